"""Synthetic workloads: the benchmark configurations mapped onto the reference's lattice model.

The reference models cloth as a woven crossing lattice (src/simulation/scene.ts): one node per
crossing, u-family spans along i (x when the layer angle is 0), v-family spans along j, per-span
axial EA (N), a shear diagonal pair per cell (N/m), per-yarn bending rigidity B (N m^2) and a mass
lumped per node. A shell material given per unit width maps onto it at lattice pitch p as:
  EA (N) = stretch (N/m) * p        shear diagonal ks = shear modulus G (N/m)
  B (N m^2) = bending (N m) * p      node mass = areal density * p^2
The family along x (u) carries the warp stretch. Linear stretch uses eaLow = eaHigh; compression
keeps the reference denim's ratio eaCompress / eaLow = 1/2. Viscosities and air drag are the
reference DENIM values (material.ts:88-138). Gravity acts along the reference's vertical axis z.
Initial jitter is N(0, sigma) per free coordinate from splitmix64 -> Box-Muller with the seed given.
"""
import numpy as np

from . import _abi
from .scene import compile_scene, layer_spec, material_preset

U64 = np.uint64


def splitmix64(seed, n):
    """n 64-bit outputs of splitmix64 seeded with `seed`."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=U64)
        z = U64(seed) + k * U64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> U64(30))) * U64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> U64(27))) * U64(0x94D049BB133111EB)
        return z ^ (z >> U64(31))


def normal(seed, n):
    """n standard normal draws (Box-Muller over splitmix64 pairs)."""
    m = (n + 1) // 2
    r = splitmix64(seed, 2 * m)
    u1 = ((r[0::2] >> U64(11)).astype(np.float64) + 1.0) / 9007199254740992.0  # (0, 1]
    u2 = (r[1::2] >> U64(11)).astype(np.float64) / 9007199254740992.0
    rad = np.sqrt(-2.0 * np.log(u1))
    z = np.empty(2 * m)
    z[0::2] = rad * np.cos(2 * np.pi * u2)
    z[1::2] = rad * np.sin(2 * np.pi * u2)
    return z[:n]


def shell_material(pitch, stretch=(8e3, 4e3), shear=200.0, bending=1e-5, areal_density=0.35, break_strain=0.08):
    """A lattice material for a shell of the given per-width stiffnesses at lattice pitch `pitch`."""
    m = material_preset(0)
    m.name = b"shell"
    m.pitch_u = pitch
    m.pitch_v = pitch
    for f in range(2):
        y = m.yarns[f]
        ea = stretch[f] * pitch
        y.linear_density = 0.5 * areal_density * pitch
        y.ea_low = ea
        y.ea_high = ea
        y.ea_compress = 0.5 * ea
        y.bend_rigidity = bending * pitch
        y.strength = ea * break_strain  # linear law: T(eps_break)
        y.yarns_per_span = 0
    m.shear_stiffness = shear
    return m


def hanging_patch(n, size=0.3, seed=1, jitter=1e-4, **mat):
    """An n x n shell patch (n = (nx, ny): nx x ny at the pitch size / (nx - 1)), top row (j = ny - 1)
    pinned, flat plus N(0, jitter) on free coordinates."""
    nx, ny = (n, n) if np.isscalar(n) else (int(n[0]), int(n[1]))
    pitch = size / (nx - 1)
    m = shell_material(pitch, **mat)
    sc = compile_scene(layer_spec(m, (nx - 0.5) * pitch, (ny - 0.5) * pitch, collar_rows=0, seed=seed))
    assert sc.nx == nx and sc.ny == ny, (sc.nx, sc.ny)
    pinned = np.zeros((ny, nx), np.uint8)
    pinned[ny - 1, :] = 1
    sc.pinned[:] = pinned.reshape(-1)
    free = sc.pinned == 0
    pos = sc.position.reshape(-1, 3)
    z = normal(seed, 3 * int(free.sum())).reshape(-1, 3)
    pos[free] += jitter * z
    sc.position[:] = pos.reshape(-1)
    return sc


# Solver schedules of the configurations.
CONFIG0 = dict(n=64, size=0.3, h=1 / 60, newton_iterations=4, pcg_rel_tol=1e-6, steps=60, max_coarsest_nodes=400)


def config0(seed=1):
    """Plain method, small size: 64 x 64 hanging patch, 0.3 m, top row pinned, dt = 1/60, 4 Newton,
    3-level MG-PCG to relative residual 1e-6, no contact, 60 steps."""
    return hanging_patch(64, 0.3, seed=seed)


# Yarn damage: a 128 x 128 lattice over 0.3 m bundled [2, 2], so that the yarn field resolves two
# warps and two picks per span: the central 32 x 32 cells hold 64 warp and 64 weft yarns.
CONFIG1 = dict(n=128, size=0.3, bundle=(2, 2), region=32, yarn_ea=2e3, yarn_bending=1e-7, crossing_friction=0.3,
               break_strain=0.08, break_sigma=0.25, grip_speed=0.2, grip_stiffness=2e4, h=1 / 120, newton_iterations=4,
               pcg_rel_tol=1e-6, steps=120)


def yarn_material(pitch, ea, bending, crossing_friction, areal_density=0.35, shear=200.0):
    """A weave of linear yarns at yarn pitch `pitch`: per-yarn EA (N) and rigidity (N m^2), the areal
    density shared by the two families, DENIM's viscosities, drag and crossing law otherwise."""
    m = material_preset(0)
    m.name = b"yarns"
    m.pitch_u = pitch
    m.pitch_v = pitch
    for f in range(2):
        y = m.yarns[f]
        y.linear_density = 0.5 * areal_density * pitch
        y.ea_low = ea
        y.ea_high = ea
        y.ea_compress = 0.5 * ea
        y.bend_rigidity = bending
        y.strength = ea * 10.0
        y.yarns_per_span = 0
    m.shear_stiffness = shear
    m.crossing_friction = crossing_friction
    return m


def config1(seed=11):
    """Yarn damage: CONFIG1's lattice, no pins. Outside the central region the yarns hold (break at
    1000 % strain); inside, each yarn segment at a crossing breaks at a strain drawn from
    lognormal(ln 0.08, 0.25), its field strength the tension T(eps) = EA eps of the linear law.
    Returns the scene and the two grips: the edge columns i = 0, 1 and i = n - 2, n - 1."""
    return _yarn_region_patch(CONFIG1, seed)


# Learned coarse correction: the tearing patch - CONFIG1's yarn lattice at 256 x 256 over 0.6 m (the
# same pitch), a central 64 x 64-cell region of lognormal break strains, self-contact on, the two
# edge grips pulled apart at 0.5 m/s; the network (3 layers, hidden 64) guarded at a mean contraction
# of 0.9 per PCG iteration.
CONFIG4 = dict(CONFIG1, n=256, size=0.6, region=64, grip_speed=0.5, self_contact=True, hidden=64, guard=0.9)


def config4(seed=41, n=None, region=None):
    """CONFIG4's scene and grips as config1 returns them; n and region scale it down at the same pitch
    (a 64 x 64 patch with a 16 x 16-cell region keeps its proportions)."""
    c = dict(CONFIG4)
    if n is not None:
        c["size"] = c["size"] / (c["n"] - 1) * (n - 1)
        c["n"] = n
    if region is not None:
        c["region"] = region
    return _yarn_region_patch(c, seed)


def _yarn_region_patch(c, seed):
    n, bu, bv = c["n"], c["bundle"][0], c["bundle"][1]
    pitch = c["size"] / (n - 1)
    m = yarn_material(pitch / bu, c["yarn_ea"], c["yarn_bending"], c["crossing_friction"])
    sc = compile_scene(layer_spec(m, (n - 0.5) * pitch, (n - 0.5) * pitch, bundle=(bu, bv), collar_rows=0, seed=seed))
    assert sc.nx == n and sc.ny == n, (sc.nx, sc.ny)
    sc.pinned[:] = 0
    L = sc.layers[0]
    K, M = L.field_k, L.field_m
    # field strength of yarn family f at crossing (pick m, warp k): index 2 (m K + k) + f
    strength = np.full((M, K, 2), c["yarn_ea"] * 10.0, np.float32)
    lo = (n - c["region"]) // 2
    ks, ms = slice(lo * bu, (lo + c["region"]) * bu), slice(lo * bv, (lo + c["region"]) * bv)
    eps = np.exp(np.log(c["break_strain"]) + c["break_sigma"] * normal(seed + 1, strength[ms, ks].size))
    strength[ms, ks] = (c["yarn_ea"] * eps).reshape(strength[ms, ks].shape)
    sc.field_strength[:] = strength.reshape(-1)
    left = np.array([j * n + i for j in range(n) for i in (0, 1)], np.int32)
    right = np.array([j * n + i for j in range(n) for i in (n - 2, n - 1)], np.int32)
    return sc, left, right


def break_events(field, seg_flags):
    """The break-event set (yarnField.ts:36-43, 483-492): (crossing, family) pairs whose damage code
    separates the yarn (cut 255 or pulled out 254), and the spans that ruptured (broken, not an
    initial defect)."""
    f = np.asarray(field).reshape(-1)
    sep = set(np.nonzero(f >= 254)[0].tolist())
    flags = np.asarray(seg_flags).reshape(-1)
    spans = set(np.nonzero(((flags & 2) != 0) & ((flags & 4) == 0))[0].tolist())
    return sep, spans


# Contact: 256 x 256 over 0.6 m of the configuration-0 material, folded about 1-3 seeded lines and
# dropped from 0.3 m onto the floor at z = 0, self-contact on (SELF_CONTACT), 200 steps.
CONFIG2 = dict(n=256, size=0.6, folds=(1, 3), fold_gap=3e-3, drop=0.3, h=1 / 60, newton_iterations=4, pcg_rel_tol=1e-6,
               steps=200, floor=0.0)


def fold(points, normal, offset, gap):
    """Fold a sheet about the line {p . normal = offset} of its plane: the part beyond the line turns
    over, each point rolling on a circle about an axis along the line gap / 2 above the sheet's
    highest point (radius = its depth below the axis), by the angle that keeps its arc length, so
    every layer folds without stretch and lands mirrored on top, its layers gap or more apart."""
    p = np.array(points, np.float64)
    nrm = np.array([normal[0], normal[1], 0.0])
    s = p @ nrm - offset
    H = p[:, 2].max() + 0.5 * gap
    over = s > 0
    rho = H - p[over, 2]
    theta = np.minimum(s[over] / rho, np.pi)
    on_arc = s[over] < np.pi * rho
    along = np.where(on_arc, rho * np.sin(theta), -(s[over] - np.pi * rho))
    out = p.copy()
    out[over] = p[over] + np.outer(along - s[over], nrm)
    out[over, 2] = np.where(on_arc, H - rho * np.cos(theta), H + rho)
    return out


def config2(seed=29, n=None, size=None, folds=None, drop=None):
    """Contact: a free sheet (no pins) of the configuration-0 material folded about k parallel lines
    (k uniform in CONFIG2's range, direction seeded), then lifted to the drop height above the floor.
    Each fold turns over a part of the sheet still single and uncreased - the first the far side of a
    line 55-70 % across, later ones the near side of a line within the remaining single region - so
    every fold is isometric (a fold across an earlier crease would have to shear its layers)."""
    c = CONFIG2
    n = n or c["n"]
    size = size or c["size"]
    pitch = size / (n - 1)
    m = shell_material(pitch)
    sc = compile_scene(layer_spec(m, (n - 0.5) * pitch, (n - 0.5) * pitch, collar_rows=0, seed=seed))
    assert sc.nx == n and sc.ny == n, (sc.nx, sc.ny)
    sc.pinned[:] = 0
    r = splitmix64(seed, 16).astype(np.float64) / 2.0**64
    k = folds if folds is not None else c["folds"][0] + int(r[0] * (c["folds"][1] - c["folds"][0] + 1))
    ang = 2 * np.pi * r[1]
    nrm = np.array([np.cos(ang), np.sin(ang)])
    pos = sc.position.reshape(-1, 3).copy()
    proj = pos[:, :2] @ nrm
    a, b = proj.min(), proj.max()
    o = a + (b - a) * (0.55 + 0.15 * r[2])
    pos = fold(pos, nrm, o, c["fold_gap"])
    lo, hi = a, o - (b - o)  # the single, uncreased region left
    for q in range(1, k):
        if hi - lo < 8 * c["fold_gap"] + 0.1 * (b - a):
            break
        o = lo + (hi - lo) * (0.35 + 0.3 * r[2 + q])
        pos = fold(pos, -nrm, -o, c["fold_gap"])  # the near side, p . nrm < o
        lo, hi = o, min(hi, o + (o - lo))
    pos[:, 2] += (c["drop"] if drop is None else drop) - pos[:, 2].min() + c["floor"]
    sc.position[:] = pos.reshape(-1)
    return sc


# Batch: independent hanging patches, all seeded: side uniform in [16, 128] nodes at configuration
# 0's pitch, stiffness factor uniform in (0.5, 2) on stretch, shear and bending, a central yarn region
# of 0-30 % of the area whose crossings break at lognormal(ln 0.08, 0.25) strains, and one grip on a
# 3 x 3 patch in the lower third pulled at 0.05-0.2 m/s in a random direction.
CONFIG3 = dict(count=512, sides=(16, 128), pitch=0.3 / 63, stiffness=(0.5, 2.0), region=(0.0, 0.3), grip_speed=(0.05, 0.2),
               grip_stiffness=50.0, grip_lead=0.006, h=1 / 60, newton_iterations=4, pcg_rel_tol=1e-6)


def _scaled_patch(n, pitch, f, seed, cache):
    """hanging_patch(n) with stretch, shear and bending scaled by f: the compiled scene of each size is
    made once and copied, its layer's material scaled (the compile itself does not depend on them),
    the jitter drawn with the patch's own seed."""
    if n not in cache:
        cache[n] = hanging_patch(n, (n - 1) * pitch, seed=1, jitter=0.0)
    sc = cache[n].copy()
    for mat in (sc.layers[0].material, sc.layers[0].weave):
        for y in mat.yarns:
            y.ea_low *= f
            y.ea_high *= f
            y.ea_compress *= f
            y.bend_rigidity *= f
        mat.shear_stiffness *= f
    free = sc.pinned == 0
    pos = sc.position.reshape(-1, 3)
    pos[free] += 1e-4 * normal(seed, 3 * int(free.sum())).reshape(-1, 3)
    sc.position[:] = pos.reshape(-1)
    return sc


def config3_sides(seed=31, count=None, sides=None):
    """The patches' lattice sides (nodes a side) of config3, without building them."""
    c = CONFIG3
    count = count or c["count"]
    lo, hi = sides or c["sides"]
    r = splitmix64(seed, 8 * count).astype(np.float64) / 2.0**64
    return [lo + int(r[8 * b] * (hi - lo + 1)) for b in range(count)]


def shard_patches(sides, world):
    """Patches of a batch dealt to `world` GPUs by estimated bytes (proportional to the node count):
    largest first, each to the least loaded rank (ties to the lowest rank), so every rank gets the
    same list whatever its own index. Returns one sorted index list a rank."""
    load = [0] * world
    out = [[] for _ in range(world)]
    for b in sorted(range(len(sides)), key=lambda b: (-sides[b] ** 2, b)):
        k = min(range(world), key=lambda q: (load[q], q))
        load[k] += sides[b] ** 2
        out[k].append(b)
    return [sorted(o) for o in out]


def config3(seed=31, count=None, sides=None, only=None):
    """The batch: a list of patches, each (scene, grip) with grip = dict(picked, nodes, weights,
    velocity, stiffness, max_lead); with `only`, the patches of those indices (each patch depends on
    its index alone)."""
    c = CONFIG3
    count = count or c["count"]
    lo, hi = sides or c["sides"]
    r = splitmix64(seed, 8 * count).astype(np.float64) / 2.0**64
    out = []
    cache = {}
    for b in (range(count) if only is None else only):
        u = r[8 * b: 8 * b + 8]
        n = lo + int(u[0] * (hi - lo + 1))
        f = c["stiffness"][0] + (c["stiffness"][1] - c["stiffness"][0]) * u[1]
        pitch = c["pitch"]
        sc = _scaled_patch(n, pitch, f, seed * 1000 + b, cache)
        # the yarn region: a central square of the given share of the cells
        share = c["region"][0] + (c["region"][1] - c["region"][0]) * u[2]
        side = int(round(np.sqrt(share) * (n - 1)))
        ea = np.array([8e3 * f * pitch, 4e3 * f * pitch])
        strength = np.repeat((10.0 * ea)[None, :], sc.C, axis=0).astype(np.float32)
        if side > 0:
            a0 = (n - side) // 2
            ii, jj = np.meshgrid(np.arange(a0, a0 + side), np.arange(a0, a0 + side))
            cross = (jj * n + ii).reshape(-1)
            eps = np.exp(np.log(0.08) + 0.25 * normal(seed * 1000 + b, 2 * cross.size)).reshape(-1, 2)
            strength[cross] = (eps * ea[None, :]).astype(np.float32)
        sc.field_strength[:] = strength.reshape(-1)
        gi = int(n // 4 + u[3] * (n // 2))
        gj = int(1 + u[4] * max(1, n // 3 - 2))
        gi, gj = min(max(gi, 1), n - 2), min(max(gj, 1), n - 2)
        nodes = np.array([(gj + dj) * n + gi + di for dj in (-1, 0, 1) for di in (-1, 0, 1)], np.int32)
        ang, el = 2 * np.pi * u[5], np.pi * (u[6] - 0.5)
        speed = c["grip_speed"][0] + (c["grip_speed"][1] - c["grip_speed"][0]) * u[7]
        vel = speed * np.array([np.cos(el) * np.cos(ang), np.cos(el) * np.sin(ang), np.sin(el)])
        out.append((sc, dict(picked=int(gj * n + gi), nodes=nodes, weights=np.ones(9), velocity=vel,
                             stiffness=c["grip_stiffness"] * f, max_lead=c["grip_lead"])))
    return out


def solver_params(h, newton_iterations, pcg_rel_tol, pcg_cap=500, **kw):
    from .solver import default_params

    kw.setdefault("newton_max", newton_iterations)
    kw.setdefault("self_contact", 0)  # the configurations without contact
    return default_params(h=h, newton_iterations=newton_iterations, pcg_iterations=pcg_cap, pcg_rel_tol=pcg_rel_tol, **kw)
