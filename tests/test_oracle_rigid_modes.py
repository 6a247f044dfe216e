"""The detached pieces' rigid modes (rigid_frame.wgsl, rigid_apply.wgsl, rigid_spin.wgsl; solver.ts:612-716)
restated in the oracle, pinned by the reference's own contracts for them (tests/gpu/detached.ts): a free
piece thrown with a spin about its normal keeps its shape and its spin and falls (tumble, :139-192),
and a piece cut out of a mounted sheet falls as freely as drag lets it at the shipped solver settings
of two Newton and two PCG iterations (cutOut, :305-352) - which without the rigid-mode start of the
Newton direction it does not (a few percent of its fall: the piece hovers). Two more of its detached
contracts: an intact span between two detached nodes pulled apart resists the extension
(differential, :84-106), and bending viscosity does not resist a rigid rotation of a bent triple
(bendViscosity, :246-304).

The pieces come from the host topology analysis (topology.ts restated in btd_b200.topology) over the
oracle's spans. The scenes are small (the product scene's node pitch, 3.42 x 3.48 mm) so the oracle
finishes in seconds."""
import numpy as np
import pytest

import btd_b200 as btd
from btd_b200.scene import SEG_BROKEN
from btd_b200.topology import Lattice, label_pieces, pack_bits, search
from oracle import Oracle

G = 9.81
H = 1 / 120
SHIPPED = dict(h=H, newton_iterations=2, pcg_iterations=2, pcg_rel_tol=0.0, max_coarsest_nodes=400, coarse_sweeps=2,
               line_colors=3, lag_coarse=True, line_search=True)


def pieces_of(o, sc, anchors=()):
    """The analysis of topology.ts over the oracle's spans: what no mount or anchor reaches, as pieces."""
    flags = o.segments()["seg_flags"]
    bits = pack_bits(flags, np.zeros(sc.N, np.float32))
    lattice = Lattice(sc.layers, sc.N)
    freed = search(bits, sc.pinned, anchors, lattice)
    piece_of, start, nodes, _ = label_pieces(bits, freed, lattice)
    return piece_of, start, nodes


def span_strain(o, sc):
    """Largest |strain| of the intact spans."""
    x = o.x
    seg = o.segments()
    worst = 0.0
    L = sc.layers[0]
    for n in range(sc.N):
        i, j = n % L.nx, n // L.nx
        for f, m in ((0, n + 1 if i + 1 < L.nx else -1), (1, n + L.nx if j + 1 < L.ny else -1)):
            s = 2 * n + f
            if m < 0 or seg["seg_flags"][s] & SEG_BROKEN or not seg["seg_flags"][s] & 1:
                continue
            worst = max(worst, abs(np.linalg.norm(x[m] - x[n]) / seg["rest_length"][s] - 1))
    return worst


def test_a_free_piece_keeps_its_shape_spins_and_falls():
    """tumble (detached.ts:139-192): a 4 x 4 piece thrown with 10 rad/s about its normal falls for 0.25 s
    at the shipped settings; its spans stay within 2 % of their rest length, it keeps more than 80 % of
    its spin (what it loses is backward Euler's dissipation) and falls faster than half of free fall."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.011, 0.011, bundle=(9, 6), z=0.1, seed=3)])
    assert (sc.layers[0].nx, sc.layers[0].ny) == (4, 4)
    sc.pinned[:] = 0
    o = Oracle(sc, **SHIPPED)
    x = sc.position.reshape(-1, 3).astype(np.float64)
    c = x.mean(axis=0)
    omega = 10.0
    v = np.zeros_like(x)
    v[:, 0] = -omega * (x[:, 1] - c[1])
    v[:, 1] = omega * (x[:, 0] - c[0])
    o.set_state(x, v)
    piece_of, start, nodes = pieces_of(o, sc)
    assert len(start) == 2 and len(nodes) == 16
    o.set_pieces(piece_of, start, nodes)
    steps = 6 * round(0.25 / 6 / H)
    worst = 0.0
    for k in range(steps):
        o.substep()
        worst = max(worst, span_strain(o, sc))
    x, v, _, _ = o.state()
    com, vcom = x.mean(axis=0), v.mean(axis=0)
    r, u = x - com, v - vcom
    spin = np.sum(r[:, 0] * u[:, 1] - r[:, 1] * u[:, 0]) / np.sum(r[:, 0] ** 2 + r[:, 1] ** 2)
    t = steps * H
    assert worst < 0.02, worst
    assert spin > 0.8 * omega, spin
    assert vcom[2] < -0.5 * G * t, (vcom[2], G * t)


def cut_out(shape, pieces=True):
    """A sheet mounted at its rim with an 8 x 7 comb or serpentine cut out of its middle (every span
    across the outline broken, and the inner cuts of the shape); 0.25 s at the shipped settings. Returns
    the piece's mean vertical velocity and the time."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.06, 0.055, bundle=(9, 6), z=0.0, seed=3)])
    L = sc.layers[0]
    nx, ny = L.nx, L.ny
    i, j = np.arange(sc.N) % nx, np.arange(sc.N) // nx
    sc.pinned[:] = ((i == 0) | (j == 0) | (i == nx - 1) | (j == ny - 1)).astype(np.uint8)
    o = Oracle(sc, **SHIPPED)
    i0, j0 = (nx - 8) // 2, (ny - 7) // 2
    inside = lambda a, b: i0 <= a < i0 + 8 and j0 <= b < j0 + 7  # noqa: E731
    seg = o.segments()
    flags = seg["seg_flags"].copy()
    piece = []
    for b in range(j0 - 1, j0 + 8):
        for a in range(i0 - 1, i0 + 9):
            n = b * nx + a
            if inside(a, b) != inside(a + 1, b):
                flags[2 * n] |= SEG_BROKEN
            if inside(a, b) != inside(a, b + 1):
                flags[2 * n + 1] |= SEG_BROKEN
            if not inside(a, b):
                continue
            piece.append(n)
            if shape == "comb" and b > j0 and inside(a + 1, b):
                flags[2 * n] |= SEG_BROKEN
            if shape == "serpentine" and inside(a, b + 1) and a != (i0 + 7 if (b - j0) % 2 == 0 else i0):
                flags[2 * n + 1] |= SEG_BROKEN
    o.set_segments(seg_flags=flags)
    piece_of, start, nodes = pieces_of(o, sc)
    assert sorted(nodes.tolist()) == sorted(piece), "the analysis detaches exactly the cut-out piece"
    if pieces:
        o.set_pieces(piece_of, start, nodes)
    steps = round(0.25 / H)
    for _ in range(steps):
        o.substep()
    return o.v[piece, 2].mean(), steps * H


@pytest.mark.parametrize("shape", ["comb", "serpentine"])
def test_a_piece_cut_out_of_the_sheet_falls_as_freely_as_drag_lets_it(shape):
    """cutOut (detached.ts:305-352): after 0.25 s the piece falls faster than half of free fall."""
    vz, t = cut_out(shape)
    assert -vz > 0.5 * G * t, (vz, G * t)


def test_without_the_rigid_modes_a_cut_out_piece_hovers():
    """The reason for the correction (rigid_apply.wgsl, detached.ts:311-314): the same comb without its
    pieces set resolves only a few percent of its fall in two PCG iterations."""
    vz, t = cut_out("comb", pieces=False)
    assert -vz < 0.2 * G * t, (vz, G * t)


def test_a_free_fall_with_the_rigid_start_matches_the_converged_solve():
    """A free layer as one piece: two PCG iterations from the rigid start give the velocity the
    converged solve (200 iterations) gives, to 1e-6 of it; without the start they give almost none."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.02, 0.02, bundle=(1, 1), z=0.1, seed=3)])
    sc.pinned[:] = 0
    out = {}
    for name, pcg, pieces in (("rigid", 2, True), ("plain", 2, False), ("converged", 200, False)):
        o = Oracle(sc, **{**SHIPPED, "pcg_iterations": pcg})
        if pieces:
            o.set_pieces(np.zeros(sc.N, np.uint32), np.array([0, sc.N], np.uint32), np.arange(sc.N, dtype=np.uint32))
        for _ in range(10):
            o.substep()
        out[name] = o.v[:, 2].mean()
    assert abs(out["rigid"] - out["converged"]) < 1e-6 * abs(out["converged"]), out
    assert abs(out["plain"]) < 0.05 * abs(out["converged"]), out


def test_setting_no_pieces_removes_the_correction():
    """An empty set (setPieces with one start entry) restores the plain solve exactly."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.011, 0.011, bundle=(9, 6), z=0.1, seed=3)])
    sc.pinned[:] = 0
    a, b = Oracle(sc, **SHIPPED), Oracle(sc, **SHIPPED)
    b.set_pieces(np.zeros(sc.N, np.uint32), np.array([0, sc.N], np.uint32), np.arange(sc.N, dtype=np.uint32))
    b.substep()
    b.set_pieces(np.full(sc.N, 0xFFFFFFFF, np.uint32), np.zeros(1, np.uint32), np.zeros(0, np.uint32))
    b.set_state(a.x, a.v)
    a.substep()
    b.substep()
    assert np.array_equal(a.x, b.x)


def isolated(spans):
    """A free 9 x 9 layer at zero gravity with only the given spans (owner, family) intact."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.028, 0.028, bundle=(9, 6), z=0.08, seed=3)])
    sc.pinned[:] = 0
    o = Oracle(sc, **{**SHIPPED, "gravity": (0.0, 0.0, 0.0)})
    seg = o.segments()
    flags = seg["seg_flags"].copy()
    keep = {2 * n + f for n, f in spans}
    for q in range(2 * sc.N):
        if q not in keep:
            flags[q] |= SEG_BROKEN
    o.set_segments(seg_flags=flags)
    return sc, o, seg["rest_length"]


def test_an_intact_span_pulled_apart_by_its_nodes_resists_the_extension():
    """differential (detached.ts:84-106): two detached nodes joined by one intact span, moving apart
    along it at 0.2 m/s at zero gravity: over 0.25 s the span stays within 1 % of its rest length and
    intact."""
    sc, o, rest = isolated([(40, 0)])
    a, b = 40, 41
    L = rest[2 * a]
    x = o.x.copy()
    x[a] = x[b] = (0.0, 0.0, 0.08)
    x[a, 0], x[b, 0] = -L / 2, L / 2
    v = np.zeros_like(x)
    v[a, 0], v[b, 0] = -0.1, 0.1
    o.set_state(x, v)
    o.set_pieces(*pieces_of(o, sc)[:3])
    worst = 0.0
    for _ in range(30):
        o.substep()
        worst = max(worst, abs(np.linalg.norm(o.x[b] - o.x[a]) / L - 1))
    flags = o.segments()["seg_flags"][2 * a]
    assert worst < 0.01 and flags == 1, (worst, flags)


def test_bending_viscosity_does_not_resist_a_rigid_rotation():
    """bendViscosity (detached.ts:246-304): a triple bent by 0.3 rad, both spans at rest length. Its
    viscous gradient (the gradient less that of the same scene without bending viscosity) vanishes for
    a rigid rotation step (30 degrees about the vertical, then about the first span's axis) and is not
    zero for a step that bends it further (the far node turned by another 0.1 rad)."""
    m = btd.material_preset(0)
    a = 40
    out = {}
    for visc in (True, False):
        mat = btd.material_preset(0)
        if not visc:
            for f in range(2):
                mat.yarns[f].bend_viscosity = 0.0
        sc = btd.compile_scene([btd.layer_spec(mat, 0.028, 0.028, bundle=(9, 6), z=0.08, seed=3)])
        sc.pinned[:] = 0
        o = Oracle(sc, **{**SHIPPED, "gravity": (0.0, 0.0, 0.0)})
        seg = o.segments()
        flags = seg["seg_flags"].copy()
        for q in range(2 * sc.N):
            if q not in (2 * a, 2 * (a + 1)):
                flags[q] |= SEG_BROKEN
        o.set_segments(seg_flags=flags)
        La, Lc = seg["rest_length"][2 * a], seg["rest_length"][2 * (a + 1)]
        th = 0.3
        p = np.array([[-La, 0, 0], [0, 0, 0], [Lc * np.cos(th), Lc * np.sin(th), 0]])
        rz = lambda q, t: np.array([q[0] * np.cos(t) - q[1] * np.sin(t), q[0] * np.sin(t) + q[1] * np.cos(t), q[2]])  # noqa: E731
        rx = lambda q, t: np.array([q[0], q[1] * np.cos(t) - q[2] * np.sin(t), q[1] * np.sin(t) + q[2] * np.cos(t)])  # noqa: E731
        x = o.x.copy()
        x[a:a + 3] = p
        o.set_state(x, np.zeros_like(x))
        for name, move in (("rigid", lambda q, k: rx(rz(q, np.pi / 6), np.pi / 6)), ("bend", lambda q, k: rz(q, 0.1) if k == 2 else q)):
            dx = np.zeros_like(x)
            for k in range(3):
                dx[a + k] = move(p[k], k) - p[k]
            o.set_dx(dx, np.zeros_like(x))
            out[name, visc] = o.node_gradient(a + 1)
    rigid = np.linalg.norm(out["rigid", True] - out["rigid", False])
    bend = np.linalg.norm(out["bend", True] - out["bend", False])
    assert bend > 0 and rigid < 1e-4 * bend, (rigid, bend)
