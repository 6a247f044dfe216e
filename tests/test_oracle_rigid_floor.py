"""The detached pieces' rigid modes together with the floor (FLOOR_CONTACT: common.wgsl floorLowest,
assemble.wgsl:191-209, step.wgsl:77-86) in the oracle, pinned by the reference's own floor contracts for
pieces (tests/gpu/floor.ts): a piece sliding on the floor stops within the Coulomb distance (slide,
:174-194), a piece spinning flat on it stops within twice its Coulomb time (spin, :196-237; "a piece in
the solve's first iterations kept spinning for a second"), and a piece cut out of a mounted sheet falls
to the floor and rests there (torn, :124-161). Without the rigid-mode correction the same pieces slide
and spin on as on ice, which is why the reference carries it. Shipped settings: two Newton and two PCG
iterations at h = 1/120; the product scene's node pitch."""
import numpy as np
import pytest

import btd_b200 as btd
from btd_b200.scene import SEG_BROKEN
from btd_b200.topology import Lattice, label_pieces, pack_bits, search
from oracle import Oracle

G = 9.81
H = 1 / 120
MU = 0.35  # FLOOR_CONTACT.friction (floor.ts:5-28)
FLOOR_Z = -0.02
SHIPPED = dict(h=H, newton_iterations=2, pcg_iterations=2, pcg_rel_tol=0.0, max_coarsest_nodes=400, coarse_sweeps=2,
               line_colors=3, lag_coarse=True, line_search=True)
HALF = 0.5 * btd.material_preset(0).thickness
DELTA = HALF + 0.3e-3  # the floor's contact reach: half the thickness plus its bulge


def one_piece(sc):
    return np.zeros(sc.N, np.uint32), np.array([0, sc.N], np.uint32), np.arange(sc.N, dtype=np.uint32)


def resting_piece(pieces=True):
    """A free 5 x 5 piece settled flat on the floor (0.3 s from just above its contact reach)."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.014, 0.014, bundle=(9, 6), z=0.0, seed=3)])
    assert (sc.layers[0].nx, sc.layers[0].ny) == (5, 5)
    sc.pinned[:] = 0
    o = Oracle(sc, **SHIPPED)
    o.set_floor(FLOOR_Z)
    x = sc.position.reshape(-1, 3).astype(np.float64)
    x[:, 2] = FLOOR_Z + HALF + 0.3e-3
    o.set_state(x, np.zeros_like(x))
    if pieces:
        o.set_pieces(*one_piece(sc))
    for _ in range(36):
        o.substep()
    assert np.abs(o.v).max() < 1e-6
    return sc, o


def spin_rate(x, v):
    """Spin about the vertical through the centre: sum r x v / sum r^2 (equal masses)."""
    r = x[:, :2] - x[:, :2].mean(axis=0)
    return np.sum(r[:, 0] * v[:, 1] - r[:, 1] * v[:, 0]) / np.sum(r ** 2)


def spin(pieces):
    sc, o = resting_piece(pieces)
    x = o.x
    r = x[:, :2] - x[:, :2].mean(axis=0)
    w0 = 10.0
    v = np.zeros_like(x)
    v[:, 0], v[:, 1] = -w0 * r[:, 1], w0 * r[:, 0]
    o.set_state(x, v)
    coulomb = w0 / (MU * G * np.hypot(r[:, 0], r[:, 1]).sum() / np.sum(r ** 2))
    for k in range(1, round(0.1 / H) + 1):
        o.substep()
        w = spin_rate(o.x, o.v)
        if abs(w) < 0.01 * w0:
            return k * H, coulomb, w
    return np.inf, coulomb, w


def test_a_piece_spinning_on_the_floor_stops_within_the_coulomb_time():
    stopped, coulomb, w = spin(True)
    assert stopped <= 2 * coulomb, (stopped, coulomb, w)


def test_without_the_rigid_modes_it_spins_on():
    stopped, coulomb, w = spin(False)
    assert stopped == np.inf and w > 0.5 * 10.0, (stopped, w)


def slide(pieces):
    sc, o = resting_piece(pieces)
    x = o.x
    x0 = x[:, 0].mean()
    v0 = 0.25
    v = np.zeros_like(x)
    v[:, 0] = v0
    o.set_state(x, v)
    lowest, late = np.inf, 0.0
    for k in range(round(0.4 / H)):
        o.substep()
        lowest = min(lowest, (o.x[:, 2] - FLOOR_Z).min())
        if k >= round(0.3 / H):
            late = max(late, np.abs(o.v).max())
    return (o.x[:, 0].mean() - x0) / (v0 * v0 / (2 * MU * G)), late, lowest


def test_a_piece_sliding_on_the_floor_stops_within_the_coulomb_distance():
    """slide (floor.ts:174-194): 0.25 m/s; slides 0.8 to 1.1 of v^2 / (2 mu g), below 2 mm/s over
    0.3-0.4 s, never below half its thickness."""
    ratio, late, lowest = slide(True)
    assert 0.8 < ratio < 1.1 and late < 0.002 and lowest >= 0.999 * HALF, (ratio, late, lowest)


def test_without_the_rigid_modes_it_slides_on():
    ratio, late, _ = slide(False)
    assert ratio > 3 and late > 0.05, (ratio, late)


def test_a_piece_torn_out_of_the_sheet_lands_on_the_floor_and_rests_there():
    """torn (floor.ts:124-161): an 8 x 7 piece cut out of a sheet mounted at its rim 12 cm above the
    floor falls onto it: after 1.5 s every node lies between half the thickness and the contact reach
    above the floor, below 2 mm/s over 1-1.5 s, spans within 2 % of rest."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.06, 0.055, bundle=(9, 6), z=0.0, seed=3)])
    L = sc.layers[0]
    nx, ny = L.nx, L.ny
    i, j = np.arange(sc.N) % nx, np.arange(sc.N) // nx
    sc.pinned[:] = ((i == 0) | (j == 0) | (i == nx - 1) | (j == ny - 1)).astype(np.uint8)
    o = Oracle(sc, **SHIPPED)
    floor_z = -0.12
    o.set_floor(floor_z)
    i0, j0 = (nx - 8) // 2, (ny - 7) // 2
    inside = lambda a, b: i0 <= a < i0 + 8 and j0 <= b < j0 + 7  # noqa: E731
    seg = o.segments()
    flags = seg["seg_flags"].copy()
    piece, spans = [], []
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
            if inside(a + 1, b):
                spans.append((n, n + 1, 2 * n))
            if inside(a, b + 1):
                spans.append((n, n + nx, 2 * n + 1))
    o.set_segments(seg_flags=flags)
    bits = pack_bits(flags, np.zeros(sc.N, np.float32))
    lattice = Lattice(sc.layers, sc.N)
    piece_of, start, nodes, _ = label_pieces(bits, search(bits, sc.pinned, (), lattice), lattice)
    assert sorted(nodes.tolist()) == sorted(piece)
    o.set_pieces(piece_of, start, nodes)
    lowest, late = np.inf, 0.0
    for k in range(round(1.5 / H)):
        o.substep()
        lowest = min(lowest, (o.x[piece, 2] - floor_z).min())
        if k >= round(1.0 / H):
            late = max(late, np.abs(o.v[piece]).max())
    x = o.x
    rest = o.segments()["rest_length"]
    highest = (x[piece, 2] - floor_z).max()
    strain = max(abs(np.linalg.norm(x[b] - x[a]) / rest[s] - 1) for a, b, s in spans)
    assert lowest >= 0.999 * HALF and highest < DELTA and late < 0.002 and strain < 0.02, (lowest, highest, late, strain)
