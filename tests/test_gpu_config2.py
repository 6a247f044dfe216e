"""Self-contact (configuration 2) on the CUDA path: a sheet folded about parallel lines and dropped
onto the floor, against the oracle's FP64 restatement of the contact shader math (the reference's
f64 solver has none; selfcontact.wgsl), and the full configuration's behaviour on the GPU alone.
"""
import numpy as np
import pytest

import btd_b200 as btd
from helpers import MG, copy_state
from oracle import Oracle

pytestmark = pytest.mark.gpu

HALF = 0.5 * btd.material_preset(0).thickness
HARD_CORE = 0.3e-3


def layer_order_kept(x0, x, cell=2e-3, apart=1e-3):
    """Nodes that started in different layers of the stack (initial heights more than `apart` apart)
    and now lie within one `cell` of each other horizontally keep their order, the higher at least
    the hard core above the lower (face-to-node contact keeps about the contact distance)."""
    key = np.floor(x[:, :2] / cell).astype(np.int64)
    order = np.lexsort((key[:, 1], key[:, 0]))
    k = key[order]
    starts = np.nonzero(np.any(np.diff(k, axis=0) != 0, axis=1))[0] + 1
    worst = np.inf
    for grp in np.split(order, starts):
        if len(grp) < 2:
            continue
        z0, z = x0[grp, 2], x[grp, 2]
        hi = z0[:, None] - z0[None, :] > apart
        if hi.any():
            worst = min(worst, float((z[:, None] - z[None, :])[hi].min()))
    return worst


def two_sheets():
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.15, 0.15, bundle=(9, 6), z=z, seed=3) for z in (0.0, 0.004)])
    L0 = sc.layers[0]
    nx, ny, n = L0.nx, L0.ny, L0.node_count
    i, j = np.arange(n) % nx, np.arange(n) // nx
    sc.pinned[:] = 0
    sc.pinned[:n] = ((i == 0) | (j == 0) | (i == nx - 1) | (j == ny - 1)).astype(np.uint8)
    h = 1 / 120
    cpu = Oracle(sc, h=h, newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, self_contact=True, **MG)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(h, 4, 1e-6, self_contact=1))
    x0, _ = copy_state(cpu, gpu)
    # the free upper sheet is a detached piece (nothing anchors it): its rigid modes on both sides
    from btd_b200.topology import Lattice, label_pieces, pack_bits, search

    bits = pack_bits(cpu.segments()["seg_flags"], np.zeros(sc.N, np.float32))
    lattice = Lattice(sc.layers, sc.N)
    piece_of, start, nodes, _ = label_pieces(bits, search(bits, sc.pinned, (), lattice), lattice)
    assert len(start) == 2 and len(nodes) == sc.N - n
    cpu.set_pieces(piece_of, start, nodes)
    gpu.set_pieces(piece_of, start, nodes)
    return sc, cpu, gpu, x0, (nx, ny, n)


def test_two_sheets_contact_matches_oracle():
    """The sheet-on-sheet drop of test_gpu_contact, GPU against the oracle with self-contact. The free
    sheet slides on the sagging one under friction near its stick limit, which amplifies rounding
    differences laterally, so the trajectory is compared substep by substep (each from the oracle's
    state rounded to float32: the largest node error over the substep's largest displacement, median
    under 5 %), and the free runs' resting gaps between the sheets after 60 substeps agree to 0.1 mm."""
    sc, cpu, gpu, x0, (nx, ny, n) = two_sheets()
    errs = []
    for _ in range(60):
        xs, _ = copy_state(cpu, gpu)
        cpu.substep()
        gpu.substep()
        errs.append(np.abs(gpu.x.astype(np.float64) - cpu.x).max() / max(np.abs(cpu.x - xs).max(), 1e-12))
    assert np.median(errs) < 0.05, np.round(errs, 4).tolist()
    sc, cpu, gpu, x0, (nx, ny, n) = two_sheets()
    for _ in range(60):
        cpu.substep()
        gpu.substep()
    xc, xg = cpu.x, gpu.x.astype(np.float64)
    gc = (xc[n:, 2] - xc[:n, 2]).reshape(ny, nx)[2:-2, 2:-2]
    gg = (xg[n:, 2] - xg[:n, 2]).reshape(ny, nx)[2:-2, 2:-2]
    assert gc.min() > HARD_CORE and gg.min() > HARD_CORE, (gc.min(), gg.min())
    assert np.abs(gg - gc).max() < 1e-4, np.abs(gg - gc).max()


def test_folded_drop_matches_oracle():
    """Configuration 2 at 64 x 64 over 0.15 m (three layers, folds 3 mm apart), 4 steps of 1/60 s:
    the folded stack starts to fall with its layers' contact bounds engaged (each node's step may
    close only 0.45 of its clearance to the face below, so the upper layers lag and the stack opens
    up); GPU within 0.03 of the motion of the oracle's, both keeping the stack's order. Later the
    bounds' switching (which face is nearest, which one the path crosses) makes the opening stack's
    trajectory diverge between any two roundings, so parity is taken here."""
    c = btd.configs.CONFIG2
    sc = btd.configs.config2(n=64, size=0.15)
    cpu = Oracle(sc, h=c["h"], newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, self_contact=True, **MG)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(c["h"], 4, 1e-6, self_contact=1))
    cpu.set_floor(c["floor"])
    gpu.set_floor(c["floor"])
    x0, _ = copy_state(cpu, gpu)
    for _ in range(4):
        cpu.substep()
        gpu.substep()
    xc, xg = cpu.x, gpu.x.astype(np.float64)
    moved = np.abs(xc - x0).max()
    assert moved > 0.01, moved
    assert np.abs(xg - xc).max() < 0.03 * moved, (np.abs(xg - xc).max(), moved)
    assert layer_order_kept(x0, xg) > HARD_CORE
    assert layer_order_kept(x0, xc) > HARD_CORE


def test_config2_on_the_gpu():
    """The full configuration (256 x 256 over 0.6 m, three parallel folds dropped from 0.3 m, 200
    steps): no value goes non-finite, no node below half thickness above the floor, and the stack's
    bottom reaches the floor. (The contact bounds cap each node's step toward the face below at 0.45
    of the clearance per substep, so the upper layers cannot keep up with the free fall; the crease
    spans tearing between the layers in flight is the model's behaviour - the same in the oracle.)"""
    c = btd.configs.CONFIG2
    sc = btd.configs.config2()
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(c["h"], c["newton_iterations"], c["pcg_rel_tol"], self_contact=1))
    gpu.set_floor(c["floor"])
    for _ in range(c["steps"] // 25):
        gpu.substeps(25)
        x, v = gpu.state()
        assert np.isfinite(x).all() and np.isfinite(v).all()
        assert x[:, 2].min() >= c["floor"] + HALF * 0.999, x[:, 2].min()
    assert x[:, 2].min() < c["floor"] + 2e-3, "the stack's bottom must reach the floor"


def test_folded_sheet_set_on_the_floor_settles():
    """The folded stack (128 x 128 over 0.3 m, three layers) set 2 mm above the floor: it comes to
    rest in 1 s with no span ruptured, above half thickness, its layers kept apart by at least the
    hard core, every node slower than 1 cm/s at the end."""
    c = btd.configs.CONFIG2
    sc = btd.configs.config2(n=128, size=0.3, drop=2e-3)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(c["h"], c["newton_iterations"], c["pcg_rel_tol"], self_contact=1))
    gpu.set_floor(c["floor"])
    x0 = gpu.x.astype(np.float64)
    gpu.clear_counters()
    gpu.substeps(60)
    x, v = gpu.state()
    assert gpu.counter_dict()["ruptures"] == 0
    assert x[:, 2].min() >= c["floor"] + HALF * 0.999
    assert layer_order_kept(x0, x.astype(np.float64)) > HARD_CORE
    assert np.linalg.norm(v[:, :3], axis=1).max() < 0.01


def test_folded_drop_substep_by_substep_against_the_oracle():
    """Configuration 2 at 64 x 64 over 0.15 m, 60 steps of 1/60 s (the fall, the impact and the stack
    settling on the floor), each step from the oracle's state rounded to float32 (the opening stack's
    own trajectory is sensitive to rounding once its contact bounds switch): the GPU's step against the
    oracle's, as the largest node error over the step's largest displacement. Printed per step; the
    typical step agrees to 1 % of its motion."""
    c = btd.configs.CONFIG2
    sc = btd.configs.config2(n=64, size=0.15)
    cpu = Oracle(sc, h=c["h"], newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, self_contact=True, **MG)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(c["h"], 4, 1e-6, self_contact=1))
    cpu.set_floor(c["floor"])
    gpu.set_floor(c["floor"])
    errs = []
    for _ in range(60):
        x0, _ = copy_state(cpu, gpu)
        cpu.substep()
        gpu.substep()
        moved = np.abs(cpu.x - x0).max()
        errs.append(np.abs(gpu.x.astype(np.float64) - cpu.x).max() / max(moved, 1e-12))
    errs = np.array(errs)
    print("config2 64x64 per-step error / motion: median %.2e, 90th %.2e, max %.2e" % (np.median(errs), np.quantile(errs, 0.9), errs.max()))
    assert np.median(errs) < 0.01, np.round(errs, 5).tolist()
    assert np.isfinite(gpu.x).all()
