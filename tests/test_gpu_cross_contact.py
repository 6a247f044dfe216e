"""Cross-layer contact (contact.ts:7-19, contact.wgsl:31-164) on the CUDA path against the oracle's
restatement, on the contracts the oracle's own tests pin (two plies at crossing pitch, contact distance
the mean of their thicknesses, 0.7 mm): a ply laid on a mounted ply rests at the contact distance, and
mounted plies overlapping by half of it are pushed apart to it; from the same start the GPU's plies
follow the oracle's. The reference gives a multi-layer scene this contact in place of self-contact
(solver.ts:364); the solver does so with the cross_layer parameter.
"""
import numpy as np
import pytest
from scipy.interpolate import LinearNDInterpolator

import btd_b200 as btd
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


def test_a_ply_laid_on_a_mounted_ply_rests_at_the_contact_distance():
    """The upper ply is free: nothing anchors it, so it is a detached piece whose rigid modes start
    every Newton direction, at the reference's shipped schedule of two PCG iterations (without them the
    near-singular free ply is beyond an FP32 preconditioner). Over 60 substeps it never comes closer to
    the lower ply than 0.75 of the contact distance, and its gaps follow the oracle's."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.015, 0.015, bundle=(1, 1), z=z, seed=3) for z in (0.0, 0.0009)])
    L0 = sc.layers[0]
    n = L0.nx * L0.ny
    i, j = np.arange(n) % L0.nx, np.arange(n) // L0.nx
    sc.pinned[:] = 0
    sc.pinned[:n] = ((i == 0) | (j == 0) | (i == L0.nx - 1) | (j == L0.ny - 1)).astype(np.uint8)
    cpu, gpu = pair(sc, pieces=True)
    worst = np.inf
    for s in range(60):
        cpu.substep()
        gpu.substep()
        if s % 5 == 4:
            worst = min(worst, gaps(gpu.x.astype(np.float64), n).min())
    g, gc = gaps(gpu.x.astype(np.float64), n), gaps(cpu.x, n)
    assert worst > 0.75 * R, worst
    assert abs(np.median(g) - np.median(gc)) < 0.1 * R, (np.median(g), np.median(gc))
    assert abs(g.min() - gc.min()) < 0.1 * R, (g.min(), gc.min())


def test_overlapping_mounted_plies_are_pushed_apart_like_the_oracle():
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
    assert np.abs(xg - xc).max() < 0.05 * moved, (np.abs(xg - xc).max(), moved)
