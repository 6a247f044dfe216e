"""Cross-layer contact (contact.ts:7-19, contact.wgsl) restated in the oracle: a scene of several
layers gets node-node contact between its layers in place of self-contact, as the reference does
(solver.ts:364). The reference has no CPU version and no test of it; these check its own contracts on
two plies at crossing pitch (node spacing 0.38 x 0.58 mm under the 0.7 mm contact distance, the
mean of the plies' thicknesses): a ply laid on a mounted ply rests at the contact distance, a ply
overlapping mounted plies are pushed apart to that distance, and one layer is unaffected.

As in the reference, detection runs at the predicted iterate (after the predictor, solver.ts:741-743)
and the bound keeps each node on the side of its nearest foreign node there: an approach faster than
the contact distance per substep can already predict a node through the other ply (a 2 mm drop at
h = 1/120 does). A free ply resting on another for long is left to the missing rigid-mode
correction: its near-rigid in-plane modes, held by contact and friction alone, are not carried by
the multigrid hierarchy, and after some 0.4 s at rest the inexact solves let it go unstable."""
import numpy as np
import pytest
from scipy.interpolate import LinearNDInterpolator

import btd_b200 as btd
from oracle import Oracle

R = btd.material_preset(0).thickness  # contact distance of two plies of one material, 0.7 mm
MG = dict(max_coarsest_nodes=400, coarse_sweeps=2, line_colors=3, lag_coarse=True, line_search=True)


def plies(z_upper, size=0.015):
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, size, size, bundle=(1, 1), z=z, seed=3) for z in (0.0, z_upper)])
    L0 = sc.layers[0]
    n = L0.nx * L0.ny
    i, j = np.arange(n) % L0.nx, np.arange(n) // L0.nx
    sc.pinned[:] = 0
    sc.pinned[:n] = ((i == 0) | (j == 0) | (i == L0.nx - 1) | (j == L0.ny - 1)).astype(np.uint8)
    return sc, n


def gaps(o, n):
    """Height of every upper node above the lower ply's surface beneath it."""
    x = o.x
    zl = LinearNDInterpolator(x[:n, :2], x[:n, 2])(x[n:, :2])
    ok = np.isfinite(zl)
    return x[n:, 2][ok] - zl[ok]


def run(z_upper, h, steps):
    sc, n = plies(z_upper)
    o = Oracle(sc, h=h, newton_iterations=4, pcg_iterations=200, pcg_rel_tol=1e-6, self_contact=True, cross_layer=True, **MG)
    worst = np.inf
    for s in range(steps):
        o.substep()
        if s % 5 == 4 or s == steps - 1:
            g = gaps(o, n)
            worst = min(worst, g.min())
    return worst, g


def test_a_ply_laid_on_a_mounted_ply_rests_at_the_contact_distance():
    worst, g = run(0.0009, 1 / 120, 60)
    assert worst > 0.75 * R, worst
    assert abs(np.median(g) - R) < 0.03 * R and g.min() > 0.95 * R, (np.median(g), g.min())


def test_mounted_plies_overlapping_by_half_the_distance_are_pushed_apart():
    """Both plies mounted at their borders, the upper one 0.35 mm above the lower (half the contact
    distance): contact pushes the interiors apart to at least the contact distance."""
    m = btd.material_preset(0)
    sc = btd.compile_scene([btd.layer_spec(m, 0.015, 0.015, bundle=(1, 1), z=z, seed=3) for z in (0.0, 0.5 * R)])
    L0 = sc.layers[0]
    n = L0.nx * L0.ny
    k = np.arange(2 * n) % n
    i, j = k % L0.nx, k // L0.nx
    sc.pinned[:] = ((i == 0) | (j == 0) | (i == L0.nx - 1) | (j == L0.ny - 1)).astype(np.uint8)
    o = Oracle(sc, h=1 / 120, newton_iterations=4, pcg_iterations=200, pcg_rel_tol=1e-6, self_contact=True, cross_layer=True, **MG)
    for _ in range(20):
        o.substep()
    x = o.x
    d = (x[n:, 2] - x[:n, 2]).reshape(L0.ny, L0.nx)[3:-3, 3:-3]
    assert d.min() > 0.95 * R, d.min()


def test_one_layer_keeps_self_contact():
    sc = btd.configs.hanging_patch(12, 0.04, seed=2)
    a, b = (Oracle(sc, h=1 / 120, newton_iterations=2, pcg_iterations=50, pcg_rel_tol=1e-6, self_contact=True, cross_layer=c, **MG)
            for c in (False, True))
    for _ in range(5):
        a.substep()
        b.substep()
    assert np.array_equal(a.x, b.x)
