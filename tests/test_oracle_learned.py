"""The learned coarse correction of configuration 4 (an extension with no counterpart in the reference),
on the oracle: a learned coarse space on the coarsest V-cycle level, its network trained on the
residual / exact-correction pairs the solver logs.

Checked here: the network's backward pass against central finite differences of its objective; the
C++ evaluation used inside the V-cycle against the numpy one; the logged pairs (the exact correction
solves the whitened coarsest system); the plain method unchanged, bit for bit, when the network is
off or only logging; what the trained network gains over the method without it on a held-out seed
(PCG iterations per Newton step to relative residual 1e-6, same positions within the solve tolerance);
and the guard that falls back to plain Galerkin MG-PCG when a solve does not contract.

Scenes: the plain configuration's 64 x 64 hanging patch (0.3 m, dt 1/60, 4 projected-Newton
iterations, lagged 3-level hierarchy, rel-res 1e-6), seeded jitter, training on seed 1 and evaluation
on seed 2, also with the hierarchy rebuilt every Newton iteration; and configuration 4's tearing patch
scaled down to 64 x 64 at its pitch (16 x 16-cell yarn region of lognormal break strains, self-contact,
edge grips pulled apart at 0.5 m/s), training on seed 41 together with the hanging patch's material,
evaluation on seed 42."""
import numpy as np
import pytest

from btd_b200 import configs
from oracle import Oracle, learned_dims, learned_forward
from oracle import learned as L

P = dict(h=1 / 60, newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, max_coarsest_nodes=400, coarse_sweeps=2,
         line_colors=3, lag_coarse=True, line_search=True)


def run(o, substeps):
    its, rel = [], []
    for _ in range(substeps):
        o.predict()
        for _ in range(P["newton_iterations"]):
            r = o.newton_step()
            its.append(r["pcg_iterations"])
            rel.append(r["rel_residual"])
        o.finalize()
        o.update_damage()
    return np.array(its), np.array(rel)


@pytest.fixture(scope="module")
def logged():
    o = Oracle(configs.hanging_patch(64, 0.3, seed=1), **P)
    o.learned_log(True, 4000)
    run(o, 6)
    return o.learned_samples()


@pytest.fixture(scope="module")
def trained(logged):
    ops, calls = logged
    w, hist = L.train(ops, calls, steps=500)
    return w, hist


C4 = configs.CONFIG4


def tearing(seed, substeps, weights=None, log=False):
    """Configuration 4 scaled to 64 x 64 on the oracle: the two edge grips move apart at its speed."""
    sc, left, right = configs.config4(seed, n=64, region=16)
    o = Oracle(sc, h=C4["h"], newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, max_coarsest_nodes=400,
               coarse_sweeps=2, line_colors=3, lag_coarse=True, line_search=True, self_contact=True)
    if weights is not None:
        o.set_learned(weights, on=True, guard=C4["guard"])
    if log:
        o.learned_log(True, 4000)
    x0 = o.x
    grips = [(int(nodes[len(nodes) // 2]), sign) for nodes, sign in ((left, -1.0), (right, 1.0))]
    for (picked, _), nodes in zip(grips, (left, right)):
        o.add_grip(nodes, np.ones(len(nodes)), (x0[nodes] - x0[picked]).reshape(-1), x0[picked], C4["grip_stiffness"])
    its, rel = [], []
    for s in range(1, substeps + 1):
        for g, (picked, sign) in enumerate(grips):
            o.set_grip_goal(g, x0[picked] + np.array([sign * 0.5 * C4["grip_speed"] * s * C4["h"], 0, 0]))
        o.predict()
        for _ in range(4):
            r = o.newton_step()
            its.append(r["pcg_iterations"])
            rel.append(r["rel_residual"])
        o.finalize()
        o.update_damage()
    return o, np.array(its), np.array(rel)


@pytest.fixture(scope="module")
def trained_mix(logged):
    """Trained on the hanging patch's material and a tearing patch's (seed 41)."""
    o, _, _ = tearing(41, 8, log=True)
    ops4, calls4 = o.learned_samples()
    ops0, calls0 = logged
    ops = ops0 + ops4
    calls = calls0 + [(op + len(ops0), r, d) for op, r, d in calls4]
    w, _ = L.train(ops, calls, steps=800)
    return w


def test_dimensions():
    assert learned_dims() == (L.IN, L.HID, L.K)
    assert L.SIZE == L.IN * L.HID + L.HID + L.HID * L.HID + L.HID + L.HID * L.OUT + L.OUT


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    n = 12
    Q = rng.standard_normal((3 * n, 3 * n))
    At = Q @ Q.T + 3 * n * np.eye(3 * n)
    X = rng.standard_normal((n, L.IN))
    ops = [(At, X)]
    calls = []
    for _ in range(3):
        r = rng.standard_normal(3 * n)
        calls.append((0, r, np.linalg.solve(At, r)))
    w = L.init(3) * 0.7
    f0, g = L.loss_grad(w, ops, calls)
    assert 0 < f0 < 1
    for _ in range(6):
        u = rng.standard_normal(L.SIZE)
        u /= np.linalg.norm(u)
        e = 1e-5
        fd = (L.loss_grad(w + e * u, ops, calls)[0] - L.loss_grad(w - e * u, ops, calls)[0]) / (2 * e)
        assert abs(fd - g @ u) <= 1e-6 * max(1e-3, abs(fd)), (fd, g @ u)


def test_cpp_forward_matches_numpy():
    rng = np.random.default_rng(9)
    w = L.init(1)
    X = rng.standard_normal((257, L.IN))
    np.testing.assert_allclose(learned_forward(w, X), L.forward(w, X), rtol=1e-12, atol=1e-12)


def test_logged_pairs_solve_the_coarsest_system(logged):
    ops, calls = logged
    assert len(ops) == 6  # lagged hierarchy: one coarsest operator per substep
    assert len(calls) > 100
    for At, X in ops:
        assert At.shape == (3 * len(X), 3 * len(X)) and X.shape[1] == L.IN
        np.testing.assert_allclose(At, At.T, atol=1e-9 * np.abs(At).max())
    for op, r, d in calls[:: max(1, len(calls) // 20)]:
        At = ops[op][0]
        assert np.linalg.norm(At @ d - r) <= 1e-8 * np.linalg.norm(r)


def test_plain_method_unchanged_when_off_or_logging(trained):
    w, _ = trained
    sc = configs.hanging_patch(64, 0.3, seed=2)
    a, b, c = Oracle(sc, **P), Oracle(sc, **P), Oracle(sc, **P)
    b.set_learned(w, on=False)
    c.learned_log(True, 50)
    ia, _ = run(a, 2)
    ib, _ = run(b, 2)
    ic, _ = run(c, 2)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.x, c.x)
    assert np.array_equal(ia, ib) and np.array_equal(ia, ic)


def test_trained_network_gains_on_a_held_out_seed(trained):
    w, hist = trained
    assert hist[-1] < 0.75 * hist[0]  # the captured share of the error energy grows in training
    sc = configs.hanging_patch(64, 0.3, seed=2)
    x0 = sc.position.reshape(-1, 3).copy()
    plain, learn = Oracle(sc, **P), Oracle(sc, **P)
    learn.set_learned(w, on=True, guard=0.9)
    ip, rp = run(plain, 4)
    il, rl = run(learn, 4)
    stats = learn.learned_stats()
    print(f"PCG iterations per Newton step: plain {ip.mean():.2f}, learned {il.mean():.2f} "
          f"({ip.mean() / il.mean():.2f}x fewer); {stats}")
    assert il.mean() <= 0.85 * ip.mean()
    assert rp.max() <= 1e-6 and rl.max() <= 1e-6
    assert stats["solves"] == len(il) and stats["fallbacks"] == 0 and stats["applied"] > 0
    motion = np.abs(plain.x - x0).max()
    assert np.abs(plain.x - learn.x).max() <= 1e-2 * motion


def test_guard_falls_back_to_plain_mg_pcg(trained):
    w, _ = trained
    sc = configs.hanging_patch(64, 0.3, seed=2)
    o = Oracle(sc, **P)
    o.set_learned(w, on=True, guard=0.05)  # no solve contracts 20x per iteration: every one falls back
    its, rel = run(o, 1)
    s = o.learned_stats()
    assert s["fallbacks"] == s["solves"] == len(its)
    assert rel.max() <= 1e-6


def test_trained_network_gains_with_a_fresh_hierarchy(trained):
    """Trained on the lagged hierarchy's material, used with the hierarchy rebuilt every Newton iteration."""
    w, _ = trained
    sc = configs.hanging_patch(64, 0.3, seed=2)
    p = dict(P, lag_coarse=False)
    plain, learn = Oracle(sc, **p), Oracle(sc, **p)
    learn.set_learned(w, on=True, guard=0.9)
    ip, _ = run(plain, 3)
    il, rl = run(learn, 3)
    print(f"fresh hierarchy: plain {ip.mean():.2f}, learned {il.mean():.2f} PCG iterations per Newton step")
    assert il.mean() <= 0.8 * ip.mean()
    assert rl.max() <= 1e-6


def test_tearing_patch_gains_on_a_held_out_seed(trained_mix):
    o_p, ip, rp = tearing(42, 8)
    o_l, il, rl = tearing(42, 8, weights=trained_mix)
    broken_p, broken_l = o_p.counts()[0], o_l.counts()[0]
    print(f"tearing patch: plain {ip.mean():.2f}, learned {il.mean():.2f} PCG iterations per Newton step; "
          f"{o_l.learned_stats()}; spans broken {broken_p} / {broken_l}")
    assert broken_p > 0  # the patch tears within these substeps
    assert il.mean() <= 0.95 * ip.mean()
    assert rp.max() <= 1e-6 and rl.max() <= 1e-6


def test_headline_size_with_a_fresh_hierarchy(trained):
    """The 256 x 256 hanging patch (0.6 m, 5 levels, coarsest 17 x 17), hierarchy rebuilt every Newton
    iteration, with the network trained on the 64 x 64 patch's material."""
    w, _ = trained
    sc = configs.hanging_patch(256, 0.6, seed=1)
    p = dict(P, lag_coarse=False)
    plain, learn = Oracle(sc, **p), Oracle(sc, **p)
    learn.set_learned(w, on=True, guard=0.9)
    ip, _ = run(plain, 2)
    il, rl = run(learn, 2)
    print(f"256 x 256, fresh hierarchy: plain {ip.mean():.2f}, learned {il.mean():.2f} PCG iterations per Newton step")
    assert il.mean() <= 0.8 * ip.mean()
    assert rl.max() <= 1e-6


def test_committed_weights_gain_without_costing():
    """The network trained by oracle/train_learned.py on 1.7 M node pairs logged by the plain solver on
    configurations 0, 1, 3 and 4 (tests/golden/learned_coarse.npy): fewer PCG iterations per Newton step
    on the held-out hanging patch, lagged or rebuilt hierarchy, and none more on the held-out tearing
    patch."""
    import os
    w = np.load(os.path.join(os.path.dirname(__file__), "golden", "learned_coarse.npy")).astype(np.float64)
    assert w.shape == (L.SIZE,)
    for lag, bound in ((True, 0.8), (False, 0.7)):
        p = dict(P, lag_coarse=lag)
        sc = configs.hanging_patch(64, 0.3, seed=2)
        plain, learn = Oracle(sc, **p), Oracle(sc, **p)
        learn.set_learned(w, on=True, guard=0.9)
        ip, _ = run(plain, 2)
        il, rl = run(learn, 2)
        print(f"committed weights, hanging patch, lagged={lag}: plain {ip.mean():.2f}, learned {il.mean():.2f}")
        assert il.mean() <= bound * ip.mean() and rl.max() <= 1e-6
    _, ip, _ = tearing(42, 4)
    o, il, rl = tearing(42, 4, weights=w)
    print(f"committed weights, tearing patch: plain {ip.mean():.2f}, learned {il.mean():.2f}")
    assert il.mean() <= 1.02 * ip.mean() and rl.max() <= 1e-6


def test_config4_scene():
    """Configuration 4's tearing patch at full size: 256 x 256 over 0.6 m bundled [2, 2], the central
    64 x 64 cells' crossings with lognormal(ln 0.08, 0.25) break strains (as tensions EA eps), the rest
    holding to 10 EA, no pins, grips on the two edge column pairs; scaled, the same pitch."""
    c = configs.CONFIG4
    sc, left, right = configs.config4()
    assert (sc.nx, sc.ny) == (256, 256) and not sc.pinned.any()
    pos = sc.position.reshape(-1, 3)
    assert np.isclose(pos[1, 0] - pos[0, 0], 0.6 / 255, rtol=1e-4)
    L = sc.layers[0]
    s = sc.field_strength.reshape(L.field_m, L.field_k, 2)
    lo = (256 - 64) // 2
    inner = s[2 * lo:2 * (lo + 64), 2 * lo:2 * (lo + 64)]
    eps = inner / c["yarn_ea"]
    assert abs(np.median(np.log(eps)) - np.log(0.08)) < 0.01 and abs(np.log(eps).std() - 0.25) < 0.01
    mask = np.ones(s.shape[:2], bool)
    mask[2 * lo:2 * (lo + 64), 2 * lo:2 * (lo + 64)] = False
    assert np.allclose(s[mask], 10 * c["yarn_ea"])
    assert len(left) == len(right) == 2 * 256
    small, _, _ = configs.config4(n=64, region=16)
    p = small.position.reshape(-1, 3)
    assert (small.nx, small.ny) == (64, 64) and np.isclose(p[1, 0] - p[0, 0], 0.6 / 255, rtol=1e-4)
