"""The reference's own property tests, run against the FP64 oracle (no GPU).

The reference pins its CPU solver with property tests rather than golden vectors
(tests/unit/newtonMultigrid.test.ts, tests/unit/referenceSolver.test.ts). Each test below restates
one of them with the same fixture (seeded LCG, coupon spec) and the same bound, so the oracle is
held to exactly what the reference holds its own solver to.
"""
import math

import numpy as np
import pytest

import btd_b200 as btd
from oracle import Oracle, solve_penta


def rng(seed):
    """The tests' LCG (newtonMultigrid.test.ts:19-25): uniform in [-0.5, 0.5)."""
    s = [seed & 0xFFFFFFFF]

    def nxt():
        s[0] = (s[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return s[0] / 4294967296 - 0.5

    return nxt


DENIM = btd.material_preset(0)


def coupon_mg(nu, nv):
    """coupon() of newtonMultigrid.test.ts:27-43."""
    return btd.layer_spec(DENIM, (nu - 1) * DENIM.pitch_u, (nv - 1) * DENIM.pitch_v, angle=0.3, compress_u=0.02,
                          compress_v=0.01, shear=0.01, collar_rows=2, seed=3, perturbation=0.3e-3)


def coupon_rs(nu, nv, **kw):
    """coupon() of referenceSolver.test.ts:7-23."""
    args = dict(angle=0.3, compress_u=0.01, compress_v=0.005, shear=0.01, collar_rows=1, seed=7, perturbation=0.2e-3)
    args.update(kw)
    return btd.layer_spec(DENIM, (nu - 1) * DENIM.pitch_u, (nv - 1) * DENIM.pitch_v, **args)


def to_dense(A, nx, ny):
    """toDense (newtonMultigrid.test.ts:45-59) for a single layer."""
    N = nx * ny
    M = np.zeros((3 * N, 3 * N))
    for n in range(N):
        j, i = divmod(n, nx)
        for dj in range(-2, 3):
            for di in range(-2, 3):
                if not (0 <= i + di < nx and 0 <= j + dj < ny):
                    continue
                m = n + dj * nx + di
                M[3 * n:3 * n + 3, 3 * m:3 * m + 3] = A[n, (dj + 2) * 5 + di + 2]
    return M


def test_block_pentadiagonal_solve_matches_the_system():
    """newtonMultigrid.test.ts:62-93: residual < 1e-12."""
    r = rng(9)
    n = 9
    D = np.zeros((n, 3, 3))
    E = np.zeros((n, 3, 3))
    F = np.zeros((n, 3, 3))
    for k in range(n):
        for q in range(9):
            E[k].flat[q] = r()
            F[k].flat[q] = 0.5 * r()
        for a in range(3):
            for b in range(3):
                D[k, a, b] = 12 if a == b else 0.3 * (a + b - 2)
    rhs = np.array([r() for _ in range(3 * n)])
    x = solve_penta(D, E, F, rhs)
    for k in range(n):
        s = D[k] @ x[k]
        if k + 1 < n:
            s += E[k] @ x[k + 1]
        if k + 2 < n:
            s += F[k] @ x[k + 2]
        if k >= 1:
            s += E[k - 1].T @ x[k - 1]
        if k >= 2:
            s += F[k - 2].T @ x[k - 2]
        assert np.abs(s - rhs[3 * k:3 * k + 3]).max() < 1e-12


def test_operator_symmetric_and_galerkin_equals_ptap():
    """newtonMultigrid.test.ts:95-151: asymmetry < 1e-12, coarse = P^T A P < 1e-10."""
    sc = btd.compile_scene(coupon_mg(11, 9))
    o = Oracle(sc)
    o.predict()
    A, fixed, _ = o.assemble()
    nx, ny = sc.nx, sc.ny
    M = to_dense(A, nx, ny)
    assert np.abs(M - M.T).max() / np.abs(M).max() < 1e-12
    o.build_levels(A)
    Ac, fixc = o.level(1)
    idx, w = o.prolongation(0)
    nxc, nyc = (nx - 1 + 1) // 2 + 1, (ny - 1 + 1) // 2 + 1
    Mc = to_dense(Ac, nxc, nyc)
    N, Nc = sc.N, nxc * nyc
    Pd = np.zeros((3 * N, 3 * Nc))
    for f in range(N):
        for k in range(4):
            c = idx[f, k]
            if c < 0:
                continue
            for q in range(3):
                Pd[3 * f + q, 3 * c + q] = w[f, k]
    Mf = M.copy()
    for n in np.nonzero(fixed)[0]:
        Mf[3 * n:3 * n + 3, :] = 0
        Mf[:, 3 * n:3 * n + 3] = 0
    S = Pd.T @ Mf @ Pd
    keep = np.repeat(fixc == 0, 3)
    err = np.abs(S - Mc)[np.ix_(keep, keep)].max()
    assert err / np.abs(S[np.ix_(keep, keep)]).max() < 1e-10


def test_smoothing_vcycle_and_pcg_reduce_the_residual():
    """newtonMultigrid.test.ts:153-194."""
    sc = btd.compile_scene(coupon_mg(40, 30))
    o = Oracle(sc)
    o.predict()
    A, fixed, _ = o.assemble()
    o.build_levels(A)
    r = rng(4)
    b = np.array([r() for _ in range(3 * sc.N)]).reshape(-1, 3)
    b[fixed != 0] = 0

    def norm(x):
        return math.sqrt(((b - o.apply(0, x)) ** 2).sum())

    x = np.zeros_like(b)
    r0 = norm(x)
    assert norm(o.smooth(0, x, b)) < r0
    assert o.level_count() > 2
    assert norm(o.vcycle(b)) < 0.5 * r0
    xs = np.array([1e-5 * r() for _ in range(3 * sc.N)]).reshape(-1, 3)
    xs[fixed != 0] = 0
    bs = o.apply(0, xs)

    def enorm(x):
        e = x - xs
        return math.sqrt((e * o.apply(0, e)).sum())

    e0 = enorm(np.zeros_like(xs))
    z, done, _ = o.pcg(bs, 3)
    assert done == 3
    assert enorm(z) / e0 < 5e-3


def randomize(o, amp, seed=1):
    """randomize (referenceSolver.test.ts:25-35)."""
    s = [seed]

    def rnd():
        s[0] = (s[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return s[0] / 4294967296 - 0.5

    _, _, dx, pred = o.state()
    dx = dx.copy()
    for n in range(o.N):
        if o.scene.pinned[n]:
            continue
        for q in range(3):
            dx[n, q] = amp * rnd()
    o.set_dx(dx, pred)
    return dx


def test_gradient_matches_finite_differences_of_the_potential():
    """referenceSolver.test.ts:39-64: relative error < 2e-4 for the first 20 free nodes."""
    sc = btd.compile_scene(coupon_rs(9, 8))
    o = Oracle(sc)
    v = np.array([0.01 * math.sin(q * 1.7) for q in range(3 * sc.N)])
    o.set_state(sc.position, v)
    o.predict()
    dx = randomize(o, 2e-5)
    _, _, _, pred = o.state()
    free = [n for n in range(sc.N) if not sc.pinned[n]]
    for n in free[:20]:
        g = o.node_gradient(n)
        for q in range(3):
            h = 1e-9
            d = dx.copy()
            d[n, q] += h
            o.set_dx(d, pred)
            ep = o.potential()
            d[n, q] -= 2 * h
            o.set_dx(d, pred)
            em = o.potential()
            o.set_dx(dx, pred)
            fd = (ep - em) / (2 * h)
            scale = max(1e-6, abs(fd), abs(g[q]))
            assert abs(fd - g[q]) / scale < 2e-4


def test_elastic_energy_invariant_under_rigid_motion():
    """referenceSolver.test.ts:66-99: relative change < 1e-7."""
    sc = btd.compile_scene(coupon_rs(8, 7, compress_u=0.0, compress_v=0.0, shear=0.0))
    o = Oracle(sc)
    dx = randomize(o, 3e-5, 5)
    o.set_dx(dx, dx)
    e0 = o.potential()
    ax = np.array([0.3, -0.5, 0.81])
    kx, ky, kz = ax / np.linalg.norm(ax)
    th = 0.7
    c, s = math.cos(th), math.sin(th)
    R = np.array([
        [c + kx * kx * (1 - c), kx * ky * (1 - c) - kz * s, kx * kz * (1 - c) + ky * s],
        [ky * kx * (1 - c) + kz * s, c + ky * ky * (1 - c), ky * kz * (1 - c) - kx * s],
        [kz * kx * (1 - c) - ky * s, kz * ky * (1 - c) + kx * s, c + kz * kz * (1 - c)],
    ])
    t = np.array([0.01, -0.02, 0.005])
    x = o.x
    y = x + dx
    rx = x @ R.T + t
    ry = y @ R.T + t
    o.set_state(rx)
    o.set_dx(ry - rx, ry - rx)
    e1 = o.potential()
    assert abs(e1 - e0) / max(e0, 1e-12) < 1e-7


def test_projected_newton_pcg_decreases_the_potential():
    """referenceSolver.test.ts:103-118."""
    sc = btd.compile_scene(coupon_rs(30, 24))
    o = Oracle(sc, h=1 / 240, newton_iterations=2, pcg_iterations=4)
    for _ in range(10):
        o.substep()
    o.predict()
    e0 = o.potential()
    prev = e0
    for _ in range(4):
        o.newton_step()
        e = o.potential()
        assert e <= prev * 1.02
        prev = e
    assert prev < e0


def test_settles_under_gravity_within_the_mounts():
    """referenceSolver.test.ts:120-135: 240 substeps, max |v| < 0.02, max |z| < 5 mm, no ruptures."""
    sc = btd.compile_scene(coupon_rs(20, 16))
    o = Oracle(sc, h=1 / 240, newton_iterations=2, pcg_iterations=4)
    for _ in range(240):
        o.substep()
    x, v, _, _ = o.state()
    assert np.isfinite(x).all()
    assert np.linalg.norm(v, axis=1).max() < 0.02
    assert np.abs(x[:, 2]).max() < 0.005
    assert o.counts()[0] == 0


def test_pulling_apart_ruptures_spans_and_conserves_yarn_length():
    """referenceSolver.test.ts:137-160: ruptures occur and the yarn-length ledger holds to 1e-9."""
    sc = btd.compile_scene(coupon_rs(14, 10, compress_u=0.0, compress_v=0.0, shear=0.0, perturbation=0.0))
    o = Oracle(sc, h=1 / 240, gravity=(0, 0, 0), newton_iterations=2, pcg_iterations=4)
    L0 = o.yarn_material_length()
    L = sc.layers[0]
    top = [L.node_offset + (L.ny - 1) * L.nx + i for i in range(L.nx)]
    vdir = np.array([L.map_a[1], L.map_a[3]])
    vdir /= np.linalg.norm(vdir)
    for _ in range(400):
        if o.counts()[0] >= 6:
            break
        x, v, _, _ = o.state()
        x = x.copy()
        x[top, 0] += (0.02 / 240) * vdir[0]
        x[top, 1] += (0.02 / 240) * vdir[1]
        o.set_state(x, v)
        o.substep()
    broken_count = o.counts()[0]
    assert broken_count > 0
    seg = o.segments()
    assert ((seg["seg_flags"] & btd.SEG_BROKEN) != 0).sum() >= broken_count
    assert abs(o.yarn_material_length() - L0) / L0 < 1e-9
