"""Shared fixtures of the parity tests: the reference's GPU-test coupon and state transfer."""
import numpy as np

import btd_b200 as btd

DENIM = btd.material_preset(0)


def correctness_coupon(nu=48, nv=40, **kw):
    """coupon() of tests/gpu/correctness.ts:27-45: bundled [3, 2], worn, so every wear-dependent term varies."""
    wear = dict(center=(0, 0), axis=(1, 0), radii=(0.03, 0.03), amount=1, cell_size=0, feature_scale=0.01,
                defect_threshold=2, defect_density=0, sparse_from=2)
    args = dict(bundle=(3, 2), angle=0.3, compress_u=0.03, compress_v=0.02, shear=0.02, collar_rows=2, seed=7,
                perturbation=0.4e-3, wear=wear, wear_strength_loss=(0.45, 0.9))
    args.update(kw)
    return btd.layer_spec(DENIM, (nu - 1) * 3 * DENIM.pitch_u, (nv - 1) * 2 * DENIM.pitch_v, **args)


def reference_params(**kw):
    """PARAMS of the reference's GPU parity suite: GPU_DEFAULTS without self-contact, which its f64
    CPU solver lacks (correctness.ts:24)."""
    kw.setdefault("self_contact", 0)
    return btd.default_params(**kw)


# The reference schedule matching GPU_DEFAULTS (correctness.ts:20-24).
MG = dict(max_coarsest_nodes=400, coarse_sweeps=2, line_colors=3, lag_coarse=True, line_search=True)


def max_abs_rel_to_scale(a, b):
    """maxAbsRelToScale (correctness.ts:79-87)."""
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def copy_state(oracle, gpu):
    """copyState (correctness.ts:146-163): both continue from the float32-rounded state."""
    x, v, _, _ = oracle.state()
    xf = x.astype(np.float32).astype(np.float64)
    vf = v.astype(np.float32).astype(np.float64)
    oracle.set_state(xf, vf)
    gpu.set_state(xf, vf)
    seg = oracle.segments()
    gpu.set_segments(**seg)
    gpu.set_field(oracle.field())
    return xf, vf


def kink_rows(oracle):
    """kinkRows (correctness.ts:53-68): rows touched by a span within rounding of the axial kink."""
    x, _, dx, _ = oracle.state()
    seg = oracle.segments()
    sc = oracle.scene
    nx = sc.nx
    rows = set()
    for s in range(2 * sc.N):
        if (seg["seg_flags"][s] & 3) != 1:
            continue
        a = s >> 1
        b = a + (1 if s & 1 == 0 else nx)
        l = np.linalg.norm((x[b] + dx[b]) - (x[a] + dx[a]))
        if abs(l / seg["rest_length"][s] - 1) < 1e-6:
            rows.update((a, b))
    return rows


def operator_apply(A, nx, ny, d, fixed=None):
    """y = A d in FP64 with a single-layer level operator read back in the reference's 25-offset
    layout (offset o: di = o % 5 - 2, dj = o // 5 - 2; newtonMultigrid.ts:38-48), rows of fixed nodes
    zero when `fixed` is given (StencilOperator.apply, newtonMultigrid.ts:96-125)."""
    d = np.asarray(d, np.float64).reshape(-1, 3)
    y = np.zeros_like(d)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny))
    i, j = i.reshape(-1), j.reshape(-1)
    for o in range(25):
        di, dj = o % 5 - 2, o // 5 - 2
        ok = (i + di >= 0) & (i + di < nx) & (j + dj >= 0) & (j + dj < ny)
        n = np.nonzero(ok)[0]
        m = (j[ok] + dj) * nx + (i[ok] + di)
        y[n] += np.einsum("nab,nb->na", A[n, o], d[m])
    if fixed is not None:
        y[np.asarray(fixed).reshape(-1) != 0] = 0.0
    return y
