"""PSD projection of near-degenerate element blocks (an extension: the reference's projections are
closed forms, newtonMultigrid.ts:127-157, assemble.wgsl:53-65): the device's FP64 eigen-clamp (cyclic
Jacobi) against numpy's symmetric eigensolver on random, clustered, rank-deficient and indefinite 3 x 3
blocks, and the spring block of a near-degenerate element against the closed form it equals in exact
arithmetic (eigenvalues K along the element and f / l across it, each clamped at zero). The element
matrices of the lattice reduce to such 3 x 3 problems: a span or shear diagonal is [[H, -H], [-H, H]]
(PSD exactly when H is), a bending triple (w w^T) x M with w w^T PSD, and the contact terms enter as
diagonal blocks (selfcontact.wgsl:521-534).
"""
import ctypes as C

import numpy as np
import pytest

from btd_b200 import _abi

pytestmark = pytest.mark.gpu


def run(blocks, mode):
    a = np.ascontiguousarray(blocks, np.float64).reshape(-1, 6)
    out = np.zeros_like(a)
    _abi.check("btd_debug_projection", a.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p), len(a), mode)
    return out


def sym6(M):
    return np.stack([M[:, 0, 0], M[:, 0, 1], M[:, 0, 2], M[:, 1, 1], M[:, 1, 2], M[:, 2, 2]], 1)


def full(S):
    i = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
    return S[:, i]


def clamp_ref(M):
    w, V = np.linalg.eigh(M)
    return np.einsum("nij,nj,nkj->nik", V, np.maximum(w, 0), V)


def test_eigen_clamp_matches_numpy():
    rng = np.random.default_rng(3)
    n = 4000
    Q, _ = np.linalg.qr(rng.standard_normal((n, 3, 3)))
    lam = rng.standard_normal((n, 3)) * 10.0 ** rng.uniform(-3, 3, (n, 1))
    lam[: n // 4, 1] = lam[: n // 4, 0]                       # a repeated eigenvalue
    lam[n // 4: n // 2, 2] = lam[n // 4: n // 2, 0] * (1 + 1e-9)  # nearly repeated
    lam[n // 2: 5 * n // 8, 1:] = 0.0                         # rank one
    lam[5 * n // 8: 3 * n // 4] = -np.abs(lam[5 * n // 8: 3 * n // 4])  # negative definite
    M = np.einsum("nij,nj,nkj->nik", Q, lam, Q)
    M = 0.5 * (M + M.transpose(0, 2, 1))
    got = full(run(sym6(M), 0))
    ref = clamp_ref(M)
    scale = np.abs(M).reshape(n, -1).max(1)[:, None, None]
    assert np.abs(got - ref).max(axis=(1, 2)).max() <= 1e-12 * scale.max()
    assert (np.abs(got - ref) <= 1e-12 * scale + 1e-300).all()
    # already diagonal and zero blocks
    D = np.zeros((3, 3, 3))
    D[1] = np.diag([3.0, -1.0, 2.0])
    np.testing.assert_allclose(full(run(sym6(D), 0)), clamp_ref(D), atol=1e-15)


def test_spring_block_equals_the_closed_form():
    rng = np.random.default_rng(4)
    n = 2000
    d = rng.standard_normal((n, 3)) * 10.0 ** rng.uniform(-9, -3, (n, 1))
    K = rng.uniform(0, 1e4, n)
    f = rng.standard_normal(n) * 10.0
    got = full(run(np.column_stack([K, f, d, np.zeros(n)]), 1))
    l = np.linalg.norm(d, axis=1)
    e = d / l[:, None]
    kperp = np.maximum(f, 0) / l
    ref = (K - kperp)[:, None, None] * np.einsum("ni,nj->nij", e, e) + kperp[:, None, None] * np.eye(3)
    scale = np.maximum(K, kperp)[:, None, None]
    assert (np.abs(got - ref) <= 1e-6 * scale).all()
    # a zero-length element: max(K, 0) I
    z = run(np.array([[5.0, -1.0, 0.0, 0.0, 0.0, 0.0]]), 1)
    np.testing.assert_allclose(z[0], [5, 0, 0, 5, 0, 5])
