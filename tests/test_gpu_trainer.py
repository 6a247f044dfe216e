"""Training of the learned coarse correction's network on the GPU (configuration 4's extension; no
counterpart in the reference) against the oracle's FP64 numpy restatement (oracle/learned.py).

Checked: the GPU's loss and gradient (BF16 forward and backward on the tensor cores, FP32 accumulation)
against the FP64 loss and backward of the same BF16-rounded weights on the same material (logged by the
oracle); GPU training from the same start lowers the loss as the FP64 training does; the material the
GPU solver logs on the device and the trainer whitens and solves (whitened diagonal blocks are the
identity, the operators symmetric, the exact corrections solve them); and a network trained on the GPU
from the GPU solver's own log makes PCG converge in fewer iterations on a held-out seed.
"""
import numpy as np
import pytest

import btd_b200 as btd
from btd_b200 import learned
from helpers import MG
from oracle import Oracle
from oracle import learned as L

pytestmark = pytest.mark.gpu

P0 = dict(h=1 / 60, newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, **MG)


def bf16(w):
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)).view(np.float32)


@pytest.fixture(scope="module")
def material():
    """The oracle's logged material on the plain configuration's hanging patch (seed 1, 3 substeps)."""
    o = Oracle(btd.configs.hanging_patch(64, 0.3, seed=1), **P0)
    o.learned_log(True, 2000)
    for _ in range(3):
        o.substep()
    return o.learned_samples()


@pytest.fixture(scope="module")
def trainer(material):
    ops, calls = material
    tr = learned.Trainer()
    by = {}
    for op, r, d in calls:
        by.setdefault(op, []).append((r, d))
    for k, (At, X) in enumerate(ops):
        rd = by.get(k, [])
        tr.add_op(At, X, np.array([a for a, _ in rd]), np.array([b for _, b in rd]))
    return tr


def test_loss_and_gradient_match_the_fp64_backward(material, trainer):
    ops, calls = material
    w = bf16(L.init(3).astype(np.float32) * 0.7)
    loss_ref, g_ref = L.loss_grad(w.astype(np.float64), ops, calls)
    loss, g = trainer.loss_grad(w, list(range(len(ops))))
    assert abs(loss - loss_ref) <= 1e-2 * max(loss_ref, 1e-3) + 1e-4, (loss, loss_ref)
    err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    cos = float(g @ g_ref) / (np.linalg.norm(g) * np.linalg.norm(g_ref))
    assert err < 5e-2 and cos > 0.998, (err, cos)
    # per layer too: the backward of each weight matrix and bias
    q = 0
    for s in L.SHAPES:
        n = int(np.prod(s))
        a, b = g[q:q + n], g_ref[q:q + n]
        assert np.linalg.norm(a - b) <= 8e-2 * np.linalg.norm(b) + 1e-9, (s, np.linalg.norm(a - b) / np.linalg.norm(b))
        q += n


def test_gpu_training_lowers_the_loss_like_fp64_training(material, trainer):
    ops, calls = material
    w0 = L.init(0).astype(np.float32)
    steps = 300
    w_gpu, hist = trainer.train(w0, steps=steps, batch_ops=3, lr=3e-3, seed=0)
    l0 = L.loss_grad(bf16(w0).astype(np.float64), ops, calls)[0]
    l_gpu = L.loss_grad(bf16(w_gpu).astype(np.float64), ops, calls)[0]
    w_ref, _ = L.train(ops, calls, steps=steps, batch_ops=3, lr=3e-3, seed=0, w=w0.astype(np.float64))
    l_ref = L.loss_grad(w_ref, ops, calls)[0]
    assert np.isfinite(hist).all()
    assert l_gpu < l0 - 0.5 * (l0 - l_ref), (l0, l_gpu, l_ref)


@pytest.fixture(scope="module")
def gpu_logged():
    """The GPU solver's own log on the hanging patch (seeds 1 and 3, 4 substeps each), in a trainer."""
    tr = learned.Trainer()
    for seed in (1, 3):
        g = btd.GpuSolver(btd.configs.hanging_patch(64, 0.3, seed=seed), btd.configs.solver_params(1 / 60, 4, 1e-6))
        learned.log_run(g, 4)
        st = g.learned_stats()
        assert st["logged_ops"] == 4 and st["logged_calls"] > 100, st
        assert tr.add_log(g) == 4
        g.close()
    return tr


def test_logging_leaves_the_plain_solve_unchanged():
    sc = btd.configs.hanging_patch(32, 0.15, seed=6)
    xs = []
    for log in (False, True):
        g = btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6))
        if log:
            g.learned_log(True, 8, 2048)
        g.substeps(3)
        g.synchronize()
        xs.append(g.x.copy())
        g.close()
    assert np.array_equal(xs[0], xs[1])


def test_device_material_is_whitened_and_solved(gpu_logged):
    ops, calls = gpu_logged.counts()
    assert ops == 8 and calls > 400
    for k in (0, ops - 1):
        At, X, R, D, E = gpu_logged.op(k)
        n = len(X)
        assert At.shape == (3 * n, 3 * n) and n > 200
        np.testing.assert_allclose(At, At.T, atol=1e-5 * np.abs(At).max())
        for i in range(0, n, 17):  # the whitened diagonal blocks are the identity
            np.testing.assert_allclose(At[3 * i:3 * i + 3, 3 * i:3 * i + 3], np.eye(3), atol=1e-4)
        A64 = At.astype(np.float64)
        for c in range(0, len(R), max(1, len(R) // 8)):
            res = A64 @ D[c] - R[c]
            assert np.linalg.norm(res) <= 1e-3 * np.linalg.norm(R[c]), np.linalg.norm(res) / np.linalg.norm(R[c])
            assert abs(E[c] - float(R[c].astype(np.float64) @ D[c])) <= 1e-4 * E[c]
        # inputs: lattice position in [0, 1], trace-normalised diagonal summing to 1
        assert (X[:, 0] >= 0).all() and (X[:, 0] <= 1).all()
        np.testing.assert_allclose(X[:, 10] + X[:, 11] + X[:, 12], 1.0, atol=1e-5)


def test_network_trained_on_the_gpu_gains_on_a_held_out_seed(gpu_logged):
    w, hist = gpu_logged.train(learned.init_weights(0), steps=600, batch_ops=4, lr=3e-3, seed=0)
    assert hist[-50:].mean() < hist[:50].mean() - 0.1, (hist[:50].mean(), hist[-50:].mean())
    sc = btd.configs.hanging_patch(64, 0.3, seed=2)
    its = {}
    for on in (False, True):
        g = btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6))
        if on:
            g.set_learned(w, on=True, guard=0.9)
        g.substeps(4)
        c = g.counter_dict()
        its[on] = c["pcg_total"] / c["newton"]
        g.close()
    assert its[True] <= 0.85 * its[False], its
