"""The learned coarse correction's network and its training on the GPU (configuration 4's extension;
no counterpart in the reference, whose coarsest V-cycle level is two line sweeps,
src/simulation/reference/newtonMultigrid.ts:495-502).

`Trainer` wraps btd_trainer of the C ABI: material comes from a solver's device-side log
(GpuSolver.learned_log, then Trainer.add_log) or from host arrays; `train` runs Adam on the GPU with the
library's BF16 forward and backward kernels. `train_network` is the product's training recipe: it
logs the plain solver's coarsest operators and residuals on the GPU over the configurations' scenes
and trains a network on them.

Weights: flat float32, W1[20][64] b1[64] W2[64][64] b2[64] W3[64][24] b3[24], row-major [in][out].
"""
import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import check

WEIGHTS = 7064
IN, HID, K = 20, 64, 8
SHAPES = ((IN, HID), (HID,), (HID, HID), (HID,), (HID, 3 * K), (3 * K,))
DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "learned_coarse.f32")


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def init_weights(seed=0):
    """Glorot-scaled weights (zero biases)."""
    rng = np.random.default_rng(seed)
    out = []
    for s in SHAPES:
        out.append(rng.standard_normal(s) * np.sqrt(1.0 / s[0]) if len(s) == 2 else np.zeros(s))
    return np.concatenate([a.reshape(-1) for a in out]).astype(np.float32)


def load(path=DEFAULT_PATH):
    w = np.fromfile(path, np.float32)
    if w.size != WEIGHTS:
        raise ValueError(f"{path}: {w.size} floats, expected {WEIGHTS}")
    return w


def save(w, path=DEFAULT_PATH):
    np.ascontiguousarray(w, np.float32).reshape(-1).tofile(path)


class Trainer:
    """Training material and Adam on the GPU (btd_trainer)."""

    def __init__(self):
        h = C.c_void_p()
        check("btd_trainer_create", C.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().btd_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def add_op(self, At, X, R, D, group=0):
        """Host material: At (3n, 3n), X (n, 20), R and D (calls, 3n), all whitened."""
        At = np.ascontiguousarray(At, np.float64)
        X = np.ascontiguousarray(X, np.float64)
        R = np.ascontiguousarray(R, np.float64).reshape(-1, At.shape[0])
        D = np.ascontiguousarray(D, np.float64).reshape(-1, At.shape[0])
        check("btd_trainer_add_op", self._h, len(X), _p(At), _p(X), len(R), _p(R), _p(D), int(group))

    def add_log(self, solver, group=0):
        """The solver's device-side log; returns the number of operators added."""
        n = C.c_int32()
        check("btd_trainer_add_log", self._h, solver._h, int(group), C.byref(n))
        return n.value

    def counts(self):
        ops, calls = C.c_int32(), C.c_int32()
        check("btd_trainer_counts", self._h, C.byref(ops), C.byref(calls))
        return ops.value, calls.value

    def op(self, k):
        """(At, X, R, D, E) of operator k as stored (float32; E float64)."""
        n, c = C.c_int32(), C.c_int32()
        check("btd_trainer_read_op", self._h, k, C.byref(n), C.byref(c), None, None, None, None, None)
        D3 = 3 * n.value
        At, X = np.zeros((D3, D3), np.float32), np.zeros((n.value, IN), np.float32)
        R, D, E = np.zeros((c.value, D3), np.float32), np.zeros((c.value, D3), np.float32), np.zeros(c.value)
        check("btd_trainer_read_op", self._h, k, C.byref(n), C.byref(c), _p(At), _p(X), _p(R), _p(D), _p(E))
        return At, X, R, D, E

    def loss_grad(self, weights, ops):
        w = np.ascontiguousarray(weights, np.float32)
        o = np.ascontiguousarray(ops, np.int32)
        loss, g = C.c_double(), np.zeros(WEIGHTS, np.float32)
        check("btd_trainer_loss_grad", self._h, _p(w), _p(o), len(o), C.byref(loss), _p(g))
        return loss.value, g

    def train(self, weights, steps=1500, batch_ops=6, lr=3e-3, seed=0, group_weights=None):
        """Adam on the GPU; returns (weights, loss of every step's minibatch)."""
        w = np.ascontiguousarray(weights, np.float32).copy()
        gw = None if group_weights is None else np.ascontiguousarray(group_weights, np.float32)
        hist = np.zeros(steps, np.float32)
        check("btd_trainer_train", self._h, _p(w), int(steps), int(batch_ops), C.c_float(lr), C.c_uint64(seed), _p(gw),
              0 if gw is None else len(gw), _p(hist))
        return w, hist


def log_run(solver, substeps, drive=None, capacity_ops=64, capacity_calls=8192):
    """Logs `substeps` substeps of the plain solve (the correction off) on the GPU; drive(s) sets the
    grip targets before substep s (1-based)."""
    solver.learned_log(True, capacity_ops, capacity_calls)
    for s in range(1, substeps + 1):
        if drive:
            drive(s)
        solver.substep()
    solver.synchronize()


def train_network(steps=1500, seed=0, verbose=True):
    """The product's training recipe, all on the GPU: the plain solver (lagged hierarchy, PCG to rel-res
    1e-6) logs its coarsest operators and residuals on the plain configuration's hanging patch (64 x 64,
    seeds 1 and 3, 6 substeps each), on the yarn-damage configuration (128 x 128 with its two edge grips,
    6 substeps), on eight patches of the batch (4 substeps each, grips moving) and on configuration 4's
    tearing patch scaled to 64 x 64 (8 substeps) and at its full 256 x 256 with another seed of its
    break strains than the benchmark's (seed 43, 24 substeps: the grips' pull and the start of the
    tear); then Adam over minibatches of 6 operators, each configuration weighing the same. Returns
    (weights, loss history)."""
    from . import configs
    from .solver import GpuSolver

    tr = Trainer()

    def edge(g, left, right, speed, h, k):
        x0 = g.x.astype(np.float32)
        grips = []
        for slot, (nodes, sign) in enumerate(((left, -1.0), (right, 1.0))):
            picked = int(nodes[len(nodes) // 2])
            g.attach_patch(slot, picked, nodes, np.ones(len(nodes)), x0[picked], k, max_lead=1.0)
            grips.append((x0[picked].astype(np.float64), sign))

        def drive(s):
            for slot, (a, sign) in enumerate(grips):
                g.set_target((a + np.array([sign * 0.5 * speed * s * h, 0, 0])).astype(np.float32), slot=slot)

        return drive

    groups = []
    c0 = configs.CONFIG0
    for seed_ in (1, 3):
        g = GpuSolver(configs.hanging_patch(64, 0.3, seed=seed_), configs.solver_params(c0["h"], 4, 1e-6))
        log_run(g, 6)
        groups.append(("config0", tr.add_log(g, 0)))
        g.close()
    c1 = configs.CONFIG1
    sc, left, right = configs.config1()
    g = GpuSolver(sc, configs.solver_params(c1["h"], 4, 1e-6))
    log_run(g, 6, edge(g, left, right, c1["grip_speed"], c1["h"], c1["grip_stiffness"]))
    groups.append(("config1", tr.add_log(g, 1)))
    g.close()
    c3 = configs.CONFIG3
    picked = 0
    for sc, gr in configs.config3(31, only=range(32)):
        if sc.N <= 400 or picked == 8:
            continue
        g = GpuSolver(sc, configs.solver_params(c3["h"], 4, 1e-6))
        p = gr["picked"]
        a = g.x[p].astype(np.float32)
        g.attach_patch(0, p, gr["nodes"], gr["weights"], a, gr["stiffness"], max_lead=gr["max_lead"])
        log_run(g, 4, lambda s, g=g, a=a, v=gr["velocity"]: g.set_target((a + v * s * c3["h"]).astype(np.float32)))
        groups.append(("config3", tr.add_log(g, 2)))
        g.close()
        picked += 1
    c4 = configs.CONFIG4
    sc, left, right = configs.config4(41, n=64, region=16)
    g = GpuSolver(sc, configs.solver_params(c4["h"], 4, 1e-6, self_contact=1))
    log_run(g, 8, edge(g, left, right, c4["grip_speed"], c4["h"], c4["grip_stiffness"]))
    groups.append(("config4", tr.add_log(g, 3)))
    g.close()
    sc, left, right = configs.config4(43)
    g = GpuSolver(sc, configs.solver_params(c4["h"], 4, 1e-6, self_contact=1))
    log_run(g, 24, edge(g, left, right, c4["grip_speed"], c4["h"], c4["grip_stiffness"]))
    groups.append(("config4-256", tr.add_log(g, 4)))
    g.close()
    if verbose:
        print("logged:", groups, "operators, calls:", tr.counts(), flush=True)
    w, hist = tr.train(init_weights(seed), steps=steps, batch_ops=6, lr=3e-3, seed=seed, group_weights=[1, 1, 1, 1, 1])
    tr.close()
    return w, hist
