"""GpuSolver: the host-side mirror of the reference's `GpuSolver` (src/simulation/gpu/solver.ts:194-838).

Method names follow the reference (setState -> set_state, encodeSubstep -> substep, ...); every
call goes through the C ABI of libbtd.so (include/btd.h). There is no CPU path: constructing a
solver without a CUDA device raises.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._abi import check

FINE_ROW = 72  # the reference's fine row floats (solver.ts:99), for readers of its layouts
COARSE_ROW = 200

COUNTER_NAMES = {0: "ruptures", 1: "pulled_out", 2: "max_speed", 3: "alpha", 12: "rejected", 16: "pcg_last",
                 17: "pcg_total", 18: "newton", 19: "rel_residual", 20: "errors", 21: "rel_residual_max",
                 22: "pcg_missed"}


def default_params(**kw):
    """GPU_DEFAULTS (solver.ts:61-72) with keyword overrides (field names of btd_params)."""
    p = _abi.Params()
    check("btd_default_params", C.byref(p))
    for k, v in kw.items():
        if k == "gravity":
            p.gravity[0], p.gravity[1], p.gravity[2] = v
        else:
            setattr(p, k, v)
    return p


def _f(a, n, dt=np.float32):
    a = np.ascontiguousarray(a, dt)
    assert a.size == n, (a.size, n)
    return a


class GpuSolver:
    """One patch (or several layers) on one GPU; owns its device memory and CUDA stream."""

    def __init__(self, scene, params=None, **kw):
        self.scene = scene
        self.params = params if params is not None else default_params(**kw)
        self.N = scene.N
        self.C = scene.C
        h = C.c_void_p()
        check("btd_create", C.byref(scene.c()), C.byref(self.params), C.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().btd_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # ---- per substep
    def substep(self, min_iterations=0, max_iterations=0):
        """encodeSubstep (solver.ts:737-760), launched on the solver's stream."""
        check("btd_substep", self._h, min_iterations, max_iterations)

    def substeps(self, count):
        check("btd_substeps", self._h, count)

    def synchronize(self):
        check("btd_synchronize", self._h)

    def settle_drape(self):
        """settleDrape (settle.ts:24-62): 420 damped substeps of 5 Newton / 2 PCG iterations, history
        off; the solver's settings are restored afterwards."""
        check("btd_settle_drape", self._h)

    # ---- state I/O
    def set_state(self, position, velocity=None):
        """setState (solver.ts:833-837): positions (N, 3) or (N, 4) (w >= 0.5 retires a node); velocities or zero."""
        pos = np.zeros((self.N, 4), np.float32)
        src = np.asarray(position, np.float64).reshape(self.N, -1)
        pos[:, :src.shape[1]] = src[:, :4]
        vel = None
        if velocity is not None:
            vel = np.zeros((self.N, 4), np.float32)
            vel[:, :3] = np.asarray(velocity, np.float64).reshape(self.N, -1)[:, :3]
        check("btd_set_state", self._h, pos.ctypes.data_as(C.c_void_p), None if vel is None else vel.ctypes.data_as(C.c_void_p))

    def state(self):
        pos = np.zeros((self.N, 4), np.float32)
        vel = np.zeros((self.N, 4), np.float32)
        check("btd_get_state", self._h, pos.ctypes.data_as(C.c_void_p), vel.ctypes.data_as(C.c_void_p))
        return pos, vel

    @property
    def x(self):
        return self.state()[0][:, :3]

    def set_segments(self, rest_length=None, intact=None, cut_mask=None, seg_flags=None, fail_site=None, tails=None):
        """setSegments (solver.ts:821-824)."""
        n2 = 2 * self.N
        arrs = [None if rest_length is None else _f(rest_length, n2), None if intact is None else _f(intact, n2),
                None if cut_mask is None else _f(cut_mask, n2, np.uint32),
                None if seg_flags is None else _f(seg_flags, n2, np.uint32),
                None if fail_site is None else _f(fail_site, n2), None if tails is None else _f(tails, 4 * self.N)]
        check("btd_set_segments", self._h, *[None if a is None else a.ctypes.data_as(C.c_void_p) for a in arrs])

    def segments(self):
        n2 = 2 * self.N
        rest, intact, fail = (np.zeros(n2, np.float32) for _ in range(3))
        cut, flags = np.zeros(n2, np.uint32), np.zeros(n2, np.uint32)
        tails = np.zeros(4 * self.N, np.float32)
        check("btd_get_segments", self._h, *[a.ctypes.data_as(C.c_void_p) for a in (rest, intact, cut, flags, fail, tails)])
        return dict(rest_length=rest, intact=intact, cut_mask=cut, seg_flags=flags, fail_site=fail, tails=tails)

    def set_field(self, damage):
        """setField (solver.ts:827-830): 2 damage codes per crossing."""
        d = _f(damage, 2 * self.C, np.uint8)
        check("btd_set_field", self._h, d.ctypes.data_as(C.c_void_p))

    def field(self):
        d = np.zeros(2 * self.C, np.uint8)
        check("btd_get_field", self._h, d.ctypes.data_as(C.c_void_p))
        return d

    def reset_state(self):
        check("btd_reset_state", self._h)

    # ---- knobs
    def set_floor(self, z):
        """setFloor (solver.ts:796-801); None removes the floor."""
        check("btd_set_floor", self._h, 0 if z is None else 1, 0.0 if z is None else float(z))

    def set_timestep(self, h):
        check("btd_set_timestep", self._h, float(h))

    def set_history_enabled(self, on):
        check("btd_set_history", self._h, int(bool(on)))

    def set_newton_tolerance(self, tol):
        check("btd_set_newton_tolerance", self._h, float(tol))

    def set_graph_mode(self, use_graphs):
        """True: one captured graph per substep; False: kernel by kernel (for per-kernel profilers)."""
        check("btd_set_graph_mode", self._h, int(bool(use_graphs)))

    def set_gradient_precision(self, fp64=True):
        """The Newton right-hand side in FP64 (default) or FP32 (the reference shader's precision)."""
        check("btd_set_gradient_precision", self._h, int(bool(fp64)))

    def set_operator_precision(self, fp64=True):
        """The operator PCG solves with: the fine rows assembled in FP64 as well (default; PCG's products and
        the V-cycle's fine residual take them), or the FP32 rows throughout (the reference shader's
        precision); the smoothers and coarse levels keep the FP32 rows either way."""
        check("btd_set_operator_precision", self._h, int(bool(fp64)))

    def set_pcg_flexible(self, on=True):
        """PCG's beta in the flexible (Polak-Ribiere) form, or the reference's form (default)."""
        check("btd_set_pcg_flexible", self._h, int(bool(on)))

    def set_pcg(self, max_iterations, rel_tol=0.0):
        check("btd_set_pcg", self._h, int(max_iterations), float(rel_tol))

    def counters(self):
        out = np.zeros(32, np.uint32)
        check("btd_read_counters", self._h, out.ctypes.data_as(C.c_void_p), 32)
        return out

    def counter_dict(self):
        c = self.counters()
        f = c.view(np.float32)
        d = {name: int(c[k]) for k, name in COUNTER_NAMES.items()}
        d["max_speed"] = float(f[2])
        d["alpha"] = float(f[3])
        d["rel_residual"] = float(f[19])
        d["rel_residual_max"] = float(f[21])
        d["max_update"] = [float(f[4 + k]) for k in range(8)]
        return d

    def clear_counters(self):
        check("btd_clear_counters", self._h)

    # ---- stage encoders (solver.ts:574-728)
    def encode_predict(self):
        check("btd_stage_predict", self._h)

    def encode_assemble(self, coarse=True):
        check("btd_stage_assemble", self._h, int(coarse))

    def encode_vcycle(self):
        check("btd_stage_vcycle", self._h)

    def encode_pcg(self):
        check("btd_stage_pcg", self._h)

    def encode_line_search(self):
        e, m = np.zeros(4), np.zeros(4)
        check("btd_stage_linesearch", self._h, e.ctypes.data_as(C.c_void_p), m.ctypes.data_as(C.c_void_p))
        return e, m

    def encode_apply(self, iteration=0):
        check("btd_stage_apply", self._h, iteration)

    def encode_newton_iteration(self, iteration=0):
        check("btd_stage_newton", self._h, iteration)

    def encode_smooth(self, level=0, reverse=False):
        """encodeSmooth (solver.ts:601-622): one line sweep of `level`, X <- S(X, B) in place."""
        check("btd_stage_smooth", self._h, level, int(reverse))

    def encode_finalize(self):
        check("btd_stage_finalize", self._h)

    def encode_damage(self):
        check("btd_stage_damage", self._h)

    # ---- grips (Interaction, src/simulation/gpu/interaction.ts:223-318)
    GRIPS = 4
    GRIP_ENTRIES = 512

    def attach_patch(self, slot, picked, nodes, weights, anchor, stiffness, max_lead, sides=None, pad_pitch=0.0, slip=0.0):
        """attachPatch (interaction.ts:223-261): grip `slot` holds `nodes` with `weights` (GripPatch
        fields); offsets and the handle's origin are taken from node `picked` on the device."""
        nodes = np.ascontiguousarray(nodes, np.int32)
        w = _f(weights, nodes.size)
        sd = None if sides is None else _f(sides, nodes.size)
        a = _f(anchor, 3)
        check("btd_set_grip", self._h, slot, nodes.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p),
              None if sd is None else sd.ctypes.data_as(C.c_void_p), nodes.size, int(picked),
              a.ctypes.data_as(C.c_void_p), stiffness, max_lead, pad_pitch, slip)

    def set_target(self, target, slot=0):
        """setTarget (interaction.ts:276-281): requested handle in the frame of the attach anchor."""
        t = _f(target, 3)
        check("btd_set_grip_target", self._h, slot, t.ctypes.data_as(C.c_void_p))

    def set_pinch(self, scale, slot=0):
        check("btd_set_grip_pinch", self._h, slot, scale)

    def set_hold(self, fraction, slot=0):
        check("btd_set_grip_hold", self._h, slot, fraction)

    def release(self, slot=0):
        check("btd_release_grip", self._h, slot)

    def read_grip(self, slot=0):
        """(nodes, current weights, handle (3,), origin (3,), closing axis (3,)) of grip `slot`."""
        count = C.c_int32()
        nodes = np.zeros(self.GRIP_ENTRIES, np.int32)
        w = np.zeros(self.GRIP_ENTRIES, np.float32)
        goal = np.zeros(12, np.float32)
        check("btd_read_grip", self._h, slot, nodes.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p),
              self.GRIP_ENTRIES, goal.ctypes.data_as(C.c_void_p), C.byref(count))
        n = count.value
        g = goal.reshape(3, 4)[:, :3].astype(np.float64)
        return nodes[:n].copy(), w[:n].copy(), g[0], g[1], g[2]

    STAGES = {"matvec": 0, "smooth": 1, "assemble": 2, "vcycle": 3, "hierarchy": 4, "substep": 5}

    def set_pieces(self, piece_of, start, nodes):
        """setPieces (solver.ts:664-676): detached pieces as the topology analysis labels them (piece of each
        node or 0xFFFFFFFF, start offsets, node lists); empty start clears."""
        start = np.ascontiguousarray(start, np.uint32)
        count = max(0, len(start) - 1)
        po = np.ascontiguousarray(piece_of, np.uint32)
        nd = np.ascontiguousarray(nodes, np.uint32)
        check("btd_set_pieces", self._h, po.ctypes.data_as(C.c_void_p), start.ctypes.data_as(C.c_void_p),
              nd.ctypes.data_as(C.c_void_p) if nd.size else None, count)

    # ---- learned coarse correction (extension; no counterpart in the reference)
    LEARNED_WEIGHTS = 7064  # W1[20][64] b1[64] W2[64][64] b2[64] W3[64][24] b3[24], row-major [in][out]

    def set_learned(self, weights=None, on=True, guard=0.9):
        """Add the learned coarse space of `weights` (flat FP32, LEARNED_WEIGHTS values; rounded to BF16 on
        the device) on the coarsest level of every V-cycle; a PCG solve whose mean contraction per
        iteration exceeds `guard` after three iterations falls back to the plain V-cycle."""
        w = None if weights is None else np.ascontiguousarray(weights, np.float32).reshape(-1)
        check("btd_set_learned", self._h, None if w is None else w.ctypes.data_as(C.c_void_p), 0 if w is None else w.size,
              int(bool(on)), C.c_double(guard))

    def learned_stats(self):
        """dict(solves, applied, fallbacks, logged_ops, logged_calls) since the correction was set."""
        out = np.zeros(5, np.int64)
        check("btd_learned_stats", self._h, out.ctypes.data_as(C.c_void_p))
        return dict(zip(("solves", "applied", "fallbacks", "logged_ops", "logged_calls"), (int(v) for v in out)))

    def learned_basis(self):
        """The last PCG solve's learned basis: (Phi (3 M, 8), G factor (8, 8), dead (8,) or -1 when no basis
        was built, coarsest flags (M,): bit 0 damage, bit 1 contact)."""
        M = C.c_int32()
        check("btd_learned_basis", self._h, None, None, None, None, C.byref(M))
        m = M.value
        phi, G = np.zeros((3 * m, 8), np.float32), np.zeros((8, 8))
        dead, flags = np.zeros(8, np.int32), np.zeros(m, np.uint8)
        check("btd_learned_basis", self._h, phi.ctypes.data_as(C.c_void_p), G.ctypes.data_as(C.c_void_p),
              dead.ctypes.data_as(C.c_void_p), flags.ctypes.data_as(C.c_void_p), C.byref(M))
        return phi, G, dead, flags

    def learned_log(self, on=True, capacity_ops=64, capacity_calls=8192):
        """Log training material on the device: each new coarsest operator (rows, fixed flags, network
        inputs) and the coarsest residual of every learned-correction call."""
        check("btd_learned_log", self._h, int(bool(on)), int(capacity_ops), int(capacity_calls))

    def autotune(self, reps=10):
        """Time every level's sweep launch shapes (CTA size, staging tile) on the current operator and keep
        the fastest; returns [(threads, tile, ms)] per level."""
        L = self.level_count()
        t, tile, ms = np.zeros(L, np.int32), np.zeros(L, np.int32), np.zeros(L, np.float32)
        check("btd_autotune", self._h, int(reps), t.ctypes.data_as(C.c_void_p), tile.ctypes.data_as(C.c_void_p),
              ms.ctypes.data_as(C.c_void_p))
        return [(int(a), int(b), float(c)) for a, b, c in zip(t, tile, ms)]

    def launch_count(self, substeps, newton_iterations, pcg_iterations):
        """Kernel launches of `substeps` substeps with the given Newton and PCG iteration totals."""
        out = C.c_int64()
        check("btd_launch_count", self._h, substeps, newton_iterations, pcg_iterations, C.byref(out))
        return out.value

    def profile_stage(self, stage, reps=10, flush=True):
        """Mean device ms of one launch of a stage (CUDA events on the solver's stream)."""
        ms = C.c_float()
        check("btd_profile_stage", self._h, self.STAGES[stage], reps, int(flush), C.byref(ms))
        return ms.value

    # ---- levels and buffers
    def level_count(self):
        n = C.c_int32()
        check("btd_level_count", self._h, C.byref(n))
        return n.value

    def level_nodes(self, k):
        n = C.c_int32()
        check("btd_level_nodes", self._h, k, C.byref(n))
        return n.value

    def read_operator(self, k):
        """Level k's operator in the CPU reference's 25-offset layout: (N, 25, 3, 3), fixed (N,)."""
        n = self.level_nodes(k)
        A = np.zeros(n * 225)
        fixed = np.zeros(n, np.uint8)
        check("btd_read_operator", self._h, k, A.ctypes.data_as(C.c_void_p), fixed.ctypes.data_as(C.c_void_p))
        return A.reshape(n, 25, 3, 3), fixed

    VEC = {"X": 0, "B": 1, "R": 2, "delta": 3, "dx": 4, "pred": 5}
    BUF = {"op": 16, "fixed": 17, "x": 18, "v": 19, "contact": 20}

    def device_buffer(self, which, level=0):
        """(device pointer, bytes) of a solver buffer, for zero-copy consumers."""
        ptr, n = C.c_void_p(), C.c_size_t()
        code = self.BUF[which] if which in self.BUF else self.VEC[which]
        check("btd_device_buffer", self._h, code, level, C.byref(ptr), C.byref(n))
        return ptr.value, n.value

    def matvec(self, x):
        """y = A x and x . y with the last assembled fine operator (x: (N, 3))."""
        xb = np.zeros((self.N, 4), np.float32)
        xb[:, :3] = np.asarray(x).reshape(self.N, 3)
        yb = np.zeros((self.N, 4), np.float32)
        xy = C.c_double()
        check("btd_stage_matvec", self._h, xb.ctypes.data_as(C.c_void_p), yb.ctypes.data_as(C.c_void_p), C.byref(xy))
        return yb[:, :3].astype(np.float64), xy.value

    def read_vector(self, which, level=0):
        n = self.level_nodes(level) if self.VEC[which] <= 2 else self.N
        out = np.zeros((n, 4), np.float32)
        check("btd_read_vector", self._h, self.VEC[which], level, out.ctypes.data_as(C.c_void_p))
        return out[:, :3].astype(np.float64)

    def delta_f64(self):
        """The last PCG iterate accumulated in FP64, (N, 3)."""
        out = np.zeros((self.N, 3))
        check("btd_read_delta_f64", self._h, out.ctypes.data_as(C.c_void_p))
        return out

    def write_vector(self, which, values, level=0):
        n = self.level_nodes(level) if self.VEC[which] <= 2 else self.N
        buf = np.zeros((n, 4), np.float32)
        buf[:, :3] = np.asarray(values).reshape(n, 3)
        check("btd_write_vector", self._h, self.VEC[which], level, buf.ctypes.data_as(C.c_void_p))


def batch_substeps(solvers, substeps):
    """btd_batch_substeps: `substeps` substeps of every solver, concurrently on their own streams."""
    arr = (C.c_void_p * len(solvers))(*[s._h for s in solvers])
    check("btd_batch_substeps", arr, len(solvers), substeps)


class Batch:
    """A batch of solvers stepped by one graph launch per substep (btd_batch_*)."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        h = C.c_void_p()
        check("btd_batch_create", arr, len(self.solvers), C.byref(h))
        self._h = h

    def run(self, substeps=1):
        check("btd_batch_run", self._h, int(substeps))

    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().btd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
