"""TEST INFRASTRUCTURE ONLY: Python binding of the FP64 oracle (oracle.cpp).

The oracle restates the reference's own CPU solver (src/simulation/reference/solver.ts and
newtonMultigrid.ts with laws.ts, axial.ts, lattice.ts, yarnField.ts) in C++. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it, to compare against and to time;
the product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    """Compile liboracle.so with the committed Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


class OraParams(C.Structure):
    _fields_ = [
        ("h", C.c_double),
        ("gravity", C.c_double * 3),
        ("newton_iterations", C.c_int32),
        ("pcg_iterations", C.c_int32),
        ("pcg_rel_tol", C.c_double),
        ("max_coarsest_nodes", C.c_int32),
        ("coarse_sweeps", C.c_int32),
        ("line_colors", C.c_int32),
        ("lag_coarse", C.c_int32),
        ("line_search", C.c_int32),
        ("threads", C.c_int32),
        ("self_contact", C.c_int32),
        ("cross_layer", C.c_int32),
        ("coarse_bf16", C.c_int32),
        ("fp32_rows", C.c_int32),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        h = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sig = {
            "ora_create": ([vp, vp], vp),
            "ora_destroy": ([vp], None),
            "ora_last_error": ([], C.c_char_p),
            "ora_potential": ([vp], C.c_double),
            "ora_yarn_material_length": ([vp], C.c_double),
            "ora_solve_penta": ([C.c_int32, vp, vp, vp, vp, vp, C.c_double], C.c_int),
            "ora_law_axial": ([vp, C.c_double, vp], None),
            "ora_law_strain_at_tension": ([vp, C.c_double], C.c_double),
            "ora_law_yarn_damage": ([vp] + [C.c_double] * 5, C.c_double),
            "ora_law_bend_psi": ([C.c_double, C.c_double, vp], None),
            "ora_law_bend_psi_delta": ([C.c_double] * 4, C.c_double),
            "ora_law_bend_geometry": ([C.c_double, C.c_double, vp], None),
            "ora_law_bend_scale": ([C.c_double, C.c_double, C.c_uint32, C.c_uint32, C.c_int32], C.c_double),
            "ora_law_shear_jam": ([C.c_double], C.c_double),
            "ora_law_cell_area": ([C.c_double] * 4, C.c_double),
            "ora_law_shear": ([C.c_double] * 4 + [vp], None),
            "ora_law_constants": ([vp], None),
            "ora_field_layer": ([vp, C.c_int32, vp], C.c_int),
            "ora_field_span_crossing": ([vp] + [C.c_int32] * 6, C.c_int32),
            "ora_field_own_span": ([vp] + [C.c_int32] * 4 + [vp], C.c_int32),
            "ora_field_interpolated_strain": ([vp] + [C.c_int32] * 4 + [vp], C.c_double),
            "ora_field_couple": ([vp], C.c_int32),
            "ora_field_update": ([vp, vp], C.c_int),
            "ora_field_pull_out": ([vp, vp], C.c_int32),
            "ora_field_recoil_length": ([vp] + [C.c_double] * 9, C.c_double),
            "ora_field_share_reach": ([vp, C.c_int32, C.c_int32], C.c_int32),
            "ora_field_share_factor": ([vp, C.c_int32, vp] + [C.c_int32] * 4 + [C.c_double], C.c_double),
            "ora_field_share_cap": ([C.c_int32] + [C.c_double] * 5, C.c_double),
            "ora_field_constants": ([vp], None),
            "ora_learned_size": ([], C.c_int32),
            "ora_learned_dims": ([vp], C.c_int32),
            "ora_learned_set": ([vp, vp, C.c_int32, C.c_int32, C.c_double], C.c_int),
            "ora_learned_log": ([vp, C.c_int32, C.c_int64], C.c_int),
            "ora_learned_ops": ([vp], C.c_int32),
            "ora_learned_op_nodes": ([vp, C.c_int32], C.c_int32),
            "ora_learned_op": ([vp, C.c_int32, vp, vp], C.c_int),
            "ora_learned_calls": ([vp], C.c_int32),
            "ora_learned_call": ([vp, C.c_int32, vp, vp, vp], C.c_int),
            "ora_learned_stats": ([vp, vp], C.c_int),
            "ora_learned_forward": ([vp, vp, C.c_int64, vp], C.c_int),
            "ora_break_margins": ([vp, vp], C.c_int),
            "ora_learned_basis_of": ([vp, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp], C.c_int),
        }
        for name, (a, r) in sig.items():
            getattr(h, name).argtypes = a
            getattr(h, name).restype = r
        _lib = h
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _call(name, *args):
    f = getattr(lib(), name)
    rc = f(*args)
    if isinstance(rc, int) and rc < 0:
        raise RuntimeError(f"{name}: {lib().ora_last_error().decode()}")
    return rc


def solve_penta(D, E, F, r, shift=0.0):
    """solvePenta (newtonMultigrid.ts:435-473) on (n, 3, 3) blocks."""
    n = len(D)
    x = np.zeros(3 * n)
    _call("ora_solve_penta", n, _ptr(np.ascontiguousarray(D, np.float64)), _ptr(np.ascontiguousarray(E, np.float64)),
          _ptr(np.ascontiguousarray(F, np.float64)), _ptr(np.ascontiguousarray(r, np.float64)), _ptr(x), C.c_double(shift))
    return x.reshape(n, 3)


class Oracle:
    """ReferenceSolver (solver.ts(ref):41-749) with the multigrid of newtonMultigrid.ts.

    Defaults follow the reference's own defaults (MG_DEFAULTS, no lag, no line search); pass the GPU
    schedule explicitly to compare with the CUDA path.
    """

    def __init__(self, scene, h=1 / 240, gravity=(0, 0, -9.81), newton_iterations=2, pcg_iterations=4,
                 pcg_rel_tol=0.0, max_coarsest_nodes=48, coarse_sweeps=6, line_colors=3, lag_coarse=False,
                 line_search=False, threads=0, self_contact=False, cross_layer=False, coarse_bf16=False,
                 fp32_rows=0):
        p = OraParams()
        p.h = h
        p.gravity[0], p.gravity[1], p.gravity[2] = gravity
        p.newton_iterations = newton_iterations
        p.pcg_iterations = pcg_iterations
        p.pcg_rel_tol = pcg_rel_tol
        p.max_coarsest_nodes = max_coarsest_nodes
        p.coarse_sweeps = coarse_sweeps
        p.line_colors = line_colors
        p.lag_coarse = int(lag_coarse)
        p.line_search = int(line_search)
        p.threads = threads
        p.self_contact = int(self_contact)
        p.cross_layer = int(cross_layer)
        p.coarse_bf16 = int(coarse_bf16)  # 0 off, 1 all blocks, 2 couplings only
        p.fp32_rows = int(fp32_rows)  # fine level (units) and coarse levels (tens): 0 kept, 1 float32 blocks, 2 float32 row-sum form
        self.scene = scene
        self.N = scene.N
        self.params = p
        self._h = _call("ora_create", C.byref(scene.c()), C.byref(p))
        if not self._h:
            raise RuntimeError(lib().ora_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ora_destroy(self._h)
            self._h = None

    # ---- state
    def state(self):
        n3 = 3 * self.N
        x, v, dx, pred = (np.zeros(n3) for _ in range(4))
        _call("ora_get_state", C.c_void_p(self._h), _ptr(x), _ptr(v), _ptr(dx), _ptr(pred))
        return x.reshape(-1, 3), v.reshape(-1, 3), dx.reshape(-1, 3), pred.reshape(-1, 3)

    @property
    def x(self):
        return self.state()[0]

    @property
    def v(self):
        return self.state()[1]

    def set_state(self, x, v=None):
        x = np.ascontiguousarray(x, np.float64).reshape(-1)
        v = None if v is None else np.ascontiguousarray(v, np.float64).reshape(-1)
        _call("ora_set_state", C.c_void_p(self._h), _ptr(x), _ptr(v))

    def set_dx(self, dx=None, pred=None):
        dx = None if dx is None else np.ascontiguousarray(dx, np.float64).reshape(-1)
        pred = None if pred is None else np.ascontiguousarray(pred, np.float64).reshape(-1)
        _call("ora_set_dx", C.c_void_p(self._h), _ptr(dx), _ptr(pred))

    def segments(self):
        n2 = 2 * self.N
        rest, intact, fail = np.zeros(n2), np.zeros(n2), np.zeros(n2)
        cut = np.zeros(n2, np.uint32)
        flags = np.zeros(n2, np.uint16)
        tails = np.zeros(4 * self.N)
        _call("ora_get_segments", C.c_void_p(self._h), _ptr(rest), _ptr(intact), _ptr(cut), _ptr(flags), _ptr(fail), _ptr(tails))
        return dict(rest_length=rest, intact=intact, cut_mask=cut, seg_flags=flags, fail_site=fail, tails=tails)

    def set_segments(self, rest_length=None, intact=None, cut_mask=None, seg_flags=None, fail_site=None, tails=None):
        conv = lambda a, t: None if a is None else np.ascontiguousarray(a, t)
        a = [conv(rest_length, np.float64), conv(intact, np.float64), conv(cut_mask, np.uint32),
             conv(seg_flags, np.uint16), conv(fail_site, np.float64), conv(tails, np.float64)]
        _call("ora_set_segments", C.c_void_p(self._h), *[_ptr(q) for q in a])

    def field(self):
        d = np.zeros(2 * self.scene.C, np.uint8)
        _call("ora_get_field", C.c_void_p(self._h), _ptr(d))
        return d

    def set_field(self, damage):
        _call("ora_set_field", C.c_void_p(self._h), _ptr(np.ascontiguousarray(damage, np.uint8)))

    # ---- the yarn damage field's steps on this solver's field and spans (yarnField.ts)
    def break_margins(self):
        """Per (crossing, family) the last damage update's relative distance to the separation threshold of
        the yarn there (cut or pull-out; +inf where none was evaluated)."""
        d = np.zeros(2 * self.scene.C)
        _call("ora_break_margins", C.c_void_p(self._h), _ptr(d))
        return d

    def field_layer(self, layer=0):
        """dict(offset, K, M, bu, bv, nx, ny, node_offset) of a layer's field."""
        out = np.zeros(8, np.int32)
        _call("ora_field_layer", C.c_void_p(self._h), layer, _ptr(out))
        return dict(zip(("offset", "K", "M", "bu", "bv", "nx", "ny", "node_offset"), (int(v) for v in out)))

    def span_crossing(self, i, j, f, q, p, layer=0):
        """spanCrossing (yarnField.ts:201-204): the absolute crossing index."""
        return lib().ora_field_span_crossing(C.c_void_p(self._h), layer, i, j, f, q, p)

    def own_span(self, k, m, f, layer=0):
        """ownSpan (yarnField.ts:187-196): (i, j), or None."""
        ij = np.zeros(2, np.int32)
        ok = lib().ora_field_own_span(C.c_void_p(self._h), layer, k, m, f, _ptr(ij))
        return (int(ij[0]), int(ij[1])) if ok else None

    def interpolated_strain(self, f, k, m, strain, layer=0):
        return lib().ora_field_interpolated_strain(C.c_void_p(self._h), layer, f, k, m, _ptr(np.ascontiguousarray(strain, np.float64)))

    def couple_spans(self):
        """coupleSpans (yarnField.ts:443-499) on the current field and spans; returns the ruptures."""
        return lib().ora_field_couple(C.c_void_p(self._h))

    def update_field(self, strain):
        """updateField (yarnField.ts:323-415) with the given strain of every span (2 per node)."""
        _call("ora_field_update", C.c_void_p(self._h), _ptr(np.ascontiguousarray(strain, np.float64)))

    def pull_out(self, strain):
        """pullOut (yarnField.ts:125-152) with the given strains; returns the crossings pulled."""
        return lib().ora_field_pull_out(C.c_void_p(self._h), _ptr(np.ascontiguousarray(strain, np.float64)))

    def share_reach(self, f, layer=0):
        return lib().ora_field_share_reach(C.c_void_p(self._h), layer, f)

    def share_factor(self, sep, f, k, m, reach, cap=float("inf"), layer=0):
        return lib().ora_field_share_factor(C.c_void_p(self._h), layer, _ptr(np.ascontiguousarray(sep, np.uint8)), f, k, m, reach, cap)

    def set_history(self, on):
        _call("ora_set_history", C.c_void_p(self._h), int(on))

    def counts(self):
        b, p = C.c_int32(), C.c_int32()
        _call("ora_counts", C.c_void_p(self._h), C.byref(b), C.byref(p))
        return b.value, p.value

    # ---- grips and floor
    def clear_grips(self):
        _call("ora_clear_grips", C.c_void_p(self._h))

    def add_grip(self, nodes, w, offset, goal, k):
        nodes = np.ascontiguousarray(nodes, np.int32)
        return _call("ora_add_grip", C.c_void_p(self._h), _ptr(nodes), _ptr(np.ascontiguousarray(w, np.float64)),
                     _ptr(np.ascontiguousarray(offset, np.float64)), len(nodes), _ptr(np.ascontiguousarray(goal, np.float64)),
                     C.c_double(k))

    def set_grip_goal(self, grip, goal):
        _call("ora_set_grip_goal", C.c_void_p(self._h), grip, _ptr(np.ascontiguousarray(goal, np.float64)))

    def set_pieces(self, piece_of, start, nodes):
        """setPieces (solver.ts:664-677): the detached pieces whose rigid modes the solve carries; an
        empty set (start of one entry) removes them."""
        piece_of = np.ascontiguousarray(piece_of, np.uint32)
        start = np.ascontiguousarray(start, np.uint32)
        nodes = np.ascontiguousarray(nodes, np.uint32)
        count = max(0, len(start) - 1)
        _call("ora_set_pieces", C.c_void_p(self._h), _ptr(piece_of), _ptr(start), count,
              _ptr(nodes) if len(nodes) else None)

    def set_floor(self, z, bulge=0.3e-3, stiffness=1300.0, friction=0.35, friction_speed=0.002, enabled=True):
        _call("ora_set_floor", C.c_void_p(self._h), int(enabled), C.c_double(z), C.c_double(bulge), C.c_double(stiffness),
              C.c_double(friction), C.c_double(friction_speed))

    # ---- stepping
    def predict(self):
        _call("ora_predict", C.c_void_p(self._h))

    def newton_step(self):
        m, rel, alpha = C.c_double(), C.c_double(), C.c_double()
        it = C.c_int32()
        _call("ora_newton_step", C.c_void_p(self._h), C.byref(m), C.byref(it), C.byref(rel), C.byref(alpha))
        return dict(max_update=m.value, pcg_iterations=it.value, rel_residual=rel.value, alpha=alpha.value)

    def finalize(self):
        _call("ora_finalize", C.c_void_p(self._h))

    def update_damage(self):
        _call("ora_update_damage", C.c_void_p(self._h))

    def substep(self):
        _call("ora_substep", C.c_void_p(self._h))

    # ---- energies
    def node_gradient(self, n):
        g = np.zeros(3)
        _call("ora_node_gradient", C.c_void_p(self._h), n, _ptr(g))
        return g

    def potential(self):
        return lib().ora_potential(self._h)

    def energy_change(self, d):
        e, m = np.zeros(4), np.zeros(4)
        _call("ora_energy_change", C.c_void_p(self._h), _ptr(np.ascontiguousarray(d, np.float64).reshape(-1)), _ptr(e), _ptr(m))
        return e, m

    def yarn_material_length(self):
        return lib().ora_yarn_material_length(self._h)

    # ---- multigrid stages
    def assemble(self):
        """(A (N, 25, 3, 3), fixed (N,), b (N, 3)) at the current iterate."""
        A = np.zeros(self.N * 25 * 9)
        fixed = np.zeros(self.N, np.uint8)
        b = np.zeros(3 * self.N)
        _call("ora_assemble", C.c_void_p(self._h), _ptr(A), _ptr(fixed), _ptr(b))
        return A.reshape(self.N, 25, 3, 3), fixed, b.reshape(-1, 3)

    def build_levels(self, A=None):
        a = None if A is None else np.ascontiguousarray(A, np.float64).reshape(-1)
        _call("ora_build_levels", C.c_void_p(self._h), _ptr(a))

    def level_count(self):
        return _call("ora_level_count", C.c_void_p(self._h))

    def level(self, k):
        n = _call("ora_level_nodes", C.c_void_p(self._h), k)
        A = np.zeros(n * 25 * 9)
        fixed = np.zeros(n, np.uint8)
        _call("ora_read_level", C.c_void_p(self._h), k, _ptr(A), _ptr(fixed))
        return A.reshape(n, 25, 3, 3), fixed

    def prolongation(self, k):
        n = _call("ora_level_nodes", C.c_void_p(self._h), k)
        idx = np.zeros(4 * n, np.int32)
        w = np.zeros(4 * n)
        _call("ora_read_prolongation", C.c_void_p(self._h), k, _ptr(idx), _ptr(w))
        return idx.reshape(n, 4), w.reshape(n, 4)

    def apply(self, k, x):
        x = np.ascontiguousarray(x, np.float64).reshape(-1)
        y = np.zeros_like(x)
        _call("ora_apply", C.c_void_p(self._h), k, _ptr(x), _ptr(y))
        return y.reshape(-1, 3)

    def smooth(self, k, x, b, reverse=False):
        x = np.ascontiguousarray(x, np.float64).reshape(-1).copy()
        _call("ora_smooth", C.c_void_p(self._h), k, _ptr(x), _ptr(np.ascontiguousarray(b, np.float64).reshape(-1)), int(reverse))
        return x.reshape(-1, 3)

    def vcycle(self, b):
        b = np.ascontiguousarray(b, np.float64).reshape(-1)
        z = np.zeros_like(b)
        _call("ora_vcycle", C.c_void_p(self._h), _ptr(b), _ptr(z))
        return z.reshape(-1, 3)

    def pcg(self, b, iterations, rel_tol=0.0, x0=None):
        b = np.ascontiguousarray(b, np.float64).reshape(-1)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).reshape(-1).copy()
        done, rel = C.c_int32(), C.c_double()
        _call("ora_pcg", C.c_void_p(self._h), _ptr(b), _ptr(x), iterations, C.c_double(rel_tol), C.byref(done), C.byref(rel))
        return x.reshape(-1, 3), done.value, rel.value

    # ---- learned coarse correction (extension; no counterpart in the reference)
    def set_learned(self, weights=None, on=True, guard=0.9):
        """Add the learned coarse space of `weights` (flat, ora_learned_size() values) on the coarsest level
        of every V-cycle; on=False returns to the plain method."""
        w = None if weights is None else np.ascontiguousarray(weights, np.float64).reshape(-1)
        _call("ora_learned_set", C.c_void_p(self._h), _ptr(w), 0 if w is None else len(w), int(on), C.c_double(guard))

    def learned_log(self, on=True, capacity=1 << 20):
        """Start (clearing) or stop logging the coarsest level's training material, at most `capacity` calls."""
        _call("ora_learned_log", C.c_void_p(self._h), int(on), capacity)

    def learned_samples(self):
        """The logged material: ops, a list of (At, X) - the whitened coarsest operator over its free
        unknowns (3n, 3n) and its node inputs (n, 20) - and calls, a list of (op, r, d) - the whitened
        residual and exact correction (3n each) of one coarsest-level call."""
        h = C.c_void_p(self._h)
        ops = []
        for k in range(lib().ora_learned_ops(h)):
            n = _call("ora_learned_op_nodes", h, k)
            At, X = np.zeros((3 * n, 3 * n)), np.zeros((n, learned_dims()[0]))
            _call("ora_learned_op", h, k, _ptr(At), _ptr(X))
            ops.append((At, X))
        calls = []
        for q in range(lib().ora_learned_calls(h)):
            op = C.c_int32()
            _call("ora_learned_call", h, q, C.byref(op), None, None)
            n3 = 3 * len(ops[op.value][1])
            r, d = np.zeros(n3), np.zeros(n3)
            _call("ora_learned_call", h, q, C.byref(op), _ptr(r), _ptr(d))
            calls.append((op.value, r, d))
        return ops, calls

    def learned_basis_of(self, weights, A, fixed, nx, ny, flags):
        """The learned basis of a given coarsest operator (A (M, 25, 3, 3), fixed (M,), flags (M, 2) damage
        and contact): (X (M, 20), Phi (3 M, 8), G factor (8, 8), dead (8,)), or None if none was built."""
        M = nx * ny
        w = np.ascontiguousarray(weights, np.float64)
        A = np.ascontiguousarray(A, np.float64).reshape(-1)
        fx = np.ascontiguousarray(fixed, np.uint8)
        fl = np.ascontiguousarray(flags, np.float32).reshape(-1)
        X, phi, G, dead = np.zeros((M, 20)), np.zeros((3 * M, 8)), np.zeros((8, 8)), np.zeros(8, np.int32)
        rc = lib().ora_learned_basis_of(C.c_void_p(self._h), _ptr(w), _ptr(A), _ptr(fx), nx, ny, _ptr(fl), _ptr(X), _ptr(phi),
                                        _ptr(G), _ptr(dead))
        return None if rc != 0 else (X, phi, G, dead)

    def learned_stats(self):
        """dict(applied, fallbacks, solves) since creation."""
        out = np.zeros(3, np.int64)
        _call("ora_learned_stats", C.c_void_p(self._h), _ptr(out))
        return dict(zip(("applied", "fallbacks", "solves"), (int(v) for v in out)))


def learned_dims():
    """(inputs, hidden, basis vectors) of the coarsest-level network."""
    out = np.zeros(3, np.int32)
    lib().ora_learned_dims(_ptr(out))
    return tuple(int(v) for v in out)


def learned_forward(weights, X):
    """The network on node inputs X (rows, 20) as the oracle's V-cycle evaluates it: (rows, 24)."""
    X = np.ascontiguousarray(X, np.float64)
    out = np.zeros((len(X), 3 * learned_dims()[2]))
    _call("ora_learned_forward", _ptr(np.ascontiguousarray(weights, np.float64)), _ptr(X), len(X), _ptr(out))
    return out


class laws:
    """The oracle's constitutive laws on their own (axial.ts, laws.ts), for the reference's unit-test
    properties; a yarn is (eaLow, eaHigh, crimpStrain, eaCompress)."""

    @staticmethod
    def _y(y):
        return _ptr(np.ascontiguousarray(y, np.float64))

    @staticmethod
    def axial(y, eps):
        """(tension, stiffness, energy density) at strain eps (axial.ts:16-42)."""
        out = np.zeros(3)
        lib().ora_law_axial(laws._y(y), eps, _ptr(out))
        return tuple(out)

    @staticmethod
    def strain_at_tension(y, t):
        return lib().ora_law_strain_at_tension(laws._y(y), t)

    @staticmethod
    def yarn_damage(y, yarns, area, peak, soft, eps):
        return lib().ora_law_yarn_damage(laws._y(y), yarns, area, peak, soft, eps)

    @staticmethod
    def bend_psi(q, a):
        out = np.zeros(3)
        lib().ora_law_bend_psi(q, a, _ptr(out))
        return tuple(out)

    @staticmethod
    def bend_psi_delta(q0, q1, dq, a):
        return lib().ora_law_bend_psi_delta(q0, q1, dq, a)

    @staticmethod
    def bend_geometry(La, Lc):
        """(wa, wc, kPerB, fold) (laws.ts:54-58)."""
        out = np.zeros(4)
        lib().ora_law_bend_geometry(La, Lc, _ptr(out))
        return tuple(out)

    @staticmethod
    def bend_scale(ia, ic, mask_a, mask_c, B):
        return lib().ora_law_bend_scale(ia, ic, mask_a, mask_c, B)

    @staticmethod
    def shear_jam(area):
        return lib().ora_law_shear_jam(area)

    @staticmethod
    def cell_area(cu, tu, cv, rv):
        return lib().ora_law_cell_area(cu, tu, cv, rv)

    @staticmethod
    def shear(ks, Ld, l, jam=None):
        """(force, stiffness, energy) (laws.ts:140-159); jam defaults to SHEAR_JAM."""
        out = np.zeros(3)
        lib().ora_law_shear(ks, Ld, l, laws.constants()[1] if jam is None else jam, _ptr(out))
        return tuple(out)

    @staticmethod
    def constants():
        """(BEND_S0, SHEAR_JAM, SHEAR_RAMP)."""
        out = np.zeros(3)
        lib().ora_law_constants(_ptr(out))
        return tuple(out)


def recoil_length(yarn, B, area, peak, eps, mu, n0, wrap, t_cross, pitch):
    """recoilLength (yarnField.ts:109-115); yarn = (eaLow, eaHigh, crimpStrain, eaCompress)."""
    return lib().ora_field_recoil_length(_ptr(np.ascontiguousarray(yarn, np.float64)), B, area, peak, eps, mu, n0, wrap, t_cross, pitch)


def share_cap(reach, mu, n0, wrap, t_cross, peak):
    return lib().ora_field_share_cap(reach, mu, n0, wrap, t_cross, peak)


def field_constants():
    """(SHARE.fraction, DAMAGE_CUT, DAMAGE_PULLED)."""
    out = np.zeros(3)
    lib().ora_field_constants(_ptr(out))
    return float(out[0]), int(out[1]), int(out[2])

