"""ctypes mirror of include/btd.h (the C ABI of the CUDA solve) and the library loader.

The structures here must stay field-for-field identical to btd.h; tests/test_abi.py checks their
sizes against the C compiler's.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbtd.so")


class Yarn(C.Structure):
    """btd_yarn: YarnFamily (src/simulation/material.ts:18-54)."""

    _fields_ = [
        (n, C.c_double)
        for n in (
            "linear_density", "ea_low", "ea_high", "crimp_strain", "ea_compress", "axial_viscosity",
            "bend_rigidity", "bend_viscosity", "strength", "softening_opening", "width", "height",
            "crimp_amplitude",
        )
    ] + [("yarns_per_span", C.c_int32), ("pad_", C.c_int32)]


class Material(C.Structure):
    """btd_material: WeaveMaterial (src/simulation/material.ts:56-85)."""

    _fields_ = [
        ("id", C.c_int32),
        ("name", C.c_char * 60),
        ("pitch_u", C.c_double),
        ("pitch_v", C.c_double),
        ("yarns", Yarn * 2),
        ("twill_repeat", C.c_int32),
        ("twill_warp_over", C.c_int32),
    ] + [
        (n, C.c_double)
        for n in (
            "shear_stiffness", "crossing_friction", "crossing_normal0", "crossing_wrap", "thickness",
            "cloth_friction", "air_drag",
        )
    ]


class Wear(C.Structure):
    """btd_wear: WearSpec (src/simulation/scene.ts:27-46)."""

    _fields_ = [("center", C.c_double * 2), ("axis", C.c_double * 2), ("radii", C.c_double * 2)] + [
        (n, C.c_double)
        for n in ("amount", "cell_size", "feature_scale", "defect_threshold", "defect_density", "sparse_from")
    ]


class LayerSpec(C.Structure):
    """btd_layer_spec: LayerSpec (src/simulation/scene.ts:48-71)."""

    _fields_ = [
        ("material", Material),
        ("bundle", C.c_int32 * 2),
        ("size_u", C.c_double),
        ("size_v", C.c_double),
        ("z", C.c_double),
        ("angle", C.c_double),
        ("compress_u", C.c_double),
        ("compress_v", C.c_double),
        ("shear", C.c_double),
        ("collar_rows", C.c_int32),
        ("seed", C.c_int32),
        ("wear", Wear),
        ("wear_strength_loss", C.c_double * 2),
        ("perturbation", C.c_double),
    ]


class LayerInfo(C.Structure):
    """btd_layer_info: LayerInfo (src/simulation/scene.ts:73-89) with its field layout."""

    _fields_ = [
        ("index", C.c_int32),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("node_offset", C.c_int32),
        ("node_count", C.c_int32),
        ("bundle", C.c_int32 * 2),
        ("field_offset", C.c_int32),
        ("field_k", C.c_int32),
        ("field_m", C.c_int32),
        ("material", Material),
        ("weave", Material),
        ("map_a", C.c_double * 4),
        ("map_origin", C.c_double * 3),
        ("rest_center", C.c_double * 2),
    ]


def _p(t):
    return C.POINTER(t)


class SceneC(C.Structure):
    """btd_scene: CompiledScene (src/simulation/scene.ts:91-125)."""

    _fields_ = [
        ("n_layers", C.c_int32),
        ("node_count", C.c_int32),
        ("crossing_count", C.c_int32),
        ("pad_", C.c_int32),
        ("layers", _p(LayerInfo)),
        ("rest_uv", _p(C.c_double)),
        ("position", _p(C.c_double)),
        ("mass", _p(C.c_double)),
        ("pinned", _p(C.c_uint8)),
        ("wear", _p(C.c_float)),
        ("structural_wear", _p(C.c_float)),
        ("rest_length", _p(C.c_double)),
        ("softening", _p(C.c_double)),
        ("seg_flags", _p(C.c_uint16)),
        ("intact", _p(C.c_double)),
        ("cut_mask", _p(C.c_uint32)),
        ("fail_site", _p(C.c_float)),
        ("field_strength", _p(C.c_float)),
        ("field_damage", _p(C.c_uint8)),
        ("field_area", _p(C.c_uint8)),
        ("crossing_normal0", _p(C.c_double)),
        ("tails", _p(C.c_double)),
    ]


class Params(C.Structure):
    """btd_params: GpuSolverParams (src/simulation/gpu/solver.ts:26-53) + MG schedule."""

    _fields_ = [
        ("h", C.c_double),
        ("gravity", C.c_double * 3),
        ("newton_iterations", C.c_int32),
        ("newton_max", C.c_int32),
        ("newton_tolerance", C.c_double),
        ("history_tolerance", C.c_double),
        ("pcg_iterations", C.c_int32),
        ("coarse_sweeps", C.c_int32),
        ("max_coarsest_nodes", C.c_int32),
        ("self_contact", C.c_int32),
        ("pcg_rel_tol", C.c_double),
        ("line_search", C.c_int32),
        ("lag_coarse", C.c_int32),
        ("overlap_launches", C.c_int32),
        ("cross_layer", C.c_int32),
    ]


# Every exported symbol of include/btd.h with its argument types (checked by tests/test_abi.py).
SIGNATURES = {
    "btd_scene_compile": ([_p(LayerSpec), C.c_int32, _p(_p(SceneC))], C.c_int),
    "btd_scene_free": ([_p(SceneC)], C.c_int),
    "btd_scene_hash": ([_p(SceneC), _p(C.c_uint32)], C.c_int),
    "btd_material_preset": ([C.c_int32, _p(Material)], C.c_int),
    "btd_bundle_weave": ([_p(Material), C.c_int32, C.c_int32, _p(Material)], C.c_int),
    "btd_default_scene_spec": ([_p(LayerSpec)], C.c_int),
    "btd_default_params": ([_p(Params)], C.c_int),
    "btd_create": ([_p(SceneC), _p(Params), _p(C.c_void_p)], C.c_int),
    "btd_destroy": ([C.c_void_p], C.c_int),
    "btd_substep": ([C.c_void_p, C.c_int32, C.c_int32], C.c_int),
    "btd_substeps": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_batch_substeps": ([C.c_void_p, C.c_int32, C.c_int32], C.c_int),
    "btd_synchronize": ([C.c_void_p], C.c_int),
    "btd_set_state": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "btd_get_state": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "btd_set_segments": ([C.c_void_p] + [C.c_void_p] * 6, C.c_int),
    "btd_get_segments": ([C.c_void_p] + [C.c_void_p] * 6, C.c_int),
    "btd_set_field": ([C.c_void_p, C.c_void_p], C.c_int),
    "btd_get_field": ([C.c_void_p, C.c_void_p], C.c_int),
    "btd_reset_state": ([C.c_void_p], C.c_int),
    "btd_set_floor": ([C.c_void_p, C.c_int32, C.c_float], C.c_int),
    "btd_set_timestep": ([C.c_void_p, C.c_float], C.c_int),
    "btd_set_history": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_set_newton_tolerance": ([C.c_void_p, C.c_float], C.c_int),
    "btd_set_pcg": ([C.c_void_p, C.c_int32, C.c_double], C.c_int),
    "btd_set_graph_mode": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_read_counters": ([C.c_void_p, C.c_void_p, C.c_int32], C.c_int),
    "btd_clear_counters": ([C.c_void_p], C.c_int),
    "btd_settle_drape": ([C.c_void_p], C.c_int),
    "btd_stage_predict": ([C.c_void_p], C.c_int),
    "btd_stage_assemble": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_stage_vcycle": ([C.c_void_p], C.c_int),
    "btd_stage_pcg": ([C.c_void_p], C.c_int),
    "btd_stage_smooth": ([C.c_void_p, C.c_int32, C.c_int32], C.c_int),
    "btd_stage_linesearch": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "btd_stage_apply": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_stage_newton": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_stage_finalize": ([C.c_void_p], C.c_int),
    "btd_stage_damage": ([C.c_void_p], C.c_int),
    "btd_level_count": ([C.c_void_p, _p(C.c_int32)], C.c_int),
    "btd_level_nodes": ([C.c_void_p, C.c_int32, _p(C.c_int32)], C.c_int),
    "btd_read_operator": ([C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p], C.c_int),
    "btd_read_vector": ([C.c_void_p, C.c_int32, C.c_int32, C.c_void_p], C.c_int),
    "btd_read_delta_f64": ([C.c_void_p, C.c_void_p], C.c_int),
    "btd_write_vector": ([C.c_void_p, C.c_int32, C.c_int32, C.c_void_p], C.c_int),
    "btd_profile_stage": ([C.c_void_p, C.c_int32, C.c_int32, C.c_int32, _p(C.c_float)], C.c_int),
    "btd_launch_count": ([C.c_void_p, C.c_int32, C.c_int32, C.c_int32, _p(C.c_int64)], C.c_int),
    "btd_device_buffer": ([C.c_void_p, C.c_int32, C.c_int32, _p(C.c_void_p), _p(C.c_size_t)], C.c_int),
    "btd_stage_matvec": ([C.c_void_p, C.c_void_p, C.c_void_p, _p(C.c_double)], C.c_int),
    "btd_matvec_noalloc": ([C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.c_void_p], C.c_int),
    "btd_set_grip": ([C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                      C.c_float, C.c_float, C.c_float, C.c_float], C.c_int),
    "btd_set_grip_target": ([C.c_void_p, C.c_int32, C.c_void_p], C.c_int),
    "btd_set_grip_pinch": ([C.c_void_p, C.c_int32, C.c_float], C.c_int),
    "btd_set_grip_hold": ([C.c_void_p, C.c_int32, C.c_float], C.c_int),
    "btd_release_grip": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_read_grip": ([C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, _p(C.c_int32)], C.c_int),
    "btd_set_wait_bound": ([C.c_int32], C.c_int),
    "btd_batch_create": ([C.c_void_p, C.c_int32, C.c_void_p], C.c_int),
    "btd_batch_run": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_batch_destroy": ([C.c_void_p], C.c_int),
    "btd_autotune": ([C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "btd_set_pieces": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32], C.c_int),
    "btd_debug_projection": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_int32], C.c_int),
    "btd_set_gradient_precision": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_set_operator_precision": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_set_pcg_flexible": ([C.c_void_p, C.c_int32], C.c_int),
    "btd_set_learned": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_double], C.c_int),
    "btd_learned_stats": ([C.c_void_p, C.c_void_p], C.c_int),
    "btd_learned_basis": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "btd_learned_log": ([C.c_void_p, C.c_int32, C.c_int32, C.c_int32], C.c_int),
    "btd_trainer_create": ([C.c_void_p], C.c_int),
    "btd_trainer_destroy": ([C.c_void_p], C.c_int),
    "btd_trainer_add_op": ([C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32], C.c_int),
    "btd_trainer_add_log": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p], C.c_int),
    "btd_trainer_counts": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "btd_trainer_read_op": ([C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p], C.c_int),
    "btd_trainer_loss_grad": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p], C.c_int),
    "btd_trainer_train": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_uint64, C.c_void_p, C.c_int32,
                           C.c_void_p], C.c_int),
    "btd_last_error": ([C.c_char_p, C.c_size_t], C.c_int),
}

_lib = None


class BtdError(RuntimeError):
    """A negative return code from the C ABI, with its btd_last_error message."""

    def __init__(self, fn, rc, msg):
        super().__init__(f"{fn} failed ({rc}): {msg}")
        self.rc = rc


def lib():
    """Load libbtd.so (built by csrc/Makefile). Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it first (python __graft_entry__.py build)")
        h = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(h, name, None)
            if f is None:  # a missing export is reported by tests/test_abi.py
                continue
            f.argtypes = args
            f.restype = res
        _lib = h
    return _lib


def last_error():
    buf = C.create_string_buffer(1024)
    lib().btd_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(fn, *args):
    rc = getattr(lib(), fn)(*args)
    if rc < 0:
        raise BtdError(fn, rc, last_error())
    return rc
