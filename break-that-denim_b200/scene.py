"""Compiled scenes as numpy arrays (CompiledScene, src/simulation/scene.ts:91-125).

`compile_scene` runs the library's host-side `compileScene` (scene.ts:233-278) and copies the result
into numpy arrays owned by Python; `Scene.c()` exposes them to the C ABI (btd_create, the oracle)
without copying.
"""
import ctypes as C

import numpy as np

from . import _abi

SEG_EXISTS = 1
SEG_BROKEN = 2
SEG_INITIAL_DEFECT = 4
SEG_SLIPPED = 8

# (field name, dtype, count multiplier over N or C)
_NODE_ARRAYS = [
    ("rest_uv", np.float64, 2), ("position", np.float64, 3), ("mass", np.float64, 1), ("pinned", np.uint8, 1),
    ("wear", np.float32, 1), ("structural_wear", np.float32, 1), ("rest_length", np.float64, 2),
    ("softening", np.float64, 2), ("seg_flags", np.uint16, 2), ("intact", np.float64, 2),
    ("cut_mask", np.uint32, 2), ("fail_site", np.float32, 2), ("crossing_normal0", np.float64, 1),
    ("tails", np.float64, 4),
]
_CROSSING_ARRAYS = [("field_strength", np.float32, 2), ("field_damage", np.uint8, 2), ("field_area", np.uint8, 2)]

_CTYPE = {np.float64: C.c_double, np.float32: C.c_float, np.uint8: C.c_uint8, np.uint16: C.c_uint16,
          np.uint32: C.c_uint32}


class Scene:
    """A compiled scene: layer infos plus per-node, per-span and per-crossing arrays."""

    def __init__(self, layers, node_count, crossing_count, arrays):
        self.layers = layers  # list of _abi.LayerInfo (copies)
        self.N = node_count
        self.C = crossing_count
        for k, v in arrays.items():
            setattr(self, k, v)
        self._keep = None

    @classmethod
    def from_c(cls, p):
        s = p.contents
        layers = [_abi.LayerInfo.from_buffer_copy(s.layers[i]) for i in range(s.n_layers)]
        arrays = {}
        for name, dt, m in _NODE_ARRAYS:
            arrays[name] = np.ctypeslib.as_array(getattr(s, name), shape=(m * s.node_count,)).astype(dt, copy=True)
        for name, dt, m in _CROSSING_ARRAYS:
            arrays[name] = np.ctypeslib.as_array(getattr(s, name), shape=(m * s.crossing_count,)).astype(dt, copy=True)
        return cls(layers, s.node_count, s.crossing_count, arrays)

    def copy(self):
        arrays = {name: getattr(self, name).copy() for name, _, _ in _NODE_ARRAYS + _CROSSING_ARRAYS}
        return Scene([_abi.LayerInfo.from_buffer_copy(L) for L in self.layers], self.N, self.C, arrays)

    def c(self):
        """A btd_scene pointing at this scene's arrays (valid while the Scene lives)."""
        s = _abi.SceneC()
        s.n_layers = len(self.layers)
        s.node_count = self.N
        s.crossing_count = self.C
        larr = (_abi.LayerInfo * len(self.layers))(*self.layers)
        s.layers = C.cast(larr, C.POINTER(_abi.LayerInfo))
        keep = [larr]
        for name, dt, _ in _NODE_ARRAYS + _CROSSING_ARRAYS:
            a = getattr(self, name)
            assert a.dtype == dt and a.flags.c_contiguous, name
            setattr(s, name, a.ctypes.data_as(C.POINTER(_CTYPE[dt])))
            keep.append(a)
        self._keep = (s, keep)
        return s

    def hash(self):
        """sceneHash (scene.ts:134-150)."""
        out = C.c_uint32()
        _abi.check("btd_scene_hash", C.byref(self.c()), C.byref(out))
        return out.value

    @property
    def nx(self):
        return self.layers[0].nx

    @property
    def ny(self):
        return self.layers[0].ny


def material_preset(index=0):
    """DENIM (0) or BACKING (1), material.ts:88-187."""
    m = _abi.Material()
    _abi.check("btd_material_preset", index, C.byref(m))
    return m


def bundle_weave(m, bu, bv=None):
    out = _abi.Material()
    _abi.check("btd_bundle_weave", C.byref(m), bu, bu if bv is None else bv, C.byref(out))
    return out


def default_spec():
    """defaultSceneSpecs (scene.ts:438-469): the shipped 182 x 115 coupon."""
    s = _abi.LayerSpec()
    _abi.check("btd_default_scene_spec", C.byref(s))
    return s


def layer_spec(material, size_u, size_v, *, bundle=(1, 1), z=0.0, angle=0.0, compress_u=0.0, compress_v=0.0,
               shear=0.0, collar_rows=0, seed=1, wear=None, wear_strength_loss=(0.0, 0.0), perturbation=0.0):
    """A LayerSpec; `wear=None` is the unworn spec of the reference's coupon tests."""
    s = _abi.LayerSpec()
    s.material = material
    s.bundle[0], s.bundle[1] = bundle
    s.size_u, s.size_v, s.z, s.angle = size_u, size_v, z, angle
    s.compress_u, s.compress_v, s.shear = compress_u, compress_v, shear
    s.collar_rows, s.seed = collar_rows, seed
    w = s.wear
    if wear is None:
        wear = dict(center=(0, 0), axis=(1, 0), radii=(1, 1), amount=0, cell_size=0, feature_scale=0.01,
                    defect_threshold=2, defect_density=0, sparse_from=2)
    w.center[0], w.center[1] = wear["center"]
    w.axis[0], w.axis[1] = wear["axis"]
    w.radii[0], w.radii[1] = wear["radii"]
    for k in ("amount", "cell_size", "feature_scale", "defect_threshold", "defect_density", "sparse_from"):
        setattr(w, k, wear[k])
    s.wear_strength_loss[0], s.wear_strength_loss[1] = wear_strength_loss
    s.perturbation = perturbation
    return s


def compile_scene(specs):
    """compileScene (scene.ts:233-278) on the host."""
    if isinstance(specs, _abi.LayerSpec):
        specs = [specs]
    arr = (_abi.LayerSpec * len(specs))(*specs)
    p = C.POINTER(_abi.SceneC)()
    _abi.check("btd_scene_compile", arr, len(specs), C.byref(p))
    try:
        return Scene.from_c(p)
    finally:
        _abi.lib().btd_scene_free(p)
