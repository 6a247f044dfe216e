"""B200-native implicit cloth solve behind the reference's GpuSolver interface.

The solve (projected Newton over the woven crossing lattice, Galerkin-multigrid-preconditioned PCG
with exact yarn-line smoothers, line search, damage field and crossing slip) runs as CUDA kernels
for sm_100a in libbtd.so; this package is the host-side mirror of the reference's
`GpuSolver` (src/simulation/gpu/solver.ts) over the library's C ABI (include/btd.h).
"""
from . import _abi, configs, drape, learned, topology
from .scene import (Scene, bundle_weave, compile_scene, default_spec, layer_spec, material_preset, SEG_BROKEN,
                    SEG_EXISTS, SEG_INITIAL_DEFECT, SEG_SLIPPED)
from ._abi import BtdError
from .solver import COARSE_ROW, FINE_ROW, Batch, GpuSolver, batch_substeps, default_params

__all__ = ["Scene", "bundle_weave", "compile_scene", "default_spec", "layer_spec", "material_preset", "SEG_BROKEN",
           "SEG_EXISTS", "SEG_INITIAL_DEFECT", "SEG_SLIPPED", "GpuSolver", "default_params", "FINE_ROW", "COARSE_ROW",
           "configs", "drape", "learned", "topology", "BtdError", "batch_substeps", "Batch"]
