"""The allocation-free matvec (btd_matvec_noalloc) against the solver's own matvec stage.

Callers that cannot allocate device memory where they call in (a host with its own fixed device
pool, a frame-budgeted thread, code running during a stream capture) use btd_matvec_noalloc on
buffers they own; its scratch is a static device array. This checks, through the C ABI, that two
calls in a row give the matvec stage's y = A x and x . y, and that oversized lattices are refused.
Collected last so that a stop at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import btd_b200 as btd
from btd_b200 import _abi

pytestmark = pytest.mark.gpu


def test_noalloc_matvec_matches_the_stage_on_two_calls():
    import torch

    sc = btd.configs.config0()
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6))
    gpu.encode_predict()
    gpu.encode_assemble(False)
    op, _ = gpu.device_buffer("op", 0)
    fixed, _ = gpu.device_buffer("fixed", 0)
    nx, ny, N = sc.nx, sc.ny, sc.N
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    lib = _abi.lib()
    rng = np.random.default_rng(7)
    for call in range(2):
        x = rng.standard_normal((N, 3)) * 1e-3
        y_ref, xy_ref = gpu.matvec(x)
        xd = torch.zeros((N, 4), dtype=torch.float32, device=dev)
        xd[:, :3] = torch.from_numpy(x.astype(np.float32)).to(dev)
        yd = torch.full((N, 4), float("nan"), dtype=torch.float32, device=dev)
        xyd = torch.zeros(1, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        rc = lib.btd_matvec_noalloc(nx, ny, C.c_void_p(op), C.c_void_p(fixed), C.c_void_p(xd.data_ptr()),
                                    C.c_void_p(yd.data_ptr()), C.c_void_p(xyd.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0, _abi.last_error()
        stream.synchronize()
        y = yd[:, :3].double().cpu().numpy()
        assert np.abs(y - y_ref).max() <= 1e-6 * np.abs(y_ref).max(), call
        assert abs(xyd.item() - xy_ref) <= 1e-6 * abs(xy_ref), (call, xyd.item(), xy_ref)
    gpu.close()


def test_noalloc_matvec_rejects_lattices_beyond_its_scratch():
    lib = _abi.lib()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.btd_matvec_noalloc(1024, 1024, one, one, one, one, one, None)
    assert rc == -1
    assert "allocation-free maximum" in _abi.last_error()
