"""The allocation-free matvec (btd_matvec_noalloc) against the FP64 oracle's operator product.

Some callers of this library cannot call cudaMalloc at the point where they call in: a host that
hands out device memory only from its own fixed pool, a frame-budgeted thread where cudaMalloc's
implicit device synchronisation is not allowed, or code running while a stream is being captured.
They use btd_matvec_noalloc on buffers they own; its reduction scratch is a static device array.
This checks, through the C ABI, that two calls in a row give y = A x and x . y as the FP64 product
of the same operator read back from the device (rows of fixed nodes zero), on the square plain
configuration and on a non-square lattice (where swapping the lattice's sides would show), and that
lattices beyond the scratch array are refused. Collected last, so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import btd_b200 as btd
from btd_b200 import _abi
from helpers import operator_apply

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,ny", [(64, 64), (48, 80)])
def test_noalloc_matvec_matches_the_fp64_product_on_two_calls(nx, ny):
    import torch

    sc = btd.configs.config0() if (nx, ny) == (64, 64) else btd.configs.hanging_patch((nx, ny), 0.3, seed=5)
    assert (sc.nx, sc.ny) == (nx, ny)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6))
    gpu.encode_predict()
    gpu.encode_assemble(False)
    A, fixed = gpu.read_operator(0)
    op, _ = gpu.device_buffer("op", 0)
    fx, _ = gpu.device_buffer("fixed", 0)
    N = sc.N
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    lib = _abi.lib()
    rng = np.random.default_rng(7)
    for call in range(2):
        x = (rng.standard_normal((N, 3)) * 1e-3).astype(np.float32).astype(np.float64)
        y_ref = operator_apply(A, nx, ny, x, fixed)
        xy_ref = float(np.sum(x * y_ref))
        xd = torch.zeros((N, 4), dtype=torch.float32, device=dev)
        xd[:, :3] = torch.from_numpy(x.astype(np.float32)).to(dev)
        yd = torch.full((N, 4), float("nan"), dtype=torch.float32, device=dev)
        xyd = torch.zeros(1, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        rc = lib.btd_matvec_noalloc(nx, ny, C.c_void_p(op), C.c_void_p(fx), C.c_void_p(xd.data_ptr()),
                                    C.c_void_p(yd.data_ptr()), C.c_void_p(xyd.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0, _abi.last_error()
        stream.synchronize()
        y = yd[:, :3].double().cpu().numpy()
        # fp32 products and sums of at most 13 blocks against the FP64 product
        assert np.abs(y - y_ref).max() <= 1e-5 * np.abs(y_ref).max(), call
        assert abs(xyd.item() - xy_ref) <= 1e-5 * abs(xy_ref), (call, xyd.item(), xy_ref)
    gpu.close()


def test_noalloc_matvec_rejects_lattices_beyond_its_scratch():
    lib = _abi.lib()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.btd_matvec_noalloc(1024, 1024, one, one, one, one, one, None)
    assert rc == -1
    assert "allocation-free maximum" in _abi.last_error()
