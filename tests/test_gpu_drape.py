"""Drape settling (settleDrape, src/simulation/gpu/settle.ts:24-62) on the CUDA path, end to end on
the reference's product scene (182 x 115 nodes, sceneHash 0xfa77387b): btd_settle_drape from the
compiled scene with GPU_DEFAULTS lands where the oracle's settle by the same schedule lands (every
ninth free node; golden/make_settled.py), the mounted collar does not move, velocities and counters
end cleared, and the settled state round-trips through the drape file.

Against the reference's own file public/drape.bin the settled state differs by up to 3.2 mm (rms
0.57 mm) in a band of the slack-driven wrinkle where the sheet moves most (4-5 mm), and the oracle
differs from that file by the same amounts while the GPU and the oracle agree to 8 um: the file was
settled by the reference's WebGPU solver, whose arithmetic its CPU solver (what the oracle restates)
does not reproduce on this buckling mode. That comparison is kept, at the size of that difference.
"""
import os

import numpy as np
import pytest

import btd_b200 as btd

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def settled():
    sc = btd.compile_scene(btd.default_spec())
    gpu = btd.GpuSolver(sc, btd.default_params())
    x0 = gpu.state()[0].copy()
    gpu.settle_drape()
    return sc, gpu, x0


def test_settled_drape_matches_the_reference_drape(settled):
    sc, gpu, x0 = settled
    x, v = gpu.state()
    assert np.isfinite(x).all()
    o = np.load(os.path.join(GOLDEN, "drape_settled_oracle.npz"))
    d = np.linalg.norm(x[o["index"], :3].astype(np.float64) - o["position"], axis=1)
    motion = np.linalg.norm(o["position"] - x0[o["index"], :3], axis=1).max()  # up to 4.7 mm
    assert d.max() < 3e-5, f"vs oracle: max {d.max():.3e} m, motion {motion:.3e} m"
    g = np.load(os.path.join(GOLDEN, "drape_settled.npz"))
    d = np.linalg.norm(x[g["index"], :3].astype(np.float64) - g["position"], axis=1)
    msg = f"vs public/drape.bin: max {d.max():.3e} m, rms {np.sqrt((d ** 2).mean()):.3e} m"
    assert d.max() < 4e-3 and np.sqrt((d ** 2).mean()) < 8e-4, msg
    c = np.load(os.path.join(GOLDEN, "drape_collar.npz"))
    assert np.array_equal(x[c["index"], :3], c["position"])  # mounted: not moved
    assert not v[:, :3].any()
    assert not gpu.counters().any()


def test_settled_drape_round_trips_through_the_drape_file(settled):
    sc, gpu, _ = settled
    data = btd.drape.encode_drape(gpu)
    assert len(data) == 16 + 16 * sc.N
    other = btd.GpuSolver(sc, btd.default_params())
    assert btd.drape.load_drape(other, data)
    assert np.array_equal(other.state()[0], gpu.state()[0])
    patch = btd.configs.hanging_patch(16, 0.1)
    assert not btd.drape.load_drape(btd.GpuSolver(patch, btd.default_params()), data)
