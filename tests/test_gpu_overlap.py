"""Programmatic dependent launch in the PCG loop (params.overlap_launches): each kernel of the loop
may start while its predecessor drains, the smoother staging its line factors meanwhile, and reads
its predecessor's output only after the grid-dependency wait. The results must be those of the
serialised launches bit for bit: one V-cycle, and whole substeps with the same PCG iteration counts.
"""
import numpy as np
import pytest

import btd_b200 as btd

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 256])
def test_overlapped_launches_equal_serialised(n):
    sc = btd.configs.hanging_patch(n, 0.6 * (n - 1) / 255, seed=5)
    on, off = (btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6, overlap_launches=v)) for v in (1, 0))
    for s in (on, off):
        s.clear_counters()
        s.substeps(3)
    assert np.array_equal(on.x, off.x)
    assert on.counters()[17] == off.counters()[17]  # PCG iterations
    rhs = np.random.default_rng(n).standard_normal((sc.N, 3))
    for s in (on, off):
        s.encode_assemble(True)
        s.write_vector("B", rhs)
        s.encode_vcycle()
    z = on.read_vector("X")
    assert np.isfinite(z).all() and np.abs(z).max() > 0
    assert np.array_equal(z, off.read_vector("X"))
    assert on.counters()[20] == 0  # no staging wait ran out
    on.close()
    off.close()
