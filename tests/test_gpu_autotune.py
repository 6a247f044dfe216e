"""The sweep autotuner (btd_autotune): per multigrid level it times the yarn-line sweep's CTA sizes and
staging tiles on the current operator and keeps the fastest. The choice changes only the launch shape,
never the arithmetic, so a run tuned after its first substep ends bit for bit where an untuned run does.
"""
import numpy as np
import pytest

import btd_b200 as btd

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 200])
def test_autotuned_run_equals_the_untuned_one(n):
    sc = btd.configs.hanging_patch(n, 0.3 * (n - 1) / 63, seed=2)
    params = btd.configs.solver_params(1 / 60, 4, 1e-6)
    a = btd.GpuSolver(sc, params)
    a.substeps(3)
    a.synchronize()
    xa = a.x.copy()
    b = btd.GpuSolver(sc, params)
    b.substeps(1)
    choice = b.autotune(reps=5)
    assert len(choice) == b.level_count()
    for threads, tile, ms in choice:
        assert threads % 32 == 0 and 64 <= threads <= 256
        assert 0 < tile <= 256
        assert ms > 0
    if n > 128:
        assert any(t in (128, 200) for _, t, _ in choice)
    b.substeps(2)
    b.synchronize()
    assert np.array_equal(b.x, xa)
