"""The smoother's bounded wait for its staging copies (the kernels never hang on a wait): a test hook
sets the wait's first bound to zero tries, so its error flag is raised on every sweep while the copies
still land under the second bound. btd_synchronize then reports BTD_E_TIMEOUT exactly once, the next
call returns 0, and the positions equal a run with the default bound bit for bit (the copies did land).
"""
import numpy as np
import pytest

import btd_b200 as btd
from btd_b200 import _abi

pytestmark = pytest.mark.gpu


def run(substeps):
    sc = btd.configs.hanging_patch(32, 0.15, seed=4)
    g = btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6))
    g.substeps(substeps)
    return g


def test_first_bound_runs_out_and_is_reported_once():
    ref = run(2)
    ref.synchronize()
    x_ref = ref.x.copy()
    ref.close()
    _abi.check("btd_set_wait_bound", 0)
    try:
        g = run(2)
        with pytest.raises(_abi.BtdError) as e:
            g.synchronize()
        assert e.value.rc == -5, e.value
        assert "bounded device-side wait" in str(e.value)
        g.synchronize()  # reported once: the flag was cleared
        assert np.array_equal(g.x, x_ref)
        g.close()
    finally:
        _abi.check("btd_set_wait_bound", -1)
    g = run(1)
    g.synchronize()  # the default bound again: nothing to report
    g.close()
