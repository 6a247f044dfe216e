"""The batched configuration (configuration 3): independent hanging patches of seeded sizes,
stiffnesses, yarn regions and grips, run as one batch (btd_batch_substeps: every patch on its own
stream, queued round robin). The reference has no batch; parity is the plain path: each patch of
the batch ends bit for bit where it ends when run alone.
"""
import numpy as np
import pytest

import btd_b200 as btd

pytestmark = pytest.mark.gpu


def make(patch):
    sc, g = patch
    c = btd.configs.CONFIG3
    s = btd.GpuSolver(sc, btd.configs.solver_params(c["h"], c["newton_iterations"], c["pcg_rel_tol"]))
    x = s.x
    anchor = x[g["picked"]].astype(np.float32)
    s.attach_patch(0, g["picked"], g["nodes"], g["weights"], anchor, g["stiffness"], max_lead=g["max_lead"])
    return s, anchor


def test_batch_equals_each_patch_alone():
    c = btd.configs.CONFIG3
    patches = btd.configs.config3(count=12, sides=(16, 48))
    steps = 15
    batch = [make(p) for p in patches]
    for k in range(1, steps + 1):
        for (s, anchor), (_, g) in zip(batch, patches):
            s.set_target((anchor + k * c["h"] * g["velocity"]).astype(np.float32))
        btd.batch_substeps([s for s, _ in batch], 1)
    for s, _ in batch:
        s.synchronize()
    for (s, _), p in zip(batch, patches):
        alone, anchor = make(p)
        for k in range(1, steps + 1):
            alone.set_target((anchor + k * c["h"] * p[1]["velocity"]).astype(np.float32))
            alone.substep()
        assert np.array_equal(alone.x, s.x)
        assert np.array_equal(alone.field(), s.field())
        alone.close()
    for s, _ in batch:
        assert np.isfinite(s.x).all()
        s.close()
