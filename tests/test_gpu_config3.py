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


def test_batch_graph_equals_each_patch_alone():
    """The batch as one graph (btd_batch_create / btd_batch_run): every patch's substep a branch of a
    single graph launch, grip targets queued on each patch's stream before it; each patch ends bit for
    bit where it ends alone, also after the sweeps' launch shapes were autotuned."""
    c = btd.configs.CONFIG3
    patches = btd.configs.config3(count=12, sides=(16, 64))
    steps = 12
    batch = [make(p) for p in patches]
    s0, a0 = batch[0]
    s0.set_target((a0 + c["h"] * patches[0][1]["velocity"]).astype(np.float32))
    s0.substep()  # an assembled system to tune on (patch 0 is one substep ahead)
    batch[0][0].autotune(reps=3)
    first = batch[0][0].x.copy()
    graph = btd.Batch([s for s, _ in batch])
    for k in range(1, steps + 1):
        for i, ((s, anchor), (_, g)) in enumerate(zip(batch, patches)):
            kk = k + 1 if i == 0 else k
            s.set_target((anchor + kk * c["h"] * g["velocity"]).astype(np.float32))
        graph.run(1)
    for s, _ in batch:
        s.synchronize()
    for i, ((s, _), p) in enumerate(zip(batch, patches)):
        alone, anchor = make(p)
        total = steps + 1 if i == 0 else steps
        for k in range(1, total + 1):
            alone.set_target((anchor + k * c["h"] * p[1]["velocity"]).astype(np.float32))
            alone.substep()
            if i == 0 and k == 1:
                assert np.array_equal(alone.x, first)
        assert np.array_equal(alone.x, s.x), i
        alone.close()
    graph.close()
    for s, _ in batch:
        s.close()
