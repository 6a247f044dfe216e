"""The V-cycle's bottom two levels in one thread-block cluster launch (btd_set_vcycle_tail, k_vtail)
against the launch-per-colour-pass path: the same device code in the same order, so the results must
agree bit for bit - one V-cycle, a PCG solve, whole substeps with the learned correction (which splits
the cluster launch around its own kernel) - and both against the oracle's V-cycle."""
import numpy as np
import pytest

import btd_b200 as btd
from helpers import MG, copy_state, max_abs_rel_to_scale
from oracle import Oracle

pytestmark = pytest.mark.gpu


def staged(n=64):
    """A hanging patch's Newton system (after two oracle substeps at 64 x 64; from rest at 256 x 256)."""
    sc = btd.configs.hanging_patch(n, 0.3, seed=2)
    cpu = Oracle(sc, h=1 / 60, newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, **MG)
    for _ in range(2 if n <= 64 else 0):
        cpu.substep()
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6))
    copy_state(cpu, gpu)
    cpu.predict()
    gpu.encode_predict()
    gpu.encode_assemble(True)
    return sc, cpu, gpu


@pytest.mark.parametrize("n", [64, 256])
def test_one_vcycle_is_the_same_bit_for_bit_and_matches_the_oracle(n):
    sc, cpu, gpu = staged(n)
    assert gpu.level_count() >= 3
    b = gpu.read_vector("B")
    out = {}
    for tail in (True, False):
        gpu.set_vcycle_tail(tail)
        gpu.write_vector("B", b)
        gpu.encode_vcycle()
        out[tail] = gpu.read_vector("X")
    gpu.set_vcycle_tail(True)
    assert np.array_equal(out[True], out[False])
    A_gpu, _ = gpu.read_operator(0)
    cpu.build_levels(A_gpu)
    zc = cpu.vcycle(b)
    assert max_abs_rel_to_scale(out[True], zc) < 5e-3


def test_pcg_is_the_same_bit_for_bit():
    sc, cpu, gpu = staged(64)
    b = gpu.read_vector("B")
    out = {}
    for tail in (True, False):
        gpu.set_vcycle_tail(tail)
        gpu.set_pcg(500, 1e-6)
        gpu.write_vector("B", b)
        gpu.encode_pcg()
        out[tail] = (gpu.delta_f64(), gpu.counter_dict()["pcg_last"])
    gpu.set_vcycle_tail(True)
    assert out[True][1] == out[False][1]
    assert np.array_equal(out[True][0], out[False][0])


def test_substeps_with_the_learned_correction_are_the_same_bit_for_bit():
    weights = btd.learned.load(btd.learned.DEFAULT_PATH)
    c = btd.configs.CONFIG4
    sc, left, right = btd.configs.config4(n=64, region=16)
    runs = {}
    for tail in (True, False):
        g = btd.GpuSolver(sc, btd.configs.solver_params(c["h"], c["newton_iterations"], c["pcg_rel_tol"], self_contact=1))
        g.set_vcycle_tail(tail)
        g.set_learned(weights, on=True, guard=c["guard"])
        x0 = g.x
        for slot, (nodes, sign) in enumerate(((left, -1.0), (right, 1.0))):
            picked = int(nodes[len(nodes) // 2])
            g.attach_patch(slot, picked, nodes, np.ones(len(nodes)), x0[picked].astype(np.float32), c["grip_stiffness"], max_lead=1.0)
        for s in range(1, 13):
            for slot, (nodes, sign) in enumerate(((left, -1.0), (right, 1.0))):
                picked = int(nodes[len(nodes) // 2])
                t = x0[picked].astype(np.float64) + np.array([sign * 0.5 * c["grip_speed"] * s * c["h"], 0, 0])
                g.set_target(t.astype(np.float32), slot=slot)
            g.substep()
        runs[tail] = (g.state()[0], g.counter_dict()["pcg_total"], g.learned_stats()["applied"])
        g.close()
    assert runs[True][2] > 0  # the correction ran
    assert runs[True][1] == runs[False][1]
    assert np.array_equal(runs[True][0], runs[False][0])
