"""Crossing slip (slipNode / updateSlip, reference/solver.ts:668-740; step.wgsl:149-233) on the CUDA
path against the oracle, state by state: configuration 1's yarn lattice pulled apart by its two edge
grips (crossing friction 0.3), where hundreds of crossings slip from the first substep on and the first
yarns pull out of their spans after about 20. From the same state (the GPU synchronised to the
oracle's positions, velocities, segments, tails and damage field before every substep), one substep
on each side, then the changes the substep made to the span rest lengths (the friction-limited
transfer), to the tails (pull-out) and to the span flags (slipped, broken) are compared.
"""
import numpy as np
import pytest

import btd_b200 as btd
from helpers import MG, copy_state
from oracle import Oracle

pytestmark = pytest.mark.gpu


def test_slip_transfers_match_the_oracle_state_by_state():
    c = btd.configs.CONFIG1
    sc, left, right = btd.configs.config1()
    cpu = Oracle(sc, h=c["h"], newton_iterations=c["newton_iterations"], pcg_iterations=500, pcg_rel_tol=c["pcg_rel_tol"], **MG)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(c["h"], c["newton_iterations"], c["pcg_rel_tol"]))
    x0 = cpu.x.astype(np.float32).astype(np.float64)
    grips = []
    for slot, (nodes, sign) in enumerate(((left, -1.0), (right, 1.0))):
        picked = int(nodes[len(nodes) // 2])
        a = x0[picked].copy()
        gpu.attach_patch(slot, picked, nodes, np.ones(len(nodes)), a.astype(np.float32), c["grip_stiffness"], max_lead=1.0)
        cpu.add_grip(nodes, np.ones(len(nodes)), (x0[nodes] - x0[picked]).reshape(-1), a, c["grip_stiffness"])
        grips.append((slot, a, sign))
    slipped_total = tails_total = 0
    for s in range(1, 23):
        for slot, a, sign in grips:
            t = (a + np.array([sign * 0.5 * c["grip_speed"] * s * c["h"], 0, 0])).astype(np.float32)
            gpu.set_target(t, slot=slot)
            cpu.set_grip_goal(slot, t.astype(np.float64))
        copy_state(cpu, gpu)
        before = gpu.segments()
        cpu.substep()
        gpu.substep()
        sc_, sg = cpu.segments(), gpu.segments()
        # the state both started from, as float32 (the GPU's)
        r0, t0 = before["rest_length"].astype(np.float64), before["tails"].astype(np.float64)
        dr_c, dr_g = sc_["rest_length"] - r0, sg["rest_length"].astype(np.float64) - r0
        dt_c, dt_g = sc_["tails"] - t0, sg["tails"].astype(np.float64) - t0
        scale = max(np.abs(dr_c).max(), 1e-9)
        # transfers: the same spans move, by the same amounts (fp32 positions and tensions on the GPU)
        moving_c, moving_g = np.abs(dr_c) > 1e-3 * scale, np.abs(dr_g) > 1e-3 * scale
        mismatch = moving_c ^ moving_g
        assert mismatch.sum() <= max(2, 0.02 * moving_c.sum()), (s, int(mismatch.sum()), int(moving_c.sum()))
        assert np.abs(dr_g - dr_c).sum() <= 0.03 * np.abs(dr_c).sum() + 1e-9, (s, np.abs(dr_g - dr_c).sum(), np.abs(dr_c).sum())
        # the yarn length ledger: slip moves rest length between spans and tails, it creates none
        # (rupture splits a span's rest length into the tails on both sides)
        assert abs(np.abs(dt_g).sum() - np.abs(dt_c).sum()) <= 0.05 * np.abs(dt_c).sum() + 1e-7, (s, np.abs(dt_g).sum(), np.abs(dt_c).sum())
        # flags: slipped and broken spans
        fc, fg = sc_["seg_flags"].astype(np.int64), sg["seg_flags"].astype(np.int64)
        assert ((fc ^ fg) != 0).sum() <= max(2, 0.02 * ((fc & 2) != 0).sum()), (s, int(((fc ^ fg) != 0).sum()))
        slipped_total += int(moving_c.sum())
        tails_total += int((np.abs(dt_c) > 0).sum())
    assert slipped_total > 10000 and tails_total > 20, (slipped_total, tails_total)
