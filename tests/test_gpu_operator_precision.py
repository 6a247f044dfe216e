"""The operator PCG solves with in FP64 (btd_set_operator_precision; the precision ladder's FP64 outer
operator, the V-cycle's smoothers and coarse levels in FP32), on a torn state.

On torn cloth, loose strands are held by their inertia (m / h^2 ~ 0.03 N/m a node at configuration 4's
pitch) against span stiffnesses of ~8.5e5 N/m. In FP32 a row's span terms cancel on a rigid motion
only to ~6e-8 of their size (~0.05 N/m), so the FP32 rows are a different operator there - no longer
positive definite on the 256 x 256 patch, where the FP64 oracle given FP32-rounded fine rows breaks
down as the GPU's FP32 solve does (the oracle's precision study, fp32_rows). The FP64 rows - each
span's block formed in FP64 from its element vector, every row summed in FP64 - are the oracle's
operator to the FP32 rounding of the laws' scalars: a solve to rel-res 1e-6 on them meets 1e-6 against
the oracle's own operator, which a solve on the FP32 rows misses."""
import numpy as np
import pytest

import btd_b200 as btd
from helpers import MG, copy_state, operator_apply
from oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torn():
    """Configuration 4's tearing patch at 64 x 64 (its pitch, a 16 x 16-cell region): 14 substeps of
    the oracle with the grips pulling (the yarns separate from substep 8); then, the grips' columns
    pinned where they are, the next substep's first Newton system staged on both sides from the same
    float32 state (spans, slip tails and damage field copied)."""
    c = btd.configs.CONFIG4
    sc, left, right = btd.configs.config4(n=64, region=16)
    run = Oracle(sc, h=c["h"], newton_iterations=c["newton_iterations"], pcg_iterations=500, pcg_rel_tol=c["pcg_rel_tol"], **MG)
    x0 = run.x.astype(np.float32).astype(np.float64)
    grips = []
    for slot, (nodes, sign) in enumerate(((left, -1.0), (right, 1.0))):
        picked = int(nodes[len(nodes) // 2])
        a = x0[picked].copy()
        run.add_grip(nodes, np.ones(len(nodes)), (x0[nodes] - x0[picked]).reshape(-1), a, c["grip_stiffness"])
        grips.append((slot, a, sign))
    for s in range(1, 15):
        for slot, a, sign in grips:
            run.set_grip_goal(slot, a + np.array([sign * 0.5 * c["grip_speed"] * s * c["h"], 0, 0]))
        run.substep()
    separated = int((run.field() >= 254).sum())
    sc.pinned[left] = 1
    sc.pinned[right] = 1
    cpu = Oracle(sc, h=c["h"], newton_iterations=c["newton_iterations"], pcg_iterations=500, pcg_rel_tol=c["pcg_rel_tol"], **MG)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(c["h"], c["newton_iterations"], c["pcg_rel_tol"]))
    cpu.set_segments(**run.segments())
    cpu.set_field(run.field())
    x, v, _, _ = run.state()
    cpu.set_state(x, v)
    copy_state(cpu, gpu)
    cpu.predict()
    gpu.encode_predict()
    gpu.encode_assemble(True)
    A_cpu, _, _ = cpu.assemble()
    cpu.build_levels()
    return sc, cpu, gpu, A_cpu, separated


def solve(gpu, b, fp64):
    gpu.set_operator_precision(fp64)
    try:
        gpu.set_pcg(500, 1e-6)
        gpu.write_vector("B", b)
        gpu.encode_pcg()
        d = gpu.delta_f64()
        c = gpu.counter_dict()
    finally:
        gpu.set_operator_precision(True)
        gpu.write_vector("B", b)
    return d, c


def test_the_fp64_operator_solves_the_oracles_system_on_torn_cloth(torn):
    sc, cpu, gpu, A_cpu, separated = torn
    assert separated > 300, separated
    b = gpu.read_vector("B")
    nb = np.linalg.norm(b)
    d64, c64 = solve(gpu, b, True)
    d32, c32 = solve(gpu, b, False)
    rel64 = np.linalg.norm(b - operator_apply(A_cpu, sc.nx, sc.ny, d64)) / nb
    rel32 = np.linalg.norm(b - operator_apply(A_cpu, sc.nx, sc.ny, d32)) / nb
    assert c64["pcg_missed"] == 0 and c64["rel_residual"] <= 1e-6, c64
    # against the oracle's operator: the tolerance and the FP32 rounding of the laws' scalars
    assert rel64 <= 2e-6, (rel64, rel32)
    assert rel64 < rel32, (rel64, rel32)
    # and the oracle's own solve of the same system
    dc, _, rel_c = cpu.pcg(b, 500, 1e-6)
    assert rel_c <= 1e-6
    assert np.abs(d64 - dc).max() <= 1e-4 * np.abs(dc).max(), (np.abs(d64 - dc).max(), np.abs(dc).max())
