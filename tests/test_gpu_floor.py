"""Floor contact on the CUDA path (floor.ts:5-28; assemble.wgsl:191-209; energy.wgsl:112-125;
step.wgsl:77-86) against the oracle's restatement of the same terms, and the reference's floor
contracts (tests/gpu/floor.ts) restated on a mounted sheet: cloth never passes below half its
thickness, and a flap that reaches the floor comes to rest lying along it.
"""
import numpy as np
import pytest

import btd_b200 as btd
from helpers import MG, copy_state
from oracle import Oracle

pytestmark = pytest.mark.gpu

H = 1 / 120
NP = 32
FLOOR_Z = -0.06
HALF = 0.5 * btd.material_preset(0).thickness


def sheet():
    return btd.configs.hanging_patch(NP, 0.15, seed=9)


def test_floor_trajectory_matches_oracle():
    """The free edge of a sheet mounted along one edge falls onto a floor 6 cm below: 90 substeps
    within 0.03 of the motion of the oracle's (converged schedule, correctness.ts:271)."""
    sc = sheet()
    cpu = Oracle(sc, h=H, newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, **MG)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(H, 4, 1e-6))
    cpu.set_floor(FLOOR_Z)
    gpu.set_floor(FLOOR_Z)
    x0, _ = copy_state(cpu, gpu)
    lowest = np.inf
    for _ in range(90):
        cpu.substep()
        gpu.substep()
        lowest = min(lowest, float(gpu.x[:, 2].min()) - FLOOR_Z)
    xc, xg = cpu.x, gpu.x.astype(np.float64)
    moved = np.abs(xc - x0).max()
    assert xc[:, 2].min() - FLOOR_Z < 3 * HALF, "the sheet must reach the floor"
    assert np.abs(xg - xc).max() < 0.03 * moved, (np.abs(xg - xc).max(), moved)
    assert lowest >= HALF * 0.999, lowest


def test_thrown_sheet_never_passes_below_half_thickness():
    """floor.ts:154-176: cloth thrown at the floor at 3 m/s stops above half its thickness."""
    sc = sheet()
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(H, 2, 1e-6))
    gpu.set_floor(-0.01)
    x = gpu.x.copy()
    v = np.zeros_like(x)
    free = sc.pinned == 0
    v[free, 2] = -3.0
    gpu.set_state(x, v)
    lowest = np.inf
    for _ in range(40):
        gpu.substep()
        lowest = min(lowest, float(gpu.x[free, 2].min()) + 0.01)
    assert lowest >= HALF * 0.999, lowest


def test_flap_lies_along_the_floor_and_rests():
    """floor.ts:240-277: a flap hanging from its mount lies along the floor where it reaches it and
    comes to rest there (2 s), above half its thickness and without stretching."""
    sc = sheet()
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6))
    gpu.set_floor(-0.1)
    gpu.substeps(120)
    x, v = gpu.state()
    height = x[:, 2] - (-0.1)
    assert height.min() >= HALF * 0.999, height.min()
    lying = int((height < HALF + 1e-3).sum())
    assert lying > NP, lying
    assert np.abs(v[:, :3]).max() < 0.01, np.abs(v[:, :3]).max()
    pitch = 0.15 / (NP - 1)
    span = np.linalg.norm(x[1:, :3] - x[:-1, :3], axis=1).reshape(-1)
    horiz = span.reshape(-1)[np.arange(len(span)) % NP != NP - 1]
    assert np.abs(horiz / pitch - 1).max() < 0.02, np.abs(horiz / pitch - 1).max()
