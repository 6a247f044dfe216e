"""Adaptive Newton gate on the CUDA path (encodeSubstep's optional iterations, solver.ts:729-757;
gate.wgsl:12-23): the first newton_iterations always run; each further one up to newton_max runs only
while the previous one still moved some node by more than newton_tolerance, and a skipped one keeps
every later one off. Each optional iteration is a conditional node of the substep graph.
"""
import numpy as np
import pytest

import btd_b200 as btd

pytestmark = pytest.mark.gpu

H = 1 / 60
NP = 32


def solver(newton, newton_max, tol, graphs=True):
    sc = btd.configs.hanging_patch(NP, 0.15, seed=5)
    s = btd.GpuSolver(sc, btd.configs.solver_params(H, newton, 1e-6, newton_max=newton_max, newton_tolerance=tol))
    s.set_graph_mode(graphs)
    return s


def run(s, steps, **kw):
    newton = []
    updates = []
    for _ in range(steps):
        s.clear_counters()
        s.substep(**kw)
        c = s.counter_dict()
        newton.append(c["newton"])
        updates.append(c["max_update"])
    return s.x.copy(), newton, updates


def test_gate_closed_equals_fewer_iterations():
    """A tolerance no update reaches keeps every optional iteration off: the same run, bit for bit,
    as newton_iterations alone."""
    xa, na, _ = run(solver(1, 3, 1.0), 6)
    xb, nb, _ = run(solver(1, 1, 1.0), 6)
    assert na == [1] * 6 and nb == [1] * 6
    assert np.array_equal(xa, xb)


def test_gate_open_equals_more_iterations():
    """A zero tolerance runs every optional iteration: the same run as newton_max unconditional ones."""
    xa, na, _ = run(solver(1, 3, 0.0), 6)
    xb, nb, _ = run(solver(3, 3, 0.0), 6)
    assert na == [3] * 6 and nb == [3] * 6
    assert np.array_equal(xa, xb)


def test_gate_stops_at_the_first_small_update():
    """In between, iteration k runs exactly when k < newton_iterations or iteration k - 1 moved some
    node by more than the tolerance and ran itself; eager launches decide the same way."""
    # a tolerance between the second and third updates of the first substep: it runs three
    _, _, u0 = run(solver(1, 4, 0.0), 1)
    tol = float(np.sqrt(u0[0][1] * u0[0][2]))
    xg, ng, ug = run(solver(1, 4, tol), 8)
    xe, ne, ue = run(solver(1, 4, tol, graphs=False), 8)
    assert ng == ne and np.array_equal(xg, xe)
    assert ng[0] == 3, (ng, u0[0][:4], tol)
    for n, u in zip(ng, ug):
        ran = 1
        for k in range(1, 4):
            if u[k - 1] > tol and ran == k:
                ran += 1
        assert n == ran, (n, u)
        assert all(v == 0.0 for v in u[n:4])


def test_substep_min_and_max_iterations():
    """encodeSubstep(min, max): min raises the unconditional count, max the gated bound."""
    _, n, _ = run(solver(1, 1, 0.0), 2, min_iterations=2)
    assert n == [2, 2]
    _, n, _ = run(solver(1, 1, 0.0), 2, max_iterations=3)
    assert n == [3, 3]
    s = solver(1, 3, 0.0)
    assert s.launch_count(1, 3, 12) > solver(1, 1, 0.0).launch_count(1, 3, 12)


def test_gated_substeps_match_the_oracle_with_the_same_gate():
    """The gated schedule against the oracle driven through the same gate (gate.wgsl:12-23): from the
    same state, the oracle runs newton_iterations Newton iterations, then more up to newton_max while the
    last one moved some node by more than the tolerance; the GPU's substep graph decides on the device.
    Per substep the same number of Newton iterations runs and the positions agree."""
    import sys

    from helpers import MG, copy_state
    from oracle import Oracle

    sc = btd.configs.hanging_patch(NP, 0.15, seed=5)
    _, _, u0 = run(solver(1, 4, 0.0), 1)
    tol = float(np.sqrt(u0[0][1] * u0[0][2]))
    gpu = solver(1, 4, tol)
    cpu = Oracle(sc, h=H, newton_iterations=1, pcg_iterations=500, pcg_rel_tol=1e-6, **MG)
    errs = []
    for s in range(8):
        copy_state(cpu, gpu)
        gpu.clear_counters()
        gpu.substep()
        ng = gpu.counter_dict()["newton"]
        cpu.predict()
        nc = 0
        while nc < 4:
            r = cpu.newton_step()
            nc += 1
            if not r["max_update"] > tol:
                break
        cpu.finalize()
        assert ng == nc, (s, ng, nc)
        xc = cpu.x
        errs.append(np.abs(gpu.x.astype(np.float64) - xc).max() / np.abs(xc).max())
    assert np.median(errs) < 1e-5 and max(errs) < 3e-4, errs
