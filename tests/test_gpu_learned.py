"""The learned coarse correction (configuration 4's extension; no counterpart in the reference) on the
CUDA path against the FP64 oracle, with the network's weights rounded to BF16 on both sides.

Checked: the coarsest nodes' damage flags against the fine lattice's damaged spans restricted through
the oracle's prolongation weights; the basis (Phi and the Cholesky factor of Phi^T A Phi) against the
oracle's basis of the same coarsest operator (the GPU evaluates the network in BF16 with FP32
accumulation); PCG to relative residual 1e-6 with the correction against the oracle's solve of the same
system (same solution, iteration counts within a quarter, fewer than without the correction); a
tearing patch's substeps against the oracle's with the correction on both sides; the guard (a guard no
solve can meet makes every solve fall back after three iterations and still converge, as the oracle's);
and the gain of the committed network over plain MG-PCG on a held-out seed.
"""
import os

import numpy as np
import pytest

import btd_b200 as btd
from helpers import MG, copy_state, max_abs_rel_to_scale
from oracle import Oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
C4 = btd.configs.CONFIG4


def bf16(w):
    """Round float32 values to BF16 (nearest, ties to even), as the device stores the weights."""
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


@pytest.fixture(scope="module")
def weights():
    return bf16(np.load(os.path.join(HERE, "golden", "learned_coarse.npy")))


def tearing_pair(seed, weights=None, guard=C4["guard"], steps_before=0, contact=True):
    """Configuration 4's tearing patch scaled to 64 x 64 at its pitch on the oracle and the GPU, grips
    attached on both; returns (oracle, gpu, drive(s))."""
    sc, left, right = btd.configs.config4(seed, n=64, region=16)
    cpu = Oracle(sc, h=C4["h"], newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, self_contact=contact, **MG)
    gpu = btd.GpuSolver(sc, btd.configs.solver_params(C4["h"], 4, 1e-6, self_contact=1 if contact else 0))
    x0 = cpu.x.astype(np.float32).astype(np.float64)
    grips = []
    for slot, (nodes, sign) in enumerate(((left, -1.0), (right, 1.0))):
        picked = int(nodes[len(nodes) // 2])
        a = x0[picked].copy()
        cpu.add_grip(nodes, np.ones(len(nodes)), (x0[nodes] - x0[picked]).reshape(-1), a, C4["grip_stiffness"])
        gpu.attach_patch(slot, picked, nodes, np.ones(len(nodes)), a.astype(np.float32), C4["grip_stiffness"], max_lead=1.0)
        grips.append((a, sign))

    def drive(s):
        for slot, (a, sign) in enumerate(grips):
            t = (a + np.array([sign * 0.5 * C4["grip_speed"] * s * C4["h"], 0, 0])).astype(np.float32)
            cpu.set_grip_goal(slot, t.astype(np.float64))
            gpu.set_target(t, slot=slot)

    if weights is not None:
        cpu.set_learned(weights.astype(np.float64), on=True, guard=guard)
        gpu.set_learned(weights, on=True, guard=guard)
    for s in range(1, steps_before + 1):
        drive(s)
        cpu.substep()
    return cpu, gpu, drive


def staged(weights, steps_before=24, seed=42):
    """A Newton system of the tearing patch after `steps_before` oracle substeps, assembled on the GPU.
    Self-contact is off here, so that both sides' contact flags (the oracle's come from its last contact
    terms, the GPU's from its own) cannot differ."""
    cpu, gpu, drive = tearing_pair(seed, weights, steps_before=steps_before, contact=False)
    copy_state(cpu, gpu)
    drive(steps_before + 1)
    cpu.predict()
    gpu.encode_predict()
    # a Newton iteration puts the grips' springs into the external terms (the assembly stage alone
    # leaves them out, and a sheet held by nothing is beyond an FP32 preconditioner at rel-res 1e-6),
    # then the system is assembled afresh at the new iterate
    gpu.encode_newton_iteration(0)
    gpu.encode_assemble(True)
    return cpu, gpu


def test_damage_flags_restrict_through_the_prolongation(weights):
    cpu, gpu = staged(weights, steps_before=30)
    gpu.set_pcg(5, 0.0)
    gpu.encode_pcg()
    _, _, _, flags = gpu.learned_basis()
    # fine damage flags from the spans (a span at the node exists but is broken or not fully intact)
    seg = gpu.segments()
    sc = cpu.scene
    nx, ny = sc.nx, sc.ny
    fl, it = seg["seg_flags"].reshape(-1, 2), seg["intact"].reshape(-1, 2)
    dam = np.zeros(sc.N, bool)
    for n in range(sc.N):
        i, j = n % nx, n // nx
        for f, (pi, pj) in enumerate(((i - 1, j), (i, j - 1))):
            nxt = (i + 1 < nx) if f == 0 else (j + 1 < ny)
            spans = ([(n, f)] if nxt else []) + ([(pj * nx + pi, f)] if pi >= 0 and pj >= 0 else [])
            for m, g in spans:
                if (fl[m, g] & 1) and ((fl[m, g] & 2) or it[m, g] < 1):
                    dam[n] = True
    assert dam.any(), "the staged state has no damage"
    A0, _ = gpu.read_operator(0)
    cpu.build_levels(A0)
    f = dam
    for k in range(gpu.level_count() - 1):
        idx, w = cpu.prolongation(k)
        c = np.zeros(gpu.level_nodes(k + 1), bool)
        for q in range(4):
            ok = (idx[:, q] >= 0) & (w[:, q] > 0) & f
            c[idx[ok, q]] = True
        f = c
    assert np.array_equal((flags & 1) != 0, f)


def test_basis_matches_the_oracle(weights):
    cpu, gpu = staged(weights)
    gpu.set_pcg(5, 0.0)
    gpu.encode_pcg()
    phi, G, dead, flags = gpu.learned_basis()
    k = gpu.level_count() - 1
    A, fixed = gpu.read_operator(k)
    M = len(fixed)
    n = int(round(np.sqrt(M)))
    assert n * n == M
    fl = np.stack([(flags & 1) != 0, (flags & 2) != 0], 1).astype(np.float32)
    out = cpu.learned_basis_of(weights.astype(np.float64), A, fixed, n, n, fl)
    assert out is not None
    X, phi_c, G_c, dead_c = out
    assert np.array_equal(dead, dead_c)
    # BF16 inputs and activations against FP64: a few parts in a thousand of the basis
    err = np.linalg.norm(phi - phi_c) / np.linalg.norm(phi_c)
    assert err < 2e-2, err
    L, Lc = np.tril(G), np.tril(G_c)
    assert np.linalg.norm(L @ L.T - Lc @ Lc.T) < 4e-2 * np.linalg.norm(Lc @ Lc.T)


def test_learned_pcg_matches_the_oracle(weights):
    cpu, gpu = staged(weights, steps_before=6)
    A0, _ = gpu.read_operator(0)
    b = gpu.read_vector("B")
    cpu.build_levels(A0)
    gpu.set_pcg(500, 1e-6)
    gpu.encode_pcg()
    dg = gpu.read_vector("delta")
    its_g = gpu.counter_dict()["pcg_last"]
    dc, its_c, rel_c = cpu.pcg(b, 500, 1e-6)
    assert rel_c <= 1e-6 and gpu.counter_dict()["rel_residual"] <= 1e-6
    assert abs(its_g - its_c) <= max(2, 0.25 * its_c), (its_g, its_c)
    assert max_abs_rel_to_scale(dg, dc) < 1e-3
    st = gpu.learned_stats()
    assert st["solves"] >= 1 and st["applied"] >= its_g and st["fallbacks"] == 0
    # the same system without the correction takes more iterations
    gpu.set_learned(None, on=False)
    gpu.write_vector("B", b)
    gpu.encode_pcg()
    assert gpu.counter_dict()["pcg_last"] > its_g


def run_pair(cpu, gpu, drive, first, count):
    errs, its_c, its_g = [], 0, 0
    for s in range(first, first + count):
        copy_state(cpu, gpu)
        drive(s)
        gpu.clear_counters()
        cpu.predict()
        for _ in range(4):
            its_c += cpu.newton_step()["pcg_iterations"]
        cpu.finalize()
        gpu.substep()
        its_g += gpu.counter_dict()["pcg_total"]
        xc = cpu.x
        errs.append(np.abs(gpu.x.astype(np.float64) - xc).max() / np.abs(xc).max())
    return np.array(errs), its_c, its_g


def test_learned_substeps_match_the_oracle(weights):
    cpu, gpu, drive = tearing_pair(42, weights, steps_before=0)
    errs, its_c, its_g = run_pair(cpu, gpu, drive, 1, 8)
    assert np.median(errs) < 1e-5, errs
    assert errs.max() < 3e-4, errs
    assert abs(its_g - its_c) <= 0.25 * its_c, (its_g, its_c)
    assert gpu.learned_stats()["applied"] > 0


def test_guard_falls_back_like_the_oracle(weights):
    cpu, gpu, drive = tearing_pair(42, weights, guard=1e-9)
    errs, its_c, its_g = run_pair(cpu, gpu, drive, 1, 2)
    st, sc = gpu.learned_stats(), cpu.learned_stats()
    # every solve that runs three iterations without converging falls back (a later Newton iteration
    # may converge sooner); the same solves on both sides
    assert st["solves"] == sc["solves"] == 8, (st, sc)
    assert st["fallbacks"] == sc["fallbacks"] and st["fallbacks"] >= st["solves"] - 2, (st, sc)
    assert gpu.counter_dict()["rel_residual"] <= 1e-6
    assert errs.max() < 3e-4, errs


def test_committed_network_gains_on_a_held_out_seed(weights):
    """The hanging patch of the plain configuration (64 x 64, seed 2: not among the training seeds):
    PCG iterations per Newton step to rel-res 1e-6 with the committed network against without."""
    cfg = btd.configs.CONFIG0
    sc = btd.configs.hanging_patch(64, 0.3, seed=2)
    its = {}
    for on in (False, True):
        g = btd.GpuSolver(sc, btd.configs.solver_params(cfg["h"], 4, 1e-6))
        if on:
            g.set_learned(weights, on=True, guard=C4["guard"])
        g.substeps(4)
        c = g.counter_dict()
        its[on] = c["pcg_total"] / c["newton"]
        g.close()
    assert its[True] <= 0.85 * its[False], its
