"""The reference's unit tests of its constitutive laws (tests/unit/axial.test.ts, laws.test.ts),
restated on the oracle's laws (the FP64 restatement the CUDA path is checked against), with the same
fixtures and tolerances: vitest's toBeCloseTo(x, d) is |a - x| < 10^-d / 2."""
import math

import numpy as np

import btd_b200 as btd
from oracle import laws


def close(a, x, d):
    return abs(a - x) < 0.5 * 10.0 ** (-d)


def denim_yarn(k=1):
    """DENIM.yarns[k] (material.ts) as the scene compiler holds it: (eaLow, eaHigh, crimpStrain, eaCompress)."""
    y = btd.material_preset(0).yarns[k]
    return np.array([y.ea_low, y.ea_high, y.crimp_strain, y.ea_compress])


# ---- axial.test.ts

def test_tension_is_the_derivative_of_energy_and_stiffness_of_tension():  # axial.test.ts:8-16
    p = denim_yarn()
    for eps in (-0.01, 0.001, 0.01, 0.02, 0.03, 0.05, 0.08):
        h = 1e-6
        dE = (laws.axial(p, eps + h)[2] - laws.axial(p, eps - h)[2]) / (2 * h)
        assert close(dE, laws.axial(p, eps)[0], 5), eps
        dT = (laws.axial(p, eps + h)[0] - laws.axial(p, eps - h)[0]) / (2 * h)
        assert close(dT, laws.axial(p, eps)[1], 3), eps


def test_strain_at_tension_inverts_the_curve():  # axial.test.ts:18-20
    p = denim_yarn()
    for t in (0.01, 0.1, 0.5, 2, 11):
        assert close(laws.axial(p, laws.strain_at_tension(p, t))[0], t, 9)


def test_cohesive_softening_dissipates_peak_times_softening_over_two():  # axial.test.ts:22-41
    p = denim_yarn()
    B = 9
    y = np.array([B * p[0], B * p[1], p[2], B * p[3]])  # one warp of a 9-warp bundle law
    peak, es = 3.0, 0.05
    ep = laws.strain_at_tension(y, peak * B)
    steps = 20000
    work = 0.0
    for k in range(steps):
        eps = ep + ((k + 0.5) / steps) * es
        work += ((1 - laws.yarn_damage(y, B, 1, peak, es, eps)) * laws.axial(y, eps)[0] * es) / B / steps
    assert close(work, peak * es / 2, 6)
    assert laws.yarn_damage(y, B, 1, peak, es, 0.99 * ep) == 0
    assert laws.yarn_damage(y, B, 1, peak, es, ep + es) == 1
    # an abraded yarn with strength in proportion to its cross-section fails at the same strain
    assert laws.yarn_damage(y, B, 0.3, 0.3 * peak, es, 0.99 * ep) == 0
    assert laws.yarn_damage(y, B, 0.3, 0.3 * peak, es, ep + es) == 1


def test_damage_grows_monotonically_with_strain():  # axial.test.ts:43-51
    p = denim_yarn()
    peak, es = 3.0, 0.05
    ep = laws.strain_at_tension(p, peak)
    prev = 0.0
    for k in range(51):
        d = laws.yarn_damage(p, 1, 1, peak, es, ep + (k / 50) * es)
        assert d >= prev
        prev = d


# ---- laws.test.ts

A = 4 * 1.2e-3 * 1.2e-3
BEND_S0, SHEAR_JAM, SHEAR_RAMP = laws.constants()


def fd(f, x, h):
    return (f(x + h) - f(x - h)) / (2 * h)


def test_bending_quadratic_for_gentle_bends_tan2_toward_a_fold():  # laws.test.ts:8-15
    q = 1e-4 * A
    assert close(laws.bend_psi(q, A)[0] / q, 1, 3)
    th = 2.0
    s = math.sin(th / 2) ** 2
    assert close(laws.bend_psi(s * A, A)[0], A * math.tan(th / 2) ** 2, 12)


def test_bending_derivatives_consistent_and_c2_at_the_joint():  # laws.test.ts:16-27
    for s in (0.1, 0.5, 0.8, BEND_S0, 0.95, 1.3):
        q = s * A
        _, d1, d2 = laws.bend_psi(q, A)
        assert close(fd(lambda x: laws.bend_psi(x, A)[0], q, 1e-7 * A) / d1, 1, 5), s
        assert close(fd(lambda x: laws.bend_psi(x, A)[1], q, 1e-7 * A) / d2, 1, 4), s
    q0 = BEND_S0 * A
    lo = laws.bend_psi(q0 * (1 - 1e-12), A)
    hi = laws.bend_psi(q0 * (1 + 1e-12), A)
    for k in range(3):
        assert close(hi[k] / lo[k], 1, 6)


def test_bending_energy_change_without_cancellation():  # laws.test.ts:28-32
    q0 = 0.3 * A
    dq = 1e-9 * A
    assert close(laws.bend_psi_delta(q0, q0 + dq, dq, A) / (laws.bend_psi(q0, A)[1] * dq), 1, 6)


def test_bending_energy_change_agrees_across_branches():  # laws.test.ts:33-44
    for s0, s1 in ((0.2, 0.5), (0.8, 0.9), (0.9, 0.8), (0.95, 3.0), (40, 41), (41, 40)):
        ref = laws.bend_psi(s1 * A, A)[0] - laws.bend_psi(s0 * A, A)[0]
        assert close(laws.bend_psi_delta(s0 * A, s1 * A, (s1 - s0) * A, A) / ref, 1, 9), (s0, s1)
    assert laws.bend_psi_delta(50 * A, 50 * A, 0, A) == 0


KS, LD = 60.0, 1.6e-3


def test_shear_linear_until_the_jam_then_stiffens_over_the_ramp():  # laws.test.ts:49-53
    assert laws.shear(KS, LD, LD * 1.1)[1] == KS
    assert laws.shear(KS, LD, LD * (1 - SHEAR_JAM + 0.01))[1] == KS
    assert close(laws.shear(KS, LD, LD * (1 - SHEAR_JAM - SHEAR_RAMP - 0.05))[1], 40 * KS, 9)


def test_shear_force_and_stiffness_are_derivatives_of_the_energy():  # laws.test.ts:54-61
    for r in (1.2, 0.9, 1 - SHEAR_JAM - 0.5 * SHEAR_RAMP, 1 - SHEAR_JAM - 2 * SHEAR_RAMP):
        l = r * LD
        f, k, _ = laws.shear(KS, LD, l)
        assert close(fd(lambda x: laws.shear(KS, LD, x)[2], l, 1e-9) / f, 1, 5), r
        assert close(fd(lambda x: laws.shear(KS, LD, x)[0], l, 1e-9) / k, 1, 5), r


def test_wear_dependent_shear_jam():  # laws.test.ts:65-78
    assert close(laws.shear_jam(1), SHEAR_JAM, 12)
    g = math.asin(1 - (1 - laws.shear_jam(0.5)) ** 2)
    assert 44 < g * 180 / math.pi < 50
    a = 0.05
    while a < 1:
        assert laws.shear_jam(a) > laws.shear_jam(a + 0.05)
        a += 0.05
    assert laws.cell_area(1, 1, 0.2, 0.4) == 1
    assert close(laws.cell_area(0, 0.4, 0.3, 0.3), 0.3, 12)


def curvature(La, Lc, pa, pb, pc):
    wa, wc, _, _ = laws.bend_geometry(La, Lc)
    return [wa * pa[k] - 2 * pb[k] + wc * pc[k] for k in range(3)]


def test_unequal_spans_reduce_to_the_second_difference_when_equal():  # laws.test.ts:86-93
    L = 3.4e-3
    wa, wc, kPerB, fold = laws.bend_geometry(L, L)
    assert close(wa, 1, 14) and close(wc, 1, 14)
    assert close(kPerB * L ** 3, 1, 12)
    assert close(fold / (4 * L * L), 1, 12)


def test_no_bending_in_a_straight_chain_of_unequal_spans_strained_alike():  # laws.test.ts:94-101
    for strain in (0, 0.05):
        s = 1 + strain
        r = curvature(3e-3, 4e-3, [0, 0, 0], [3e-3 * s, 0, 0], [7e-3 * s, 0, 0])
        assert math.hypot(*r) < 1e-18


def test_rod_energy_on_a_circular_arc():  # laws.test.ts:102-114
    B, R, La, Lc = 2.4e-7, 0.02, 2.6e-3, 4.1e-3
    at = lambda s: [R * math.sin(s / R), R * (1 - math.cos(s / R)), 0]
    r = curvature(La, Lc, at(-La), at(0), at(Lc))
    kPerB = laws.bend_geometry(La, Lc)[2]
    e = 0.5 * B * kPerB * (r[0] ** 2 + r[1] ** 2 + r[2] ** 2)
    exact = (0.5 * B * (0.5 * (La + Lc))) / (R * R)
    assert close(e / exact, 1, 2)


def test_bending_only_through_yarns_continuous_across_the_node():  # laws.test.ts:115-122
    B = 9
    assert close(laws.bend_scale(1, 1, 0, 0, B), 1, 12)
    assert close(laws.bend_scale(6 / 9, 0.5, 0b111, 0b111, B), 0.5, 12)
    assert laws.bend_scale(4 / 9, 4 / 9, 0b000011111, 0b111110000, B) == 0
