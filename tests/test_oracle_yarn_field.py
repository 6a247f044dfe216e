"""The reference's unit tests of its yarn damage field (tests/unit/yarnField.test.ts), restated on the
oracle's restatement of yarnField.ts (what the CUDA path's damage field is checked against), on the
same coupon - DENIM bundled 9 x 6, 12 x 10 cells, one collar row, unworn, seed 3 - with the same
cuts, strains and tolerances (vitest toBeCloseTo(x, d): |a - x| < 10^-d / 2). The field defines the
break-event set of the damage configuration."""
import math

import numpy as np
import pytest

import btd_b200 as btd
from oracle import Oracle, field_constants, recoil_length, share_cap

SHARE_FRACTION, DAMAGE_CUT, DAMAGE_PULLED = field_constants()
SEG_EXISTS, SEG_BROKEN, SEG_SLIPPED = btd.SEG_EXISTS, btd.SEG_BROKEN, btd.SEG_SLIPPED


def close(a, x, d):
    return abs(a - x) < 0.5 * 10.0 ** (-d)


def coupon():
    m = btd.material_preset(0)
    sc = btd.compile_scene(btd.layer_spec(m, 12 * 9 * m.pitch_u, 10 * 6 * m.pitch_v, bundle=(9, 6), collar_rows=1, seed=3))
    return sc, Oracle(sc)


@pytest.fixture
def field():
    sc, o = coupon()
    return sc, o, o.field_layer(), sc.field_damage.copy()


def span_length(fl, f):
    return fl["bv"] if f == 1 else fl["bu"]


def test_every_crossing_of_a_span_maps_back_to_it(field):  # yarnField.test.ts:32-47
    sc, o, fl, _ = field
    for f in (0, 1):
        for i, j in ((2, 3), (5, 1)):
            B = fl["bu"] if f == 1 else fl["bv"]
            for q in range(B):
                for p in range(span_length(fl, f)):
                    c = o.span_crossing(i, j, f, q, p) - fl["offset"]
                    assert o.own_span(c % fl["K"], c // fl["K"], f) == (i, j)


def test_interpolates_a_uniform_strain_and_ignores_spans_without_one(field):  # yarnField.test.ts:49-57
    sc, o, fl, _ = field
    strain = np.full(2 * sc.N, 0.02)
    assert close(o.interpolated_strain(1, 40, 30, strain), 0.02, 12)
    strain[:] = np.nan
    strain[2 * (3 * sc.nx + 4) + 1] = 0.05
    c = o.span_crossing(4, 3, 1, 4, 2) - fl["offset"]
    assert close(o.interpolated_strain(1, c % fl["K"], c // fl["K"], strain), 0.05, 12)


def test_a_span_keeps_its_intact_fraction_and_separates_conserving_length(field):  # yarnField.test.ts:59-80
    sc, o, fl, damage = field
    i, j, f = 4, 3, 1
    s_idx = 2 * (j * sc.nx + i) + f
    for q in range(3):
        damage[2 * o.span_crossing(i, j, f, q, q + 1) + f] = DAMAGE_CUT
    damage[2 * o.span_crossing(i, j, f, 3, 0) + f] = 127
    o.set_field(damage)
    assert o.couple_spans() == 0
    seg = o.segments()
    assert close(seg["intact"][s_idx], (5 + (1 - 127 / 255)) / 9, 9)
    assert seg["cut_mask"][s_idx] == 0b111
    total = seg["tails"].sum()
    for q in range(9):
        damage[2 * o.span_crossing(i, j, f, q, 2) + f] = DAMAGE_CUT
    o.set_field(damage)
    assert o.couple_spans() == 1
    seg = o.segments()
    assert seg["seg_flags"][s_idx] & SEG_BROKEN == SEG_BROKEN
    assert seg["intact"][s_idx] == 0
    assert close(seg["tails"].sum() - total, seg["rest_length"][s_idx], 12)


def test_a_ruptured_spans_yarns_slide_out_of_the_other_sides_weave(field):  # yarnField.test.ts:82-106
    sc, o, fl, damage = field
    i, j, f = 4, 3, 0
    P = span_length(fl, f)
    cuts = [[0], [P - 1], [4], [1, 6]]
    for q in range(fl["bv"]):
        for p in (cuts[q] if q < len(cuts) else [2]):
            damage[2 * o.span_crossing(i, j, f, q, p) + f] = DAMAGE_CUT
    before = damage.copy()
    o.set_field(damage)
    assert o.couple_spans() == 1
    damage = o.field()
    assert P - P // 2 == 5
    pulled = lambda q: "".join("1" if damage[2 * o.span_crossing(i, j, f, q, p) + f] == DAMAGE_PULLED else "0" for p in range(P))
    assert [pulled(q) for q in range(5)] == ["011110000", "000001110", "000000000", "001110000", "000110000"]
    changed = np.nonzero(damage != before)[0]
    assert (changed % 2 == f).all()


def test_slipped_yarns_part_from_their_nodes_weave_only_once(field):  # yarnField.test.ts:108-129
    sc, o, fl, damage = field
    f = 1
    P = span_length(fl, f)
    seg = o.segments()
    flags, site = seg["seg_flags"].copy(), seg["fail_site"].copy()
    for i, s in ((4, 0), (6, 1)):
        s_idx = 2 * (3 * sc.nx + i) + f
        flags[s_idx] |= SEG_BROKEN | SEG_SLIPPED
        site[s_idx] = s
    o.set_segments(seg_flags=flags, fail_site=site)
    damage[2 * o.span_crossing(6, 3, f, 0, 1) + f] = DAMAGE_CUT
    o.set_field(damage)
    assert o.couple_spans() == 0
    assert P == 6
    damage = o.field()
    pulled = lambda i, q: "".join("1" if damage[2 * o.span_crossing(i, 3, f, q, p) + f] == DAMAGE_PULLED else "0" for p in range(P))
    for q in range(fl["bu"]):
        assert pulled(4, q) == "111000"
        assert pulled(6, q) == "000111"
    assert o.segments()["seg_flags"][2 * (3 * sc.nx + 4) + f] & SEG_SLIPPED == 0


def test_an_overstretched_yarn_separates_at_its_weakest_crossing_only(field):  # yarnField.test.ts:131-156
    sc, o, fl, damage = field
    o.set_field(damage)
    o.update_field(np.full(2 * sc.N, 0.5))
    damage = o.field()
    strength, area = sc.field_strength, sc.field_area
    for f in (0, 1):
        B = fl["bu"] if f == 1 else fl["bv"]
        for q in range(B):
            cuts, weakest, low = 0, -1, math.inf
            for p in range(span_length(fl, f)):
                c = o.span_crossing(4, 3, f, q, p)
                cuts += damage[2 * c + f] == DAMAGE_CUT
                peak = strength[2 * c + f] / (area[2 * c + f] / 255)
                if peak < low:
                    low, weakest = peak, c
            assert cuts == 1 and damage[2 * weakest + f] == DAMAGE_CUT, (f, q)


def test_a_cut_end_pulls_out_by_its_shear_lag_retraction_under_load_only(field):  # yarnField.test.ts:158-193
    sc, o, fl, damage = field
    c0 = fl["offset"] + 30 * fl["K"] + 40
    damage[2 * c0] = DAMAGE_CUT
    o.set_field(damage)

    def pull_all(strain):
        total, n = 0, o.pull_out(strain)
        while n > 0:
            total += n
            n = o.pull_out(strain)
        return total

    assert pull_all(np.zeros(2 * sc.N)) == 0
    strain = np.zeros(2 * sc.N)
    strain[0::2] = 0.06
    pull_all(strain)
    mat, weave = sc.layers[0].material, sc.layers[0].weave
    yy = mat.yarns[0]
    y = (yy.ea_low, yy.ea_high, yy.crimp_strain, yy.ea_compress)
    from oracle import laws

    B = fl["bv"]
    T, _, W = laws.axial(y, 0.06)
    comp = (T * 0.06 - W) / B
    p = weave.pitch_u
    n0 = sc.crossing_normal0[0] / (fl["bu"] * fl["bv"])
    delta = comp * p / (mat.crossing_friction * n0)
    assert close(recoil_length(y, B, 1, 1e3, 0.06, mat.crossing_friction, n0, mat.crossing_wrap, 0, p), delta, 12)
    peak = float(sc.field_strength[2 * c0])
    capped = recoil_length(y, B, 1, peak, 0.6, mat.crossing_friction, n0, mat.crossing_wrap, 0, p)
    assert close(capped, recoil_length(y, B, 1, peak, 0.2, mat.crossing_friction, n0, mat.crossing_wrap, 0, p), 12)
    run = min(12, math.floor(delta / p + 0.5))
    assert run > 0
    damage = o.field()
    for d in (-1, 1):
        for k in range(1, run + 1):
            assert damage[2 * (c0 + d * k)] == DAMAGE_PULLED
        assert damage[2 * (c0 + d * (run + 1))] < DAMAGE_PULLED
    assert pull_all(np.zeros(2 * sc.N)) == 0
    assert o.field()[2 * (c0 + 1)] == DAMAGE_PULLED


def test_overloads_the_yarns_beside_a_run_of_separated_neighbours(field):  # yarnField.test.ts:195-208
    sc, o, fl, _ = field
    sep = np.zeros(len(sc.field_damage), np.uint8)
    reach = o.share_reach(1)
    for k in range(40, 43):
        sep[2 * (fl["offset"] + 30 * fl["K"] + k) + 1] = 1
    assert close(o.share_factor(sep, 1, 43, 30, reach), 1 + SHARE_FRACTION * 3 / 2, 12)
    assert close(o.share_factor(sep, 1, 39, 30 + reach, reach), 1 + SHARE_FRACTION * 3 / 2, 12)
    assert o.share_factor(sep, 1, 43, 30 + reach + 1, reach) == 1
    assert o.share_factor(sep, 1, 45, 30, reach) == 1
    assert close(o.share_factor(sep, 1, 43, 30, reach, 0.1), 1.1, 12)
    assert close(share_cap(2, 0.35, 0.25, 0.3, 0, 11), 5 * 0.35 * 0.25 / 11, 12)


def test_a_crack_runs_on_beside_the_last_break_across_bundles(field):  # yarnField.test.ts:210-227
    sc, o, fl, damage = field
    k_edge = 4 * fl["bu"] - 1
    m_cut = 3 * fl["bv"] + fl["bv"] // 2 + 1
    damage[2 * (fl["offset"] + m_cut * fl["K"] + k_edge) + 1] = DAMAGE_CUT
    o.set_field(damage)
    o.couple_spans()
    o.update_field(np.full(2 * sc.N, 0.2))
    damage = o.field()
    reach = o.share_reach(1)
    at = [m for m in range(fl["M"]) if damage[2 * (fl["offset"] + m * fl["K"] + k_edge + 1) + 1] == DAMAGE_CUT and abs(m - m_cut) <= reach]
    assert at
