"""Scene compiler pinned against the reference's own known answers (no GPU).

The reference ships one precomputed state, public/drape.bin, whose header carries sceneHash
(src/simulation/scene.ts:134-150) of its default scene: a content hash over the materials' JSON,
sampled field damage/area codes, float32 positions and span flags. Reproducing it bit for bit pins
compileScene (scene.ts:233-278) and its noise, wear, field and initial span coupling.
"""
import json
import os

import numpy as np

import btd_b200 as btd

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_default_scene_hash_matches_reference_drape():
    hdr = json.load(open(os.path.join(GOLDEN, "drape_header.json")))
    sc = btd.compile_scene(btd.default_spec())
    assert sc.N == hdr["node_count"] == 182 * 115
    assert (sc.nx, sc.ny) == (182, 115)
    assert sc.hash() == hdr["scene_hash"]
    assert hdr["bytes"] == 16 + 16 * sc.N


def test_collar_positions_match_reference_drape():
    g = np.load(os.path.join(GOLDEN, "drape_collar.npz"))
    sc = btd.compile_scene(btd.default_spec())
    pos = sc.position.reshape(-1, 3)[g["index"]].astype(np.float32)
    assert np.array_equal(pos, g["position"])
    assert sc.pinned[g["index"]].all()


def test_bundle_weave_and_crossing_mass():
    d = btd.material_preset(0)
    b = btd.bundle_weave(d, 9, 6)
    assert b.name == b"denim-3x1/b9x6"
    assert abs(b.pitch_u - 9 * 0.38e-3) < 1e-18 and abs(b.pitch_v - 6 * 0.58e-3) < 1e-18
    # u-family spans (picks) carry bv = 6 yarns, v-family (warps) bu = 9 (material.ts:201-212)
    assert b.yarns[0].yarns_per_span == 6 and b.yarns[1].yarns_per_span == 9
    assert abs(b.yarns[0].ea_low - 36) < 1e-12 and abs(b.yarns[1].ea_low - 90) < 1e-12
    assert abs(b.crossing_normal0 - 54 * 0.25) < 1e-12


def test_initial_defects_flagged_and_spans_coupled():
    sc = btd.compile_scene(btd.default_spec())
    broken = (sc.seg_flags & btd.SEG_BROKEN) != 0
    assert np.array_equal(broken, (sc.seg_flags & btd.SEG_INITIAL_DEFECT) != 0)
    act = (sc.seg_flags & 3) == 1
    assert (sc.intact[act] > 0).all() and (sc.intact[act] <= 1 + 1e-12).all()
    # rest length is conserved into the tails of initially ruptured spans (yarnField.ts:483-492)
    assert abs(sc.tails.sum() - sc.rest_length[broken].sum()) < 1e-9


def test_layer_spec_coupon_extent():
    d = btd.material_preset(0)
    sc = btd.compile_scene(btd.layer_spec(d, 10 * d.pitch_u, 8 * d.pitch_v, angle=0.3, collar_rows=2, seed=3))
    assert sc.N == sc.nx * sc.ny
    assert sc.pinned.reshape(sc.ny, sc.nx)[2:-2, 2:-2].sum() == 0


def test_scene_compile_rejects_bad_specs():
    """No layer, a bundle wider than the 32-bit cut masks, and a layer too small for two nodes a family
    are BTD_E_INVALID with a message, not a crash or an empty scene."""
    import ctypes as C

    from btd_b200 import _abi

    m = btd.material_preset(0)
    p = C.POINTER(_abi.SceneC)()
    rc = _abi.lib().btd_scene_compile(None, 0, C.byref(p))
    assert rc == -1 and "layer" in _abi.last_error(), (rc, _abi.last_error())
    for spec in (btd.layer_spec(m, 0.05, 0.05, bundle=(33, 1), seed=3), btd.layer_spec(m, 1e-4, 0.05, bundle=(9, 6), seed=3)):
        try:
            btd.compile_scene([spec])
        except _abi.BtdError as e:
            assert e.rc == -1, e
        else:
            raise AssertionError("compile_scene accepted a bad spec")
