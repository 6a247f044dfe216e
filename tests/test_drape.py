"""The drape file of the reference (src/simulation/gpu/settle.ts:4-22) on the host: the header our
scene compiler produces for the default scene is the one public/drape.bin carries, and a file
loads only onto its own scene (size, magic, version, node count, scene hash all checked)."""
import json
import os

import numpy as np

import btd_b200 as btd

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_drape_header_of_the_default_scene_is_the_reference_file_header():
    hdr = json.load(open(os.path.join(GOLDEN, "drape_header.json")))
    sc = btd.compile_scene(btd.default_spec())
    head = btd.drape.drape_header(sc.N, sc.hash())
    assert np.frombuffer(head, "<u4").tolist() == [hdr["magic"], hdr["version"], hdr["node_count"], hdr["scene_hash"]]
    assert len(head) + 16 * sc.N == hdr["bytes"]


def test_a_drape_loads_only_onto_its_own_scene():
    n, h = 7, 0xFA77387B
    x = np.arange(4 * n, dtype=np.float32).reshape(n, 4)
    data = btd.drape.drape_header(n, h) + x.astype("<f4").tobytes()
    assert np.array_equal(btd.drape.parse_drape(data, n, h), x)
    assert btd.drape.parse_drape(data, n, h ^ 1) is None  # another scene
    assert btd.drape.parse_drape(data, n + 1, h) is None  # another node count (and size)
    assert btd.drape.parse_drape(data[:-4], n, h) is None  # truncated
    bad = bytearray(data)
    bad[0] ^= 1
    assert btd.drape.parse_drape(bytes(bad), n, h) is None  # magic
    bad = bytearray(data)
    bad[4] = 2
    assert btd.drape.parse_drape(bytes(bad), n, h) is None  # version
