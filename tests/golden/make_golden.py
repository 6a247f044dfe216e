"""Regenerates the committed golden fixtures from a checkout of the reference.

Usage: python tests/golden/make_golden.py <reference checkout>  (or set BTD_REFERENCE to its path).

drape_header.json: the header of the reference's precomputed drape (public/drape.bin:
[magic, version, node count, sceneHash], src/simulation/gpu/settle.ts:4-22) for its default scene.
drape_collar.npz: the drape's positions of the mounted collar nodes (scene.ts:309 pins 2 rows on
every side); settling never moves mounted nodes, so these are the compiled initial positions
rounded to float32, a known answer for the scene compiler.
drape_settled.npz: the drape's positions of every ninth free node, the reference's settled state.
"""
import json
import os
import struct
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BTD_REFERENCE")
if not REF:
    sys.exit("usage: make_golden.py <reference checkout> (or set BTD_REFERENCE)")
HERE = os.path.dirname(os.path.abspath(__file__))

data = open(os.path.join(REF, "public", "drape.bin"), "rb").read()
magic, version, n, h = struct.unpack("<4I", data[:16])
pos = np.frombuffer(data[16:], dtype="<f4").reshape(n, 4)
json.dump({"magic": magic, "version": version, "node_count": n, "scene_hash": h, "bytes": len(data)},
          open(os.path.join(HERE, "drape_header.json"), "w"), indent=1)
nx, ny, cr = 182, 115, 2  # defaultSceneSpecs (scene.ts:438-469) compiles to 182 x 115 with 2 collar rows
j, i = np.divmod(np.arange(n), nx)
collar = (i < cr) | (j < cr) | (i >= nx - cr) | (j >= ny - cr)
idx = np.nonzero(collar)[0].astype(np.int32)
np.savez_compressed(os.path.join(HERE, "drape_collar.npz"), index=idx, position=pos[idx, :3].copy())
# drape_settled.npz: the settled positions of every ninth free node (the reference's own GPU solve of
# settleDrape, settle.ts:24-62), for the end-to-end check of btd_settle_drape
free = np.nonzero(~collar)[0][::9].astype(np.int32)
np.savez_compressed(os.path.join(HERE, "drape_settled.npz"), index=free, position=pos[free, :3].copy())
print("wrote", len(idx), "collar nodes,", len(free), "settled free nodes, hash", hex(h))
