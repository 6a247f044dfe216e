"""The settled drape (src/simulation/gpu/settle.ts): settling the authored drape before interaction,
and the precomputed drape file that lets a session skip it.

File (settle.ts:4-13): a 16-byte header of four little-endian u32 - magic 0x50415244, version 1, node
count, sceneHash of the compiled scene (scene.ts:134-150) - then 4 float32 a node (the positions
buffer, w included). A file loads only onto a solver of exactly that scene (settle.ts:16-22).
"""
import struct

import numpy as np

DRAPE_MAGIC = 0x50415244
DRAPE_VERSION = 1


def drape_header(node_count, scene_hash):
    """The 16 header bytes for a scene of `node_count` nodes and hash `scene_hash`."""
    return struct.pack("<4I", DRAPE_MAGIC, DRAPE_VERSION, node_count, scene_hash & 0xFFFFFFFF)


def parse_drape(data, node_count, scene_hash):
    """The positions (node_count x 4 float32) of a drape file when it matches the scene, else None
    (loadDrape's checks: size, magic, version, node count, scene hash)."""
    data = bytes(data)
    if len(data) != 16 + 16 * node_count or data[:16] != drape_header(node_count, scene_hash):
        return None
    return np.frombuffer(data, dtype="<f4", offset=16).reshape(node_count, 4).copy()


def encode_drape(solver, positions=None):
    """encodeDrape (settle.ts:8-13): the file bytes of `positions` (N x 4, default the solver's
    current positions)."""
    x = solver.state()[0] if positions is None else np.asarray(positions, np.float32).reshape(solver.N, 4)
    return drape_header(solver.N, solver.scene.hash()) + np.ascontiguousarray(x, dtype="<f4").tobytes()


def load_drape(solver, data):
    """loadDrape (settle.ts:16-22): upload the file's positions if it matches the solver's scene
    exactly (velocities kept); returns whether it did."""
    x = parse_drape(data, solver.N, solver.scene.hash())
    if x is None:
        return False
    solver.set_state(x, solver.state()[1])
    return True


def settle_drape(solver):
    """settleDrape (settle.ts:24-62) on the GPU: btd_settle_drape."""
    solver.settle_drape()
