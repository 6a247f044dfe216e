"""Detached-piece detection (src/simulation/gpu/topology.ts, state.wgsl), host side.

After ruptures (or a grip release) the active span graph is read back and flooded from its anchors
- the mounted nodes and, while gripping, the grip patch cores. Cloth nodes that no longer reach an
anchor become detached (x.w = 1, irreversible): they stay in the solve, but no grip holds them and
self-contact treats them as a lip. Every analysis also labels the detached pieces (connected through
active spans), each piece's nodes contiguous, for a rigid-mode correction of the solve.

Per node the packed bits are (state.wgsl:17-26): 1 the +u span is active, 2 the +v span is active,
4 detached (x.w > 0.5), 8 retired (x.w > 1.5).
"""
from collections import deque

import numpy as np

from .scene import SEG_BROKEN, SEG_EXISTS

NO_PIECE = 0xFFFFFFFF


class Lattice:
    """Row stride, column and row of every node (one lattice a layer)."""

    def __init__(self, layers, node_count):
        self.stride = np.zeros(node_count, np.int64)
        self.column = np.zeros(node_count, np.int64)
        self.row = np.zeros(node_count, np.int64)
        for L in layers:
            k = np.arange(L.nx * L.ny)
            self.stride[L.node_offset + k] = L.nx
            self.column[L.node_offset + k] = k % L.nx
            self.row[L.node_offset + k] = k // L.nx

    def neighbours(self, bits, n):
        """Nodes joined to n by an active span (topology.ts:201-205)."""
        nx = self.stride[n]
        out = []
        if bits[n] & 1:
            out.append(n + 1)
        if bits[n] & 2:
            out.append(n + nx)
        if self.column[n] > 0 and bits[n - 1] & 1:
            out.append(n - 1)
        if self.row[n] > 0 and bits[n - nx] & 2:
            out.append(n - nx)
        return out


def pack_bits(seg_flags, w):
    """pack (state.wgsl:17-26): the bits of every node from its two spans' flags and its x.w."""
    f = np.asarray(seg_flags, np.uint32).reshape(-1, 2)
    active = (f & (SEG_EXISTS | SEG_BROKEN)) == SEG_EXISTS
    w = np.asarray(w, np.float32)
    return (active[:, 0] * 1 | active[:, 1] * 2 | (w > 0.5) * 4 | (w > 1.5) * 8).astype(np.uint32)


def search(bits, pinned, anchors, lattice):
    """search (topology.ts:155-178): flood the active span graph from the mounts, then from each
    anchor not yet reached; the nodes neither reached nor detached before are freed. Returns the
    freed mask (uint32, 1 = freed)."""
    N = len(bits)
    vis = np.zeros(N, bool)
    queue = deque()

    def push(n):
        if vis[n] or bits[n] & 4:
            return
        vis[n] = True
        queue.append(n)

    def flood():
        while queue:
            for m in lattice.neighbours(bits, queue.popleft()):
                push(m)

    for n in np.nonzero(np.asarray(pinned))[0]:
        push(int(n))
    flood()
    for a in anchors:
        if vis[a] or bits[a] & 4:
            continue
        push(int(a))
        flood()
    return ((~vis) & ((bits & 4) == 0)).astype(np.uint32)


def label_pieces(bits, freed, lattice):
    """labelPieces (topology.ts:184-218): the detached pieces (detached and not retired, or freed
    now) connected through active spans, in order of their lowest node. Returns (piece_of, start,
    nodes, signature): piece_of[n] the piece of node n (NO_PIECE outside every piece), piece p's
    nodes nodes[start[p]:start[p + 1]], and the FNV-style signature that tells a changed labelling."""
    N = len(bits)
    detached = (((bits & 4) != 0) & ((bits & 8) == 0)) | (np.asarray(freed) == 1)
    piece_of = np.full(N, NO_PIECE, np.uint32)
    nodes = np.zeros(N, np.uint32)
    start = [0]
    tail = 0
    h = 2166136261
    for seed in range(N):
        if piece_of[seed] != NO_PIECE or not detached[seed]:
            continue
        p = len(start) - 1
        head = tail
        piece_of[seed] = p
        nodes[tail] = seed
        tail += 1
        while head < tail:
            n = int(nodes[head])
            head += 1
            for m in lattice.neighbours(bits, n):
                if piece_of[m] != NO_PIECE or not detached[m]:
                    continue
                piece_of[m] = p
                nodes[tail] = m
                tail += 1
        start.append(tail)
        h = ((((h ^ (seed + 1)) * 16777619) & 0xFFFFFFFF) ^ tail) & 0xFFFFFFFF
    h = (h ^ len(start)) & 0xFFFFFFFF
    return piece_of, np.array(start, np.uint32), nodes[:tail].copy(), h


def grip_core(nodes, weights):
    """The core of a grip patch (interaction.ts:231-237): its nodes held with weight 0.5 or more -
    the anchors that grip gives an analysis while it is held and not being let go."""
    return [int(n) for n, w in zip(nodes, weights) if w >= 0.5]


class Topology:
    """The analysis of topology.ts run to completion on a solver (GpuSolver, or anything with
    scene, state(), set_state() and segments()): read the spans and positions back, free the nodes
    no anchor reaches (x.w = 1 written back, velocities kept), label the detached pieces."""

    def __init__(self, solver):
        self.solver = solver
        self.scene = solver.scene
        self.lattice = Lattice(self.scene.layers, self.scene.N)
        self.freed_count = 0
        self.piece_of = np.full(self.scene.N, NO_PIECE, np.uint32)
        self.start = np.zeros(1, np.uint32)
        self.nodes = np.zeros(0, np.uint32)
        self.signature = 0

    def analyze(self, anchors=()):
        """One analysis with the given extra anchors (grip patch cores). Returns the number of nodes
        freed by it; the pieces are in piece_of / start / nodes, `changed` tells a new labelling."""
        x, v = self.solver.state()
        bits = pack_bits(self.solver.segments()["seg_flags"], x[:, 3])
        freed = search(bits, self.scene.pinned, anchors, self.lattice)
        count = int(freed.sum())
        if count:
            x = x.copy()
            x[(freed == 1) & (x[:, 3] <= 0.5), 3] = 1.0  # applyFreed (state.wgsl:28-35)
            self.solver.set_state(x, v)
        self.freed_count += count
        piece_of, start, nodes, sig = label_pieces(bits, freed, self.lattice)
        self.changed = sig != self.signature
        if self.changed:
            self.piece_of, self.start, self.nodes, self.signature = piece_of, start, nodes, sig
        return count
