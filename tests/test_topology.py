"""Detached-piece detection (src/simulation/gpu/topology.ts, state.wgsl) on the host: nodes that no
active span path joins to a mount or a grip anchor are freed, detached pieces are labelled through
active spans with each piece's nodes contiguous, and an analysis writes x.w = 1 back to the solver
for the nodes it frees (velocities kept)."""
from types import SimpleNamespace

import numpy as np

import btd_b200 as btd
from btd_b200.topology import NO_PIECE, Lattice, Topology, label_pieces, pack_bits, search

SEG_EXISTS = btd.SEG_EXISTS
SEG_BROKEN = btd.SEG_BROKEN


def lattice(layers):
    """Layers of (nx, ny, pinned top row?); every span exists."""
    infos, pinned, off = [], [], 0
    for nx, ny, pin in layers:
        infos.append(SimpleNamespace(nx=nx, ny=ny, node_offset=off, node_count=nx * ny))
        p = np.zeros((ny, nx), np.uint8)
        if pin:
            p[ny - 1, :] = 1
        pinned.append(p.reshape(-1))
        off += nx * ny
    flags = np.full(2 * off, SEG_EXISTS, np.uint32)
    for L in infos:  # no +u span off the row end, no +v span off the top
        k = np.arange(L.node_count)
        flags[2 * (L.node_offset + k[k % L.nx == L.nx - 1])] = 0
        flags[2 * (L.node_offset + k[k // L.nx == L.ny - 1]) + 1] = 0
    return infos, np.concatenate(pinned), flags


def cut_island(flags, nx, i0, i1, j0, j1, off=0):
    """Break every span joining the block [i0, i1] x [j0, j1] to the rest of its layer."""
    node = lambda i, j: off + j * nx + i
    for j in range(j0, j1 + 1):
        flags[2 * node(i0 - 1, j)] |= SEG_BROKEN
        flags[2 * node(i1, j)] |= SEG_BROKEN
    for i in range(i0, i1 + 1):
        flags[2 * node(i, j0 - 1) + 1] |= SEG_BROKEN
        flags[2 * node(i, j1) + 1] |= SEG_BROKEN
    return {node(i, j) for i in range(i0, i1 + 1) for j in range(j0, j1 + 1)}


def analyse(infos, pinned, flags, w, anchors=()):
    lat = Lattice(infos, len(pinned))
    bits = pack_bits(flags, w)
    freed = search(bits, pinned, anchors, lat)
    return bits, freed, label_pieces(bits, freed, lat)


def test_an_island_cut_loose_is_freed_and_is_one_piece():
    infos, pinned, flags = lattice([(12, 10, True)])
    island = cut_island(flags, 12, 4, 6, 3, 5)
    bits, freed, (piece_of, start, nodes, sig) = analyse(infos, pinned, flags, np.zeros(120))
    assert set(np.nonzero(freed)[0]) == island
    assert start.tolist() == [0, 9] and set(nodes.tolist()) == island
    assert all(piece_of[n] == 0 for n in island) and (piece_of == NO_PIECE).sum() == 120 - 9


def test_a_grip_anchor_keeps_what_it_holds():
    infos, pinned, flags = lattice([(12, 10, True)])
    island = cut_island(flags, 12, 4, 6, 3, 5)
    _, freed, (_, start, _, _) = analyse(infos, pinned, flags, np.zeros(120), anchors=[min(island)])
    assert not freed.any() and start.tolist() == [0]


def test_detached_and_retired_nodes():
    infos, pinned, flags = lattice([(12, 10, True)])
    island = sorted(cut_island(flags, 12, 4, 6, 3, 5))
    w = np.zeros(120)
    w[island] = 1.0  # detached by an earlier analysis: labelled, not freed again
    _, freed, (_, start, nodes, _) = analyse(infos, pinned, flags, w)
    assert not freed.any() and start.tolist() == [0, 9]
    w[island[0]] = 2.0  # retired: out of every piece
    _, _, (piece_of, start, _, _) = analyse(infos, pinned, flags, w)
    assert piece_of[island[0]] == NO_PIECE and start.tolist() == [0, 8]


def test_two_islands_two_pieces_in_node_order_and_a_new_signature():
    infos, pinned, flags = lattice([(12, 10, True)])
    a = cut_island(flags, 12, 1, 2, 1, 2)
    _, _, (_, _, _, sig1) = analyse(infos, pinned, flags, np.zeros(120))
    b = cut_island(flags, 12, 7, 9, 4, 6)
    _, freed, (piece_of, start, nodes, sig2) = analyse(infos, pinned, flags, np.zeros(120))
    assert set(np.nonzero(freed)[0]) == a | b
    assert start.tolist() == [0, 4, 13]
    assert set(nodes[:4].tolist()) == a and set(nodes[4:].tolist()) == b
    assert sig1 != sig2


def test_an_unmounted_layer_is_freed_whole():
    infos, pinned, flags = lattice([(8, 6, True), (5, 4, False)])
    _, freed, (piece_of, start, nodes, _) = analyse(infos, pinned, flags, np.zeros(68))
    assert np.array_equal(np.nonzero(freed)[0], np.arange(48, 68))
    assert start.tolist() == [0, 20] and sorted(nodes.tolist()) == list(range(48, 68))


def test_an_analysis_writes_detached_nodes_back_to_the_solver():
    infos, pinned, flags = lattice([(12, 10, True)])
    island = cut_island(flags, 12, 4, 6, 3, 5)

    class FakeSolver:
        def __init__(self):
            self.scene = SimpleNamespace(layers=infos, N=120, pinned=pinned)
            self.x = np.zeros((120, 4), np.float32)
            self.v = np.ones((120, 4), np.float32)

        def state(self):
            return self.x.copy(), self.v.copy()

        def set_state(self, x, v):
            self.x, self.v = np.array(x, np.float32), np.array(v, np.float32)

        def segments(self):
            return {"seg_flags": flags}

    s = FakeSolver()
    topo = Topology(s)
    assert topo.analyze() == 9 and topo.changed
    assert set(np.nonzero(s.x[:, 3] == 1.0)[0]) == island and (s.v == 1).all()
    assert topo.analyze() == 0 and not topo.changed  # already detached: the same pieces
    assert topo.start.tolist() == [0, 9]


def test_two_claw_centre_piece_classification_on_the_product_scene():
    """tests/gpu/twohand-topology.ts (classification checks) on the host analysis: on the default
    scene, a 9 x 3 strip left in the scene (everything else retired) with only its own spans, held by
    two claws at its ends (each with a weak rim entry on the centre, which is no anchor); the centre
    three columns are cut free on both sides in either order or at once: after one cut the centre
    stays held by the other hand, after both it is detached as one piece and the held sides are kept;
    with both hands let go the whole strip detaches."""
    from btd_b200.topology import grip_core

    sc = btd.compile_scene(btd.default_spec())
    nx = sc.layers[0].nx
    node = lambda i, j: (50 + j) * nx + 50 + i
    strip = [node(k % 9, k // 9) for k in range(27)]
    centre = [n for n in strip if 53 <= n % nx <= 55]
    lat = Lattice(sc.layers, sc.N)
    w = np.full(sc.N, 2.0)
    w[strip] = 0.0

    def setup():
        flags = sc.seg_flags.astype(np.uint32) | SEG_BROKEN
        for j in range(3):
            for i in range(9):
                if i < 8:
                    flags[2 * node(i, j)] = SEG_EXISTS
                if j < 2:
                    flags[2 * node(i, j) + 1] = SEG_EXISTS
        return flags, w.copy()

    def cut(flags, side):
        for j in range(3):
            flags[2 * node(2 if side == 0 else 5, j)] |= SEG_BROKEN

    cores = [grip_core([node(0 if slot == 0 else 8, 1), centre[slot]], [1, 0.25]) for slot in (0, 1)]
    assert cores == [[node(0, 1)], [node(8, 1)]]  # the rim entries are no anchors

    def analyze(flags, ww, anchors):
        bits = pack_bits(flags, ww)
        freed = search(bits, sc.pinned, anchors, lat)
        ww[(freed == 1) & (ww <= 0.5)] = 1.0
        return label_pieces(bits, freed, lat)

    def verify(ww, pieces):
        piece_of = pieces[0]
        assert all(ww[n] == (1.0 if n in centre else 0.0) for n in strip)
        assert piece_of[centre[0]] != NO_PIECE and all(piece_of[n] == piece_of[centre[0]] for n in centre)
        assert all(piece_of[n] == NO_PIECE for n in strip if n not in centre)

    anchors = cores[0] + cores[1]
    for first in (0, 1):
        flags, ww = setup()
        analyze(flags, ww, anchors)
        cut(flags, first)
        analyze(flags, ww, anchors)
        assert all(ww[n] == 0.0 for n in centre)  # still held by the other hand
        cut(flags, 1 - first)
        verify(ww, analyze(flags, ww, anchors))
    flags, ww = setup()
    analyze(flags, ww, anchors)
    cut(flags, 0)
    cut(flags, 1)
    verify(ww, analyze(flags, ww, anchors))
    flags, ww = setup()
    analyze(flags, ww, anchors)
    analyze(flags, ww, [])  # both hands let go
    assert all(ww[n] == 1.0 for n in strip)
