"""Self-contact contracts of the reference (tests/gpu/interaction.ts:185-250) on the CUDA path, on
the shipped 182 x 115 scene with every node retired but a face and a node placed by hand: a Newton
update that would drive a node and a face through each other leaves them apart (the directional and
reciprocal bounds), a node predicted through a face at 2.4 m/s is stopped by the face its path
crosses, and the lattice exclusion window skips the node's own cloth but not a lip across a tear.
Plus a dynamic check: a sheet dropped onto a second sheet lies on it without passing through.
"""
import numpy as np
import pytest

import btd_b200 as btd

pytestmark = pytest.mark.gpu

PU, PV = 0.00342, 0.00348


@pytest.fixture(scope="module")
def scene():
    sc = btd.compile_scene(btd.default_spec())
    gpu = btd.GpuSolver(sc, btd.default_params(line_search=0))
    return sc, gpu


def placed_state(sc, placed):
    x = np.zeros((sc.N, 4), np.float32)
    x[:, :3] = sc.position.reshape(-1, 3)
    x[:, 3] = 2.0  # retired: out of the scene
    for n, p in placed.items():
        x[n, :3] = p
        x[n, 3] = 0.0
    return x


def apply(gpu, sc, placed, delta, velocity=None, seg_flags=None):
    """One full Newton update of `delta` after detection at the (predicted) iterate; returns dx."""
    x = placed_state(sc, placed)
    v = np.zeros((sc.N, 3))
    for n, q in (velocity or {}).items():
        v[n] = q
    gpu.set_state(x, v)
    if seg_flags is not None:
        gpu.set_segments(seg_flags=seg_flags)
    gpu.encode_predict()
    d = np.zeros((sc.N, 3))
    for n, q in delta.items():
        d[n] = q
    gpu.write_vector("delta", d)
    gpu.encode_line_search()
    gpu.encode_apply(0)
    return gpu.read_vector("dx")


def test_contact_contracts(scene):
    sc, gpu = scene
    nx = sc.nx
    f = 20 * nx + 20
    cs = [f, f + 1, f + nx, f + nx + 1]
    node = 50 * nx + 50
    face = {c: (((q % 2) - 0.5) * PU, ((q // 2) - 0.5) * PV, 0.0) for q, c in enumerate(cs)}
    above = dict(face)
    above[node] = (0.0, 0.0, 0.0015)

    def gap(dx):
        return 0.0015 + dx[node, 2] - np.mean([dx[c, 2] for c in cs])

    cases = {
        "a node driven through a still face": {node: (0, 0, -0.002)},
        "a face driven through a still node": {c: (0, 0, 0.003) for c in cs},
        "node and face driven through each other": {node: (0, 0, -0.002), **{c: (0, 0, 0.002) for c in cs}},
    }
    for name, delta in cases.items():
        g = gap(apply(gpu, sc, above, delta))
        assert g > 0.3e-3, (name, g)
    # 2.4 m/s through the face in one substep: the predictor itself is the iterate (no direction)
    g = gap(apply(gpu, sc, above, {}, velocity={node: (0, 0, -2.4)}))
    assert g > 0.3e-3, ("a fast node is stopped by the face its path crosses", g)

    # a lip three rows above the face is linked to it through its column while that holds, and is
    # another lip once the column is cut
    lip, link = f + 3 * nx, f + 2 * nx
    torn = dict(face)
    torn[lip] = (0.0, 0.0, 0.0015)
    torn[link] = (0.01, 0.0, 0.0)
    segs = gpu.segments()["seg_flags"].copy()
    linked = apply(gpu, sc, torn, {lip: (0, 0, -0.002)}, seg_flags=segs)
    cut = segs.copy()
    cut[2 * (f + nx) + 1] |= 2
    severed = apply(gpu, sc, torn, {lip: (0, 0, -0.002)}, seg_flags=cut)
    gpu.set_segments(seg_flags=segs)
    assert 0.0015 + linked[lip, 2] < 0, "its own linked cloth in the exclusion window is not a contact"
    assert 0.0015 + severed[lip, 2] > 0.3e-3, "a lip across a tear in the exclusion window is"


def test_sheet_dropped_on_a_sheet_stays_above_it():
    """Two 0.15 m sheets of the shipped denim lattice, the upper one 4 mm above the lower, whose
    edges are mounted: the upper falls onto it and rests on it, every interior node at least the
    hard core (0.3 mm) above the node under it, with self-contact on and gravity only."""
    m = btd.material_preset(0)
    specs = [btd.layer_spec(m, 0.15, 0.15, bundle=(9, 6), z=z, seed=3) for z in (0.0, 0.004)]
    sc = btd.compile_scene(specs)
    L0 = sc.layers[0]
    nx, ny = L0.nx, L0.ny
    i = np.arange(L0.node_count) % nx
    j = np.arange(L0.node_count) // nx
    sc.pinned[:] = 0
    sc.pinned[:L0.node_count] = ((i == 0) | (j == 0) | (i == nx - 1) | (j == ny - 1)).astype(np.uint8)
    gpu = btd.GpuSolver(sc, btd.default_params(newton_iterations=3, newton_max=3, pcg_iterations=20))
    n = L0.node_count
    worst = np.inf
    for _ in range(8):
        gpu.substeps(15)
        x = gpu.x
        assert np.isfinite(x).all()
        gap = (x[n:, 2] - x[:n, 2]).reshape(ny, nx)[2:-2, 2:-2]
        worst = min(worst, float(gap.min()))
    assert worst > 0.3e-3, worst
    assert worst < 2e-3, "the upper sheet must have come down onto the lower one"
    v = gpu.state()[1]
    assert np.abs(v[n:, :3]).max() < 0.05, np.abs(v[n:, :3]).max()
