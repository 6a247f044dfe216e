"""The numeric firewalls of the CUDA path, with the failures made on the host (no device fault):
non-finite directions are zeroed by the Newton update (step.wgsl:105-106), non-finite nodes are left
out of the line search's energy sums (energy.wgsl:89-218), a zero right-hand side stops PCG at once and a
non-positive curvature p . Ap stops it with a zero step (pcg.wgsl:82-85 safeDiv; the reference's pcg()
breaks there, newtonMultigrid.ts:553-556). In every case the solver's state stays finite and the next
substep runs normally.
"""
import numpy as np
import pytest

import btd_b200 as btd

pytestmark = pytest.mark.gpu


def staged():
    sc = btd.configs.hanging_patch(32, 0.15, seed=8)
    g = btd.GpuSolver(sc, btd.configs.solver_params(1 / 60, 4, 1e-6))
    g.substeps(2)
    g.encode_predict()
    g.encode_assemble(True)
    return sc, g


def test_non_finite_direction_is_zeroed_by_the_update():
    sc, g = staged()
    g.encode_pcg()
    d = g.read_vector("delta")
    bad = [5, 100, 700]
    d[bad[0], 0] = np.nan
    d[bad[1], 1] = np.inf
    d[bad[2], 2] = -np.inf
    g.write_vector("delta", d)
    dx0 = g.read_vector("dx")
    g.encode_apply(0)
    dx1 = g.read_vector("dx")
    assert np.isfinite(dx1).all()
    np.testing.assert_array_equal(dx1[bad], dx0[bad])
    moved = np.abs(dx1 - dx0).max(1) > 0
    assert moved.sum() > 0.9 * (sc.N - 32 - len(bad))
    g.substep()
    assert np.isfinite(g.x).all()


def test_line_search_leaves_non_finite_nodes_out():
    sc, g = staged()
    g.encode_pcg()
    d = g.read_vector("delta")
    e_ref, m_ref = g.encode_line_search()
    d[40, 0] = np.nan
    g.write_vector("delta", d)
    e, m = g.encode_line_search()
    assert np.isfinite(e).all() and np.isfinite(m).all()
    # one node's terms (and its neighbours' terms through it) fewer: the sums barely move
    assert np.abs(e - e_ref).max() <= 0.05 * np.abs(m_ref).max()
    assert g.counter_dict()["alpha"] in (0.0, 0.125, 0.25, 0.5, 1.0)


def test_zero_right_hand_side_stops_pcg_at_once():
    sc, g = staged()
    g.set_pcg(500, 1e-6)
    g.write_vector("B", np.zeros((sc.N, 3), np.float32))
    g.encode_pcg()
    d = g.read_vector("delta")
    c = g.counter_dict()
    assert np.isfinite(d).all() and np.abs(d).max() == 0.0
    assert c["pcg_last"] <= 1


class _DeviceArray:
    """A view of a library-owned device buffer for torch (__cuda_array_interface__)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (ptr, False), "version": 3}


def test_non_positive_curvature_stops_pcg_with_a_zero_step():
    import torch

    sc, g = staged()
    b = g.read_vector("B")
    ptr, nbytes = g.device_buffer("op", 0)
    assert nbytes == 15 * sc.N * 16
    # the fine operator replaced by -I (the smoother keeps the factors of the assembled operator, a
    # positive preconditioner), so the first direction has p . Ap < 0. Row floats 0..5 are the diagonal
    # block xx xy xz yy yz zz: plane 0 = (xx, xy, xz, yy), plane 1 = (yz, zz, ...).
    planes = torch.zeros((15, sc.N, 4), dtype=torch.float32, device="cuda")
    planes[0, :, 0] = -1.0
    planes[0, :, 3] = -1.0
    planes[1, :, 1] = -1.0
    g.synchronize()
    torch.as_tensor(_DeviceArray(ptr, (15, sc.N, 4)), device="cuda").copy_(planes)
    torch.cuda.synchronize()
    g.set_pcg(500, 1e-6)
    g.write_vector("B", b)
    g.set_operator_precision(False)  # PCG's operator: the fp32 rows written above
    g.encode_pcg()
    d = g.read_vector("delta")
    c = g.counter_dict()
    g.set_operator_precision(True)
    assert np.isfinite(d).all() and np.abs(d).max() == 0.0
    assert c["pcg_last"] == 1
    # the next substep assembles afresh and runs normally
    g.substep()
    assert np.isfinite(g.x).all()
