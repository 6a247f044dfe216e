"""Precision study on the oracle: coarse multigrid levels stored in BF16 (the precision ladder's "coarse
levels may be stored in BF16"; no counterpart in the reference, whose GPU levels are FP32). Each coarse
level's operator is rounded to BF16 as it is built and the next level is built from the rounded one.
Rounding the 24 coupling blocks and keeping the diagonal block (about half the coarse-row bytes) still
solves every Newton system to rel-res 1e-6 at a few percent more PCG iterations on the lagged
hierarchy; the plain configuration's 64 x 64 hanging patch, seed 2, 2 substeps."""
import numpy as np

from btd_b200 import configs
from oracle import Oracle

P = dict(h=1 / 60, newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, max_coarsest_nodes=400, coarse_sweeps=2,
         line_colors=3, lag_coarse=True, line_search=True)


def run(o, substeps):
    its, rel = [], []
    for _ in range(substeps):
        o.predict()
        for _ in range(4):
            r = o.newton_step()
            its.append(r["pcg_iterations"])
            rel.append(r["rel_residual"])
        o.finalize()
        o.update_damage()
    return np.mean(its), max(rel)


def test_bf16_coupling_blocks_cost_few_iterations():
    sc = configs.hanging_patch(64, 0.3, seed=2)
    i32, r32 = run(Oracle(sc, **P), 2)
    i16, r16 = run(Oracle(sc, **P, coarse_bf16=2), 2)
    print(f"PCG iterations per Newton step: coarse levels FP64 {i32:.2f}, BF16 couplings {i16:.2f}")
    assert r32 <= 1e-6 and r16 <= 1e-6
    assert i16 <= 1.1 * i32


def test_fp32_rows_study_modes():
    """The operator as FP32 storage would hold it (fp32_rows; the study behind PCG's FP64 operator):
    on the hanging patch (no loose material) every mode still solves each Newton system to rel-res
    1e-6, and keeping PCG's operator exact while the V-cycle takes FP32-rounded rows (mode 3) changes
    the iteration count by at most one a Newton step against all-FP64 rows."""
    sc = configs.hanging_patch(64, 0.3, seed=2)
    i64, r64 = run(Oracle(sc, **P), 1)
    out = {}
    for mode in (1, 2, 3, 11, 13):
        out[mode] = run(Oracle(sc, **P, fp32_rows=mode), 1)
    for mode, (i, r) in out.items():
        assert r <= 1e-6, (mode, r)
    assert abs(out[3][0] - i64) <= 1.0, (out[3][0], i64)
    assert abs(out[13][0] - i64) <= 1.0, (out[13][0], i64)
