"""Regenerates drape_settled_oracle.npz: the oracle's (FP64 restatement of the reference's CPU solver)
settled drape of the default scene at the node subsample of drape_settled.npz, by settleDrape's
schedule (src/simulation/gpu/settle.ts:24-62) - GPU_DEFAULTS with 5 Newton and a fixed 2 PCG
iterations, history off, velocities cleared after every tenth of the first 360 of 420 substeps.
About two minutes on 8 host cores."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import conftest  # noqa: E402,F401  (registers the package)
import btd_b200 as btd  # noqa: E402
from oracle import Oracle  # noqa: E402

sc = btd.compile_scene(btd.default_spec())
o = Oracle(sc, h=1 / 120, newton_iterations=5, pcg_iterations=2, pcg_rel_tol=0.0, max_coarsest_nodes=400, coarse_sweeps=2,
           line_colors=3, lag_coarse=True, line_search=True, self_contact=True)
o.set_history(False)
for k in range(420):
    o.substep()
    if k % 10 == 9 and k < 360:
        o.set_state(o.x, np.zeros((sc.N, 3)))
idx = np.load(os.path.join(HERE, "drape_settled.npz"))["index"]
np.savez_compressed(os.path.join(HERE, "drape_settled_oracle.npz"), index=idx, position=o.x[idx])
print("wrote", len(idx), "oracle-settled nodes")
