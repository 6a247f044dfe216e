"""TEST INFRASTRUCTURE ONLY: trains the learned coarse space's network (configuration 4's learned coarse
correction, an extension with no counterpart in the reference) on the material the plain oracle solver
logs, and writes the weights (float32, the flat layout of oracle/learned.py) to
tests/golden/learned_coarse.npy. Each configuration weighs the same in the training minibatches.

Material: every coarsest-level call of plain MG-PCG (lagged hierarchy, rel-res 1e-6) on
  - configuration 0's hanging patch, 64 x 64 over 0.3 m, dt 1/60, 4 Newton: seeds 1 and 3, 6 substeps each;
  - configuration 1's yarn-damage patch, 128 x 128 with the bundle-[2, 2] region, the two edge grips
    moving apart at 0.2 m/s, dt 1/120: 6 substeps;
  - configuration 3's batch: its first 8 patches (seed 31) with a coarse level, each grip moving at its
    velocity, dt 1/60: 4 substeps each;
  - configuration 4's tearing patch scaled to 64 x 64 at its pitch (seed 41): 8 substeps.
Configuration 2 (the folded drop) is left out: its contact-engaged solves run PCG to the iteration cap,
which makes its material slow to log on the CPU.

Usage: python oracle/train_learned.py [--steps 1500] [--out tests/golden/learned_coarse.npy]
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
import conftest  # noqa: E402,F401  (registers the product package as btd_b200)
from btd_b200 import configs  # noqa: E402
from oracle import Oracle  # noqa: E402
from oracle import learned as L  # noqa: E402

MG = dict(max_coarsest_nodes=400, coarse_sweeps=2, line_colors=3, lag_coarse=True, line_search=True)


def newton_substeps(o, substeps, goals=None):
    """`substeps` substeps of 4 Newton iterations; goals(s) -> [(grip, goal)] before substep s (1-based)."""
    for s in range(1, substeps + 1):
        for g, goal in (goals(s) if goals else []):
            o.set_grip_goal(g, goal)
        o.predict()
        for _ in range(4):
            o.newton_step()
        o.finalize()
        o.update_damage()


def edge_grips(o, left, right, speed, h, k):
    x0 = o.x
    grips = []
    for nodes, sign in ((left, -1.0), (right, 1.0)):
        picked = int(nodes[len(nodes) // 2])
        o.add_grip(nodes, np.ones(len(nodes)), (x0[nodes] - x0[picked]).reshape(-1), x0[picked], k)
        grips.append((x0[picked].copy(), sign))
    return lambda s: [(g, a + np.array([sign * 0.5 * speed * s * h, 0, 0])) for g, (a, sign) in enumerate(grips)]


def material():
    runs = []
    c0 = configs.CONFIG0
    for seed in (1, 3):
        o = Oracle(configs.hanging_patch(64, 0.3, seed=seed), h=c0["h"], newton_iterations=4, pcg_iterations=500,
                   pcg_rel_tol=1e-6, **MG)
        runs.append(("config0 seed %d" % seed, o, 6, None))
    c1 = configs.CONFIG1
    sc, left, right = configs.config1()
    o = Oracle(sc, h=c1["h"], newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, **MG)
    runs.append(("config1", o, 6, edge_grips(o, left, right, c1["grip_speed"], c1["h"], c1["grip_stiffness"])))
    c3 = configs.CONFIG3
    picked = []
    for b, (sc, g) in enumerate(configs.config3(31, only=range(32))):
        if sc.N <= 400 or len(picked) == 8:
            continue
        o = Oracle(sc, h=c3["h"], newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, **MG)
        x0 = o.x
        p = g["picked"]
        o.add_grip(g["nodes"], g["weights"], (x0[g["nodes"]] - x0[p]).reshape(-1), x0[p], g["stiffness"])
        a, vel = x0[p].copy(), g["velocity"]
        picked.append(b)
        runs.append(("config3 patch %d" % b, o, 4, lambda s, a=a, vel=vel: [(0, a + vel * s * c3["h"])]))
    c4 = configs.CONFIG4
    sc, left, right = configs.config4(41, n=64, region=16)
    o = Oracle(sc, h=c4["h"], newton_iterations=4, pcg_iterations=500, pcg_rel_tol=1e-6, self_contact=True, **MG)
    runs.append(("config4 64x64", o, 8, edge_grips(o, left, right, c4["grip_speed"], c4["h"], c4["grip_stiffness"])))

    ops, calls, group = [], [], []
    for name, o, substeps, goals in runs:
        t = time.time()
        o.learned_log(True, 1 << 20)
        newton_substeps(o, substeps, goals)
        o_ops, o_calls = o.learned_samples()
        base = len(ops)
        ops += o_ops
        group += [name.split()[0]] * len(o_ops)
        calls += [(op + base, r, d) for op, r, d in o_calls]
        pairs = sum(len(o_ops[op][1]) for op, _, _ in o_calls)
        print(f"{name}: {len(o_ops)} operators, {len(o_calls)} calls, {pairs} node pairs, {time.time() - t:.1f} s",
              flush=True)
    return ops, calls, group


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "learned_coarse.npy"))
    args = ap.parse_args()
    ops, calls, group = material()
    pairs = sum(len(ops[op][1]) for op, _, _ in calls)
    print(f"total: {len(ops)} operators, {len(calls)} calls, {pairs} node pairs", flush=True)
    # each configuration weighs the same in the minibatches, whatever its number of operators
    count = {g: group.count(g) for g in set(group)}
    op_weights = [1.0 / count[g] for g in group]
    t = time.time()
    w, hist = L.train(ops, calls, steps=args.steps, batch_ops=6, op_weights=op_weights)
    print("loss every 50 steps:", " ".join(f"{h:.3f}" for h in hist), f"({time.time() - t:.1f} s)")
    np.save(args.out, w.astype(np.float32))
    print("wrote", args.out)


if __name__ == "__main__":
    main()
