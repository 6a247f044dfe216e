#!/usr/bin/env python
"""Benchmark: Newton steps/s of the implicit cloth solve at relative residual 1e-6 on B200.

A step is one substep of the workload: predictor, 4 projected-Newton iterations each solved by
Galerkin-multigrid PCG to relative residual 1e-6, line search, commit, damage field and crossing
slip. `value` is Newton iterations per second over all ranks, timed with CUDA events on the
solver's stream with a cold L2 before every step (a 256 MiB buffer is rewritten between steps,
outside the timed events); `e2e` is the same metric through the public C ABI from pinned host
buffers (state in, state out every step). One patch does not shard: with --gpus N each rank runs
an independent replica (weak scaling) and the time is the max over ranks.

--impl reference times the reference's CPU solver (its FP64 restatement: the reference is
TypeScript and has no runnable CPU path here) on the host cores, on the same workload and metric.
"""
import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "break-that-denim_b200")
METRIC = "Newton steps/s at rel-res 1e-6: learned-precond vs plain MG-PCG, 1 B200"
FALLBACK_HBM_GBS = 6650.0

# workloads: (lattice side, patch size m, dt, Newton iterations, relative residual)
WORKLOADS = {
    "hanging-256": dict(n=256, size=0.6, h=1 / 60, newton=4, rel=1e-6,
                        desc="256x256-vertex hanging shell patch (0.6 m, config-0 material and schedule: top row pinned, "
                             "dt 1/60, 4 projected-Newton, MG-PCG to rel-res 1e-6, no contact), seeded N(0,1e-4) jitter"),
    "config0-64": dict(n=64, size=0.3, h=1 / 60, newton=4, rel=1e-6,
                       desc="64x64-vertex hanging shell patch (0.3 m), dt 1/60, 4 projected-Newton, 3-level MG-PCG to rel-res 1e-6"),
}
WORKLOADS["config2-256"] = dict(n=256, size=0.6, h=1 / 60, newton=4, rel=1e-6, contact=True,
                                desc="configuration 2: a free 256x256-vertex sheet (0.6 m, config-0 material) folded about 1-3 seeded "
                                     "parallel lines, dropped from 0.3 m onto the floor with self-contact on (SELF_CONTACT law); "
                                     "dt 1/60, 4 projected-Newton, MG-PCG to rel-res 1e-6; timed from the drop")
BATCH = "batch-512"
WORKLOADS[BATCH] = dict(n=None, size=None, h=1 / 60, newton=4, rel=1e-6,
                        desc="512 independent hanging patches (the batched configuration): sides uniform in [16, 128] nodes at "
                             "the config-0 pitch, stiffness factors U(0.5, 2), central yarn regions of 0-30 % with lognormal "
                             "break strains, one edge grip each pulled at 0.05-0.2 m/s, all seeded; dt 1/60, 4 projected-Newton, "
                             "MG-PCG to rel-res 1e-6; sharded across GPUs by estimated bytes")
PRODUCT = "product-21k"
WORKLOADS[PRODUCT] = dict(n=None, size=None, h=1 / 120, newton=2, rel=0.0, pcg=2, contact=True, product=True,
                          desc="the product scene: the default 182 x 115 denim panel (20,930 nodes, scene.ts defaults), "
                               "settled by the drape schedule (settle.ts), then hanging at the shipped solver settings "
                               "(GPU_DEFAULTS: h 1/120, 2 Newton x 2 PCG iterations - fixed counts, no residual stop - "
                               "self-contact on)")
METRIC_PRODUCT = "Newton steps/s of the product scene's substep at the shipped settings (2 Newton x 2 PCG, self-contact)"
# the reference's published substep times on this scene (Apple M5, WebGPU): 2 Newton x 2 PCG 6.9 ms plus
# 0.6 ms of self-contact (docs/decisions/2026-10-10-feedback-round2.md:11-14)
PRODUCT_PUBLISHED_MS = 6.9 + 0.6
DEFAULT_WORKLOAD = "hanging-256"
HIST_EDGES = [0, 5, 10, 15, 20, 25, 30, 40, 60, 100, 500]
MG = dict(max_coarsest_nodes=400, coarse_sweeps=2, line_colors=3, lag_coarse=True, line_search=True)


def package():
    if "btd_b200" in sys.modules:
        return sys.modules["btd_b200"]
    spec = importlib.util.spec_from_file_location("btd_b200", os.path.join(PKG, "__init__.py"), submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["btd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def build_scene(btd, w):
    if w.get("product"):
        return btd.compile_scene(btd.default_spec())
    if w.get("contact"):
        return btd.configs.config2()
    return btd.configs.hanging_patch(w["n"], w["size"], seed=1)


def solver_params(btd, w):
    if w.get("product"):
        return btd.default_params()
    return btd.configs.solver_params(w["h"], w["newton"], w["rel"], self_contact=1 if w.get("contact") else 0)


# Multigrid settings measured beside the default one: the Galerkin hierarchy rebuilt at every Newton
# iteration instead of lagged from the first (the reference lags it, newtonMultigrid.ts:579, for its
# fixed two PCG iterations), and that coarsened down to at most 30 nodes instead of 400. On the oracle
# they take the PCG iterations per Newton step of the 256 x 256 hanging patch from 37 to 20 and 13,
# and of the folded drop with self-contact at 64 x 64 from 94 to 59 and 41; each extra level costs
# its launches in every V-cycle, so the device decides between them.
MG_VARIANTS = (dict(lag_coarse=0), dict(lag_coarse=0, max_coarsest_nodes=30))


def measure_variant(btd, w, sc, steps, warmup, settings):
    """The workload's substeps with other multigrid settings: Newton steps/s from the device-timed
    substep graph (L2 flushed before each, as the default's), PCG iterations per Newton step and the
    level count."""
    p = solver_params(btd, w)
    for k, v in settings.items():
        setattr(p, k, v)
    g = btd.GpuSolver(sc, p)
    if w.get("contact"):
        g.set_floor(btd.configs.CONFIG2["floor"])
    try:
        for _ in range(warmup):
            g.substep()
        g.synchronize()
        g.clear_counters()
        ms = g.profile_stage("substep", reps=steps, flush=True)
        c = g.counter_dict()
        return {"settings": dict(settings), "levels": g.level_count(),
                "value": c["newton"] / (ms * steps / 1e3), "unit": "Newton steps/s", "ms_per_step": ms,
                "pcg_iterations_per_newton": c["pcg_total"] / max(1, c["newton"])}
    finally:
        g.close()


def workload_oracle(btd, w, threads=0):
    """The oracle configured as the workload's solve (PCG to the relative residual, or the fixed count)."""
    sys.path.insert(0, ROOT)
    from oracle import Oracle

    sc = build_scene(btd, w)
    o = Oracle(sc, h=w["h"], newton_iterations=w["newton"], pcg_iterations=w.get("pcg", 500), pcg_rel_tol=w["rel"],
               threads=threads, self_contact=bool(w.get("contact")), **MG)
    if w.get("contact") and not w.get("product"):
        o.set_floor(btd.configs.CONFIG2["floor"])
    return o


def peaks():
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 4 + k and r[4 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_sample(btd, w, substeps, threads=0):
    """The oracle (the reference's CPU solver restated, FP64, OpenMP) on `substeps` substeps."""
    o = workload_oracle(btd, w, threads)
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    if w.get("contact") and not w.get("product"):
        # bounded sample: one Newton iteration with the contacts engaged - the first substep's second
        # (its prediction and first iteration, untimed, converge in ~50 PCG iterations; the later
        # ones, ~30 s each on 8 host cores, are the representative work)
        o.predict()
        o.newton_step()
        t = time.perf_counter()
        o.newton_step()
        dt = time.perf_counter() - t
        return 1.0 / dt, dt, cores
    t = time.perf_counter()
    for _ in range(substeps):
        o.substep()
    dt = time.perf_counter() - t
    return substeps * w["newton"] / dt, dt, cores


def across_ranks(dist, values, op="max", device="cuda"):
    """Every rank's `values` combined over the ranks (the max of the device times: the job takes as
    long as its slowest rank; the sum of counts); unchanged on a single process."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def cpu_sample_single_core(btd, w):
    """The oracle on one host thread, bounded: the first substep's prediction and first Newton
    iteration of the workload (a whole substep takes tens of seconds on one core at 256 x 256)."""
    o = workload_oracle(btd, w, threads=1)
    t = time.perf_counter()
    o.predict()
    o.newton_step()
    dt = time.perf_counter() - t
    return 1.0 / dt, dt


def batch_cpu_sample(btd, patches=2):
    """The oracle on the first `patches` patches of the batch, one substep each, grips held."""
    sys.path.insert(0, ROOT)
    from oracle import Oracle

    c = btd.configs.CONFIG3
    dt = 0.0
    newton = 0
    for sc, g in btd.configs.config3(only=list(range(patches))):
        o = Oracle(sc, h=c["h"], newton_iterations=c["newton_iterations"], pcg_iterations=500, pcg_rel_tol=c["pcg_rel_tol"], **MG)
        x = o.x
        nodes = np.asarray(g["nodes"])
        anchor = x[g["picked"]].copy()
        o.add_grip(nodes, np.asarray(g["weights"], np.float64), (x[nodes] - x[g["picked"]]).reshape(-1), anchor, g["stiffness"])
        o.set_grip_goal(0, anchor + c["h"] * g["velocity"])
        t = time.perf_counter()
        o.substep()
        dt += time.perf_counter() - t
        newton += c["newton_iterations"]
    return newton / dt, dt, os.cpu_count() or 1


def run_reference(args, w, rank):
    if rank != 0:
        return
    btd = package()
    if args.workload == BATCH:
        value, dt, cores = batch_cpu_sample(btd, max(1, args.steps))
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Newton steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / max(1, args.steps), "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": args.workload, "description": w["desc"]},
                "cpu_baseline": {"value": value, "unit": "Newton steps/s", "cores": cores, "kind": "port",
                                 "sample": f"one substep of each of the first {max(1, args.steps)} patches"},
                "e2e": {"value": value, "unit": "Newton steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    for _ in range(args.warmup):
        pass  # the CPU solver has no warm-up state worth timing; warm-up steps run inside the sample below
    steps = max(1, args.steps)
    value, dt, cores = cpu_sample(btd, w, steps)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Newton steps/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": {"workload": args.workload, "description": w["desc"]},
            "cpu_baseline": {"value": value, "unit": "Newton steps/s", "cores": cores, "kind": "port",
                             "sample": f"{steps} substeps x {w['newton']} Newton of the workload from its initial state"},
            "e2e": {"value": value, "unit": "Newton steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_batch(args, w, rank, world, local, dist):
    """The batched configuration: this rank's shard of the patches (by estimated bytes), each a solver
    on its own stream and graph, driven one substep of every patch at a time (grip targets set, then
    btd_batch_substeps); the per-patch Newton and PCG counts gathered to rank 0 at the end."""
    import torch

    btd = package()
    c = btd.configs.CONFIG3
    sides = btd.configs.config3_sides(count=args.patches)
    mine = btd.configs.shard_patches(sides, world)[rank]
    t_setup = time.perf_counter()
    patches = btd.configs.config3(count=args.patches, only=mine)
    params = btd.configs.solver_params(c["h"], c["newton_iterations"], c["pcg_rel_tol"])
    solvers, anchors = [], []
    for sc, g in patches:
        s = btd.GpuSolver(sc, params)
        a = s.x[g["picked"]].astype(np.float32)
        s.attach_patch(0, g["picked"], g["nodes"], g["weights"], a, g["stiffness"], max_lead=g["max_lead"])
        solvers.append(s)
        anchors.append(a)
    t_setup = time.perf_counter() - t_setup
    step = [0]

    def advance():
        step[0] += 1
        for s, a, (_, g) in zip(solvers, anchors, patches):
            s.set_target((a + step[0] * c["h"] * g["velocity"]).astype(np.float32))
        btd.batch_substeps(solvers, 1)

    def barrier():
        if dist is not None:
            dist.barrier()
        for s in solvers:
            s.synchronize()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        advance()
    barrier()
    for s in solvers:
        s.clear_counters()
    idx = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        idx = vis.split(",")[local]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(idx) as clocks:
        ev0.record()
        for _ in range(args.steps):
            advance()
        for s in solvers:
            s.synchronize()
        torch.cuda.synchronize()
        ev1.record()
        ev1.synchronize()
    t_dev = ev0.elapsed_time(ev1) / 1e3
    stats = {}
    for b, s in zip(mine, solvers):
        cd = s.counter_dict()
        stats[b] = (int(cd["newton"]), int(cd["pcg_total"]), sides[b])
    launches = sum(s.launch_count(args.steps, stats[b][0], stats[b][1]) for b, s in zip(mine, solvers))

    # end to end through the C ABI: every patch's state in from pinned host buffers, the batch
    # substep, every state out
    lib_check = btd._abi.check
    host = []
    for s in solvers:
        xh = torch.empty((s.N, 4), dtype=torch.float32, pin_memory=True)
        vh = torch.empty((s.N, 4), dtype=torch.float32, pin_memory=True)
        lib_check("btd_get_state", s._h, xh.data_ptr(), vh.data_ptr())
        host.append((xh, vh))
    for s in solvers:
        s.clear_counters()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for s, (xh, vh) in zip(solvers, host):
            lib_check("btd_set_state", s._h, xh.data_ptr(), vh.data_ptr())
        btd.batch_substeps(solvers, 1)
        for s, (xh, vh) in zip(solvers, host):
            lib_check("btd_get_state", s._h, xh.data_ptr(), vh.data_ptr())
    barrier()
    t_e2e = time.perf_counter() - t0
    newton_e2e = sum(s.counter_dict()["newton"] for s in solvers)
    bytes_step = sum(2 * 16 * s.N for s in solvers)

    gathered = [stats]
    if dist is not None:
        t_dev, t_e2e = across_ranks(dist, [t_dev, t_e2e], "max")
        newton_e2e, bytes_step, launches = across_ranks(dist, [newton_e2e, bytes_step, launches], "sum")
        gathered = [None] * world
        dist.all_gather_object(gathered, stats)
    for s in solvers:
        s.close()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    merged = {}
    for d in gathered:
        merged.update(d)
    newton = sum(v[0] for v in merged.values())
    per = np.array([v[1] / max(1, v[0]) for v in merged.values()])
    hist, _ = np.histogram(per, bins=HIST_EDGES)
    line = {
        "metric": METRIC, "value": newton / t_dev, "unit": "Newton steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": w["desc"], "patches": len(merged),
                   "nodes": int(sum(v[2] ** 2 for v in merged.values())),
                   "substeps_per_s": len(merged) * args.steps / t_dev,
                   "pcg_iterations_per_newton": float(per.mean()),
                   "pcg_iterations_per_newton_histogram": {"edges": HIST_EDGES, "patches": hist.tolist()},
                   "l2": "inputs larger than L2 (every patch's state and operators, about 1.5 GB)",
                   "setup_s": t_setup, "parallelism": f"patches sharded x{world}"},
        "e2e": {"value": newton_e2e / t_e2e, "unit": "Newton steps/s", "h2d_bytes_per_step": int(bytes_step),
                "d2h_bytes_per_step": int(bytes_step)},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        v_cpu, dt_cpu, cores = batch_cpu_sample(btd)
        line["cpu_baseline"] = {"value": v_cpu, "unit": "Newton steps/s", "cores": cores, "kind": "port",
                                "sample": f"one substep of each of the first 2 patches, {dt_cpu:.1f} s"}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    # the batched workload runs one stream a patch: let up to 32 of them reach the GPU's hardware
    # queues at once (the default is 8); read when CUDA initialises, so set before it does
    if BATCH in sys.argv:
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--eager", action="store_true", help="launch kernel by kernel (for per-kernel profilers)")
    ap.add_argument("--patches", type=int, default=512, help="patches of the batch workload")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    w = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, w, rank)
        return

    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    if args.workload == BATCH:
        run_batch(args, w, rank, world, local, dist)
        return
    btd = package()
    sc = build_scene(btd, w)
    params = solver_params(btd, w)
    gpu = btd.GpuSolver(sc, params)
    if w.get("product"):
        gpu.settle_drape()  # the product starts from its settled drape (drape.bin / settleDrape)
    elif w.get("contact"):
        gpu.set_floor(btd.configs.CONFIG2["floor"])
    if args.eager:
        gpu.set_graph_mode(False)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        gpu.synchronize()

    # warm-up (captures the substep graph, fills caches)
    for _ in range(args.warmup):
        gpu.substep()
    gpu.synchronize()
    gpu.clear_counters()

    # ---- device-timed region: K substeps, cold L2 before each (flush outside the events)
    barrier()
    idx = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        idx = vis.split(",")[local]
    with ClockSampler(idx) as clocks:
        ms_step = gpu.profile_stage("substep", reps=args.steps, flush=True)
        barrier()
    c = gpu.counter_dict()
    newton_total = c["newton"]
    pcg_total = c["pcg_total"]
    t_dev = ms_step * args.steps / 1e3
    if dist is not None:
        t_dev = across_ranks(dist, [t_dev], "max")[0]
    value = world * newton_total / t_dev
    launches = gpu.launch_count(args.steps, newton_total, pcg_total)

    # ---- end to end through the C ABI from pinned host buffers: state in, substep, state out
    N = sc.N
    xh = torch.empty((N, 4), dtype=torch.float32, pin_memory=True)
    vh = torch.empty((N, 4), dtype=torch.float32, pin_memory=True)
    lib = btd._abi.lib()
    h = gpu._h
    btd._abi.check("btd_get_state", h, xh.data_ptr(), vh.data_ptr())
    gpu.clear_counters()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        btd._abi.check("btd_set_state", h, xh.data_ptr(), vh.data_ptr())
        btd._abi.check("btd_substep", h, 0, 0)
        btd._abi.check("btd_get_state", h, xh.data_ptr(), vh.data_ptr())
    barrier()
    t_e2e = time.perf_counter() - t0
    cd_e2e = gpu.counter_dict()
    newton_e2e = cd_e2e["newton"]
    pcg_e2e = cd_e2e["pcg_total"] / max(1, cd_e2e["newton"])
    if dist is not None:
        t_e2e = across_ranks(dist, [t_e2e], "max")[0]
    e2e = world * newton_e2e / t_e2e

    # ---- roofline of the dominant kernel (fine-level smoother sweep), live, cold L2 per launch
    peak, peak_kind = peaks()
    R0 = 232.0  # fine row algorithmic bytes
    ms_sweep = gpu.profile_stage("smooth", reps=10, flush=True)
    bytes_sweep = 2.0 * N * (R0 + 36.0)
    achieved = bytes_sweep / (ms_sweep / 1e3) / 1e9
    ms_mv = gpu.profile_stage("matvec", reps=10, flush=True)
    mv_gbs = N * (R0 + 24.0) / (ms_mv / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(args.workload, {}).get("smooth_sweep_dram_bytes")
        except Exception:
            traffic = None

    variants = None
    if world == 1 and not w.get("product"):
        variants = []
        for settings in MG_VARIANTS:
            try:
                variants.append(measure_variant(btd, w, sc, args.steps, args.warmup, settings))
            except Exception as e:  # reported, never fatal to the default measurement
                variants.append({"settings": dict(settings), "error": f"{type(e).__name__}: {e}"})

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC_PRODUCT if w.get("product") else METRIC, "value": value, "unit": "Newton steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "description": w["desc"], "nodes": N, "levels": gpu.level_count(),
                   "newton_per_step": w["newton"], "pcg_iterations_per_newton": pcg_total / max(1, newton_total),
                   "l2": "flushed before every timed step (256 MiB rewrite outside the events)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e, "unit": "Newton steps/s", "h2d_bytes_per_step": 2 * 16 * N, "d2h_bytes_per_step": 2 * 16 * N,
                "pcg_iterations_per_newton": pcg_e2e,
                "loop": "each step: the state in from pinned host memory (the previous step's output), one substep, the state out"},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "k_smooth<FineRows> (fine yarn-line sweep, 6 colour launches)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_sweep": bytes_sweep, "ms_per_sweep": ms_sweep,
                     "matvec_gbs": mv_gbs, "matvec_ms": ms_mv},
        "clocks": clocks.summary(),
    }
    if variants is not None:
        line["config"]["mg_variants"] = variants
    # the metric's learned arm: the learned coarse space runs in the FP64 oracle only (its CUDA kernels
    # are not built), so this line measures the plain MG-PCG path
    line["config"]["learned_arm"] = "not on the CUDA path: this value is plain MG-PCG"
    if w.get("product"):
        line["config"]["ms_per_substep"] = ms_step
        line["config"]["reference_published"] = {
            "ms_per_substep": PRODUCT_PUBLISHED_MS, "hardware": "Apple M5, WebGPU",
            "source": "docs/decisions/2026-10-10-feedback-round2.md:11-14 (2 Newton x 2 PCG 6.9 ms + self-contact 0.6 ms)",
            "substep_time_ratio": PRODUCT_PUBLISHED_MS / ms_step}
    if world == 1 and not args.no_cpu_baseline:
        v_cpu, dt_cpu, cores = cpu_sample(btd, w, 1)
        what = ("the first substep's second Newton iteration (contacts engaged)" if w.get("contact") and not w.get("product")
                else f"1 substep ({w['newton']} Newton) of the workload from its initial state")
        line["cpu_baseline"] = {"value": v_cpu, "unit": "Newton steps/s", "cores": cores, "kind": "port",
                                "sample": f"{what}, {dt_cpu:.1f} s"}
        if not w.get("contact") or w.get("product"):
            v1, dt1 = cpu_sample_single_core(btd, w)
            line["cpu_baseline_single_core"] = {"value": v1, "unit": "Newton steps/s", "cores": 1, "kind": "port",
                                                "sample": f"the first substep's prediction and first Newton iteration, {dt1:.1f} s"}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
