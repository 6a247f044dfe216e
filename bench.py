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
CPU_SAMPLE_BUDGET_S = 20.0  # timed oracle work of the GPU arm's CPU baseline (after its untimed warm-up)
REFERENCE_BUDGET_S = 120.0  # timed oracle work of the reference arm (after its untimed warm-up)

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
TEARING = "config4-256"
WORKLOADS[TEARING] = dict(n=256, size=0.6, h=1 / 120, newton=4, rel=1e-6, contact=True, tearing=True,
                          desc="configuration 4's tearing patch: the 256x256 yarn lattice (0.6 m, yarn EA 2e3 N, bending "
                               "1e-7 N m^2, crossing friction 0.3, bundled [2, 2]) with a central 64x64-cell region of "
                               "lognormal(ln 0.08, 0.25) break strains, self-contact on, two edge grips (columns 0-1 and "
                               "n-2..n-1) pulled apart at 0.5 m/s; dt 1/120, 4 projected-Newton, MG-PCG to rel-res 1e-6")
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
DEFAULT_WORKLOAD = TEARING
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


class Patch:
    """The workload's scene and its grips: (nodes, sign) per grip, the grip moving along x by
    sign * speed / 2 per second (the two edges of the tearing patch separate at `speed`)."""

    def __init__(self, sc, grips=(), speed=0.0, stiffness=0.0):
        self.sc, self.grips, self.speed, self.stiffness = sc, list(grips), speed, stiffness

    @classmethod
    def build(cls, btd, w):
        if w.get("product"):
            return cls(btd.compile_scene(btd.default_spec()))
        if w.get("tearing"):
            c = btd.configs.CONFIG4
            sc, left, right = btd.configs.config4()
            return cls(sc, [(left, -1.0), (right, 1.0)], c["grip_speed"], c["grip_stiffness"])
        if w.get("contact"):
            return cls(btd.configs.config2())
        return cls(btd.configs.hanging_patch(w["n"], w["size"], seed=1))

    def anchors(self, x0):
        """(picked node, anchor) per grip: the middle node of its patch at its float32 position."""
        out = []
        for nodes, _ in self.grips:
            picked = int(nodes[len(nodes) // 2])
            out.append((picked, np.asarray(x0, np.float64)[picked].astype(np.float32).astype(np.float64)))
        return out

    def goals(self, anchors, s, h):
        """Grip targets before substep s (1-based)."""
        return [a + np.array([sign * 0.5 * self.speed * s * h, 0.0, 0.0]) for (_, a), (_, sign) in zip(anchors, self.grips)]

    # the reference arm builds its scene in a child process (the scene compiler lives in the product
    # library, which the reference arm must not map) and loads it from a file
    def save(self, path):
        sc = self.sc
        arrays = {name: getattr(sc, name) for name in sc.__dict__ if isinstance(getattr(sc, name), np.ndarray)}
        layers = np.frombuffer(b"".join(bytes(L) for L in sc.layers), np.uint8)
        grips = {f"grip{k}": np.asarray(nodes, np.int32) for k, (nodes, _) in enumerate(self.grips)}
        np.savez(path, _layers=layers, _meta=np.array([sc.N, sc.C, len(sc.layers), len(self.grips)], np.int64),
                 _signs=np.array([g[1] for g in self.grips] + [0.0]), _grip=np.array([self.speed, self.stiffness]),
                 **arrays, **grips)

    @classmethod
    def load(cls, btd, path):
        import ctypes

        d = np.load(path)
        N, C, nl, ng = (int(v) for v in d["_meta"])
        size = ctypes.sizeof(btd._abi.LayerInfo)
        raw = d["_layers"].tobytes()
        layers = [btd._abi.LayerInfo.from_buffer_copy(raw[k * size:(k + 1) * size]) for k in range(nl)]
        arrays = {k: d[k].copy() for k in d.files if not k.startswith("_") and not k.startswith("grip")}
        sc = btd.Scene(layers, N, C, arrays)
        grips = [(d[f"grip{k}"], float(d["_signs"][k])) for k in range(ng)]
        return cls(sc, grips, float(d["_grip"][0]), float(d["_grip"][1]))


def solver_params(btd, w, settings=None):
    if w.get("product"):
        p = btd.default_params()
    else:
        p = btd.configs.solver_params(w["h"], w["newton"], w["rel"], self_contact=1 if w.get("contact") else 0)
    for k, v in (settings or {}).items():
        setattr(p, k, v)
    return p


def gpu_arm(btd, w, patch, settings=None, learned=None):
    """A GpuSolver set up as the workload (floor, drape, grips; the learned coarse correction with the
    given weights) and its per-substep driver."""
    g = btd.GpuSolver(patch.sc, solver_params(btd, w, settings))
    if learned is not None:
        g.set_learned(learned, on=True, guard=btd.configs.CONFIG4["guard"])
    if w.get("product"):
        g.settle_drape()  # the product starts from its settled drape (drape.bin / settleDrape)
    elif w.get("contact") and not w.get("tearing"):
        g.set_floor(btd.configs.CONFIG2["floor"])
    anchors = patch.anchors(g.x)
    for slot, ((nodes, _), (picked, a)) in enumerate(zip(patch.grips, anchors)):
        g.attach_patch(slot, picked, nodes, np.ones(len(nodes)), a.astype(np.float32), patch.stiffness, max_lead=1.0)

    def drive(s):
        for slot, goal in enumerate(patch.goals(anchors, s, w["h"])):
            g.set_target(goal.astype(np.float32), slot=slot)

    return g, drive


def timed_substeps(g, drive, first, count):
    """Device time (ms) of `count` substeps from substep `first`, L2 flushed before each (outside the
    CUDA events on the solver's stream); the grip targets are set before each."""
    total = 0.0
    for s in range(first, first + count):
        drive(s)
        total += g.profile_stage("substep", reps=1, flush=True)
    return total


def learned_weights(btd):
    """The learned coarse correction's network: the committed weights (trained on the GPU by
    break-that-denim_b200/train_learned.py), else trained here on the GPU (about a minute)."""
    path = btd.learned.DEFAULT_PATH
    if os.path.exists(path):
        return btd.learned.load(path), {"weights": os.path.basename(path), "trained": "on the GPU by train_learned.py"}
    t = time.perf_counter()
    w, hist = btd.learned.train_network(verbose=False)
    return w, {"weights": "trained in this run on the GPU", "train_s": time.perf_counter() - t,
               "final_loss": float(np.mean(hist[-50:]))}


# Multigrid settings measured beside the reference's schedule (hierarchy lagged from a substep's first
# Newton iteration, newtonMultigrid.ts:579; coarsest level at most 400 nodes, solver.ts:70): the
# Galerkin hierarchy rebuilt at every Newton iteration, and that coarsened down to at most 30 nodes.
# On the oracle they take the PCG iterations per Newton step of the 256 x 256 hanging patch from 37 to
# 20 and 13; each extra level costs its launches in every V-cycle, so the device decides.
MG_VARIANTS = {"rebuilt": dict(lag_coarse=0), "rebuilt_deep": dict(lag_coarse=0, max_coarsest_nodes=30)}


def measure_arm(btd, w, patch, steps, warmup, settings=None, learned=None):
    """The workload's substeps W + 1 .. W + K on a fresh solver with `settings` (and the learned coarse
    correction when weights are given): Newton steps/s from the device-timed substeps, PCG iterations
    per Newton step, levels and kernel launches."""
    g, drive = gpu_arm(btd, w, patch, settings, learned)
    try:
        for s in range(1, warmup + 1):
            drive(s)
            g.substep()
        g.synchronize()
        g.clear_counters()
        ms = timed_substeps(g, drive, warmup + 1, steps)
        g.synchronize()
        c = g.counter_dict()
        out = {"settings": dict(settings or {}), "learned": learned is not None, "levels": g.level_count(),
               "value": c["newton"] / (ms / 1e3), "unit": "Newton steps/s", "ms_per_step": ms / steps,
               "pcg_iterations_per_newton": c["pcg_total"] / max(1, c["newton"]),
               "solves_short_of_tolerance": c["pcg_missed"], "worst_rel_residual": c["rel_residual_max"],
               "gpu_launches": int(g.launch_count(steps, c["newton"], c["pcg_total"]))}
        if learned is not None:
            out["learned_stats"] = g.learned_stats()
        return out
    finally:
        g.close()


def workload_oracle(w, patch, threads=0):
    """The oracle configured as the workload's solve (PCG to the relative residual, or the fixed count),
    with the workload's floor and grips; returns it and its per-substep driver."""
    sys.path.insert(0, ROOT)
    from oracle import Oracle

    o = Oracle(patch.sc, h=w["h"], newton_iterations=w["newton"], pcg_iterations=w.get("pcg", 500), pcg_rel_tol=w["rel"],
               threads=threads, self_contact=bool(w.get("contact")), **MG)
    if w.get("contact") and not w.get("product") and not w.get("tearing"):
        o.set_floor(CONFIG2_FLOOR)
    x0 = o.x.astype(np.float32).astype(np.float64)
    anchors = patch.anchors(x0)
    for (nodes, _), (picked, a) in zip(patch.grips, anchors):
        o.add_grip(nodes, np.ones(len(nodes)), (x0[nodes] - x0[picked]).reshape(-1), a, patch.stiffness)

    def drive(s):
        for slot, goal in enumerate(patch.goals(anchors, s, w["h"])):
            o.set_grip_goal(slot, goal.astype(np.float32).astype(np.float64))

    return o, drive


CONFIG2_FLOOR = 0.0  # the folded drop's floor height (configs.CONFIG2["floor"])


def peaks():
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clock and throttle-reason samples during the timed region: NVML polled every 5 ms (short
    timed regions still get samples), else nvidia-smi every 200 ms. Reads only."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.rows = []  # (sm MHz, max sm MHz, [reason names])
        self.proc = None
        self.stop = threading.Event()
        self.source = None

    def __enter__(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(int(self.index))
            bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def poll():
                while not self.stop.is_set():
                    try:
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), float(mx),
                                          [n for n, b in zip(self.NAMES, bits) if r & b]))
                    except Exception:
                        pass
                    self.stop.wait(0.005)

            self.source = "nvml"
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            r = [c.strip() for c in line.split(",")]
            if len(r) < 8 or not r[0].replace(".", "").isdigit():
                continue
            self.rows.append((float(r[0]), float(r[1]) if r[1].replace(".", "").isdigit() else None,
                              [self.NAMES[k] for k in range(4) if r[4 + k] == "Active"]))

    def __exit__(self, *a):
        self.stop.set()
        if self.source == "nvml":
            self.thread.join(timeout=1)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows if r[1]]
        reasons = sorted({n for r in self.rows for n in r[2]})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows), "source": self.source}


def cpu_sample(w, patch, substeps, threads=0, warmup=0, budget=None):
    """The oracle (the reference's CPU solver restated, FP64, OpenMP) on substeps warmup + 1 ..
    warmup + substeps of the workload (the warm-up ones untimed), or fewer when `budget` seconds of
    timed work run out first (a bounded sample: at least one substep); returns Newton steps/s, seconds,
    cores and the substeps timed."""
    o, drive = workload_oracle(w, patch, threads)
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    if w.get("contact") and not w.get("product") and not w.get("tearing"):
        # bounded sample: one Newton iteration with the contacts engaged - the first substep's second
        # (its prediction and first iteration, untimed, converge in ~50 PCG iterations; the later
        # ones, ~30 s each on 8 host cores, are the representative work)
        o.predict()
        o.newton_step()
        t = time.perf_counter()
        o.newton_step()
        dt = time.perf_counter() - t
        return 1.0 / dt, dt, cores, 0
    for s in range(1, warmup + 1):
        drive(s)
        o.substep()
    t = time.perf_counter()
    done = 0
    for s in range(warmup + 1, warmup + substeps + 1):
        drive(s)
        o.substep()
        done += 1
        if budget is not None and time.perf_counter() - t >= budget:
            break
    dt = time.perf_counter() - t
    return done * w["newton"] / dt, dt, cores, done


def across_ranks(dist, values, op="max", device="cuda"):
    """Every rank's `values` combined over the ranks (the max of the device times: the job takes as
    long as its slowest rank; the sum of counts); unchanged on a single process."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def cpu_baselines(w, patch, warmup, steps, budget):
    """The oracle on the GPU arm's substep window: substeps 1..warmup untimed on all host cores, then
    substeps warmup + 1 .. timed on all cores until `steps` or `budget` seconds (at least one), then the
    next substep's prediction and first Newton iteration on one core. Returns (Newton steps/s, seconds,
    cores, substeps timed) on all cores and (Newton steps/s, seconds, substep) on one."""
    import ctypes

    o, drive = workload_oracle(w, patch)
    cores = os.cpu_count() or 1
    for s in range(1, warmup + 1):
        drive(s)
        o.substep()
    t = time.perf_counter()
    done = 0
    for s in range(warmup + 1, warmup + steps + 1):
        drive(s)
        o.substep()
        done += 1
        if time.perf_counter() - t >= budget:
            break
    dt = time.perf_counter() - t
    gomp = ctypes.CDLL("libgomp.so.1")
    gomp.omp_set_num_threads(1)
    s1 = warmup + done + 1
    drive(s1)
    t = time.perf_counter()
    o.predict()
    o.newton_step()
    dt1 = time.perf_counter() - t
    gomp.omp_set_num_threads(cores)
    return (done * w["newton"] / dt, dt, cores, done), (1.0 / dt1, dt1, s1)


def batch_patches(btd, count):
    """The first `count` patches of the batch with their grips, as Patch objects whose single grip moves
    with the patch's velocity (the Patch's goals are replaced by the velocity's)."""
    out = []
    for sc, g in btd.configs.config3(only=list(range(count))):
        p = Patch(sc, [(np.asarray(g["nodes"], np.int32), 0.0)], 0.0, float(g["stiffness"]))
        p.picked, p.weights, p.velocity = int(g["picked"]), np.asarray(g["weights"], np.float64), np.asarray(g["velocity"])
        out.append(p)
    return out


def batch_cpu_sample(w, patches, steps, warmup=0):
    """The oracle on the given batch patches: substeps warmup + 1 .. warmup + steps of each (the warm-up
    ones untimed), its grip held and moved with the patch's velocity."""
    sys.path.insert(0, ROOT)
    from oracle import Oracle

    dt, newton = 0.0, 0
    for p in patches:
        o = Oracle(p.sc, h=w["h"], newton_iterations=w["newton"], pcg_iterations=500, pcg_rel_tol=w["rel"], **MG)
        x = o.x
        nodes = np.asarray(p.grips[0][0])
        anchor = x[p.picked].copy()
        o.add_grip(nodes, p.weights, (x[nodes] - x[p.picked]).reshape(-1), anchor, p.stiffness)
        for s in range(1, warmup + steps + 1):
            o.set_grip_goal(0, anchor + s * w["h"] * p.velocity)
            t = time.perf_counter()
            o.substep()
            if s > warmup:
                dt += time.perf_counter() - t
                newton += w["newton"]
    return newton / dt, dt, os.cpu_count() or 1


def dump_patches(args, path):
    """Child process of the reference arm: writes the workload's patches (scene, grips) to files."""
    btd = package()
    w = WORKLOADS[args.workload]
    if args.workload == BATCH:
        for k, p in enumerate(batch_patches(btd, 2)):
            p.save(f"{path}.{k}.npz")
            np.savez(f"{path}.{k}.grip.npz", picked=p.picked, weights=p.weights, velocity=p.velocity)
    else:
        Patch.build(btd, w).save(f"{path}.0.npz")


def load_patches(btd, args, path):
    if args.workload != BATCH:
        return [Patch.load(btd, f"{path}.0.npz")]
    out = []
    for k in range(2):
        p = Patch.load(btd, f"{path}.{k}.npz")
        g = np.load(f"{path}.{k}.grip.npz")
        p.picked, p.weights, p.velocity = int(g["picked"]), g["weights"], g["velocity"]
        out.append(p)
    return out


def run_reference(args, w, rank):
    """The reference arm: the reference's CPU solver (its FP64 restatement, the oracle) on the host
    cores, on the same workload, metric and substep window (W warm-up substeps untimed, then K timed).
    The scenes are compiled in a child process and read from files, so that this process maps no
    library of the product."""
    if rank != 0:
        return
    import tempfile

    btd = package()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "patch")
        subprocess.run([sys.executable, os.path.abspath(__file__), "--workload", args.workload, "--dump-patches", path],
                       check=True)
        patches = load_patches(btd, args, path)
    steps = max(1, args.steps)
    if args.workload == BATCH:
        value, dt, cores = batch_cpu_sample(w, patches, steps, args.warmup)
        sample = f"substeps {args.warmup + 1}..{args.warmup + steps} of the first {len(patches)} patches (warm-up untimed)"
        scaling = "strong"
    else:
        value, dt, cores, done = cpu_sample(w, patches[0], steps, warmup=args.warmup, budget=REFERENCE_BUDGET_S)
        sample = (f"substeps {args.warmup + 1}..{args.warmup + done} x {w['newton']} Newton of the workload (warm-up untimed"
                  + (f"; {steps - done} of the {steps} steps left out when {REFERENCE_BUDGET_S} s of timed work ran out)" if done < steps else ")"))
        scaling = "weak"
        if w.get("contact") and not w.get("tearing"):
            sample = "the first substep's second Newton iteration (contacts engaged)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Newton steps/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": scaling, "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": {"workload": args.workload, "description": w["desc"]},
            "cpu_baseline": {"value": value, "unit": "Newton steps/s", "cores": cores, "kind": "port", "sample": sample},
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

    graph = [None]

    def advance():
        step[0] += 1
        for s, a, (_, g) in zip(solvers, anchors, patches):
            s.set_target((a + step[0] * c["h"] * g["velocity"]).astype(np.float32))
        if graph[0] is not None:
            graph[0].run(1)
        else:
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
    # the sweeps' launch shapes of every patch picked by the autotuner on its current operators, then
    # the batch as one graph: one launch per batch substep
    t_tune = time.perf_counter()
    if not args.batch_streams:
        for s in solvers:
            s.autotune(reps=3)
        graph[0] = btd.Batch(solvers)
    t_tune = time.perf_counter() - t_tune
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
        if graph[0] is not None:
            graph[0].run(1)
        else:
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
    if graph[0] is not None:
        graph[0].close()
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
                   "setup_s": t_setup, "autotune_and_capture_s": t_tune,
                   "launch": ("one graph per batch substep (btd_batch_run), sweep shapes autotuned per patch"
                              if not args.batch_streams else "one graph per patch, round robin over streams"),
                   "parallelism": f"patches sharded x{world}"},
        "e2e": {"value": newton_e2e / t_e2e, "unit": "Newton steps/s", "h2d_bytes_per_step": int(bytes_step),
                "d2h_bytes_per_step": int(bytes_step)},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        v_cpu, dt_cpu, cores = batch_cpu_sample(w, batch_patches(btd, 2), 1)
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
    ap.add_argument("--no-variants", action="store_true",
                    help="measure the headline arm alone (no plain arm, no multigrid variants; for profilers)")
    ap.add_argument("--eager", action="store_true", help="launch the timed substeps kernel by kernel (for per-kernel profilers)")
    ap.add_argument("--patches", type=int, default=512, help="patches of the batch workload")
    ap.add_argument("--dump-patches", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--batch-streams", action="store_true", help="batch workload: one graph per patch on its stream")
    args = ap.parse_args()
    if args.dump_patches:
        dump_patches(args, args.dump_patches)
        return
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
    patch = Patch.build(btd, w)
    sc = patch.sc
    # the metric's learned arm (the tearing workload): the learned coarse correction on top of the
    # reference's schedule; the plain arm is measured beside it on the same substep window
    learned, learned_info = (learned_weights(btd) if w.get("tearing") else (None, None))
    gpu, drive = gpu_arm(btd, w, patch, learned=learned)

    current = [gpu]

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        current[0].synchronize()

    # warm-up: substeps 1..W (captures the substep graph, fills caches)
    for s in range(1, args.warmup + 1):
        drive(s)
        gpu.substep()
    gpu.synchronize()
    gpu.clear_counters()
    if args.eager:  # the timed substeps kernel by kernel, the warm-up's graphs left out of a profiler's count
        gpu.set_graph_mode(False)

    # ---- device-timed region: substeps W + 1 .. W + K, cold L2 before each (flush outside the events)
    barrier()
    idx = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        idx = vis.split(",")[local]
    with ClockSampler(idx) as clocks:
        ms_total = timed_substeps(gpu, drive, args.warmup + 1, args.steps)
        barrier()
    ms_step = ms_total / args.steps
    c = gpu.counter_dict()
    newton_total = c["newton"]
    pcg_total = c["pcg_total"]
    t_dev = ms_total / 1e3
    if dist is not None:
        t_dev = across_ranks(dist, [t_dev], "max")[0]
    value = world * newton_total / t_dev
    launches = gpu.launch_count(args.steps, newton_total, pcg_total)
    levels = gpu.level_count()
    learned_stats = gpu.learned_stats() if learned is not None else None

    # ---- roofline of the dominant kernel (fine-level smoother sweep), live, cold L2 per launch, on the
    # system of the last timed substep
    peak, peak_kind = peaks()
    N = sc.N
    R0 = 232.0  # fine row algorithmic bytes
    ms_sweep = gpu.profile_stage("smooth", reps=10, flush=True)
    bytes_sweep = 2.0 * N * (R0 + 36.0)
    achieved = bytes_sweep / (ms_sweep / 1e3) / 1e9
    ms_mv = gpu.profile_stage("matvec", reps=10, flush=True)
    # PCG's matvec reads the FP64 rows (58 doubles a node), p and the fixed flag, and writes Ap
    R64 = 464.0
    mv_gbs = N * (R64 + 16.0 + 4.0 + 16.0) / (ms_mv / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(args.workload, {}).get("smooth_sweep_dram_bytes")
        except Exception:
            traffic = None
    gpu.close()

    # ---- end to end through the C ABI from pinned host buffers: the state in (the previous step's
    # output), the grip targets, one substep, the state out; substeps W + 1 .. W + K of a fresh solver
    g2, drive2 = gpu_arm(btd, w, patch, learned=learned)
    current[0] = g2
    for s in range(1, args.warmup + 1):
        drive2(s)
        g2.substep()
    xh = torch.empty((N, 4), dtype=torch.float32, pin_memory=True)
    vh = torch.empty((N, 4), dtype=torch.float32, pin_memory=True)
    h = g2._h
    btd._abi.check("btd_get_state", h, xh.data_ptr(), vh.data_ptr())
    g2.synchronize()
    g2.clear_counters()
    barrier()
    t0 = time.perf_counter()
    for s in range(args.warmup + 1, args.warmup + args.steps + 1):
        btd._abi.check("btd_set_state", h, xh.data_ptr(), vh.data_ptr())
        drive2(s)
        btd._abi.check("btd_substep", h, 0, 0)
        btd._abi.check("btd_get_state", h, xh.data_ptr(), vh.data_ptr())
    barrier()
    t_e2e = time.perf_counter() - t0
    cd_e2e = g2.counter_dict()
    g2.close()
    newton_e2e = cd_e2e["newton"]
    pcg_e2e = cd_e2e["pcg_total"] / max(1, cd_e2e["newton"])
    if dist is not None:
        t_e2e = across_ranks(dist, [t_e2e], "max")[0]
    e2e = world * newton_e2e / t_e2e

    # ---- the plain arm and other multigrid settings on the same substep window (one GPU only)
    variants, plain = None, None
    if learned is not None and not args.no_variants:
        plain = measure_arm(btd, w, patch, args.steps, args.warmup, {})
    if world == 1 and not w.get("product") and not args.no_variants:
        variants = {}
        for name, settings in MG_VARIANTS.items():
            for lw, suffix in ((None, ""), (learned, "_learned")):
                if lw is None and suffix:
                    continue
                try:
                    variants[name + suffix] = measure_arm(btd, w, patch, args.steps, args.warmup, settings, lw)
                except Exception as e:  # reported, never fatal to the default measurement
                    variants[name + suffix] = {"settings": dict(settings), "error": f"{type(e).__name__}: {e}"}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC_PRODUCT if w.get("product") else METRIC, "value": value, "unit": "Newton steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "description": w["desc"], "nodes": N, "levels": None,
                   "newton_per_step": w["newton"], "pcg_iterations_per_newton": pcg_total / max(1, newton_total),
                   "solves_short_of_tolerance": c["pcg_missed"], "worst_rel_residual": c["rel_residual_max"],
                   "substeps_timed": [args.warmup + 1, args.warmup + args.steps],
                   "l2": "flushed before every timed step (256 MiB rewrite outside the events)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e, "unit": "Newton steps/s", "h2d_bytes_per_step": 2 * 16 * N, "d2h_bytes_per_step": 2 * 16 * N,
                "pcg_iterations_per_newton": pcg_e2e,
                "loop": "each step: the state in from pinned host memory (the previous step's output), the grip targets, "
                        "one substep, the state out"},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "k_smooth<FineRows> (fine yarn-line sweep, 6 colour launches)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_sweep": bytes_sweep, "ms_per_sweep": ms_sweep,
                     "matvec_gbs": mv_gbs, "matvec_ms": ms_mv, "matvec_frac": mv_gbs / peak,
                     "matvec_bytes_per_node": R64 + 36.0},
        "clocks": clocks.summary(),
    }
    line["config"]["levels"] = levels
    if variants is not None:
        line["config"]["mg_variants"] = variants
    if learned is not None:
        line["config"]["arm"] = ("learned: the learned coarse correction (BF16 MLP basis on the coarsest level, "
                                 "guard 0.9) on the reference's schedule (hierarchy lagged from each substep's first "
                                 "Newton iteration, coarsest level <= 400 nodes)")
        line["config"]["learned"] = dict(learned_info, stats=learned_stats)
        if plain is not None:
            line["config"]["plain"] = plain
            line["config"]["learned_over_plain"] = value / plain["value"]
    else:
        line["config"]["arm"] = "plain MG-PCG (the reference's schedule)"
    if w.get("product"):
        line["config"]["ms_per_substep"] = ms_step
        line["config"]["reference_published"] = {
            "ms_per_substep": PRODUCT_PUBLISHED_MS, "hardware": "Apple M5, WebGPU",
            "source": "docs/decisions/2026-10-10-feedback-round2.md:11-14 (2 Newton x 2 PCG 6.9 ms + self-contact 0.6 ms)",
            "substep_time_ratio": PRODUCT_PUBLISHED_MS / ms_step}
    if world == 1 and not args.no_cpu_baseline:
        if w.get("contact") and not w.get("product") and not w.get("tearing"):
            v_cpu, dt_cpu, cores, _ = cpu_sample(w, patch, 1)
            line["cpu_baseline"] = {"value": v_cpu, "unit": "Newton steps/s", "cores": cores, "kind": "port",
                                    "sample": f"the first substep's second Newton iteration (contacts engaged), {dt_cpu:.1f} s"}
        else:
            (v_cpu, dt_cpu, cores, done), (v1, dt1, s1) = cpu_baselines(w, patch, args.warmup, args.steps, CPU_SAMPLE_BUDGET_S)
            line["cpu_baseline"] = {"value": v_cpu, "unit": "Newton steps/s", "cores": cores, "kind": "port",
                                    "sample": f"substeps {args.warmup + 1}..{args.warmup + done} ({w['newton']} Newton each) of the "
                                              f"timed window, {dt_cpu:.1f} s (substeps 1..{args.warmup} untimed)"}
            line["cpu_baseline_single_core"] = {"value": v1, "unit": "Newton steps/s", "cores": 1, "kind": "port",
                                                "sample": f"substep {s1}'s prediction and first Newton iteration, {dt1:.1f} s"}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
