"""Sharding of the batched configuration across GPUs (one process a GPU, no data-path collective):
every patch on exactly one rank, loads balanced by estimated bytes, each patch built the same
whichever subset asks for it, and the end-of-run gather of per-patch statistics over a world of two
gloo ranks on the CPU (the path an NCCL all-gather takes on GPUs)."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

try:
    import btd_b200 as btd
except ImportError:  # a spawned rank: register the package as the test session does
    from conftest import _load_package

    btd = _load_package()


def test_shards_cover_every_patch_once_and_balance():
    sides = btd.configs.config3_sides()
    assert len(sides) == 512 and min(sides) >= 16 and max(sides) <= 128
    for world in (1, 2, 4, 8):
        shards = btd.configs.shard_patches(sides, world)
        flat = sorted(b for s in shards for b in s)
        assert flat == list(range(512))
        loads = [sum(sides[b] ** 2 for b in s) for s in shards]
        assert max(loads) - min(loads) <= 128 ** 2, (world, loads)


def test_a_patch_is_the_same_built_alone():
    full = btd.configs.config3(count=6, sides=(16, 24))
    some = btd.configs.config3(count=6, sides=(16, 24), only=[4, 1])
    for (sc, g), b in zip(some, (4, 1)):
        sf, gf = full[b]
        assert np.array_equal(sc.position, sf.position) and np.array_equal(sc.field_strength, sf.field_strength)
        assert np.array_equal(g["nodes"], gf["nodes"]) and np.allclose(g["velocity"], gf["velocity"])


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sides = btd.configs.config3_sides(count=40, sides=(16, 48))
    mine = btd.configs.shard_patches(sides, world)[rank]
    stats = {b: (b, sides[b]) for b in mine}  # stand-in for (Newton steps, PCG iterations) a patch
    got = [None] * world
    dist.all_gather_object(got, stats)
    if rank == 0:
        merged = {}
        for d in got:
            assert not set(d) & set(merged)
            merged.update(d)
        out.put(sorted(merged))
    dist.destroy_process_group()


def test_per_patch_statistics_gather_over_two_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == list(range(40))


def _bench_rank(rank, world, port, out):
    import importlib.util
    import sys

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    sys.modules["bench_under_test"] = bench
    spec.loader.exec_module(bench)
    # replicas: rank r took 1 + r seconds for 10 Newton steps; the job time is the slowest rank's
    t = bench.across_ranks(dist, [1.0 + rank, 0.5 * (1 + rank)], "max", device="cpu")
    n = bench.across_ranks(dist, [10.0], "sum", device="cpu")
    if rank == 0:
        out.put((t, n))
    dist.destroy_process_group()


def test_replica_timing_is_the_slowest_rank_over_two_ranks():
    """bench.py --gpus N runs N replicas (one patch does not shard): value = all ranks' Newton steps
    over the slowest rank's device time; the reduction over two gloo ranks."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_bench_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, n = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert t == [2.0, 1.0] and n == [20.0]
