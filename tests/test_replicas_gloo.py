"""The multi-GPU path of bench.py is independent replicas: each rank renders its own sample
indices and only the timings meet, as a max over ranks.  Two gloo ranks on the CPU check that
the replicas' sample ranges are disjoint and that every rank gets the slowest rank's time."""
import importlib.util
import os
import pathlib

import pytest
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = _bench()
        warmup, steps = 3, 5
        base = b.replica_sample_base(rank, warmup, steps)
        used = [(base, base + 1)]  # counting pass
        used += [(b.step_samples(base, 0, w), b.step_samples(base, 0, w) + b.SPP_PER_STEP) for w in range(warmup)]
        used += [(b.step_samples(base, warmup, k), b.step_samples(base, warmup, k) + b.SPP_PER_STEP) for k in range(steps)]
        t = b.max_over_ranks(10.0 + 7.0 * rank, dist, "cpu")
        out[rank] = (used, t)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_disjoint_samples_and_max_time():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = 29500 + (os.getpid() % 1000)
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    ranges = {r: out[r][0] for r in range(world)}
    for r in range(world):
        assert out[r][1] == 17.0  # the slowest rank's time on every rank
        spans = sorted(ranges[r])
        assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:]))  # no overlap within a rank
    lo0, hi0 = min(a for a, _ in ranges[0]), max(b for _, b in ranges[0])
    lo1, hi1 = min(a for a, _ in ranges[1]), max(b for _, b in ranges[1])
    assert hi0 <= lo1 or hi1 <= lo0  # ranks never render the same sample index
