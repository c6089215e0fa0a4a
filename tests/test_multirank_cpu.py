"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1.

Each rank of `python -m torch.distributed.run ... bench.py --gpus N` transforms
its own shard (weak scaling, no collective on the data path); the step time is
the slowest rank's, taken with one all-reduce, and the whole-job GB/s counts
every rank's bytes.  The GPU work itself cannot run here; the reduction, the
per-rank seeds and the job accounting can."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 10.0 + 5.0 * rank               # rank 1 is the slow one
        ms = bench.max_over_ranks(torch, dist, local_ms, "cpu")
        wl = bench.C3Fxcorr()
        cfg = wl.config(world)
        gbs = bench.whole_job_gbs(wl.bytes_per_step(), world, ms)
        out.put((rank, ms, cfg["global_batch_points"], gbs))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_step_and_count_every_shard():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(out.get(timeout=10) for _ in range(world))
    per_rank_bytes = 256 * (1 << 20) * 16
    for rank, ms, points, gbs in res:
        assert ms == pytest.approx(15.0)           # the max over ranks, on every rank
        assert points == 256 * (1 << 20) * world   # weak scaling: every rank its own 256 channels
        assert gbs == pytest.approx(per_rank_bytes * world / 15e-3 / 1e9)
