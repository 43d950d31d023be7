"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2).

The path does not shard: every rank filters its own copy of the workload and
no collective touches the data.  What runs across ranks is the timing
protocol — barriers around the timed region and the maximum of the per-rank
times — and the per-rank seeding of the inputs; both are checked here with
the gloo backend, no GPU involved.
"""
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


def _worker(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ws, rk, lr = bench.rank_info()
        # the slowest rank's time is the job's time
        t = bench.max_over_ranks(1.5 + rk, torch.device("cpu"))
        # inputs are seeded by rank: replicas filter different signals
        w = bench.load_workload("cfg1", "cpu", seed=rk, B=2, T=64)
        xs = [torch.empty_like(w["x"]) for _ in range(world)]
        dist.all_gather(xs, w["x"].contiguous())
        same = all(torch.equal(xs[0], xi) for xi in xs[1:])
        # the reference arm: ranks other than 0 exit at once without work
        args = type("A", (), {"config": "cfg1", "B": 2, "T": 64, "steps": 1, "warmup": 1})()
        ref_rc = bench.run_reference(args) if rk != 0 else None
        out.put((rk, ws, t, same, ref_rc))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_timing_protocol():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rk, ws, t, same, ref_rc in res:
        assert ws == world
        assert t == pytest.approx(2.5)  # the max over ranks, on every rank
        assert not same
    assert res[1][4] == 0
