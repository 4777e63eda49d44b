"""The multi-process paths of bench.py on CPU (gloo, world size 2): the
device-time maximum over ranks, the barrier, and the reference arm running on
rank 0 only (the other ranks return without work)."""

import argparse
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        out[f"max{rank}"] = bench.max_over_ranks(float(rank + 1) * 1.5, world)
        bench.barrier(world)
        args = argparse.Namespace(workload="gemm", gemm_n=64, steps=1, warmup=1)
        line = bench.run_reference(args, world, rank)
        out[f"ref{rank}"] = None if line is None else line["impl"]
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_bench_rank_helpers_gloo_world2():
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    assert out["max0"] == out["max1"] == 3.0
    assert out["ref0"] == "reference"
    assert out["ref1"] is None
