"""The N > 1 logic of bench.py on CPU: two gloo ranks (one process each, 127.0.0.1) take the same
collective steps the GPU replicas take -- disjoint sample ranges, a barrier, the max-over-ranks time --
and rank 0's whole-job throughput counts both ranks' paths over the slowest rank's time."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        spp = 64
        offset = bench.replica_sample_offset(rank, spp)
        gathered = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(gathered, torch.tensor([offset], dtype=torch.int64))
        dist.barrier()
        seconds = bench.max_over_ranks(dist, 1.0 + 0.5 * rank, torch.device("cpu"))
        value = bench.whole_job_mpaths(world, 1_000_000, 2, seconds)
        out[rank] = (sorted(int(g.item()) for g in gathered), seconds, value)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replica_logic():
    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    offsets, seconds, value = out[0]
    assert offsets == [0, 64]                       # disjoint sample ranges [0, 64) and [64, 128)
    assert out[1][1] == seconds == pytest.approx(1.5)  # both ranks see the slowest rank's time
    assert value == pytest.approx(2 * 1_000_000 * 2 / 1.5 / 1e6)

