"""The multi-GPU path is replicas only: each rank serves its own share of the
request stream and the ranks meet only to time the run (barrier, max of the
step times, sum of the request counts).  These tests run that plumbing as two
gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        class A:
            requests, n_hi, seed, rate = 6, 512, 4, 0.0

        bench.barrier(world)
        mx = bench.max_over_ranks(10.0 + rank, world)
        sm = bench.sum_over_ranks(float(rank + 1), world)
        specs = bench.step_specs(A, 0, rank, False)
        out.put((rank, mx, sm, [(s.n, s.m, s.algo, s.seed) for s in specs]))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_and_shard():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(world):
            rank, mx, sm, specs = out.get(timeout=120)
            got[rank] = (mx, sm, specs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    # the slowest rank's time and the total request count, on every rank
    assert got[0][0] == got[1][0] == 11.0
    assert got[0][1] == got[1][1] == 3.0
    # each rank draws its own requests (no shared data, no collective on the data path)
    assert got[0][2] != got[1][2]
    assert len(got[0][2]) == len(got[1][2]) == 6


def test_single_rank_helpers_are_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.sum_over_ranks(7.0, 1) == 7.0
    bench.barrier(1)
