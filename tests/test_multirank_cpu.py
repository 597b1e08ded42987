"""The N>1 path of bench.py on CPU: one process per rank (gloo, world size 2),
as torchrun launches it on the GPUs with NCCL.  Replicas are independent
(their own seeds, no data-path collective); the job's time is the slowest
rank's, taken by one all-reduce; a rank that leaves makes the others'
next collective end with an error instead of waiting for good."""
import datetime
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))


def _aggregate_worker(rank, world, port, q):
    import bench

    _init(rank, world, port, 60)
    ms_rank = 100.0 + 25.0 * rank  # rank 1 is the slow one
    ms_max = bench.max_over_ranks(torch, dist, ms_rank)
    value = bench.whole_job_mlups(world, bench.NX * bench.NY, 10, ms_max)
    q.put((rank, ms_max, value, bench.rank_seed(rank)))
    dist.barrier()
    dist.destroy_process_group()


def _leaver_worker(rank, world, port, q):
    _init(rank, world, port, 5)
    dist.barrier()
    if rank == 1:
        q.put((rank, "left"))
        return  # leaves between steps, with nothing in flight
    try:
        dist.barrier()
        q.put((rank, "no error"))
    except Exception as e:  # the short process-group timeout ends the collective
        q.put((rank, "error: " + type(e).__name__))


def _run(worker, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_two_ranks_take_the_slowest_time_and_sum_the_work():
    import bench

    out = _run(_aggregate_worker)
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 125.0 for o in out)  # both ranks see the max
    nodes = bench.NX * bench.NY
    assert all(o[2] == pytest.approx(2 * nodes * 10 / (125.0 * 1e3)) for o in out)
    assert out[0][3] != out[1][3]  # independent replicas


def test_a_rank_that_leaves_ends_the_others_collective_with_an_error():
    out = dict(_run(_leaver_worker))
    assert out[1] == "left"
    assert out[0].startswith("error")
