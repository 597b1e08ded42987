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


# ------------------------------------------------ independent units over ranks
def test_lpt_puts_every_unit_in_exactly_one_part_and_balances():
    from lagrangianrbnudging_b200 import shard

    rng = __import__("numpy").random.default_rng(3)
    for n, parts in [(64, 2), (64, 8), (4, 8), (7, 3), (1, 1), (0, 2)]:
        costs = [float(c) for c in rng.choice([32768, 131072, 524288], n)]
        split = shard.lpt(costs, parts)
        assert len(split) == parts
        flat = sorted(i for p in split for i in p)
        assert flat == list(range(n))
        assert all(p == sorted(p) for p in split)
        if n:
            loads = [sum(costs[i] for i in p) for p in split]
            # list scheduling: no part exceeds the mean load by more than one unit
            assert max(loads) <= sum(costs) / parts + max(costs) + 1e-9
        # every rank computes the same split
        for r in range(parts):
            assert shard.my_units(costs, r, parts) == split[r]
    # equal costs go round robin
    assert shard.lpt([1.0] * 4, 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.my_units([1.0], 2, 2)


def test_ensemble_members_split_by_node_count_cover_the_ensemble():
    import bench
    from lagrangianrbnudging_b200 import shard

    desc = bench.ensemble_desc()
    assert len(desc) == bench.ENS_N and desc == bench.ensemble_desc()  # seeded, same on every rank
    costs = [nx * ny for nx, ny, _, _ in desc]
    for world in (1, 2, 4, 8):
        units = [shard.my_units(costs, r, world) for r in range(world)]
        assert sorted(i for u in units for i in u) == list(range(bench.ENS_N))
        loads = [sum(costs[i] for i in u) for u in units]
        assert max(loads) - min(loads) <= max(costs)


def _gather_worker(rank, world, port, q):
    from lagrangianrbnudging_b200 import shard

    _init(rank, world, port, 60)
    ndir = 8
    mine = shard.my_units([1.0] * ndir, rank, world)
    errs = {k: 1e-9 * (k + 1) for k in mine}  # each rank's share of the FD directions
    merged = {}
    for part in shard.gather(dist, errs):
        merged.update(part)
    q.put((rank, sorted(mine), [merged[k] for k in range(ndir)]))
    dist.barrier()
    dist.destroy_process_group()


def test_split_units_are_gathered_once_in_rank_order():
    out = _run(_gather_worker)
    assert [o[0] for o in out] == [0, 1]
    assert out[0][1] == [0, 2, 4, 6] and out[1][1] == [1, 3, 5, 7]
    expect = [1e-9 * (k + 1) for k in range(8)]
    assert out[0][2] == expect and out[1][2] == expect
