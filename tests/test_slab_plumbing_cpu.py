"""The one-process-per-GPU exchange of y-slabs with particles
(lagrangianrbnudging_b200.slabrank) on CPU: one process per rank over gloo,
as torchrun launches it on GPUs over NCCL, each rank a stand-in slab
(tests/slab_standin.py) that writes its messages in the library's byte
layout and checks every message it receives against the oracle's whole
domain.  Two ranks (both neighbours are the same rank, around the ring) and
three; the particles end up held once each, with the oracle's states."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

NX, NYT = 32, 24


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _params():
    from oracle.oracle import closure

    return dict(**closure(NX, NYT, Ra=1e6, Pr=1.0, U=0.1))


def _particles(n: int, edges):
    """particles beside every slab boundary (and the walls), moving across
    them on the first steps (tracers step by 1.5 u - 0.5 u_old)"""
    rng = np.random.default_rng(5)
    y = np.concatenate([e + rng.uniform(-0.3, 0.3, n // (len(edges) + 1)) for e in edges]
                       + [rng.uniform(1.0, NYT, n - (n // (len(edges) + 1)) * len(edges))])
    y = np.clip(y, 1.0, NYT - 1e-3)
    x = rng.uniform(0.5, NX + 0.5, n)
    v = rng.choice([-0.6, 0.6], n)
    ptype = (np.arange(n) % 3 == 0).astype(np.int32)  # tracers and some inertial particles
    return dict(id=(np.arange(n, dtype=np.int32) * 7 + 3)[::-1].copy(), x=x, y=y, u=rng.uniform(-0.1, 0.1, n),
                v=v, type=ptype, invtau=np.where(ptype == 1, 0.05, 0.0))


def _worker(rank, world, heights, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from lagrangianrbnudging_b200 import slabrank
        from tests.slab_standin import StandInSlab

        j0s = np.concatenate([[0], np.cumsum(heights)])
        parts = _particles(240, list(j0s[1:-1] + 1) + [1.0, NYT - 0.5])
        slab = StandInSlab(_params(), int(j0s[rank]), int(heights[rank]), 11, parts, xcap=240)
        r = slabrank.SlabRank(slab, slab.bufs, particles=True)
        for n in (1, 4, 9):
            slabrank.run_distributed(r, n, dist, rank, world)
        held = dict(id=slab.ids.tolist(), P=slab.P.tolist())
        out = [None] * world
        dist.all_gather_object(out, (held, slab.handed, slab.istep))
        if rank == 0:
            ids = np.concatenate([np.asarray(h["id"], np.int32) for h, _, _ in out])
            P = np.concatenate([np.asarray(h["P"]).reshape(9, -1) for h, _, _ in out], axis=1)
            idx = slab._oracle_index(ids)
            same = all(np.array_equal(P[k], slab.orc.pa[f][idx]) for k, f in enumerate(
                ["x", "y", "u", "v", "xo", "yo", "uo", "vo", "invtau"]))
            q.put(("ok", sorted(ids.tolist()) == sorted(parts["id"].tolist()), same,
                   sum(h for _, h, _ in out), {s for _, _, s in out}))
        dist.barrier()
    except Exception as e:  # reported to the test, then the group ends
        q.put(("error", rank, repr(e)))
    finally:
        dist.destroy_process_group()


def _run(heights):
    world = len(heights)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, heights, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
    res = []
    while not q.empty():
        res.append(q.get())
    return res


@pytest.mark.parametrize("heights", [(12, 12), (8, 9, 7)])
def test_slab_ranks_exchange_ghosts_moments_and_particles_over_gloo(heights):
    res = _run(heights)
    errors = [r for r in res if r[0] == "error"]
    assert not errors, errors
    (ok, covered, same, handed, steps), = res
    assert covered, "every particle held by exactly one slab"
    assert same, "particle states equal the oracle's"
    assert handed > 20, "particles crossed the slab boundaries"
    assert steps == {14}


def test_neighbours_and_operation_order():
    from lagrangianrbnudging_b200 import slabrank

    assert slabrank.neighbours(0, 3, False) == (1, None)
    assert slabrank.neighbours(2, 3, False) == (None, 1)
    assert slabrank.neighbours(2, 3, True) == (0, 1)
    assert slabrank.neighbours(0, 1, True) == (0, 0)

    class D:
        isend, irecv = "send", "recv"

        @staticmethod
        def P2POp(op, t, peer):
            return (op, t, peer)

    ex = slabrank.Exchange("mom", "up", "down", "lo", "hi", True)
    # two ranks in a ring: sends (up, down) then receives (lo, hi) to one peer
    assert slabrank.p2p_ops(D, ex, 0, 2) == [("send", "up", 1), ("send", "down", 1), ("recv", "lo", 1),
                                              ("recv", "hi", 1)]
    wall = slabrank.Exchange("ghost", "up", "down", None, "hi", False)
    assert slabrank.p2p_ops(D, wall, 0, 3) == [("send", "up", 1), ("recv", "hi", 1)]


def test_message_layout_matches_the_library():
    import ctypes as C

    from lagrangianrbnudging_b200 import build, lib
    from tests.slab_standin import HEADER, PLANES_OFF, RECORD

    build.build()
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    assert lib().lbrb_slab_particle_format(C.byref(a), C.byref(b), C.byref(c)) == 0
    assert (a.value, b.value, c.value) == (HEADER.itemsize, RECORD.itemsize, PLANES_OFF)
