"""One domain over several GPUs, one process per GPU: the per-step exchange
between y-slabs (lbrb_slab_*), as a protocol that a driver carries out.

The reference decomposes its domain over MPI ranks: each step it refreshes
the population halos (pbc, temppart_dump.c:234-250) and hands the particles
that leave a rank's block to the neighbour (toggle_prtcl,
Trajectories/code/mympi2.h:568-760).  Here a rank holds one y-slab (a handle
after lbrb_slab_set) and, per step:

    lbrb_slab_pack                 ghost rows   up -> s+1 lo, down -> s-1 hi
    [lbrb_slab_particles_recv]     (the previous step's hand-off lists)
    lbrb_step(h, 1)
    lbrb_slab_moments_pack         moment rows  up -> s+1 lo, down -> s-1 hi (ring)
    [lbrb_slab_nudge]              (bilinear nudging)
    lbrb_slab_particles_step       hand-off     up -> s+1 lo, down -> s-1 hi (ring)

The hand-off lists of a step travel with the next step's ghost rows (one
batch of point-to-point operations); a call of `steps` ends with their own
exchange and receive, so the slab's particles are complete between calls.
With `pairs`, two steps go per launch (lbrb_slab_pack2, lbrb_step(h, 2)),
the particle exchange of each following in turn (no nudging).

`SlabRank.steps(n)` yields, at each exchange, a list of `Exchange`
requests; a driver fills them and resumes it.  `run_distributed` drives one
rank over torch.distributed point-to-point operations (NCCL on GPUs, gloo on
CPU); `run_local` drives several ranks of one process in lockstep with
copies (slabs on one GPU, or a test).  Message buffers are torch tensors of
bytes: device memory of the handle (`device_buffers`), or host arrays of a
stand-in slab in a CPU test.  On GPUs the handles' work and the exchange
share one stream (`bind_stream`).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable, Iterator


@dataclass
class Exchange:
    """Send `up` to the rank above (it lands in that rank's `lo`) and `down`
    to the rank below (its `hi`).  ring: the ranks form a ring (rank world-1
    sends up to rank 0), else the ends send nothing past the walls and their
    outer buffers are None."""
    name: str
    up: Any
    down: Any
    lo: Any
    hi: Any
    ring: bool


def neighbours(rank: int, world: int, ring: bool):
    """(rank above, rank below), None past a wall"""
    up = (rank + 1) % world if ring or rank + 1 < world else None
    dn = (rank - 1) % world if ring or rank > 0 else None
    return up, dn


def p2p_ops(dist, ex: Exchange, rank: int, world: int) -> list:
    """the point-to-point operations of one exchange.  Sends go first (up,
    then down) and receives after (lo, then hi): with two ranks in a ring
    both neighbours are the same rank, and operations between two ranks match
    in the order they are posted, so `up` lands in the peer's `lo` and
    `down` in its `hi`."""
    up, dn = neighbours(rank, world, ex.ring)
    ops = []
    if up is not None:
        ops.append(dist.P2POp(dist.isend, ex.up, up))
    if dn is not None:
        ops.append(dist.P2POp(dist.isend, ex.down, dn))
    if dn is not None:
        ops.append(dist.P2POp(dist.irecv, ex.lo, dn))
    if up is not None:
        ops.append(dist.P2POp(dist.irecv, ex.hi, up))
    return ops


class SlabRank:
    """The protocol of one slab.  `slab` has the lbrb.Run slab methods
    (slab_pack, slab_pack2, step, slab_moments_pack, slab_nudge,
    slab_particles_step, slab_particles_recv); `bufs` maps the buffer names
    of `device_buffers` to tensors.  particles: the slab holds particles;
    nudging: bilinear nudging (every rank alike; both need the moment
    messages, lbrb_slab_particles_set)."""

    def __init__(self, slab, bufs: dict, particles: bool, pairs: bool = False, nudging: bool = False):
        self.slab, self.b, self.particles, self.nudging = slab, bufs, particles, nudging
        self.pairs = pairs and not nudging
        self.pending = False  # hand-off lists packed, not yet exchanged

    def _ghosts(self, two: bool) -> Exchange:
        k = "2" if two else ""
        b = self.b
        return Exchange("ghost" + k, b["up" + k], b["down" + k], b["ghost_lo" + k], b["ghost_hi" + k], False)

    def _hand(self) -> Exchange:
        b = self.b
        return Exchange("hand", b["hand_up"], b["hand_down"], b["hand_lo"], b["hand_hi"], True)

    def _mom(self) -> Exchange:
        b = self.b
        return Exchange("mom", b["mom_up"], b["mom_down"], b["mom_lo"], b["mom_hi"], True)

    def steps(self, n: int) -> Iterator[list]:
        s = self.slab
        left = int(n)
        while left > 0:
            two = self.pairs and left >= 2
            if two:
                s.slab_pack2()
            else:
                s.slab_pack()
            ex = [self._ghosts(two)]
            if self.pending:
                ex.append(self._hand())
            yield ex
            if self.pending:
                s.slab_particles_recv()
                self.pending = False
            s.step(2 if two else 1)
            left -= 2 if two else 1
            if self.particles or self.nudging:
                # each step of the launch in turn; after a two-step launch the
                # first step's receive moves the handle on to the second step
                for q in range(2 if two else 1):
                    s.slab_moments_pack()
                    yield [self._mom()]
                    if self.nudging:
                        s.slab_nudge()
                    if self.particles:
                        s.slab_particles_step()
                        if two and q == 0:
                            yield [self._hand()]
                            s.slab_particles_recv()
                        else:
                            self.pending = True
        if self.pending:
            yield [self._hand()]
            s.slab_particles_recv()
            self.pending = False


def run_distributed(rank_obj: SlabRank, n: int, dist, rank: int, world: int,
                    local_copy: Callable[[Any, Any], None] | None = None) -> None:
    """n steps of one rank over torch.distributed (every rank calls this with
    the same n).  With one rank the ring exchanges are copies to itself
    (`local_copy(dst, src)`, default dst.copy_(src))."""
    copy = local_copy or (lambda d, s_: d.copy_(s_))
    for exchanges in rank_obj.steps(n):
        ops = []
        for ex in exchanges:
            if world == 1:
                if ex.ring:
                    copy(ex.lo, ex.up)
                    copy(ex.hi, ex.down)
                continue
            ops += p2p_ops(dist, ex, rank, world)
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


def run_local(ranks: list, n: int, local_copy: Callable[[Any, Any], None] | None = None) -> None:
    """n steps of every slab of a domain held in this process, in lockstep:
    each exchange is a copy into the neighbours' buffers"""
    copy = local_copy or (lambda d, s_: d.copy_(s_))
    world = len(ranks)
    gens = [r.steps(n) for r in ranks]
    while True:
        reqs = [next(g, None) for g in gens]
        if all(q is None for q in reqs):
            return
        if any(q is None for q in reqs) or len({len(q) for q in reqs}) != 1:
            raise RuntimeError("slab ranks out of step")
        for e in range(len(reqs[0])):
            for r in range(world):
                ex = reqs[r][e]
                up, dn = neighbours(r, world, ex.ring)
                if up is not None:
                    copy(reqs[up][e].lo, ex.up)
                if dn is not None:
                    copy(reqs[dn][e].hi, ex.down)


def bind_stream(runs, torch, stream=None):
    """Queue every handle's work on one torch stream (a new one of the first
    handle's device by default) and return it.  Run the drivers under
    `torch.cuda.stream(stream)`: the copies between slabs and the NCCL
    operations are then ordered against the handles' kernels.  (A handle
    given stream 0 keeps its own non-blocking stream, which the legacy
    default stream does not order against, so that stream is refused.)"""
    if stream is None:
        stream = torch.cuda.Stream(device=torch.device("cuda", runs[0].p.device))
    if stream.cuda_stream == 0:
        raise ValueError("the slab exchange needs a stream other than the legacy default stream")
    for r in runs:
        r.set_stream(stream.cuda_stream)
    return stream


def device_buffers(run, torch) -> dict:
    """the handle's message buffers as uint8 tensors on its device (views of
    its memory, no copy): ghost rows (up, down, ghost_lo, ghost_hi; the
    two-row blocks with suffix 2; None past a wall) and, with particles, the
    moment and hand-off messages"""
    dev = torch.device("cuda", run.p.device)

    def view(ptr: int, nbytes: int):
        if not ptr:
            return None

        class _Mem:
            __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                        "version": 3, "strides": None}

        return torch.as_tensor(_Mem(), device=dev)

    out = {}
    for two in (False, True):
        ptrs, nb = run.slab_buffers(two)
        k = "2" if two else ""
        for name, p in zip(("up", "down", "ghost_lo", "ghost_hi"), ptrs):
            out[name + k] = view(p, nb)
    try:
        pb = run.slab_particle_buffers()
    except Exception:
        pb = {}
    for name, (p, nb) in pb.items():
        out[name] = view(p, nb)
    return out
