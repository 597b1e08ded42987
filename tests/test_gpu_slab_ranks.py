"""One process per GPU with particles (lbrb_slab_particles_* and
lagrangianrbnudging_b200.slabrank), with the ranks' exchanges done as
copies between slab handles on one GPU (slabrank.run_local): each slab holds
the particles in its rows, hands the leavers to its neighbours and receives
theirs; states, records and populations equal the whole domain's bit for
bit.  Also the protocol's checks: a message missing from the exchange, a
full hand-off list, calls out of order."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build, slabrank

pytestmark = pytest.mark.gpu

NX, NY = 64, 48


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def params(precision, **kw):
    return dict(**lb.closure(NX, NY, Ra=1e6, Pr=1.0, U=0.1), precision=precision, **kw)


def seed(d, n, s):
    rng = np.random.default_rng(s)
    x = rng.uniform(0.5, NX + 0.5, n)
    y = rng.uniform(1.0, NY, n)
    y[:8] = [1.0, 19.9, 20.0, 20.05, 36.98, 37.0, NY - 0.01, NY - 0.5]  # beside the slab edges and walls
    ptype = (np.arange(n) % 2).astype(np.int32)
    invtau = np.where(ptype == 1, 1.0 / 40.0, 0.0)
    u0 = rng.uniform(-0.02, 0.02, n)
    d.set_particles((np.arange(n, dtype=np.int32) * 5 + 1)[::-1].copy(), x, y, u0, -u0, ptype, invtau)


def developed(precision):
    with lb.Run(**params(precision)) as dev:
        dev.init_conduction(23, 5e-2)
        dev.step(3000)
        return dev.get_populations(), dev.get_moments()


def ranks_of(dom, torch, pairs=False):
    """the slabs as ranks, their work on one stream with the copies between
    them (run the drivers under torch.cuda.stream(dom.stream))"""
    dom.stream = slabrank.bind_stream(dom.slabs, torch)
    return [slabrank.SlabRank(r, slabrank.device_buffers(r, torch), particles=dom.np > 0, pairs=pairs)
            for r in dom.slabs]


def drive(dom, ranks, n, torch):
    with torch.cuda.stream(dom.stream):
        slabrank.run_local(ranks, n)
    torch.cuda.synchronize()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("heights,beta,full", [((20, 17, 11), 0.0, 0), ((20, 17, 11), 0.5, 1),
                                                ((24, 24), 0.5, 0), ((16, 3, 29), 0.0, 1)])
def test_slab_ranks_match_the_whole_domain(precision, heights, beta, full):
    torch = pytest.importorskip("torch")
    npart = 400
    kw = params(precision, nprtcl=npart, noutconfig=7, record_slots=64, beta=beta, record_full=full)
    (f, g), m = developed(precision)
    with lb.Run(**kw) as whole, lb.SlabDomain(heights, **kw) as dom:
        for d in (whole, dom):
            d.set_populations(f, g)
            d.set_moments(m["rho"], m["u"], m["v"], m["T"])
            seed(d, npart, 4)
        y0 = whole.get_particles()["y"]
        ranks = ranks_of(dom, torch)
        for n in (1, 6, 90, 200):
            whole.step(n)
            drive(dom, ranks, n, torch)
            for r in dom.slabs:
                r.sync()
            pw, ps = whole.get_particles(), dom.get_particles()
            for k in pw:
                np.testing.assert_array_equal(ps[k], pw[k])
            sw, rw = whole.drain_records_array()
            ss, rs = dom.drain_records_array()
            np.testing.assert_array_equal(ss, sw)
            np.testing.assert_array_equal(rs, rw)
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)
        assert sum(dom.slab_counts()) == npart
        edges = np.cumsum(heights)[:-1]
        moved = (np.searchsorted(edges, np.floor(y0) - 1, side="right")
                 != np.searchsorted(edges, np.floor(pw["y"]) - 1, side="right"))
        assert moved.sum() > 10, "particles changed slabs"


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_slab_step_in_one_process_holds_particles_by_owner(precision):
    """lbrb_slab_step with particles: the same exchange by peer copies; each
    slab holds only its own particles"""
    npart = 300
    kw = params(precision, nprtcl=npart, noutconfig=5, record_slots=64, beta=0.5)
    (f, g), m = developed(precision)
    with lb.Run(**kw) as whole, lb.SlabDomain((20, 17, 11), **kw) as dom:
        for d in (whole, dom):
            d.set_populations(f, g)
            d.set_moments(m["rho"], m["u"], m["v"], m["T"])
            seed(d, npart, 9)
        counts0 = dom.slab_counts()
        assert sum(counts0) == npart and max(counts0) < npart
        for n in (1, 2, 3, 150):
            whole.step(n)
            dom.step(n)
            pw, ps = whole.get_particles(), dom.get_particles()
            for k in pw:
                np.testing.assert_array_equal(ps[k], pw[k])
            sw, rw = whole.drain_records_array()
            ss, rs = dom.drain_records_array()
            np.testing.assert_array_equal(ss, sw)
            np.testing.assert_array_equal(rs, rw)
        assert sum(dom.slab_counts()) == npart


def test_one_slab_rank_of_the_whole_domain():
    """a single rank: the ring messages go to itself (run_distributed, world 1)"""
    torch = pytest.importorskip("torch")
    npart = 200
    kw = params("fp32", nprtcl=npart, noutconfig=4, record_slots=64)
    (f, g), m = developed("fp32")
    with lb.Run(**kw) as whole, lb.SlabDomain((NY,), **kw) as dom:
        for d in (whole, dom):
            d.set_populations(f, g)
            d.set_moments(m["rho"], m["u"], m["v"], m["T"])
            seed(d, npart, 2)
        (rank,) = ranks_of(dom, torch)
        whole.step(40)
        with torch.cuda.stream(dom.stream):
            slabrank.run_distributed(rank, 40, None, 0, 1)
        torch.cuda.synchronize()
        pw, ps = whole.get_particles(), dom.get_particles()
        for k in pw:
            np.testing.assert_array_equal(ps[k], pw[k])
        np.testing.assert_array_equal(dom.drain_records_array()[1], whole.drain_records_array()[1])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_slab_ranks_two_steps_per_exchange_without_particles(precision):
    torch = pytest.importorskip("torch")
    with lb.Run(**params(precision)) as whole, lb.SlabDomain((20, 17, 11), **params(precision)) as dom:
        whole.init_conduction(19, 3e-2)
        dom.init_conduction(19, 3e-2)
        ranks = ranks_of(dom, torch, pairs=True)
        for n in (1, 8, 33):
            whole.step(n)
            drive(dom, ranks, n, torch)
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)


def test_missing_message_and_full_list_are_reported():
    torch = pytest.importorskip("torch")
    npart = 300
    kw = params("fp32", nprtcl=npart)
    (f, g), m = developed("fp32")
    # a moment message that never arrives: the receiver's header is stale
    with lb.SlabDomain((24, 24), **kw) as dom:
        dom.set_populations(f, g)
        dom.set_moments(m["rho"], m["u"], m["v"], m["T"])
        seed(dom, npart, 3)
        ranks = ranks_of(dom, torch)
        drive(dom, ranks, 3, torch)
        a, b = dom.slabs
        with torch.cuda.stream(dom.stream):
            for r in (a, b):
                r.slab_pack()
            # (the ghost exchange and the step, then no moment exchange)
            bufs = [slabrank.device_buffers(r, torch) for r in (a, b)]
            bufs[1]["ghost_lo"].copy_(bufs[0]["up"])
            bufs[0]["ghost_hi"].copy_(bufs[1]["down"])
            for r in (a, b):
                r.step(1)
                r.slab_moments_pack()
                r.slab_particles_step()
        torch.cuda.synchronize()
        with pytest.raises(lb.LbrbError) as e:
            a.sync()
        assert e.value.code == lb.ERR_CODES["LBRB_ERR_STATE"]
    # a hand-off list of one record while many particles cross
    with lb.SlabDomain((24, 24), **kw) as dom:
        dom.set_populations(f, g)
        dom.set_moments(m["rho"], m["u"], m["v"], m["T"])
        rng = np.random.default_rng(1)
        y = 24.9 + rng.uniform(-0.05, 0.05, npart)  # all beside the inner edge, moving across it
        dom.set_particles(np.arange(npart, dtype=np.int32), rng.uniform(1, NX, npart), y, np.zeros(npart),
                          np.where(np.arange(npart) % 2 == 0, 0.8, -0.8), np.zeros(npart, np.int32),
                          np.zeros(npart), handoff_capacity=1)
        ranks = ranks_of(dom, torch)
        drive(dom, ranks, 2, torch)
        codes = []
        for r in dom.slabs:
            try:
                r.sync()
            except lb.LbrbError as err:
                codes.append(err.code)
        assert lb.ERR_CODES["LBRB_ERR_OVERFLOW"] in codes


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("npart", [0, 150])
def test_slab_ranks_with_bilinear_nudging_match_the_whole_domain(precision, npart):
    """one process per GPU with bilinear nudging (lbrb_slab_nudge after the
    moment exchange): each slab interpolates T at an observation's corners
    from its own rows and the received moment rows, and adds the shares at
    its own corners.  Observations straddle both inner edges and, through
    the periodic wrap of the cell rows, the walls; with and without
    particles (a slab without them holds the moment messages only)."""
    torch = pytest.importorskip("torch")
    nobs, nst = 90, 5
    rng = np.random.default_rng(31)
    ox = rng.uniform(0.0, NX + 1.0, (nst, nobs))
    oy = rng.uniform(0.5, NY + 0.5, (nst, nobs))
    oy[:, :9] = [19.5, 20.0, 20.5, 21.0, 36.2, 37.0, 37.9, 0.7, NY + 0.3]
    oT = rng.uniform(-0.5, 0.5, (nst, nobs))
    kw = params(precision, nudge="bilinear", alpha=0.3, nobs=nobs, obs_cycle=1, nprtcl=npart,
                noutconfig=5 if npart else 0, record_slots=64)
    with lb.Run(**kw) as whole, lb.SlabDomain((20, 17, 11), **kw) as dom:
        for d in (whole, dom):
            d.init_conduction(41, 2e-2)
            d.nudge_obs(1, ox, oy, oT)
            if npart:
                seed(d, npart, 8)
        if not npart:
            for r in dom.slabs:
                r.slab_messages_only()
        dom.stream = slabrank.bind_stream(dom.slabs, torch)
        ranks = [slabrank.SlabRank(r, slabrank.device_buffers(r, torch), particles=npart > 0, nudging=True)
                 for r in dom.slabs]
        for n in (1, 4, 60):
            whole.step(n)
            drive(dom, ranks, n, torch)
            for r in dom.slabs:
                r.sync()
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)
            if npart:
                pw, ps = whole.get_particles(), dom.get_particles()
                for k in pw:
                    np.testing.assert_array_equal(ps[k], pw[k])
                np.testing.assert_array_equal(dom.drain_records_array()[1], whole.drain_records_array()[1])
        # the nudging acted, and a nudged slab does not step on before it ran
        with lb.Run(**dict(kw, nudge="none", nobs=0)) as free:
            free.init_conduction(41, 2e-2)
            if npart:
                seed(free, npart, 8)
            free.step(65)
            assert not np.array_equal(free.get_populations()[1], gw)
        a = dom.slabs[0]
        with torch.cuda.stream(dom.stream):
            a.slab_pack()
            a.step(1)
            a.slab_moments_pack()
            with pytest.raises(lb.LbrbError):
                a.slab_pack()
                a.step(1)  # lbrb_slab_nudge of the last step first


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("heights", [(20, 17, 11), (24, 24)])
def test_slab_ranks_with_particles_two_steps_per_launch(precision, heights):
    """lbrb_step(h, 2) on slabs holding particles: one two-step launch, then
    the particle exchange of each of its steps in turn (the first step's
    receive moves the handle on to the second); odd call lengths end with a
    single step.  States, records (at odd and even steps) and populations
    equal the whole domain's bit for bit."""
    torch = pytest.importorskip("torch")
    npart = 400
    kw = params(precision, nprtcl=npart, noutconfig=7, record_slots=64, beta=0.5, record_full=1)
    (f, g), m = developed(precision)
    with lb.Run(**kw) as whole, lb.SlabDomain(heights, **kw) as dom:
        for d in (whole, dom):
            d.set_populations(f, g)
            d.set_moments(m["rho"], m["u"], m["v"], m["T"])
            seed(d, npart, 5)
        ranks = ranks_of(dom, torch, pairs=True)
        for n in (1, 6, 91, 200):
            whole.step(n)
            drive(dom, ranks, n, torch)
            for r in dom.slabs:
                r.sync()
            pw, ps = whole.get_particles(), dom.get_particles()
            for k in pw:
                np.testing.assert_array_equal(ps[k], pw[k])
            sw, rw = whole.drain_records_array()
            ss, rs = dom.drain_records_array()
            np.testing.assert_array_equal(ss, sw)
            np.testing.assert_array_equal(rs, rw)
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)
        assert sum(dom.slab_counts()) == npart
        # after a two-step launch the handle takes no further step until
        # both steps' particle exchanges have run
        a = dom.slabs[0]
        with torch.cuda.stream(dom.stream):
            a.slab_pack2()
            a.step(2)
            with pytest.raises(lb.LbrbError):
                a.step(1)
