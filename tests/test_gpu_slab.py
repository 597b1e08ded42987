"""One domain cut into y-slabs (lbrb_slab_set / lbrb_slab_step): the slabs
advance exactly as the whole domain in one handle, bit for bit, in both
precisions and with uneven slab heights, particles, their records,
bilinear nudging and adiabatic walls included; box nudging bit for bit against
the reference's own run; the slabs' initial state is the whole domain's; the
height-weighted Nu is the whole domain's.  On one GPU the
slabs are handles on the same device: the exchange is the same peer copy as
across GPUs (cudaMemcpyPeerAsync), ordered by the same events."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build
from tests.golden import cases

pytestmark = pytest.mark.gpu

NX, NY = 64, 48


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def params(precision):
    return dict(**lb.closure(NX, NY, Ra=1e6, Pr=1.0, U=0.1), precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("heights", [(24, 24), (20, 17, 11), (3, 42, 3)])
@pytest.mark.parametrize("shape", [-1, 0, 9, 10])
def test_slabs_advance_as_the_whole_domain(precision, heights, shape):
    """shape: the two-step launch shape of the slabs (-1 tuned; 0 a tile;
    9, 10 marching strips, whose rows beyond an inner boundary come from
    the ghost blocks)"""
    with lb.Run(**params(precision)) as whole, lb.SlabDomain(heights, **params(precision)) as dom:
        if shape >= 0:
            for r in dom.slabs:
                r.set_pair_shape(shape)
        whole.init_conduction(17, 2e-2)
        dom.init_conduction(17, 2e-2)
        fw, gw = whole.get_populations()
        fs, gs = dom.get_populations()
        np.testing.assert_array_equal(fs, fw)
        np.testing.assert_array_equal(gs, gw)
        for n in (1, 37, 300):
            whole.step(n)
            dom.step(n)
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)
        mw, ms = whole.get_moments(), dom.get_moments()
        for k in ("rho", "u", "v", "T"):
            np.testing.assert_array_equal(ms[k], mw[k])
        assert dom.nusselt() == pytest.approx(whole.nusselt(), rel=1e-12, abs=1e-12)


def test_slabs_from_a_developed_state():
    """populations set from a whole-domain state after 2000 steps"""
    with lb.Run(**params("fp32")) as whole, lb.SlabDomain((16, 16, 16), **params("fp32")) as dom:
        whole.init_conduction(5, 5e-2)
        whole.step(2000)
        f, g = whole.get_populations()
        m = whole.get_moments()
        dom.set_populations(f, g)
        dom.set_moments(m["rho"], m["u"], m["v"], m["T"])
        # the whole run's state again from the same host copy (same rounding)
        whole.set_populations(f, g)
        whole.set_moments(m["rho"], m["u"], m["v"], m["T"])
        whole.step(500)
        dom.step(500)
        fw, gw = whole.get_populations()
        fs, gs = dom.get_populations()
        np.testing.assert_array_equal(fs, fw)
        np.testing.assert_array_equal(gs, gw)


def test_slab_mode_rejects_what_it_does_not_cover():
    with lb.Run(**dict(params("fp32"), ny=24)) as r:
        with pytest.raises(lb.LbrbError):
            r._ck(lb.lib().lbrb_slab_set(r.h, 30, NY))  # rows outside the domain
        r._ck(lb.lib().lbrb_slab_set(r.h, 0, NY))
        r.init_conduction(1, 1e-3)
        with pytest.raises(lb.LbrbError):
            r.step(3)  # one step, or two after lbrb_slab_pack2, per boundary exchange
    with lb.Run(**dict(params("fp32"), ny=24)) as r:
        r.slab_set(0, NY)
        r.init_conduction(1, 1e-3)
        with pytest.raises(lb.LbrbError):
            r.step(2)  # two steps need lbrb_slab_pack2 first
    with lb.Run(**dict(params("fp32"), ny=24, nprtcl=8)) as r:
        with pytest.raises(lb.LbrbError):
            r.slab_set(0, NY)  # a slab holds its own particles (lbrb_slab_particles_set)
    with lb.Run(**dict(params("fp32"), ny=24)) as r:
        r.slab_set(0, NY)
        r.init_conduction(1, 1e-3)
        with pytest.raises(lb.LbrbError):
            r.slab_particles_step()  # no particles set
        r.slab_particles_set(np.arange(8, dtype=np.int32), np.full(8, 5.0), np.linspace(1.5, 40.0, 8),
                             np.zeros(8), np.zeros(8), np.zeros(8, np.int32), np.zeros(8))
        assert r.slab_particles_count() == 5  # (y in the whole domain: cells in rows 0-23)
        with pytest.raises(lb.LbrbError):
            r.slab_moments_pack()  # after the slab's step
        r.slab_pack()
        r.step(1)
        with pytest.raises(lb.LbrbError):
            r.slab_particles_step()  # after the moment pack (and its exchange)
        with pytest.raises(lb.LbrbError):
            r.step(1)  # the particles of the last step first
    with pytest.raises(ValueError):
        lb.SlabDomain((20, 20), **params("fp32"))  # heights must add up to ny
    with lb.SlabDomain((24, 24), **params("fp32")) as dom:
        dom.init_conduction(1, 1e-3)
        rev = (lb.C.c_void_p * 2)(dom.slabs[1].h, dom.slabs[0].h)
        assert lb.ERRORS[lb.lib().lbrb_slab_step(rev, 2, 1)] == "LBRB_ERR_ARG"  # slabs out of order


def seed_particles(run, n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.5, NX + 0.5, n)
    y = rng.uniform(1.0, NY, n)
    y[:6] = [1.0, 20.5, 21.0, 36.99, 37.0, NY - 0.01]  # on and beside the slab boundaries and walls
    ptype = (np.arange(n) % 2).astype(np.int32)  # tracers and inertial particles
    invtau = np.where(ptype == 1, 1.0 / 40.0, 0.0)
    u0 = rng.uniform(-0.01, 0.01, n)
    run.set_particles(np.arange(n, dtype=np.int32)[::-1].copy(), x, y, u0, -u0, ptype, invtau)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("beta,full", [(0.0, 0), (0.5, 1)])
def test_slab_particles_and_records_match_the_whole_domain(precision, beta, full):
    """particles cross the inner boundaries of three uneven slabs; states and
    records equal the whole domain's bit for bit"""
    npart = 300
    kw = dict(params(precision), nprtcl=npart, noutconfig=7, record_slots=64, beta=beta, record_full=full)
    with lb.Run(**params(precision)) as dev:  # a developed flow (no particles)
        dev.init_conduction(23, 5e-2)
        dev.step(3000)
        f, g = dev.get_populations()
        m = dev.get_moments()
    with lb.Run(**kw) as whole, lb.SlabDomain((20, 17, 11), **kw) as dom:
        for d in (whole, dom):
            d.set_populations(f, g)
            d.set_moments(m["rho"], m["u"], m["v"], m["T"])
        seed_particles(whole, npart, 4)
        seed_particles(dom, npart, 4)
        y0 = whole.get_particles()["y"]
        for n in (1, 6, 90, 300):
            whole.step(n)
            dom.step(n)
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
        assert dom.istep == whole.istep
        # the particles did change slabs
        edges = np.array([20, 37])
        moved = np.searchsorted(edges, y0 - 1, side="right") != np.searchsorted(edges, pw["y"] - 1, side="right")
        assert moved.sum() > 10


def test_slab_particle_record_ring_overflow_is_reported():
    kw = dict(params("fp32"), nprtcl=16, noutconfig=2, record_slots=2)
    with lb.SlabDomain((24, 24), **kw) as dom:
        dom.init_conduction(3, 1e-2)
        seed_particles(dom, 16, 1)
        dom.step(4)
        assert dom.pending_records() == 2
        with pytest.raises(lb.LbrbError):
            dom.step(2)
        steps, _ = dom.drain_records_array()
        assert list(steps) == [2, 4]
        dom.step(2)
        assert dom.pending_records() == 1


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("npart", [0, 120])
def test_slab_bilinear_nudging_matches_the_whole_domain(precision, npart):
    """observations cycling over 5 steps, cells straddling the inner
    boundaries among them; with and without particles"""
    nobs, nst = 90, 5
    rng = np.random.default_rng(31)
    ox = rng.uniform(0.0, NX + 1.0, (nst, nobs))
    oy = rng.uniform(0.5, NY + 0.5, (nst, nobs))
    oy[:, :8] = [19.5, 20.0, 20.5, 21.0, 36.2, 37.0, 37.9, 0.7]  # cells across the slab edges and the wall
    oT = rng.uniform(-0.5, 0.5, (nst, nobs))
    kw = dict(params(precision), nudge="bilinear", alpha=0.3, nobs=nobs, obs_cycle=1, nprtcl=npart,
              noutconfig=5 if npart else 0, record_slots=64)
    with lb.Run(**kw) as whole, lb.SlabDomain((20, 17, 11), **kw) as dom:
        for d in (whole, dom):
            d.init_conduction(41, 2e-2)
            d.nudge_obs(1, ox, oy, oT)
            if npart:
                seed_particles(d, npart, 8)
        for n in (1, 4, 60):
            whole.step(n)
            dom.step(n)
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)
            mw, ms = whole.get_moments(), dom.get_moments()
            for k in ("rho", "u", "v", "T"):
                np.testing.assert_array_equal(ms[k], mw[k])
            if npart:
                pw, ps = whole.get_particles(), dom.get_particles()
                for k in pw:
                    np.testing.assert_array_equal(ps[k], pw[k])
                sw, rw = whole.drain_records_array()
                ss, rs = dom.drain_records_array()
                np.testing.assert_array_equal(ss, sw)
                np.testing.assert_array_equal(rs, rw)
        # the nudging did act: without it the state differs
        with lb.Run(**dict(kw, nudge="none", nobs=0)) as free:
            free.init_conduction(41, 2e-2)
            if npart:
                seed_particles(free, npart, 8)
            free.step(65)
            assert not np.array_equal(free.get_moments()["T"], mw["T"])


def cudart():
    """the CUDA runtime, for device-to-device copies standing in for the
    neighbour sends of one process per GPU"""
    import ctypes as C
    for name in ("/usr/local/cuda/lib64/libcudart.so", "libcudart.so", "libcudart.so.12"):
        try:
            L = C.CDLL(name)
            break
        except OSError:
            continue
    L.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    L.cudaMemcpy.restype = C.c_int
    return L


def exchange(dom, two):
    """what each rank of one process per GPU does: pack its boundary rows,
    then send `up` to the slab above's ghost_lo and `down` to the slab
    below's ghost_hi (here copies between handles of one process)"""
    import ctypes as C
    L, rt = lb.lib(), cudart()
    pack = L.lbrb_slab_pack2 if two else L.lbrb_slab_pack
    bufs_of = L.lbrb_slab_buffers2 if two else L.lbrb_slab_buffers
    nbytes = (L.lbrb_slab_ghost2_bytes if two else L.lbrb_slab_ghost_bytes)(dom.slabs[0].h)
    bufs = []
    for r in dom.slabs:
        r._ck(pack(r.h))
        b = [C.c_void_p() for _ in range(4)]  # up, down, ghost_lo, ghost_hi
        r._ck(bufs_of(r.h, *[C.byref(x) for x in b]))
        bufs.append(b)
    for r in dom.slabs:
        r.sync()
    n = len(dom.slabs)
    for s in range(n):
        if s + 1 < n:
            assert rt.cudaMemcpy(bufs[s + 1][2], bufs[s][0], nbytes, 3) == 0
        if s > 0:
            assert rt.cudaMemcpy(bufs[s - 1][3], bufs[s][1], nbytes, 3) == 0
    # a device-to-device cudaMemcpy may return before the copy ends, and the
    # handles' streams do not wait for the legacy stream: finish the copies
    # before any slab steps (a rank's NCCL recv on its stream orders this)
    assert rt.cudaDeviceSynchronize() == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_one_process_per_gpu_exchange(precision):
    """the exchange a rank does over NCCL, done here with copies: one step per
    exchange (lbrb_slab_pack, lbrb_step(h, 1)) and two steps per exchange
    (lbrb_slab_pack2, lbrb_step(h, 2)) both give the whole domain's state"""
    with lb.Run(**params(precision)) as whole, lb.SlabDomain((20, 17, 11), **params(precision)) as dom:
        whole.init_conduction(19, 3e-2)
        dom.init_conduction(19, 3e-2)
        for two, calls in ((False, 9), (True, 12), (False, 3), (True, 5)):
            for _ in range(calls):
                exchange(dom, two)
                for r in dom.slabs:
                    r.step(2 if two else 1)
            whole.step(calls * (2 if two else 1))
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)
            mw, ms = whole.get_moments(), dom.get_moments()
            for k in ("rho", "u", "v", "T"):
                np.testing.assert_array_equal(ms[k], mw[k])
        with pytest.raises(lb.LbrbError):
            dom.slabs[0].step(3)  # one or two steps per exchange
        # two steps need this slab's lbrb_slab_pack2 since its last step
        with pytest.raises(lb.LbrbError):
            dom.slabs[0].step(2)
        exchange(dom, False)  # a one-step pack does not count
        with pytest.raises(lb.LbrbError):
            dom.slabs[0].step(2)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_slabs_with_adiabatic_walls_advance_as_the_whole_domain(precision):
    """adiabatic T walls (the nudging run's) hold at the domain's walls only;
    inner slab edges take ghost rows"""
    kw = dict(params(precision), twall="adiabatic")
    with lb.Run(**kw) as whole, lb.SlabDomain((20, 17, 11), **kw) as dom:
        whole.init_conduction(17, 2e-2)
        dom.init_conduction(17, 2e-2)
        for n in (1, 37, 300):
            whole.step(n)
            dom.step(n)
            fw, gw = whole.get_populations()
            fs, gs = dom.get_populations()
            np.testing.assert_array_equal(fs, fw)
            np.testing.assert_array_equal(gs, gw)


@pytest.mark.parametrize("name", list(cases.NUDGE_CASES))
@pytest.mark.parametrize("heights,protocol", [((12, 11, 9), "slab_step"), ((8, 8, 8, 8), "slab_step"),
                                              ((16, 16), "ranks")])
def test_slab_box_nudging_bit_exact_vs_reference(name, heights, protocol):
    """the reference's box nudging (FP64, adiabatic walls) on y-slabs, as the
    reference runs it over ranks in y: every slab takes all observations and
    keeps the running means of the boxes' nodes in its own rows.  Populations
    and moments equal the reference's own run bit for bit, through
    lbrb_slab_step and through the one-process-per-GPU protocol (box nudging
    needs no exchange beyond the ghost rows)."""
    c = cases.nudge_case(name)
    z = cases.load_golden(name)
    st = cases.nudge_initial_state(c)
    kw = dict(**c["base"], precision="fp64", twall="adiabatic", nudge="refbox", alpha=c["alpha"],
              ntempread=c["ntempread"], nobs=c["nprtcl"])
    with lb.SlabDomain(heights, **kw) as dom:
        dom.set_populations(st["f"], st["g"])
        dom.set_moments(st["rho"], st["u"], st["v"], st["T"])
        io = c["init_obs"]
        dom.nudge_init(io["x"], io["y"], io["T"], io["id"])
        nt = c["ntempread"]
        if protocol == "ranks":
            torch = pytest.importorskip("torch")
            from lagrangianrbnudging_b200 import slabrank
            stream = slabrank.bind_stream(dom.slabs, torch)
            ranks = [slabrank.SlabRank(r, slabrank.device_buffers(r, torch), particles=False) for r in dom.slabs]
        for s in range(1, c["nsteps"] + 1):
            if s % nt == 1:
                d = c["files"][s + nt - 1]
                dom.nudge_load(d["x"], d["y"], d["id"], d["temp"])
            if protocol == "ranks":
                with torch.cuda.stream(stream):
                    slabrank.run_local(ranks, 1)
                torch.cuda.synchronize()
            else:
                dom.step(1)
        for r in dom.slabs:
            r.sync()
        f, g = dom.get_populations()
        m = dom.get_moments()
    np.testing.assert_array_equal(f, z["f"])
    np.testing.assert_array_equal(g, z["g"])
    s = c["nsteps"]
    np.testing.assert_array_equal(m["T"], z[f"snap{s}_T"])
    np.testing.assert_array_equal(m["u"], z[f"snap{s}_u"])
    np.testing.assert_array_equal(m["v"], z[f"snap{s}_v"])
