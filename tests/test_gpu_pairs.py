"""Two steps per launch (lb_pair_kernel, lb_march_kernel, lbrb_set_pairs): a
run stepped in pairs ends bit-identical to the same run stepped one launch at
a time --
populations, moments, post-stream populations of the last step, particles
and records -- for every launch shape (tiles and marching strips) and the tuned one, in
both precisions, on
grids whose width and height are not multiples of the tile, with records on
the first and on the second step of a pair, tracers and inertial particles
with the Maxey-Riley stencil and full records, and without particles."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

pytestmark = pytest.mark.gpu

CALLS = (1, 2, 5, 8, 31)  # odd calls end on a single step, even calls on a pair


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def make(precision, nx, ny, nprtcl, beta, full, pairs, shape):
    r = lb.Run(**lb.closure(nx, ny, Ra=1e6, Pr=1.0, U=0.1), precision=precision, nprtcl=nprtcl,
               noutconfig=3 if nprtcl else 0, record_slots=64, beta=beta, record_full=full)
    r.set_graph(0)  # (small grids would otherwise replay graphs of single steps)
    r.set_pairs(pairs)
    if shape >= 0:
        r.set_pair_shape(shape)
    r.init_conduction(29, 3e-2)
    if nprtcl:
        rng = np.random.default_rng(7)
        x = rng.uniform(0.5, nx + 0.5, nprtcl)
        y = rng.uniform(1.0, ny, nprtcl)
        y[:2] = [1.0, ny - 1e-9]
        ptype = (np.arange(nprtcl) % 2).astype(np.int32)
        invtau = np.where(ptype == 1, 1.0 / 25.0, 0.0)
        z = np.zeros(nprtcl)
        r.set_particles(np.arange(nprtcl, dtype=np.int32), x, y, z, z, ptype, invtau)
    return r


def state(r, nprtcl):
    f, g = r.get_populations()
    fp, gp = r.get_poststream()
    out = dict(f=f, g=g, fp=fp, gp=gp, **r.get_moments())
    if nprtcl:
        out.update({"p" + k: v for k, v in r.get_particles().items()})
        s, rec = r.drain_records_array()
        out.update(rec_steps=s, rec=rec)
    return out


NSHAPES = 15  # lbrb_pair_shapes(): 9 tiles, then 6 marching shapes
MARCH = list(range(9, NSHAPES))


def test_shape_count():
    assert lb.Run.pair_shapes() == NSHAPES


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("nprtcl,beta,full", [(0, 0.0, 0), (80, 0.0, 0), (80, 0.5, 1)])
@pytest.mark.parametrize("shape", [-1] + list(range(NSHAPES)))
def test_pairs_equal_single_steps(precision, nprtcl, beta, full, shape):
    nx, ny = 200, 37
    with make(precision, nx, ny, nprtcl, beta, full, 0, -1) as a, \
            make(precision, nx, ny, nprtcl, beta, full, 1, shape) as b:
        for n in CALLS:
            a.step(n)
            b.step(n)
            sa, sb = state(a, nprtcl), state(b, nprtcl)
            for k in sa:
                np.testing.assert_array_equal(sb[k], sa[k], err_msg=k)
        assert a.istep == b.istep == sum(CALLS)
        ps = b.pair_shape()
        assert ps["shape"] == (shape if shape >= 0 else ps["shape"]) and ps["shape"] >= 0
        assert a.pair_shape()["shape"] == -1


@pytest.mark.parametrize("shape", [0, 9, 10, 11])
def test_pairs_on_a_tile_multiple_grid(shape):
    with make("fp32", 64, 48, 40, 0.0, 0, 0, -1) as a, make("fp32", 64, 48, 40, 0.0, 0, 1, shape) as b:
        a.step(100)
        b.step(100)
        sa, sb = state(a, 40), state(b, 40)
        for k in sa:
            np.testing.assert_array_equal(sb[k], sa[k], err_msg=k)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("shape", MARCH)
def test_march_on_many_chunks(precision, shape):
    """a grid tall enough for several chunks per strip and several strips,
    width not a multiple of 32: chunk edges, strip edges and the x wrap"""
    with make(precision, 232, 700, 60, 0.5, 1, 0, -1) as a, make(precision, 232, 700, 60, 0.5, 1, 1, shape) as b:
        for n in (9, 14):
            a.step(n)
            b.step(n)
            sa, sb = state(a, 60), state(b, 60)
            for k in sa:
                np.testing.assert_array_equal(sb[k], sa[k], err_msg=k)


def test_record_ring_overflow_is_reported_at_the_same_step():
    """a pair whose records would overflow the ring runs as single steps"""
    kw = dict(**lb.closure(64, 32, Ra=1e6, Pr=1.0, U=0.1), precision="fp32", nprtcl=16, noutconfig=2,
              record_slots=3)
    for pairs in (0, 1):
        with lb.Run(**kw) as r:
            r.set_graph(0)
            r.set_pairs(pairs)
            r.init_conduction(3, 1e-2)
            r.set_particles(np.arange(16, dtype=np.int32), np.full(16, 10.5), np.linspace(2, 30, 16),
                            np.zeros(16), np.zeros(16), np.zeros(16, np.int32), np.zeros(16))
            with pytest.raises(lb.LbrbError):
                r.step(9)  # records at 2, 4, 6 fill the ring; step 8 overflows
            assert r.istep == 7
            assert r.pending_records() == 3


def test_pair_arguments_checked():
    with lb.Run(**lb.closure(64, 32, Ra=1e6, Pr=1.0, U=0.1), precision="fp32") as r:
        for bad in (-2, 2):
            with pytest.raises(lb.LbrbError):
                r.set_pairs(bad)
        for bad in (-2, NSHAPES):
            with pytest.raises(lb.LbrbError):
                r.set_pair_shape(bad)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_pairs_on_grids_smaller_than_a_tile(precision):
    """8 x 5 nodes: the ring wraps onto the tile itself in x, and every row
    is a wall row or next to one"""
    for shape in (0, 5, 8, *MARCH):
        with make(precision, 8, 5, 6, 0.0, 0, 0, -1) as a, make(precision, 8, 5, 6, 0.0, 0, 1, shape) as b:
            for n in (3, 7):
                a.step(n)
                b.step(n)
                sa, sb = state(a, 6), state(b, 6)
                for k in sa:
                    np.testing.assert_array_equal(sb[k], sa[k], err_msg=f"shape {shape}: {k}")


def test_pairs_are_the_default_above_the_graph_size():
    """a grid of more than 2^20 nodes steps two per launch by default (and
    keeps the result of single launches)"""
    kw = dict(**lb.closure(1040, 1024, Ra=1e6, Pr=1.0, U=0.1), precision="fp32")
    with lb.Run(**kw) as a, lb.Run(**kw) as b:
        a.set_pairs(0)
        for r in (a, b):
            r.init_conduction(2, 1e-2)
            r.step(9)
        assert b.pair_shape()["shape"] >= 0 and a.pair_shape()["shape"] == -1
        ma, mb = a.get_moments(), b.get_moments()
        for k in ma:
            np.testing.assert_array_equal(mb[k], ma[k])


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("shape", [-1, 0, 5, 9, 10])
def test_nudged_pairs_equal_single_steps(precision, shape):
    """bilinear nudging with two steps per launch (step n's innovations
    formed before the launch from T^n pulled from the previous state, added
    to g inside it; step n+1's applied after it): bit-identical to single
    steps, with tracers, inertial particles and records; observations
    repeating over 7 steps, some at the walls and the x wrap"""
    nx, ny, nobs, rows = 200, 37, 150, 7
    rng = np.random.default_rng(11)
    ox = rng.uniform(0.0, nx + 1.0, (rows, nobs))
    oy = rng.uniform(1.0, ny, (rows, nobs))
    ox[:, :3] = [0.2, nx + 0.7, 0.99]
    oy[:, 3:6] = [1.0, ny - 1e-9, 1.5]
    oT = rng.uniform(-0.5, 0.5, (rows, nobs))

    def run(pairs):
        r = lb.Run(**lb.closure(nx, ny, Ra=1e6, Pr=1.0, U=0.1), precision=precision, nprtcl=40, noutconfig=3,
                   record_slots=64, beta=0.5, record_full=1, nudge="bilinear", alpha=0.3, nobs=nobs, obs_cycle=1)
        r.set_pairs(pairs)
        if pairs and shape >= 0:
            r.set_pair_shape(shape)
        r.init_conduction(29, 3e-2)
        x = np.random.default_rng(7).uniform(0.5, nx + 0.5, 40)
        y = np.random.default_rng(8).uniform(1.0, ny, 40)
        ptype = (np.arange(40) % 2).astype(np.int32)
        z = np.zeros(40)
        r.set_particles(np.arange(40, dtype=np.int32), x, y, z, z, ptype, np.where(ptype == 1, 1 / 25.0, 0.0))
        r.nudge_obs(1, ox, oy, oT)
        return r

    with run(0) as a, run(1) as b:
        for n in (1, 2, 5, 8, 31):
            a.step(n)
            b.step(n)
            sa, sb = state(a, 40), state(b, 40)
            for k in sa:
                np.testing.assert_array_equal(sb[k], sa[k], err_msg=k)
        assert b.pair_shape()["shape"] >= 0 and a.pair_shape()["shape"] == -1
