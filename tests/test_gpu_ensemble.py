"""The ensemble (lbrb_ensemble_*): members of uneven grid size, closure,
particles and nudging advanced by one launch per phase of the step, or two
steps per launch (a marching or tile kernel over all members, nudged
members included), replayed from CUDA graphs, end bit-identical to the same handles
advanced alone by lbrb_step -- whatever the launch variant, with or without
the graphs, and with per-member steps in between."""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build

pytestmark = pytest.mark.gpu

# uneven members: grid, Rayleigh number, nudging, particles (mixed types)
SPECS = [
    dict(nx=64, ny=32, Ra=1e5, alpha=0.0, nprtcl=100, seed=1),
    dict(nx=128, ny=64, Ra=3e5, alpha=0.1, nprtcl=256, seed=2),
    dict(nx=96, ny=48, Ra=2e5, alpha=0.1, nprtcl=0, seed=3),
    dict(nx=256, ny=24, Ra=1e6, alpha=0.0, nprtcl=300, seed=4),
]
NOBS, OBS_ROWS = 64, 5


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def make_member(spec, precision):
    nx, ny = spec["nx"], spec["ny"]
    kw = dict(**lb.closure(nx, ny, Ra=spec["Ra"], Pr=1.0, U=0.1), precision=precision,
              nprtcl=spec["nprtcl"], beta=0.1)
    if spec["alpha"] > 0:
        kw.update(nudge="bilinear", alpha=spec["alpha"], nobs=NOBS, obs_cycle=1)
    r = lb.Run(**kw)
    r.init_conduction(spec["seed"], 1e-2)
    rng = np.random.default_rng(100 + spec["seed"])
    n = spec["nprtcl"]
    if n:
        x = rng.uniform(0.5, nx + 0.5, n)
        y = rng.uniform(1.0, ny, n)
        ptype = (np.arange(n) % 2).astype(np.int32)
        r.set_particles(np.arange(n, dtype=np.int32), x, y, np.zeros(n), np.zeros(n), ptype,
                        np.full(n, 1.0 / 40.0))
    if spec["alpha"] > 0:
        ox = rng.uniform(0.5, nx + 0.5, (OBS_ROWS, NOBS))
        oy = rng.uniform(1.0, ny, (OBS_ROWS, NOBS))
        oT = 0.5 - (oy - 0.5) / ny + 0.05 * rng.standard_normal((OBS_ROWS, NOBS))
        r.nudge_obs(1, ox, oy, oT)
    return r


def snapshot(r):
    f, g = r.get_populations()
    out = {"f": f, "g": g, **r.get_moments()}
    if r.np:
        out.update({"p" + k: v for k, v in r.get_particles().items()})
    return out


def assert_same(a, b):
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("pairs", [1, 0])
def test_ensemble_matches_members_stepped_alone(precision, pairs):
    """pairs: 20 steps = 9 pairs (one graph of 6 pairs, 3 direct) + 2 single
    steps, then 7 = 3 pairs + 1; singles: 3 graph replays of 6 steps, then
    single steps"""
    A = [make_member(s, precision) for s in SPECS]
    B = [make_member(s, precision) for s in SPECS]
    with lb.Ensemble(A) as ens:
        ens.set_pairs(pairs)
        ens.step(20)
        ens.sync()
        for r in B:
            r.step(20)
        for a, b in zip(A, B):
            assert a.istep == b.istep == 20
            assert_same(snapshot(a), snapshot(b))
        ens.step(7)
        ens.sync()
    for r in B:
        r.step(7)
    for a, b in zip(A, B):
        assert_same(snapshot(a), snapshot(b))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_every_pair_variant_matches_members_stepped_alone(precision):
    """each two-step launch variant (marching groups, 32 x 8 and 30 x 8
    tiles, ragged at the members' edges), 14 steps = 6 pairs from the graph
    + 1 pair + 1 single step"""
    B = [make_member(s, precision) for s in SPECS]
    for r in B:
        r.step(14)
    ref = [snapshot(b) for b in B]
    for v in range(lb.Ensemble.pair_variants()):
        A = [make_member(s, precision) for s in SPECS]
        with lb.Ensemble(A) as ens:
            ens.set_pairs(1)
            ens.set_pair_variant(v)
            ens.step(14)
            ens.sync()
            p = ens.pairs()
        assert p["variant"] == v and p["tuned_ms"] == 0
        for a, b in zip(A, ref):
            assert_same(snapshot(a), b)


def test_every_launch_variant_gives_identical_results():
    ref = None
    for v in range(lb.Ensemble.nvariants()):
        A = [make_member(s, "fp32") for s in SPECS]
        with lb.Ensemble(A) as ens:
            ens.set_pairs(0)  # (every step in the variant under test)
            ens.set_schedule(v)
            ens.step(9)
            ens.sync()
            assert ens.schedule()["variant"] == v
        snap = [snapshot(a) for a in A]
        if ref is None:
            ref = snap
        else:
            for x, y in zip(snap, ref):
                assert_same(x, y)


def test_members_step_alone_between_ensemble_steps():
    A = [make_member(s, "fp32") for s in SPECS]
    B = [make_member(s, "fp32") for s in SPECS]
    with lb.Ensemble(A) as ens:
        ens.step(5)
        A[1].step(3)  # the member's own stream is ordered after the ensemble
        ens.step(8)
        ens.sync()
    B[1].step(16)
    for i, b in enumerate(B):
        if i != 1:
            b.step(13)
    for a, b in zip(A, B):
        assert_same(snapshot(a), snapshot(b))


def test_timing_mode_launches_directly_with_same_results():
    A = [make_member(s, "fp32") for s in SPECS]
    B = [make_member(s, "fp32") for s in SPECS]
    with lb.Ensemble(A) as ea, lb.Ensemble(B) as eb:
        eb.set_schedule(ea_variant := 4)
        ea.set_schedule(ea_variant)
        ea.set_pairs(0)
        eb.set_pairs(0)
        ea.set_timing(True)
        ea.step(14)
        t = ea.get_timing()
        eb.step(14)
        ea.sync()
        eb.sync()
    assert t["lb_step"][1] == 14 and t["aux"][1] == 14 and t["apply"][1] == 14
    assert t["lb_step"][0] > 0
    for a, b in zip(A, B):
        assert_same(snapshot(a), snapshot(b))


def test_pair_timing_mode_launches_directly_with_same_results():
    """14 steps in pairs: 6 pairs (pre-innovations, marching launch, aux,
    apply each) + 2 single steps, launched directly"""
    A = [make_member(s, "fp32") for s in SPECS]
    B = [make_member(s, "fp32") for s in SPECS]
    with lb.Ensemble(A) as ea, lb.Ensemble(B) as eb:
        ea.set_timing(True)
        ea.step(14)
        t = ea.get_timing()
        eb.step(14)
        ea.sync()
        eb.sync()
        p = ea.pairs()
    assert p["mode"] == -1 and p["rows"] in (6, 8) and p["tuned_ms"] > 0
    assert 0 <= p["variant"] < lb.Ensemble.pair_variants() and p["tile_cols"] in (0, 30, 32)
    assert t["lb_step"][1] == 8 and t["aux"][1] == 8 and t["apply"][1] == 2 * 6 + 2
    for a, b in zip(A, B):
        assert_same(snapshot(a), snapshot(b))


def test_ensemble_pairs_match_single_steps_over_many_calls():
    """calls of odd and even lengths (a pair never takes a call's last step)"""
    A = [make_member(s, "fp32") for s in SPECS]
    B = [make_member(s, "fp32") for s in SPECS]
    with lb.Ensemble(A) as ea, lb.Ensemble(B) as eb:
        eb.set_pairs(0)
        for n in (1, 2, 3, 4, 13, 26):
            ea.step(n)
            eb.step(n)
        ea.sync()
        eb.sync()
    for a, b in zip(A, B):
        assert_same(snapshot(a), snapshot(b))


def test_ensemble_autotuner_picks_a_variant():
    A = [make_member(s, "fp32") for s in SPECS]
    with lb.Ensemble(A) as ens:
        ens.step(3)
        ens.sync()
        s = ens.schedule()
    assert 0 <= s["variant"] < lb.Ensemble.nvariants() and s["tuned_ms"] > 0


def test_ensemble_rejects_incompatible_members():
    a = make_member(SPECS[0], "fp32")
    b = make_member(SPECS[1], "fp64")
    with pytest.raises(lb.LbrbError) as ei:
        lb.Ensemble([a, b])
    assert ei.value.code == -1
    rec = lb.Run(**lb.closure(64, 32, Ra=1e5, Pr=1.0, U=0.1), precision="fp32", nprtcl=8,
                 noutconfig=5)
    with pytest.raises(lb.LbrbError) as ei:
        lb.Ensemble([a, rec])
    assert ei.value.code == -9


def test_ensemble_reports_missing_observations():
    spec = dict(SPECS[1])
    r = make_member(spec, "fp32")
    r2 = lb.Run(**lb.closure(64, 32, Ra=1e5, Pr=1.0, U=0.1), precision="fp32", nudge="bilinear",
                alpha=0.1, nobs=NOBS)
    r2.init_conduction(5, 1e-2)
    rng = np.random.default_rng(0)
    r2.nudge_obs(1, rng.uniform(1, 60, (3, NOBS)), rng.uniform(1, 30, (3, NOBS)),
                 np.zeros((3, NOBS)))
    with lb.Ensemble([r, r2]) as ens:
        ens.step(3)  # covered
        with pytest.raises(lb.LbrbError) as ei:
            ens.step(1)  # step 4 has no observation row and the series does not repeat
        assert ei.value.code == -4
        ens.sync()
