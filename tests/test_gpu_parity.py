"""Parity of the CUDA path (liblbrb.so through the C-ABI) with the reference.

FP64 path: bit-identical to the reference (golden fixtures made by running the
reference's own sources) and to the oracle, including particle records.
FP32 shifted path: within the tolerances written in each test.
"""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build
from oracle.oracle import Oracle
from tests.golden import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def traj_run(c, precision="fp64", **extra):
    kw = dict(c["base"], precision=precision, twall="dirichlet", nudge="none", beta=c["beta"],
              nprtcl=c["nprtcl"], noutconfig=c["noutconfig"], record_full=True, record_slots=64)
    kw.update(extra)
    r = lb.Run(**kw)
    r.set_populations(c["f0"], c["g0"])
    r.moments_from_pre(c["f0"], c["g0"])
    r.set_particles(c["ids"], c["px"], c["py"], c["pu"], c["pv"], c["ptype"], c["invtau"])
    return r


@pytest.mark.parametrize("launch", ["default", "pairs", "single"])
@pytest.mark.parametrize("name", list(cases.TRAJ_CASES))
def test_fp64_trajectories_bit_exact_vs_reference(name, launch):
    """default: graph replays of one-step launches on these small grids;
    pairs: two steps per fused launch (and per particle launch); single: one
    launch per step, no graphs"""
    c = cases.traj_case(name)
    z = cases.load_golden(name)
    with traj_run(c) as r:
        if launch != "default":
            r.set_graph(0)
            r.set_pairs(1 if launch == "pairs" else 0)
        r.step(c["nsteps"])
        r.sync()
        f, g = r.get_populations()
        recs = r.drain_records()
    np.testing.assert_array_equal(f, z["f"])
    np.testing.assert_array_equal(g, z["g"])
    steps = sorted({int(k[3:].split("_")[0]) for k in z if k.startswith("rec")})
    assert sorted(recs) == steps
    for s in steps:
        rr = recs[s]
        order = np.argsort(rr["id"])
        np.testing.assert_array_equal(rr["id"][order], z[f"rec{s}_id"])
        for k in lb.REC_NAMES:
            np.testing.assert_array_equal(rr[k][order], z[f"rec{s}_{k}"], err_msg=f"step {s} {k}")


def test_fp64_moments_particles_energy_match_oracle():
    c = cases.traj_case("traj_inertial")
    o = cases.run_oracle_traj(c)
    with traj_run(c) as r:
        r.step(c["nsteps"])
        r.sync()
        m = r.get_moments()
        pr = r.get_particles()
        ke, tm = r.energy()
        nu = r.nusselt()
    for k in ("rho", "u", "v", "T"):
        np.testing.assert_array_equal(m[k], o[k])
    np.testing.assert_array_equal(pr["x"], o["px"])
    np.testing.assert_array_equal(pr["y"], o["py"])
    # compensated sums vs the reference's running sums: 1e-12 relative
    assert abs(ke - o["energy"][0]) <= 1e-12 * abs(o["energy"][0])
    assert abs(tm - o["energy"][1]) <= 1e-12 * max(abs(o["energy"][1]), 1e-12)
    oo = Oracle(c["params"], 0)
    oo.rho[:], oo.u[:], oo.v[:], oo.T[:] = o["rho"], o["u"], o["v"], o["T"]
    assert abs(nu - oo.nusselt()) <= 1e-12 * abs(oo.nusselt())


@pytest.mark.parametrize("name", list(cases.NUDGE_CASES))
def test_fp64_box_nudging_bit_exact_vs_reference(name):
    c = cases.nudge_case(name)
    z = cases.load_golden(name)
    st = cases.nudge_initial_state(c)
    with lb.Run(**c["base"], precision="fp64", twall="adiabatic", nudge="refbox",
                alpha=c["alpha"], ntempread=c["ntempread"], nobs=c["nprtcl"]) as r:
        r.set_populations(st["f"], st["g"])
        r.set_moments(st["rho"], st["u"], st["v"], st["T"])
        io = c["init_obs"]
        r.nudge_init(io["x"], io["y"], io["T"], io["id"])
        nt = c["ntempread"]
        for s in range(1, c["nsteps"] + 1):
            if s % nt == 1:
                d = c["files"][s + nt - 1]
                r.nudge_load(d["x"], d["y"], d["id"], d["temp"])
            r.step(1)
        r.sync()
        f, g = r.get_populations()
        m = r.get_moments()
    np.testing.assert_array_equal(f, z["f"])
    np.testing.assert_array_equal(g, z["g"])
    s = c["nsteps"]
    np.testing.assert_array_equal(m["T"], z[f"snap{s}_T"])
    np.testing.assert_array_equal(m["u"], z[f"snap{s}_u"])
    np.testing.assert_array_equal(m["v"], z[f"snap{s}_v"])


def _check_profile(p, o):
    """lbrb_profile against the oracle: compensated sums against the
    reference's running sums, so 1e-12 relative, with an absolute floor of
    1e-15 for means that cancel to about zero (u, v over a row)"""
    np.testing.assert_allclose(p[:, :8], o[:, :8], rtol=1e-12, atol=1e-15)
    # the row Nusselt number divides by kappa dT / ny
    np.testing.assert_allclose(p[:, 8], o[:, 8], rtol=1e-10, atol=1e-10)


def test_fp64_profile_matches_oracle_trajectories():
    c = cases.traj_case("traj_wide")
    o = Oracle(c["params"], c["nprtcl"])
    o.f[:] = c["f0"]
    o.g[:] = c["g0"]
    o.moments_from_pre(c["f0"], c["g0"])
    o.set_particles(c["ids"], c["px"], c["py"], c["pu"], c["pv"], c["ptype"], c["invtau"])
    with traj_run(c) as r:
        for s in range(1, c["nsteps"] + 1):
            o.step(s)
            o.record()
            if s % 40 == 0:
                r.step(40)
                r.sync()
                _check_profile(r.profile(), o.profile())


@pytest.mark.parametrize("name", list(cases.NUDGE_CASES))
def test_fp64_profile_matches_oracle_box_nudging(name):
    """the whole-domain profile of a box-nudged run (above the top row, the
    periodic halo row without the 1/2 nud_term, as the reference forms it)"""
    c = cases.nudge_case(name)
    out = cases.run_oracle_nudge(c, ranks_y=1)
    st = cases.nudge_initial_state(c)
    with lb.Run(**c["base"], precision="fp64", twall="adiabatic", nudge="refbox",
                alpha=c["alpha"], ntempread=c["ntempread"], nobs=c["nprtcl"]) as r:
        r.set_populations(st["f"], st["g"])
        r.set_moments(st["rho"], st["u"], st["v"], st["T"])
        io = c["init_obs"]
        r.nudge_init(io["x"], io["y"], io["T"], io["id"])
        nt = c["ntempread"]
        for s in range(1, c["nsteps"] + 1):
            if s % nt == 1:
                d = c["files"][s + nt - 1]
                r.nudge_load(d["x"], d["y"], d["id"], d["temp"])
            r.step(1)
            if s in out["profiles"]:
                r.sync()
                _check_profile(r.profile(), out["profiles"][s])


def test_init_conduction_matches_oracle():
    base = lb.closure(96, 48, Ra=1e6, Pr=1.0, U=0.1)
    o = Oracle(dict(base), 0)
    o.init_conduction(seed=12345, noise=1e-3)
    with lb.Run(**base, precision="fp64") as r:
        r.init_conduction(12345, 1e-3)
        f, g = r.get_populations()
        m = r.get_moments()
    np.testing.assert_array_equal(f, o.f)
    np.testing.assert_array_equal(g, o.g)
    for k, a in (("rho", o.rho), ("u", o.u), ("v", o.v), ("T", o.T)):
        np.testing.assert_array_equal(m[k], a)


def test_reference_layout_roundtrip_and_halo():
    c = cases.traj_case("traj_tracer")
    nx, ny = c["nx"], c["ny"]
    with lb.Run(**c["base"], precision="fp64") as r:
        ref = np.zeros((nx + 2, ny + 2, 9))
        ref[1:-1, 1:-1, :] = np.transpose(c["f0"], (2, 1, 0))
        r.set_populations(ref, ref, layout="ref")
        f, g = r.get_populations(layout="soa")
        np.testing.assert_array_equal(f, c["f0"])
        fr, _ = r.get_populations(layout="ref")
    np.testing.assert_array_equal(fr[1:-1, 1:-1], ref[1:-1, 1:-1])
    # halo filled periodically in x and y (as pbc leaves it)
    np.testing.assert_array_equal(fr[0, 1:-1], fr[nx, 1:-1])
    np.testing.assert_array_equal(fr[nx + 1, 1:-1], fr[1, 1:-1])
    np.testing.assert_array_equal(fr[:, 0], fr[:, ny])
    np.testing.assert_array_equal(fr[:, ny + 1], fr[:, 1])


@pytest.mark.parametrize("launch", ["single", "pairs"])
@pytest.mark.parametrize("shape", [-1, 0, 9])
def test_fp64_bilinear_nudging_matches_oracle(launch, shape):
    """single: one launch per step; pairs: two steps per launch, step n's
    innovations formed before the launch and added inside it (shape -1
    tuned, 0 a tile, 9 a marching strip)"""
    if launch == "single" and shape != -1:
        pytest.skip("the launch shape applies to pairs")
    nx, ny, nobs, K = 64, 32, 200, 40
    base = lb.closure(nx, ny, Ra=1e5, Pr=1.0, U=0.1)
    rng = np.random.default_rng(5)
    ox = rng.uniform(0.0, nx, (K, nobs))
    oy = rng.uniform(1.0, ny, (K, nobs))
    oT = rng.uniform(-0.5, 0.5, (K, nobs))
    o = Oracle(dict(base, nudge="bilinear", alpha=0.1), 0)
    o.init_conduction(seed=3, noise=1e-2)
    with lb.Run(**base, precision="fp64", nudge="bilinear", alpha=0.1, nobs=nobs) as r:
        r.set_pairs(1 if launch == "pairs" else 0)
        if shape >= 0:
            r.set_pair_shape(shape)
        r.init_conduction(3, 1e-2)
        r.nudge_obs(1, ox, oy, oT)
        r.step(K)
        r.sync()
        f, g = r.get_populations()
    for s in range(1, K + 1):
        o.nudge_obs(ox[s - 1], oy[s - 1], oT[s - 1])
        o.step(s)
    np.testing.assert_array_equal(f, o.f)
    np.testing.assert_array_equal(g, o.g)


def test_fp64_large_grid_one_step_bit_exact():
    """Many chunks per row and a row length that is not a multiple of the warp
    chunk: 1000x260, 3 steps against the oracle."""
    base = lb.closure(1000, 260, Ra=1e7, Pr=1.0, U=0.1)
    o = Oracle(dict(base), 0)
    o.init_conduction(seed=99, noise=1e-2)
    with lb.Run(**base, precision="fp64") as r:
        r.init_conduction(99, 1e-2)
        r.step(3)
        f, g = r.get_populations()
        m = r.get_moments()
    for s in range(1, 4):
        o.step(s)
    np.testing.assert_array_equal(f, o.f)
    np.testing.assert_array_equal(g, o.g)
    np.testing.assert_array_equal(m["T"], o.T)


def test_fp32_shifted_close_to_fp64():
    """FP32 shifted populations against the FP64 oracle after 200 steps of a
    convecting case; tolerances: T (range 1) 2e-5 absolute, u and v 2e-6
    absolute (|u| ~ 1e-3 here), particle positions 1e-4."""
    c = cases.traj_case("traj_inertial")
    o = cases.run_oracle_traj(c)
    with traj_run(c, precision="fp32") as r:
        r.step(c["nsteps"])
        r.sync()
        m = r.get_moments()
        pr = r.get_particles()
    eT = np.abs(m["T"] - o["T"]).max()
    eu = max(np.abs(m["u"] - o["u"]).max(), np.abs(m["v"] - o["v"]).max())
    ex = max(np.abs(pr["x"] - o["px"]).max(), np.abs(pr["y"] - o["py"]).max())
    print(f"fp32 vs fp64: T {eT:.3e} u,v {eu:.3e} x,y {ex:.3e}")
    assert eT < 2e-5 and eu < 2e-6 and ex < 1e-4


def test_record_ring_overflow_is_a_status():
    c = cases.traj_case("traj_tracer")
    with traj_run(c, noutconfig=1, record_slots=2) as r:
        with pytest.raises(lb.LbrbError) as e:
            r.step(3)
        assert e.value.code == -7
        assert r.istep == 2
        recs = r.drain_records()
        assert sorted(recs) == [1, 2]
        r.step(2)
        assert sorted(r.drain_records()) == [3, 4]


def test_particle_outside_domain_rejected():
    c = cases.traj_case("traj_tracer")
    with lb.Run(**c["base"], nprtcl=c["nprtcl"]) as r:
        x = c["px"].copy()
        x[3] = c["nx"] + 5.0
        with pytest.raises(lb.LbrbError) as e:
            r.set_particles(c["ids"], x, c["py"], c["pu"], c["pv"], c["ptype"], c["invtau"])
        assert e.value.code == -6


def test_nonfinite_state_detected():
    c = cases.traj_case("traj_tracer")
    with lb.Run(**c["base"]) as r:
        f = c["f0"].copy()
        f[3, 5, 7] = np.nan
        r.set_populations(f, c["g0"])
        with pytest.raises(lb.LbrbError) as e:
            r.check_finite()
        assert e.value.code == -5


def test_box_nudging_missing_file_is_a_status():
    c = cases.nudge_case("nudge_box")
    with lb.Run(**c["base"], twall="adiabatic", nudge="refbox", alpha=0.1,
                ntempread=c["ntempread"], nobs=c["nprtcl"]) as r:
        r.set_moments(np.ones((c["ny"], c["nx"])), *(np.zeros((c["ny"], c["nx"])),) * 2,
                      c["Tic"])
        io = c["init_obs"]
        r.nudge_init(io["x"], io["y"], io["T"], io["id"])
        with pytest.raises(lb.LbrbError) as e:
            r.step(1)
        assert e.value.code == -4
        d = c["files"][c["ntempread"]]
        bad = d["id"].copy()
        bad[0] = -12345
        with pytest.raises(lb.LbrbError) as e:
            r.nudge_load(d["x"], d["y"], bad, d["temp"])
        assert e.value.code == -8


def test_fp32_full_size_conservation():
    """4096x2048 (the production grid), 50 steps: total mass is conserved by
    the bounce-back walls and periodic x (FP32 rounding only), T stays within
    the wall temperatures."""
    base = lb.closure(4096, 2048, Ra=1e8, Pr=1.0, U=0.05)
    with lb.Run(**base, precision="fp32") as r:
        r.init_conduction(1, 1e-3)
        m0 = r.get_moments()
        r.step(50)
        r.sync()
        r.check_finite()
        m = r.get_moments()
    drift = abs(m["rho"].mean() - m0["rho"].mean())
    assert drift < 1e-6, drift
    assert m["T"].max() <= 0.5 + 2e-3 and m["T"].min() >= -0.5 - 2e-3
