"""Parity of the CUDA path with the reference at the configurations' own sizes.

The fixtures (tests/golden/cfg*_traj.npz, made by make_golden.py from the
reference's own sources run on the same seeded inputs) hold SHA-256 digests of
the full populations f, g after the run, of every particle record, and of the
final moments rho, u, v, T (from the oracle, kept only after its populations
and records matched the reference's bit for bit), plus sampled rows.

  cfg0_traj  512x256, Ra=1e6, U=0.1, 4096 tracers, 1000 steps, records every 10
  cfg1_traj  4096x2048, Ra=1e8, U=0.05, 2^17 inertial particles (St=0.5),
             10 steps, records every 5

FP64: bit-exact (digest equality) in every launch mode.  FP32 shifted
populations: within the tolerances written in the test.
"""
import numpy as np
import pytest

import lagrangianrbnudging_b200 as lb
from lagrangianrbnudging_b200 import build
from tests.golden import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


_CASES = {}


def case(name):
    if name not in _CASES:
        _CASES[name] = (cases.traj_case(name), cases.load_golden(name))
    return _CASES[name]


def run_case(c, precision, launch):
    kw = dict(c["base"], precision=precision, twall="dirichlet", nudge="none", beta=c["beta"],
              nprtcl=c["nprtcl"], noutconfig=c["noutconfig"], record_full=True,
              record_slots=c["nsteps"] // c["noutconfig"] + 2)
    with lb.Run(**kw) as r:
        r.set_populations(c["f0"], c["g0"])
        r.moments_from_pre(c["f0"], c["g0"])
        r.set_particles(c["ids"], c["px"], c["py"], c["pu"], c["pv"], c["ptype"], c["invtau"])
        if launch != "default":
            r.set_graph(0)
            r.set_pairs(1 if launch == "pairs" else 0)
        r.step(c["nsteps"])
        r.sync()
        f, g = r.get_populations()
        m = r.get_moments()
        recs = r.drain_records()
    return f, g, m, recs


def check_fp64(name, launch):
    c, _ = case(name)
    check_fp64_outputs(name, *run_case(c, "fp64", launch))


def check_fp64_outputs(name, f, g, m, recs, fields_only=False):
    c, z = case(name)
    rows = cases.sample_rows(c["ny"])
    np.testing.assert_array_equal(cases.sample_pops(f), z["f_sample"])
    np.testing.assert_array_equal(cases.sample_pops(g), z["g_sample"])
    assert cases.sha256(f) == str(z["f_sha"])
    assert cases.sha256(g) == str(z["g_sha"])
    for k in ("rho", "u", "v", "T"):
        np.testing.assert_array_equal(m[k][rows][:, ::64], z[f"{k}_sample"], err_msg=k)
        assert cases.sha256(m[k]) == str(z[f"{k}_sha"]), k
    if fields_only:
        return
    fields = [str(k) for k in z["rec_fields"]]
    steps = [int(s) for s in z["rec_steps"]]
    assert sorted(recs) == steps
    last = recs[steps[-1]]
    order = np.argsort(last["id"], kind="stable")[:64]
    np.testing.assert_array_equal(last["id"][order], z["rec_last_id"])
    for k in fields:
        np.testing.assert_array_equal(last[k][order], z[f"rec_last_{k}"], err_msg=k)
    for s in steps:
        assert cases.record_digest(recs[s], fields) == str(z[f"rec{s}_sha"]), f"record of step {s}"


@pytest.mark.parametrize("launch", ["default", "pairs", "single"])
def test_config0_fp64_bit_exact_vs_reference(launch):
    """default: graph replays of one-step launches (a grid below 2^20 nodes);
    pairs: two steps per fused launch; single: one launch per step"""
    check_fp64("cfg0_traj", launch)


@pytest.mark.parametrize("launch", ["default", "single"])
def test_config1_fp64_bit_exact_vs_reference(launch):
    """default: two steps per fused launch (a grid above 2^20 nodes)"""
    check_fp64("cfg1_traj", launch)


@pytest.mark.parametrize("name", ["cfg0_traj", "cfg1_traj"])
def test_config_fp32_shifted_close_to_reference(name):
    """FP32 shifted populations against the reference's FP64 run: sampled
    moments and the last record of the 64 lowest ids"""
    c, z = case(name)
    f, g, m, recs = run_case(c, "fp32", "default")
    rows = cases.sample_rows(c["ny"])
    # tolerances: |dT| < 2e-5, |du|, |dv| < 2e-6 (|u| <= 1e-3 here), positions < 1e-4
    np.testing.assert_allclose(m["T"][rows][:, ::64], z["T_sample"], rtol=0, atol=2e-5)
    np.testing.assert_allclose(m["u"][rows][:, ::64], z["u_sample"], rtol=0, atol=2e-6)
    np.testing.assert_allclose(m["v"][rows][:, ::64], z["v_sample"], rtol=0, atol=2e-6)
    np.testing.assert_allclose(m["rho"][rows][:, ::64], z["rho_sample"], rtol=0, atol=1e-5)
    last = recs[int(z["rec_steps"][-1])]
    order = np.argsort(last["id"], kind="stable")[:64]
    np.testing.assert_array_equal(last["id"][order], z["rec_last_id"])
    np.testing.assert_allclose(last["x"][order], z["rec_last_x"], rtol=0, atol=1e-4)
    np.testing.assert_allclose(last["y"][order], z["rec_last_y"], rtol=0, atol=1e-4)
    np.testing.assert_allclose(last["temp"][order], z["rec_last_temp"], rtol=0, atol=2e-5)


def run_case_slabs(c, heights, protocol):
    """the same run as one domain cut into y-slabs on this GPU: through
    lbrb_slab_step (one process), or the one-process-per-GPU protocol with
    two steps per launch (slabrank, copies between the slabs)"""
    kw = dict(c["base"], precision="fp64", twall="dirichlet", nudge="none", beta=c["beta"],
              nprtcl=c["nprtcl"], noutconfig=c["noutconfig"], record_full=True,
              record_slots=c["nsteps"] // c["noutconfig"] + 2)
    with lb.SlabDomain(heights, **kw) as dom:
        dom.set_populations(c["f0"], c["g0"])
        dom.moments_from_pre(c["f0"], c["g0"])
        dom.set_particles(c["ids"], c["px"], c["py"], c["pu"], c["pv"], c["ptype"], c["invtau"])
        if protocol == "slab_step":
            dom.step(c["nsteps"])
        else:
            import torch

            from lagrangianrbnudging_b200 import slabrank
            st = slabrank.bind_stream(dom.slabs, torch)
            ranks = [slabrank.SlabRank(r, slabrank.device_buffers(r, torch), particles=True, pairs=True)
                     for r in dom.slabs]
            with torch.cuda.stream(st):
                slabrank.run_local(ranks, c["nsteps"])
            torch.cuda.synchronize()
        for r in dom.slabs:
            r.sync()
        f, g = dom.get_populations()
        m = dom.get_moments()
        recs = dom.drain_records()
    return f, g, m, recs


@pytest.mark.parametrize("protocol", ["slab_step", "ranks_pairs"])
def test_config0_fp64_slabs_bit_exact_vs_reference(protocol):
    """three uneven y-slabs, each holding its own particles, against the
    reference's digests: populations, moments and every record"""
    c, _ = case("cfg0_traj")
    check_fp64_outputs("cfg0_traj", *run_case_slabs(c, (100, 90, 66), protocol))


def test_config1_fp64_slabs_bit_exact_vs_reference():
    """4096x2048 with 2^17 particles as two slabs through the
    one-process-per-GPU protocol, against the reference's digests"""
    c, _ = case("cfg1_traj")
    check_fp64_outputs("cfg1_traj", *run_case_slabs(c, (1024, 1024), "ranks_pairs"))


def test_config0_fp64_ensemble_member_bit_exact_vs_reference():
    """the configuration's fields as a member of an ensemble (two-step
    launches in graph replays, beside a member of another size) against the
    reference's digests of f, g and the moments (ensemble members keep no
    records; the particles do not act on the fields)"""
    c, _ = case("cfg0_traj")
    kw = dict(c["base"], precision="fp64", twall="dirichlet", nudge="none", nprtcl=0)
    a = lb.Run(**kw)
    b = lb.Run(**lb.closure(256, 128, Ra=1e6, Pr=1.0, U=0.1), precision="fp64")
    try:
        a.set_populations(c["f0"], c["g0"])
        a.moments_from_pre(c["f0"], c["g0"])
        b.init_conduction(5, 1e-2)
        with lb.Ensemble([a, b]) as e:
            e.step(c["nsteps"])
            e.sync()
        f, g = a.get_populations()
        m = a.get_moments()
    finally:
        a.close()
        b.close()
    check_fp64_outputs("cfg0_traj", f, g, m, None, fields_only=True)
