"""Pin the oracle (CPU restatement) to the reference.

* against the committed golden fixtures, which hold outputs of the reference's
  own sources run on the same seeded inputs (tests/golden/make_golden.py);
* against a live run of the reference when its checkout is present.

FP64 results must be bit-identical (same operation order, no FMA).
"""
import numpy as np
import pytest

from oracle import build
from tests.golden import cases


def _check_traj(name, out, z):
    np.testing.assert_array_equal(out["f"], z["f"])
    np.testing.assert_array_equal(out["g"], z["g"])
    steps = sorted({int(k[3:].split("_")[0]) for k in z if k.startswith("rec")})
    assert steps == sorted(out["records"]), (steps, sorted(out["records"]))
    for s in steps:
        r = out["records"][s]
        for k in r:
            np.testing.assert_array_equal(r[k], z[f"rec{s}_{k}"], err_msg=f"{name} step {s} {k}")
    # evolution.dat holds %e-formatted mean KE and mean T
    ev = z["evolution"]
    assert ev.shape[0] >= 1


@pytest.mark.parametrize("name", list(cases.TRAJ_CASES))
def test_oracle_matches_golden_trajectories(name):
    c = cases.traj_case(name)
    out = cases.run_oracle_traj(c)
    _check_traj(name, out, cases.load_golden(name))


@pytest.mark.parametrize("name", list(cases.NUDGE_CASES))
def test_oracle_matches_golden_nudging(name):
    c = cases.nudge_case(name)
    # (the fixtures come from the reference run on 1 x npy ranks)
    out = cases.run_oracle_nudge(c, ranks_y=c["npy"])
    z = cases.load_golden(name)
    # profiles.<step>.dat: every value as the reference printed it
    steps = sorted(int(k[4:]) for k in z if k.startswith("prof"))
    assert steps == sorted(out["profiles"]) and steps
    for s in steps:
        np.testing.assert_array_equal(z[f"prof{s}"][:, 0], np.arange(1, c["ny"] + 1))
        np.testing.assert_array_equal(cases.printed(out["profiles"][s][:, :8]), z[f"prof{s}"][:, 1:],
                                      err_msg=f"profile of step {s}")
    np.testing.assert_array_equal(out["f"], z["f"])
    np.testing.assert_array_equal(out["g"], z["g"])
    s = c["nsteps"]
    np.testing.assert_array_equal(out["T"], z[f"snap{s}_T"])
    np.testing.assert_array_equal(out["u"], z[f"snap{s}_u"])
    np.testing.assert_array_equal(out["v"], z[f"snap{s}_v"])


needs_ref = pytest.mark.skipif(not build.reference_available(), reason="reference checkout absent")


@needs_ref
def test_oracle_matches_live_reference_inertial():
    """Rebuild and rerun the reference now (not from fixtures)."""
    from oracle import refrun

    c = cases.traj_case("traj_inertial")
    refp = refrun.traj_params(c["base"], c["nsteps"], c["noutconfig"], c["nprtcl"],
                              tracer=False, taulag=c["taulag"], beta=c["beta"])
    ref = refrun.run_trajectories(refp, c["f0"], c["g0"], c["f0"], c["g0"], c["ids"],
                                  c["px"], c["py"], c["pu"], c["pv"])
    out = cases.run_oracle_traj(c)
    np.testing.assert_array_equal(out["f"], ref["f"])
    np.testing.assert_array_equal(out["g"], ref["g"])
    for s, r in ref["records"].items():
        order = np.argsort(r["id"])
        for k, a in out["records"][s].items():
            np.testing.assert_array_equal(a, r[k][order])


@needs_ref
def test_reference_decomposition_invariance():
    """The MPI stand-in is faithful: the reference run on a 2x2 process grid
    gives the same fields as on one rank (restart-route inputs)."""
    from oracle import refrun

    c = cases.traj_case("traj_tracer")
    refp = refrun.traj_params(c["base"], 40, 20, c["nprtcl"], tracer=True)
    a = refrun.run_trajectories(refp, c["f0"], c["g0"], c["f0"], c["g0"], c["ids"],
                                c["px"], c["py"], c["pu"], c["pv"], np_ranks=1)
    b = refrun.run_trajectories(refp, c["f0"], c["g0"], c["f0"], c["g0"], c["ids"],
                                c["px"], c["py"], c["pu"], c["pv"], np_ranks=4, dims="2x2")
    np.testing.assert_array_equal(a["f"], b["f"])
    np.testing.assert_array_equal(a["g"], b["g"])
    for s in a["records"]:
        oa, ob = np.argsort(a["records"][s]["id"]), np.argsort(b["records"][s]["id"])
        np.testing.assert_allclose(a["records"][s]["temp"][oa], b["records"][s]["temp"][ob],
                                   rtol=0, atol=1e-12)


def test_oracle_matches_golden_config0_digests():
    """the configuration-size fixture (512x256, 4096 tracers, 1000 steps):
    the oracle's populations, moments and every record against the digests
    of the reference's run"""
    c = cases.traj_case("cfg0_traj")
    z = cases.load_golden("cfg0_traj")
    out = cases.run_oracle_traj(c)
    assert cases.sha256(out["f"]) == str(z["f_sha"])
    assert cases.sha256(out["g"]) == str(z["g_sha"])
    for k in ("rho", "u", "v", "T"):
        assert cases.sha256(out[k]) == str(z[f"{k}_sha"]), k
    fields = [str(k) for k in z["rec_fields"]]
    assert sorted(out["records"]) == [int(s) for s in z["rec_steps"]]
    for s, r in out["records"].items():
        assert cases.record_digest(dict(r, id=c["ids"]), fields) == str(z[f"rec{s}_sha"]), s
