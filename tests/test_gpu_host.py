"""The host program (lbrb_host) as a drop-in for the reference's main():
same parameters, same input files, same output files -- compared with the
outputs of the reference's own programs (golden fixtures)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from lagrangianrbnudging_b200 import build
from oracle import refrun
from tests.golden import cases

HOST = Path(build.__file__).resolve().parent / "lbrb_host"
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def run_host(program: str, params: dict, wd: Path):
    args = [str(HOST), program] + [f"{k}={float(v)!r}" if isinstance(v, float) else f"{k}={v}"
                                   for k, v in params.items()] + [f"dir={wd}"]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr


def read_pops(path: Path, nx: int, ny: int) -> np.ndarray:
    return refrun._from_ref_pops(np.fromfile(path), nx, ny)


def check_records(wd: Path, z: dict):
    steps = sorted({int(k[3:].split("_")[0]) for k in z if k.startswith("rec")})
    assert steps
    for s in steps:
        d = wd / "Prtcl_Veldata1" / f"Particles{s}.h5.d"
        ids = np.fromfile(d / "id.bin", dtype=np.int32)
        order = np.argsort(ids)
        np.testing.assert_array_equal(ids[order], z[f"rec{s}_id"])
        for k in refrun.REC_FIELDS:
            if f"rec{s}_{k}" in z:
                np.testing.assert_array_equal(np.fromfile(d / f"{k}.bin")[order], z[f"rec{s}_{k}"],
                                              err_msg=f"step {s} {k}")


def test_host_trajectories_restart_route(tmp_path):
    """restart files + prtcl_dump -> records, confnew, confpre identical to the reference"""
    c = cases.traj_case("traj_inertial")
    z = cases.load_golden("traj_inertial")
    wd = tmp_path
    refrun._write_ds(wd / "conf.h5.d" / "f.bin", refrun._to_ref_pops(c["f0"]))
    refrun._write_ds(wd / "cong.h5.d" / "g.bin", refrun._to_ref_pops(c["g0"]))
    refrun._write_ds(wd / "confpre.h5.d" / "f.bin", refrun._to_ref_pops(c["f0"]))
    refrun._write_ds(wd / "congpre.h5.d" / "g.bin", refrun._to_ref_pops(c["g0"]))
    refrun._write_ds(wd / "Prtcl_Veldata1" / "Particles0.h5.d" / "id.bin", c["ids"])
    rec = np.zeros((c["nprtcl"], 8))
    rec[:, 0], rec[:, 1], rec[:, 2], rec[:, 3] = c["px"], c["py"], c["pu"], c["pv"]
    rec.tofile(wd / "prtcl_dump0.in")
    b = c["base"]
    run_host("trajectories", dict(nx=c["nx"], ny=c["ny"], scratch=0, nsteps=c["nsteps"],
                                  nout=c["noutconfig"], noutconfig=c["noutconfig"],
                                  relax=b["relax"], relaxg=b["relaxg"], Tup=b["Tup"],
                                  Tdown=b["Tdown"], gravity=b["gravity"], Particle_scratch=0,
                                  Nprtcl=c["nprtcl"], tracer=0, heavyprtcl=1,
                                  taulag=c["taulag"], beta=c["beta"], Prtcl_Writefull=1), wd)
    last = c["nsteps"] + 1
    np.testing.assert_array_equal(read_pops(wd / f"confnew{last}.h5.d" / "f.bin", c["nx"], c["ny"]), z["f"])
    np.testing.assert_array_equal(read_pops(wd / f"congnew{last}.h5.d" / "g.bin", c["nx"], c["ny"]), z["g"])
    np.testing.assert_array_equal(read_pops(wd / f"confpre{c['nsteps']}.h5.d" / "f.bin", c["nx"], c["ny"]), z["fpre"])
    np.testing.assert_array_equal(read_pops(wd / f"congpre{c['nsteps']}.h5.d" / "g.bin", c["nx"], c["ny"]), z["gpre"])
    check_records(wd, z)
    ev = np.loadtxt(wd / "evolution.dat", ndmin=2)
    np.testing.assert_allclose(ev[:, 1:], z["evolution"][:, 1:], rtol=1e-5)  # %e text


def test_host_trajectories_scratch_state_and_lattice(tmp_path):
    """the reference's own scratch state (tanh + rand()) and particle lattice"""
    c = cases.SCRATCH_TRAJ_CASES["traj_scratch"]
    z = cases.load_golden("traj_scratch")
    b = cases.closure(c["nx"], c["ny"], Ra=c["Ra"], Pr=1.0, U=c["U"])
    run_host("trajectories", dict(nx=c["nx"], ny=c["ny"], scratch=1, nsteps=c["nsteps"],
                                  nout=c["noutconfig"], noutconfig=c["noutconfig"],
                                  relax=b["relax"], relaxg=b["relaxg"], Tup=b["Tup"],
                                  Tdown=b["Tdown"], gravity=b["gravity"], Particle_scratch=1,
                                  Nprtcl=c["nprtcl"], tracer=1, heavyprtcl=0,
                                  taulag=c["taulag"], beta=c["beta"], Prtcl_Writefull=1), tmp_path)
    last = c["nsteps"] + 1
    np.testing.assert_array_equal(np.fromfile(tmp_path / "init_prtclx0.in"), z["init_x"])
    np.testing.assert_array_equal(np.fromfile(tmp_path / "init_prtcly0.in"), z["init_y"])
    np.testing.assert_array_equal(read_pops(tmp_path / f"confnew{last}.h5.d" / "f.bin", c["nx"], c["ny"]), z["f"])
    np.testing.assert_array_equal(read_pops(tmp_path / f"congnew{last}.h5.d" / "g.bin", c["nx"], c["ny"]), z["g"])
    np.testing.assert_array_equal(read_pops(tmp_path / f"confpre{c['nsteps']}.h5.d" / "f.bin", c["nx"], c["ny"]), z["fpre"])
    check_records(tmp_path, z)


def test_host_nudging_restart_route(tmp_path):
    """observation files + restart files -> fields identical to the reference
    (run there on a 1 x 2 process grid)"""
    c = cases.nudge_case("nudge_restart")
    z = cases.load_golden("nudge_restart")
    wd = tmp_path
    obs = wd / "obs"
    (obs / "Prtcl_Veldata1").mkdir(parents=True)
    io = c["init_obs"]
    np.asarray(io["x"], np.float64).tofile(obs / "init_prtclx0.in")
    np.asarray(io["y"], np.float64).tofile(obs / "init_prtcly0.in")
    np.asarray(io["T"], np.float64).tofile(obs / "init_prtclT0.in")
    np.asarray(io["id"], np.int32).tofile(obs / "init_prtcl_id0.in")
    for s, d in c["files"].items():
        base = obs / "Prtcl_Veldata1" / f"Particles{s}.h5.d"
        for k, dt in (("x", np.float64), ("y", np.float64), ("id", np.int32), ("temp", np.float64)):
            refrun._write_ds(base / f"{k}.bin", np.asarray(d[k], dt))
    rp = c["restart_pops"]
    for name, key, a in (("conf", "f", rp["f"]), ("cong", "g", rp["g"]), ("confpre", "f", rp["fpre"]),
                         ("congpre", "g", rp["gpre"])):
        refrun._write_ds(wd / f"{name}.h5.d" / f"{key}.bin", refrun._to_ref_pops(a))
    b = c["base"]
    run_host("nudging", dict(nx=c["nx"], ny=c["ny"], scratch=0, nsteps=c["nsteps"], nout=cases.PROFILE_EVERY,
                             noutconfig=10, ntempread=c["ntempread"], alpha=c["alpha"],
                             relax=b["relax"], relaxg=b["relaxg"], Tup=b["Tup"], Tdown=b["Tdown"],
                             gravity=b["gravity"], Nprtcl=c["nprtcl"]), wd)
    last = c["nsteps"] + 1
    np.testing.assert_array_equal(read_pops(wd / f"confnew{last}.h5.d" / "f.bin", c["nx"], c["ny"]), z["f"])
    np.testing.assert_array_equal(read_pops(wd / f"congnew{last}.h5.d" / "g.bin", c["nx"], c["ny"]), z["g"])
    for s in range(10, c["nsteps"] + 1, 10):
        d = wd / "Tempfolder" / f"snaptemp{s}.h5.d"
        for k in ("T", "u", "v"):
            a = np.fromfile(d / f"{k}.bin").reshape(c["nx"], c["ny"]).T
            np.testing.assert_array_equal(a, z[f"snap{s}_{k}"], err_msg=f"snap {s} {k}")
    # profiles.<step>.dat against the reference's (run on 1 x npy ranks).  The
    # host program is one whole domain: at the last row of an inner y-rank the
    # reference's dT/dy took T(j+1) from a halo row without the 1/2 nud_term,
    # there the expected value is the whole domain's (the oracle's, printed)
    whole = cases.run_oracle_nudge(c, ranks_y=1)["profiles"]
    nyr = c["ny"] // c["npy"]
    for s in range(cases.PROFILE_EVERY, c["nsteps"] + 1, cases.PROFILE_EVERY):
        got = np.loadtxt(wd / f"profiles.{s}.dat", ndmin=2)
        ref = z[f"prof{s}"].copy()
        for j in range(nyr - 1, c["ny"] - 1, nyr):
            ref[j, 8] = cases.printed(whole[s][j, 7])
        np.testing.assert_array_equal(got[:, 0], ref[:, 0])
        # both are "%e" text (7 significant digits) of sums taken in different
        # orders: one unit in the 7th digit, and 1e-15 for means near zero
        np.testing.assert_allclose(got[:, 1:], ref[:, 1:], rtol=1.000001e-6, atol=1e-15,
                                   err_msg=f"profile of step {s}")
