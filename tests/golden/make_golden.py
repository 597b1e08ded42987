"""Generate the golden fixtures by running the reference's OWN sources.

Run from the repository root, where the reference checkout is available:

    python tests/golden/make_golden.py

For each case in cases.py this builds the reference program with the case's
compile-time parameters (oracle/build.py: gcc -O2 against the in-repo MPI and
HDF5 stand-ins), injects the seeded inputs through the reference's restart
route (or, for the nudging program, its scratch initial state and observation
files) and stores the reference's outputs as compressed .npz files here.
The GPU box has no reference checkout; these fixtures carry its results there.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refrun  # noqa: E402
from tests.golden import cases  # noqa: E402


def make_traj(name: str) -> dict:
    c = cases.traj_case(name)
    refp = refrun.traj_params(c["base"], c["nsteps"], c["noutconfig"], c["nprtcl"],
                              tracer=not c["inertial"], taulag=c["taulag"], beta=c["beta"])
    out = refrun.run_trajectories(refp, c["f0"], c["g0"], c["f0"], c["g0"], c["ids"],
                                  c["px"], c["py"], c["pu"], c["pv"])
    z = {"f": out["f"], "g": out["g"], "evolution": out["evolution"]}
    if name == "traj_inertial":
        z["fpre"], z["gpre"] = out["fpre"], out["gpre"]
    for s, r in out["records"].items():
        order = np.argsort(r["id"], kind="stable")
        z[f"rec{s}_id"] = r["id"][order]
        for k in refrun.REC_FIELDS:
            if k in r:
                z[f"rec{s}_{k}"] = r[k][order]
    return z


def make_config(name: str) -> dict:
    """A configuration-size run: the reference's outputs as digests (and
    samples), the oracle's final moments beside them.  The oracle's moments
    are kept only after its populations and records have matched the
    reference's bit for bit on the same run."""
    c = cases.traj_case(name)
    refp = refrun.traj_params(c["base"], c["nsteps"], c["noutconfig"], c["nprtcl"],
                              tracer=not c["inertial"], taulag=c["taulag"], beta=c["beta"])
    out = refrun.run_trajectories(refp, c["f0"], c["g0"], c["f0"], c["g0"], c["ids"],
                                  c["px"], c["py"], c["pu"], c["pv"])
    o = cases.run_oracle_traj(c)
    assert np.array_equal(o["f"], out["f"]) and np.array_equal(o["g"], out["g"]), "oracle vs reference"
    steps = sorted(out["records"])
    assert steps == sorted(o["records"]), (steps, sorted(o["records"]))
    fields = [k for k in refrun.REC_FIELDS if k in out["records"][steps[0]]]
    z = {"f_sha": np.array(cases.sha256(out["f"])), "g_sha": np.array(cases.sha256(out["g"])),
         "f_sample": cases.sample_pops(out["f"]), "g_sample": cases.sample_pops(out["g"]),
         "rec_fields": np.array(fields), "rec_steps": np.array(steps, np.int32),
         "evolution": out["evolution"]}
    for s in steps:
        r = out["records"][s]
        orr = dict(o["records"][s], id=np.asarray(c["ids"]))
        z[f"rec{s}_sha"] = np.array(cases.record_digest(r, fields))
        assert cases.record_digest(orr, fields) == z[f"rec{s}_sha"], f"oracle record {s}"
    # the last record of the 64 lowest ids, in full
    r = out["records"][steps[-1]]
    order = np.argsort(r["id"], kind="stable")[:64]
    z["rec_last_id"] = r["id"][order]
    for k in fields:
        z[f"rec_last_{k}"] = r[k][order]
    rows = cases.sample_rows(c["ny"])
    for k in ("rho", "u", "v", "T"):
        z[f"{k}_sha"] = np.array(cases.sha256(o[k]))
        z[f"{k}_sample"] = np.ascontiguousarray(o[k][rows][:, ::64])
    return z


def make_scratch(name: str) -> dict:
    c = dict(cases.SCRATCH_TRAJ_CASES[name])
    base = cases.closure(c["nx"], c["ny"], Ra=c["Ra"], Pr=1.0, U=c["U"])
    refp = refrun.traj_params(base, c["nsteps"], c["noutconfig"], c["nprtcl"], tracer=c["tracer"],
                              taulag=c["taulag"], beta=c["beta"])
    refp.update(scratch=1, Particle_scratch=1)
    out = refrun.run_trajectories_scratch(refp)
    z = {"f": out["f"], "g": out["g"], "fpre": out["fpre"], "gpre": out["gpre"],
         "init_x": out["init_x"], "init_y": out["init_y"]}
    for s, r in out["records"].items():
        order = np.argsort(r["id"], kind="stable")
        z[f"rec{s}_id"] = r["id"][order]
        for k in refrun.REC_FIELDS:
            if k in r:
                z[f"rec{s}_{k}"] = r[k][order]
    return z


def make_nudge(name: str) -> dict:
    c = cases.nudge_case(name)
    refp = refrun.nudge_params(c["base"], c["nsteps"], c["ntempread"], c["alpha"],
                               noutconfig=10, nout=cases.PROFILE_EVERY, scratch=0 if c.get("restart") else 1)
    out = refrun.run_nudging(refp, c["init_obs"], c["files"], np_ranks=c["npy"],
                             dims=f"1x{c['npy']}", restart=c.get("restart_pops"))
    z = {"f": out["f"], "g": out["g"]}
    for s, d in out["snaps"].items():
        for k, a in d.items():
            z[f"snap{s}_{k}"] = a
    for s, a in out["profiles"].items():
        z[f"prof{s}"] = a  # [ny][j, rho, u, v, u^2, v^2, T, vT, dT/dy] as printed (%e)
    return z


def main(only=()):
    """all fixtures, or only the named ones (command-line arguments)"""
    makers = [(cases.TRAJ_CASES, make_traj), (cases.CONFIG_CASES, make_config),
              (cases.SCRATCH_TRAJ_CASES, make_scratch), (cases.NUDGE_CASES, make_nudge)]
    for table, make in makers:
        for name in table:
            if only and name not in only:
                continue
            z = make(name)
            np.savez_compressed(cases.golden_path(name), **z)
            print("wrote", cases.golden_path(name))


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
