"""Run the reference's own programs (built by ``build.build_ref``) on injected
inputs and read their outputs back.  TEST INFRASTRUCTURE ONLY.

Inputs go in through the reference's restart route (temppart_dump.c:1649-1654,
restore* :348-668, restore_prtcl :252-346) in the HDF5 stand-in's raw layout;
outputs are read from the files the reference writes (dumpf/dumpg :52-141,
dumpfpre/dumpgpre :143-232, prtcl_write :1467-1571 + Writefull
mympi2.h:441-565, snapshottemp tempvel_nudge.c:1784-1862, evolution.dat).
"""
from __future__ import annotations

import ctypes
import math
import os
import resource
import subprocess
import tempfile
from pathlib import Path

import numpy as np

from . import build

REC_FIELDS = ["x", "y", "u", "v", "xo", "yo", "uo", "vo", "temp",
              "dtu", "dtv", "dxu", "dxv", "dyu", "dyv", "fu", "fv"]


def _unlimited_stack():
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass


def _to_ref_pops(a: np.ndarray) -> np.ndarray:
    """(9, ny, nx) -> reference dataset layout [nx][ny][9]"""
    return np.ascontiguousarray(np.transpose(a, (2, 1, 0)))


def _from_ref_pops(b: np.ndarray, nx: int, ny: int) -> np.ndarray:
    return np.ascontiguousarray(np.transpose(b.reshape(nx, ny, 9), (2, 1, 0)))


def _write_ds(path: Path, arr: np.ndarray):
    path.parent.mkdir(parents=True, exist_ok=True)
    np.ascontiguousarray(arr).tofile(path)


def run_exe(exe: Path, workdir: Path, np_ranks: int = 1, dims: str | None = None,
            timeout: float = 600.0) -> float:
    env = dict(os.environ)
    env["LBRB_SHIM_NP"] = str(np_ranks)
    if dims:
        env["LBRB_SHIM_DIMS"] = dims
    else:
        env.pop("LBRB_SHIM_DIMS", None)
    import time
    t0 = time.perf_counter()
    with open(workdir / "stdout.txt", "wb") as out, open(workdir / "stderr.txt", "wb") as err:
        r = subprocess.run([str(exe)], cwd=workdir, env=env, stdout=out, stderr=err,
                           preexec_fn=_unlimited_stack, timeout=timeout)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed rc={r.returncode}: "
                           f"{(workdir / 'stderr.txt').read_text()[-2000:]}")
    return dt


def traj_params(base: dict, nsteps: int, noutconfig: int, nprtcl: int, tracer: bool,
                taulag: float = 100.0, beta: float = 0.0, writefull: bool = True,
                nout: int | None = None) -> dict:
    """compile-time parameters of temppart_dump.c / its mympi2.h"""
    return dict(
        nx=int(base["nx"]), ny=int(base["ny"]), scratch=0, nstart=0, nsteps=int(nsteps),
        nout=int(nout or noutconfig), noutconfig=int(noutconfig),
        relax=float(base["relax"]), relaxg=float(base["relaxg"]),
        Tup=float(base["Tup"]), Tdown=float(base["Tdown"]), gravity=float(base["gravity"]),
        Particle=1, Particle_scratch=0,
        Nprtcl=int(nprtcl), tracer=1 if tracer else 0, heavyprtcl=0 if tracer else 1,
        taulag=float(taulag), beta=float(beta), Prtcl_Writefull=1 if writefull else 0,
    )


def run_trajectories_scratch(refp: dict, workdir: Path | None = None, tag: str | None = None) -> dict:
    """Run temppart_dump with scratch=1, Particle_scratch=1 on one rank."""
    exe = build.build_ref("temppart_dump", refp, tag)
    nx, ny, nsteps, nout_c = refp["nx"], refp["ny"], refp["nsteps"], refp["noutconfig"]
    wd = Path(tempfile.mkdtemp(prefix="lbrb_refs_")) if workdir is None else Path(workdir)
    (wd / "Prtcl_Veldata1").mkdir(parents=True, exist_ok=True)
    (wd / "Tempfolder").mkdir(exist_ok=True)
    run_exe(exe, wd, 1, None)
    out = {"workdir": wd}
    last = nsteps + 1
    out["f"] = _from_ref_pops(np.fromfile(wd / f"confnew{last}.h5.d" / "f.bin"), nx, ny)
    out["g"] = _from_ref_pops(np.fromfile(wd / f"congnew{last}.h5.d" / "g.bin"), nx, ny)
    out["fpre"] = _from_ref_pops(np.fromfile(wd / f"confpre{nsteps}.h5.d" / "f.bin"), nx, ny)
    out["gpre"] = _from_ref_pops(np.fromfile(wd / f"congpre{nsteps}.h5.d" / "g.bin"), nx, ny)
    recs = {}
    for s in range(nout_c, nsteps + 1, nout_c):
        d = wd / "Prtcl_Veldata1" / f"Particles{s}.h5.d"
        r = {"id": np.fromfile(d / "id.bin", dtype=np.int32)}
        for name in REC_FIELDS:
            if (d / f"{name}.bin").exists():
                r[name] = np.fromfile(d / f"{name}.bin")
        recs[s] = r
    out["records"] = recs
    out["init_x"] = np.fromfile(wd / "init_prtclx0.in")
    out["init_y"] = np.fromfile(wd / "init_prtcly0.in")
    return out


def run_trajectories(refp: dict, f0, g0, fpre0, gpre0, ids, px, py, pu, pv,
                     np_ranks: int = 1, dims: str | None = None, workdir: Path | None = None,
                     tag: str | None = None) -> dict:
    """Run temppart_dump with restart-route inputs; returns the outputs."""
    exe = build.build_ref("temppart_dump", refp, tag)
    nx, ny, nsteps, nout_c = refp["nx"], refp["ny"], refp["nsteps"], refp["noutconfig"]
    own = workdir is None
    wd = Path(tempfile.mkdtemp(prefix="lbrb_ref_")) if own else Path(workdir)
    (wd / "Prtcl_Veldata1").mkdir(parents=True, exist_ok=True)
    (wd / "Tempfolder").mkdir(exist_ok=True)
    _write_ds(wd / "conf.h5.d" / "f.bin", _to_ref_pops(f0))
    _write_ds(wd / "cong.h5.d" / "g.bin", _to_ref_pops(g0))
    _write_ds(wd / "confpre.h5.d" / "f.bin", _to_ref_pops(fpre0))
    _write_ds(wd / "congpre.h5.d" / "g.bin", _to_ref_pops(gpre0))
    n = len(ids)
    _write_ds(wd / "Prtcl_Veldata1" / "Particles0.h5.d" / "id.bin", np.asarray(ids, np.int32))
    rec = np.zeros((n, 8))
    rec[:, 0], rec[:, 1], rec[:, 2], rec[:, 3] = px, py, pu, pv
    rec[:, 4], rec[:, 5], rec[:, 6], rec[:, 7] = px, py, pu, pv
    rec.tofile(wd / "prtcl_dump0.in")
    wall = run_exe(exe, wd, np_ranks, dims)
    out = {"wall_s": wall, "workdir": wd}
    last = nsteps + 1  # the reference's loop counter after the loop
    out["f"] = _from_ref_pops(np.fromfile(wd / f"confnew{last}.h5.d" / "f.bin"), nx, ny)
    out["g"] = _from_ref_pops(np.fromfile(wd / f"congnew{last}.h5.d" / "g.bin"), nx, ny)
    out["fpre"] = _from_ref_pops(np.fromfile(wd / f"confpre{nsteps}.h5.d" / "f.bin"), nx, ny)
    out["gpre"] = _from_ref_pops(np.fromfile(wd / f"congpre{nsteps}.h5.d" / "g.bin"), nx, ny)
    recs = {}
    if nout_c > 0:
        for s in range(nout_c, nsteps + 1, nout_c):
            d = wd / "Prtcl_Veldata1" / f"Particles{s}.h5.d"
            r = {"id": np.fromfile(d / "id.bin", dtype=np.int32)}
            for name in REC_FIELDS:
                p = d / f"{name}.bin"
                if p.exists():
                    r[name] = np.fromfile(p)
            recs[s] = r
    out["records"] = recs
    ev = wd / "evolution.dat"
    out["evolution"] = np.loadtxt(ev, ndmin=2) if ev.exists() and ev.stat().st_size else np.zeros((0, 3))
    return out


def nudge_params(base: dict, nsteps: int, ntempread: int, alpha: float, noutconfig: int,
                 nout: int, scratch: int = 1) -> dict:
    """compile-time parameters of tempvel_nudge.c (Nprtcl stays 40*40)"""
    return dict(
        nx=int(base["nx"]), ny=int(base["ny"]), scratch=int(scratch), contin=0, nstart=0,
        nsteps=int(nsteps), nout=int(nout), noutconfig=int(noutconfig),
        ntempread=int(ntempread), relax=float(base["relax"]), relaxg=float(base["relaxg"]),
        Tup=float(base["Tup"]), Tdown=float(base["Tdown"]), gravity=float(base["gravity"]),
        alpha=float(alpha),
    )


def scratch_ic_T(nx: int, ny: int, Tup: float, Tdown: float, npy: int) -> np.ndarray:
    """Temperature of the reference's scratch initial state (inithydro,
    temppart_dump.c:686-701 / tempvel_nudge.c:580-595) for a 1 x npy process
    grid: rank r = mey seeds srand(r) and draws one rand() per haloed node in
    i-major order.  Uses the C library's own rand() and tanh()."""
    libc = ctypes.CDLL(None)
    libc.rand.restype = ctypes.c_int
    RAND_MAX = 2147483647
    randnorm = 1.0 / RAND_MAX
    epstan = 10.0
    NY = ny // npy
    T = np.zeros((ny, nx))
    for mey in range(npy):
        libc.srand(mey)
        for i in range(nx + 2):
            for j in range(NY + 2):
                yyy = float(j - 1 + NY * mey)
                y_c = float(ny) * 1 / 2.0 + (randnorm * libc.rand() - 0.5) * 2.0 * epstan
                t = Tdown + (Tup - Tdown) * (math.tanh((yyy - y_c) / epstan) + 1.0) / 2.0
                if 1 <= i <= nx and 1 <= j <= NY:
                    T[j - 1 + NY * mey, i - 1] = t
    return T


def run_nudging(refp: dict, init_obs: dict, files: dict, np_ranks: int = 2, dims: str = "1x2",
                workdir: Path | None = None, tag: str | None = None, restart: dict | None = None) -> dict:
    """Run tempvel_nudge (scratch IC, contin=0).  init_obs: x,y,T,id arrays
    (init_prtcl*0.in); files: {step: dict(x,y,id,temp)} observation files."""
    exe = build.build_ref("tempvel_nudge", refp, tag)
    nx, ny, nsteps = refp["nx"], refp["ny"], refp["nsteps"]
    own = workdir is None
    wd = Path(tempfile.mkdtemp(prefix="lbrb_refn_")) if own else Path(workdir)
    (wd / "Tempfolder").mkdir(parents=True, exist_ok=True)
    obs = wd / "obs"
    (obs / "Prtcl_Veldata1").mkdir(parents=True, exist_ok=True)
    np.asarray(init_obs["x"], np.float64).tofile(obs / "init_prtclx0.in")
    np.asarray(init_obs["y"], np.float64).tofile(obs / "init_prtcly0.in")
    np.asarray(init_obs["T"], np.float64).tofile(obs / "init_prtclT0.in")
    np.asarray(init_obs["id"], np.int32).tofile(obs / "init_prtcl_id0.in")
    if restart is not None:
        # restart route (scratch=0): conf/cong/confpre/congpre in the run directory
        _write_ds(wd / "conf.h5.d" / "f.bin", _to_ref_pops(restart["f"]))
        _write_ds(wd / "cong.h5.d" / "g.bin", _to_ref_pops(restart["g"]))
        _write_ds(wd / "confpre.h5.d" / "f.bin", _to_ref_pops(restart["fpre"]))
        _write_ds(wd / "congpre.h5.d" / "g.bin", _to_ref_pops(restart["gpre"]))
    for s, d in files.items():
        base = obs / "Prtcl_Veldata1" / f"Particles{s}.h5.d"
        _write_ds(base / "x.bin", np.asarray(d["x"], np.float64))
        _write_ds(base / "y.bin", np.asarray(d["y"], np.float64))
        _write_ds(base / "id.bin", np.asarray(d["id"], np.int32))
        _write_ds(base / "temp.bin", np.asarray(d["temp"], np.float64))
    wall = run_exe(exe, wd, np_ranks, dims)
    out = {"wall_s": wall, "workdir": wd}
    last = nsteps + 1
    out["f"] = _from_ref_pops(np.fromfile(wd / f"confnew{last}.h5.d" / "f.bin"), nx, ny)
    out["g"] = _from_ref_pops(np.fromfile(wd / f"congnew{last}.h5.d" / "g.bin"), nx, ny)
    snaps = {}
    nc = refp["noutconfig"]
    for s in range(nc, nsteps + 1, nc):
        d = wd / "Tempfolder" / f"snaptemp{s}.h5.d"
        if d.exists():
            snaps[s] = {k: np.ascontiguousarray(np.fromfile(d / f"{k}.bin").reshape(nx, ny).T)
                        for k in ("T", "u", "v")}
    out["snaps"] = snaps
    # profiles.<istep>.dat (profile(), tempvel_nudge.c:1104-1260, every nout
    # steps): "j rho u v u^2 v^2 T vT dT/dy" per row, each %e; the format has
    # one %e more than its arguments (:1229), so a tenth column is whatever
    # printf finds there and is dropped
    profs = {}
    for s in range(refp["nout"], nsteps + 1, refp["nout"]):
        p = wd / f"profiles.{s}.dat"
        if p.exists():
            rows = [ln.split()[:9] for ln in p.read_text().splitlines() if ln.strip()]
            profs[s] = np.array([[float(x) for x in r] for r in rows])
    out["profiles"] = profs
    return out
