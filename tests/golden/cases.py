"""Canonical parity cases: seeded inputs shared by the golden-fixture
generator (make_golden.py), the oracle pin tests and the GPU parity tests.

Every input is synthetic and seeded; nothing is read from the reference
checkout here.  The oracle is imported only as the checker.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from oracle.oracle import Oracle, closure  # noqa: F401  (closure re-exported for the generator)

GOLDEN = Path(__file__).resolve().parent
W = np.array([16 / 36, 4 / 36, 4 / 36, 4 / 36, 4 / 36, 1 / 36, 1 / 36, 1 / 36, 1 / 36])


def bilinear_np(fld: np.ndarray, xx: float, yy: float) -> float:
    ny, nx = fld.shape
    x1, y1 = int(xx), int(yy)
    x2, y2 = x1 + 1, y1 + 1
    F = lambda i, j: fld[(j - 1) % ny, (i - 1) % nx]
    return (F(x1, y1) * (x2 - xx) * (y2 - yy) + F(x2, y1) * (xx - x1) * (y2 - yy)
            + F(x1, y2) * (x2 - xx) * (yy - y1) + F(x2, y2) * (xx - x1) * (yy - y1))


TRAJ_CASES = {
    # name: grid, closure, particles, steps
    "traj_tracer": dict(nx=48, ny=24, Ra=1e5, U=0.1, seed=7, noise=1e-2, nprtcl=64,
                        inertial=False, taulag=50.0, beta=0.0, nsteps=200, noutconfig=50),
    "traj_inertial": dict(nx=48, ny=24, Ra=1e5, U=0.1, seed=9, noise=1e-2, nprtcl=64,
                          inertial=True, taulag=50.0, beta=0.1, nsteps=200, noutconfig=50),
    "traj_wide": dict(nx=136, ny=20, Ra=3e5, U=0.1, seed=21, noise=2e-2, nprtcl=300,
                      inertial=True, taulag=30.0, beta=0.1, nsteps=120, noutconfig=40),
    # the 1000-step window: f, g, u, T and every record bit for bit
    "traj_long": dict(nx=64, ny=32, Ra=1e6, U=0.1, seed=31, noise=2e-2, nprtcl=128,
                      inertial=True, taulag=40.0, beta=0.1, nsteps=1000, noutconfig=250),
}

# the configurations' own sizes, checked through SHA-256 digests of the full
# arrays (the arrays themselves are too large to commit) plus sampled values
CONFIG_CASES = {
    # plain FP64 run: 512x256, Ra=1e6, U=0.1, conduction + 1e-3 noise, 4096
    # seeded uniform tracers, 1000 steps, records every 10
    "cfg0_traj": dict(nx=512, ny=256, Ra=1e6, U=0.1, seed=20240101, noise=1e-3, nprtcl=4096,
                      inertial=False, taulag=100.0, beta=0.0, nsteps=1000, noutconfig=10),
    # production grid: 4096x2048, Ra=1e8, U=0.05, 2^17 inertial particles of
    # one Stokes number (the reference compiles one particle type; St=0.5:
    # tau_p = St*Ny/U = 20480), beta=0, 10 steps, records every 5
    "cfg1_traj": dict(nx=4096, ny=2048, Ra=1e8, U=0.05, seed=20240102, noise=1e-3, nprtcl=1 << 17,
                      inertial=True, taulag=0.5 * 2048 / 0.05, beta=0.0, nsteps=10, noutconfig=5),
}

# runs of the host program against the reference's own scratch / restart paths
SCRATCH_TRAJ_CASES = {
    # the reference's scratch state (tanh + rand(), one rank) and its 40x40
    # particle lattice, which places 2 particles on a 48x24 grid
    "traj_scratch": dict(nx=48, ny=24, Ra=1e5, U=0.1, nprtcl=2, tracer=True, taulag=50.0,
                         beta=0.0, nsteps=100, noutconfig=25),
}

NUDGE_CASES = {
    "nudge_box": dict(nx=64, ny=32, Ra=1e5, U=0.1, nsteps=30, ntempread=5, alpha=0.1,
                      nprtcl=1600, seed=11, npy=2),
    # restart route of the nudging program (scratch=0, contin=0)
    "nudge_restart": dict(nx=64, ny=32, Ra=1e5, U=0.1, nsteps=30, ntempread=5, alpha=0.1,
                          nprtcl=1600, seed=13, npy=2, restart=True),
}


def bilinear_vec(fld: np.ndarray, xs: np.ndarray, ys: np.ndarray) -> np.ndarray:
    """bilinear_np at many points: the same corner order and the same
    operation order element by element, so the results are identical"""
    ny, nx = fld.shape
    x1 = xs.astype(np.int64)
    y1 = ys.astype(np.int64)
    x2, y2 = x1 + 1, y1 + 1
    F = lambda i, j: fld[(j - 1) % ny, (i - 1) % nx]
    return (F(x1, y1) * (x2 - xs) * (y2 - ys) + F(x2, y1) * (xs - x1) * (y2 - ys)
            + F(x1, y2) * (x2 - xs) * (ys - y1) + F(x2, y2) * (xs - x1) * (ys - y1))


def traj_case(name: str) -> dict:
    c = dict(TRAJ_CASES[name] if name in TRAJ_CASES else CONFIG_CASES[name])
    base = closure(c["nx"], c["ny"], Ra=c["Ra"], Pr=1.0, U=c["U"])
    params = dict(base, twall="dirichlet", nudge="none", beta=c["beta"],
                  noutconfig=c["noutconfig"], record_full=True)
    o = Oracle(params, c["nprtcl"])
    o.init_conduction(seed=c["seed"], noise=c["noise"])
    rng = np.random.default_rng(c["seed"] + 1000)
    n, nx, ny = c["nprtcl"], c["nx"], c["ny"]
    px = rng.uniform(0.01, nx - 0.01, n)
    py = rng.uniform(1.01, ny - 0.01, n)
    pu = bilinear_vec(o.u, px, py)
    pv = bilinear_vec(o.v, px, py)
    c.update(base=base, params=params, f0=o.f.copy(), g0=o.g.copy(),
             rho0=o.rho.copy(), u0=o.u.copy(), v0=o.v.copy(), T0=o.T.copy(),
             ids=np.arange(n, dtype=np.int32), px=px, py=py, pu=pu, pv=pv,
             ptype=np.full(n, 1 if c["inertial"] else 0, np.int32),
             invtau=np.full(n, 1.0 / c["taulag"]))
    return c


def run_oracle_traj(c: dict) -> dict:
    o = Oracle(c["params"], c["nprtcl"])
    o.f[:] = c["f0"]
    o.g[:] = c["g0"]
    o.moments_from_pre(c["f0"], c["g0"])
    o.set_particles(c["ids"], c["px"], c["py"], c["pu"], c["pv"], c["ptype"], c["invtau"])
    recs = {}
    for s in range(1, c["nsteps"] + 1):
        o.step(s)
        st, r = o.record()
        if st == s:
            recs[s] = r
    return dict(f=o.f.copy(), g=o.g.copy(), rho=o.rho.copy(), u=o.u.copy(), v=o.v.copy(),
                T=o.T.copy(), records=recs, energy=o.energy(),
                px=o.pa["x"][: c["nprtcl"]].copy(), py=o.pa["y"][: c["nprtcl"]].copy())


def nudge_case(name: str) -> dict:
    from oracle import refrun

    c = dict(NUDGE_CASES[name])
    nx, ny, N, nt, nsteps = c["nx"], c["ny"], c["nprtcl"], c["ntempread"], c["nsteps"]
    base = closure(nx, ny, Ra=c["Ra"], Pr=1.0, U=c["U"])
    rng = np.random.default_rng(c["seed"])
    ids0 = (rng.permutation(N) + 100).astype(np.int32)
    x0 = rng.uniform(0, nx, N)
    y0 = rng.uniform(1, ny, N)
    T0 = rng.uniform(-0.5, 0.5, N)
    files = {}
    x, y, T = x0.copy(), y0.copy(), T0.copy()
    for s in range(nt, nsteps + nt, nt):
        x = (x + rng.normal(0, 2.0, N)) % nx
        y = np.clip(y + rng.normal(0, 1.0, N), 1.0, ny)
        jump = rng.random(N) < 0.01
        y[jump] = np.where(y[jump] > ny / 2, y[jump] - ny + 2, y[jump] + ny - 2)
        T = T + rng.normal(0, 0.05, N)
        perm = rng.permutation(N)
        files[s] = dict(x=x[perm].copy(), y=y[perm].copy(), id=ids0[perm].copy(),
                        temp=T[perm].copy())
    Tic = refrun.scratch_ic_T(nx, ny, base["Tup"], base["Tdown"], c["npy"])
    params = dict(base, twall="adiabatic", nudge="refbox", alpha=c["alpha"], ntempread=nt)
    c.update(base=base, params=params, Tic=Tic,
             init_obs=dict(x=x0, y=y0, T=T0, id=ids0), files=files)
    if c.get("restart"):
        # positive restart populations (restore* abort on an exact zero)
        rr = np.random.default_rng(c["seed"] + 500)
        Tr = rr.uniform(-0.5, 0.5, (ny, nx))
        Tr[np.abs(Tr) < 1e-3] = 1e-3
        c["restart_pops"] = dict(
            f=W[:, None, None] * (1.0 + 1e-3 * rr.uniform(-1, 1, (9, ny, nx))),
            g=Tr[None] * W[:, None, None] * (1.0 + 1e-3 * rr.uniform(-1, 1, (9, ny, nx))),
            fpre=W[:, None, None] * (1.0 + 1e-3 * rr.uniform(-1, 1, (9, ny, nx))),
            gpre=Tr[None] * W[:, None, None] * (1.0 + 1e-3 * rr.uniform(-1, 1, (9, ny, nx))))
    return c


def initial_box_mask(nx: int, ny: int) -> np.ndarray:
    """nudge_vol of set_nudge_vol (contin==0, tempvel_nudge.c:2054-2079): the
    7x7 boxes around the 40x40 particle lattice of a 1680x840 run"""
    xs = [5]
    for i in range(1, 40):
        xs.append(xs[-1] + 42 + (i % 2))
    xs[-1] += 3
    ys = [10 + 21 * i for i in range(40)]
    i = np.arange(1, nx + 1)[None, :]
    j = np.arange(1, ny + 1)[:, None]
    m = np.zeros((ny, nx), bool)
    for a in xs:
        for b in ys:
            m |= (np.abs(i - a) < 4) & (np.abs(j - b) < 4)
    return m


def nudge_initial_state(c: dict) -> dict:
    """f, g, rho, u, v, T at the start of the nudging run (interior arrays)"""
    ny, nx = c["ny"], c["nx"]
    if c.get("restart"):
        rp = c["restart_pops"]
        T = np.zeros((ny, nx))
        m = initial_box_mask(nx, ny)
        # inithydro contin==0 (tempvel_nudge.c:598-617): sum of congpre in k order
        t = np.zeros((ny, nx))
        for k in range(9):
            t = t + rp["gpre"][k]
        T[m] = t[m]
        return dict(f=W[:, None, None] * np.ones((1, ny, nx)), g=rp["g"].copy(),
                    rho=np.ones((ny, nx)), u=np.zeros((ny, nx)), v=np.zeros((ny, nx)), T=T)
    return dict(f=W[:, None, None] * np.ones((1, ny, nx)), g=c["Tic"][None] * W[:, None, None],
                rho=np.ones((ny, nx)), u=np.zeros((ny, nx)), v=np.zeros((ny, nx)), T=c["Tic"].copy())


PROFILE_EVERY = 10  # the nudging fixtures' nout: the reference writes profiles.<step>.dat


def run_oracle_nudge(c: dict, ranks_y: int = 1) -> dict:
    """the nudging run on the oracle; profiles every PROFILE_EVERY steps as
    the reference prints them from a run on `ranks_y` ranks in y"""
    o = Oracle(c["params"], c["nprtcl"])
    st = nudge_initial_state(c)
    o.f[:] = st["f"]
    o.g[:] = st["g"]
    o.rho[:] = st["rho"]
    o.T[:] = st["T"]
    o.u[:] = 0.0
    o.v[:] = 0.0
    io = c["init_obs"]
    o.nudge_init(io["x"], io["y"], io["T"], io["id"])
    nt = c["ntempread"]
    profiles = {}
    for s in range(1, c["nsteps"] + 1):
        if s % nt == 1:
            d = c["files"][s + nt - 1]
            o.nudge_load(d["x"], d["y"], d["id"], d["temp"])
        o.step(s)
        if s % PROFILE_EVERY == 0:
            profiles[s] = o.profile(ranks_y)
    return dict(f=o.f.copy(), g=o.g.copy(), T=o.T.copy(), u=o.u.copy(), v=o.v.copy(),
                nudge_vol=o.nudge_vol.copy(), tempreadint=o.tempreadint.copy(), profiles=profiles)


def sha256(a: np.ndarray) -> str:
    """digest of an array's values in C order (little-endian)"""
    import hashlib

    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()).hexdigest()


def record_digest(rec: dict, fields) -> str:
    """digest of one particle record: ids in increasing order, then each
    field in `fields` order, rows ordered by id"""
    import hashlib

    order = np.argsort(rec["id"], kind="stable")
    h = hashlib.sha256(np.ascontiguousarray(rec["id"][order], "<i4").tobytes())
    for k in fields:
        h.update(np.ascontiguousarray(rec[k][order], "<f8").tobytes())
    return h.hexdigest()


# the sampled values kept beside the digests: rows and every 64th column
def sample_rows(ny: int):
    return np.array(sorted({0, 1, ny // 2, ny - 2, ny - 1}), np.int64)


def sample_pops(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a[:, sample_rows(a.shape[1])][:, :, ::64])


def printed(a: np.ndarray) -> np.ndarray:
    """values as the reference's "%e" prints them"""
    return np.vectorize(lambda v: float("%e" % v))(a)


def golden_path(name: str) -> Path:
    return GOLDEN / f"{name}.npz"


def load_golden(name: str) -> dict:
    z = np.load(golden_path(name), allow_pickle=False)
    return {k: z[k] for k in z.files}


def adjoint_case(seed: int, nx: int = 48, ny: int = 24, nsteps: int = 40, every: int = 4,
                 nobs: int = 30) -> dict:
    """Assimilation window: observations of a truth run (seeded conduction
    state with its own noise) at fixed random positions every `every` steps;
    the window starts from another seeded state."""
    base = closure(nx, ny, Ra=1e5, Pr=1.0, U=0.1)
    params = dict(base, twall="dirichlet", nudge="none")
    rng = np.random.default_rng(seed)
    j = np.arange(ny)
    Tcol = base["Tdown"] + (base["Tup"] - base["Tdown"]) * ((j + 0.5) / ny)
    T_truth = Tcol[:, None] + 2e-2 * rng.uniform(-1, 1, (ny, nx))
    T0 = Tcol[:, None] + 2e-2 * rng.uniform(-1, 1, (ny, nx))
    steps = np.arange(every, nsteps + 1, every, dtype=np.int32)
    ox = rng.uniform(0.5, nx - 0.5, (len(steps), nobs))
    oy = rng.uniform(1.0, ny, (len(steps), nobs))
    oT = truth_obs(params, T_truth, nsteps, steps, ox, oy)
    return dict(params=params, base=base, nx=nx, ny=ny, nsteps=nsteps, steps=steps, ox=ox, oy=oy,
                oT=oT, T0=T0, T_truth=T_truth)


def truth_obs(params: dict, T_truth: np.ndarray, nsteps: int, steps, ox, oy) -> np.ndarray:
    """temperatures of the truth run at the observation points"""
    nx, ny = int(params["nx"]), int(params["ny"])
    o = Oracle(params, 0)
    f = W[:, None, None] * np.ones((1, ny, nx))
    g = np.empty((9, ny, nx))
    for k in range(9):
        g[k] = T_truth * W[k]
    o.f[:] = f
    o.g[:] = g
    o.moments_from_pre(o.f.copy(), o.g.copy())
    out = np.zeros((len(steps), ox.shape[1]))
    a = 0
    for s in range(1, nsteps + 1):
        o.step(s)
        if a < len(steps) and steps[a] == s:
            out[a] = [bilinear_np(o.T, x, y) for x, y in zip(ox[a], oy[a])]
            a += 1
    return out
