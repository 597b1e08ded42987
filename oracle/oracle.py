"""ctypes binding of the CPU restatement (``lbrb_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

TWALL = {"dirichlet": 0, "adiabatic": 1}
NUDGE = {"none": 0, "refbox": 1, "bilinear": 2}

F, G, RHO, U, V, T, UBEF, VBEF, FY, TEMPREADINT, NUDTERM, NUDGE_SRC = range(12)
PX, PY, PU, PV, PXO, PYO, PUO, PVO, PINVTAU = range(9)
REC_NAMES = ["x", "y", "u", "v", "xo", "yo", "uo", "vo", "temp",
             "dtu", "dtv", "dxu", "dxv", "dyu", "dyv", "fu", "fv"]


class OrcParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("relax", C.c_double), ("relaxg", C.c_double),
        ("Tup", C.c_double), ("Tdown", C.c_double), ("gravity", C.c_double),
        ("twall", C.c_int), ("nudge", C.c_int), ("alpha", C.c_double),
        ("ntempread", C.c_int), ("beta", C.c_double),
        ("noutconfig", C.c_int), ("record_full", C.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build_oracle()
        L = C.CDLL(str(path))
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams), C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_field.restype = dp
        L.orc_field.argtypes = [C.c_void_p, C.c_int]
        L.orc_nudge_vol.restype = ip
        L.orc_nudge_vol.argtypes = [C.c_void_p]
        L.orc_prtcl.restype = dp
        L.orc_prtcl.argtypes = [C.c_void_p, C.c_int]
        L.orc_prtcl_ids.restype = ip
        L.orc_prtcl_ids.argtypes = [C.c_void_p]
        L.orc_prtcl_type.restype = ip
        L.orc_prtcl_type.argtypes = [C.c_void_p]
        L.orc_record.restype = dp
        L.orc_record.argtypes = [C.c_void_p, ip]
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_moments_from_pre.argtypes = [C.c_void_p, dp, dp]
        L.orc_init_conduction.argtypes = [C.c_void_p, C.c_ulonglong, C.c_double]
        L.orc_splitmix_uniform.restype = C.c_double
        L.orc_splitmix_uniform.argtypes = [C.c_ulonglong, C.c_ulonglong]
        L.orc_nudge_init.argtypes = [C.c_void_p, dp, dp, dp, ip]
        L.orc_nudge_load.argtypes = [C.c_void_p, dp, dp, ip, dp]
        L.orc_nudge_obs.argtypes = [C.c_void_p, C.c_int, dp, dp, dp]
        L.orc_energy.argtypes = [C.c_void_p, dp, dp]
        L.orc_profile.argtypes = [C.c_void_p, dp]
        L.orc_profile_ranks.argtypes = [C.c_void_p, C.c_int, dp]
        L.orc_nusselt.restype = C.c_double
        L.orc_nusselt.argtypes = [C.c_void_p]
        L.orc_tlm_window.argtypes = [C.c_void_p, dp, dp, C.c_int, C.c_int, ip, C.c_int, dp, dp,
                                     dp, dp, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


def make_params(p: dict) -> OrcParams:
    return OrcParams(
        nx=int(p["nx"]), ny=int(p["ny"]),
        relax=float(p["relax"]), relaxg=float(p["relaxg"]),
        Tup=float(p["Tup"]), Tdown=float(p["Tdown"]), gravity=float(p["gravity"]),
        twall=TWALL[p.get("twall", "dirichlet")], nudge=NUDGE[p.get("nudge", "none")],
        alpha=float(p.get("alpha", 0.0)), ntempread=int(p.get("ntempread", 1)),
        beta=float(p.get("beta", 0.0)), noutconfig=int(p.get("noutconfig", 0)),
        record_full=int(bool(p.get("record_full", False))),
    )


class Oracle:
    """FP64 CPU restatement of one whole-domain reference run."""

    def __init__(self, params: dict, nprtcl: int = 0):
        self.params = dict(params)
        self.nx, self.ny = int(params["nx"]), int(params["ny"])
        self.np = int(nprtcl)
        self._p = make_params(params)
        self._h = lib().orc_create(C.byref(self._p), self.np)
        if not self._h:
            raise MemoryError("orc_create failed")
        L = lib()
        nx, ny = self.nx, self.ny

        def fview(w, shape):
            return np.ctypeslib.as_array(L.orc_field(self._h, w), shape=shape)

        self.f = fview(F, (9, ny, nx))
        self.g = fview(G, (9, ny, nx))
        self.rho, self.u, self.v, self.T = (fview(w, (ny, nx)) for w in (RHO, U, V, T))
        self.ubef, self.vbef, self.Fy = (fview(w, (ny, nx)) for w in (UBEF, VBEF, FY))
        self.tempreadint = fview(TEMPREADINT, (ny, nx))
        self.nudterm = fview(NUDTERM, (ny, nx))
        self.nudge_src = fview(NUDGE_SRC, (ny, nx))
        self.nudge_vol = np.ctypeslib.as_array(L.orc_nudge_vol(self._h), shape=(ny, nx))
        m = max(self.np, 1)
        self.pa = {n: np.ctypeslib.as_array(L.orc_prtcl(self._h, w), shape=(m,))
                   for n, w in zip(["x", "y", "u", "v", "xo", "yo", "uo", "vo", "invtau"], range(9))}
        self.pid = np.ctypeslib.as_array(L.orc_prtcl_ids(self._h), shape=(m,))
        self.ptype = np.ctypeslib.as_array(L.orc_prtcl_type(self._h), shape=(m,))
        self._rec = np.ctypeslib.as_array(L.orc_record(self._h, None), shape=(17, m))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    # -- state --------------------------------------------------------------
    def init_conduction(self, seed: int, noise: float):
        lib().orc_init_conduction(self._h, seed, noise)

    def moments_from_pre(self, fpre: np.ndarray, gpre: np.ndarray):
        fpre = np.ascontiguousarray(fpre, dtype=np.float64)
        gpre = np.ascontiguousarray(gpre, dtype=np.float64)
        lib().orc_moments_from_pre(self._h, _dp(fpre), _dp(gpre))

    def set_particles(self, ids, x, y, u, v, ptype, invtau):
        n = self.np
        self.pid[:n] = ids
        for k, a in (("x", x), ("y", y), ("u", u), ("v", v)):
            self.pa[k][:n] = a
        self.pa["xo"][:n] = x
        self.pa["yo"][:n] = y
        self.pa["uo"][:n] = u
        self.pa["vo"][:n] = v
        self.ptype[:n] = ptype
        self.pa["invtau"][:n] = invtau

    def step(self, istep: int):
        lib().orc_step(self._h, int(istep))

    def record(self):
        st = C.c_int(-1)
        lib().orc_record(self._h, C.byref(st))
        return st.value, {n: self._rec[i, : self.np].copy() for i, n in enumerate(REC_NAMES)}

    # -- nudging ------------------------------------------------------------
    def nudge_init(self, x, y, T, ids):
        x, y, T = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, T))
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        lib().orc_nudge_init(self._h, _dp(x), _dp(y), _dp(T), _ip(ids))

    def nudge_load(self, x, y, ids, T):
        x, y, T = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, T))
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        lib().orc_nudge_load(self._h, _dp(x), _dp(y), _ip(ids), _dp(T))

    def nudge_obs(self, x, y, T):
        x, y, T = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, T))
        lib().orc_nudge_obs(self._h, len(x), _dp(x), _dp(y), _dp(T))

    # -- diagnostics ----------------------------------------------------------
    def energy(self):
        ke, tm = C.c_double(), C.c_double()
        lib().orc_energy(self._h, C.byref(ke), C.byref(tm))
        return ke.value, tm.value

    def profile(self, ranks_y: int = 1):
        """per-row profiles; ranks_y: the reference's ranks in y (the last
        row of each rank takes T(j+1) from its halo row)"""
        out = np.zeros((self.ny, 9))
        lib().orc_profile_ranks(self._h, int(ranks_y), _dp(out))
        return out

    def nusselt(self) -> float:
        return lib().orc_nusselt(self._h)

    def tlm_window(self, T0, dT0, nsteps, steps, ox, oy, oT):
        """misfit J and its directional derivative along dT0 (FP64 tangent-linear model)"""
        T0, dT0 = np.ascontiguousarray(T0, np.float64), np.ascontiguousarray(dT0, np.float64)
        steps = np.ascontiguousarray(steps, np.int32)
        ox, oy, oT = (np.ascontiguousarray(np.atleast_2d(a), np.float64) for a in (ox, oy, oT))
        J, dJ = C.c_double(), C.c_double()
        lib().orc_tlm_window(self._h, _dp(T0), _dp(dT0), int(nsteps), len(steps), _ip(steps),
                             ox.shape[1], _dp(ox), _dp(oy), _dp(oT), C.byref(J), C.byref(dJ))
        return J.value, dJ.value


def splitmix_uniform(seed: int, index: int) -> float:
    return lib().orc_splitmix_uniform(seed, index)


def closure(nx: int, ny: int, Ra: float, Pr: float, U: float, dT: float = 1.0) -> dict:
    """Closure of the configurations: nu = U*Ny*sqrt(Pr/Ra), kappa =
    U*Ny/sqrt(Ra*Pr), tau = 3 nu + 0.5, g*beta = U^2/Ny (gravity is negative
    in the reference's sign convention)."""
    nu = U * ny * np.sqrt(Pr / Ra)
    kappa = U * ny / np.sqrt(Ra * Pr)
    return dict(nx=nx, ny=ny, relax=3.0 * nu + 0.5, relaxg=3.0 * kappa + 0.5,
                Tup=-0.5 * dT, Tdown=0.5 * dT, gravity=-(U * U) / ny)
