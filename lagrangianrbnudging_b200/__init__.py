"""B200-native thermal lattice-Boltzmann Rayleigh-Benard step loop with
Lagrangian particles and temperature nudging.

The compute path is liblbrb.so (hand-written CUDA for sm_100a behind the
C-ABI of include/lbrb.h).  This module binds that ABI with ctypes for the
tests, the benchmark and Python callers; there is no CPU fallback: when the
library or a CUDA device is missing, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "liblbrb.so"

OK = 0
ERRORS = {
    -1: "LBRB_ERR_ARG", -2: "LBRB_ERR_CUDA", -3: "LBRB_ERR_NOMEM", -4: "LBRB_ERR_STATE",
    -5: "LBRB_ERR_NONFINITE", -6: "LBRB_ERR_RANGE", -7: "LBRB_ERR_OVERFLOW", -8: "LBRB_ERR_IDS",
    -9: "LBRB_ERR_UNSUPPORTED",
}
ERR_CODES = {v: k for k, v in ERRORS.items()}
PREC = {"fp64": 0, "fp32": 1}
TWALL = {"dirichlet": 0, "adiabatic": 1}
NUDGE = {"none": 0, "refbox": 1, "bilinear": 2}
LAYOUT = {"ref": 0, "soa": 1}
REC_NAMES = ["x", "y", "u", "v", "xo", "yo", "uo", "vo", "temp",
             "dtu", "dtv", "dxu", "dxv", "dyu", "dyv", "fu", "fv"]

# every symbol declared in include/lbrb.h
EXPORTS = [
    "lbrb_params_default", "lbrb_create", "lbrb_destroy", "lbrb_last_error", "lbrb_abi_version",
    "lbrb_set_populations", "lbrb_get_populations", "lbrb_set_moments", "lbrb_get_moments",
    "lbrb_moments_from_pre", "lbrb_init_conduction", "lbrb_step", "lbrb_sync", "lbrb_get_istep",
    "lbrb_set_istep", "lbrb_check_finite", "lbrb_particles_set", "lbrb_particles_get",
    "lbrb_record_pending", "lbrb_record_drain", "lbrb_nudge_init", "lbrb_nudge_load",
    "lbrb_nudge_obs", "lbrb_energy", "lbrb_nusselt", "lbrb_profile", "lbrb_set_stream",
    "lbrb_set_timing", "lbrb_get_timing", "lbrb_stats_noalloc", "lbrb_get_launch_shape",
    "lbrb_get_poststream", "lbrb_adjoint_set_obs", "lbrb_adjoint_window",
    "lbrb_ensemble_create", "lbrb_ensemble_destroy", "lbrb_ensemble_last_error",
    "lbrb_ensemble_step", "lbrb_ensemble_sync", "lbrb_ensemble_set_stream",
    "lbrb_ensemble_nvariants", "lbrb_ensemble_set_schedule", "lbrb_ensemble_get_schedule",
    "lbrb_ensemble_set_pairs", "lbrb_ensemble_get_pairs", "lbrb_ensemble_pair_variants",
    "lbrb_ensemble_set_pair_variant", "lbrb_ensemble_get_pair_variant",
    "lbrb_ensemble_set_timing", "lbrb_ensemble_get_timing",
    "lbrb_adjoint_variants", "lbrb_adjoint_set_variant", "lbrb_adjoint_get_variant",
    "lbrb_adjoint_set_store", "lbrb_adjoint_get_store",
    "lbrb_slab_set", "lbrb_slab_ghost_bytes", "lbrb_slab_buffers", "lbrb_slab_pack", "lbrb_slab_step",
    "lbrb_slab_ghost2_bytes", "lbrb_slab_buffers2", "lbrb_slab_pack2",
    "lbrb_slab_particles_set", "lbrb_slab_particle_bytes", "lbrb_slab_particle_buffers",
    "lbrb_slab_moments_pack", "lbrb_slab_particles_step", "lbrb_slab_particles_recv",
    "lbrb_slab_particles_count", "lbrb_slab_particles_get", "lbrb_slab_record_pending",
    "lbrb_slab_record_drain", "lbrb_slab_particle_format", "lbrb_slab_nudge",
    "lbrb_set_graph", "lbrb_set_pairs", "lbrb_set_pair_shape", "lbrb_get_pair_shape", "lbrb_pair_shapes",
]


class LbrbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("relax", C.c_double), ("relaxg", C.c_double),
        ("Tup", C.c_double), ("Tdown", C.c_double), ("gravity", C.c_double),
        ("precision", C.c_int), ("twall", C.c_int), ("nudge", C.c_int),
        ("alpha", C.c_double), ("ntempread", C.c_int), ("nobs", C.c_int),
        ("beta", C.c_double), ("nprtcl", C.c_int), ("noutconfig", C.c_int),
        ("record_full", C.c_int), ("record_slots", C.c_int), ("device", C.c_int),
        ("autotune", C.c_int), ("launch_shape", C.c_int), ("obs_cycle", C.c_int),
    ]


_lib = None


def lib() -> C.CDLL:
    """Load liblbrb.so (built in-tree by lagrangianrbnudging_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} is missing: run python -m lagrangianrbnudging_b200.build")
    L = C.CDLL(str(LIB_PATH))
    dp, ip, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
    sig = {
        "lbrb_params_default": (None, [C.POINTER(Params)]),
        "lbrb_create": (C.c_int, [C.POINTER(Params), C.POINTER(vp)]),
        "lbrb_destroy": (C.c_int, [vp]),
        "lbrb_last_error": (C.c_char_p, [vp]),
        "lbrb_abi_version": (C.c_int, []),
        "lbrb_set_populations": (C.c_int, [vp, dp, dp, C.c_int]),
        "lbrb_get_populations": (C.c_int, [vp, dp, dp, C.c_int]),
        "lbrb_set_moments": (C.c_int, [vp, dp, dp, dp, dp, C.c_int]),
        "lbrb_get_moments": (C.c_int, [vp, dp, dp, dp, dp, C.c_int]),
        "lbrb_moments_from_pre": (C.c_int, [vp, dp, dp, C.c_int]),
        "lbrb_init_conduction": (C.c_int, [vp, C.c_uint64, C.c_double]),
        "lbrb_step": (C.c_int, [vp, C.c_int]),
        "lbrb_sync": (C.c_int, [vp]),
        "lbrb_get_istep": (C.c_int, [vp, ip]),
        "lbrb_set_istep": (C.c_int, [vp, C.c_int]),
        "lbrb_check_finite": (C.c_int, [vp]),
        "lbrb_particles_set": (C.c_int, [vp, C.c_int, ip, dp, dp, dp, dp, ip, dp]),
        "lbrb_particles_get": (C.c_int, [vp, C.c_int, ip, dp, dp, dp, dp, dp, dp, dp, dp]),
        "lbrb_record_pending": (C.c_int, [vp, ip]),
        "lbrb_record_drain": (C.c_int, [vp, C.c_int, ip, dp, ip, ip]),
        "lbrb_nudge_init": (C.c_int, [vp, C.c_int, dp, dp, dp, ip]),
        "lbrb_nudge_load": (C.c_int, [vp, C.c_int, dp, dp, ip, dp]),
        "lbrb_nudge_obs": (C.c_int, [vp, C.c_int, C.c_int, dp, dp, dp]),
        "lbrb_energy": (C.c_int, [vp, dp, dp]),
        "lbrb_nusselt": (C.c_int, [vp, dp]),
        "lbrb_profile": (C.c_int, [vp, dp]),
        "lbrb_set_stream": (C.c_int, [vp, vp]),
        "lbrb_set_timing": (C.c_int, [vp, C.c_int]),
        "lbrb_get_timing": (C.c_int, [vp, dp, ip, C.c_int]),
        "lbrb_get_poststream": (C.c_int, [vp, dp, dp, C.c_int]),
        "lbrb_adjoint_set_obs": (C.c_int, [vp, C.c_int, ip, C.c_int, dp, dp, dp]),
        "lbrb_adjoint_window": (C.c_int, [vp, dp, C.c_int, C.c_int, dp, dp]),
        "lbrb_get_launch_shape": (C.c_int, [vp, ip, ip, ip, C.POINTER(C.c_float)]),
        "lbrb_stats_noalloc": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_double, C.c_double, C.c_double, vp, dp]),
        "lbrb_ensemble_create": (C.c_int, [C.POINTER(vp), C.c_int, C.POINTER(vp)]),
        "lbrb_ensemble_destroy": (C.c_int, [vp]),
        "lbrb_ensemble_last_error": (C.c_char_p, [vp]),
        "lbrb_ensemble_step": (C.c_int, [vp, C.c_int]),
        "lbrb_ensemble_sync": (C.c_int, [vp]),
        "lbrb_ensemble_set_stream": (C.c_int, [vp, vp]),
        "lbrb_ensemble_nvariants": (C.c_int, []),
        "lbrb_ensemble_set_schedule": (C.c_int, [vp, C.c_int]),
        "lbrb_ensemble_set_pairs": (C.c_int, [vp, C.c_int]),
        "lbrb_ensemble_get_pairs": (C.c_int, [vp, ip, ip, C.POINTER(C.c_float)]),
        "lbrb_ensemble_pair_variants": (C.c_int, []),
        "lbrb_ensemble_set_pair_variant": (C.c_int, [vp, C.c_int]),
        "lbrb_ensemble_get_pair_variant": (C.c_int, [vp, ip, ip]),
        "lbrb_ensemble_get_schedule": (C.c_int, [vp, ip, ip, ip, ip, ip, C.POINTER(C.c_float)]),
        "lbrb_ensemble_set_timing": (C.c_int, [vp, C.c_int]),
        "lbrb_ensemble_get_timing": (C.c_int, [vp, dp, ip, C.c_int]),
        "lbrb_adjoint_variants": (C.c_int, []),
        "lbrb_adjoint_set_variant": (C.c_int, [vp, C.c_int]),
        "lbrb_adjoint_get_variant": (C.c_int, [vp, ip]),
        "lbrb_adjoint_set_store": (C.c_int, [vp, C.c_int]),
        "lbrb_adjoint_get_store": (C.c_int, [vp, ip, ip, C.POINTER(C.c_size_t)]),
        "lbrb_slab_set": (C.c_int, [vp, C.c_int, C.c_int]),
        "lbrb_slab_ghost_bytes": (C.c_size_t, [vp]),
        "lbrb_slab_buffers": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
        "lbrb_slab_pack": (C.c_int, [vp]),
        "lbrb_slab_ghost2_bytes": (C.c_size_t, [vp]),
        "lbrb_slab_buffers2": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
        "lbrb_slab_pack2": (C.c_int, [vp]),
        "lbrb_slab_step": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int]),
        "lbrb_slab_particles_set": (C.c_int, [vp, C.c_int, ip, dp, dp, dp, dp, ip, dp, C.c_int, C.c_int]),
        "lbrb_slab_particle_bytes": (C.c_int, [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                               C.POINTER(C.c_size_t)]),
        "lbrb_slab_particle_buffers": (C.c_int, [vp] + [C.POINTER(vp)] * 8),
        "lbrb_slab_moments_pack": (C.c_int, [vp]),
        "lbrb_slab_particles_step": (C.c_int, [vp]),
        "lbrb_slab_particles_recv": (C.c_int, [vp]),
        "lbrb_slab_particles_count": (C.c_int, [vp, ip]),
        "lbrb_slab_particles_get": (C.c_int, [vp, C.c_int, ip, ip] + [dp] * 8),
        "lbrb_slab_record_pending": (C.c_int, [vp, ip]),
        "lbrb_slab_record_drain": (C.c_int, [vp, C.c_int, ip, ip, ip, dp]),
        "lbrb_slab_particle_format": (C.c_int, [ip, ip, ip]),
        "lbrb_slab_nudge": (C.c_int, [vp]),
        "lbrb_set_graph": (C.c_int, [vp, C.c_int]),
        "lbrb_set_pairs": (C.c_int, [vp, C.c_int]),
        "lbrb_set_pair_shape": (C.c_int, [vp, C.c_int]),
        "lbrb_pair_shapes": (C.c_int, []),
        "lbrb_get_pair_shape": (C.c_int, [vp, ip, ip, ip, C.POINTER(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "float64 C-contiguous array required"
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous, "int32 C-contiguous array required"
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def make_params(**kw) -> Params:
    p = Params()
    lib().lbrb_params_default(C.byref(p))
    for k, v in kw.items():
        if k == "precision":
            v = PREC.get(v, v)
        elif k == "twall":
            v = TWALL.get(v, v)
        elif k == "nudge":
            v = NUDGE.get(v, v)
        elif k == "record_full":
            v = int(bool(v))
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class Run:
    """One whole-domain run on one GPU, through the C-ABI."""

    def __init__(self, **params):
        self.p = make_params(**params)
        h = C.c_void_p()
        rc = lib().lbrb_create(C.byref(self.p), C.byref(h))
        if rc != OK:
            raise LbrbError(rc, "lbrb_create failed (arguments, device or memory)")
        self.h = h
        self.nx, self.ny, self.np = self.p.nx, self.p.ny, self.p.nprtcl
        self.nrec = 17 if self.p.record_full else 9

    def _ck(self, rc: int):
        if rc != OK:
            msg = lib().lbrb_last_error(self.h)
            raise LbrbError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            lib().lbrb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- state
    def set_populations(self, f, g, layout="soa"):
        f, g = _f64(f), _f64(g)
        self._ck(lib().lbrb_set_populations(self.h, _dp(f), _dp(g), LAYOUT[layout]))

    def get_populations(self, layout="soa"):
        if layout == "soa":
            shape = (9, self.ny, self.nx)
        else:
            shape = (self.nx + 2, self.ny + 2, 9)
        f = np.empty(shape)
        g = np.empty(shape)
        self._ck(lib().lbrb_get_populations(self.h, _dp(f), _dp(g), LAYOUT[layout]))
        return f, g

    def get_poststream(self, layout="soa"):
        """post-stream populations of the last step (dumpfpre/dumpgpre)"""
        shape = (9, self.ny, self.nx) if layout == "soa" else (self.nx + 2, self.ny + 2, 9)
        f = np.empty(shape)
        g = np.empty(shape)
        self._ck(lib().lbrb_get_poststream(self.h, _dp(f), _dp(g), LAYOUT[layout]))
        return f, g

    def set_moments(self, rho, u, v, T, layout="soa"):
        a = [_f64(x) for x in (rho, u, v, T)]
        self._ck(lib().lbrb_set_moments(self.h, *[_dp(x) for x in a], LAYOUT[layout]))

    def get_moments(self, layout="soa"):
        shape = (self.ny, self.nx) if layout == "soa" else (self.nx + 2, self.ny + 2)
        out = [np.empty(shape) for _ in range(4)]
        self._ck(lib().lbrb_get_moments(self.h, *[_dp(x) for x in out], LAYOUT[layout]))
        return dict(zip(("rho", "u", "v", "T"), out))

    def moments_from_pre(self, fpre, gpre, layout="soa"):
        fpre, gpre = _f64(fpre), _f64(gpre)
        self._ck(lib().lbrb_moments_from_pre(self.h, _dp(fpre), _dp(gpre), LAYOUT[layout]))

    def init_conduction(self, seed: int, noise: float):
        self._ck(lib().lbrb_init_conduction(self.h, C.c_uint64(seed), noise))

    # ---- loop
    def step(self, n: int = 1):
        self._ck(lib().lbrb_step(self.h, int(n)))

    def sync(self):
        self._ck(lib().lbrb_sync(self.h))

    @property
    def istep(self) -> int:
        s = C.c_int()
        self._ck(lib().lbrb_get_istep(self.h, C.byref(s)))
        return s.value

    def check_finite(self):
        self._ck(lib().lbrb_check_finite(self.h))

    # ---- particles
    def set_particles(self, ids, x, y, u, v, ptype, invtau):
        ids, ptype = _i32(ids), _i32(ptype)
        x, y, u, v, invtau = (_f64(a) for a in (x, y, u, v, invtau))
        self._ck(lib().lbrb_particles_set(self.h, len(ids), _ip(ids), _dp(x), _dp(y), _dp(u),
                                          _dp(v), _ip(ptype), _dp(invtau)))

    def get_particles(self):
        n = self.np
        ids = np.empty(n, np.int32)
        arrs = [np.empty(n) for _ in range(8)]
        self._ck(lib().lbrb_particles_get(self.h, n, _ip(ids), *[_dp(a) for a in arrs]))
        return dict(id=ids, **dict(zip(["x", "y", "u", "v", "xo", "yo", "uo", "vo"], arrs)))

    def pending_records(self) -> int:
        c = C.c_int()
        self._ck(lib().lbrb_record_pending(self.h, C.byref(c)))
        return c.value

    def drain_records(self, max_records: int | None = None):
        """Returns {step: {field: array}} for the drained records."""
        k = self.pending_records() if max_records is None else max_records
        if k == 0:
            return {}
        steps = np.empty(k, np.int32)
        buf = np.empty((k, self.nrec, self.np))
        ids = np.empty(self.np, np.int32)
        got = C.c_int()
        self._ck(lib().lbrb_record_drain(self.h, k, _ip(steps), _dp(buf), _ip(ids), C.byref(got)))
        out = {}
        for r in range(got.value):
            d = {"id": ids.copy()}
            for f in range(self.nrec):
                d[REC_NAMES[f]] = buf[r, f].copy()
            out[int(steps[r])] = d
        return out

    def drain_records_array(self):
        """All pending records as (steps[k], buf[k][field][nprtcl]), particles in id order."""
        k = self.pending_records()
        steps = np.empty(k, np.int32)
        buf = np.empty((k, self.nrec, self.np))
        if k == 0:
            return steps, buf
        got = C.c_int()
        self._ck(lib().lbrb_record_drain(self.h, k, _ip(steps), _dp(buf), None, C.byref(got)))
        return steps[: got.value], buf[: got.value]

    # ---- nudging
    def nudge_init(self, x, y, T, ids):
        x, y, T, ids = _f64(x), _f64(y), _f64(T), _i32(ids)
        self._ck(lib().lbrb_nudge_init(self.h, len(x), _dp(x), _dp(y), _dp(T), _ip(ids)))

    def nudge_load(self, x, y, ids, T):
        x, y, T, ids = _f64(x), _f64(y), _f64(T), _i32(ids)
        self._ck(lib().lbrb_nudge_load(self.h, len(x), _dp(x), _dp(y), _ip(ids), _dp(T)))

    def nudge_obs(self, first_step: int, x, y, T):
        x, y, T = _f64(np.atleast_2d(x)), _f64(np.atleast_2d(y)), _f64(np.atleast_2d(T))
        self._ck(lib().lbrb_nudge_obs(self.h, int(first_step), x.shape[0], _dp(x), _dp(y), _dp(T)))

    # ---- adjoint
    @staticmethod
    def adjoint_variants() -> int:
        return lib().lbrb_adjoint_variants()

    def adjoint_set_variant(self, variant: int):
        self._ck(lib().lbrb_adjoint_set_variant(self.h, int(variant)))

    def adjoint_variant(self) -> int:
        v = C.c_int()
        self._ck(lib().lbrb_adjoint_get_variant(self.h, C.byref(v)))
        return v.value

    def adjoint_set_store(self, mode: int):
        """1: keep every forward state's F and moments; 0: checkpoints and
        recompute; -1: the store when it fits (lbrb_adjoint_set_store)"""
        self._ck(lib().lbrb_adjoint_set_store(self.h, int(mode)))

    def adjoint_store(self) -> dict:
        m, u, b = C.c_int(), C.c_int(), C.c_size_t()
        self._ck(lib().lbrb_adjoint_get_store(self.h, C.byref(m), C.byref(u), C.byref(b)))
        return {"mode": m.value, "used_last": u.value, "bytes": b.value}

    def adjoint_set_obs(self, steps, x, y, T):
        steps = _i32(steps)
        x, y, T = _f64(np.atleast_2d(x)), _f64(np.atleast_2d(y)), _f64(np.atleast_2d(T))
        self._ck(lib().lbrb_adjoint_set_obs(self.h, len(steps), _ip(steps), x.shape[1], _dp(x),
                                            _dp(y), _dp(T)))

    def adjoint_window(self, T0, nsteps: int, checkpoint_every: int, gradient: bool = True):
        T0 = _f64(T0)
        J = C.c_double()
        g = np.empty((self.ny, self.nx)) if gradient else None
        self._ck(lib().lbrb_adjoint_window(self.h, _dp(T0), int(nsteps), int(checkpoint_every),
                                           C.byref(J), _dp(g)))
        return (J.value, g) if gradient else J.value

    # ---- y-slab of a larger domain (lbrb_slab_*)
    def slab_set(self, j0: int, ny_total: int):
        self._ck(lib().lbrb_slab_set(self.h, int(j0), int(ny_total)))
        self.j0, self.ny_total = int(j0), int(ny_total)

    def slab_pack(self):
        self._ck(lib().lbrb_slab_pack(self.h))

    def slab_pack2(self):
        self._ck(lib().lbrb_slab_pack2(self.h))

    def slab_buffers(self, two: bool = False):
        """device pointers (up, down, ghost_lo, ghost_hi) of the ghost-row
        exchange (two: the two-row blocks of lbrb_slab_pack2), and its bytes"""
        b = [C.c_void_p() for _ in range(4)]
        fn = lib().lbrb_slab_buffers2 if two else lib().lbrb_slab_buffers
        self._ck(fn(self.h, *[C.byref(x) for x in b]))
        nbytes = (lib().lbrb_slab_ghost2_bytes if two else lib().lbrb_slab_ghost_bytes)(self.h)
        return [x.value for x in b], int(nbytes)

    def slab_particles_set(self, ids, x, y, u, v, ptype, invtau, capacity: int = 0, handoff_capacity: int = 0):
        """keep, of the particles given (the whole domain's), those whose cell
        lies in this slab's rows"""
        ids, ptype = _i32(ids), _i32(ptype)
        x, y, u, v, invtau = (_f64(a) for a in (x, y, u, v, invtau))
        self._ck(lib().lbrb_slab_particles_set(self.h, len(ids), _ip(ids), _dp(x), _dp(y), _dp(u), _dp(v),
                                               _ip(ptype), _dp(invtau), int(capacity), int(handoff_capacity)))

    def slab_particle_buffers(self):
        """{name: (device pointer, bytes)} of the particle messages: mom_up,
        mom_down (sent), mom_lo, mom_hi (received), hand_up, hand_down,
        hand_lo, hand_hi"""
        sz = [C.c_size_t() for _ in range(3)]
        self._ck(lib().lbrb_slab_particle_bytes(self.h, *[C.byref(x) for x in sz]))
        b = [C.c_void_p() for _ in range(8)]
        self._ck(lib().lbrb_slab_particle_buffers(self.h, *[C.byref(x) for x in b]))
        names = ["mom_up", "mom_down", "mom_lo", "mom_hi", "hand_up", "hand_down", "hand_lo", "hand_hi"]
        nbytes = [sz[0].value, sz[1].value, sz[0].value, sz[1].value] + [sz[2].value] * 4
        return {k: (p.value, n) for k, p, n in zip(names, b, nbytes)}

    def slab_moments_pack(self):
        self._ck(lib().lbrb_slab_moments_pack(self.h))

    def slab_nudge(self):
        """this step's bilinear nudging at the slab's corners (after the moment exchange)"""
        self._ck(lib().lbrb_slab_nudge(self.h))

    def slab_messages_only(self):
        """the moment messages without particles (a nudged slab without particles)"""
        e = np.empty(0)
        i = np.empty(0, np.int32)
        self._ck(lib().lbrb_slab_particles_set(self.h, 0, _ip(i), _dp(e), _dp(e), _dp(e), _dp(e), _ip(i), _dp(e),
                                               -1, 0))

    def slab_particles_step(self):
        self._ck(lib().lbrb_slab_particles_step(self.h))

    def slab_particles_recv(self):
        self._ck(lib().lbrb_slab_particles_recv(self.h))

    def slab_particles_count(self) -> int:
        n = C.c_int()
        self._ck(lib().lbrb_slab_particles_count(self.h, C.byref(n)))
        return n.value

    def slab_particles_get(self):
        cap = self.slab_particles_count()
        ids = np.empty(cap, np.int32)
        arrs = [np.empty(cap) for _ in range(8)]
        n = C.c_int()
        self._ck(lib().lbrb_slab_particles_get(self.h, cap, C.byref(n), _ip(ids), *[_dp(a) for a in arrs]))
        k = n.value
        return dict(id=ids[:k], **{f: a[:k] for f, a in zip(["x", "y", "u", "v", "xo", "yo", "uo", "vo"], arrs)})

    def slab_record_pending(self) -> int:
        c = C.c_int()
        self._ck(lib().lbrb_slab_record_pending(self.h, C.byref(c)))
        return c.value

    def slab_record_drain(self, max_n: int):
        """the oldest record of this slab: (step, ids[count], buf[field][count]),
        or None when none is pending"""
        ids = np.empty(max_n, np.int32)
        buf = np.empty(self.nrec * max_n)
        step, cnt = C.c_int(), C.c_int()
        self._ck(lib().lbrb_slab_record_drain(self.h, int(max_n), C.byref(step), C.byref(cnt), _ip(ids),
                                              _dp(buf)))
        if step.value < 0:
            return None
        k = cnt.value
        return step.value, ids[:k].copy(), buf[: self.nrec * k].reshape(self.nrec, k).copy()

    # ---- streams and timing
    def set_stream(self, stream_handle: int | None):
        self._ck(lib().lbrb_set_stream(self.h, C.c_void_p(stream_handle or 0)))

    def set_graph(self, mode: int):
        """CUDA-graph replay of plain steps: -1 small grids (default), 0 off, 1 on"""
        self._ck(lib().lbrb_set_graph(self.h, int(mode)))

    def set_pairs(self, mode: int):
        """two steps per fused launch: -1 (default) and 1 where eligible, 0 off"""
        self._ck(lib().lbrb_set_pairs(self.h, int(mode)))

    @staticmethod
    def pair_shapes() -> int:
        """launch shapes of the two-step kernel (tiles, then marching strips)"""
        return lib().lbrb_pair_shapes()

    def set_pair_shape(self, shape: int):
        """fixed launch shape of the two-step kernel (0 .. pair_shapes() - 1), or -1: timed on first use"""
        self._ck(lib().lbrb_set_pair_shape(self.h, int(shape)))

    def pair_shape(self):
        sh, tx, ty, ms = C.c_int(), C.c_int(), C.c_int(), C.c_float()
        self._ck(lib().lbrb_get_pair_shape(self.h, C.byref(sh), C.byref(tx), C.byref(ty), C.byref(ms)))
        return {"shape": sh.value, "tile": [tx.value, ty.value], "tuned_ms": ms.value}

    def set_timing(self, enable: bool):
        self._ck(lib().lbrb_set_timing(self.h, int(bool(enable))))

    def get_timing(self):
        ms = np.zeros(4)
        cnt = np.zeros(4, np.int32)
        self._ck(lib().lbrb_get_timing(self.h, _dp(ms), _ip(cnt), 4))
        names = ["lb_step", "particles", "nudging", "record_copy"]
        return {n: (float(ms[i]), int(cnt[i])) for i, n in enumerate(names)}

    def launch_shape(self):
        sh, b, m, ms = C.c_int(), C.c_int(), C.c_int(), C.c_float()
        self._ck(lib().lbrb_get_launch_shape(self.h, C.byref(sh), C.byref(b), C.byref(m), C.byref(ms)))
        return {"shape": sh.value, "block": b.value, "min_blocks": m.value,
                "pull": "interior fast path" if sh.value <= 6 else "general",
                "tuned_ms": ms.value}

    # ---- diagnostics
    def energy(self):
        ke, tm = C.c_double(), C.c_double()
        self._ck(lib().lbrb_energy(self.h, C.byref(ke), C.byref(tm)))
        return ke.value, tm.value

    def nusselt(self) -> float:
        nu = C.c_double()
        self._ck(lib().lbrb_nusselt(self.h, C.byref(nu)))
        return nu.value

    def profile(self):
        out = np.empty((self.ny, 9))
        self._ck(lib().lbrb_profile(self.h, _dp(out)))
        return out


class SlabDomain:
    """One domain of nx x ny_total nodes cut into y-slabs, one handle each
    (on one or several GPUs of this process): lbrb_slab_set on each slab and
    lbrb_slab_step for the whole domain.  The slabs advance exactly as the
    whole domain in one handle would.

    heights: rows per slab, bottom to top; devices: one CUDA device per slab
    (default: all on `device`); params as for Run, with ny the whole
    domain's rows (each slab gets its own height) and nprtcl the whole
    domain's particles: each slab holds those in its rows
    (lbrb_slab_particles_set); particles and records come back merged, in
    the order the particles were set."""

    def __init__(self, heights, devices=None, **params):
        ny_total = int(params["ny"])
        heights = [int(h) for h in heights]
        if sum(heights) != ny_total or min(heights) < 3:
            raise ValueError("slab heights must be >= 3 (a handle's minimum) and add up to ny")
        devices = list(devices) if devices is not None else [params.get("device", 0)] * len(heights)
        if len(devices) != len(heights):
            raise ValueError("one device per slab")
        self.nx, self.ny = int(params["nx"]), ny_total
        self.heights = heights
        self.np = int(params.get("nprtcl", 0))
        self.nrec = 17 if params.get("record_full") else 9
        self._order = None
        self.slabs = []
        j0 = 0
        try:
            for hgt, dev in zip(heights, devices):
                r = Run(**dict(params, ny=hgt, device=dev, nprtcl=0))
                self.slabs.append(r)
                r.slab_set(j0, ny_total)
                j0 += hgt
        except Exception:
            self.close()
            raise
        self._arr = (C.c_void_p * len(self.slabs))(*[r.h for r in self.slabs])

    def close(self):
        for r in self.slabs:
            r.close()
        self.slabs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def init_conduction(self, seed: int, noise: float):
        """the whole domain's seeded conduction state, each slab its rows"""
        for r in self.slabs:
            r.init_conduction(seed, noise)

    def step(self, n: int):
        rc = lib().lbrb_slab_step(self._arr, len(self.slabs), int(n))
        if rc:
            for r in self.slabs:
                msg = lib().lbrb_last_error(r.h)
                if msg:
                    raise LbrbError(rc, msg.decode())
            raise LbrbError(rc, "slab_step")

    def set_populations(self, f, g):
        """whole-domain populations, SoA (9, ny, nx) each"""
        j0 = 0
        for r, hgt in zip(self.slabs, self.heights):
            r.set_populations(f[:, j0:j0 + hgt], g[:, j0:j0 + hgt])
            j0 += hgt

    def set_moments(self, rho, u, v, T):
        j0 = 0
        for r, hgt in zip(self.slabs, self.heights):
            r.set_moments(rho[j0:j0 + hgt], u[j0:j0 + hgt], v[j0:j0 + hgt], T[j0:j0 + hgt])
            j0 += hgt

    def moments_from_pre(self, fpre, gpre):
        """the restart route's moments from whole-domain post-stream
        populations, SoA (9, ny, nx) each (node by node: each slab its rows)"""
        j0 = 0
        for r, hgt in zip(self.slabs, self.heights):
            r.moments_from_pre(np.ascontiguousarray(fpre[:, j0:j0 + hgt]), np.ascontiguousarray(gpre[:, j0:j0 + hgt]))
            j0 += hgt

    def get_populations(self):
        parts = [r.get_populations() for r in self.slabs]
        return np.concatenate([p[0] for p in parts], axis=1), np.concatenate([p[1] for p in parts], axis=1)

    def get_moments(self):
        parts = [r.get_moments() for r in self.slabs]
        return {k: np.concatenate([p[k] for p in parts], axis=0) for k in ("rho", "u", "v", "T")}

    def nusselt(self) -> float:
        """the slabs' values weighted by their heights"""
        return float(sum(hgt * r.nusselt() for r, hgt in zip(self.slabs, self.heights)) / self.ny)

    # ---- particles: each slab holds those whose cell lies in its rows
    @property
    def istep(self) -> int:
        return self.slabs[0].istep

    def set_particles(self, ids, x, y, u, v, ptype, invtau, capacity: int = 0, handoff_capacity: int = 0):
        """the whole domain's particles (ids unique); capacity and
        handoff_capacity per slab as lbrb_slab_particles_set takes them"""
        ids = _i32(ids)
        if len(ids) != self.np or len(np.unique(ids)) != len(ids):
            raise ValueError("nprtcl particles with unique ids required")
        for r in self.slabs:
            r.slab_particles_set(ids, x, y, u, v, ptype, invtau, capacity, handoff_capacity)
        self._order = ids.copy()
        self._sorter = np.argsort(ids, kind="stable")

    def _place(self, ids):
        """positions of `ids` in the order the particles were set (each once)"""
        srt = self._order[self._sorter]
        k = np.searchsorted(srt, ids)
        if len(ids) != self.np or np.any(k >= self.np) or np.any(srt[np.minimum(k, self.np - 1)] != ids):
            raise RuntimeError("slab particles do not cover the domain's particles")
        pos = self._sorter[k]
        if len(np.unique(pos)) != self.np:
            raise RuntimeError("a particle is held by two slabs")
        return pos

    def get_particles(self):
        parts = [r.slab_particles_get() for r in self.slabs]
        pos = self._place(np.concatenate([p["id"] for p in parts]))
        out = {"id": self._order.copy()}
        for k in ("x", "y", "u", "v", "xo", "yo", "uo", "vo"):
            a = np.empty(self.np)
            a[pos] = np.concatenate([p[k] for p in parts])
            out[k] = a
        return out

    def slab_counts(self):
        return [r.slab_particles_count() for r in self.slabs]

    def pending_records(self) -> int:
        return min(r.slab_record_pending() for r in self.slabs)

    def drain_records_array(self, max_records: int | None = None):
        """The pending records (all, or the oldest max_records) as (steps[k],
        buf[k][field][nprtcl]), particles in the order they were set (each
        slab's part of a step's record placed by id)"""
        k = self.pending_records()
        if max_records is not None:
            k = min(k, int(max_records))
        steps = np.empty(k, np.int32)
        buf = np.empty((k, self.nrec, self.np))
        for q in range(k):
            recs = [r.slab_record_drain(self.np) for r in self.slabs]
            st = {rec[0] for rec in recs}
            if len(st) != 1:
                raise RuntimeError("slab records of different steps")
            steps[q] = st.pop()
            pos = self._place(np.concatenate([rec[1] for rec in recs]))
            buf[q][:, pos] = np.concatenate([rec[2] for rec in recs], axis=1)
        return steps, buf

    def drain_records(self, max_records: int | None = None):
        """{step: {field: array}} as Run.drain_records gives it"""
        steps, buf = self.drain_records_array(max_records)
        out = {}
        for q in range(len(steps)):
            d = {"id": self._order.copy()}
            for f in range(self.nrec):
                d[REC_NAMES[f]] = buf[q, f].copy()
            out[int(steps[q])] = d
        return out

    def check_finite(self):
        for r in self.slabs:
            r.check_finite()

    def nudge_obs(self, first_step: int, x, y, T):
        """bilinear observations in the whole domain's coordinates, given to
        every slab (each nudges the corners in its own rows)"""
        for r in self.slabs:
            r.nudge_obs(first_step, x, y, T)

    def nudge_init(self, x, y, T, ids):
        """box nudging: the initial observations, given to every slab (each
        keeps the running means of the boxes' nodes in its own rows)"""
        for r in self.slabs:
            r.nudge_init(x, y, T, ids)

    def nudge_load(self, x, y, ids, T):
        """box nudging: the next observation file, given to every slab"""
        for r in self.slabs:
            r.nudge_load(x, y, ids, T)


class Ensemble:
    """Independent runs advanced together (lbrb_ensemble_*): one launch per
    phase of the step covers every member, replayed from a CUDA graph.  The
    members are Run objects; their state stays theirs, so every Run method
    works between ensemble steps.  Close the ensemble before its members."""

    def __init__(self, members):
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.h for m in self.members])
        e = C.c_void_p()
        rc = lib().lbrb_ensemble_create(arr, len(self.members), C.byref(e))
        if rc != OK:
            raise LbrbError(rc, "lbrb_ensemble_create: members must share device, precision and "
                                "wall mode; no box nudging; no trajectory records")
        self.e = e

    def _ck(self, rc: int):
        if rc != OK:
            msg = lib().lbrb_ensemble_last_error(self.e)
            raise LbrbError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "e", None):
            lib().lbrb_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, n: int):
        self._ck(lib().lbrb_ensemble_step(self.e, int(n)))

    def sync(self):
        self._ck(lib().lbrb_ensemble_sync(self.e))

    def set_stream(self, cuda_stream):
        self._ck(lib().lbrb_ensemble_set_stream(self.e, C.c_void_p(cuda_stream or 0)))

    @staticmethod
    def nvariants() -> int:
        return lib().lbrb_ensemble_nvariants()

    def set_schedule(self, variant: int):
        self._ck(lib().lbrb_ensemble_set_schedule(self.e, int(variant)))

    def set_pairs(self, mode: int):
        """two steps per launch: -1 / 1 on (default), 0 off"""
        self._ck(lib().lbrb_ensemble_set_pairs(self.e, int(mode)))

    def pairs(self) -> dict:
        mode, rows, ms = C.c_int(), C.c_int(), C.c_float()
        self._ck(lib().lbrb_ensemble_get_pairs(self.e, C.byref(mode), C.byref(rows), C.byref(ms)))
        v, cols = C.c_int(), C.c_int()
        self._ck(lib().lbrb_ensemble_get_pair_variant(self.e, C.byref(v), C.byref(cols)))
        return {"mode": mode.value, "rows": rows.value, "tuned_ms": ms.value, "variant": v.value,
                "tile_cols": cols.value}

    def set_pair_variant(self, variant: int) -> None:
        """-1: time the two-step launch variants at the next paired call;
        else use that one (pair_variants() of them)"""
        self._ck(lib().lbrb_ensemble_set_pair_variant(self.e, int(variant)))

    @staticmethod
    def pair_variants() -> int:
        return int(lib().lbrb_ensemble_pair_variants())

    def schedule(self) -> dict:
        v, b, r, s, f, ms = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_float()
        self._ck(lib().lbrb_ensemble_get_schedule(self.e, C.byref(v), C.byref(b), C.byref(r),
                                                  C.byref(s), C.byref(f), C.byref(ms)))
        return {"variant": v.value, "block": b.value, "rows": r.value,
                "schedule": ["one block per tile", "persistent grid stride",
                             "persistent atomic counter"][s.value] if s.value >= 0 else None,
                "pull": {1: "interior fast path", 0: "general"}.get(f.value),
                "tuned_ms": ms.value}

    def set_timing(self, enable: bool):
        self._ck(lib().lbrb_ensemble_set_timing(self.e, int(bool(enable))))

    def get_timing(self) -> dict:
        ms = np.zeros(3)
        cnt = np.zeros(3, dtype=np.int32)
        self._ck(lib().lbrb_ensemble_get_timing(self.e, _dp(ms), _ip(cnt), 3))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(("lb_step", "aux", "apply"))}


def closure(nx: int, ny: int, Ra: float, Pr: float, U: float, dT: float = 1.0) -> dict:
    """Run parameters of the configurations: nu = U*Ny*sqrt(Pr/Ra),
    kappa = U*Ny/sqrt(Ra*Pr), tau = 3 nu + 1/2, g*beta = U^2/Ny (gravity
    negative in the reference's sign convention), T_bottom = +dT/2."""
    nu = U * ny * np.sqrt(Pr / Ra)
    kappa = U * ny / np.sqrt(Ra * Pr)
    return dict(nx=nx, ny=ny, relax=3.0 * nu + 0.5, relaxg=3.0 * kappa + 0.5,
                Tup=-0.5 * dT, Tdown=0.5 * dT, gravity=-(U * U) / ny)
