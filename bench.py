#!/usr/bin/env python
"""Benchmark of the B200 step loop on the production-trajectory workload.

Workload (one GPU): 4096 x 2048 Rayleigh-Benard, Ra = 1e8, Pr = 1, U = 0.05,
2^17 Lagrangian particles split over Stokes numbers {0 (tracer), 0.1, 0.5, 1,
2} (26215, 26215, 26214, 26214, 26214), tau_p = St*Ny/U, beta = 0, particle
record (x, y, u, v, xo, yo, uo, vo, T) every 20 steps.  Synthetic seeded
initial state: linear conduction + 1e-3 uniform noise; particles uniform.

One "step" = one time step of the whole loop: fused stream/collide kernel,
particle kernel, and every 20th step a record copied to pinned host memory.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  With N > 1 (torchrun) every rank advances its
own independent instance (different seed): weak scaling, no per-step
collective; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import signal
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NX, NY = 4096, 2048
RA, PR, U = 1e8, 1.0, 0.05
ST = [0.0, 0.1, 0.5, 1.0, 2.0]
NPRTCL = 1 << 17
NOUTCONFIG = 20
SEED = 20240531
WORKLOAD = (f"production trajectories: {NX}x{NY} Ra=1e8 Pr=1 U=0.05, 2^17 particles over "
            f"St {{0,0.1,0.5,1,2}} (tau_p=St*Ny/U, beta=0), record every {NOUTCONFIG} steps")
# algorithmic bytes per node and step of the fused kernel: 18 populations read + written
ALG_BYTES = {"fp32": 144, "fp64": 288}
FALLBACK_HBM_GBS = 6650.0
REF_TAG = "bench_c1"
REF_STEPS_CAP_S = 60.0  # bound on the reference's timed window
# one metric string for both arms (ours and the reference build), so the two
# lines compare directly; the precision is a key of each line
METRIC = "MLUPS (lattice updates/s, whole step incl. particles)"


def st_counts(n: int = NPRTCL) -> list[int]:
    base, extra = divmod(n, len(ST))
    return [base + (1 if i < extra else 0) for i in range(len(ST))]


def particle_setup(seed: int, n: int = NPRTCL):
    """Seeded uniform positions in the reference frame, per-particle type and 1/tau_p."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, NX, n)
    x[x <= 0.0] = 0.5
    y = rng.uniform(1.0, NY, n)
    ptype = np.empty(n, np.int32)
    invtau = np.empty(n)
    k = 0
    for st, c in zip(ST, st_counts(n)):
        ptype[k:k + c] = 0 if st == 0.0 else 1
        invtau[k:k + c] = 0.0 if st == 0.0 else U / (st * NY)
        k += c
    return np.arange(n, dtype=np.int32), x, y, ptype, invtau


def bilinear_np(fld: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    ny, nx = fld.shape
    x1 = x.astype(np.int64)
    y1 = y.astype(np.int64)
    ix1, ix2 = (x1 - 1) % nx, x1 % nx
    jy1, jy2 = (y1 - 1) % ny, y1 % ny
    wx2, wy2 = x - x1, y - y1
    wx1, wy1 = (x1 + 1) - x, (y1 + 1) - y
    return (fld[jy1, ix1] * wx1 * wy1 + fld[jy1, ix2] * wx2 * wy1
            + fld[jy2, ix1] * wx1 * wy2 + fld[jy2, ix2] * wx2 * wy2)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), [c.strip() for c in line.split(",")]))

    def mark(self):
        return time.time()

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0: float, t1: float) -> dict:
        rows = [r for t, r in self.rows if t0 <= t <= t1 + 0.1] or [r for _, r in self.rows]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------- our arm
PAIRS_MODE = -1  # lbrb_set_pairs of the handles bench creates (--no-pairs: 0)


def make_run(lb, precision: str, seed: int, device: int, slots: int):
    base = lb.closure(NX, NY, Ra=RA, Pr=PR, U=U)
    r = lb.Run(**base, precision=precision, twall="dirichlet", nudge="none", beta=0.0,
               nprtcl=NPRTCL, noutconfig=NOUTCONFIG, record_full=False, record_slots=slots,
               device=device)
    r.set_pairs(PAIRS_MODE)
    return r, base


def init_run(r, seed: int):
    r.init_conduction(seed, 1e-3)
    m = r.get_moments()
    ids, x, y, ptype, invtau = particle_setup(seed + 1)
    u = bilinear_np(m["u"], x, y)
    v = bilinear_np(m["v"], x, y)
    r.set_particles(ids, x, y, u, v, ptype, invtau)
    return m


def timed_steps(r, torch, steps: int, warmup: int, dist, device: int, clock=None):
    """W warm-up steps, then the timed region: K steps as a user runs them
    (CUDA events around the region only, on the handle's stream).  Then the
    same K steps again with an event pair around every launch of the handle
    (lbrb_set_timing), for the per-kernel figures: that instrumentation
    serialises the launches (no programmatic dependent launch between them),
    so it stays out of the timed region; the launch sequence is the same.
    clock: a ClockSampler, whose samples during the timed region are kept."""
    r.step(warmup)
    r.sync()
    r.drain_records()
    # a real (non-default) stream: the events and all of the handle's work share it
    stream = torch.cuda.Stream()
    r.set_stream(stream.cuda_stream)

    def window(instrumented: bool):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        r.set_timing(instrumented)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.time()
        e0.record(stream)
        r.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        t1 = time.time()
        if dist is not None:
            dist.barrier()
        timing = r.get_timing() if instrumented else None
        r.set_timing(False)
        r.sync()
        return e0.elapsed_time(e1), timing, (t0, t1)

    ms, _, span = window(False)
    clocks = clock.summary(*span) if clock is not None else None
    recs = r.drain_records()
    ms_inst, timing, _ = window(True)
    r.drain_records()
    r.set_stream(None)
    timing["window_ms"] = (ms_inst, 0)
    return ms, timing, recs, span if clock is None else clocks


def max_over_ranks(torch, dist, v: float) -> float:
    """the slowest rank's time: one all-reduce (NCCL on the GPUs, gloo on CPU)"""
    if dist is None:
        return v
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(rank: int) -> int:
    """each replica's own seed (independent instances, no shared state)"""
    return SEED + 7919 * rank


def whole_job_mlups(world: int, nodes: int, steps: int, ms_max: float) -> float:
    """lattice updates of all ranks over the slowest rank's time"""
    return world * nodes * steps / (ms_max * 1e3)


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


# the sources of the fused kernels: a traffic capture counts only for the build it measured
KERNEL_SOURCES = ["lb_kernels.cu", "lb_pair.cuh", "lb_node.cuh", "lbrb_internal.cuh"]


def kernel_sources_sha() -> str:
    import hashlib

    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        h.update((ROOT / "lagrangianrbnudging_b200" / "csrc" / name).read_bytes())
    return h.hexdigest()[:16]


def profiled_traffic(precision: str, kernel: str):
    """DRAM bytes per node of one launch of `kernel` ("lb_pair_kernel<float>",
    ...) from the committed ncu summary (profiles/lb_step_traffic.json: per
    precision, an entry per kernel), or None when that capture was made on
    other kernel sources than this build's or holds no such kernel."""
    p = ROOT / "profiles" / "lb_step_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        if d.get("kernel_sources_sha") != kernel_sources_sha():
            return None
        return float(d[precision][kernel]["bytes_per_node"])
    except Exception:
        return None


def e2e(lb, torch, precision: str, seed: int, steps: int, device: int, dist):
    r, base = make_run(lb, precision, seed, device, steps // NOUTCONFIG + 2)
    w = np.array([16 / 36, 4 / 36, 4 / 36, 4 / 36, 4 / 36, 1 / 36, 1 / 36, 1 / 36, 1 / 36])
    rng = np.random.default_rng(seed)
    j = np.arange(NY)
    Tcol = base["Tdown"] + (base["Tup"] - base["Tdown"]) * ((j + 0.5) / NY)

    def pinned(n, torch_dtype):
        return torch.empty(n, dtype=torch_dtype, pin_memory=True).numpy()

    nh = (NX + 2) * (NY + 2)
    f = pinned(nh * 9, torch.float64).reshape(NX + 2, NY + 2, 9)
    g = pinned(nh * 9, torch.float64).reshape(NX + 2, NY + 2, 9)
    T = np.empty((NX + 2, NY + 2))
    T[1:-1, 1:-1] = Tcol[None, :] + 1e-3 * (2.0 * rng.random((NX, NY)) - 1.0)
    T[0], T[-1] = T[-2], T[1]
    T[:, 0], T[:, -1] = T[:, -2], T[:, 1]
    f[:] = w
    np.multiply(T[:, :, None], w[None, None, :], out=g)
    rho = pinned(nh, torch.float64).reshape(NX + 2, NY + 2)
    uu = pinned(nh, torch.float64).reshape(NX + 2, NY + 2)
    vv = pinned(nh, torch.float64).reshape(NX + 2, NY + 2)
    Th = pinned(nh, torch.float64).reshape(NX + 2, NY + 2)
    rho[:] = 1.0
    uu[:] = 0.0
    vv[:] = 0.5 * (-base["gravity"]) * T
    Th[:] = T
    ids, x, y, ptype, invtau = particle_setup(seed + 1)
    pu = np.zeros(NPRTCL)
    pv = bilinear_np(vv[1:-1, 1:-1].T.copy(), x, y)
    out_m = [pinned(nh, torch.float64).reshape(NX + 2, NY + 2) for _ in range(4)]
    stream = torch.cuda.Stream()
    r.set_stream(stream.cuda_stream)
    nrec = steps // NOUTCONFIG
    recbuf = pinned(max(nrec, 1) * 9 * NPRTCL, torch.float64).reshape(max(nrec, 1), 9, NPRTCL)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r.set_populations(f, g, layout="ref")
    r.set_moments(rho, uu, vv, Th, layout="ref")
    r.set_particles(ids, x, y, pu, pv, ptype, invtau)
    import ctypes as C
    st = np.empty(max(nrec, 1), np.int32)
    got = C.c_int()
    # as a host program runs: the steps go out in chunks, and the records of
    # one chunk are drained (into the caller's arrays) while the next runs
    chunk = 25 * NOUTCONFIG
    done = drained = 0
    prev = 0  # records of the chunk before the one in flight
    while done < steps:
        n = min(chunk, steps - done)
        r.step(n)
        done += n
        if prev:
            r._ck(lb.lib().lbrb_record_drain(r.h, prev, lb._ip(st[drained:]), lb._dp(recbuf[drained:]), None,
                                             C.byref(got)))
            drained += got.value
        prev = (done // NOUTCONFIG) - ((done - n) // NOUTCONFIG)
    r._ck(lb.lib().lbrb_record_drain(r.h, nrec - drained, lb._ip(st[drained:]), lb._dp(recbuf[drained:]), None,
                                     C.byref(got)))
    drained += got.value
    got.value = drained
    r._ck(lb.lib().lbrb_get_moments(r.h, *[lb._dp(a) for a in out_m], lb.LAYOUT["ref"]))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    r.set_stream(None)
    h2d = 2 * f.nbytes + 4 * rho.nbytes + NPRTCL * (4 * 8 + 4 + 4 + 8)
    d2h = got.value * 9 * NPRTCL * 8 + 4 * rho.nbytes
    r.close()
    return ms, h2d, d2h


def pinned_copy_rates(torch, device: int, nbytes: int = 1 << 29) -> tuple[float, float]:
    """host<->device copy rates (GB/s) of pinned memory on this box: one
    cudaMemcpyAsync each way of `nbytes`, timed with CUDA events after a
    warm-up copy"""
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{device}")
    rates = []
    for to_dev in (True, False):
        for rep in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if to_dev:
                d.copy_(h, non_blocking=True)
            else:
                h.copy_(d, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
        rates.append(nbytes / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del h, d
    return rates[0], rates[1]


def run_ours(args, torch, dist, rank: int, world: int, device: int) -> dict | None:
    import lagrangianrbnudging_b200 as lb
    from lagrangianrbnudging_b200 import build as b

    if rank == 0:
        b.build()
    if dist is not None:
        dist.barrier()
    seed = rank_seed(rank)
    K, W = args.steps, args.warmup
    nodes = NX * NY
    out = {}
    # -- headline: FP32 shifted populations
    r, base = make_run(lb, "fp32", seed, device, K // NOUTCONFIG + W // NOUTCONFIG + 4)
    init_run(r, seed)
    with ClockSampler(device) as clk:
        ms, timing, recs, clocks = timed_steps(r, torch, K, W, dist, device, clock=clk)
    shape32 = r.launch_shape()
    pair32 = r.pair_shape()
    nu32 = r.nusselt()
    ke32, _ = r.energy()
    r.close()
    ms = max_over_ranks(torch, dist, ms)
    lb_ms, lb_n = timing["lb_step"]
    pt_ms, pt_n = timing["particles"]
    # -- FP64 reference-order populations on the same workload
    K64 = max(K // 2, 10)
    r64, _ = make_run(lb, "fp64", seed, device, K64 // NOUTCONFIG + W // NOUTCONFIG + 4)
    init_run(r64, seed)
    ms64, timing64, _, _ = timed_steps(r64, torch, K64, W, dist, device)
    shape64 = r64.launch_shape()
    pair64 = r64.pair_shape()
    # the same number of steps as the FP32 run (two windows each) for the Nu
    # comparison, draining the records as they come
    rest = 2 * (K - K64)
    r64.drain_records()
    while rest > 0:
        n = min(rest, 4 * NOUTCONFIG)  # (fewer records per call than the ring holds)
        r64.step(n)
        r64.drain_records()
        rest -= n
    r64.sync()
    nu64 = r64.nusselt()
    ke64, _ = r64.energy()
    r64.close()
    ms64 = max_over_ranks(torch, dist, ms64)
    # -- end to end through the C-ABI with host buffers
    e2e_ms = e2e_h2d = e2e_d2h = None
    if not args.no_e2e:
        e2e_ms, e2e_h2d, e2e_d2h = e2e(lb, torch, "fp32", seed, K, device, dist)
        e2e_ms = max_over_ranks(torch, dist, e2e_ms)
        h2d_gbs, d2h_gbs = pinned_copy_rates(torch, device)
    # sections with independent units: every rank takes its share (replicas
    # for the adjoint window's timing), results gathered once
    sec = {}
    if not args.no_adjoint:
        sec["adjoint"] = run_adjoint_bench(lb, torch, device, dist=dist, rank=rank, world=world)
    if world == 1 and not args.no_accuracy:
        sec["accuracy"] = run_accuracy(lb, device)
    if not args.no_nudging:
        sec["nudging"] = run_nudging_bench(lb, torch, device, args.nudging_steps, dist=dist, rank=rank,
                                           world=world)
    if not args.no_ensemble:
        sec["ensemble"] = run_ensemble_bench(lb, torch, device, args.ensemble_steps, dist=dist, rank=rank,
                                             world=world)
    if world == 1 and not args.no_slab:
        sec["slab"] = run_slab_bench(lb, torch, device)
    if rank != 0:
        return None
    mlups = whole_job_mlups(world, nodes, K, ms)
    mlups64 = whole_job_mlups(world, nodes, K64, ms64)
    peak, peak_kind = measured_peak()
    # the fused launches of the instrumented window: node-steps per launch
    # (2 for a two-step launch; the call's last step is a single one)
    avg_lb = lb_ms / max(lb_n, 1)
    spl = K / max(lb_n, 1)
    achieved = ALG_BYTES["fp32"] * nodes * spl / (avg_lb * 1e-3) / 1e9
    tr = None  # (set below, once the kernel of the launches is known)
    spl64 = K64 / max(timing64["lb_step"][1], 1)
    avg_lb64 = timing64["lb_step"][0] / max(timing64["lb_step"][1], 1)
    achieved64 = ALG_BYTES["fp64"] * nodes * spl64 / (avg_lb64 * 1e-3) / 1e9
    if pair32["shape"] >= 0 and spl > 1.5:
        kernel32 = "lb_march_kernel<float>" if pair32["shape"] >= 9 else "lb_pair_kernel<float>"
    else:
        kernel32 = "lb_node_kernel<float>"
    tr = profiled_traffic("fp32" if spl > 1.5 else "fp32_single", kernel32)
    out.update({
        "metric": METRIC,
        "value": round(mlups, 1),
        # the FP64 path on the same workload: bit-identical to the reference's
        # arithmetic, the like-for-like figure against the reference arm
        "value_fp64": round(mlups64, 1),
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(ms / K, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic (seeded conduction + noise; seeded uniform particles)",
        "config": {"workload": WORKLOAD, "grid": f"{NX}x{NY}", "particles": NPRTCL,
                   "precision": "fp32-shifted populations, fp64 particles",
                   "l2": "state 1.5 GB > 126 MB L2 on every step (no flush needed)",
                   "parallelism": f"{world} independent instances (replicas), no collective"},
        "roofline": {"bound": "hbm", "kernel": kernel32,
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "alg_bytes_per_node": ALG_BYTES["fp32"],
                     "node_steps_per_launch": round(spl, 4),
                     "avg_launch_ms": round(avg_lb, 5),
                     "traffic": (round(tr * nodes) if tr else None),
                     "traffic_source": ("profiles/lb_step_traffic.json, captured on these kernel sources "
                                        f"(sha {kernel_sources_sha()})" if tr else
                                        "none: no ncu capture of this build's kernel on record"),
                     "traffic_gbs": (round(tr * nodes / (avg_lb * 1e-3) / 1e9, 1) if tr else None),
                     "share_of_step": round(lb_ms / timing["window_ms"][0], 4),
                     "launch_shape": shape32, "pair_shape": pair32,
                     "note": "achieved = 144 B x node-steps per launch / launch time (a two-step launch moves "
                             "the populations through HBM once for two steps); per-kernel times from an "
                             "instrumented second window of the same K steps"},
        "fp64": {"value": round(mlups64, 1), "unit": "MLUPS", "steps": K64,
                 "lb_achieved_gbs": round(achieved64, 1),
                 "lb_frac": round(achieved64 / peak, 4),
                 "fp32_over_fp64": round(mlups / mlups64, 3),
                 "launch_shape": shape64, "pair_shape": pair64},
        "accuracy_end_of_timed_run": {"nu_fp32": nu32, "nu_fp64": nu64,
                     "nu_rel_err": abs(nu32 - nu64) / abs(nu64),
                     "ke_rel_err": abs(ke32 - ke64) / max(abs(ke64), 1e-300),
                     "note": f"after {2 * K + W} steps from the same initial state"},
        "kernels_ms": {k: round(v[0], 3) for k, v in timing.items()},
        "kernel_launches": {k: v[1] for k, v in timing.items() if k != "window_ms"},
        "gpu_launches": int(lb_n + pt_n),
        "clocks": clocks,
        "records": len(recs),
    })
    out.update(sec)
    if e2e_ms is not None:
        out["e2e"] = {"value": round(world * nodes * K / (e2e_ms * 1e3), 1), "unit": "MLUPS",
                      "h2d_bytes_per_step": int(e2e_h2d / K), "d2h_bytes_per_step": int(e2e_d2h / K),
                      "ms": round(e2e_ms, 2),
                      # the copies alone at this box's pinned rates, plus the device-timed steps
                      "pinned_h2d_gbs": round(h2d_gbs, 1), "pinned_d2h_gbs": round(d2h_gbs, 1),
                      "copy_bound_ms": round(e2e_h2d / h2d_gbs / 1e6 + e2e_d2h / d2h_gbs / 1e6 + ms, 2),
                      "path": "lbrb_set_populations(REF_AOS_HALO fp64) + set_moments + particles_set + "
                              "lbrb_step in chunks of 500 steps, each chunk's records drained (lbrb_record_drain) "
                              "while the next runs + get_moments"}
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args)
    return out


# ------------------------------------------------------------- adjoint
ADJ_NX, ADJ_NY, ADJ_STEPS, ADJ_K, ADJ_EVERY, ADJ_NOBS = 1024, 512, 2000, 100, 10, 4096


def adjoint_problem(lb, device: int, seed: int = 31):
    """Assimilation window of the adjoint configuration: 1024x512, Ra=1e6,
    Pr=1, U=0.1; observations = T along 4096 tracer trajectories of a seeded
    truth run, every 10 steps over 2000 steps; the window starts from an
    initial state with other noise."""
    base = lb.closure(ADJ_NX, ADJ_NY, Ra=1e6, Pr=1.0, U=0.1)
    nrec = ADJ_STEPS // ADJ_EVERY
    with lb.Run(**base, precision="fp64", nprtcl=ADJ_NOBS, noutconfig=ADJ_EVERY, record_slots=nrec + 1,
                device=device) as r:
        r.init_conduction(seed, 1e-2)
        m = r.get_moments()
        rng = np.random.default_rng(seed)
        x = rng.uniform(0.5, ADJ_NX - 0.5, ADJ_NOBS)
        y = rng.uniform(1.0, ADJ_NY, ADJ_NOBS)
        r.set_particles(np.arange(ADJ_NOBS, dtype=np.int32), x, y, bilinear_np(m["u"], x, y),
                        bilinear_np(m["v"], x, y), np.zeros(ADJ_NOBS, np.int32), np.zeros(ADJ_NOBS))
        r.step(ADJ_STEPS)
        recs = r.drain_records()
    steps = np.array(sorted(recs), np.int32)
    ox = np.stack([recs[s]["x"] for s in steps])
    oy = np.stack([recs[s]["y"] for s in steps])
    oT = np.stack([recs[s]["temp"] for s in steps])
    rng = np.random.default_rng(seed + 1)
    j = np.arange(ADJ_NY)
    T0 = (base["Tdown"] + (base["Tup"] - base["Tdown"]) * ((j + 0.5) / ADJ_NY))[:, None] \
        + 1e-2 * rng.uniform(-1, 1, (ADJ_NY, ADJ_NX))
    return base, steps, ox, oy, oT, T0


def sync_ranks(torch, dist):
    """all ranks at the same point with their GPU work done"""
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()


def run_adjoint_bench(lb, torch, device: int, nsteps: int = ADJ_STEPS, K: int = ADJ_K,
                      variant: int = -1, dist=None, rank: int = 0, world: int = 1) -> dict:
    """The adjoint window's cost (every rank times the same window: replicas,
    the slowest rank's times) and the FD check (directions split over the
    ranks)."""
    base, steps, ox, oy, oT, T0 = adjoint_problem(lb, device)
    keep = steps <= nsteps
    steps, ox, oy, oT = steps[keep], ox[keep], oy[keep], oT[keep]
    with lb.Run(**base, precision="fp32", device=device) as w:
        w.adjoint_set_obs(steps, ox, oy, oT)
        if variant >= 0:
            w.adjoint_set_variant(variant)
        stream = torch.cuda.Stream()
        w.set_stream(stream.cuda_stream)
        # warm-up at the window's own size: the state store (the default when
        # it fits) or checkpoint and segment buffers, launch-shape and
        # pair-kernel autotuning happen here, untimed
        w.adjoint_window(T0, nsteps, K, gradient=True)
        pair_variant = w.adjoint_variant()
        store = w.adjoint_store()
        sync_ranks(torch, dist)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(8)]
        ev[0].record(stream)
        w.adjoint_window(T0, nsteps, K, gradient=False)
        ev[1].record(stream)
        ev[2].record(stream)
        J, grad = w.adjoint_window(T0, nsteps, K, gradient=True)
        ev[3].record(stream)
        # the same gradient window with checkpoints every K steps and the
        # segments recomputed (the form for windows whose store does not
        # fit), after its own untimed warm-up
        w.adjoint_set_store(0)
        w.adjoint_window(T0, nsteps, K, gradient=True)
        ev[6].record(stream)
        Jr, gradr = w.adjoint_window(T0, nsteps, K, gradient=True)
        ev[7].record(stream)
        # plain forward steps of the same grid, for the cost ratio
        w.init_conduction(1, 1e-3)
        w.step(10)
        ev[4].record(stream)
        w.step(nsteps)
        ev[5].record(stream)
        torch.cuda.synchronize()
        t_fwd_window = max_over_ranks(torch, dist, ev[0].elapsed_time(ev[1]))
        t_adj = max_over_ranks(torch, dist, ev[2].elapsed_time(ev[3]))
        t_rec = max_over_ranks(torch, dist, ev[6].elapsed_time(ev[7]))
        t_step = max_over_ranks(torch, dist, ev[4].elapsed_time(ev[5]) / nsteps)
        w.set_stream(None)
    fd = adjoint_fd_check(lb, base, steps, ox, oy, oT, T0, nsteps, device, ndir=8, dist=dist, rank=rank,
                          world=world)
    return {"grid": f"{ADJ_NX}x{ADJ_NY}", "window_steps": nsteps, "checkpoint_every": K,
            "ranks": world,
            "observations": f"{ADJ_NOBS} tracers every {ADJ_EVERY} steps (seeded truth run)",
            "fd_check": fd, "pair_kernel_variant": pair_variant,
            "precision": "fp32 forward, fp64 adjoint", "J": J,
            "grad_norm": float(np.linalg.norm(grad)),
            # all ranks' adjoint steps over the slowest rank's window
            "adjoint_steps_per_s": round(world * nsteps / (t_adj * 1e-3), 1),
            "ms_gradient_window": round(t_adj, 2), "ms_misfit_window": round(t_fwd_window, 2),
            "ms_forward_step": round(t_step, 5),
            # gradient (forward + recompute + backward) per window step, in plain forward steps
            "cost_vs_forward_steps": round(t_adj / (nsteps * t_step), 2),
            # the backward sweep alone (recompute + adjoint) per step, in plain forward steps
            "backward_sweep_vs_forward_steps": round((t_adj - t_fwd_window) / (nsteps * t_step), 2),
            # gradient over function: the gradient window against the misfit window
            "gradient_over_misfit": round(t_adj / t_fwd_window, 2),
            "states": ("store of every state's F and moments, " f"{store['bytes'] / 1e9:.1f} GB"
                       if store["used_last"] else f"checkpoints every {K} steps, segments recomputed"),
            "checkpoint_recompute": {"ms_gradient_window": round(t_rec, 2),
                                     "cost_vs_forward_steps": round(t_rec / (nsteps * t_step), 2),
                                     "same_gradient": bool(J == Jr and np.array_equal(grad, gradr))}}


def adjoint_fd_check(lb, base, steps, ox, oy, oT, T0, nsteps, device, ndir, h=1e-6, seed=2024,
                     dist=None, rank: int = 0, world: int = 1) -> dict:
    """<gradient, d> of the FP64 adjoint against central differences (h) of the
    FP64 forward on ndir seeded directions, split over the ranks (each rank
    its own gradient and its directions; the errors gathered once);
    FP32-forward gradient against it"""
    from lagrangianrbnudging_b200 import shard

    mine = set(shard.my_units([1.0] * ndir, rank, world))
    errs = {}
    with lb.Run(**base, precision="fp64", device=device) as w:
        w.adjoint_set_obs(steps, ox, oy, oT)
        J, g64 = w.adjoint_window(T0, nsteps, ADJ_K)
        rng = np.random.default_rng(seed)
        for k in range(ndir):
            d = rng.standard_normal(T0.shape)  # every rank draws every direction, in order
            if k not in mine:
                continue
            Jp = w.adjoint_window(T0 + h * d, nsteps, ADJ_K, gradient=False)
            Jm = w.adjoint_window(T0 - h * d, nsteps, ADJ_K, gradient=False)
            fd = (Jp - Jm) / (2 * h)
            ad = float(np.sum(g64 * d))
            errs[k] = abs(fd - ad) / abs(ad)
    for part in shard.gather(dist, errs):
        errs.update(part)
    errs = [errs[k] for k in range(ndir)]
    with lb.Run(**base, precision="fp32", device=device) as w:
        w.adjoint_set_obs(steps, ox, oy, oT)
        J32, g32 = w.adjoint_window(T0, nsteps, ADJ_K)
    return {"directions": ndir, "h": h, "fd_rel_err_max": float(max(errs)),
            "fd_rel_err_median": float(np.median(errs)), "tolerance": 1e-4,
            "J_fp64": J, "J_fp32": J32,
            "fp32_grad_rel_l2_vs_fp64": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))}


def run_adjoint_check(lb, torch, device: int, ndir: int = 64, h: float = 1e-6) -> dict:
    """the adjoint configuration's full check: 64 seeded directions"""
    base, steps, ox, oy, oT, T0 = adjoint_problem(lb, device)
    return {"mode": "adjoint-check", "grid": f"{ADJ_NX}x{ADJ_NY}", "window_steps": ADJ_STEPS,
            **adjoint_fd_check(lb, base, steps, ox, oy, oT, T0, ADJ_STEPS, device, ndir, h)}


# ------------------------------------------------------------- accuracy
ACC_STEPS, ACC_EVERY = 8000, 100


def run_accuracy(lb, device: int, steps: int = ACC_STEPS, every: int = ACC_EVERY) -> dict:
    """FP32-shifted against FP64 (reference operation order) on the headline
    grid from the same seeded state: time-averaged Nu and <u^2> over the
    run (sampled every `every` steps) and the T-field error at its end."""
    base = lb.closure(NX, NY, Ra=RA, Pr=PR, U=U)
    res = {}
    for prec in ("fp32", "fp64"):
        with lb.Run(**base, precision=prec, device=device) as r:
            r.init_conduction(SEED, 1e-3)
            nus, kes = [], []
            for _ in range(steps // every):
                r.step(every)
                nus.append(r.nusselt())
                kes.append(r.energy()[0])
            res[prec] = (np.array(nus), np.array(kes), r.get_moments()["T"])
    n32, k32, T32 = res["fp32"]
    n64, k64, T64 = res["fp64"]
    dT = T32 - T64
    return {"grid": f"{NX}x{NY}", "steps": steps, "sampled_every": every,
            "nu_avg_fp32": float(n32.mean()), "nu_avg_fp64": float(n64.mean()),
            "nu_avg_rel_err": float(abs(n32.mean() - n64.mean()) / abs(n64.mean())),
            "nu_final_rel_err": float(abs(n32[-1] - n64[-1]) / abs(n64[-1])),
            "u2_avg_rel_err": float(abs(k32.mean() - k64.mean()) / abs(k64.mean())),
            "T_max_abs_err": float(np.abs(dT).max()), "T_l2_err": float(np.sqrt(np.mean(dT ** 2))),
            "bar": "time-averaged Nu within 0.5% of FP64"}


def batch_mean_se(x: np.ndarray, nbatch: int = 10) -> tuple[float, float]:
    """mean and its standard error from `nbatch` batch means (the samples of
    a turbulent time series are correlated; batches longer than the
    correlation time are not)"""
    n = len(x) // nbatch * nbatch
    b = x[len(x) - n:].reshape(nbatch, -1).mean(axis=1)
    return float(x.mean()), float(b.std(ddof=1) / np.sqrt(nbatch))


def run_stationary_nu(lb, device: int, tff: float = 6.0, discard: float = 3.0, every: int = 200) -> dict:
    """FP32-shifted against FP64 on the production grid (4096x2048, Ra=1e8,
    U=0.05) from the same seeded state over `tff` free-fall times Ny/U
    (40,960 steps each), the first `discard` dropped as the onset transient:
    time-averaged volume Nusselt number, row-profile Nusselt number (the
    per-row ingredients of the reference's profile(): (<vT> - kappa dT/dy) /
    (kappa dT / H) averaged over rows 0..ny-2), <u^2> and their standard
    errors, sampled every `every` steps, and the volume Nu once per
    free-fall time."""
    base = lb.closure(NX, NY, Ra=RA, Pr=PR, U=U)
    t_ff = int(NY / U)
    total, skip = int(tff * t_ff) // every * every, int(discard * t_ff) // every
    out = {"mode": "nu-stationary", "grid": f"{NX}x{NY}", "Ra": RA, "free_fall_steps": t_ff,
           "steps": total, "discarded_steps": skip * every, "sampled_every": every}
    series = {}
    for prec in ("fp32", "fp64"):
        with lb.Run(**base, precision=prec, device=device) as r:
            r.init_conduction(SEED, 1e-3)
            nu, nup, u2 = [], [], []
            t0 = time.perf_counter()
            for _ in range(total // every):
                r.step(every)
                nu.append(r.nusselt())
                # (rows 0..ny-2: the top row's dT/dy wraps to the bottom row, and over all
                # rows the conduction terms telescope to zero)
                nup.append(float(np.mean(r.profile()[:-1, 8])))
                u2.append(2.0 * r.energy()[0])
            wall = time.perf_counter() - t0
        series[prec] = {k: np.array(v)[skip:] for k, v in (("nu", nu), ("nu_profile", nup), ("u2", u2))}
        out[prec] = {"wall_s": round(wall, 1), "nu_series_every_ff": [round(nu[i], 4) for i in
                                                                         range(0, len(nu), t_ff // every)]}
        for k, a in series[prec].items():
            m, se = batch_mean_se(a)
            out[prec][k] = {"mean": m, "se": se}
    for k in ("nu", "nu_profile", "u2"):
        a, b = out["fp32"][k], out["fp64"][k]
        out[f"{k}_rel_diff"] = abs(a["mean"] - b["mean"]) / abs(b["mean"])
        out[f"{k}_rel_se_of_diff"] = float(np.hypot(a["se"], b["se"]) / abs(b["mean"]))
    out["bar"] = "time-averaged Nu of FP32 within 0.5% of FP64"
    return out


# ------------------------------------------------------------- nudging twin
NUD_NX, NUD_NY, NUD_RA, NUD_TRACERS, NUD_STEPS, NUD_CHUNK = 2048, 1024, 1e7, 1 << 14, 50000, 250
NUD_ALPHAS = (0.01, 0.1, 1.0)


def run_nudging_bench(lb, torch, device: int, steps: int = NUD_STEPS, chunk: int = NUD_CHUNK,
                      dist=None, rank: int = 0, world: int = 1) -> dict:
    """Twin experiment: run A (seed A, 2^14 tracers) records T along the
    trajectories every step; runs from seed B relax T toward those records at
    the recorded positions (bilinear, alpha in {0.01, 0.1, 1} per step), beside
    a free run (alpha = 0) from seed B.  All FP32-shifted populations, FP64
    positions; the L2 error of T against run A is sampled along the way.
    With several ranks the four runs from seed B are split over them; each
    rank with runs computes run A itself (deterministic), and the results are
    gathered once."""
    from lagrangianrbnudging_b200 import shard

    alphas_all = (0.0,) + NUD_ALPHAS
    mine = [alphas_all[i] for i in shard.my_units([1.0] * len(alphas_all), rank, world)]
    base = lb.closure(NUD_NX, NUD_NY, Ra=NUD_RA, Pr=1.0, U=0.1)
    seed_a, seed_b = 1001, 2002
    n = NUD_TRACERS
    nodes = NUD_NX * NUD_NY
    part = {"ms_truth": None, "runs": {}}
    if mine:
        rng = np.random.default_rng(seed_a)
        x = rng.uniform(0.5, NUD_NX + 0.5, n)
        y = rng.uniform(1.0, NUD_NY, n)
        truth = lb.Run(**base, precision="fp32", nprtcl=n, noutconfig=1, record_slots=chunk + 1,
                       device=device)
        truth.init_conduction(seed_a, 1e-3)
        m = truth.get_moments()
        truth.set_particles(np.arange(n, dtype=np.int32), x, y, bilinear_np(m["u"], x, y),
                            bilinear_np(m["v"], x, y), np.zeros(n, np.int32), np.zeros(n))
        runs = {}
        for a in mine:
            kw = dict(base, precision="fp32", device=device)
            if a > 0:
                kw.update(nudge="bilinear", alpha=a, nobs=n)
            r = lb.Run(**kw)
            r.init_conduction(seed_b, 1e-3)
            runs[a] = r
        stream = torch.cuda.Stream()
        ms = {a: 0.0 for a in runs}
        ms_truth = 0.0
        samples = {a: [] for a in runs}
        sample_every = max(steps // 20, chunk)

        def l2(ra, rb):
            ta = ra.get_moments()["T"]
            tb = rb.get_moments()["T"]
            return float(np.sqrt(np.mean((tb - ta) ** 2)))

        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for r in [truth, *runs.values()]:
            r.set_stream(stream.cuda_stream)
        done = 0
        while done < steps:
            c = min(chunk, steps - done)
            e0.record(stream)
            truth.step(c)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_truth += e0.elapsed_time(e1)
            st, buf = truth.drain_records_array()
            ox, oy, oT = buf[:, 0, :], buf[:, 1, :], buf[:, 8, :]
            for a, r in runs.items():
                if a > 0:
                    r.nudge_obs(int(st[0]), ox, oy, oT)
                e0.record(stream)
                r.step(c)
                e1.record(stream)
                torch.cuda.synchronize()
                ms[a] += e0.elapsed_time(e1)
            done += c
            if done % sample_every == 0 or done == steps:
                for a, r in runs.items():
                    samples[a].append((done, float(f"{l2(truth, r):.4g}")))
        for r in [truth, *runs.values()]:
            r.set_stream(None)
            r.close()
        part = {"ms_truth": ms_truth, "runs": {a: (samples[a], ms[a]) for a in runs}}
    parts = shard.gather(dist, part)
    ms_truth = next(p["ms_truth"] for p in parts if p["ms_truth"] is not None)
    samples, ms = {}, {}
    for p in parts:
        for a, (sm, m_) in p["runs"].items():
            samples[a], ms[a] = sm, m_
    out = {"grid": f"{NUD_NX}x{NUD_NY}", "Ra": NUD_RA, "tracers": n, "steps": steps,
           "obs": "run A's records (x, y, T) every step, fed in chunks of %d steps" % chunk,
           "truth_mlups_with_records": round(nodes * steps / (ms_truth * 1e3), 1),
           "free_run": {"l2_final": samples[0.0][-1][1], "l2": samples[0.0]},
           "nudged": {str(a): {"l2_final": samples[a][-1][1], "l2": samples[a],
                               "mlups": round(nodes * steps / (ms[a] * 1e3), 1)} for a in NUD_ALPHAS},
           "metric": "L2 T-field error vs run A, sqrt(mean((T_B - T_A)^2))"}
    if world > 1:
        out["ranks"] = world
        out["split"] = "the four runs from seed B over the ranks (longest processing time first)"
    return out


# ------------------------------------------------------------- ensemble
ENS_N, ENS_STEPS, ENS_TRACERS, ENS_OBS_ROWS = 64, 10000, 1024, 100


def ensemble_members(lb, device: int, seed: int = 41, keep=None, precision: str = "fp32"):
    """The uneven ensemble: 64 members with Nx x Ny drawn from {256x128,
    512x256, 1024x512} and Ra log-uniform in [1e5, 1e7] (Pr=1, U=0.1), each
    with 1024 tracers and a nudging alpha drawn from {0, 0.1}; FP32-shifted
    populations.  Nudged members relax T toward synthetic observations at
    1024 seeded positions (a repeating series of 100 rows; T = conduction
    profile + 0.01 seeded noise).  Every member's draws are taken in order;
    only the members in `keep` (all when None) are built.  Returns the built
    members and the description of all 64."""
    rng = np.random.default_rng(seed)
    sizes = [(256, 128), (512, 256), (1024, 512)]
    members, desc = [], []
    for i in range(ENS_N):
        nx, ny = sizes[int(rng.integers(3))]
        Ra = float(10 ** rng.uniform(5, 7))
        alpha = [0.0, 0.1][int(rng.integers(2))]
        x = rng.uniform(0.5, nx + 0.5, ENS_TRACERS)
        y = rng.uniform(1.0, ny, ENS_TRACERS)
        if alpha:
            ox = rng.uniform(0.5, nx + 0.5, (ENS_OBS_ROWS, ENS_TRACERS))
            oy = rng.uniform(1.0, ny, (ENS_OBS_ROWS, ENS_TRACERS))
            oT = 0.5 - (oy - 0.5) / ny + 0.01 * rng.standard_normal(oy.shape)
        desc.append((nx, ny, Ra, alpha))
        if keep is not None and i not in keep:
            continue
        kw = dict(**lb.closure(nx, ny, Ra=Ra, Pr=1.0, U=0.1), precision=precision, nprtcl=ENS_TRACERS,
                  device=device)
        if alpha:
            kw.update(nudge="bilinear", alpha=alpha, nobs=ENS_TRACERS, obs_cycle=1)
        r = lb.Run(**kw)
        r.init_conduction(seed * 1000 + i, 1e-3)
        z = np.zeros(ENS_TRACERS)
        r.set_particles(np.arange(ENS_TRACERS, dtype=np.int32), x, y, z, z,
                        np.zeros(ENS_TRACERS, np.int32), z)
        if alpha:
            r.nudge_obs(1, ox, oy, oT)
        members.append(r)
    return members, desc


def ensemble_member_checks(lb, device: int, desc, checks: dict, steps: int, every: int = 500) -> dict:
    """Every member: mass conserved, T inside the walls' range (plus the
    nudging targets' spread); the member of lowest Nu stepped again alone,
    in FP32 (bit-identical to the ensemble: the same Nu) and in FP64 (the
    reference-order arithmetic), with its Nu every `every` steps."""
    worst = min(checks, key=lambda i: checks[i]["nu"])
    nx, ny, Ra, alpha = desc[worst]
    alone = {}
    for prec in ("fp32", "fp64"):
        (r,), _ = ensemble_members(lb, device, keep={worst}, precision=prec)
        series, done = [], 0
        while done < steps:
            n = min(every, steps - done)
            r.step(n)
            done += n
            series.append(round(r.nusselt(), 4))
        alone[prec] = {"nu": r.nusselt(), "nu_every_%d" % every: series}
        r.close()
    return {"max_mass_err": max(c["mass_err"] for c in checks.values()),
            "T_range": [min(c["T_min"] for c in checks.values()), max(c["T_max"] for c in checks.values())],
            "lowest_nu_member": {"index": worst, "grid": f"{nx}x{ny}", "Ra": Ra, "alpha": alpha,
                                 "nu_in_ensemble": checks[worst]["nu"], "alone": alone,
                                 "fp32_alone_equals_ensemble": alone["fp32"]["nu"] == checks[worst]["nu"]}}


def ensemble_desc(seed: int = 41):
    """the 64 members' (nx, ny, Ra, alpha) without building any"""
    return ensemble_members(None, 0, seed, keep=())[1]


def run_ensemble_bench(lb, torch, device: int, steps: int = ENS_STEPS, variant: int = -1, dist=None,
                       rank: int = 0, world: int = 1) -> dict:
    """The 64-member ensemble under its CUDA graph.  With several ranks the
    members are split over them by node count (longest processing time
    first), each rank runs its share as one ensemble, and the aggregate is
    all nodes x steps over the slowest rank's time."""
    from lagrangianrbnudging_b200 import shard

    desc = ensemble_desc()
    costs = [nx * ny for nx, ny, _, _ in desc]
    keep = shard.my_units(costs, rank, world)
    members, _ = ensemble_members(lb, device, keep=set(keep))
    nodes = sum(costs)
    my_nodes = sum(costs[i] for i in keep)
    ms_mine, sched, t, pairs = 0.0, None, None, None
    ens = lb.Ensemble(members) if members else None
    if ens is not None:
        if variant >= 0:
            ens.set_schedule(variant)
        stream = torch.cuda.Stream()
        ens.set_stream(stream.cuda_stream)
        ens.step(12)  # autotune + graph capture + warm-up
        ens.step(25)  # (a pair graph of 12 steps needs 25-step calls)
        ens.sync()
        sched = ens.schedule()
        pairs = ens.pairs()
        # per-launch timing of the phases (direct launches, no graph)
        ens.set_timing(True)
        ens.step(60)
        t = ens.get_timing()
        ens.set_timing(False)
    sync_ranks(torch, dist)
    if ens is not None:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_mine = e0.elapsed_time(e1)
        ens.sync()
        ens.set_stream(None)
        ens.close()
    ms = max_over_ranks(torch, dist, ms_mine)

    def is_finite(r):
        try:
            r.check_finite()
            return True
        except lb.LbrbError:
            return False

    def sanity(r):
        """mass (mean rho - 1), T range and Nu of a member"""
        m = r.get_moments()
        return {"mass_err": float(abs(m["rho"].mean() - 1.0)), "T_min": float(m["T"].min()),
                "T_max": float(m["T"].max()), "nu": r.nusselt()}

    mine = {"members": len(keep), "nodes": my_nodes, "ms": ms_mine, "schedule": sched, "timing": t, "pairs": pairs,
            "finite": all(is_finite(r) for r in members), "ids": list(keep),
            "checks": [sanity(r) for r in members]}
    for r in members:
        r.close()
    parts = shard.gather(dist, mine)
    finite = all(p["finite"] for p in parts)
    checks = {i: c for p in parts for i, c in zip(p["ids"], p["checks"])}
    nus = [c["nu"] for c in checks.values()]
    t = parts[0]["timing"]
    sched = parts[0]["schedule"]
    peak, _ = measured_peak()
    lb_ms = t["lb_step"][0] / max(t["lb_step"][1], 1)
    agg = nodes * ALG_BYTES["fp32"] * steps / (ms * 1e-3) / 1e9
    # the fused phase over the 60-step timing window (a launch takes one or two steps)
    lb_gbs = parts[0]["nodes"] * ALG_BYTES["fp32"] * 60 / (t["lb_step"][0] * 1e-3) / 1e9
    nudged = sum(1 for d in desc if d[3] > 0)
    out = {"members": ENS_N, "nodes": nodes, "steps": steps, "ms": round(ms, 2),
           "mlups": round(nodes * steps / (ms * 1e3), 1),
           "aggregate_gbs": round(agg, 1), "aggregate_frac": round(agg / (peak * world), 4),
           "lb_phase_ms": round(lb_ms, 5), "lb_phase_gbs": round(lb_gbs, 1),
           "lb_phase_frac": round(lb_gbs / peak, 4),
           "phase_share": {k: round(v[0] / sum(x[0] for x in t.values()), 4) for k, v in t.items()},
           "launches_per_step": round(sum(v[1] for v in t.values()) / 60, 3), "schedule": sched,
           "pairs": parts[0].get("pairs"), "finite": bool(finite),
           "nu_range": [round(min(nus), 3), round(max(nus), 3)],
           # (every member took 12 + 25 + 60 steps of tuning, capture and timing before the timed steps)
           "member_checks": ensemble_member_checks(lb, device, desc, checks, 97 + steps) if rank == 0 else None,
           "config": f"{ENS_N} members from {{256x128, 512x256, 1024x512}}, Ra log-uniform "
                     f"[1e5,1e7], Pr=1, U=0.1, {ENS_TRACERS} tracers each, alpha in {{0,0.1}} "
                     f"({nudged} nudged), fp32-shifted; {steps} steps in CUDA-graph replays",
           "alg_bytes": "sum of nodes x 144 B per step"}
    if world > 1:
        out["ranks"] = [{"members": p["members"], "nodes": p["nodes"], "ms": round(p["ms"], 2)}
                        for p in parts]
        out["split"] = "members over the ranks by node count (longest processing time first)"
        out["lb_phase"] = "rank 0's share"
    return out


# ------------------------------------------------------------- y-slabs
SLAB_STEPS = 200


def run_slab_bench(lb, torch, device: int, steps: int = SLAB_STEPS, devices=None) -> dict:
    """The headline grid (FP32-shifted, no particles) as one handle and as a
    domain of 2 and 4 y-slabs (lbrb_slab_step: per step a pack kernel and
    peer copies of the crossing populations, then the fused kernel per slab).
    With one GPU the slabs share it (all on one stream), which measures the
    exchange's cost; the end states must equal the single handle's bit for
    bit (T and u compared)."""
    base = dict(**lb.closure(NX, NY, Ra=RA, Pr=PR, U=U), precision="fp32")
    stream = torch.cuda.Stream()

    def timed(obj, set_stream):
        set_stream(stream.cuda_stream)
        obj.init_conduction(SEED, 1e-3)
        obj.step(20)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        obj.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        m = obj.get_moments()
        return e0.elapsed_time(e1), m

    nodes = NX * NY
    with lb.Run(**base, device=device) as whole:
        ms1, m1 = timed(whole, whole.set_stream)
    out = {"grid": f"{NX}x{NY}", "steps": steps, "single_handle_mlups": round(nodes * steps / (ms1 * 1e3), 1)}
    for n in (2, 4):
        with lb.SlabDomain([NY // n] * n, devices=devices, **base, device=device) as dom:
            ms, m = timed(dom, lambda st: [r.set_stream(st) for r in dom.slabs])
            exact = all(np.array_equal(m[k], m1[k]) for k in ("T", "u"))
            for r in dom.slabs:
                r.set_stream(None)
        out[f"slabs_{n}"] = {"mlups": round(nodes * steps / (ms * 1e3), 1),
                             "vs_single_handle": round(ms1 / ms, 4), "bit_exact_T_u": bool(exact)}
    # the production workload with its 2^17 particles and records: one handle
    # against 2 slabs (owner slab advances, the others copy in)
    pk = dict(base, nprtcl=NPRTCL, noutconfig=NOUTCONFIG, record_slots=steps // NOUTCONFIG + 4)

    def timed_p(obj, set_stream):
        set_stream(stream.cuda_stream)
        init_run(obj, SEED)
        obj.step(20)
        obj.drain_records_array()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        obj.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), obj.get_particles(), obj.drain_records_array()

    with lb.Run(**pk, device=device) as whole:
        ms1, p1, r1 = timed_p(whole, whole.set_stream)
    # each slab holds the particles in its rows (owner arrays, hand-off lists
    # between neighbours each step)
    for n in (2, 4):
        with lb.SlabDomain([NY // n] * n, devices=devices, **pk, device=device) as dom:
            ms, p2, r2 = timed_p(dom, lambda st: [r.set_stream(st) for r in dom.slabs])
            counts = dom.slab_counts()
            for r in dom.slabs:
                r.set_stream(None)
        exact = all(np.array_equal(p1[k], p2[k]) for k in p1) and all(np.array_equal(a, b) for a, b in zip(r1, r2))
        out[f"particles_{n}_slabs"] = {"nprtcl": NPRTCL, "records_every": NOUTCONFIG,
                                       "single_handle_mlups": round(nodes * steps / (ms1 * 1e3), 1),
                                       "mlups": round(nodes * steps / (ms * 1e3), 1),
                                       "vs_single_handle": round(ms1 / ms, 4), "particles_per_slab": counts,
                                       "bit_exact_particles_records": bool(exact)}
    # the one-process-per-GPU protocol (lagrangianrbnudging_b200.slabrank),
    # its ranks' sends done as copies on one GPU: per step a ghost exchange
    # (with the last step's hand-off lists), the step, a moment exchange and
    # the particle step, one step per launch
    from lagrangianrbnudging_b200 import slabrank
    with lb.SlabDomain([NY // 2] * 2, devices=devices, **pk, device=device) as dom:
        st = slabrank.bind_stream(dom.slabs, torch, stream)
        init_run(dom, SEED)
        ranks = [slabrank.SlabRank(r, slabrank.device_buffers(r, torch), particles=True, pairs=True)
                 for r in dom.slabs]
        with torch.cuda.stream(st):
            slabrank.run_local(ranks, 20)
        dom.drain_records_array()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(st):
            e0.record(st)
            slabrank.run_local(ranks, steps)
            e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        p2, r2 = dom.get_particles(), dom.drain_records_array()
        for r in dom.slabs:
            r.set_stream(None)
    exact = all(np.array_equal(p1[k], p2[k]) for k in p1) and all(np.array_equal(a, b) for a, b in zip(r1, r2))
    out["rank_protocol_2_slabs"] = {"nprtcl": NPRTCL, "mlups": round(nodes * steps / (ms * 1e3), 1),
                                    "vs_single_handle": round(ms1 / ms, 4),
                                    "bit_exact_particles_records": bool(exact),
                                    "note": "two steps per launch, the particle exchange of each step in turn; "
                                            "across GPUs the copies are NCCL send/recv"}
    out["note"] = ("slabs on one GPU and one stream: the figure is the exchange's overhead; "
                   "across GPUs each slab runs on its own device")
    return out


# ---------------------------------------------------------- reference arm
def ref_params() -> dict:
    nu = U * NY * np.sqrt(PR / RA)
    kappa = U * NY / np.sqrt(RA * PR)
    return dict(nx=NX, ny=NY, scratch=1, nstart=0, nsteps=1000000, nout=1000000,
                noutconfig=NOUTCONFIG, relax=3.0 * nu + 0.5, relaxg=3.0 * kappa + 0.5,
                Tup=-0.5, Tdown=0.5, gravity=-(U * U) / NY, Particle=1, Particle_scratch=0,
                Nprtcl=NPRTCL, tracer=0, heavyprtcl=1, taulag=0.5 * NY / U, beta=0.0,
                Prtcl_Writefull=0)


def build_reference_baseline():
    """Build the reference's own temppart_dump for the production-trajectory
    workload and for the 512x256 case (needs the reference checkout; the
    binaries travel in oracle/_ref)."""
    from oracle import build as ob

    ob.build_ref("temppart_dump", c0_ref_params(), C0_REF_TAG)
    return ob.build_ref("temppart_dump", ref_params(), REF_TAG)


# ------------------------------------------------------ 512x256 tracer case
C0_NX, C0_NY, C0_RA, C0_U, C0_TRACERS, C0_EVERY, C0_STEPS = 512, 256, 1e6, 0.1, 4096, 10, 20000
C0_REF_TAG = "bench_c0"


def c0_ref_params() -> dict:
    nu = C0_U * C0_NY * np.sqrt(1.0 / C0_RA)
    return dict(nx=C0_NX, ny=C0_NY, scratch=1, nstart=0, nsteps=1000000, nout=1000000,
                noutconfig=C0_EVERY, relax=3.0 * nu + 0.5, relaxg=3.0 * nu + 0.5, Tup=-0.5, Tdown=0.5,
                gravity=-(C0_U * C0_U) / C0_NY, Particle=1, Particle_scratch=0, Nprtcl=C0_TRACERS,
                tracer=1, heavyprtcl=0, taulag=1.0, beta=0.0, Prtcl_Writefull=0)


def run_config0(lb, torch, device: int, steps: int = C0_STEPS) -> dict:
    """The reference's CPU-runnable case: 512x256, Ra=1e6, U=0.1, 4096 seeded
    uniform tracers, records (x, y, u, v, T, ...) every 10 steps, drained to
    the host every 1000 steps.  GPU FP32-shifted and FP64, and the
    reference's own build on the host cores at several rank counts."""
    base = lb.closure(C0_NX, C0_NY, Ra=C0_RA, Pr=1.0, U=C0_U)
    rng = np.random.default_rng(SEED + 5)
    n = C0_TRACERS
    x = rng.uniform(0.5, C0_NX + 0.5, n)
    y = rng.uniform(1.0, C0_NY, n)
    ids = np.arange(n, dtype=np.int32)
    out = {"grid": f"{C0_NX}x{C0_NY}", "tracers": n, "records_every": C0_EVERY, "steps": steps}
    chunk = 1000
    for prec in ("fp32", "fp64"):
        with lb.Run(**base, precision=prec, nprtcl=n, noutconfig=C0_EVERY, record_slots=chunk // C0_EVERY + 2,
                    device=device) as r:
            r.init_conduction(SEED, 1e-3)
            m = r.get_moments()
            r.set_particles(ids, x, y, bilinear_np(m["u"], x, y), bilinear_np(m["v"], x, y),
                            np.zeros(n, np.int32), np.zeros(n))
            r.step(chunk)
            r.sync()
            r.drain_records_array()
            stream = torch.cuda.Stream()
            r.set_stream(stream.cuda_stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            dev_ms = 0.0
            nrec = 0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(steps // chunk):
                e0.record(stream)
                r.step(chunk)
                e1.record(stream)
                r.sync()
                dev_ms += e0.elapsed_time(e1)
                nrec += len(r.drain_records_array()[0])
            wall = time.perf_counter() - t0
            r.set_stream(None)
        out[prec] = {"mlups_device": round(C0_NX * C0_NY * steps / (dev_ms * 1e3), 1),
                     "mlups_with_record_drains": round(C0_NX * C0_NY * steps / (wall * 1e6), 1),
                     "records": nrec}
    cpu = {}
    exe = ROOT / "oracle" / "_ref" / C0_REF_TAG / "temppart_dump"
    cores = host_cores()
    np_list = [p for p in (1, 2, 4, 8, 16, 32, 64) if p <= cores]
    for p in np_list:
        try:
            res = run_reference(steps=200, warmup=5, ranks=p, time_cap=8.0, exe=exe, particles=(ids, x, y))
            cpu[str(p)] = round(C0_NX * C0_NY / res["per_step_s"] / 1e6, 3)
        except Exception as e:  # reported, never fatal
            cpu[str(p)] = f"unavailable: {e}"
    out["reference_cpu_mlups_by_ranks"] = cpu
    out["reference_note"] = ("the reference's own temppart_dump (tracers, records every 10 steps, "
                             "scratch tanh+rand initial state) timed from its per-step output line")
    return out


def ref_exe() -> Path:
    return ROOT / "oracle" / "_ref" / REF_TAG / "temppart_dump"


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def ref_ranks(cores: int) -> int:
    p = 1
    while p * 2 <= min(cores, 128):
        p *= 2
    return p


def run_reference(steps: int, warmup: int, ranks: int, time_cap: float, exe: Path | None = None,
                  particles=None) -> dict:
    """Run the reference on `ranks` processes; the per-step time comes from
    the wall-clock arrival of its per-step stdout line (temppart_dump.c:1698),
    measured over steps warmup+1 .. warmup+steps, then the run is stopped.
    exe: a reference build (default: the production-trajectory one);
    particles: (ids, x, y) of its restart particle files."""
    import resource

    exe = exe or ref_exe()
    if not exe.exists():
        raise FileNotFoundError(f"{exe} missing (built by __graft_entry__.build() where the reference is present)")
    wd = Path(tempfile.mkdtemp(prefix="lbrb_bench_ref_"))
    (wd / "Prtcl_Veldata1" / "Particles0.h5.d").mkdir(parents=True)
    (wd / "Tempfolder").mkdir()
    if particles is None:
        ids, x, y, _, _ = particle_setup(SEED + 1)
    else:
        ids, x, y = particles
    ids.astype(np.int32).tofile(wd / "Prtcl_Veldata1" / "Particles0.h5.d" / "id.bin")
    rec = np.zeros((len(ids), 8))
    rec[:, 0], rec[:, 1], rec[:, 4], rec[:, 5] = x, y, x, y
    rec.tofile(wd / "prtcl_dump0.in")

    def pre():
        for lim in (resource.RLIMIT_STACK,):
            try:
                resource.setrlimit(lim, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
            except (ValueError, OSError):
                pass
        soft, hard = resource.getrlimit(resource.RLIMIT_NOFILE)
        try:
            resource.setrlimit(resource.RLIMIT_NOFILE, (min(hard, 1 << 16), hard))
        except (ValueError, OSError):
            pass

    env = dict(os.environ, LBRB_SHIM_NP=str(ranks))
    env.pop("LBRB_SHIM_DIMS", None)
    p = subprocess.Popen([str(exe)], cwd=wd, env=env, stdout=subprocess.PIPE,
                         stderr=subprocess.DEVNULL, preexec_fn=pre, start_new_session=True,
                         text=True, bufsize=1)
    stamps = {}
    a, want = warmup, warmup + steps
    t_start = time.time()
    try:
        for line in p.stdout:
            if line.startswith("Loop "):
                s = int(line.split()[1])
                if s == max(a, 1) or s == want or s >= a:
                    stamps[s] = time.time()
                if s >= want or (s > a and time.time() - stamps.get(max(a, 1), t_start) > time_cap):
                    break
    finally:
        try:
            os.killpg(p.pid, signal.SIGKILL)
        except ProcessLookupError:
            pass
        p.wait()
        import shutil
        shutil.rmtree(wd, ignore_errors=True)
    s0 = max(a, 1)
    s1 = max(stamps)
    if s1 <= s0:
        raise RuntimeError("reference produced too few steps")
    per = (stamps[s1] - stamps[s0]) / (s1 - s0)
    return {"per_step_s": per, "steps": s1 - s0, "ranks": ranks}


def cpu_baseline(args) -> dict:
    try:
        cores = host_cores()
        ranks = ref_ranks(cores)
        res = run_reference(steps=40, warmup=3, ranks=ranks, time_cap=25.0)
        return {"value": round(NX * NY / res["per_step_s"] / 1e6, 3), "unit": "MLUPS",
                "cores": res["ranks"], "kind": "reference",
                "sample": f"reference temppart_dump (gcc -O2, {res['ranks']} ranks on {cores} host "
                          f"cores), {NX}x{NY}, 2^17 inertial particles (one St), {res['steps']} "
                          f"steps timed from its per-step output line"}
    except Exception as e:  # reported, never fatal for our arm
        return {"value": None, "unit": "MLUPS", "cores": None, "kind": "reference",
                "sample": f"unavailable: {e}"}


def run_reference_arm(args) -> dict:
    cores = host_cores()
    ranks = ref_ranks(cores)
    res = run_reference(steps=args.steps, warmup=args.warmup, ranks=ranks, time_cap=REF_STEPS_CAP_S)
    mlups = NX * NY / res["per_step_s"] / 1e6
    sample = (f"reference temppart_dump (its own C sources, gcc -O2, MPI/HDF5 stand-ins), "
              f"{res['ranks']} ranks on {cores} host cores, {NX}x{NY}, 2^17 inertial particles "
              f"(one St: the reference compiles one particle type), {res['steps']} timed steps")
    return {"impl": "reference", "metric": METRIC,
            "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": res["steps"], "warmup": args.warmup,
            "ms_per_step": round(res["per_step_s"] * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": f"{NX}x{NY}", "particles": NPRTCL},
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": res["ranks"],
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_lb_only(args, torch) -> dict:
    """The fused stream/collide kernel alone on a grid of --grid (no
    particles): the command used for ncu captures of lb_node_kernel."""
    import lagrangianrbnudging_b200 as lb
    from lagrangianrbnudging_b200 import build as b

    b.build()
    nx, ny = (int(a) for a in args.grid.lower().split("x"))
    base = lb.closure(nx, ny, Ra=RA, Pr=PR, U=U)
    fixed = dict(autotune=0, launch_shape=args.shape) if args.shape >= 0 else {}
    with lb.Run(**base, precision=args.precision, device=0, **fixed) as r:
        r.set_pairs(PAIRS_MODE)
        if args.pair_shape >= 0:
            r.set_pair_shape(args.pair_shape)
        r.init_conduction(SEED, 1e-3)
        ms, timing, _, _ = timed_steps(r, torch, args.steps, args.warmup, None, 0)
        shape = r.launch_shape()
        pair = r.pair_shape()
    lb_ms, n = timing["lb_step"]
    avg = lb_ms / max(n, 1)
    spl = args.steps / max(n, 1)  # node-steps per fused launch (2 for two-step launches)
    gbs = ALG_BYTES[args.precision] * nx * ny * spl / (avg * 1e-3) / 1e9
    return {"mode": "lb-only", "grid": f"{nx}x{ny}", "precision": args.precision,
            "steps": args.steps, "avg_lb_ms": round(avg, 5), "ms_per_step_fused": round(lb_ms / args.steps, 5),
            "node_steps_per_launch": round(spl, 4), "alg_gbs": round(gbs, 1),
            # from the fused launches' own event times (the uninstrumented window's
            # total can include one-time work after a short warm-up)
            "mlups": round(nx * ny * args.steps / (lb_ms * 1e3), 1), "window_ms": round(ms, 3),
            "launch_shape": shape, "pair_shape": pair}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=40)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-nudging", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--nudging-steps", type=int, default=NUD_STEPS)
    ap.add_argument("--nudging-only", action="store_true",
                    help="only the nudging twin experiment")
    ap.add_argument("--ensemble-steps", type=int, default=ENS_STEPS)
    ap.add_argument("--ensemble-variant", type=int, default=-1,
                    help="fixed launch variant of the ensemble's fused phase (-1: autotune)")
    ap.add_argument("--config0", action="store_true",
                    help="the 512x256 tracer case on the GPU and the reference CPU build")
    ap.add_argument("--no-slab", action="store_true", help="skip the y-slab section")
    ap.add_argument("--pair-shape", type=int, default=-1,
                    help="lb-only: fixed tile shape of the two-step launch instead of the autotuner")
    ap.add_argument("--no-pairs", action="store_true",
                    help="one fused launch per step (lbrb_set_pairs 0) instead of two steps per launch")
    ap.add_argument("--slab-only", action="store_true",
                    help="only the y-slab section (one domain as 2 and 4 slabs against one handle)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="only the adjoint window (the command used for ncu captures of the adjoint kernels)")
    ap.add_argument("--adjoint-steps", type=int, default=ADJ_STEPS)
    ap.add_argument("--adjoint-k", type=int, default=ADJ_K, help="checkpoint interval of the adjoint window")
    ap.add_argument("--adjoint-variant", type=int, default=-1,
                    help="fixed launch variant of the two-step adjoint kernel (-1: autotune)")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="only the ensemble section (the command used for ncu captures of ens_lb_kernel)")
    ap.add_argument("--adjoint-check", action="store_true",
                    help="FD check of the adjoint gradient at the adjoint configuration")
    ap.add_argument("--nu-stationary", action="store_true",
                    help="FP32 vs FP64 time-averaged Nu on a statistically stationary state (minutes of GPU time)")
    ap.add_argument("--nu-tff", type=float, default=6.0, help="free-fall times of --nu-stationary")
    ap.add_argument("--nu-discard", type=float, default=3.0, help="free-fall times dropped as the transient")
    ap.add_argument("--lb-only", action="store_true",
                    help="fused kernel alone on --grid (the ncu capture command)")
    ap.add_argument("--grid", default="2048x1024")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--shape", type=int, default=-1,
                    help="lb-only: fixed launch shape index instead of the autotuner")
    args = ap.parse_args()
    global PAIRS_MODE
    if args.no_pairs:
        PAIRS_MODE = 0
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference_arm(args)), flush=True)
        return
    import torch

    if args.lb_only:
        torch.cuda.set_device(0)
        print(json.dumps(run_lb_only(args, torch)), flush=True)
        return
    if args.config0:
        import lagrangianrbnudging_b200 as lb
        from lagrangianrbnudging_b200 import build as b

        b.build()
        torch.cuda.set_device(0)
        print(json.dumps({"mode": "config0", **run_config0(lb, torch, 0)}), flush=True)
        return
    if args.slab_only:
        import lagrangianrbnudging_b200 as lb
        from lagrangianrbnudging_b200 import build as b

        b.build()
        torch.cuda.set_device(0)
        print(json.dumps({"mode": "slab-only", **run_slab_bench(lb, torch, 0)}), flush=True)
        return
    if args.adjoint_only:
        import lagrangianrbnudging_b200 as lb
        from lagrangianrbnudging_b200 import build as b

        b.build()
        torch.cuda.set_device(0)
        print(json.dumps({"mode": "adjoint-only", **run_adjoint_bench(lb, torch, 0, args.adjoint_steps,
                                                                      args.adjoint_k, args.adjoint_variant)}),
              flush=True)
        return
    if args.nudging_only:
        import lagrangianrbnudging_b200 as lb
        from lagrangianrbnudging_b200 import build as b

        b.build()
        torch.cuda.set_device(0)
        print(json.dumps({"mode": "nudging-only", **run_nudging_bench(lb, torch, 0, args.nudging_steps)}),
              flush=True)
        return
    if args.ensemble_only:
        import lagrangianrbnudging_b200 as lb
        from lagrangianrbnudging_b200 import build as b

        b.build()
        torch.cuda.set_device(0)
        print(json.dumps({"mode": "ensemble-only",
                          **run_ensemble_bench(lb, torch, 0, args.ensemble_steps, args.ensemble_variant)}),
              flush=True)
        return
    if args.adjoint_check:
        import lagrangianrbnudging_b200 as lb
        from lagrangianrbnudging_b200 import build as b

        b.build()
        torch.cuda.set_device(0)
        print(json.dumps(run_adjoint_check(lb, torch, 0)), flush=True)
        return
    if args.nu_stationary:
        import lagrangianrbnudging_b200 as lb
        from lagrangianrbnudging_b200 import build as b

        b.build()
        torch.cuda.set_device(0)
        print(json.dumps(run_stationary_nu(lb, 0, args.nu_tff, args.nu_discard)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    else:
        torch.cuda.set_device(0)
    out = run_ours(args, torch, dist, rank, world, local)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
