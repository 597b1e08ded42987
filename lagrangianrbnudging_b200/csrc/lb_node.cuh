// lb_node.cuh -- the per-node update of the fused stream/collide step, shared
// by the single-run kernel (lb_kernels.cu) and the ensemble kernel
// (ensemble_kernels.cu), so that both execute the same arithmetic.
//
// Reference semantics (temppart_dump.c, Trajectories):
//   stream          :781-854   f_k(x) <- f_k(x - c_k) for k = 1..8, same for g
//   force           :744-755   F_y = -gravity * rho^{n-1} * T^{n-1}, F_x = 0
//   f walls         :763-777, 859-894   half-way bounce-back from the
//                              pre-stream wall row
//   g walls (T)     :896-921   g_in = -g_opp(post-stream) + 2 w T_wall
//   g walls (N)     tempvel_nudge.c:684-702, 783-962: adiabatic copy rows
//   moments         :957-987 (tempvel_nudge.c:1069-1102 adds 1/2 nud_term)
//   collision       :1097-1180, 1314-1341 (tempvel_nudge.c:1917-1945 nudged g)
#pragma once

#include <type_traits>

#include "lbrb_internal.cuh"

namespace lbrb {

template <int K, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (K > 0) {
    static_for<K - 1>(f);
    f(std::integral_constant<int, K - 1>{});
  }
}

// ------------------------------------------------ reference-order FP64 node
// SF(k, value), SG(k, value): store a post-collision population as soon as
// it is computed (short live ranges; the operation order is unchanged)
template <bool REFNUDGE, typename SF, typename SG>
__device__ __forceinline__ void node_ref(const LBView<double>& V, size_t idx, double* fs,
                                         double* gs, double& Fy_io, double& r_out, double& u_out,
                                         double& v_out, double& t_out, SF&& store_f, SG&& store_g) {
  double r = 0.0, t = 0.0;
#pragma unroll
  for (int k = 0; k < NPOP; k++) r = r + fs[k];
#pragma unroll
  for (int k = 0; k < NPOP; k++) t = t + gs[k];
  int nv = 0;
  if (REFNUDGE) {
    nv = V.nudge_vol[idx];
    if (idx < (size_t)V.pitch) V.tsum0[idx] = t;  // (row 0)
    if (nv > 0) t = (t + 0.5 * V.nud_term[idx]);
  }
  const double rhoi = 1. / r;
  double fl[NPOP];
#pragma unroll
  for (int k = 0; k < NPOP; k++) fl[k] = fs[k] * rhoi;
  const double Fx = 0.0;
  const double Fy = Fy_io;
  const double u = fl[1] - fl[3] + fl[5] - fl[6] - fl[7] + fl[8] + 0.5 * rhoi * Fx;
  const double v = fl[5] + fl[2] + fl[6] - fl[7] - fl[4] - fl[8] + 0.5 * rhoi * Fy;
  const double omega = V.omega, omegag = V.omegag;
  double feq[NPOP];
  equil_ref(r, u, v, feq);
  static_for<NPOP>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    double source = (1.0 - 0.5 * omega) * w_of(k);
    double factor = div_const((dcx(k) - u) * Fx + (dcy(k) - v) * Fy, CS2, RCP_CS2);
    factor = factor + div_const((dcx(k) * u + dcy(k) * v) * (dcx(k) * Fx + dcy(k) * Fy), DIV_CS4, RCP_CS4);
    fs[k] = fs[k] * (1. - omega) + omega * feq[k] + source * factor;
    store_f(k, fs[k]);
  });
  equil_ref(t, u, v, feq);
  if (REFNUDGE && nv > 0) {
    const double B = 1.0 - 0.5 * omegag;
    const double Q = V.alpha * (t - V.tempreadint[idx]);
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      gs[k] = gs[k] * (1. - omegag) + omegag * feq[k] - B * w_of(k) * Q;
      store_g(k, gs[k]);
    }
    V.nud_term[idx] = -1. * Q;
  } else {
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      gs[k] = gs[k] * (1. - omegag) + omegag * feq[k];
      store_g(k, gs[k]);
    }
  }
  // buoyancy of the next step from this step's moments (forcingconstructWW)
  Fy_io = V.neg_gravity * r * (t - 0.0);
  r_out = r;
  u_out = u;
  v_out = v;
  t_out = t;
}

// -------------------------------------------------- FP32 shifted-form node
// Shifted variables df_k = f_k - w_k, dg_k = g_k - w_k T0 and
//   dr = sum df, r = 1 + dr, u = jx / r, v = (jy + Fy/2) / r, t = T0 + sum dg
//   P_k = 3 c.u + 4.5 (c.u)^2 - 1.5 |u|^2
//   df_k' = df_k + om (w_k (dr + r P_k) - df_k) + (1 - om/2) w_k Fy (3 (cy - v) + 9 (c.u) cy)
//   dg_k' = dg_k + omg (w_k (dT + t P_k) - dg_k)
// in this relaxation form: the increment om (feq - df) is small near
// equilibrium, so its rounding error is small against df_k itself (a form
// that adds (1 - om) df_k and om feq_k rounds each at the scale of df_k and
// drifted 35% further from the FP64 path over 1000 steps)
// the same BGK + Guo collision as the reference, written with explicit fused
// multiply-adds (this translation unit is otherwise built without FMA
// contraction, which the FP64 reference-order form needs); c.u is picked per
// direction at compile time, so no multiplication by a zero lattice
// component is issued.
template <int K>
__device__ __forceinline__ float cdotu(float u, float v, float upv, float umv) {
  constexpr int cx = icx(K), cy = icy(K);
  if constexpr (cx == 0 && cy == 0) return 0.f;
  else if constexpr (cy == 0) return cx > 0 ? u : -u;
  else if constexpr (cx == 0) return cy > 0 ? v : -v;
  else if constexpr (cx == cy) return cx > 0 ? upv : -upv;
  else return cx > 0 ? umv : -umv;
}

__device__ __forceinline__ void node_shift(const LBView<float>& V, float* df, float* dg,
                                           float& Fy_io, float& r_out, float& u_out,
                                           float& v_out, float& t_out) {
  float dr = 0.f, dT = 0.f;
#pragma unroll
  for (int k = 0; k < NPOP; k++) dr += df[k];
#pragma unroll
  for (int k = 0; k < NPOP; k++) dT += dg[k];
  const float r = 1.f + dr;
  const float T0 = V.T0_f;
  const float t = T0 + dT;
  const float jx = (df[1] - df[3]) + (df[5] - df[6]) + (df[8] - df[7]);
  const float jy = (df[2] - df[4]) + (df[5] - df[7]) + (df[6] - df[8]);
  const float Fy = Fy_io;
  const float rinv = __frcp_rn(r);  // (the correctly rounded 1 / r)
  const float u = jx * rinv;
  const float v = fmaf(0.5f, Fy, jy) * rinv;
  const float om = V.omega_f, omg = V.omegag_f;
  const float srcFy = (1.f - 0.5f * om) * Fy;
  const float usq15 = 1.5f * fmaf(u, u, v * v);
  const float v3 = 3.f * v;
  const float upv = u + v, umv = u - v;
  static_for<NPOP>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    constexpr float w = (float)w_of(k);
    constexpr int cy = icy(k);
    const float cu = cdotu<k>(u, v, upv, umv);
    const float P = (k == 0) ? -usq15 : fmaf(cu, fmaf(4.5f, cu, 3.f), -usq15);
    // Guo source factor 3 (cy - v) + 9 (c.u) cy
    float G;
    if constexpr (cy == 0) G = -v3;
    else G = fmaf(cu, 9.f * cy, 3.f * cy - v3);
    const float dfeq = w * fmaf(r, P, dr);
    df[k] = fmaf(w * srcFy, G, fmaf(om, dfeq - df[k], df[k]));
    const float dgeq = w * fmaf(t, P, dT);
    dg[k] = fmaf(omg, dgeq - dg[k], dg[k]);
  });
  Fy_io = V.neg_gravity_f * r * t;
  r_out = r;
  u_out = u;
  v_out = v;
  t_out = t;
}

// ------------------------------------------------------------------ kernel
// Element offsets: Off = uint32_t when a population buffer (18 planes) holds
// fewer than 2^32 elements (off32_ok), else size_t.

// the 9 f and 9 g values streaming into node (x, j), walls applied for f
// (bounce-back) and for adiabatic g; Dirichlet g walls follow in dirichlet_walls
template <typename Real, int TWALL, typename Off, bool FAST = true>
__device__ __forceinline__ void pull_node(const LBView<Real>& V, int j, int x, Real* fs, Real* gs) {
  const int xl = (x == 0) ? V.nx - 1 : x - 1;       // source column of c_x = +1
  const int xr = (x == V.nx - 1) ? 0 : x + 1;       // source column of c_x = -1
  const Off pl = (Off)V.plane, pitch = (Off)V.pitch;
  const Off oc = (Off)j * pitch;
  // rows whose sources all lie inside the domain (for adiabatic g also off
  // the copy rows): no wall logic; the row is uniform over a block
  const bool interior = TWALL == LBRB_TWALL_ADIABATIC ? (j > 1 && j < V.ny - 2) : (j > 0 && j < V.ny - 1);
  if (FAST && interior) {
    static_for<NPOP>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      const int xs = icx(k) == 1 ? xl : (icx(k) == -1 ? xr : x);
      const Off row = icy(k) == 1 ? oc - pitch : (icy(k) == -1 ? oc + pitch : oc);
      const Off o = (Off)k * pl + row + (Off)xs;
      fs[k] = __ldcs(V.fsrc + o);
      gs[k] = __ldcs(V.gsrc + o);
    });
    return;
  }
  // adiabatic g walls at the domain's walls only (a y-slab's inner edge
  // has ghost rows instead)
  const bool wall_lo = !V.ghost_lo, wall_hi = !V.ghost_hi;
  const bool adia_wall = TWALL == LBRB_TWALL_ADIABATIC && ((j == 0 && wall_lo) || (j == V.ny - 1 && wall_hi));
  const int jc = (j == 0) ? 1 : V.ny - 2;
  static_for<NPOP>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    const int xs = icx(k) == 1 ? xl : (icx(k) == -1 ? xr : x);
    const int js = j - icy(k);
    // y-slab boundary inside the domain: the neighbour's boundary row
    const Real* gh = js < 0 ? V.ghost_lo : (js >= V.ny ? V.ghost_hi : nullptr);
    if (gh) {
      constexpr int slot = (k == 2 || k == 4) ? 0 : ((k == 5 || k == 7) ? 1 : 2);
      fs[k] = gh[(size_t)slot * V.nx + xs];
      gs[k] = gh[(size_t)(3 + slot) * V.nx + xs];
      return;
    }
    if (js < 0 || js >= V.ny)
      fs[k] = __ldcs(V.fsrc + ((Off)opp(k) * pl + oc + (Off)x));
    else
      fs[k] = __ldcs(V.fsrc + ((Off)k * pl + (Off)js * pitch + (Off)xs));
    if (adia_wall) {
      gs[k] = __ldcs(V.gsrc + ((Off)k * pl + (Off)jc * pitch + (Off)x));
    } else {
      int jg = js;
      if (TWALL == LBRB_TWALL_ADIABATIC) {
        if (jg == 0 && wall_lo) jg = 1;
        else if (jg == V.ny - 1 && wall_hi) jg = V.ny - 2;
      }
      gs[k] = (jg < 0 || jg >= V.ny) ? Real(0)
                                      : __ldcs(V.gsrc + ((Off)k * pl + (Off)jg * pitch + (Off)xs));
    }
  });
}

// anti-bounce-back with the post-stream opposite population
// (temppart_dump.c:896-921): g_in = -g_opp + 2 w T_wall (shifted form: T_wall - T0)
template <typename Real>
__device__ __forceinline__ void dirichlet_walls(const LBView<Real>& V, int j, Real* gs) {
  if (j == V.ny - 1 && !V.ghost_hi) {
    const Real tw = std::is_same<Real, double>::value ? (Real)V.Tup : (Real)(V.Tup - V.T0);
    gs[4] = -gs[2] + Real(2.0 * w_of(2)) * tw;
    gs[7] = -gs[5] + Real(2.0 * w_of(5)) * tw;
    gs[8] = -gs[6] + Real(2.0 * w_of(6)) * tw;
  }
  if (j == 0 && !V.ghost_lo) {
    const Real tw = std::is_same<Real, double>::value ? (Real)V.Tdown : (Real)(V.Tdown - V.T0);
    gs[2] = -gs[4] + Real(2.0 * w_of(4)) * tw;
    gs[5] = -gs[7] + Real(2.0 * w_of(7)) * tw;
    gs[6] = -gs[8] + Real(2.0 * w_of(8)) * tw;
  }
}


// moments and collision of a pulled node (idx: its element offset, for the
// box-nudging fields); SF(k, f_k'), SG(k, g_k') take the post-collision
// populations and Fy_io becomes the next step's buoyancy
template <typename Real, bool REFNUDGE, typename SF, typename SG>
__device__ __forceinline__ void lb_collide(const LBView<Real>& V, size_t idx, Real* fs, Real* gs, Real& Fy_io,
                                           Real& r, Real& u, Real& v, Real& t, SF&& store_f, SG&& store_g) {
  if constexpr (std::is_same<Real, double>::value) {
    node_ref<REFNUDGE>(V, idx, fs, gs, Fy_io, r, u, v, t, store_f, store_g);
  } else {
    node_shift(V, fs, gs, Fy_io, r, u, v, t);
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      store_f(k, fs[k]);
      store_g(k, gs[k]);
    }
  }
}

// moments, collision and stores of node o from its pulled populations and
// this step's buoyancy Fy
template <typename Real, bool REFNUDGE, typename Off>
__device__ __forceinline__ void lb_finish_node(const LBView<Real>& V, Off o, Real* fs, Real* gs, Real Fy) {
  const Off pl = (Off)V.plane;
  Real r, u, v, t;
  lb_collide<Real, REFNUDGE>(
      V, (size_t)o, fs, gs, Fy, r, u, v, t, [&](int k, Real val) { __stcs(V.fdst + ((Off)k * pl + o), val); },
      [&](int k, Real val) { __stcs(V.gdst + ((Off)k * pl + o), val); });
  V.Fout[o] = Fy;
  if (V.write_uv) {
    V.u[o] = u;
    V.v[o] = v;
  }
  if (V.write_rt & 1) V.T[o] = t;
  if (V.write_rt & 2) V.rho[o] = r;
}

// one node of one step: pull (walls applied), moments, collision, stores
// FAST: interior rows take the pull without wall logic (else every row takes
// the general pull)
template <typename Real, int TWALL, bool REFNUDGE, typename Off = size_t, bool FAST = true>
__device__ __forceinline__ void lb_update_node(const LBView<Real>& V, int j, int x) {
  Real fs[NPOP], gs[NPOP];
  pull_node<Real, TWALL, Off, FAST>(V, j, x, fs, gs);
  if (TWALL == LBRB_TWALL_DIRICHLET) dirichlet_walls(V, j, gs);
  const Off o = (Off)j * (Off)V.pitch + (Off)x;
  lb_finish_node<Real, REFNUDGE, Off>(V, o, fs, gs, V.Fin[o]);
}

}  // namespace lbrb
