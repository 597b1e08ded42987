// nudge_dev.cuh -- bilinear-4 nudging of one observation, shared by the
// single-run kernels (nudge_kernels.cu) and the ensemble kernels
// (ensemble_kernels.cu).  The innovation alpha (T_obs - T(x_p)) uses the
// reference's bilinear() form (Trajectories/code/mympi2.h:292-311) and is
// scattered to the 4 cell corners with 2^-40 fixed-point int64 atomics:
// integer sums do not depend on the order of the atomics, so the result is
// deterministic.  The apply pass takes each touched node's sum once (atomic
// exchange, leaving the accumulator cleared) and adds w_k * sum to its g.
#pragma once

#include <type_traits>

#include "lb_node.cuh"
#include "lbrb_internal.cuh"

namespace lbrb {


__device__ __forceinline__ void obs_cell(double xx, double yy, int nx, int ny, int& x1, int& y1,
                                         int& ix1, int& ix2, int& jy1, int& jy2) {
  x1 = (int)xx;
  y1 = (int)yy;
  ix1 = (x1 - 1) % nx; if (ix1 < 0) ix1 += nx;
  ix2 = x1 % nx; if (ix2 < 0) ix2 += nx;
  jy1 = (y1 - 1) % ny; if (jy1 < 0) jy1 += ny;
  jy2 = y1 % ny; if (jy2 < 0) jy2 += ny;
}

// Innovation of one observation, scattered to those of its 4 cell corners
// whose rows lie in [j0, j0 + nyl) of the accumulator (a whole domain: j0 =
// 0, nyl = ny; a y-slab: its own rows, indexed from j0).  Tat(j, i) is the
// temperature at global row j, column i.
template <typename TAt>
__device__ __forceinline__ void obs_scatter_rows(TAt Tat, int nx, int ny, int pitch, double xx, double yy,
                                                 double Tobs, double alpha, unsigned long long* __restrict__ acc,
                                                 unsigned* dflags, int j0, int nyl) {
  if (!(xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0)) {
    atomicOr(dflags, DFLAG_RANGE);
    return;
  }
  int x1, y1, ix1, ix2, jy1, jy2;
  obs_cell(xx, yy, nx, ny, x1, y1, ix1, ix2, jy1, jy2);
  const bool in1 = (unsigned)(jy1 - j0) < (unsigned)nyl, in2 = (unsigned)(jy2 - j0) < (unsigned)nyl;
  if (!in1 && !in2) return;
  const int x2 = x1 + 1, y2 = y1 + 1;
  const double u11 = (double)Tat(jy1, ix1);
  const double u12 = (double)Tat(jy2, ix1);
  const double u21 = (double)Tat(jy1, ix2);
  const double u22 = (double)Tat(jy2, ix2);
  const double val1 = u11 * ((double)x2 - xx) * ((double)y2 - yy);
  const double val2 = u21 * (xx - (double)x1) * ((double)y2 - yy);
  const double val3 = u12 * ((double)x2 - xx) * (yy - (double)y1);
  const double val4 = u22 * (xx - (double)x1) * (yy - (double)y1);
  const double tm = val1 + val2 + val3 + val4;
  const double dlt = alpha * (Tobs - tm);
  const double wx1 = (double)x2 - xx, wx2 = xx - (double)x1;
  const double wy1 = (double)y2 - yy, wy2 = yy - (double)y1;
  if (in1) {
    unsigned long long* r = acc + (size_t)(jy1 - j0) * pitch;
    atomicAdd(&r[ix1], (unsigned long long)__double2ll_rn(dlt * (wx1 * wy1) * FIX_SCALE));
    atomicAdd(&r[ix2], (unsigned long long)__double2ll_rn(dlt * (wx2 * wy1) * FIX_SCALE));
  }
  if (in2) {
    unsigned long long* r = acc + (size_t)(jy2 - j0) * pitch;
    atomicAdd(&r[ix1], (unsigned long long)__double2ll_rn(dlt * (wx1 * wy2) * FIX_SCALE));
    atomicAdd(&r[ix2], (unsigned long long)__double2ll_rn(dlt * (wx2 * wy2) * FIX_SCALE));
  }
}

template <typename Real>
__device__ __forceinline__ void obs_scatter_one(const Real* __restrict__ T, int nx, int ny, int pitch,
                                                double xx, double yy, double Tobs, double alpha,
                                                unsigned long long* __restrict__ acc,
                                                unsigned* dflags) {
  obs_scatter_rows([&](int j, int i) { return T[(size_t)j * pitch + i]; }, nx, ny, pitch, xx, yy, Tobs, alpha,
                   acc, dflags, 0, ny);
}

// corner `corner` (0..3) of the observation at (xx, yy), when its row lies
// in [j0, j0 + nyl) (rows of g and acc indexed from j0)
template <typename Real>
__device__ __forceinline__ void obs_apply_one(Real* __restrict__ g, size_t plane, int nx, int ny,
                                              int pitch, double xx, double yy, int corner,
                                              unsigned long long* __restrict__ acc, int j0 = 0, int nyl = -1) {
  if (!(xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0)) return;
  const int x1 = (int)xx + (corner & 1), y1 = (int)yy + (corner >> 1);
  int ix = (x1 - 1) % nx; if (ix < 0) ix += nx;
  int jy = (y1 - 1) % ny; if (jy < 0) jy += ny;
  if (nyl >= 0 && (unsigned)(jy - j0) >= (unsigned)nyl) return;
  const size_t q = (size_t)(jy - j0) * pitch + ix;
  const long long sfix = (long long)atomicExch(&acc[q], 0ull);
  if (sfix == 0) return;
  const double sv = (double)sfix * (1.0 / FIX_SCALE);
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    Real* a = g + (size_t)k * plane + q;
    *a = *a + nudge_increment<Real>(k, sv);
  }
}

// T^n at node (i, j) as the fused step forms it: the sum of the g streaming
// into the node (Dirichlet walls, no slab ghost rows), in the step's order --
// the g half of pull_node and dirichlet_walls
template <typename Real>
__device__ __forceinline__ Real pulled_T(const LBView<Real>& V, int j, int i) {
  const int xl = (i == 0) ? V.nx - 1 : i - 1, xr = (i == V.nx - 1) ? 0 : i + 1;
  Real gs[NPOP];
  static_for<NPOP>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    const int xs = icx(k) == 1 ? xl : (icx(k) == -1 ? xr : i);
    const int js = j - icy(k);
    gs[k] = (js < 0 || js >= V.ny) ? Real(0) : V.gsrc[(size_t)k * V.plane + (size_t)js * V.pitch + xs];
  });
  dirichlet_walls(V, j, gs);
  if constexpr (std::is_same<Real, double>::value) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < NPOP; k++) t = t + gs[k];
    return t;
  } else {
    float dT = 0.f;
#pragma unroll
    for (int k = 0; k < NPOP; k++) dT += gs[k];
    return V.T0_f + dT;
  }
}

// Two-step launch of a nudged run, before the launch: the innovation of one
// observation of step n from T^n at its cell corners, with four threads per
// observation (lanes 4p .. 4p+3 of a warp, one per corner).  T^n is the
// moment of the g populations streaming into a corner -- pulled from the
// state before the step (V's sources), walls applied, summed as the fused
// step sums it (pulled_T) -- so it equals the T the step itself forms.  The
// lanes share their corners' T by shuffles, every lane forms the innovation
// with obs_scatter_rows' expressions, and each adds its own corner's share
// to acc (fixed point, as a single step's scatter) and its bit to the node
// mask (pitch / 32 words per row), which the two-step kernels read to add
// the sums after the collision.  All 32 lanes of the warp must call it
// (live: the lane's observation exists).
template <typename Real>
__device__ __forceinline__ void obs_pre_corner(const LBView<Real>& V, bool live, double xx, double yy, double Tobs,
                                               double alpha, int corner, unsigned long long* __restrict__ acc,
                                               unsigned* __restrict__ mask, unsigned* dflags) {
  const int nx = V.nx, ny = V.ny;
  const bool inr = live && xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0;
  if (live && !inr && corner == 0) atomicOr(dflags, DFLAG_RANGE);
  int x1, y1, ix1, ix2, jy1, jy2;
  obs_cell(inr ? xx : 1.0, inr ? yy : 1.0, nx, ny, x1, y1, ix1, ix2, jy1, jy2);
  const int ix = (corner & 1) ? ix2 : ix1, jy = (corner >> 1) ? jy2 : jy1;
  const Real Tc = inr ? pulled_T(V, jy, ix) : Real(0);
  const int base = (threadIdx.x & 31) & ~3;
  const double u11 = (double)__shfl_sync(0xffffffffu, Tc, base + 0);
  const double u21 = (double)__shfl_sync(0xffffffffu, Tc, base + 1);
  const double u12 = (double)__shfl_sync(0xffffffffu, Tc, base + 2);
  const double u22 = (double)__shfl_sync(0xffffffffu, Tc, base + 3);
  if (!inr) return;
  const int x2 = x1 + 1, y2 = y1 + 1;
  const double val1 = u11 * ((double)x2 - xx) * ((double)y2 - yy);
  const double val2 = u21 * (xx - (double)x1) * ((double)y2 - yy);
  const double val3 = u12 * ((double)x2 - xx) * (yy - (double)y1);
  const double val4 = u22 * (xx - (double)x1) * (yy - (double)y1);
  const double tm = val1 + val2 + val3 + val4;
  const double dlt = alpha * (Tobs - tm);
  const double wx = (corner & 1) ? xx - (double)x1 : (double)x2 - xx;
  const double wy = (corner >> 1) ? yy - (double)y1 : (double)y2 - yy;
  atomicAdd(&acc[(size_t)jy * V.pitch + ix], (unsigned long long)__double2ll_rn(dlt * (wx * wy) * FIX_SCALE));
  atomicOr(&mask[(size_t)jy * (V.pitch >> 5) + (ix >> 5)], 1u << (ix & 31));
}

// after the launch: clear corner `corner` (0..3) of an observation of step n
__device__ __forceinline__ void obs_clear_one(int nx, int ny, int pitch, double xx, double yy, int corner,
                                              unsigned long long* __restrict__ acc, unsigned* __restrict__ mask) {
  if (!(xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0)) return;
  int ix = ((int)xx + (corner & 1) - 1) % nx;
  if (ix < 0) ix += nx;
  int jy = ((int)yy + (corner >> 1) - 1) % ny;
  if (jy < 0) jy += ny;
  acc[(size_t)jy * pitch + ix] = 0ull;
  atomicAnd(&mask[(size_t)jy * (pitch >> 5) + (ix >> 5)], ~(1u << (ix & 31)));
}

}  // namespace lbrb
