// aux_kernels.cu -- state set-up and read-out, diagnostics.
//
//  * layout conversion between the host layouts of lbrb.h (the reference's
//    haloed AoS pop_type arrays, or interior SoA) and the device layout,
//    with the FP32 shifted form (f_k - w_k, g_k - w_k T0) applied on the way;
//  * the restart-route moments (inithydro scratch==0, temppart_dump.c:703-726);
//  * the seeded conduction initial state;
//  * compensated FP64 reductions: mean kinetic energy and temperature
//    (temppart_dump.c:1739-1757), Nusselt number, per-row profiles
//    (tempvel_nudge.c:1104-1260);
//  * a NaN/Inf scan of the populations.
#include <type_traits>

#include "lbrb_internal.cuh"

namespace lbrb {

__device__ __forceinline__ int wrapn(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

// host index of interior node (i, j) (0-based) and population k
__device__ __forceinline__ size_t host_pop_index(int layout, int nx, int ny, int i, int j, int k) {
  if (layout == LBRB_LAYOUT_REF_AOS_HALO)
    return ((size_t)(j + 1) + (size_t)(ny + 2) * (size_t)(i + 1)) * NPOP + k;
  return ((size_t)k * ny + j) * nx + i;
}
__device__ __forceinline__ size_t host_scalar_index(int layout, int nx, int ny, int i, int j) {
  if (layout == LBRB_LAYOUT_REF_AOS_HALO) return (size_t)(j + 1) + (size_t)(ny + 2) * (size_t)(i + 1);
  return (size_t)j * nx + i;
}

// host -> device populations; base = rho0 (f) or T0 (g) for the shifted form
template <typename Real>
__global__ void pops_in_kernel(const double* __restrict__ h, int layout, Real* __restrict__ d,
                               int nx, int ny, int pitch, size_t plane, double base) {
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      const double a = h[host_pop_index(layout, nx, ny, i, j, k)];
      Real* o = d + (size_t)k * plane + (size_t)j * pitch + i;
      if constexpr (std::is_same<Real, double>::value) *o = a;
      else *o = (float)(a - w_of(k) * base);
    }
  }
}

// device -> host populations; the reference layout's halo is filled with
// periodic copies in x and y (what pbc() leaves, temppart_dump.c:234-250)
template <typename Real>
__global__ void pops_out_kernel(const Real* __restrict__ d, int layout, double* __restrict__ h,
                                int nx, int ny, int pitch, size_t plane, double base) {
  const int hx = layout == LBRB_LAYOUT_REF_AOS_HALO ? nx + 2 : nx;
  const int hy = layout == LBRB_LAYOUT_REF_AOS_HALO ? ny + 2 : ny;
  const long n = (long)hx * hy;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    int a = (int)(q % hx), b = (int)(q / hx);
    int i = a, j = b;
    if (layout == LBRB_LAYOUT_REF_AOS_HALO) { i = wrapn(a - 1, nx); j = wrapn(b - 1, ny); }
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      const Real v = d[(size_t)k * plane + (size_t)j * pitch + i];
      double o;
      if constexpr (std::is_same<Real, double>::value) o = v;
      else o = (double)v + w_of(k) * base;
      if (layout == LBRB_LAYOUT_REF_AOS_HALO)
        h[((size_t)b + (size_t)(ny + 2) * (size_t)a) * NPOP + k] = o;
      else
        h[((size_t)k * ny + j) * nx + i] = o;
    }
  }
}

template <typename Real>
__global__ void scalar_in_kernel(const double* __restrict__ h, int layout, Real* __restrict__ d,
                                 int nx, int ny, int pitch) {
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    d[(size_t)j * pitch + i] = (Real)h[host_scalar_index(layout, nx, ny, i, j)];
  }
}

template <typename Real>
__global__ void scalar_out_kernel(const Real* __restrict__ d, int layout, double* __restrict__ h,
                                  int nx, int ny, int pitch) {
  const int hx = layout == LBRB_LAYOUT_REF_AOS_HALO ? nx + 2 : nx;
  const int hy = layout == LBRB_LAYOUT_REF_AOS_HALO ? ny + 2 : ny;
  const long n = (long)hx * hy;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    int a = (int)(q % hx), b = (int)(q / hx);
    int i = a, j = b;
    if (layout == LBRB_LAYOUT_REF_AOS_HALO) {
      i = wrapn(a - 1, nx);
      j = wrapn(b - 1, ny);
      h[(size_t)b + (size_t)(ny + 2) * (size_t)a] = (double)d[(size_t)j * pitch + i];
    } else {
      h[(size_t)j * nx + i] = (double)d[(size_t)j * pitch + i];
    }
  }
}

// ------------------------------------------------ chunked host transfers
// A host array moves in chunks of whole units through a staging slot.  A unit
// is one halo column of the reference layout ((ny + 2) nodes of NP values:
// unit a starts at host element a (ny + 2) NP) or one row of nx values of the
// SoA layout (row r = k ny + j of population plane k, or row j of a scalar
// field: unit r starts at host element r nx).  The staging slot holds units
// [u0, u1) as they lie in the host array.  NP: 9 populations (FP32 handles
// store them shifted by w_k base), or 1 for a scalar field.
template <typename Real, int NP>
__global__ void units_in_kernel(const double* __restrict__ st, int layout, Real* __restrict__ d, int nx, int ny,
                                int pitch, size_t plane, double base, int u0, int u1) {
  auto cv = [&](double a, int k) -> Real {
    if constexpr (std::is_same<Real, double>::value) return a;
    else return NP == NPOP ? (float)(a - w_of(k) * base) : (float)a;
  };
  if (layout == LBRB_LAYOUT_REF_AOS_HALO) {
    // interior nodes of halo columns [u0, u1) (1 <= u0, u1 <= nx + 1)
    const long n = (long)(u1 - u0) * ny;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
      const int a = u0 + (int)(q / ny), j = (int)(q % ny);
      const double* src = st + ((size_t)(a - u0) * (ny + 2) + (j + 1)) * NP;
#pragma unroll
      for (int k = 0; k < NP; k++) d[(size_t)k * plane + (size_t)j * pitch + (a - 1)] = cv(src[k], k);
    }
  } else {
    const long n = (long)(u1 - u0) * nx;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
      const int r = u0 + (int)(q / nx), i = (int)(q % nx);
      const int k = r / ny, j = r % ny;
      d[(size_t)k * plane + (size_t)j * pitch + i] = cv(st[(size_t)(r - u0) * nx + i], k);
    }
  }
}

// the other way; the reference layout's halo holds periodic copies in x and
// y (what pbc() leaves, temppart_dump.c:234-250)
template <typename Real, int NP>
__global__ void units_out_kernel(const Real* __restrict__ d, int layout, double* __restrict__ st, int nx, int ny,
                                 int pitch, size_t plane, double base, int u0, int u1) {
  auto cv = [&](Real a, int k) -> double {
    if constexpr (std::is_same<Real, double>::value) return a;
    else return NP == NPOP ? (double)a + w_of(k) * base : (double)a;
  };
  if (layout == LBRB_LAYOUT_REF_AOS_HALO) {
    const long n = (long)(u1 - u0) * (ny + 2);
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
      const int a = u0 + (int)(q / (ny + 2)), b = (int)(q % (ny + 2));
      const int i = wrapn(a - 1, nx), j = wrapn(b - 1, ny);
      double* dst = st + ((size_t)(a - u0) * (ny + 2) + b) * NP;
#pragma unroll
      for (int k = 0; k < NP; k++) dst[k] = cv(d[(size_t)k * plane + (size_t)j * pitch + i], k);
    }
  } else {
    const long n = (long)(u1 - u0) * nx;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
      const int r = u0 + (int)(q / nx), i = (int)(q % nx);
      const int k = r / ny, j = r % ny;
      st[(size_t)(r - u0) * nx + i] = cv(d[(size_t)k * plane + (size_t)j * pitch + i], k);
    }
  }
}

// buoyancy of the first step from the moments in place (forcingconstructWW)
template <typename Real>
__global__ void force_kernel(const Real* __restrict__ rho, const Real* __restrict__ T,
                             Real* __restrict__ F, int nx, int ny, int pitch, double neg_gravity) {
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const size_t o = (size_t)j * pitch + i;
    if constexpr (std::is_same<Real, double>::value) F[o] = neg_gravity * rho[o] * (T[o] - 0.0);
    else F[o] = (float)neg_gravity * rho[o] * T[o];
  }
}

// restart-route moments from "pre" populations held in the host layout
template <typename Real>
__global__ void moments_from_pre_kernel(const double* __restrict__ fpre, const double* __restrict__ gpre,
                                        int layout, Real* __restrict__ rho, Real* __restrict__ u,
                                        Real* __restrict__ v, Real* __restrict__ T, int nx, int ny,
                                        int pitch, double neg_gravity) {
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    double fk[NPOP], r = 0.0, t = 0.0;
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      fk[k] = fpre[host_pop_index(layout, nx, ny, i, j, k)];
      r = r + fk[k];
    }
#pragma unroll
    for (int k = 0; k < NPOP; k++) t = t + gpre[host_pop_index(layout, nx, ny, i, j, k)];
    const double rhoi = 1. / r;
    double fl[NPOP];
#pragma unroll
    for (int k = 0; k < NPOP; k++) fl[k] = fk[k] * rhoi;
    const size_t o = (size_t)j * pitch + i;
    rho[o] = (Real)r;
    T[o] = (Real)t;
    u[o] = (Real)(fl[1] - fl[3] + fl[5] - fl[6] - fl[7] + fl[8]);
    v[o] = (Real)(fl[5] + fl[2] + fl[6] - fl[7] - fl[4] - fl[8] + (0.5 * neg_gravity * t));
  }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// seeded conduction profile; matches the oracle's orc_init_conduction
template <typename Real>
__global__ void init_conduction_kernel(Real* __restrict__ pops, Real* __restrict__ rho,
                                       Real* __restrict__ u, Real* __restrict__ v,
                                       Real* __restrict__ T, int nx, int ny, int pitch,
                                       size_t plane, double Tup, double Tdown, double T0,
                                       double neg_gravity, uint64_t seed, double noise, int j0,
                                       int ny_total) {
  // rows [j0, j0 + ny) of a domain of ny_total rows (a y-slab; j0 = 0 and
  // ny_total = ny for a whole domain): profile and noise by global node
  const long n = (long)nx * ny;
  const double dT = Tup - Tdown;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const long qg = q + (long)j0 * nx;
    const uint64_t z = splitmix64(seed + ((uint64_t)qg + 1ULL) * 0x9E3779B97F4A7C15ULL);
    const double un = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    const double t = Tdown + dT * (((double)(j0 + j) + 0.5) / (double)ny_total) + noise * (2.0 * un - 1.0);
    double feq[NPOP], geq[NPOP];
    equil_ref(1.0, 0.0, 0.0, feq);
    equil_ref(t, 0.0, 0.0, geq);
    const size_t o = (size_t)j * pitch + i;
    double r = 0.0, tt = 0.0;
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      r = r + feq[k];
      if constexpr (std::is_same<Real, double>::value) {
        pops[(size_t)k * plane + o] = feq[k];
        pops[(size_t)(k + NPOP) * plane + o] = geq[k];
      } else {
        pops[(size_t)k * plane + o] = (float)(feq[k] - w_of(k));
        pops[(size_t)(k + NPOP) * plane + o] = (float)(geq[k] - w_of(k) * T0);
      }
    }
#pragma unroll
    for (int k = 0; k < NPOP; k++) tt = tt + geq[k];
    const double rhoi = 1. / r;
    double fl[NPOP];
#pragma unroll
    for (int k = 0; k < NPOP; k++) fl[k] = feq[k] * rhoi;
    rho[o] = (Real)r;
    T[o] = (Real)tt;
    u[o] = (Real)(fl[1] - fl[3] + fl[5] - fl[6] - fl[7] + fl[8]);
    v[o] = (Real)(fl[5] + fl[2] + fl[6] - fl[7] - fl[4] - fl[8] + (0.5 * neg_gravity * tt));
  }
}

// ------------------------------------------------------------- reductions
// Neumaier-compensated FP64 accumulator
struct KSum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ double val() const { return s + c; }
};

constexpr int RED_BLOCKS = 1184;  // 8 per SM on 148 SMs
constexpr int RED_Q = 3;          // ke, T, vT

template <typename Real>
__global__ void __launch_bounds__(256) stats_partial_kernel(const Real* __restrict__ rho,
                                                            const Real* __restrict__ u,
                                                            const Real* __restrict__ v,
                                                            const Real* __restrict__ T, int nx,
                                                            int ny, int pitch,
                                                            double* __restrict__ part) {
  KSum a[RED_Q];
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const size_t o = (size_t)j * pitch + i;
    const double r = rho[o], uu = u[o], vv = v[o], t = T[o];
    a[0].add(0.5 * r * (uu * uu + vv * vv));
    a[1].add(t);
    a[2].add(vv * t);
  }
  __shared__ double sh[RED_Q][2][256];
  for (int w = 0; w < RED_Q; w++) {
    sh[w][0][threadIdx.x] = a[w].s;
    sh[w][1][threadIdx.x] = a[w].c;
  }
  __syncthreads();
  if (threadIdx.x < RED_Q) {
    KSum b;
    for (int t = 0; t < 256; t++) {
      b.add(sh[threadIdx.x][0][t]);
      b.add(sh[threadIdx.x][1][t]);
    }
    part[(size_t)blockIdx.x * 2 * RED_Q + 2 * threadIdx.x] = b.s;
    part[(size_t)blockIdx.x * 2 * RED_Q + 2 * threadIdx.x + 1] = b.c;
  }
}

// one block: every thread folds a strided share of the block partials, then
// thread 0 folds the per-thread results (all compensated)
__global__ void __launch_bounds__(256) stats_final_kernel(const double* __restrict__ part,
                                                          int nblocks, double* __restrict__ out) {
  __shared__ double sh[RED_Q][2][256];
  KSum a[RED_Q];
  for (int k = threadIdx.x; k < nblocks; k += blockDim.x)
    for (int q = 0; q < RED_Q; q++) {
      a[q].add(part[(size_t)k * 2 * RED_Q + 2 * q]);
      a[q].add(part[(size_t)k * 2 * RED_Q + 2 * q + 1]);
    }
  for (int q = 0; q < RED_Q; q++) {
    sh[q][0][threadIdx.x] = a[q].s;
    sh[q][1][threadIdx.x] = a[q].c;
  }
  __syncthreads();
  if (threadIdx.x < RED_Q) {
    KSum b;
    for (int t = 0; t < (int)blockDim.x; t++) {
      b.add(sh[threadIdx.x][0][t]);
      b.add(sh[threadIdx.x][1][t]);
    }
    out[threadIdx.x] = b.val();
  }
}

// per-row sums, one block per row
template <typename Real>
__global__ void __launch_bounds__(256) profile_kernel(const Real* __restrict__ rho,
                                                      const Real* __restrict__ u,
                                                      const Real* __restrict__ v,
                                                      const Real* __restrict__ T, int nx, int ny,
                                                      int pitch, const double* __restrict__ Ttop,
                                                      double* __restrict__ out) {
  const int j = blockIdx.x;
  KSum a[8];
  const int jt = (j + 1) % ny;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    const size_t o = (size_t)j * pitch + i, ot = (size_t)jt * pitch + i;
    const double r = rho[o], uu = u[o], vv = v[o], t = T[o];
    // above the top row: the periodic halo row (Ttop: its value without box
    // nudging's 1/2 nud_term, as the reference forms the halo)
    const double tu = (Ttop && j == ny - 1) ? Ttop[i] : (double)T[ot];
    a[0].add(r); a[1].add(uu); a[2].add(vv); a[3].add(uu * uu); a[4].add(vv * vv);
    a[5].add(t); a[6].add(vv * t); a[7].add(tu - t);
  }
  __shared__ double sh[8][2][256];
  for (int w = 0; w < 8; w++) {
    sh[w][0][threadIdx.x] = a[w].s;
    sh[w][1][threadIdx.x] = a[w].c;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    KSum b;
    for (int t = 0; t < (int)blockDim.x; t++) {
      b.add(sh[threadIdx.x][0][t]);
      b.add(sh[threadIdx.x][1][t]);
    }
    out[(size_t)j * 9 + threadIdx.x] = b.val() * (1 / (double)nx);  // (the reference's 1/nx scaling)
  }
}

template <typename Real>
__global__ void finite_kernel(const Real* __restrict__ a, size_t n, unsigned* flags) {
  bool bad = false;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    bad |= !isfinite((double)a[q]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags, DFLAG_NONFINITE);
}

// ------------------------------------------------------------- launchers
static int grid_for(long n) {
  long g = (n + 255) / 256;
  return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

cudaError_t launch_pops_in(const double* h, int layout, void* d, bool fp32, int nx, int ny,
                           int pitch, size_t plane, double base, cudaStream_t s) {
  const int g = grid_for((long)nx * ny);
  if (fp32) pops_in_kernel<float><<<g, 256, 0, s>>>(h, layout, (float*)d, nx, ny, pitch, plane, base);
  else pops_in_kernel<double><<<g, 256, 0, s>>>(h, layout, (double*)d, nx, ny, pitch, plane, base);
  return cudaGetLastError();
}

cudaError_t launch_pops_out(const void* d, int layout, double* h, bool fp32, int nx, int ny,
                            int pitch, size_t plane, double base, cudaStream_t s) {
  const int g = grid_for((long)(nx + 2) * (ny + 2));
  if (fp32) pops_out_kernel<float><<<g, 256, 0, s>>>((const float*)d, layout, h, nx, ny, pitch, plane, base);
  else pops_out_kernel<double><<<g, 256, 0, s>>>((const double*)d, layout, h, nx, ny, pitch, plane, base);
  return cudaGetLastError();
}

cudaError_t launch_units(bool in, const void* src, void* dst, int layout, int npop, bool fp32, int nx, int ny,
                         int pitch, size_t plane, double base, int u0, int u1, cudaStream_t s) {
  const long per = layout == LBRB_LAYOUT_REF_AOS_HALO ? (long)(ny + 2) : (long)nx;
  const int g = grid_for((long)(u1 - u0) * per);
  if (u1 <= u0) return cudaSuccess;
#define LBRB_UNITS(R, NPV)                                                                                   \
  if (in) units_in_kernel<R, NPV><<<g, 256, 0, s>>>((const double*)src, layout, (R*)dst, nx, ny, pitch, plane, \
                                                    base, u0, u1);                                           \
  else units_out_kernel<R, NPV><<<g, 256, 0, s>>>((const R*)src, layout, (double*)dst, nx, ny, pitch, plane,  \
                                                  base, u0, u1);
  if (fp32) {
    if (npop == NPOP) { LBRB_UNITS(float, NPOP) } else { LBRB_UNITS(float, 1) }
  } else {
    if (npop == NPOP) { LBRB_UNITS(double, NPOP) } else { LBRB_UNITS(double, 1) }
  }
#undef LBRB_UNITS
  return cudaGetLastError();
}

cudaError_t launch_scalar_in(const double* h, int layout, void* d, bool fp32, int nx, int ny,
                             int pitch, cudaStream_t s) {
  const int g = grid_for((long)nx * ny);
  if (fp32) scalar_in_kernel<float><<<g, 256, 0, s>>>(h, layout, (float*)d, nx, ny, pitch);
  else scalar_in_kernel<double><<<g, 256, 0, s>>>(h, layout, (double*)d, nx, ny, pitch);
  return cudaGetLastError();
}

cudaError_t launch_scalar_out(const void* d, int layout, double* h, bool fp32, int nx, int ny,
                              int pitch, cudaStream_t s) {
  const int g = grid_for((long)(nx + 2) * (ny + 2));
  if (fp32) scalar_out_kernel<float><<<g, 256, 0, s>>>((const float*)d, layout, h, nx, ny, pitch);
  else scalar_out_kernel<double><<<g, 256, 0, s>>>((const double*)d, layout, h, nx, ny, pitch);
  return cudaGetLastError();
}

cudaError_t launch_force(const void* rho, const void* T, void* F, bool fp32, int nx, int ny,
                         int pitch, double neg_gravity, cudaStream_t s) {
  const int g = grid_for((long)nx * ny);
  if (fp32) force_kernel<float><<<g, 256, 0, s>>>((const float*)rho, (const float*)T, (float*)F, nx, ny, pitch, neg_gravity);
  else force_kernel<double><<<g, 256, 0, s>>>((const double*)rho, (const double*)T, (double*)F, nx, ny, pitch, neg_gravity);
  return cudaGetLastError();
}

cudaError_t launch_moments_from_pre(const double* fpre, const double* gpre, int layout, void* rho,
                                    void* u, void* v, void* T, bool fp32, int nx, int ny, int pitch,
                                    double neg_gravity, cudaStream_t s) {
  const int g = grid_for((long)nx * ny);
  if (fp32)
    moments_from_pre_kernel<float><<<g, 256, 0, s>>>(fpre, gpre, layout, (float*)rho, (float*)u,
                                                     (float*)v, (float*)T, nx, ny, pitch, neg_gravity);
  else
    moments_from_pre_kernel<double><<<g, 256, 0, s>>>(fpre, gpre, layout, (double*)rho, (double*)u,
                                                      (double*)v, (double*)T, nx, ny, pitch, neg_gravity);
  return cudaGetLastError();
}

cudaError_t launch_init_conduction(void* pops, void* rho, void* u, void* v, void* T, bool fp32,
                                   int nx, int ny, int pitch, size_t plane, double Tup,
                                   double Tdown, double T0, double neg_gravity, uint64_t seed,
                                   double noise, int j0, int ny_total, cudaStream_t s) {
  const int g = grid_for((long)nx * ny);
  if (fp32)
    init_conduction_kernel<float><<<g, 256, 0, s>>>((float*)pops, (float*)rho, (float*)u, (float*)v,
                                                    (float*)T, nx, ny, pitch, plane, Tup, Tdown, T0,
                                                    neg_gravity, seed, noise, j0, ny_total);
  else
    init_conduction_kernel<double><<<g, 256, 0, s>>>((double*)pops, (double*)rho, (double*)u,
                                                     (double*)v, (double*)T, nx, ny, pitch, plane,
                                                     Tup, Tdown, T0, neg_gravity, seed, noise, j0,
                                                     ny_total);
  return cudaGetLastError();
}

// y-slab exchange: this slab's top row's upward populations (f2, f5, f6,
// g2, g5, g6) into `up` and its bottom row's downward ones (f4, f7, f8, g4,
// g7, g8) into `down`, each 6 rows of nx values: the neighbours' ghost rows
template <typename Real>
__global__ void slab_pack_kernel(const Real* __restrict__ pops, int nx, int ny, int pitch, size_t plane,
                                 Real* __restrict__ up, Real* __restrict__ down) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;  // 0..5: f then g, three populations each
  if (x >= nx) return;
  const int g = r / 3, m = r % 3;
  const int kup = m == 0 ? 2 : (m == 1 ? 5 : 6), kdn = m == 0 ? 4 : (m == 1 ? 7 : 8);
  const Real* base = pops + (size_t)g * NPOP * plane;
  up[(size_t)r * nx + x] = base[(size_t)kup * plane + (size_t)(ny - 1) * pitch + x];
  down[(size_t)r * nx + x] = base[(size_t)kdn * plane + x];
}

cudaError_t launch_slab_pack(const void* pops, bool fp32, int nx, int ny, int pitch, size_t plane, void* up,
                             void* down, cudaStream_t s) {
  dim3 grid((nx + 127) / 128, 6);
  if (fp32)
    slab_pack_kernel<float><<<grid, 128, 0, s>>>((const float*)pops, nx, ny, pitch, plane, (float*)up,
                                                 (float*)down);
  else
    slab_pack_kernel<double><<<grid, 128, 0, s>>>((const double*)pops, nx, ny, pitch, plane, (double*)up,
                                                  (double*)down);
  return cudaGetLastError();
}

// Ghost blocks of a y-slab for two steps per launch (SLAB_GH2_PLANES planes
// of nx values): the neighbour's boundary row r1 -- its three f and three g
// populations that cross into this slab (the one-step ghost layout), then its
// k = 0, 1, 3 f and g, then its F -- and the three f and three g crossing
// populations of the row r2 beyond it.  `up` goes to the slab above (r1, r2 =
// rows ny-1, ny-2; k = 2, 5, 6 cross), `down` to the slab below (rows 0, 1;
// k = 4, 7, 8).
template <typename Real>
__global__ void slab_pack2_kernel(const Real* __restrict__ pops, const Real* __restrict__ F, int nx, int ny,
                                  int pitch, size_t plane, Real* __restrict__ up, Real* __restrict__ down) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = blockIdx.y;  // 0..18
  if (x >= nx) return;
  auto value = [&](bool upward) -> Real {
    if (p == 12) return F[(size_t)(upward ? ny - 1 : 0) * pitch + x];
    const bool beyond = p >= 13;
    int q = beyond ? p - 13 : p;
    int k;
    if (q < 6) {
      const int m = q % 3;
      k = upward ? (m == 0 ? 2 : (m == 1 ? 5 : 6)) : (m == 0 ? 4 : (m == 1 ? 7 : 8));
    } else {
      q -= 6;
      const int m = q % 3;
      k = m == 0 ? 0 : (m == 1 ? 1 : 3);
    }
    const int g = q / 3;  // 0: f, 1: g
    const int row = upward ? (beyond ? ny - 2 : ny - 1) : (beyond ? 1 : 0);
    return pops[((size_t)g * NPOP + k) * plane + (size_t)row * pitch + x];
  };
  up[(size_t)p * nx + x] = value(true);
  down[(size_t)p * nx + x] = value(false);
}

cudaError_t launch_slab_pack2(const void* pops, const void* F, bool fp32, int nx, int ny, int pitch, size_t plane,
                              void* up, void* down, cudaStream_t s) {
  dim3 grid((nx + 127) / 128, SLAB_GH2_PLANES);
  if (fp32)
    slab_pack2_kernel<float><<<grid, 128, 0, s>>>((const float*)pops, (const float*)F, nx, ny, pitch, plane,
                                                  (float*)up, (float*)down);
  else
    slab_pack2_kernel<double><<<grid, 128, 0, s>>>((const double*)pops, (const double*)F, nx, ny, pitch, plane,
                                                   (double*)up, (double*)down);
  return cudaGetLastError();
}

int red_blocks() { return RED_BLOCKS; }

cudaError_t launch_stats(const void* rho, const void* u, const void* v, const void* T, bool fp32,
                         int nx, int ny, int pitch, double* part, double* out, cudaStream_t s) {
  if (fp32)
    stats_partial_kernel<float><<<RED_BLOCKS, 256, 0, s>>>((const float*)rho, (const float*)u,
                                                           (const float*)v, (const float*)T, nx, ny,
                                                           pitch, part);
  else
    stats_partial_kernel<double><<<RED_BLOCKS, 256, 0, s>>>((const double*)rho, (const double*)u,
                                                            (const double*)v, (const double*)T, nx,
                                                            ny, pitch, part);
  stats_final_kernel<<<1, 256, 0, s>>>(part, RED_BLOCKS, out);
  return cudaGetLastError();
}

cudaError_t launch_profile(const void* rho, const void* u, const void* v, const void* T, bool fp32,
                           int nx, int ny, int pitch, const double* Ttop, double* out, cudaStream_t s) {
  if (fp32)
    profile_kernel<float><<<ny, 256, 0, s>>>((const float*)rho, (const float*)u, (const float*)v,
                                             (const float*)T, nx, ny, pitch, Ttop, out);
  else
    profile_kernel<double><<<ny, 256, 0, s>>>((const double*)rho, (const double*)u, (const double*)v,
                                              (const double*)T, nx, ny, pitch, Ttop, out);
  return cudaGetLastError();
}

cudaError_t launch_finite(const void* a, size_t n, bool fp32, unsigned* flags, cudaStream_t s) {
  const int g = grid_for((long)(n / 4 + 1));
  if (fp32) finite_kernel<float><<<g, 256, 0, s>>>((const float*)a, n, flags);
  else finite_kernel<double><<<g, 256, 0, s>>>((const double*)a, n, flags);
  return cudaGetLastError();
}

}  // namespace lbrb
