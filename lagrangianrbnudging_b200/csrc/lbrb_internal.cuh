// lbrb_internal.cuh -- shared device helpers and the run handle.
//
// Device layout (one whole domain, no halo):
//   populations  pop[k][j][x]  with row pitch `pitch` (elements, multiple of 32)
//                plane = ny * pitch; f and g each hold 9 planes; two copies
//                (ping-pong: the step reads one and writes the other)
//   scalars      s[j][x] with the same pitch
// Reference node (i, j) (1-based, temppart_dump.c idx = j + (NY+2)*i) is
// device node (x = i-1, y = j-1).  The reference's periodic halos (pbc,
// communication) become index wrap.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <type_traits>

#include "../../include/lbrb.h"

namespace lbrb {

constexpr int NPOP = 9;
constexpr int WARP = 32;

// D2Q9 as the reference's dellar() builds it (temppart_dump.c:1363-1401);
// cy[3] = -cy[1] and cx[4] = -cx[2] are negative zeros there.
__host__ __device__ constexpr double w_of(int k) {
  return k == 0 ? 16. / 36. : (k < 5 ? 4. / 36. : 1. / 36.);
}
__host__ __device__ constexpr int icx(int k) {
  return (k == 1 || k == 5 || k == 8) ? 1 : ((k == 3 || k == 6 || k == 7) ? -1 : 0);
}
__host__ __device__ constexpr int icy(int k) {
  return (k == 2 || k == 5 || k == 6) ? 1 : ((k == 4 || k == 7 || k == 8) ? -1 : 0);
}
__host__ __device__ constexpr double dcx(int k) {
  return k == 4 ? -0.0 : (double)icx(k);
}
__host__ __device__ constexpr double dcy(int k) {
  return k == 3 ? -0.0 : (double)icy(k);
}
__host__ __device__ constexpr int opp(int k) {
  return k == 0 ? 0 : (k <= 4 ? ((k + 1) % 4) + 1 : ((k - 5 + 2) % 4) + 5);
}
static_assert(opp(1) == 3 && opp(2) == 4 && opp(3) == 1 && opp(4) == 2, "opp");
static_assert(opp(5) == 7 && opp(6) == 8 && opp(7) == 5 && opp(8) == 6, "opp");

constexpr double CS2 = 1.0 / 3.0;

// equilif / equilig in the reference's operation order
// (temppart_dump.c:1097-1180): r1 is rho for f and T for g.
__device__ __forceinline__ void equil_ref(double r1, double u, double v, double feq[NPOP]) {
  double usq = u * u;
  double vsq = v * v;
  double sumsq = (usq + vsq) / (2. * CS2);
  double sumsq2 = sumsq * (1. - CS2) / CS2;
  double u2 = usq / (2. / 9.);
  double v2 = vsq / (2. / 9.);
  double ui = u / CS2;
  double vi = v / CS2;
  double uv = ui * vi;
  feq[0] = r1 * w_of(0) * (1. - sumsq);
  feq[1] = r1 * w_of(1) * (1. - sumsq + u2 + ui);
  feq[2] = r1 * w_of(2) * (1. - sumsq + v2 + vi);
  feq[3] = r1 * w_of(3) * (1. - sumsq + u2 - ui);
  feq[4] = r1 * w_of(4) * (1. - sumsq + v2 - vi);
  feq[5] = r1 * w_of(5) * (1. + sumsq2 + ui + vi + uv);
  feq[6] = r1 * w_of(6) * (1. + sumsq2 - ui + vi - uv);
  feq[7] = r1 * w_of(7) * (1. + sumsq2 - ui - vi + uv);
  feq[8] = r1 * w_of(8) * (1. + sumsq2 + ui - vi - uv);
}


// device error flags (bit mask in Handle::dflags)
enum : unsigned {
  DFLAG_RANGE = 1u,      // a particle or observation left the addressable range
  DFLAG_NONFINITE = 2u,  // NaN / Inf seen
  DFLAG_BOXCAP = 4u,     // box nudging cell list inconsistent
};

// ---------------------------------------------------------------- vectors
template <typename Real>
struct Vec;
template <>
struct Vec<double> {
  static constexpr int N = 2;
  using T = double2;
  __device__ static inline void unpack(const T& v, double* o) { o[0] = v.x; o[1] = v.y; }
  __device__ static inline T pack(const double* a) { return make_double2(a[0], a[1]); }
};
template <>
struct Vec<float> {
  static constexpr int N = 4;
  using T = float4;
  __device__ static inline void unpack(const T& v, float* o) {
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
  __device__ static inline T pack(const float* a) { return make_float4(a[0], a[1], a[2], a[3]); }
};

template <typename Real>
__device__ __forceinline__ void vload(const Real* __restrict__ p, Real* o) {
  using V = Vec<Real>;
  typename V::T v = __ldcs(reinterpret_cast<const typename V::T*>(p));
  V::unpack(v, o);
}
template <typename Real>
__device__ __forceinline__ void vstore(Real* __restrict__ p, const Real* a) {
  using V = Vec<Real>;
  __stcs(reinterpret_cast<typename V::T*>(p), V::pack(a));
}

// Load VEC consecutive values of `row` pulled along x by `cx`:
//   out[m] = row[(x0 + m - cx) mod nx].
// Lanes own aligned chunks [x0, x0+VEC); the one value that lies in the
// neighbour lane's chunk comes by shuffle, and lanes at the warp or row edge
// fetch it with a scalar load (periodic wrap).
template <int CX, typename Real>
__device__ __forceinline__ void load_pull_x(const Real* __restrict__ row, int x0, int lane,
                                            int nx, Real* out) {
  constexpr int N = Vec<Real>::N;
  Real v[N];
  vload<Real>(row + x0, v);
  if (CX == 0) {
#pragma unroll
    for (int m = 0; m < N; m++) out[m] = v[m];
  } else if (CX == 1) {
    Real left = __shfl_up_sync(0xffffffffu, v[N - 1], 1);
    if (lane == 0 || x0 == 0) left = __ldcs(row + (x0 == 0 ? nx - 1 : x0 - 1));
    out[0] = left;
#pragma unroll
    for (int m = 1; m < N; m++) out[m] = v[m - 1];
  } else {
    Real right = __shfl_down_sync(0xffffffffu, v[0], 1);
    if (lane == WARP - 1 || x0 + N >= nx) right = __ldcs(row + (x0 + N >= nx ? 0 : x0 + N));
#pragma unroll
    for (int m = 0; m < N - 1; m++) out[m] = v[m + 1];
    out[N - 1] = right;
  }
}

// ------------------------------------------------------------ kernel views
template <typename Real>
struct LBView {
  const Real* __restrict__ fsrc;
  const Real* __restrict__ gsrc;
  Real* __restrict__ fdst;
  Real* __restrict__ gdst;
  Real* __restrict__ F;    // buoyancy F_y of the NEXT step; read then rewritten in place
  Real* __restrict__ rho;
  Real* __restrict__ u;
  Real* __restrict__ v;
  Real* __restrict__ T;
  int nx, ny, pitch;
  size_t plane;
  double omega, omegag;    // 1/relax, 1/relaxg
  double neg_gravity;      // -gravity
  double Tup, Tdown, T0;
  // reference box nudging
  const int* __restrict__ nudge_vol;
  const double* __restrict__ tempreadint;
  double* __restrict__ nud_term;
  double alpha;
  int write_uv, write_rt;
  int chunks_per_row;
  long ntasks;
};

// --------------------------------------------------------------- handle
struct Handle {
  lbrb_params p{};
  std::string err;
  int dev = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;
  cudaStream_t own_stream = nullptr;  // the handle's own stream (stream may be the caller's)
  cudaEvent_t join_ev = nullptr;      // last record copy, joined back into `stream`
  bool join_pending = false;
  // per-kernel timing: event pairs per class, summed on request
  bool timing = false;
  int istep = 0;  // steps done (the reference's istep of the last step)
  int pitch = 0;
  size_t plane = 0;   // ny * pitch
  size_t esize = 8;   // bytes per population value
  // populations: pops[buf] holds f (9 planes) then g (9 planes)
  void* pops[2] = {nullptr, nullptr};
  int cur = 0;        // buffer holding the current post-collision state
  // scalar fields (Real)
  void* F = nullptr;
  void* rho = nullptr;
  void* uv[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [slot][u/v]
  int uvcur = 0;      // slot of the current u, v (the other holds u^{n-1})
  void* T = nullptr;
  bool moments_valid = false;
  // particles (FP64)
  int np = 0;
  double* px = nullptr;  // [9][np]: x y u v xo yo uo vo invtau
  int* pid = nullptr;
  int* ptype = nullptr;
  bool particles_set = false;
  // records
  int nrec_fields = LBRB_REC_NBASIC;
  double* d_ring = nullptr;      // [slots][fields][np]
  double* h_ring = nullptr;      // pinned mirror
  int* h_ring_step = nullptr;
  cudaEvent_t* ring_ev = nullptr;
  long rec_head = 0, rec_tail = 0;  // produced / drained counts
  // box nudging (FP64)
  int nobs = 0;
  double* nb = nullptr;     // per-observation doubles, see nudge.cu
  int* nbi = nullptr;       // per-observation ints
  int* nudge_vol = nullptr;
  double* tempreadint = nullptr;
  double* nud_term = nullptr;
  int* cell_count = nullptr;
  int* cell_start = nullptr;
  int* cell_fill = nullptr;
  int* cell_dirty = nullptr;
  int* cell_items = nullptr;
  long cell_items_cap = 0;
  int ncx = 0, ncy = 0;
  bool nudge_init_done = false, nudge_file_loaded = false;
  int* h_chk = nullptr;     // host copy of chk_id (ids matched on the host)
  int* h_oid = nullptr;     // host copy of the initial-order ids
  // bilinear nudging
  double* obs = nullptr;    // [nsteps][3][nobs]
  int obs_first = 0, obs_nsteps = 0, obs_cap_steps = 0;
  long long* acc = nullptr;
  // scratch / staging
  void* staging = nullptr;
  size_t staging_bytes = 0;
  double* red = nullptr;    // reduction partials
  unsigned* dflags = nullptr;
  unsigned* h_flags = nullptr;
};

}  // namespace lbrb
