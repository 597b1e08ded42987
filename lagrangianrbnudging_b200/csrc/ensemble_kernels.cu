// ensemble_kernels.cu -- kernels that advance many independent runs
// ("members", of uneven grid size and closure) in one launch per phase of the
// time step.  No counterpart in the reference.
//
// Phase A, the fused stream/collide step of every member: a work list of
// equal tiles (member, first row, first column; BS columns x ROWS rows) is
// processed either one block per tile, or by a persistent grid of
// (SMs x resident blocks) walking the list statically (grid stride) or
// dynamically (an atomic tile counter).  A block copies its tile's member
// view into shared memory when the member changes, then runs lb_update_node
// -- the same per-node function as the single-run kernel, so a member's
// result is bit-identical to the same run advanced alone.
// Phase B: every member's particles (one block per 128-particle chunk) and
// the innovation scatter of its bilinear observations.
// Phase C: the nudging apply of every member.
//
// ctr[0] counts the steps of the current lbrb_ensemble_step call (phase A's
// first block increments it; B and C read it to pick observation rows);
// ctr[1] is the dynamic schedule's tile counter (cleared by phase B).
// The three kernels are launched with programmatic dependent launch (also
// inside the ensemble's CUDA graph) and wait for the previous phase before
// touching memory, so each launch overlaps only the previous one's drain.
#include <atomic>

#include "capi_internal.cuh"
#include "ensemble.cuh"
#include "lb_pair.cuh"
#include "nudge_dev.cuh"
#include "particle_dev.cuh"

namespace lbrb {

template <typename Real, int TWALL, int BS, int ROWS, int SCHED, int MINB, typename Off, bool FAST>
__global__ void __launch_bounds__(BS, MINB)
    ens_lb_kernel(const LBView<Real>* __restrict__ views, const int4* __restrict__ items, int nitems,
                  int* __restrict__ ctr) {
  __shared__ LBView<Real> sV;
  __shared__ int s_item[2];
  pdl_wait();
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&ctr[0], 1);
  constexpr int WORDS = (int)(sizeof(LBView<Real>) / sizeof(int));
  static_assert(sizeof(LBView<Real>) % sizeof(int) == 0, "view size");
  int cur_m = -1;
  int it = blockIdx.x;
  int par = 0;
  for (;;) {
    int item;
    if (SCHED == 2) {
      if (threadIdx.x == 0) s_item[par] = atomicAdd(&ctr[1], 1);
      __syncthreads();
      item = s_item[par];
      par ^= 1;
    } else {
      item = it;
      it += gridDim.x;
    }
    if (item >= nitems) break;
    const int4 w = items[item];
    if (w.x != cur_m) {
      __syncthreads();  // every thread is done with the previous member's view
      const int* src = reinterpret_cast<const int*>(views + w.x);
      int* dst = reinterpret_cast<int*>(&sV);
      for (int i = threadIdx.x; i < WORDS; i += BS) dst[i] = src[i];
      __syncthreads();
      cur_m = w.x;
    }
    const int x = w.z + threadIdx.x;
    if (x < sV.nx) {
      const int j1 = min(w.y + ROWS, sV.ny);
      for (int j = w.y; j < j1; j++) lb_update_node<Real, TWALL, false, Off, FAST>(sV, j, x);
    }
    if (SCHED == 0) break;
  }
}

template <typename Real>
__global__ void __launch_bounds__(128)
    ens_aux_kernel(const EnsAux<Real>* __restrict__ aux, const int2* __restrict__ pchunks, int npchunks,
                   const int2* __restrict__ ochunks, int nochunks, int* __restrict__ ctr) {
  pdl_wait();
  if (blockIdx.x == 0 && threadIdx.x == 0) ctr[1] = 0;
  int b = blockIdx.x;
  if (b < npchunks) {
    const int2 c = pchunks[b];
    const EnsAux<Real>& A = aux[c.x];
    const int p = c.y + threadIdx.x;
    if (p < A.P.np) particle_update(A.P, p);
    return;
  }
  b -= npchunks;
  if (b < nochunks) {
    const int2 c = ochunks[b];
    const EnsAux<Real>& A = aux[c.x];
    const int o = c.y + threadIdx.x;
    if (o >= A.nobs) return;
    const double* ob = ens_obs_row(A, ctr[0] - 1);
    obs_scatter_one(A.T, A.nx, A.ny, A.pitch, ob[o], ob[A.nobs + o], ob[2 * A.nobs + o], A.alpha,
                    A.acc, A.dflags);
  }
}

// 4 threads per observation (its cell corners), 128 observations per block
template <typename Real>
__global__ void __launch_bounds__(512)
    ens_apply_kernel(const EnsAux<Real>* __restrict__ aux, const int2* __restrict__ ochunks,
                     const int* __restrict__ ctr) {
  pdl_wait();
  const int2 c = ochunks[blockIdx.x];
  const EnsAux<Real>& A = aux[c.x];
  const int o = c.y + (threadIdx.x >> 2);
  if (o >= A.nobs) return;
  const double* ob = ens_obs_row(A, ctr[0] - 1);
  obs_apply_one(A.g, A.plane, A.nx, A.ny, A.pitch, ob[o], ob[A.nobs + o], threadIdx.x & 3, A.acc);
}

// ------------------------------------------------- two steps per launch
// The member's two step views are copied into shared memory; the ring of
// march_block follows them (dynamic shared memory).  Block 0 counts the two
// steps in ctr[0] (the later phases pick observation rows from it).
template <typename Real, int R, int MINB, bool PRE, typename Off>
__global__ void __launch_bounds__(32 * (R + 1), MINB)
    ens_march_kernel(const LBView<Real>* __restrict__ views1, const LBView<Real>* __restrict__ views2,
                     const int4* __restrict__ items, int* __restrict__ ctr) {
  __shared__ LBView<Real> sV[2];
  extern __shared__ __align__(16) unsigned char ens_march_smem[];
  pdl_wait();
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&ctr[0], 2);
  const int4 w = items[blockIdx.x];  // (member, first column, first row, rows)
  constexpr int WORDS = (int)(sizeof(LBView<Real>) / sizeof(int));
  static_assert(sizeof(LBView<Real>) % sizeof(int) == 0, "view size");
  const int* s1 = reinterpret_cast<const int*>(views1 + w.x);
  const int* s2 = reinterpret_cast<const int*>(views2 + w.x);
  int* d = reinterpret_cast<int*>(sV);
  for (int i = threadIdx.x; i < 2 * WORDS; i += blockDim.x) d[i] = i < WORDS ? s1[i] : s2[i - WORDS];
  __syncthreads();
  march_block<Real, R, PRE, Off>(sV[0], sV[1], w.y, w.z, w.w, ens_march_smem);
}

// The tile variant: work items (member, x0, y0, 0), one TX x TY tile each
// (tile_block), the views as in ens_march_kernel
template <typename Real, int TX, int TY, int NT, int MINB, typename Off>
__global__ void __launch_bounds__(NT, MINB)
    ens_tile_kernel(const LBView<Real>* __restrict__ views1, const LBView<Real>* __restrict__ views2,
                    const int4* __restrict__ items, int* __restrict__ ctr) {
  __shared__ LBView<Real> sV[2];
  extern __shared__ __align__(16) unsigned char ens_tile_smem[];
  pdl_wait();
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&ctr[0], 2);
  const int4 w = items[blockIdx.x];
  constexpr int WORDS = (int)(sizeof(LBView<Real>) / sizeof(int));
  const int* s1 = reinterpret_cast<const int*>(views1 + w.x);
  const int* s2 = reinterpret_cast<const int*>(views2 + w.x);
  int* d = reinterpret_cast<int*>(sV);
  for (int i = threadIdx.x; i < 2 * WORDS; i += NT) d[i] = i < WORDS ? s1[i] : s2[i - WORDS];
  __syncthreads();
  tile_block<Real, TX, TY, NT, Off>(sV[0], sV[1], w.y, w.z, ens_tile_smem);
}

// step n's innovations of the nudged members, before the pair's launch
// (ctr[0] steps of this call done): 4 threads per observation, one per cell
// corner (obs_pre_corner; every lane of a warp takes part)
template <typename Real>
__global__ void __launch_bounds__(4 * ENS_OCHUNK)
    ens_pre_kernel(const LBView<Real>* __restrict__ views1, const EnsAux<Real>* __restrict__ aux1,
                   const int2* __restrict__ ochunks, const int* __restrict__ ctr) {
  pdl_wait();
  const int2 c = ochunks[blockIdx.x];
  const EnsAux<Real>& A = aux1[c.x];
  const int o = c.y + (threadIdx.x >> 2);
  const bool live = o < A.nobs;
  const double* ob = ens_obs_row(A, ctr[0]);
  obs_pre_corner(views1[c.x], live, live ? ob[o] : 0.0, live ? ob[A.nobs + o] : 0.0,
                 live ? ob[2 * A.nobs + o] : 0.0, A.alpha, threadIdx.x & 3, A.acc2, A.nmask, A.dflags);
}

// every member's particles of both steps; step n+1's innovations
template <typename Real>
__global__ void __launch_bounds__(128)
    ens_aux2_kernel(const EnsAux<Real>* __restrict__ aux1, const EnsAux<Real>* __restrict__ aux2,
                    const int2* __restrict__ pchunks, int npchunks, const int2* __restrict__ ochunks, int nochunks,
                    int* __restrict__ ctr) {
  pdl_wait();
  if (blockIdx.x == 0 && threadIdx.x == 0) ctr[1] = 0;
  int b = blockIdx.x;
  if (b < npchunks) {
    const int2 c = pchunks[b];
    const int p = c.y + threadIdx.x;
    if (p < aux1[c.x].P.np) {
      particle_update(aux1[c.x].P, p);
      particle_update(aux2[c.x].P, p);
    }
    return;
  }
  b -= npchunks;
  if (b < nochunks) {
    const int2 c = ochunks[b];
    const EnsAux<Real>& A = aux2[c.x];
    const int o = c.y + threadIdx.x;
    if (o >= A.nobs) return;
    const double* ob = ens_obs_row(A, ctr[0] - 1);
    obs_scatter_one(A.T, A.nx, A.ny, A.pitch, ob[o], ob[A.nobs + o], ob[2 * A.nobs + o], A.alpha, A.acc, A.dflags);
  }
}

// step n+1's nudging apply; step n's sums and mask bits cleared (4 threads
// per observation, its cell corners)
template <typename Real>
__global__ void __launch_bounds__(512)
    ens_apply2_kernel(const EnsAux<Real>* __restrict__ aux1, const EnsAux<Real>* __restrict__ aux2,
                      const int2* __restrict__ ochunks, const int* __restrict__ ctr) {
  pdl_wait();
  const int2 c = ochunks[blockIdx.x];
  const EnsAux<Real>& A = aux2[c.x];
  const int o = c.y + (threadIdx.x >> 2);
  if (o >= A.nobs) return;
  const double* ob = ens_obs_row(A, ctr[0] - 1);
  obs_apply_one(A.g, A.plane, A.nx, A.ny, A.pitch, ob[o], ob[A.nobs + o], threadIdx.x & 3, A.acc);
  const EnsAux<Real>& A1 = aux1[c.x];
  const double* o1 = ens_obs_row(A1, ctr[0] - 2);
  obs_clear_one(A1.nx, A1.ny, A1.pitch, o1[o], o1[A1.nobs + o], threadIdx.x & 3, A1.acc2, A1.nmask);
}

// pair variants 0-2, marching: (rows per group, min blocks per SM, software
// pipelining); 3-4, tiles: (tile columns, tile rows, threads, min blocks per
// SM), as the single runs' pair shapes 6 and 5
constexpr int3 ENS_PAIR_TABLE[ENS_MARCH_VARIANTS] = {{8, 3, 0}, {8, 3, 1}, {6, 4, 1}};
constexpr int4 ENS_TILE_TABLE[ENS_PAIR_VARIANTS - ENS_MARCH_VARIANTS] = {{32, 8, 256, 5}, {30, 8, 320, 3}};
int ens_pair_rows(int variant) {
  return variant < ENS_MARCH_VARIANTS ? ENS_PAIR_TABLE[variant].x : ENS_TILE_TABLE[variant - ENS_MARCH_VARIANTS].y;
}
int ens_pair_tile_cols(int variant) {
  return variant < ENS_MARCH_VARIANTS ? 0 : ENS_TILE_TABLE[variant - ENS_MARCH_VARIANTS].x;
}

template <typename Real, int R, int MINB, bool PRE, typename Off>
static cudaError_t ens_march_launch(const void* v1, const void* v2, const int4* items, int nitems, int* ctr,
                                    cudaStream_t s) {
  constexpr int MB = std::is_same<Real, double>::value ? (MINB + 1) / 2 : MINB;
  auto k = ens_march_kernel<Real, R, MB, PRE, Off>;
  constexpr size_t smem = march_smem_bytes<Real, R>();
  static std::atomic<unsigned long long> attr_set{0};
  const cudaError_t e = smem_limit_once((const void*)k, smem, attr_set);
  if (e != cudaSuccess) return e;
  if (nitems <= 0) return cudaSuccess;
  return launch_k(k, nitems, 32 * (R + 1), smem, s, true, (const LBView<Real>*)v1, (const LBView<Real>*)v2,
                  items, ctr);
}

template <typename Real, int TX, int TY, int NT, int MINB, typename Off>
static cudaError_t ens_tile_launch(const void* v1, const void* v2, const int4* items, int nitems, int* ctr,
                                   cudaStream_t s) {
  constexpr int MB = std::is_same<Real, double>::value ? (MINB + 1) / 2 : MINB;
  auto k = ens_tile_kernel<Real, TX, TY, NT, MB, Off>;
  constexpr size_t smem = tile_smem_bytes<Real, TX, TY>();
  static std::atomic<unsigned long long> attr_set{0};
  const cudaError_t e = smem_limit_once((const void*)k, smem, attr_set);
  if (e != cudaSuccess) return e;
  if (nitems <= 0) return cudaSuccess;
  return launch_k(k, nitems, NT, smem, s, true, (const LBView<Real>*)v1, (const LBView<Real>*)v2, items, ctr);
}

template <typename Real, typename Off>
static cudaError_t ens_march_dispatch(int variant, const void* v1, const void* v2, const int4* items, int nitems,
                                      int* ctr, cudaStream_t s) {
  static_assert(ENS_PAIR_VARIANTS == 5, "pair variants");
  switch (variant) {
    case 1: return ens_march_launch<Real, 8, 3, true, Off>(v1, v2, items, nitems, ctr, s);
    case 2: return ens_march_launch<Real, 6, 4, true, Off>(v1, v2, items, nitems, ctr, s);
    case 3: return ens_tile_launch<Real, 32, 8, 256, 5, Off>(v1, v2, items, nitems, ctr, s);
    case 4: return ens_tile_launch<Real, 30, 8, 320, 3, Off>(v1, v2, items, nitems, ctr, s);
    default: return ens_march_launch<Real, 8, 3, false, Off>(v1, v2, items, nitems, ctr, s);
  }
}

cudaError_t launch_ens_march(bool f32, bool off32, int variant, const void* views1, const void* views2,
                             const int4* items, int nitems, int* ctr, cudaStream_t s) {
  if (f32)
    return off32 ? ens_march_dispatch<float, uint32_t>(variant, views1, views2, items, nitems, ctr, s)
                 : ens_march_dispatch<float, size_t>(variant, views1, views2, items, nitems, ctr, s);
  return off32 ? ens_march_dispatch<double, uint32_t>(variant, views1, views2, items, nitems, ctr, s)
               : ens_march_dispatch<double, size_t>(variant, views1, views2, items, nitems, ctr, s);
}

cudaError_t launch_ens_pre(bool f32, const void* views1, const void* aux1, const int2* ochunks, int nochunks,
                           const int* ctr, cudaStream_t s) {
  if (nochunks <= 0) return cudaSuccess;
  if (f32)
    return launch_k(ens_pre_kernel<float>, nochunks, 4 * ENS_OCHUNK, 0, s, true, (const LBView<float>*)views1,
                    (const EnsAux<float>*)aux1, ochunks, ctr);
  return launch_k(ens_pre_kernel<double>, nochunks, 4 * ENS_OCHUNK, 0, s, true, (const LBView<double>*)views1,
                  (const EnsAux<double>*)aux1, ochunks, ctr);
}

cudaError_t launch_ens_aux2(bool f32, const void* aux1, const void* aux2, const int2* pchunks, int npchunks,
                            const int2* ochunks, int nochunks, int* ctr, cudaStream_t s) {
  const int g = npchunks + nochunks;
  if (g <= 0) return cudaSuccess;
  if (f32)
    return launch_k(ens_aux2_kernel<float>, g, 128, 0, s, true, (const EnsAux<float>*)aux1,
                    (const EnsAux<float>*)aux2, pchunks, npchunks, ochunks, nochunks, ctr);
  return launch_k(ens_aux2_kernel<double>, g, 128, 0, s, true, (const EnsAux<double>*)aux1,
                  (const EnsAux<double>*)aux2, pchunks, npchunks, ochunks, nochunks, ctr);
}

cudaError_t launch_ens_apply2(bool f32, const void* aux1, const void* aux2, const int2* ochunks, int nochunks,
                              const int* ctr, cudaStream_t s) {
  if (nochunks <= 0) return cudaSuccess;
  if (f32)
    return launch_k(ens_apply2_kernel<float>, nochunks, 4 * ENS_OCHUNK, 0, s, true, (const EnsAux<float>*)aux1,
                    (const EnsAux<float>*)aux2, ochunks, ctr);
  return launch_k(ens_apply2_kernel<double>, nochunks, 4 * ENS_OCHUNK, 0, s, true, (const EnsAux<double>*)aux1,
                  (const EnsAux<double>*)aux2, ochunks, ctr);
}

// ------------------------------------------------------------ variants
// (threads per tile row, rows per tile, schedule, min blocks per SM)
template <typename Real, int TWALL, int BS, int ROWS, int SCHED, int MINB, typename Off, bool FAST>
static cudaError_t ens_lb_launch(const LBView<Real>* views, const int4* items, int nitems, int* ctr,
                                 int nsm, cudaStream_t s) {
  auto k = ens_lb_kernel<Real, TWALL, BS, ROWS, SCHED, MINB, Off, FAST>;
  int grid = nitems;
  if (SCHED != 0) {
    // resident blocks per SM of this variant, queried once (outside any
    // stream capture: the first launch of a variant is a tuning or direct one)
    static std::atomic<int> per_cached[MAX_DEVICES] = {};  // one entry per device ordinal
    int per = 0;
    const cudaError_t e = occupancy_once((const void*)k, BS, 0, per_cached, &per);
    if (e != cudaSuccess) return e;
    grid = std::max(1, std::min(nitems, per * nsm));
  }
  if (nitems <= 0) return cudaSuccess;
  return launch_k(k, grid, BS, 0, s, true, views, items, nitems, ctr);
}

// (threads per tile row, rows per tile, schedule, min blocks per SM, pull
// form: 1 interior rows without wall logic + 32-bit offsets, 0 general)
#define ENS_VARIANTS(X)    \
  X(0, 128, 1, 0, 8, 1)    \
  X(1, 128, 2, 0, 8, 1)    \
  X(2, 128, 1, 0, 6, 1)    \
  X(3, 128, 2, 1, 8, 1)    \
  X(4, 128, 4, 1, 8, 1)    \
  X(5, 128, 2, 2, 8, 1)    \
  X(6, 256, 1, 0, 4, 1)    \
  X(7, 256, 2, 1, 4, 1)    \
  X(8, 128, 1, 0, 6, 0)    \
  X(9, 128, 2, 0, 6, 0)    \
  X(10, 256, 1, 0, 3, 0)   \
  X(11, 128, 2, 1, 6, 0)

const EnsVariant ENS_TABLE[] = {
#define X(i, bs, rows, sched, minb, fast) {bs, rows, sched, minb, fast},
    ENS_VARIANTS(X)
#undef X
};
const int ENS_NVARIANTS = sizeof(ENS_TABLE) / sizeof(ENS_TABLE[0]);

template <typename Real, int TWALL, typename Off>
static cudaError_t ens_lb_dispatch(int variant, const LBView<Real>* views, const int4* items,
                                   int nitems, int* ctr, int nsm, cudaStream_t s) {
  switch (variant) {
#define X(i, bs, rows, sched, minb, fast)                                                       \
  case i:                                                                                       \
    if (fast && std::is_same<Off, uint32_t>::value)                                             \
      return ens_lb_launch<Real, TWALL, bs, rows, sched, minb, uint32_t, true>(views, items, nitems, ctr, nsm, s); \
    return ens_lb_launch<Real, TWALL, bs, rows, sched, minb, size_t, (bool)fast>(views, items, nitems, ctr, nsm, s);
    ENS_VARIANTS(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
}

template <typename Real>
static cudaError_t ens_lb_walls(bool off32, int twall, int variant, const LBView<Real>* views,
                                const int4* items, int nitems, int* ctr, int nsm, cudaStream_t s) {
  if (twall == LBRB_TWALL_DIRICHLET)
    return off32 ? ens_lb_dispatch<Real, LBRB_TWALL_DIRICHLET, uint32_t>(variant, views, items, nitems, ctr, nsm, s)
                 : ens_lb_dispatch<Real, LBRB_TWALL_DIRICHLET, size_t>(variant, views, items, nitems, ctr, nsm, s);
  return off32 ? ens_lb_dispatch<Real, LBRB_TWALL_ADIABATIC, uint32_t>(variant, views, items, nitems, ctr, nsm, s)
               : ens_lb_dispatch<Real, LBRB_TWALL_ADIABATIC, size_t>(variant, views, items, nitems, ctr, nsm, s);
}

cudaError_t launch_ens_lb(bool f32, bool off32, int twall, int variant, const void* views,
                          const int4* items, int nitems, int* ctr, int nsm, cudaStream_t s) {
  if (f32) return ens_lb_walls<float>(off32, twall, variant, (const LBView<float>*)views, items, nitems, ctr, nsm, s);
  return ens_lb_walls<double>(off32, twall, variant, (const LBView<double>*)views, items, nitems, ctr, nsm, s);
}

cudaError_t launch_ens_aux(bool f32, const void* aux, const int2* pchunks, int npchunks,
                           const int2* ochunks, int nochunks, int* ctr, cudaStream_t s) {
  const int grid = std::max(1, npchunks + nochunks);
  if (f32)
    return launch_k(ens_aux_kernel<float>, grid, 128, 0, s, true, (const EnsAux<float>*)aux, pchunks, npchunks,
                    ochunks, nochunks, ctr);
  return launch_k(ens_aux_kernel<double>, grid, 128, 0, s, true, (const EnsAux<double>*)aux, pchunks, npchunks,
                  ochunks, nochunks, ctr);
}

cudaError_t launch_ens_apply(bool f32, const void* aux, const int2* ochunks, int nochunks, const int* ctr,
                             cudaStream_t s) {
  if (nochunks <= 0) return cudaSuccess;
  if (f32) return launch_k(ens_apply_kernel<float>, nochunks, 512, 0, s, true, (const EnsAux<float>*)aux, ochunks, ctr);
  return launch_k(ens_apply_kernel<double>, nochunks, 512, 0, s, true, (const EnsAux<double>*)aux, ochunks, ctr);
}

}  // namespace lbrb
