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
#include "lb_node.cuh"
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
