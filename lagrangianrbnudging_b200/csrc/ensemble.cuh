// ensemble.cuh -- per-member views of the ensemble kernels and their launchers.
#pragma once

#include "lbrb_internal.cuh"
#include "particle_dev.cuh"

namespace lbrb {

// everything phases B and C need of one member for one step
template <typename Real>
struct EnsAux {
  PView<Real> P;            // particles of the step (np = 0: none)
  const Real* T;            // T of the new state (innovations)
  Real* g;                  // g planes of the new state (nudging apply)
  size_t plane;
  int nx, ny, pitch;
  const double* obs;        // bilinear observations [rows][3][nobs], or null
  int nobs, obs_first, obs_nsteps, obs_cycle, istep0;
  double alpha;
  unsigned long long* acc;  // fixed-point innovation sums
  unsigned* dflags;
  // two steps per launch (the first step's view of a pair): the sums formed
  // before the launch and their node mask
  unsigned long long* acc2;
  unsigned* nmask;
};

// observation row of the member's step istep0 + t + 1 (t counts the steps of
// the current call from 0); coverage is checked on the host before launch
template <typename Real>
__device__ __forceinline__ const double* ens_obs_row(const EnsAux<Real>& A, int t) {
  int row = A.istep0 + t + 1 - A.obs_first;
  if (A.obs_cycle) row %= A.obs_nsteps;
  return A.obs + (size_t)row * 3 * A.nobs;
}

// a launch variant of phase A: threads per tile row, rows per tile,
// schedule (0 one block per tile, 1 persistent grid-stride, 2 persistent
// atomic counter), min blocks per SM of the launch bounds, pull form (1
// interior rows without wall logic and 32-bit offsets where they fit, 0 the
// general pull with 64-bit offsets)
struct EnsVariant { int bs, rows, sched, minb, fast; };
extern const EnsVariant ENS_TABLE[];
extern const int ENS_NVARIANTS;

constexpr int ENS_PCHUNK = 128;  // particles per block of phase B
constexpr int ENS_OCHUNK = 128;  // observations per block of phases B and C

// off32: every member's population buffer holds fewer than 2^32 elements
cudaError_t launch_ens_lb(bool f32, bool off32, int twall, int variant, const void* views,
                          const int4* items, int nitems, int* ctr, int nsm, cudaStream_t s);
cudaError_t launch_ens_aux(bool f32, const void* aux, const int2* pchunks, int npchunks,
                           const int2* ochunks, int nochunks, int* ctr, cudaStream_t s);
cudaError_t launch_ens_apply(bool f32, const void* aux, const int2* ochunks, int nochunks,
                             const int* ctr, cudaStream_t s);

// Two steps per launch for every member (ensemble_kernels.cu).  A pair's
// launches: ens_pre (step n's innovations of the nudged members, formed from
// T^n before the launch), ens_march (the marching two-step kernel over work
// items (member, first column, first row, rows); views1/views2 hold each
// member's step n and step n+1 views), ens_aux2 (every member's particles of
// both steps; the innovations of step n+1), ens_apply2 (the nudging apply of
// step n+1 and the clearing of step n's sums).  aux1/aux2: EnsAux of steps n
// and n+1.  Pair variants: [0, ENS_MARCH_VARIANTS) march (items: a strip of
// 32 columns and a chunk of rows), the rest take tiles (ens_tile, items: a
// tile's first column and row; ens_pair_tile_cols columns).
constexpr int ENS_MARCH_VARIANTS = 3;
constexpr int ENS_PAIR_VARIANTS = 5;
int ens_pair_rows(int variant);  // rows per marching group, or per tile
int ens_pair_tile_cols(int variant);  // 0: a marching variant
cudaError_t launch_ens_pre(bool f32, const void* views1, const void* aux1, const int2* ochunks, int nochunks,
                           const int* ctr, cudaStream_t s);
cudaError_t launch_ens_march(bool f32, bool off32, int variant, const void* views1, const void* views2,
                             const int4* items, int nitems, int* ctr, cudaStream_t s);
cudaError_t launch_ens_aux2(bool f32, const void* aux1, const void* aux2, const int2* pchunks, int npchunks,
                            const int2* ochunks, int nochunks, int* ctr, cudaStream_t s);
cudaError_t launch_ens_apply2(bool f32, const void* aux1, const void* aux2, const int2* ochunks, int nochunks,
                              const int* ctr, cudaStream_t s);

}  // namespace lbrb
