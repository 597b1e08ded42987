// lb_kernels.cu -- the fused pull stream + walls + buoyancy + moments +
// collision kernel: one launch per time step, both populations f and g.
//
// Reference semantics (temppart_dump.c, Trajectories):
//   stream          :781-854   f_k(x) <- f_k(x - c_k) for k = 1..8, same for g
//   force           :744-755   F_y = -gravity * rho^{n-1} * T^{n-1}, F_x = 0
//   f walls         :763-777, 859-894   half-way bounce-back from the
//                              pre-stream wall row: f2,f5,f6(1) <- f4,f7,f8(1);
//                              f4,f7,f8(NY) <- f2,f5,f6(NY)
//   g walls (T)     :896-921   g_in = -g_opp(post-stream) + 2 w T_wall
//   g walls (N)     tempvel_nudge.c:684-702, 783-962: rows 1 and NY hold
//                              pre-stream copies of rows 2 and NY-1 and are
//                              not streamed into
//   moments         :957-987 (tempvel_nudge.c:1069-1102 adds 1/2 nud_term)
//   collision       :1097-1180, 1314-1341 (tempvel_nudge.c:1917-1945 nudged g)
//
// Two arithmetic forms:
//   Real = double: the reference's operation order exactly (built with
//     --fmad=false), bit-identical to the reference on x86-64.
//   Real = float: populations stored as deviations from their weights
//     (f_k - w_k rho0, g_k - w_k T0), collision in FP32.
//
// Mapping: one node per thread, a block covers BS consecutive nodes of one
// row (wall handling is block-uniform).  Every population is one plain
// coalesced load at its pull address: x-1 and x+1 fall in the same 128-byte
// lines as the neighbouring threads' loads, so L1/L2 absorb the shift and
// DRAM reads each value once.  All 18 loads are independent and issue back to
// back; the small register budget keeps many warps per SM and enough bytes in
// flight for HBM3e.  The buoyancy F of the next step is written to the other
// of two buffers, so a launch is a pure function of its sources: the launch
// shape (block size, blocks per SM) is picked by timing the candidates on the
// run's own grid (tune_lb).
#include <cstdlib>
#include <type_traits>

#include "lb_node.cuh"

namespace lbrb {

// post-stream populations only (walls applied): dumpfpre/dumpgpre
template <typename Real, int TWALL>
__global__ void __launch_bounds__(128) lb_pull_kernel(const LBView<Real> V, Real* __restrict__ outf,
                                                      Real* __restrict__ outg) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (x >= V.nx) return;
  Real fs[NPOP], gs[NPOP];
  pull_node<Real, TWALL, size_t>(V, j, x, fs, gs);
  if (TWALL == LBRB_TWALL_DIRICHLET) dirichlet_walls(V, j, gs);
  const size_t o = (size_t)j * V.pitch + x;
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    outf[(size_t)k * V.plane + o] = fs[k];
    outg[(size_t)k * V.plane + o] = gs[k];
  }
}

template <typename Real, int TWALL, bool REFNUDGE, int BS, int MINB, typename Off, bool FAST>
__global__ void __launch_bounds__(BS, MINB) lb_node_kernel(const LBView<Real> V) {
  pdl_wait();
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (x >= V.nx) return;
  lb_update_node<Real, TWALL, REFNUDGE, Off, FAST>(V, j, x);
}

// --------------------------------------------------------------- launch
// launch shapes tried by tune_lb: (threads per block, min blocks per SM,
// pull form: 1 = interior rows without wall logic and 32-bit offsets where
// they fit, 0 = the general pull with 64-bit offsets on every row)
struct Shape { int bs, minb, fast; };
constexpr Shape SHAPES[] = {{256, 1, 1}, {256, 2, 1}, {256, 3, 1}, {128, 4, 1}, {128, 6, 1},
                            {512, 1, 1}, {512, 2, 1}, {256, 3, 0}, {128, 4, 0}, {128, 6, 0}};
constexpr int NSHAPES = sizeof(SHAPES) / sizeof(SHAPES[0]);

template <typename Real, int TWALL, bool REFNUDGE, int BS, int MINB, bool FAST>
static cudaError_t launch_shape(const LBView<Real>& V, cudaStream_t s, bool pdl) {
  dim3 grid((V.nx + BS - 1) / BS, V.ny);
  if (FAST && off32_ok(V.plane))
    return launch_k(lb_node_kernel<Real, TWALL, REFNUDGE, BS, MINB, uint32_t, true>, grid, BS, 0, s, pdl, V);
  return launch_k(lb_node_kernel<Real, TWALL, REFNUDGE, BS, MINB, size_t, FAST>, grid, BS, 0, s, pdl, V);
}

template <typename Real, int TWALL, bool REFNUDGE>
static cudaError_t launch_lb(const LBView<Real>& V, int shape, cudaStream_t s, bool pdl) {
  switch (shape) {
    case 1: return launch_shape<Real, TWALL, REFNUDGE, 256, 2, true>(V, s, pdl);
    case 2: return launch_shape<Real, TWALL, REFNUDGE, 256, 3, true>(V, s, pdl);
    case 3: return launch_shape<Real, TWALL, REFNUDGE, 128, 4, true>(V, s, pdl);
    case 4: return launch_shape<Real, TWALL, REFNUDGE, 128, 6, true>(V, s, pdl);
    case 5: return launch_shape<Real, TWALL, REFNUDGE, 512, 1, true>(V, s, pdl);
    case 6: return launch_shape<Real, TWALL, REFNUDGE, 512, 2, true>(V, s, pdl);
    case 7: return launch_shape<Real, TWALL, REFNUDGE, 256, 3, false>(V, s, pdl);
    case 8: return launch_shape<Real, TWALL, REFNUDGE, 128, 4, false>(V, s, pdl);
    case 9: return launch_shape<Real, TWALL, REFNUDGE, 128, 6, false>(V, s, pdl);
    default: return launch_shape<Real, TWALL, REFNUDGE, 256, 1, true>(V, s, pdl);
  }
}

cudaError_t launch_lb_fp64(const LBView<double>& V, int twall, bool refnudge, int shape,
                           cudaStream_t s, bool pdl) {
  if (twall == LBRB_TWALL_DIRICHLET)
    return refnudge ? launch_lb<double, LBRB_TWALL_DIRICHLET, true>(V, shape, s, pdl)
                    : launch_lb<double, LBRB_TWALL_DIRICHLET, false>(V, shape, s, pdl);
  return refnudge ? launch_lb<double, LBRB_TWALL_ADIABATIC, true>(V, shape, s, pdl)
                  : launch_lb<double, LBRB_TWALL_ADIABATIC, false>(V, shape, s, pdl);
}

cudaError_t launch_lb_fp32(const LBView<float>& V, int twall, int shape, cudaStream_t s, bool pdl) {
  if (twall == LBRB_TWALL_DIRICHLET) return launch_lb<float, LBRB_TWALL_DIRICHLET, false>(V, shape, s, pdl);
  return launch_lb<float, LBRB_TWALL_ADIABATIC, false>(V, shape, s, pdl);
}

// Autotuner: time every launch shape on this run's grid (CUDA events, `reps`
// launches after one warm-up launch each) and return the fastest.  A trial
// launch reads the current state and writes only buffers the real step
// overwrites: the other population buffer, the other F buffer and, when the
// caller's view stores u, v (runs with particles), the u, v slot of the next
// step; rho and T are not written.  Box-nudged FP64 steps update nud_term in
// place and are not tuned (shape 0).
template <typename Real>
static int tune(const LBView<Real>& Vin, int twall, bool refnudge, cudaStream_t s, int reps,
                float* best_ms) {
  LBView<Real> V = Vin;  // u, v stores as the caller's view has them
  V.write_rt = 0;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int best = 0;
  float bt = 1e30f;
  for (int sh = 0; sh < NSHAPES; sh++) {
    cudaError_t e;
    auto go = [&]() {
      if constexpr (std::is_same<Real, double>::value) return launch_lb_fp64(V, twall, refnudge, sh, s, false);
      else return launch_lb_fp32(V, twall, sh, s, false);
    };
    e = go();
    if (e != cudaSuccess) { cudaGetLastError(); continue; }
    cudaEventRecord(a, s);
    for (int r = 0; r < reps; r++) go();
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < bt) { bt = ms; best = sh; }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (best_ms) *best_ms = bt / reps;
  return best;
}

template <typename Real>
static cudaError_t launch_pull_t(const LBView<Real>& V, int twall, void* outf, void* outg,
                                 cudaStream_t s) {
  dim3 grid((V.nx + 127) / 128, V.ny);
  if (twall == LBRB_TWALL_DIRICHLET)
    lb_pull_kernel<Real, LBRB_TWALL_DIRICHLET><<<grid, 128, 0, s>>>(V, (Real*)outf, (Real*)outg);
  else
    lb_pull_kernel<Real, LBRB_TWALL_ADIABATIC><<<grid, 128, 0, s>>>(V, (Real*)outf, (Real*)outg);
  return cudaGetLastError();
}
cudaError_t launch_pull_fp64(const LBView<double>& V, int twall, void* outf, void* outg, cudaStream_t s) {
  return launch_pull_t<double>(V, twall, outf, outg, s);
}
cudaError_t launch_pull_fp32(const LBView<float>& V, int twall, void* outf, void* outg, cudaStream_t s) {
  return launch_pull_t<float>(V, twall, outf, outg, s);
}

// launches timed per shape: enough that each shape's timed span is well above
// the event resolution and launch jitter on small grids
static int tune_reps(const LBView<float>& V) { return (long)V.nx * V.ny >= (1L << 21) ? 6 : 30; }
static int tune_reps(const LBView<double>& V) { return (long)V.nx * V.ny >= (1L << 21) ? 6 : 30; }

int tune_lb_fp64(const LBView<double>& V, int twall, cudaStream_t s, float* best_ms) {
  return tune<double>(V, twall, false, s, tune_reps(V), best_ms);
}
int tune_lb_fp32(const LBView<float>& V, int twall, cudaStream_t s, float* best_ms) {
  return tune<float>(V, twall, false, s, tune_reps(V), best_ms);
}

}  // namespace lbrb
