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
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <type_traits>

#include "lb_pair.cuh"

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

// ------------------------------------------------------- two steps per launch
// Temporal blocking of two steps n, n+1 in TX x TY tiles, one per block
// (lb_pair.cuh: tile_block, the per-block work).
template <typename Real, int TX, int TY, int NT, int MINB, typename Off>
__global__ void __launch_bounds__(NT, MINB) lb_pair_kernel(const LBView<Real> V1, const LBView<Real> V2) {
  pdl_wait();
  extern __shared__ __align__(16) unsigned char pair_smem[];
  tile_block<Real, TX, TY, NT, Off>(V1, V2, blockIdx.x * TX, blockIdx.y * TY, pair_smem);
}

template <typename Real, int R, int MINB, bool PRE, typename Off>
__global__ void __launch_bounds__(32 * (R + 1), MINB)
    lb_march_kernel(const LBView<Real> V1, const LBView<Real> V2, int H) {
  pdl_wait();
  extern __shared__ __align__(16) unsigned char march_smem[];
  const int nstrips = (V1.nx + 31) >> 5;
  const int strip = blockIdx.x % nstrips, chunk = blockIdx.x / nstrips;
  const int ya = chunk * H;
  march_block<Real, R, PRE, Off>(V1, V2, strip * 32, ya, min(H, V1.ny - ya), march_smem);
}

// pair launch shapes: (tile columns, tile rows, threads, min blocks per SM)
struct PairShape { int tx, ty, nt, minb; };
constexpr PairShape PAIR_SHAPES[] = {{32, 8, 256, 4}, {32, 4, 128, 6}, {32, 16, 512, 2}, {64, 4, 256, 3},
                                     {32, 8, 352, 2}, {30, 8, 320, 3}, {32, 8, 256, 5}, {32, 6, 192, 5},
                                     {64, 8, 512, 2}};
constexpr int NPAIR = sizeof(PAIR_SHAPES) / sizeof(PAIR_SHAPES[0]);
static_assert(NPAIR <= NUM_PAIR_SHAPES, "pair shape table");

template <typename Real, int TX, int TY, int NT, int MINB>
static cudaError_t launch_pair_t(const LBView<Real>& V1, const LBView<Real>& V2, cudaStream_t s, bool pdl) {
  constexpr size_t smem = tile_smem_bytes<Real, TX, TY>();
  dim3 grid((V1.nx + TX - 1) / TX, (V1.ny + TY - 1) / TY);
  auto go = [&](auto kernel) -> cudaError_t {
    // the shared-memory limit is a per-device attribute of the kernel: set
    // once per device (one bit per device ordinal, per instantiation)
    static std::atomic<unsigned long long> attr_set{0};
    const cudaError_t e = smem_limit_once((const void*)kernel, smem, attr_set);
    if (e != cudaSuccess) return e;
    return launch_k(kernel, grid, NT, smem, s, pdl, V1, V2);
  };
  // (FP64 holds twice the registers per value: half the blocks per SM)
  constexpr int MB = std::is_same<Real, double>::value ? (MINB + 1) / 2 : MINB;
  if (off32_ok(V1.plane)) return go(lb_pair_kernel<Real, TX, TY, NT, MB, uint32_t>);
  return go(lb_pair_kernel<Real, TX, TY, NT, MB, size_t>);
}

// marching launch shapes: (rows per group R, min blocks per SM, waves): the
// chunk height H = kR - 2 (whole groups) is chosen so that the grid of
// strips x chunks holds about `waves` waves of resident blocks
struct MarchShape { int r, minb, waves, pre; };
constexpr MarchShape MARCH_SHAPES[] = {{8, 3, 8, 0}, {8, 3, 8, 1}, {8, 2, 8, 1},
                                       {6, 4, 8, 1}, {4, 6, 8, 1}, {6, 3, 8, 1}};
constexpr int NMARCH = sizeof(MARCH_SHAPES) / sizeof(MARCH_SHAPES[0]);
static_assert(NPAIR + NMARCH == NUM_PAIR_SHAPES, "pair shape table");

template <typename Real, int R, int MINB, bool PRE>
static cudaError_t launch_march_t(const LBView<Real>& V1, const LBView<Real>& V2, int waves, cudaStream_t s,
                                  bool pdl) {
  constexpr int NT = 32 * (R + 1);
  constexpr size_t smem = march_smem_bytes<Real, R>();
  // (FP64 holds twice the registers and shared memory per value: half the blocks per SM)
  constexpr int MB = std::is_same<Real, double>::value ? (MINB + 1) / 2 : MINB;
  auto go = [&](auto kernel) -> cudaError_t {
    static std::atomic<unsigned long long> attr_set{0};
    static std::atomic<int> occ_cache[MAX_DEVICES] = {};
    cudaError_t e = smem_limit_once((const void*)kernel, smem, attr_set);
    if (e != cudaSuccess) return e;
    int occ = 0, dev = 0, nsm = 0;
    e = occupancy_once((const void*)kernel, NT, smem, occ_cache, &occ);
    if (e == cudaSuccess) e = current_device(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int nx = V1.nx, ny = V1.ny;
    const long nstrips = (nx + 31) / 32;
    const long target = std::max(1L, ((long)waves * occ * nsm + nstrips / 2) / nstrips);  // chunks
    const int h0 = (int)((ny + target - 1) / target);
    const int H = ((h0 + 2 + R - 1) / R) * R - 2;  // whole groups of R rows
    const long nchunks = (ny + H - 1) / H;
    return launch_k(kernel, dim3((unsigned)(nstrips * nchunks)), NT, smem, s, pdl, V1, V2, H);
  };
  if (off32_ok(V1.plane)) return go(lb_march_kernel<Real, R, MB, PRE, uint32_t>);
  return go(lb_march_kernel<Real, R, MB, PRE, size_t>);
}

template <typename Real>
static cudaError_t launch_march(const LBView<Real>& V1, const LBView<Real>& V2, int m, cudaStream_t s, bool pdl) {
  const int waves = MARCH_SHAPES[m].waves;
  switch (m) {
    case 1: return launch_march_t<Real, 8, 3, true>(V1, V2, waves, s, pdl);
    case 2: return launch_march_t<Real, 8, 2, true>(V1, V2, waves, s, pdl);
    case 3: return launch_march_t<Real, 6, 4, true>(V1, V2, waves, s, pdl);
    case 4: return launch_march_t<Real, 4, 6, true>(V1, V2, waves, s, pdl);
    case 5: return launch_march_t<Real, 6, 3, true>(V1, V2, waves, s, pdl);
    default: return launch_march_t<Real, 8, 3, false>(V1, V2, waves, s, pdl);
  }
}

template <typename Real>
static cudaError_t launch_pair(const LBView<Real>& V1, const LBView<Real>& V2, int shape, cudaStream_t s, bool pdl) {
  if (shape >= NPAIR) return launch_march<Real>(V1, V2, shape - NPAIR, s, pdl);
  switch (shape) {
    case 1: return launch_pair_t<Real, 32, 4, 128, 6>(V1, V2, s, pdl);
    case 2: return launch_pair_t<Real, 32, 16, 512, 2>(V1, V2, s, pdl);
    case 3: return launch_pair_t<Real, 64, 4, 256, 3>(V1, V2, s, pdl);
    case 4: return launch_pair_t<Real, 32, 8, 352, 2>(V1, V2, s, pdl);
    case 5: return launch_pair_t<Real, 30, 8, 320, 3>(V1, V2, s, pdl);
    case 6: return launch_pair_t<Real, 32, 8, 256, 5>(V1, V2, s, pdl);
    case 7: return launch_pair_t<Real, 32, 6, 192, 5>(V1, V2, s, pdl);
    case 8: return launch_pair_t<Real, 64, 8, 512, 2>(V1, V2, s, pdl);
    default: return launch_pair_t<Real, 32, 8, 256, 4>(V1, V2, s, pdl);
  }
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
  // two rounds over all shapes, each shape's faster round counts: a shape
  // timed while the clocks settle or beside a transient gets a second look
  float shape_ms[NSHAPES];
  for (float& m : shape_ms) m = 1e30f;
  for (int round = 0; round < 2; round++) {
    for (int sh = 0; sh < NSHAPES; sh++) {
      auto go = [&]() {
        if constexpr (std::is_same<Real, double>::value) return launch_lb_fp64(V, twall, refnudge, sh, s, false);
        else return launch_lb_fp32(V, twall, sh, s, false);
      };
      if (go() != cudaSuccess) { cudaGetLastError(); continue; }
      cudaEventRecord(a, s);
      for (int r = 0; r < reps; r++) go();
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      shape_ms[sh] = std::min(shape_ms[sh], ms);
    }
  }
  int best = 0;
  float bt = 1e30f;
  for (int sh = 0; sh < NSHAPES; sh++)
    if (shape_ms[sh] < bt) { bt = shape_ms[sh]; best = sh; }
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

// two steps per launch: V1 is step n (its pops and F outputs unused), V2 step
// n+1 (its pop and F inputs unused)
cudaError_t launch_pair_fp32(const LBView<float>& V1, const LBView<float>& V2, int shape, cudaStream_t s, bool pdl) {
  return launch_pair<float>(V1, V2, shape, s, pdl);
}
cudaError_t launch_pair_fp64(const LBView<double>& V1, const LBView<double>& V2, int shape, cudaStream_t s,
                             bool pdl) {
  return launch_pair<double>(V1, V2, shape, s, pdl);
}

// pair shape autotuner: as tune(), the trial launches write only buffers the
// real steps overwrite (the views' destinations; no rho or T)
template <typename Real>
static int tune_pair(const LBView<Real>& A, const LBView<Real>& B, cudaStream_t s, float* best_ms) {
  LBView<Real> V1 = A, V2 = B;
  V1.write_rt = V2.write_rt = 0;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int reps = tune_reps(V1);
  float shape_ms[NUM_PAIR_SHAPES];
  for (float& m : shape_ms) m = 1e30f;
  for (int round = 0; round < 2; round++) {  // (as tune(): each shape's faster round)
    for (int sh = 0; sh < NUM_PAIR_SHAPES; sh++) {
      if (launch_pair<Real>(V1, V2, sh, s, false) != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      cudaEventRecord(a, s);
      for (int r = 0; r < reps; r++) launch_pair<Real>(V1, V2, sh, s, false);
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      shape_ms[sh] = std::min(shape_ms[sh], ms);
    }
  }
  int best = 0;
  float bt = 1e30f;
  for (int sh = 0; sh < NUM_PAIR_SHAPES; sh++)
    if (shape_ms[sh] < bt) { bt = shape_ms[sh]; best = sh; }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (best_ms) *best_ms = bt / reps;
  return best;
}
int tune_pair_fp32(const LBView<float>& V1, const LBView<float>& V2, cudaStream_t s, float* best_ms) {
  return tune_pair<float>(V1, V2, s, best_ms);
}
int tune_pair_fp64(const LBView<double>& V1, const LBView<double>& V2, cudaStream_t s, float* best_ms) {
  return tune_pair<double>(V1, V2, s, best_ms);
}

}  // namespace lbrb
