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
#include <atomic>
#include <utility>
#include <vector>

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

// element offsets of a population buffer (18 planes) fit in 32 bits
inline bool off32_ok(size_t plane) { return plane * 2 * NPOP < (size_t(1) << 32); }

// launch shapes of the two-step kernels (lb_kernels.cu): the tiles of
// lb_pair_kernel (PAIR_SHAPES), then the marching lb_march_kernel
// (MARCH_SHAPES)
constexpr int NUM_PAIR_TILES = 9;
constexpr int NUM_PAIR_SHAPES = NUM_PAIR_TILES + 6;
// planes (of nx values) of a y-slab's ghost block for two steps per launch
// (aux_kernels.cu: slab_pack2_kernel)
constexpr int SLAB_GH2_PLANES = 19;

// Programmatic dependent launch: a kernel launched with the attribute may
// start while the kernel before it in the stream finishes; it waits here,
// before touching memory, until that kernel has completed and its writes are
// visible.  For a kernel launched without the attribute this returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Per-device caches (kernel attributes set once, occupancy queried once) keep
// one entry per device ordinal below MAX_DEVICES; the current ordinal, checked.
constexpr int MAX_DEVICES = 64;
inline cudaError_t current_device(int* dev) {
  const cudaError_t e = cudaGetDevice(dev);
  if (e != cudaSuccess) return e;
  return (*dev < 0 || *dev >= MAX_DEVICES) ? cudaErrorInvalidDevice : cudaSuccess;
}
// a kernel's dynamic shared-memory limit, set once per device: `bits` (one
// static per kernel instantiation) holds a bit per ordinal already set
inline cudaError_t smem_limit_once(const void* kernel, size_t smem, std::atomic<unsigned long long>& bits) {
  int dev = 0;
  cudaError_t e = current_device(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << dev;
  if (bits.load(std::memory_order_relaxed) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  bits.fetch_or(bit, std::memory_order_relaxed);
  return cudaSuccess;
}
// resident blocks per SM of a kernel launch shape, queried once per device
// (`cache`: one static array per kernel instantiation)
inline cudaError_t occupancy_once(const void* kernel, int threads, size_t smem, std::atomic<int>* cache, int* occ) {
  int dev = 0;
  cudaError_t e = current_device(&dev);
  if (e != cudaSuccess) return e;
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    if (v < 1) return cudaErrorInvalidConfiguration;
    cache[dev].store(v, std::memory_order_relaxed);
  }
  *occ = v;
  return cudaSuccess;
}

// launch k<<<grid, block, smem, s>>>(args...), with programmatic dependent
// launch when `pdl` (the kernel must call pdl_wait() first)
template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl,
                            Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

// a state slot of the adjoint window (planes of `plane` elements): the 18
// populations, F, then the moments the step that produced the state formed
// (rho, u, v, T; the next step's adjoint linearises around them)
constexpr int SLOT_F = 2 * NPOP, SLOT_MOM = 2 * NPOP + 1, SLOT_PLANES = 2 * NPOP + 5;
// a state's moment block, all the adjoint reads of a state: F, then rho, u,
// v, T -- a slot's planes SLOT_F .. SLOT_PLANES-1, or one entry of the
// window's moment store (every state's block, when it fits)
constexpr int MB_PLANES = SLOT_PLANES - SLOT_F;
static_assert(SLOT_MOM == SLOT_F + 1 && MB_PLANES == 5, "moment block: F then the four moments");

// x / c for a divisor c fixed at compile time, equal to the IEEE quotient
// RN(x / c) without a division: with rc = RN(1 / c), q0 = RN(x rc) is within
// one ulp of x / c, the remainder r = x - q0 c is exact in one fused
// multiply-add, and RN(q0 + r rc) is RN(x / c) (Markstein's correction step,
// P. Markstein, IBM J. Res. Dev. 34(1), 1990, the basis of correctly rounded
// division on fused multiply-add hardware).  Holds for quotients in the
// normal range, which the state's values are far from leaving; r == 0 means
// q0 is exact (and keeps the sign of a zero x).  tests/test_div_const.py
// checks it against exact rational quotients, including binade edges.
__device__ __forceinline__ double div_const(double x, double c, double rc) {
  const double q0 = __dmul_rn(x, rc);
  const double r = __fma_rn(-q0, c, x);
  return r == 0.0 ? q0 : __fma_rn(r, rc, q0);
}
// the reference's divisors and their rounded reciprocals
constexpr double DIV_2CS2 = 2. * CS2, RCP_2CS2 = 1. / (2. * CS2);
constexpr double RCP_CS2 = 1. / CS2;
constexpr double DIV_2_9 = 2. / 9., RCP_2_9 = 1. / (2. / 9.);
constexpr double DIV_CS4 = CS2 * CS2, RCP_CS4 = 1. / (CS2 * CS2);

// equilif / equilig in the reference's operation order
// (temppart_dump.c:1097-1180): r1 is rho for f and T for g; the divisions by
// lattice constants go through div_const (the same quotients)
__device__ __forceinline__ void equil_ref(double r1, double u, double v, double feq[NPOP]) {
  double usq = u * u;
  double vsq = v * v;
  double sumsq = div_const(usq + vsq, DIV_2CS2, RCP_2CS2);
  double sumsq2 = div_const(sumsq * (1. - CS2), CS2, RCP_CS2);
  double u2 = div_const(usq, DIV_2_9, RCP_2_9);
  double v2 = div_const(vsq, DIV_2_9, RCP_2_9);
  double ui = div_const(u, CS2, RCP_CS2);
  double vi = div_const(v, CS2, RCP_CS2);
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
  DFLAG_XCAP = 8u,       // a slab's particles or a hand-off list over capacity
  DFLAG_XMSG = 16u,      // a slab message from the wrong step or neighbour
};

// ------------------------------------------------------------ kernel views
template <typename Real>
struct LBView {
  const Real* __restrict__ fsrc;
  const Real* __restrict__ gsrc;
  Real* __restrict__ fdst;
  Real* __restrict__ gdst;
  const Real* __restrict__ Fin;  // buoyancy F_y of this step (from step n-1 moments)
  Real* __restrict__ Fout;       // buoyancy of the next step (this step's moments)
  Real* __restrict__ rho;
  Real* __restrict__ u;
  Real* __restrict__ v;
  Real* __restrict__ T;
  int nx, ny, pitch;
  size_t plane;
  double omega, omegag;    // 1/relax, 1/relaxg
  double neg_gravity;      // -gravity
  double Tup, Tdown, T0;
  // the same constants rounded to FP32 on the host, for the FP32 collision
  // (the values (float)omega etc. would give, without a conversion per node)
  float omega_f, omegag_f, neg_gravity_f, T0_f;
  // reference box nudging
  const int* __restrict__ nudge_vol;
  const double* __restrict__ tempreadint;
  double* __restrict__ nud_term;
  // box nudging: row 0's sum of g before the 1/2 nud_term (the reference's
  // halo row above the top row takes that value: lbrb_profile's top dT/dy)
  double* __restrict__ tsum0;
  double alpha;
  int write_uv;
  int write_rt;  // bit 0: store T (records, nudging), bit 1: also rho (a call's last step)
  int write_F;   // lb_pair_kernel: also store step n's F^{n+1} through V1.Fout (adjoint recompute)
  // y-slab of a larger domain: the rows below row 0 / above row ny-1 (the
  // neighbour slab's boundary row after its collision), 6 rows of nx values:
  // f then g of the three populations crossing the boundary; null = wall
  const Real* __restrict__ ghost_lo;
  const Real* __restrict__ ghost_hi;
  // lb_pair_kernel on a y-slab: SLAB_GH2_PLANES-plane ghost blocks (null at a
  // wall); their first six planes are the one-step ghost rows above
  const Real* __restrict__ gh2_lo;
  const Real* __restrict__ gh2_hi;
  // two-step launch of a bilinear-nudged run (first step's view only): the
  // nudging sums of this step at the nodes flagged in nmask (one bit per
  // node, pitch / 32 words per row), 2^-40 fixed point; added to g right
  // after the collision, as the apply pass of a single step adds them
  const unsigned* __restrict__ nmask;
  const unsigned long long* __restrict__ nacc;
};

// 2^-40 fixed point of the bilinear nudging sums (nudge_dev.cuh)
constexpr double FIX_SCALE = 1099511627776.0;

// the apply pass's increment of g_k: w_k * S (rounded to FP32 for FP32 runs)
template <typename Real>
__device__ __forceinline__ Real nudge_increment(int k, double sv) {
  if constexpr (std::is_same<Real, double>::value) return w_of(k) * sv;
  else return (float)(w_of(k) * sv);
}

struct SlabParts;  // particles of a y-slab held by their owner slab (slab_parts.cuh)

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
  // y-slab mode: rows [slab_j0, slab_j0 + ny) of ny_total; ghost rows below
  // and above (null at a wall), this slab's packed boundary rows (up: the top
  // row's upward populations, down: the bottom row's downward ones), events
  // ordering the exchange between neighbours
  bool slab = false;
  int slab_j0 = 0, slab_ny_total = 0;
  void* slab_ghost_lo = nullptr;
  void* slab_ghost_hi = nullptr;
  // ghost blocks for two steps per launch (SLAB_GH2_PLANES rows) and the
  // packed boundary rows sent to the neighbours
  void* slab_gh2_lo = nullptr;
  void* slab_gh2_hi = nullptr;
  void* slab_up2 = nullptr;
  void* slab_down2 = nullptr;
  // lbrb_slab_pack2 ran since this slab's last step: lbrb_step(h, 2) may use
  // the two-row ghost blocks (cleared by the step and by lbrb_slab_pack)
  bool slab_gh2_packed = false;
  void* slab_up = nullptr;
  void* slab_down = nullptr;
  cudaEvent_t slab_ev_xfer = nullptr, slab_ev_done = nullptr;
  bool slab_defer_moments = false;  // inside lbrb_slab_step: moments on its last step only
  bool slab_stepping = false;       // inside lbrb_slab_step
  // bilinear nudging of a slab domain in one process: device tables of row
  // pointers (T of every slab, 2 buffers) built for the slab list slab_sig
  void* slab_tab = nullptr;
  size_t slab_tab_bytes = 0;
  std::vector<const void*> slab_sig;
  // particles of a y-slab held by their owner slab (lbrb_slab_particles_set)
  SlabParts* sp = nullptr;
  const double* slab_obs = nullptr;  // bilinear observations of the step just taken (lbrb_slab_step applies them)
  // CUDA graphs of plain steps, one per buffer phase (cur * 9 + uvcur * 3 +
  // uvprev); graph_mode -1: small grids where two-step launches do not
  // apply, 0: off, 1: on (ahead of two-step launches)
  cudaGraphExec_t graph_exec[18] = {};
  // two steps per launch (lb_pair_kernel, NUM_PAIR_SHAPES tile shapes):
  // pair_mode -1 auto (steps that
  // do not replay graphs), 0 off, 1 on; pair_shape: tuned on first use
  int pair_mode = -1;
  int pair_shape = -1;
  float pair_ms = 0.f;
  int pair_save[3] = {0, 0, 0};  // y-slab pairs: cur, uvcur, uvprev before the launch
  int graph_mode = -1;
  size_t esize = 8;   // bytes per population value
  // populations: pops[buf] holds f (9 planes) then g (9 planes)
  void* pops[2] = {nullptr, nullptr};
  int cur = 0;        // buffer holding the current post-collision state
  bool prev_valid = false;  // pops[cur^1] holds the state before the last step
  // the call ended with a two-step launch without nudging: pops[cur^1] and
  // F[cur^1] hold the state before that launch (lbrb_get_poststream rebuilds
  // the state before the last step from them)
  bool prev_pair = false;
  // scalar fields (Real)
  void* F[2] = {nullptr, nullptr};  // buoyancy for the step after the state in pops[cur] is F[cur]
  int lb_shape = -1;                // launch shape picked by the autotuner (-1: not tuned yet)
  float lb_shape_ms = 0.f;
  // moments: rho and T of the state in pops[cur] are rho[cur], T[cur];
  // u, v rotate over three slots: u^n in uvcur, u^{n-1} in uvprev, so the
  // particle kernel of step n can run beside the fused kernel of step n+1
  void* rho[2] = {nullptr, nullptr};
  void* T[2] = {nullptr, nullptr};
  void* uv[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  int uvcur = 0, uvprev = 1;
  // second stream: the adjoint window's segment recompute (events order it
  // against `stream`)
  cudaStream_t pstream = nullptr;
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
  double* tsum0 = nullptr;  // [pitch]: row 0's sum of g without the 1/2 nud_term (LBView::tsum0)
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
  // two-step launches of a nudged run: the first step's sums (formed before
  // the launch) and their node mask, cleared after the launch
  long long* acc2 = nullptr;
  unsigned* nmask = nullptr;
  // adjoint window
  double* adj_obs = nullptr;         // [nobs_steps][3][nobs]
  int adj_nobs = 0, adj_nsteps_obs = 0;
  int* adj_steps = nullptr;          // host
  double* adj_res = nullptr;         // residuals [nobs_steps][nobs]
  void* adj_chk = nullptr;           // checkpoints: 19 planes each (pops + F)
  size_t adj_chk_bytes = 0;
  void* adj_seg = nullptr;           // two buffers of K+1 segment states
  size_t adj_seg_bytes = 0;
  double* adj_lam = nullptr;         // 2 x 18 lambda planes (ping-pong) + 2 lambda F planes
  long long* adj_lT = nullptr;       // 2 fixed-point lambda T planes (the steps of a pair)
  double* adj_T0 = nullptr;          // [ny*nx] initial temperature / gradient
  int adj_pair_variant = -1;         // launch variant of the pair kernel (-1: tune at first use)
  void* adj_store = nullptr;         // every state's moment block (store mode)
  size_t adj_store_bytes = 0;
  int adj_store_mode = -1;           // 1 store, 0 checkpoint-recompute, -1 store when it fits
  int adj_store_used = 0;            // the last gradient window stored (1) or recomputed (0)
  // scratch / staging: host transfers go through two staging slots of
  // stage_slot doubles each (allocated at create), chunk by chunk, with
  // events xfer_ev (copied[2], converted[2]) ordering the slots' reuse; the
  // restart route's moments and the post-stream dump use `big`, a full-size
  // scratch allocated on their first use
  void* staging = nullptr;
  size_t staging_bytes = 0;
  size_t stage_slot = 0;
  cudaEvent_t xfer_ev[4] = {nullptr, nullptr, nullptr, nullptr};
  void* big = nullptr;
  size_t big_bytes = 0;
  double* red = nullptr;    // reduction partials
  unsigned* dflags = nullptr;
  unsigned* h_flags = nullptr;
  double* h_scalar = nullptr;  // pinned: one device scalar read back (the misfit)
};

}  // namespace lbrb
