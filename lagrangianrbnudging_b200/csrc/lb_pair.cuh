// lb_pair.cuh -- device code of the two-step launches shared by the
// single-run kernels (lb_kernels.cu: lb_pair_kernel, lb_march_kernel) and
// the ensemble's two-step kernel (ensemble_kernels.cu): the ghost rows of a
// y-slab, the nudging sums of a nudged run, and one marching block.
//
// Reference semantics: as lb_kernels.cu (temppart_dump.c:744-1341, the loop
// body :1674-1759); two steps here equal two single steps bit for bit.
#pragma once

#include "lb_node.cuh"

namespace lbrb {

// On a y-slab, the ring row outside the slab (row -1 or ny) is the
// neighbour's boundary row r1: its populations of step n-1 come from the
// ghost block (SLAB_GH2_PLANES planes: r1's crossing populations, its k = 0,
// 1, 3, its F, then the crossing populations of the row r2 beyond), except
// those it pulls from this slab's own boundary row.  Neither r1 nor r2 is a
// wall row (slabs hold at least three rows).
template <typename Real, typename Off>
__device__ __forceinline__ void pull_ghost_row(const LBView<Real>& V, bool lo, int x, Real* fs, Real* gs, Real& Fy) {
  const Real* G = lo ? V.gh2_lo : V.gh2_hi;
  const int nx = V.nx;
  const int xl = (x == 0) ? nx - 1 : x - 1, xr = (x == nx - 1) ? 0 : x + 1;
  const Off pl = (Off)V.plane, own = (Off)(lo ? 0 : V.ny - 1) * (Off)V.pitch;
  static_for<NPOP>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    const int xs = icx(k) == 1 ? xl : (icx(k) == -1 ? xr : x);
    if constexpr (icy(k) == 0) {
      constexpr int m = k == 0 ? 0 : (k == 1 ? 1 : 2);
      fs[k] = G[(size_t)(6 + m) * nx + xs];
      gs[k] = G[(size_t)(9 + m) * nx + xs];
    } else {
      // from this slab's boundary row (k moving away from it), else from r2
      const bool from_own = lo ? icy(k) == -1 : icy(k) == 1;
      constexpr int slot = (k == 2 || k == 4) ? 0 : ((k == 5 || k == 7) ? 1 : 2);
      if (from_own) {
        fs[k] = V.fsrc[(Off)k * pl + own + (Off)xs];
        gs[k] = V.gsrc[(Off)k * pl + own + (Off)xs];
      } else {
        fs[k] = G[(size_t)(13 + slot) * nx + xs];
        gs[k] = G[(size_t)(16 + slot) * nx + xs];
      }
    }
  });
  Fy = G[(size_t)12 * nx + x];
}

// A bilinear-nudged run's two-step launch: the nudging sum of step n at
// node (y, x) (element offset o), 0 where the mask has no bit or the sum is
// 0 (the apply pass of a single step skips those nodes too)
template <typename Real>
__device__ __forceinline__ long long pair_nudge_sum(const LBView<Real>& V, int y, int x, size_t o) {
  if (!V.nmask || y < 0 || y >= V.ny) return 0;
  const unsigned w = V.nmask[(size_t)y * (size_t)(V.pitch >> 5) + (size_t)(x >> 5)];
  if (!((w >> (x & 31)) & 1u)) return 0;
  return (long long)V.nacc[o];
}

// ------------------------------------------- two steps per launch, marching
// The same two steps as lb_pair_kernel, with far less recomputation: a block
// owns a strip of 32 columns [x0, x0 + 32) and a chunk of rows [ya, ya + Hc)
// and walks down it in groups of R rows.  With ly = y - ya + 1 (ring row
// index; ly = 0 is the row below the chunk), group q does
//   phase 1: step n at rows ly in [qR, qR + R) for the 34 region columns
//            x0-1 .. x0+32 (R warps take the strip's columns of one row
//            each; one more warp takes the two halo columns of all R rows),
//            pulled from HBM exactly as lb_update_node pulls, into a ring of
//            RING = 2R + 2 rows in shared memory; the chunk's own rows also
//            store u^n, v^n (T^n on a record step) and keep F^{n+1};
//   one barrier;
//   phase 2: step n+1 at output rows ly in [qR - 1, qR + R - 1) within
//            [1, Hc], pulled from the ring with pull_node's wall rules.
// Phase 2 of group q reads ring rows [qR - 2, qR + R - 1]; phase 1 of group
// q + 1 overwrites rows [qR - R - 2, qR - 3], which only phase 2 of group
// q - 1 read, before the barrier of group q: one barrier per group orders
// the ring.  Recomputed per strip and chunk: the two halo columns and the two
// rows beyond the chunk (34/32 x (Hc + 2)/Hc node updates in phase 1,
// against 34 x 10 / (32 x 8) for the 32 x 8 tile).  The per-node arithmetic
// is lb_update_node's, so the result equals two single steps bit for bit.
// Slabs: as in lb_pair_kernel, rows -1 and ny come from the ghost blocks.
// shared memory of march_block: the ring of step-n populations, then F^{n+1}
template <typename Real, int R>
constexpr size_t march_smem_bytes() {
  return ((size_t)2 * NPOP * (2 * R + 2) * 34 + (size_t)(2 * R + 2) * 32) * sizeof(Real);
}

// One block's strip [x0, x0 + 32) and chunk of rows [ya, ya + Hc); smem:
// march_smem_bytes<Real, R>() of shared memory; 32 (R + 1) threads
// PRE: software pipelining -- a thread pulls its phase-1 inputs of group
// q + 1 right after the barrier of group q, so the loads are in flight while
// it computes phase 2 of group q (the inputs live in registers meanwhile)
template <typename Real, int R, bool PRE, typename Off>
__device__ __forceinline__ void march_block(const LBView<Real>& V1, const LBView<Real>& V2, int x0, int ya, int Hc,
                                            unsigned char* smem) {
  static_assert(2 * R <= 32, "the halo warp takes 2R nodes");
  constexpr int RING = 2 * R + 2, CW = 34, PL = RING * CW;
  Real* S = reinterpret_cast<Real*>(smem);  // [2 * NPOP][RING][CW]: f then g of step n
  Real* SF = S + 2 * NPOP * PL;             // [RING][32]: F^{n+1} at the strip's columns
  const int nx = V1.nx, ny = V1.ny;
  const int ncols = min(32, nx - x0);
  const Off pitch = (Off)V1.pitch;
  const bool glo = V1.gh2_lo != nullptr, ghi = V1.gh2_hi != nullptr;
  const int ylo = glo ? -1 : 0, yhi = ghi ? ny : ny - 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this thread's phase-1 node: row w of the group, column x, ring column c
  int w, x, c;
  bool col_ok;
  if (warp < R) {
    w = warp;
    x = x0 + lane;
    c = lane + 1;
    col_ok = lane < ncols;
  } else {
    const bool right = lane >= R;  // lanes [0, R): column x0 - 1; [R, 2R): x0 + ncols
    w = right ? lane - R : lane;
    c = right ? ncols + 1 : 0;
    x = right ? x0 + ncols : x0 - 1;
    if (x < 0) x += nx;
    else if (x >= nx) x -= nx;
    col_ok = lane < 2 * R;
  }
  // phase-1 inputs of this thread's node in group q: the pulled populations
  // (walls applied), the step's buoyancy, the nudging sum of a nudged run
  Real fs[NPOP], gs[NPOP], Fy = Real(0);
  long long nsum = 0;
  bool on = false;
  int y1 = 0, slot = 0;
  Off o1 = 0;
  auto fetch = [&](int q) {
    const int ly = q * R + w;
    y1 = ya - 1 + ly;
    on = col_ok && ly <= Hc + 1 && y1 >= ylo && y1 <= yhi;
    if (!on) return;
    slot = ly % RING;
    o1 = (Off)(y1 < 0 ? 0 : (y1 >= ny ? ny - 1 : y1)) * pitch + (Off)x;  // (ghost rows: no stores)
    if (y1 < 0 || y1 >= ny) {
      pull_ghost_row<Real, Off>(V1, y1 < 0, x, fs, gs, Fy);
    } else {
      pull_node<Real, LBRB_TWALL_DIRICHLET, Off, true>(V1, y1, x, fs, gs);
      dirichlet_walls(V1, y1, gs);
      Fy = V1.Fin[o1];
    }
    if (V1.nmask) nsum = pair_nudge_sum(V1, y1, x, (size_t)o1);
  };
  // phase 1 from the fetched inputs: collide into the ring; the chunk's own
  // nodes of the strip also store their moments and keep F^{n+1}
  auto collide = [&]() {
    if (!on) return;
    Real r, u, v, t;
    Real* Sc = S + slot * CW + c;
    double nsv = 0.0;
    if (V1.nmask && nsum != 0) nsv = (double)nsum * (1.0 / FIX_SCALE);
    lb_collide<Real, false>(
        V1, (size_t)o1, fs, gs, Fy, r, u, v, t, [&](int k, Real val) { Sc[k * PL] = val; },
        [&](int k, Real val) {
          if (nsum != 0) val = val + nudge_increment<Real>(k, nsv);
          Sc[(NPOP + k) * PL] = val;
        });
    if (warp < R && y1 >= ya && y1 < ya + Hc) {  // a node of this block's strip and chunk
      SF[slot * 32 + lane] = Fy;
      if (V1.write_F) V1.Fout[o1] = Fy;
      if (V1.write_uv) {
        V1.u[o1] = u;
        V1.v[o1] = v;
      }
      if (V1.write_rt & 1) V1.T[o1] = t;
      if (V1.write_rt & 2) V1.rho[o1] = r;
    }
  };
  const int Q = (Hc + 2 + R - 1) / R;
  if (PRE) fetch(0);
  for (int q = 0; q < Q; q++) {
    if (!PRE) fetch(q);
    collide();
    __syncthreads();
    if (PRE && q + 1 < Q) fetch(q + 1);
    if (warp < R) {
      const int ly = q * R - 1 + w, y = ya - 1 + ly;
      if (lane < ncols && ly >= 1 && ly <= Hc) {
        const int s0 = ly % RING, sm = (ly - 1) % RING, sp = (ly + 1) % RING;
        Real f2[NPOP], g2[NPOP];
        static_for<NPOP>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          const int js = y - icy(k);
          if ((js < 0 && !glo) || (js >= ny && !ghi)) {
            f2[k] = S[opp(k) * PL + s0 * CW + lane + 1];
            g2[k] = Real(0);
          } else {
            const int sl = icy(k) == 1 ? sm : (icy(k) == -1 ? sp : s0);
            const int cc = lane + 1 - icx(k);
            f2[k] = S[k * PL + sl * CW + cc];
            g2[k] = S[(NPOP + k) * PL + sl * CW + cc];
          }
        });
        dirichlet_walls(V2, y, g2);
        lb_finish_node<Real, false, Off>(V2, (Off)y * pitch + (Off)(x0 + lane), f2, g2, SF[s0 * 32 + lane]);
      }
    }
  }
}

}  // namespace lbrb
