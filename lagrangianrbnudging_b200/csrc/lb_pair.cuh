// lb_pair.cuh -- device code of the two-step launches shared by the
// single-run kernels (lb_kernels.cu: lb_pair_kernel, lb_march_kernel) and
// the ensemble's two-step kernels (ensemble_kernels.cu): the ghost rows of a
// y-slab, the nudging sums of a nudged run, one tile block and one marching
// block.
//
// Reference semantics: as lb_kernels.cu (temppart_dump.c:744-1341, the loop
// body :1674-1759); two steps here equal two single steps bit for bit.
#pragma once

#include <type_traits>

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

// ------------------------------------------------ two steps per launch, tile
// Temporal blocking of two steps n, n+1 (Dirichlet walls, no ghost rows, no
// nudging in between).  A block owns a TX x TY tile.  Phase 1 computes step n
// at the tile and a one-node ring around it (x wrapped, rows outside the
// domain skipped) from HBM, exactly as lb_update_node does, and keeps the
// post-collision populations in shared memory; at the tile it also stores
// u^n, v^n (and T^n on a record step) to HBM through V1, and keeps the next
// buoyancy F^{n+1} in shared memory.  Phase 2 computes step n+1 at the tile,
// pulling from shared memory with the same wall rules as pull_node (bounce-back
// from the node's own opposite population, anti-bounce-back for g), and
// stores through V2.  Populations and F cross HBM once per two steps; the
// ring is recomputed (34 x 10 nodes for a 32 x 8 tile).  The per-node
// arithmetic is lb_update_node's, so two steps here equal two launches of
// lb_node_kernel bit for bit.
// On a y-slab the ring rows beyond an inner boundary come from the ghost
// blocks (pull_ghost_row).

// shared memory of tile_block: the ring of step-n populations, then F^{n+1}
template <typename Real, int TX, int TY>
constexpr size_t tile_smem_bytes() {
  return ((size_t)2 * NPOP * (TX + 2) * (TY + 2) + (size_t)TX * TY) * sizeof(Real);
}

// One block's tile [x0, x0 + TX) x [y0, y0 + TY); smem: tile_smem_bytes<Real,
// TX, TY>() of shared memory.  NT threads per block: TX * TY (phase 1 takes
// the region in passes), or one per region node rounded to whole warps
// (phase 1 in one pass; phase 2 leaves the rest idle)
template <typename Real, int TX, int TY, int NT, typename Off>
__device__ __forceinline__ void tile_block(const LBView<Real>& V1, const LBView<Real>& V2, int x0, int y0,
                                           unsigned char* smem) {
  constexpr int RX = TX + 2, RY = TY + 2, RN = RX * RY;
  Real* S = reinterpret_cast<Real*>(smem);  // [2 * NPOP][RY][RX]: f then g of step n
  Real* SF = S + 2 * NPOP * RN;             // [TY][TX]: F^{n+1} at the tile
  const int nx = V1.nx, ny = V1.ny;
  const int ncols = min(TX, nx - x0), nrows = min(TY, ny - y0);
  const Off pitch = (Off)V1.pitch;
  // y-slab: the rows beyond an inner boundary are computed from ghost blocks
  const bool glo = V1.gh2_lo != nullptr, ghi = V1.gh2_hi != nullptr;
  // FP64: a full tile whose ring, and the ring's pulls, lie strictly inside
  // the domain (no x wrap, no wall row, no slab ghost row) in a run without
  // in-launch nudging sums takes phase 1 by fixed offsets from each node:
  // the values pull_node's interior path reads, without its bounds, wrap and
  // wall logic (block-uniform).  (In FP32 the second copy of the phase made
  // the launch 10% slower, so FP32 keeps the one general phase.)
  const bool fast = ncols == TX && nrows == TY && x0 >= 2 && x0 + TX + 1 <= nx - 1 && y0 >= 2 &&
                    y0 + TY + 1 <= ny - 1 && !V1.nmask;
  auto phase1 = [&](auto fastc) {
    constexpr bool FAST = decltype(fastc)::value;
    for (int q = threadIdx.x; q < RN; q += NT) {
      const int lx = q % RX, ly = q / RX;
      const int jg = y0 - 1 + ly;
      Real fs[NPOP], gs[NPOP];
      Real Fy, r, u, v, t;
      Off o;
      long long nsum = 0;
      double nsv = 0.0;
      if constexpr (FAST) {
        const int xg = x0 - 1 + lx;
        o = (Off)jg * pitch + (Off)xg;
        const Off pl = (Off)V1.plane;
        static_for<NPOP>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          const Off src = (Off)k * pl + o + (Off)(-icy(k) * V1.pitch - icx(k));  // (modular: a negative shift wraps)
          fs[k] = __ldcs(V1.fsrc + src);
          gs[k] = __ldcs(V1.gsrc + src);
        });
        Fy = V1.Fin[o];
      } else {
        if (lx > ncols + 1 || ly > nrows + 1 || jg < (glo ? -1 : 0) || jg > (ghi ? ny : ny - 1)) continue;
        int xg = x0 - 1 + lx;
        if (xg < 0) xg += nx;
        else if (xg >= nx) xg -= nx;
        o = (Off)(jg < 0 ? 0 : (jg >= ny ? ny - 1 : jg)) * pitch + (Off)xg;  // (ring rows of a slab: no stores)
        if (jg < 0 || jg >= ny) {
          pull_ghost_row<Real, Off>(V1, jg < 0, xg, fs, gs, Fy);
        } else {
          pull_node<Real, LBRB_TWALL_DIRICHLET, Off, true>(V1, jg, xg, fs, gs);
          dirichlet_walls(V1, jg, gs);
          Fy = V1.Fin[o];
        }
        // (nudged run: step n's sums join g after the collision, as the apply pass does)
        if (V1.nmask) {
          nsum = pair_nudge_sum(V1, jg, xg, (size_t)o);
          if (nsum != 0) nsv = (double)nsum * (1.0 / FIX_SCALE);
        }
      }
      lb_collide<Real, false>(
          V1, (size_t)o, fs, gs, Fy, r, u, v, t, [&](int k, Real val) { S[(k * RY + ly) * RX + lx] = val; },
          [&](int k, Real val) {
            if (!FAST && nsum != 0) val = val + nudge_increment<Real>(k, nsv);
            S[((NPOP + k) * RY + ly) * RX + lx] = val;
          });
      if (lx >= 1 && lx <= ncols && ly >= 1 && ly <= nrows) {
        SF[(ly - 1) * TX + (lx - 1)] = Fy;
        if (V1.write_F) V1.Fout[o] = Fy;
        if (V1.write_uv) {
          V1.u[o] = u;
          V1.v[o] = v;
        }
        if (V1.write_rt & 1) V1.T[o] = t;
        if (V1.write_rt & 2) V1.rho[o] = r;
      }
    }
  };
  if constexpr (std::is_same<Real, double>::value) {
    if (fast) phase1(std::true_type{});
    else phase1(std::false_type{});
  } else {
    phase1(std::false_type{});
  }
  __syncthreads();
  if (threadIdx.x >= TX * TY) return;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  if (tx >= ncols || ty >= nrows) return;
  const int x = x0 + tx, j = y0 + ty;
  Real fs[NPOP], gs[NPOP];
  // a tile whose rows and their neighbours all lie in the domain (or beyond
  // an inner slab edge) pulls with no wall rule (block-uniform)
  const bool inner = (y0 > 0 || glo) && (y0 + nrows < ny || ghi);
  if (inner) {
    static_for<NPOP>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      const int lx = tx + 1 - icx(k), ly = ty + 1 - icy(k);
      fs[k] = S[(k * RY + ly) * RX + lx];
      gs[k] = S[((NPOP + k) * RY + ly) * RX + lx];
    });
  } else {
    static_for<NPOP>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      const int js = j - icy(k);
      if ((js < 0 && !glo) || (js >= ny && !ghi)) {
        fs[k] = S[(opp(k) * RY + ty + 1) * RX + tx + 1];
        gs[k] = Real(0);
      } else {
        const int lx = tx + 1 - icx(k), ly = ty + 1 - icy(k);
        fs[k] = S[(k * RY + ly) * RX + lx];
        gs[k] = S[((NPOP + k) * RY + ly) * RX + lx];
      }
    });
    dirichlet_walls(V2, j, gs);
  }
  lb_finish_node<Real, false, Off>(V2, (Off)j * pitch + (Off)x, fs, gs, SF[ty * TX + tx]);
}

// ------------------------------------------- two steps per launch, marching
// The same two steps as tile_block, with far less recomputation: a block
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
// Slabs: as in tile_block, rows -1 and ny come from the ghost blocks.
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
