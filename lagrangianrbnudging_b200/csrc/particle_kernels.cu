// particle_kernels.cu -- Lagrangian particles: interpolate, advance, record,
// wrap/reflect.  One thread per particle (a warp advances a tile of 32).
//
// Reference semantics (Trajectories/code/mympi2.h):
//   bilinear     :292-311  cell index by C truncation, weights in the order
//                          val1+val2+val3+val4; halos periodic in x and y
//   tracer       :358-372  Adams-Bashforth 2: x += 1.5 u^n - 0.5 u_p^{n-1}
//   inertial     :373-433  Maxey-Riley, explicit Euler:
//                          v += beta (du/dt + u.grad u) - (v - u)/tau_p; x += v
//                          du/dt = u^n - u^{n-1}, central differences in x,
//                          central in y except one-sided at the wall rows
//   record       :434-565 and temppart_dump.c:1467-1571: T at the new,
//                          not yet wrapped position; Writefull terms at (xo,yo)
//   wrap/reflect :589-635, 681-723
// The reference materialises six derivative fields every step (6 extra field
// sweeps and 6 halo exchanges); here each particle evaluates the derivative
// at its 4 cell corners from a 4x4 stencil of u, v and the 2x2 u^{n-1}.
// Built with --fmad=false: the FP64 results match the reference bit for bit.
#include "particle_dev.cuh"
#include "slab_parts.cuh"

namespace lbrb {

template <typename Real, bool DERIVS>
__global__ void __launch_bounds__(128) particle_kernel(const PView<Real> V) {
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= V.np) return;
  particle_update<Real, DERIVS>(V, p);
}

template <typename Real>
cudaError_t launch_particles_t(const PView<Real>& V, cudaStream_t s, bool pdl) {
  if (V.np <= 0) return cudaSuccess;
  // the derivative stencil only where beta != 0 or full records need it
  if (V.beta != 0.0 || V.full) return launch_k(particle_kernel<Real, true>, (V.np + 127) / 128, 128, 0, s, pdl, V);
  return launch_k(particle_kernel<Real, false>, (V.np + 127) / 128, 128, 0, s, pdl, V);
}

// Two steps of a particle in one launch, after a two-step fused launch has
// stored u, v (and T) of both steps: Va is step n, Vb step n+1.  The second
// update reads the state the first one wrote (the same thread, so it sees
// its own stores); the arithmetic is particle_update's, step by step.
template <typename Real, bool DERIVS>
__global__ void __launch_bounds__(128) particle_pair_kernel(const PView<Real> Va, const PView<Real> Vb) {
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= Va.np) return;
  particle_update<Real, DERIVS>(Va, p);
  particle_update<Real, DERIVS>(Vb, p);
}

// ------------------------------------------------------------- y-slabs
// A domain held as y-slabs, one handle each (one process per GPU, or several
// in one process): each slab holds the particles whose cell lies in its rows,
// as the reference's ranks do (toggle_prtcl, Trajectories/code/mympi2.h:
// 568-760, sends the particles that leave a rank's block to the neighbour).
// Per step, after the slab's fused kernel and the exchange of the moment
// rows (slab_mom_pack_kernel): own_step_kernel advances the slab's particles,
// reading the fields through row tables (own rows, the neighbours' rows
// from the moment messages, a zero row elsewhere) and classifies each by the
// cell it ends in, and its last block turns the per-block counts into
// offsets; own_scatter_kernel compacts the kept particles, in order, into the other
// buffer and writes the leavers, in order, into the hand-off lists; after
// the exchange of the lists own_recv_kernel appends the particles from below
// and then those from above.  A particle's arithmetic is particle_update's,
// so its state equals the whole domain's bit for bit.
__device__ __forceinline__ int cell_row(double yy, int ny) {
  if (!(yy > -2.0 && yy < ny + 2.0)) return 0;  // (flagged by make_cell)
  return wrapi((int)yy - 1, ny);
}

// a row of the domain within reach of the slab [j0, j0 + nyl): its own rows,
// one below and two above (periodic in y)
__device__ __forceinline__ bool in_reach(int j, int j0, int nyl, int nyT) {
  const int d = wrapi(j - j0 + 1, nyT);  // 0: the row below
  return d <= nyl + 2;
}

struct OwnArgs {
  int* cnt;
  const int* id;
  int* rid;         // record ids (record steps) or null
  int* rcnt;        // record count (record steps) or null
  unsigned char* cls;
  int* bcnt;
  unsigned* done;   // blocks finished (the last one scans; it resets this)
  int j0, nyl, istep, xcap;
  const SlabMsg* mlo;  // moment rows from the slab below
  const SlabMsg* mhi;  // from the slab above
  SlabMsg* hup;        // hand-off headers written (own lists or the neighbours' received ones)
  SlabMsg* hdown;
};

// The last block of own_step_kernel to finish turns the per-block counts
// into exclusive offsets (each of its threads scans a run of consecutive
// blocks) and writes the kept count and the hand-off headers: the pattern of
// a reduction whose last block, found by an atomic counter after a memory
// fence, finishes it (no block waits for another).
__device__ void own_scan_last(const OwnArgs& A, unsigned* dflags) {
  __shared__ int s[3][128];
  const int t = threadIdx.x, nblk = gridDim.x;
  const int per = (nblk + 127) / 128;
  const int b0 = min(nblk, t * per), b1 = min(nblk, b0 + per);
  int loc[3] = {0, 0, 0};
  for (int b = b0; b < b1; b++)
    for (int k = 0; k < 3; k++) loc[k] += __ldcg(A.bcnt + b * 3 + k);
  for (int k = 0; k < 3; k++) s[k][t] = loc[k];
  __syncthreads();
  for (int off = 1; off < 128; off <<= 1) {
    int v[3];
    for (int k = 0; k < 3; k++) v[k] = t >= off ? s[k][t - off] : 0;
    __syncthreads();
    for (int k = 0; k < 3; k++) s[k][t] += v[k];
    __syncthreads();
  }
  int run[3];
  for (int k = 0; k < 3; k++) run[k] = s[k][t] - loc[k];
  for (int b = b0; b < b1; b++)
    for (int k = 0; k < 3; k++) {
      const int c = __ldcg(A.bcnt + b * 3 + k);
      A.bcnt[b * 3 + k] = run[k];
      run[k] += c;
    }
  if (t == 127) {
    const int kept = s[0][127], up = s[1][127], down = s[2][127];
    A.cnt[0] = kept;
    A.cnt[1] = kept;
    if (up > A.xcap || down > A.xcap) atomicOr(dflags, DFLAG_XCAP);
    const int j1 = A.j0 + A.nyl;
    *A.hup = SlabMsg{min(up, A.xcap), A.istep, A.j0, j1, MSG_HAND_UP, {0, 0, 0}};
    *A.hdown = SlabMsg{min(down, A.xcap), A.istep, A.j0, j1, MSG_HAND_DOWN, {0, 0, 0}};
    *A.done = 0u;  // (for the next launch)
  }
}

template <typename Real, bool DERIVS>
__global__ void __launch_bounds__(128) own_step_kernel(const PView<Real> V, const OwnArgs A) {
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;  // (the grid covers the capacity)
  const int n = A.cnt[1], nyT = V.ny;
  if (p == 0) {
    const SlabMsg lo = *A.mlo, hi = *A.mhi;
    const bool ok = lo.kind == MSG_MOM_UP && lo.step == A.istep && wrapi(lo.j1, nyT) == A.j0 &&
                    hi.kind == MSG_MOM_DOWN && hi.step == A.istep && hi.j0 == wrapi(A.j0 + A.nyl, nyT);
    if (!ok) atomicOr(V.dflags, DFLAG_XMSG);
    if (A.rcnt) *A.rcnt = n;
  }
  int c = 3;
  if (p < n) {
    const int cr = cell_row(V.P[V.np + p], nyT);
    if (cr < A.j0 || cr >= A.j0 + A.nyl) {
      atomicOr(V.dflags, DFLAG_RANGE);  // (a particle that moved past a neighbour slab)
      c = 0;
    } else {
      particle_update<Real, DERIVS, true>(V, p);
      if (V.record) {
        A.rid[p] = A.id[p];
        // the record's T was read at the new position: rows within reach?
        const double yr = V.rec[(size_t)LBRB_REC_Y * V.np + p];
        if (yr > -2.0 && yr < nyT + 2.0) {
          const int y1 = (int)yr;
          if (!in_reach(wrapi(y1 - 1, nyT), A.j0, A.nyl, nyT) || !in_reach(wrapi(y1, nyT), A.j0, A.nyl, nyT))
            atomicOr(V.dflags, DFLAG_RANGE);
        }
      }
      const double yn = V.P[V.np + p];
      const int cn = cell_row(yn, nyT);
      c = !(yn > -2.0 && yn < nyT + 2.0) ? 0 : (cn < A.j0 ? 2 : (cn >= A.j0 + A.nyl ? 1 : 0));
    }
  }
  A.cls[p] = (unsigned char)c;
  const int k0 = __syncthreads_count(c == 0), k1 = __syncthreads_count(c == 1), k2 = __syncthreads_count(c == 2);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    A.bcnt[blockIdx.x * 3 + 0] = k0;
    A.bcnt[blockIdx.x * 3 + 1] = k1;
    A.bcnt[blockIdx.x * 3 + 2] = k2;
    __threadfence();
    last = atomicAdd(A.done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  own_scan_last(A, V.dflags);
}

__device__ __forceinline__ void put_rec(HandoffRec* r, const double* __restrict__ P, int cap, int p, int id,
                                        int type) {
#pragma unroll
  for (int k = 0; k < 9; k++) r->P[k] = P[(size_t)k * cap + p];
  r->id = id;
  r->type = type;
}

__global__ void __launch_bounds__(128)
    own_scatter_kernel(const double* __restrict__ P, const int* __restrict__ id, const int* __restrict__ type, int cap,
                       const unsigned char* __restrict__ cls, const int* __restrict__ bcnt, double* __restrict__ P2,
                       int* __restrict__ id2, int* __restrict__ type2, HandoffRec* __restrict__ up,
                       HandoffRec* __restrict__ down, int xcap) {
  pdl_wait();
  __shared__ int wc[3][4];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = cls[p];
  unsigned m[3];
  for (int k = 0; k < 3; k++) m[k] = __ballot_sync(0xffffffffu, c == k);
  if (lane == 0)
    for (int k = 0; k < 3; k++) wc[k][w] = __popc(m[k]);
  __syncthreads();
  if (c == 3) return;
  int at = bcnt[blockIdx.x * 3 + c] + __popc(m[c] & ((1u << lane) - 1u));
  for (int q = 0; q < w; q++) at += wc[c][q];
  if (c == 0) {
#pragma unroll
    for (int k = 0; k < 9; k++) P2[(size_t)k * cap + at] = P[(size_t)k * cap + p];
    id2[at] = id[p];
    type2[at] = type[p];
  } else if (at < xcap) {
    put_rec((c == 1 ? up : down) + at, P, cap, p, id[p], type[p]);
  }
}

// the particles handed over by the slab below (lo) and the slab above (hi),
// appended after the kept ones in that order
__global__ void __launch_bounds__(128)
    own_recv_kernel(double* __restrict__ P, int* __restrict__ id, int* __restrict__ type, int cap, int* cnt,
                    const SlabMsg* hlo, const HandoffRec* __restrict__ rlo, const SlabMsg* hhi,
                    const HandoffRec* __restrict__ rhi, int xcap, int istep, int j0, int j1, int nyT,
                    unsigned* dflags) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const SlabMsg lo = *hlo, hi = *hhi;
  const bool ok = lo.kind == MSG_HAND_UP && lo.step == istep && wrapi(lo.j1, nyT) == j0 && lo.count >= 0 &&
                  lo.count <= xcap && hi.kind == MSG_HAND_DOWN && hi.step == istep && hi.j0 == wrapi(j1, nyT) &&
                  hi.count >= 0 && hi.count <= xcap;
  const int nlo = ok ? lo.count : 0, nhi = ok ? hi.count : 0;
  const int n0 = cnt[0];
  if (t == 0) {
    if (!ok) atomicOr(dflags, DFLAG_XMSG);
    if (n0 + nlo + nhi > cap) atomicOr(dflags, DFLAG_XCAP);
    cnt[1] = min(cap, n0 + nlo + nhi);
  }
  const HandoffRec* r = nullptr;
  int at = 0;
  if (t < xcap) {
    if (t < nlo) r = rlo + t, at = n0 + t;
  } else if (t - xcap < nhi) {
    r = rhi + (t - xcap), at = n0 + nlo + (t - xcap);
  }
  if (!r || at >= cap) return;
#pragma unroll
  for (int k = 0; k < 9; k++) P[(size_t)k * cap + at] = r->P[k];
  id[at] = r->id;
  type[at] = r->type;
}

// the moment rows a slab sends: up (u, v, T of its top row) and down (u, v,
// u^{n-1}, v^{n-1}, T of row 0, u, v, T of row 1)
template <typename Real>
__global__ void __launch_bounds__(256)
    slab_mom_pack_kernel(const Real* __restrict__ u, const Real* __restrict__ v, const Real* __restrict__ ub,
                         const Real* __restrict__ vb, const Real* __restrict__ T, int nx, int nyl, int pitch,
                         char* mup, char* mdown, size_t pstride, int istep, int j0) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.y;  // plane: 0-2 up, 3-10 down
  if (q == 0 && i == 0) {
    *(SlabMsg*)mup = SlabMsg{MOM_UP_PLANES, istep, j0, j0 + nyl, MSG_MOM_UP, {0, 0, 0}};
    *(SlabMsg*)mdown = SlabMsg{MOM_DOWN_PLANES, istep, j0, j0 + nyl, MSG_MOM_DOWN, {0, 0, 0}};
  }
  if (i >= nx) return;
  const size_t top = (size_t)(nyl - 1) * pitch, r1 = (size_t)pitch;
  const Real* src;
  char* dst;
  switch (q) {
    case 0: src = u + top; break;
    case 1: src = v + top; break;
    case 2: src = T + top; break;
    case 3: src = u; break;
    case 4: src = v; break;
    case 5: src = ub; break;
    case 6: src = vb; break;
    case 7: src = T; break;
    case 8: src = u + r1; break;
    case 9: src = v + r1; break;
    default: src = T + r1; break;
  }
  dst = q < 3 ? mup + MOM_PLANES_OFF + q * pstride : mdown + MOM_PLANES_OFF + (q - 3) * pstride;
  ((Real*)dst)[i] = src[i];
}

cudaError_t launch_slab_mom_pack(const void* u, const void* v, const void* ub, const void* vb, const void* T,
                                 bool fp32, int nx, int nyl, int pitch, void* mup, void* mdown, size_t pstride,
                                 int istep, int j0, cudaStream_t s, bool pdl) {
  const dim3 g((nx + 255) / 256, MOM_UP_PLANES + MOM_DOWN_PLANES);
  if (fp32)
    return launch_k(slab_mom_pack_kernel<float>, g, 256, 0, s, pdl, (const float*)u, (const float*)v,
                    (const float*)ub, (const float*)vb, (const float*)T, nx, nyl, pitch, (char*)mup, (char*)mdown,
                    pstride, istep, j0);
  return launch_k(slab_mom_pack_kernel<double>, g, 256, 0, s, pdl, (const double*)u, (const double*)v,
                  (const double*)ub, (const double*)vb, (const double*)T, nx, nyl, pitch, (char*)mup, (char*)mdown,
                  pstride, istep, j0);
}

cudaError_t launch_own_particles(const void* const* rows5, bool fp32, int nx, int ny_total, const SlabParts& S,
                                 void* hand_up, void* hand_down, int j0, int nyl, int istep, double beta, int record,
                                 int full, double* rec, int* rid, int* rcnt, unsigned* dflags, cudaStream_t s,
                                 bool pdl) {
  const int nblk = S.cap / 128, o = S.pc;
  OwnArgs A{S.cnt, S.id[o], rid, rcnt, S.cls, S.bcnt, S.done, j0, nyl, istep, S.xcap,
            (const SlabMsg*)S.mom[2], (const SlabMsg*)S.mom[3], (SlabMsg*)hand_up, (SlabMsg*)hand_down};
  auto go = [&](auto zero) -> cudaError_t {
    using Real = decltype(zero);
    using Rows = const Real* const*;
    PView<Real> V{nullptr, nullptr, nullptr, nullptr, nullptr, nx, ny_total, 0, S.P[o], S.type[o], S.cap, beta,
                  record, full, rec, dflags, (Rows)rows5[0], (Rows)rows5[1], (Rows)rows5[2], (Rows)rows5[3],
                  (Rows)rows5[4]};
    if (beta != 0.0 || full) return launch_k(own_step_kernel<Real, true>, nblk, 128, 0, s, pdl, V, A);
    return launch_k(own_step_kernel<Real, false>, nblk, 128, 0, s, pdl, V, A);
  };
  cudaError_t e = fp32 ? go(0.f) : go(0.0);
  if (e != cudaSuccess) return e;
  return launch_k(own_scatter_kernel, nblk, 128, 0, s, pdl, (const double*)S.P[o], (const int*)S.id[o],
                  (const int*)S.type[o], S.cap, (const unsigned char*)S.cls, (const int*)S.bcnt, S.P[o ^ 1],
                  S.id[o ^ 1], S.type[o ^ 1], (HandoffRec*)((char*)hand_up + HAND_RECS_OFF),
                  (HandoffRec*)((char*)hand_down + HAND_RECS_OFF), S.xcap);
}

cudaError_t launch_own_recv(const SlabParts& S, int j0, int nyl, int nyT, int istep, unsigned* dflags,
                            cudaStream_t s, bool pdl) {
  const int o = S.pc;
  return launch_k(own_recv_kernel, (2 * S.xcap + 127) / 128, 128, 0, s, pdl, S.P[o], S.id[o], S.type[o], S.cap,
                  S.cnt, (const SlabMsg*)S.hand[2], (const HandoffRec*)((const char*)S.hand[2] + HAND_RECS_OFF),
                  (const SlabMsg*)S.hand[3], (const HandoffRec*)((const char*)S.hand[3] + HAND_RECS_OFF), S.xcap,
                  istep, j0, j0 + nyl, nyT, dflags);
}

cudaError_t launch_particles_pair(const void* const* fields_a, const void* const* fields_b, bool fp32, int nx,
                                  int ny, int pitch, double* P, const int* ptype, int np, double beta, int full,
                                  double* rec_a, double* rec_b, unsigned* dflags, cudaStream_t s, bool pdl) {
  if (np <= 0) return cudaSuccess;
  auto go = [&](auto zero) -> cudaError_t {
    using Real = decltype(zero);
    auto view = [&](const void* const* f, double* rec) {
      return PView<Real>{(const Real*)f[0], (const Real*)f[1], (const Real*)f[2], (const Real*)f[3], (const Real*)f[4],
                         nx, ny, pitch, P, ptype, np, beta, rec ? 1 : 0, full, rec, dflags};
    };
    const PView<Real> Va = view(fields_a, rec_a), Vb = view(fields_b, rec_b);
    const int g = (np + 127) / 128;
    if (beta != 0.0 || full) return launch_k(particle_pair_kernel<Real, true>, g, 128, 0, s, pdl, Va, Vb);
    return launch_k(particle_pair_kernel<Real, false>, g, 128, 0, s, pdl, Va, Vb);
  };
  return fp32 ? go(0.f) : go(0.0);
}

// explicit views built by the host side
cudaError_t launch_particles(const void* u, const void* v, const void* ub, const void* vb,
                             const void* T, bool fp32, int nx, int ny, int pitch, double* P,
                             const int* ptype, int np, double beta, int record, int full,
                             double* rec, unsigned* dflags, cudaStream_t s, bool pdl) {
  if (fp32) {
    PView<float> V{(const float*)u, (const float*)v, (const float*)ub, (const float*)vb,
                   (const float*)T, nx, ny, pitch, P, ptype, np, beta, record, full, rec, dflags};
    return launch_particles_t(V, s, pdl);
  }
  PView<double> V{(const double*)u, (const double*)v, (const double*)ub, (const double*)vb,
                  (const double*)T, nx, ny, pitch, P, ptype, np, beta, record, full, rec, dflags};
  return launch_particles_t(V, s, pdl);
}

}  // namespace lbrb
