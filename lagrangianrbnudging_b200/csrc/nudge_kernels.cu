// nudge_kernels.cu -- temperature nudging toward values stored along
// trajectories.
//
// Box mode (the reference, Nudging/code/tempvel_nudge.c:1380-1781 read_prtcl):
//   every step each observation's position and temperature are advanced by
//   linear interpolation in time between files written every ntempread steps
//   (with the periodic-x and wall-y jump handling of :1489-1552, :1688-1720);
//   then every node inside the 7x7 box around (round x, round y) gets the
//   running mean tempreadint = (tempreadint*n + T)/(n+1), n = nudge_vol, in
//   the reference's contribution order: observation index k ascending, and
//   per k the main box, then its left and right periodic images.
//   The per-node order is reproduced exactly (FP64 bit-identical): the
//   contributions are binned into 8x8-node cells, each cell sorts its
//   contribution keys (3k + image), and each node walks its cell's sorted
//   list.  Only cells that hold contributions, or held some the step before,
//   touch memory.
// Bilinear mode (no reference counterpart): innovation
//   d = alpha (T_obs - T(x_obs)) spread to the 4 cell corners with bilinear
//   weights; contributions are summed in 2^-40 fixed point with integer
//   atomics, so the result does not depend on their order, then added to the
//   post-collision g as w_k * S.
#include "lbrb_internal.cuh"
#include "nudge_dev.cuh"

namespace lbrb {

constexpr int CELL = 8;

// per-observation double arrays in Handle::nb, each of length nobs
enum { NB_OX = 0, NB_OY, NB_OT, NB_FX, NB_FY, NB_FT, NB_XINT, NB_YINT, NB_TINT, NB_DX, NB_DY,
       NB_DT, NB_COUNT };
// per-observation int arrays in Handle::nbi
enum { NBI_CHK = 0, NBI_BC, NBI_XIDX, NBI_YIDX, NBI_COUNT };

struct BoxView {
  double* nb;
  int* nbi;
  // ny: the handle's rows (of nudge_vol, tempreadint and the cells); nyT:
  // the whole domain's rows (positions and boxes); j0: the handle's first
  // row in the domain (0 unless a y-slab)
  int n, nx, ny, nt, istep, nyT, j0;
  int ncx, ncy;
  int* cell_count;
  int* cell_start;
  int* cell_fill;
  int* cell_dirty;
  int* items;
  int* sorted;
  int* nudge_vol;
  double* tempreadint;
  int pitch;
  unsigned* dflags;
};

__device__ __forceinline__ double* NB(const BoxView& B, int a) { return B.nb + (size_t)a * B.n; }
__device__ __forceinline__ int* NBI(const BoxView& B, int a) { return B.nbi + (size_t)a * B.n; }

// time interpolation, one thread per observation (read_prtcl's three branches)
__global__ void box_interp_kernel(const BoxView B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B.n) return;
  const int nx = B.nx, ny = B.nyT, nt = B.nt;
  double *ox = NB(B, NB_OX), *oy = NB(B, NB_OY), *oT = NB(B, NB_OT);
  double *fx = NB(B, NB_FX), *fy = NB(B, NB_FY), *fT = NB(B, NB_FT);
  double *xint = NB(B, NB_XINT), *yint = NB(B, NB_YINT), *Tint = NB(B, NB_TINT);
  double *dxs = NB(B, NB_DX), *dys = NB(B, NB_DY), *dTs = NB(B, NB_DT);
  int *chk = NBI(B, NBI_CHK), *bc = NBI(B, NBI_BC), *xidx = NBI(B, NBI_XIDX), *yidx = NBI(B, NBI_YIDX);
  const int ph = B.istep % nt;
  if (ph == 1) {
    const int c = chk[i];
    int bci = 0;
    double xread = fx[c];
    double yread = fy[c];
    dxs[i] = (xread - xint[i]) / ((double)nt);
    if (abs((int)(xread - xint[i])) > ((double)nx / 2.0)) {
      if (xread > xint[i]) {
        xread = xread - (double)nx;
        dxs[i] = (xread - xint[i]) / ((double)nt);
      } else {
        xread = xread + (double)nx;
        dxs[i] = (xread - xint[i]) / ((double)nt);
      }
    }
    double xposnow = xint[i] + dxs[i];
    if (xposnow > (double)nx) xposnow = xposnow - (double)nx;
    if (xposnow < 0.0) xposnow = xposnow + (double)nx;
    xint[i] = xposnow;
    dys[i] = (yread - yint[i]) / ((double)nt);
    if (abs((int)(yread - yint[i])) > ((double)ny / 2.0)) {
      bci = 1;
      if (yread > yint[i]) {
        yread = yread - (double)ny + 1.0;
        dys[i] = (yread - yint[i]) / ((double)nt);
      } else {
        yread = yread + (double)ny - 1.0;
        dys[i] = (yread - yint[i]) / ((double)nt);
      }
    }
    double yposnow = yint[i] + dys[i];
    if (yposnow > (double)ny) { yposnow = yposnow - (double)ny + 1.0; bci = 2; }
    if (yposnow < 1.0) { yposnow = yposnow + (double)ny - 1.0; bci = 2; }
    yint[i] = yposnow;
    xidx[i] = (int)round(xposnow);
    yidx[i] = (int)round(yposnow);
    const double Tread = fT[c];
    dTs[i] = (Tread - Tint[i]) / ((double)nt);
    double Tnow = Tint[i] + dTs[i];
    if (bci == 1) Tnow = Tint[i];
    if (bci == 2) { Tnow = fT[c]; bci = 1; }
    Tint[i] = Tnow;
    bc[i] = bci;
  } else if (ph == 0) {
    const int c = chk[i];
    xint[i] = ox[c];
    yint[i] = oy[c];
    Tint[i] = oT[c];
    xidx[i] = (int)round(ox[c]);
    yidx[i] = (int)round(oy[c]);
  } else {
    double xposnow = xint[i] + dxs[i];
    if (xposnow > (double)nx) xposnow = xposnow - (double)nx;
    if (xposnow < 0.0) xposnow = xposnow + (double)nx;
    xint[i] = xposnow;
    int bci = bc[i];
    double yposnow = yint[i] + dys[i];
    if (yposnow > (double)ny) { yposnow = yposnow - (double)ny + 1.0; bci = 2; }
    if (yposnow < 1.0) { yposnow = yposnow + (double)ny - 1.0; bci = 2; }
    yint[i] = yposnow;
    xidx[i] = (int)round(xposnow);
    yidx[i] = (int)round(yposnow);
    double Tnow = Tint[i] + dTs[i];
    if (bci == 1) Tnow = Tint[i];
    if (bci == 2) { Tnow = oT[chk[i]]; bci = 1; }
    Tint[i] = Tnow;
    bc[i] = bci;
  }
}

// after the file branch: the loaded file becomes the "last file"
__global__ void box_commit_file_kernel(const BoxView B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B.n) return;
  NB(B, NB_OX)[i] = NB(B, NB_FX)[i];
  NB(B, NB_OY)[i] = NB(B, NB_FY)[i];
  NB(B, NB_OT)[i] = NB(B, NB_FT)[i];
}

// node box of contribution (k, img), reference 1-based node coordinates of
// the whole domain, clipped to its interior; false when empty.  img 0: main 7x7 box; img 1:
// left periodic image (xidx < 4); img 2: right periodic image (xidx > nx-2).
__device__ __forceinline__ bool contrib_box(const BoxView& B, int k, int img, int& xa, int& xb,
                                            int& ya, int& yb) {
  const int xi = NBI(B, NBI_XIDX)[k], yi = NBI(B, NBI_YIDX)[k];
  if (img == 0) {
    xa = xi - 3; xb = xi + 3;
  } else if (img == 1) {
    if (!(xi < 4)) return false;
    xa = B.nx + xi - 3; xb = B.nx + xi;
  } else {
    if (!(xi > B.nx - 2)) return false;
    xa = xi - B.nx; xb = xi - B.nx + 3;
  }
  ya = yi - 3; yb = yi + 3;
  if (xa < 1) xa = 1;
  if (xb > B.nx) xb = B.nx;
  if (ya < 1) ya = 1;
  if (yb > B.nyT) yb = B.nyT;
  return xa <= xb && ya <= yb;
}

template <bool FILL>
__global__ void box_bin_kernel(const BoxView B) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * B.n) return;
  const int k = t / 3, img = t - 3 * k;
  int xa, xb, ya, yb;
  if (!contrib_box(B, k, img, xa, xb, ya, yb)) return;
  // the rows of this handle (a y-slab bins only what reaches its rows)
  ya = max(ya, B.j0 + 1);
  yb = min(yb, B.j0 + B.ny);
  if (ya > yb) return;
  const int ca = (xa - 1) / CELL, cb = (xb - 1) / CELL;
  const int ra = (ya - 1 - B.j0) / CELL, rb = (yb - 1 - B.j0) / CELL;
  for (int cy = ra; cy <= rb; cy++)
    for (int cx = ca; cx <= cb; cx++) {
      const int c = cy * B.ncx + cx;
      if (FILL) {
        const int slot = atomicAdd(&B.cell_fill[c], 1);
        B.items[B.cell_start[c] + slot] = t;
      } else {
        atomicAdd(&B.cell_count[c], 1);
      }
    }
}

// exclusive scan of cell_count into cell_start: one block
__global__ void __launch_bounds__(1024) scan_kernel(const int* __restrict__ in, int* __restrict__ out,
                                                    int n) {
  __shared__ int part[1024];
  const int tid = threadIdx.x;
  const int per = (n + 1023) / 1024;
  const int a = tid * per, b = min(n, a + per);
  int s = 0;
  for (int q = a; q < b; q++) s += in[q];
  part[tid] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  int run = part[tid] - s;
  for (int q = a; q < b; q++) {
    out[q] = run;
    run += in[q];
  }
}

// one block of CELL*CELL threads per cell: sort the cell's keys, then every
// node applies the running mean in key order
__global__ void __launch_bounds__(CELL * CELL) box_cells_kernel(const BoxView B) {
  const int c = blockIdx.x;
  const int cnt = B.cell_count[c];
  const int dirty = B.cell_dirty[c];
  if (cnt == 0 && !dirty) return;
  const int cx = c % B.ncx, cy = c / B.ncx;
  const int tid = threadIdx.x;
  const int i = cx * CELL + (tid % CELL) + 1;  // reference node coordinates (of the domain)
  const int j = B.j0 + cy * CELL + (tid / CELL) + 1;
  const int st = B.cell_start[c];
  // rank sort (keys are unique)
  for (int a = tid; a < cnt; a += blockDim.x) {
    const int key = B.items[st + a];
    int rank = 0;
    for (int b = 0; b < cnt; b++) rank += (B.items[st + b] < key);
    B.sorted[st + rank] = key;
  }
  __syncthreads();
  int nv = 0;
  double tri = 0.0;
  const double* Tint = NB(B, NB_TINT);
  for (int a = 0; a < cnt; a++) {
    const int key = B.sorted[st + a];
    const int k = key / 3, img = key - 3 * k;
    int xa, xb, ya, yb;
    if (!contrib_box(B, k, img, xa, xb, ya, yb)) continue;
    if (i >= xa && i <= xb && j >= ya && j <= yb) {
      tri = (tri * (double)nv + Tint[k]) / ((double)nv + 1.0);
      nv = nv + 1;
    }
  }
  if (i <= B.nx && j <= B.j0 + B.ny) {
    const size_t q = (size_t)(j - 1 - B.j0) * B.pitch + (i - 1);
    B.nudge_vol[q] = nv;
    B.tempreadint[q] = tri;
  }
  if (tid == 0) B.cell_dirty[c] = cnt > 0;
}

cudaError_t launch_box_nudge(double* nb, int* nbi, int n, int nx, int ny, int ny_total, int j0, int nt, int istep,
                             int ncx, int ncy, int* cell_count, int* cell_start, int* cell_fill,
                             int* cell_dirty, int* items, int* nudge_vol, double* tempreadint,
                             int pitch, unsigned* dflags, cudaStream_t s) {
  const int ncell = ncx * ncy;
  BoxView B{nb, nbi, n, nx, ny, nt, istep, ny_total, j0, ncx, ncy, cell_count, cell_start, cell_fill,
            cell_dirty, items, items + (size_t)n * 3 * 4, nudge_vol, tempreadint, pitch, dflags};
  const int tb = 128;
  box_interp_kernel<<<(n + tb - 1) / tb, tb, 0, s>>>(B);
  if (istep % nt == 1) box_commit_file_kernel<<<(n + tb - 1) / tb, tb, 0, s>>>(B);
  cudaMemsetAsync(cell_count, 0, sizeof(int) * ncell, s);
  cudaMemsetAsync(cell_fill, 0, sizeof(int) * ncell, s);
  box_bin_kernel<false><<<(3 * n + tb - 1) / tb, tb, 0, s>>>(B);
  scan_kernel<<<1, 1024, 0, s>>>(cell_count, cell_start, ncell);
  box_bin_kernel<true><<<(3 * n + tb - 1) / tb, tb, 0, s>>>(B);
  box_cells_kernel<<<ncell, CELL * CELL, 0, s>>>(B);
  return cudaGetLastError();
}

// ------------------------------------------------------------ bilinear mode
template <typename Real>
__global__ void obs_scatter_kernel(const Real* __restrict__ T, int nx, int ny, int pitch,
                                   const double* __restrict__ ox, const double* __restrict__ oy,
                                   const double* __restrict__ oT, int nobs, double alpha,
                                   unsigned long long* __restrict__ acc, unsigned* dflags) {
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nobs) return;
  obs_scatter_one(T, nx, ny, pitch, ox[p], oy[p], oT[p], alpha, acc, dflags);
}

template <typename Real>
__global__ void obs_apply_kernel(Real* __restrict__ g, size_t plane, int nx, int ny, int pitch,
                                 const double* __restrict__ ox, const double* __restrict__ oy,
                                 int nobs, unsigned long long* __restrict__ acc) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * nobs) return;
  const int p = t >> 2;
  obs_apply_one(g, plane, nx, ny, pitch, ox[p], oy[p], t & 3, acc);
}

// Two-step launch of a nudged run: step n's innovations before the launch
// (four threads per observation, obs_pre_corner in nudge_dev.cuh), and the
// clearing of their sums and mask bits after it
template <typename Real>
__global__ void __launch_bounds__(128) obs_pre4_kernel(const LBView<Real> V, const double* __restrict__ ox,
                                                       const double* __restrict__ oy, const double* __restrict__ oT,
                                                       int nobs, double alpha, unsigned long long* __restrict__ acc,
                                                       unsigned* __restrict__ mask, unsigned* dflags) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = t >> 2;
  const bool live = p < nobs;
  obs_pre_corner(V, live, live ? ox[p] : 0.0, live ? oy[p] : 0.0, live ? oT[p] : 0.0, alpha, t & 3, acc, mask,
                 dflags);
}

// after a nudged two-step launch: step n+1's apply pass (acc) and the
// clearing of step n's in-launch sums and mask bits (acc2, mask) in one
// launch -- corner t & 3 of observation t >> 2 of each step
template <typename Real>
__global__ void obs_apply_clear_kernel(Real* __restrict__ g, size_t plane, int nx, int ny, int pitch,
                                       const double* __restrict__ ox2, const double* __restrict__ oy2, int nobs,
                                       unsigned long long* __restrict__ acc, const double* __restrict__ ox1,
                                       const double* __restrict__ oy1, unsigned long long* __restrict__ acc2,
                                       unsigned* __restrict__ mask) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * nobs) return;
  const int p = t >> 2;
  obs_apply_one(g, plane, nx, ny, pitch, ox2[p], oy2[p], t & 3, acc);
  obs_clear_one(nx, ny, pitch, ox1[p], oy1[p], t & 3, acc2, mask);
}

cudaError_t launch_obs_pre_fp32(const LBView<float>& V, const double* ox, const double* oy, const double* oT,
                                int nobs, double alpha, long long* acc, unsigned* mask, unsigned* dflags,
                                cudaStream_t s, bool pdl) {
  if (nobs <= 0) return cudaSuccess;
  return launch_k(obs_pre4_kernel<float>, (4 * nobs + 127) / 128, 128, 0, s, pdl, V, ox, oy, oT, nobs, alpha,
                  reinterpret_cast<unsigned long long*>(acc), mask, dflags);
}
cudaError_t launch_obs_pre_fp64(const LBView<double>& V, const double* ox, const double* oy, const double* oT,
                                int nobs, double alpha, long long* acc, unsigned* mask, unsigned* dflags,
                                cudaStream_t s, bool pdl) {
  if (nobs <= 0) return cudaSuccess;
  return launch_k(obs_pre4_kernel<double>, (4 * nobs + 127) / 128, 128, 0, s, pdl, V, ox, oy, oT, nobs, alpha,
                  reinterpret_cast<unsigned long long*>(acc), mask, dflags);
}
cudaError_t launch_bilinear_nudge_clear(void* T, void* g, bool fp32, size_t plane, int nx, int ny, int pitch,
                                        const double* ox, const double* oy, const double* oT, int nobs, double alpha,
                                        long long* acc, const double* ox1, const double* oy1, long long* acc2,
                                        unsigned* mask, unsigned* dflags, cudaStream_t s, bool pdl) {
  if (nobs <= 0) return cudaSuccess;
  const int tb = 128;
  unsigned long long* a = reinterpret_cast<unsigned long long*>(acc);
  unsigned long long* a2 = reinterpret_cast<unsigned long long*>(acc2);
  auto go = [&](auto zero) -> cudaError_t {
    using Real = decltype(zero);
    cudaError_t e = launch_k(obs_scatter_kernel<Real>, (nobs + tb - 1) / tb, tb, 0, s, pdl, (const Real*)T, nx, ny,
                             pitch, ox, oy, oT, nobs, alpha, a, dflags);
    if (e != cudaSuccess) return e;
    return launch_k(obs_apply_clear_kernel<Real>, (4 * nobs + tb - 1) / tb, tb, 0, s, pdl, (Real*)g, plane, nx, ny,
                    pitch, ox, oy, nobs, a, ox1, oy1, a2, mask);
  };
  return fp32 ? go(0.f) : go(0.0);
}

// y-slab: the observations' innovations read T of the whole domain through
// a table of row pointers (one per global row); the slab scatters to and
// applies at the corners in its own rows only
template <typename Real>
__global__ void obs_scatter_slab_kernel(const Real* const* __restrict__ Trow, int nx, int ny_total, int pitch,
                                        const double* __restrict__ ox, const double* __restrict__ oy,
                                        const double* __restrict__ oT, int nobs, double alpha,
                                        unsigned long long* __restrict__ acc, unsigned* dflags, int j0, int nyl) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nobs) return;
  obs_scatter_rows([&](int j, int i) { return Trow[j][i]; }, nx, ny_total, pitch, ox[p], oy[p], oT[p], alpha, acc,
                   dflags, j0, nyl);
}

template <typename Real>
__global__ void obs_apply_slab_kernel(Real* __restrict__ g, size_t plane, int nx, int ny_total, int pitch,
                                      const double* __restrict__ ox, const double* __restrict__ oy, int nobs,
                                      unsigned long long* __restrict__ acc, int j0, int nyl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * nobs) return;
  const int p = t >> 2;
  obs_apply_one(g, plane, nx, ny_total, pitch, ox[p], oy[p], t & 3, acc, j0, nyl);
}

cudaError_t launch_bilinear_nudge_slab(const void* Trows, void* g, bool fp32, size_t plane, int nx, int ny_total,
                                       int j0, int nyl, int pitch, const double* ox, const double* oy,
                                       const double* oT, int nobs, double alpha, long long* acc, unsigned* dflags,
                                       cudaStream_t s) {
  if (nobs <= 0) return cudaSuccess;
  const int tb = 128;
  unsigned long long* a = reinterpret_cast<unsigned long long*>(acc);
  auto go = [&](auto zero) {
    using Real = decltype(zero);
    obs_scatter_slab_kernel<Real><<<(nobs + tb - 1) / tb, tb, 0, s>>>(
        (const Real* const*)Trows, nx, ny_total, pitch, ox, oy, oT, nobs, alpha, a, dflags, j0, nyl);
    obs_apply_slab_kernel<Real><<<(4 * nobs + tb - 1) / tb, tb, 0, s>>>((Real*)g, plane, nx, ny_total, pitch, ox,
                                                                       oy, nobs, a, j0, nyl);
  };
  if (fp32) go(0.f);
  else go(0.0);
  return cudaGetLastError();
}

cudaError_t launch_bilinear_nudge(void* T, void* g, bool fp32, size_t plane, int nx, int ny,
                                  int pitch, const double* ox, const double* oy, const double* oT,
                                  int nobs, double alpha, long long* acc, unsigned* dflags,
                                  cudaStream_t s, bool pdl) {
  if (nobs <= 0) return cudaSuccess;
  const int tb = 128;
  unsigned long long* a = reinterpret_cast<unsigned long long*>(acc);
  auto go = [&](auto zero) -> cudaError_t {
    using Real = decltype(zero);
    cudaError_t e = launch_k(obs_scatter_kernel<Real>, (nobs + tb - 1) / tb, tb, 0, s, pdl, (const Real*)T, nx, ny,
                             pitch, ox, oy, oT, nobs, alpha, a, dflags);
    if (e != cudaSuccess) return e;
    return launch_k(obs_apply_kernel<Real>, (4 * nobs + tb - 1) / tb, tb, 0, s, pdl, (Real*)g, plane, nx, ny, pitch,
                    ox, oy, nobs, a);
  };
  return fp32 ? go(0.f) : go(0.0);
}

}  // namespace lbrb
