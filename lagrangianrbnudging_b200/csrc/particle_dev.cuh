// particle_dev.cuh -- one Lagrangian particle of one step, shared by the
// single-run particle kernel (particle_kernels.cu) and the ensemble kernels
// (ensemble_kernels.cu).  Reference semantics: see particle_kernels.cu.
#pragma once

#include "lbrb_internal.cuh"

namespace lbrb {

template <typename Real>
struct PView {
  const Real* __restrict__ u;
  const Real* __restrict__ v;
  const Real* __restrict__ ub;
  const Real* __restrict__ vb;
  const Real* __restrict__ T;
  int nx, ny, pitch;
  double* __restrict__ P;  // [9][np]: x y u v xo yo uo vo invtau
  const int* __restrict__ ptype;
  int np;
  double beta;
  int record;              // this step writes a record
  int full;                // also the 8 Writefull fields
  double* __restrict__ rec;  // ring slot base, [fields][np]
  unsigned* dflags;
  // y-slabs of one domain: for each global row, a pointer to that row of u,
  // v, ub, vb and T in the slab that holds it (nx, ny are then the whole
  // domain's); null for a whole domain in one handle
  const Real* const* __restrict__ urow;
  const Real* const* __restrict__ vrow;
  const Real* const* __restrict__ ubrow;
  const Real* const* __restrict__ vbrow;
  const Real* const* __restrict__ Trow;
};

// value of a field at row j, column i: one plane (ROWS = false) or a table of
// row pointers (ROWS = true, a domain held as y-slabs)
template <bool ROWS, typename Real>
__device__ __forceinline__ Real fat(const Real* __restrict__ f, const Real* const* __restrict__ rows, int pitch,
                                    int j, int i) {
  if constexpr (ROWS) return rows[j][i];
  else return f[(size_t)j * pitch + i];
}

__device__ __forceinline__ int wrapi(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

// Cell of a reference-frame position: corners (x1, y1), (x1+1, y1+1) and
// their device indices after periodic wrap.  Flags positions that could not
// come from a finite run (the reference would read out of its arrays).
struct Cell {
  int x1, y1;
  int ix[2], jy[2];
};

__device__ __forceinline__ bool make_cell(double xx, double yy, int nx, int ny, Cell& c,
                                          unsigned* dflags) {
  bool ok = (xx > -2.0) && (xx < nx + 2.0) && (yy > -2.0) && (yy < ny + 2.0);
  if (!ok) {
    atomicOr(dflags, isfinite(xx) && isfinite(yy) ? DFLAG_RANGE : DFLAG_NONFINITE);
    xx = 1.0;
    yy = 1.0;
  }
  c.x1 = (int)xx;
  c.y1 = (int)yy;
  c.ix[0] = wrapi(c.x1 - 1, nx);
  c.ix[1] = wrapi(c.x1, nx);
  c.jy[0] = wrapi(c.y1 - 1, ny);
  c.jy[1] = wrapi(c.y1, ny);
  return ok;
}

__device__ __forceinline__ double bil_combine(const Cell& c, double xx, double yy, double u11,
                                              double u12, double u21, double u22) {
  const int x2 = c.x1 + 1, y2 = c.y1 + 1;
  double val1 = u11 * ((double)x2 - xx) * ((double)y2 - yy);
  double val2 = u21 * (xx - (double)c.x1) * ((double)y2 - yy);
  double val3 = u12 * ((double)x2 - xx) * (yy - (double)c.y1);
  double val4 = u22 * (xx - (double)c.x1) * (yy - (double)c.y1);
  return val1 + val2 + val3 + val4;
}

template <bool ROWS = false, typename Real>
__device__ __forceinline__ double bilin(const Real* __restrict__ f, const Real* const* rows, int pitch,
                                        const Cell& c, double xx, double yy) {
  double u11 = (double)fat<ROWS>(f, rows, pitch, c.jy[0], c.ix[0]);
  double u12 = (double)fat<ROWS>(f, rows, pitch, c.jy[1], c.ix[0]);
  double u21 = (double)fat<ROWS>(f, rows, pitch, c.jy[0], c.ix[1]);
  double u22 = (double)fat<ROWS>(f, rows, pitch, c.jy[1], c.ix[1]);
  return bil_combine(c, xx, yy, u11, u12, u21, u22);
}

// derivative terms at one device node (i, j): dt, dx, dy of u and v
template <bool ROWS = false, typename Real>
__device__ __forceinline__ void node_derivs(const PView<Real>& V, int i, int j, double d[6]) {
  const int nx = V.nx, ny = V.ny, pitch = V.pitch;
  auto U = [&](int jj, int ii) { return (double)fat<ROWS>(V.u, V.urow, pitch, jj, ii); };
  auto W = [&](int jj, int ii) { return (double)fat<ROWS>(V.v, V.vrow, pitch, jj, ii); };
  const int ir = wrapi(i + 1, nx), il = wrapi(i - 1, nx);
  const int jt = wrapi(j + 1, ny), jb = wrapi(j - 1, ny);
  const double uq = U(j, i), vq = W(j, i);
  d[0] = uq - (double)fat<ROWS>(V.ub, V.ubrow, pitch, j, i);
  d[1] = vq - (double)fat<ROWS>(V.vb, V.vbrow, pitch, j, i);
  d[2] = (U(j, ir) - U(j, il)) * 0.5;
  d[3] = (W(j, ir) - W(j, il)) * 0.5;
  if (j == 0) {
    d[4] = (U(jt, i) - uq);
    d[5] = (W(jt, i) - vq);
  } else if (j == ny - 1) {
    d[4] = (uq - U(jb, i));
    d[5] = (vq - W(jb, i));
  } else {
    d[4] = (U(jt, i) - U(jb, i)) * 0.5;
    d[5] = (W(jt, i) - W(jb, i)) * 0.5;
  }
}

// bilinear of the six derivative fields over one cell
template <bool ROWS = false, typename Real>
__device__ __forceinline__ void bilin_derivs(const PView<Real>& V, const Cell& c, double xx,
                                             double yy, double out[6]) {
  double d11[6], d12[6], d21[6], d22[6];
  node_derivs<ROWS>(V, c.ix[0], c.jy[0], d11);
  node_derivs<ROWS>(V, c.ix[0], c.jy[1], d12);
  node_derivs<ROWS>(V, c.ix[1], c.jy[0], d21);
  node_derivs<ROWS>(V, c.ix[1], c.jy[1], d22);
#pragma unroll
  for (int w = 0; w < 6; w++) out[w] = bil_combine(c, xx, yy, d11[w], d12[w], d21[w], d22[w]);
}

// one particle of one step: interpolate, advance, record, wrap/reflect
// DERIVS = false: the run needs no Maxey-Riley derivative terms (beta == 0
// and no full records), so the 4x4 derivative stencil is not compiled in.
// ROWS: the fields are read through the view's row tables (y-slabs).
template <typename Real, bool DERIVS = true, bool ROWS = false>
__device__ __forceinline__ void particle_update(const PView<Real>& V, int p) {
  const int n = V.np;
  double* X = V.P;
  const double delta_t = 1.0;
  const double xx = X[0 * n + p], yy = X[1 * n + p];
  const double uold = X[2 * n + p], vold = X[3 * n + p];
  const double invtau = X[8 * n + p];
  Cell c;
  make_cell(xx, yy, V.nx, V.ny, c, V.dflags);
  const double tempup = bilin<ROWS>(V.u, V.urow, V.pitch, c, xx, yy);
  const double tempvp = bilin<ROWS>(V.v, V.vrow, V.pitch, c, xx, yy);
  const bool tracer = V.ptype[p] == LBRB_PTYPE_TRACER;
  const bool need_d = (!tracer && V.beta != 0.0) || (V.record && V.full);
  double dd[6] = {0, 0, 0, 0, 0, 0};
  if (DERIVS && need_d) bilin_derivs<ROWS>(V, c, xx, yy, dd);
  double xn, yn, un, vn;
  if (tracer) {
    xn = xx + 1.5 * delta_t * tempup - 0.5 * delta_t * uold;
    yn = yy + 1.5 * delta_t * tempvp - 0.5 * delta_t * vold;
    un = tempup;
    vn = tempvp;
  } else {
    const double beta = V.beta;
    un = uold + delta_t * (beta * (dd[0] + tempup * dd[2] + tempvp * dd[4]) - invtau * (uold - tempup));
    vn = vold + delta_t * (beta * (dd[1] + tempup * dd[3] + tempvp * dd[5]) - invtau * (vold - tempvp));
    xn = xx + delta_t * un;
    yn = yy + delta_t * vn;
  }
  if (V.record) {
    double* r = V.rec;
    r[LBRB_REC_X * n + p] = 0.0 + xn;
    r[LBRB_REC_Y * n + p] = 0.0 + yn;
    r[LBRB_REC_U * n + p] = un;
    r[LBRB_REC_V * n + p] = vn;
    r[LBRB_REC_XO * n + p] = 0.0 + xx;
    r[LBRB_REC_YO * n + p] = 0.0 + yy;
    r[LBRB_REC_UO * n + p] = uold;
    r[LBRB_REC_VO * n + p] = vold;
    Cell cn;
    make_cell(xn, yn, V.nx, V.ny, cn, V.dflags);
    r[LBRB_REC_TEMP * n + p] = bilin<ROWS>(V.T, V.Trow, V.pitch, cn, xn, yn);
    if (V.full) {
      // Writefull terms at (xo, yo): the cell this step started in
      r[LBRB_REC_DTU * n + p] = dd[0];
      r[LBRB_REC_DTV * n + p] = dd[1];
      r[LBRB_REC_DXU * n + p] = dd[2];
      r[LBRB_REC_DXV * n + p] = dd[3];
      r[LBRB_REC_DYU * n + p] = dd[4];
      r[LBRB_REC_DYV * n + p] = dd[5];
      r[LBRB_REC_FU * n + p] = tempup;
      r[LBRB_REC_FV * n + p] = tempvp;
    }
  }
  // toggle_prtcl: periodic x, mirror y about 1 and NY with v -> -v
  const double NXd = (double)V.nx, NYd = (double)V.ny;
  if (xn >= NXd) xn = xn - NXd;
  else if (xn <= 0.0) xn = xn + NXd;
  if (yn < 1.0) {
    yn = yn + 2.0 * (1.0 - yn);
    vn = -vn;
  } else if (yn >= NYd) {
    yn = yn + 2.0 * (NYd - yn);
    vn = -vn;
  }
  X[0 * n + p] = xn;
  X[1 * n + p] = yn;
  X[2 * n + p] = un;
  X[3 * n + p] = vn;
  X[4 * n + p] = xx;
  X[5 * n + p] = yy;
  X[6 * n + p] = uold;
  X[7 * n + p] = vold;
}


}  // namespace lbrb
