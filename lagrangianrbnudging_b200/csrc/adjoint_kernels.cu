// adjoint_kernels.cu -- hand-written adjoint of the time step, for the
// gradient of a trajectory-temperature misfit with respect to the initial
// temperature field.  No counterpart in the reference.
//
// Forward step n (Dirichlet walls, as lb_node_kernel): pull the previous
// post-collision populations (bounce-back / anti-bounce-back at the walls),
// moments rho, j, T with the buoyancy F^n = g*beta rho^{n-1} T^{n-1}, BGK +
// Guo collision, and F^{n+1} = g*beta rho^n T^n.  In the shifted variables
// df_k = f_k - w_k, dg_k = g_k - w_k T0 (the same mathematics as the
// reference-order FP64 arithmetic):
//   dr = sum df, r = 1 + dr, jx = sum cx df, jy = sum cy df
//   u = jx / r,  v = (jy + F/2) / r,  dT = sum dg,  t = T0 + dT
//   cu_k = c_k.u,  P_k = 3 cu + 4.5 cu^2 - 1.5 |u|^2
//   df'_k = (1-w) df_k + w w_k (dr + r P_k) + (1-w/2) w_k F (3 (cy_k - v) + 9 cu_k cy_k)
//   dg'_k = (1-wg) dg_k + wg w_k (dT + t P_k)
//   F' = g*beta r t
// The adjoint kernel of step n, one thread per node x: re-pull the forward
// state at x, apply the transposed local Jacobian to the adjoints of the
// step's outputs at x (lambda df', dg', F', plus the observation term on T),
// fold the anti-bounce-back transpose, and push the results to the nodes the
// forward pulled from (the transpose of streaming: bounce-back sends the
// adjoint to the opposite population of the same node; populations that
// stream out of the domain get zero).  Adjoints are FP64.
#include <type_traits>

#include "lbrb_internal.cuh"

namespace lbrb {

template <typename Real>
struct AdjView {
  const Real* __restrict__ fsrc;  // forward state before the step (18 planes)
  const Real* __restrict__ gsrc;
  const Real* __restrict__ Fin;   // F of the step
  const double* __restrict__ lf_out;  // lambda of the step's post-collision output
  const double* __restrict__ lg_out;
  double* __restrict__ lf_in;     // lambda of the step's input (pushed)
  double* __restrict__ lg_in;
  double* __restrict__ lF;        // in: lambda F^{n+1}; out: lambda F^n (same node)
  long long* __restrict__ lT;     // fixed-point lambda T of this step, or null; cleared
  int nx, ny, pitch;
  size_t plane;
  double omega, omegag, gbeta, T0, Tup, Tdown;
};

constexpr double ADJ_FIX = 1099511627776.0;  // 2^40

template <typename Real>
__device__ __forceinline__ void adj_pull(const AdjView<Real>& V, int j, int x, double* df, double* dg) {
  const int xl = (x == 0) ? V.nx - 1 : x - 1;
  const int xr = (x == V.nx - 1) ? 0 : x + 1;
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    const int xs = icx(k) == 1 ? xl : (icx(k) == -1 ? xr : x);
    const int js = j - icy(k);
    double fv, gv;
    if (js < 0 || js >= V.ny) {
      fv = (double)V.fsrc[(size_t)opp(k) * V.plane + (size_t)j * V.pitch + x];
      gv = 0.0;
    } else {
      fv = (double)V.fsrc[(size_t)k * V.plane + (size_t)js * V.pitch + xs];
      gv = (double)V.gsrc[(size_t)k * V.plane + (size_t)js * V.pitch + xs];
    }
    if constexpr (std::is_same<Real, double>::value) {
      // reference-order storage holds f, g themselves: go to the shifted form
      df[k] = fv - w_of(k);
      dg[k] = (js < 0 || js >= V.ny) ? 0.0 : gv - w_of(k) * V.T0;
    } else {
      df[k] = fv;
      dg[k] = gv;
    }
  }
  // anti-bounce-back on the shifted form: dg_in = -dg_opp + 2 w (Twall - T0)
  if (j == V.ny - 1) {
    const double tw = V.Tup - V.T0;
    dg[4] = -dg[2] + 2.0 * w_of(2) * tw;
    dg[7] = -dg[5] + 2.0 * w_of(5) * tw;
    dg[8] = -dg[6] + 2.0 * w_of(6) * tw;
  }
  if (j == 0) {
    const double tw = V.Tdown - V.T0;
    dg[2] = -dg[4] + 2.0 * w_of(4) * tw;
    dg[5] = -dg[7] + 2.0 * w_of(7) * tw;
    dg[6] = -dg[8] + 2.0 * w_of(8) * tw;
  }
}

template <typename Real>
__global__ void __launch_bounds__(128) adjoint_step_kernel(const AdjView<Real> V) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (x >= V.nx) return;
  const size_t o = (size_t)j * V.pitch + x;
  double df[NPOP], dg[NPOP];
  adj_pull(V, j, x, df, dg);
  // forward local quantities
  double dr = 0.0, dT = 0.0, jx = 0.0, jy = 0.0;
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    dr += df[k];
    dT += dg[k];
    jx += icx(k) * df[k];
    jy += icy(k) * df[k];
  }
  const double r = 1.0 + dr, t = V.T0 + dT;
  const double F = (double)V.Fin[o];
  const double u = jx / r, v = (jy + 0.5 * F) / r;
  const double om = V.omega, omg = V.omegag, srcf = 1.0 - 0.5 * om;
  // adjoints of the outputs
  double lfo[NPOP], lgo[NPOP];
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    lfo[k] = V.lf_out[(size_t)k * V.plane + o];
    lgo[k] = V.lg_out[(size_t)k * V.plane + o];
  }
  const double lFo = V.lF[o];
  double lt = 0.0;
  if (V.lT) {
    const long long q = V.lT[o];
    lt = (double)q * (1.0 / ADJ_FIX);
    if (q != 0) V.lT[o] = 0;
  }
  // transposed local Jacobian
  double lu = 0.0, lv = 0.0, ldr = 0.0, ldT = 0.0, lFin = 0.0;
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    const double w = w_of(k), cx = icx(k), cy = icy(k);
    const double cu = cx * u + cy * v;
    const double P = 3.0 * cu + 4.5 * cu * cu - 1.5 * (u * u + v * v);
    const double A = om * lfo[k];   // lambda of df_eq
    const double B = omg * lgo[k];  // lambda of dg_eq
    const double lP = A * w * r + B * w * t;
    const double lS = lfo[k] * srcf * w;  // lambda of S / (srcf w) scale folded
    const double lcu = lP * (3.0 + 9.0 * cu) + lS * F * 9.0 * cy;
    lu += lcu * cx - lP * 3.0 * u;
    lv += lcu * cy - lP * 3.0 * v - lS * F * 3.0;
    ldr += A * w * (1.0 + P);
    ldT += B * w * (1.0 + P);
    lFin += lS * (3.0 * (cy - v) + 9.0 * cu * cy);
  }
  lFin += lv * 0.5 / r;
  const double lt_tot = lt + lFo * V.gbeta * r;
  const double lr = lFo * V.gbeta * t - (lu * u + lv * v) / r;
  const double ljx = lu / r, ljy = lv / r;
  ldr += lr;
  ldT += lt_tot;
  double lfs[NPOP], lgs[NPOP];
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    lfs[k] = (1.0 - om) * lfo[k] + ldr + icx(k) * ljx + icy(k) * ljy;
    lgs[k] = (1.0 - omg) * lgo[k] + ldT;
  }
  // anti-bounce-back transpose: the replaced population feeds its opposite
  if (j == V.ny - 1) {
    lgs[2] -= lgs[4]; lgs[4] = 0.0;
    lgs[5] -= lgs[7]; lgs[7] = 0.0;
    lgs[6] -= lgs[8]; lgs[8] = 0.0;
  }
  if (j == 0) {
    lgs[4] -= lgs[2]; lgs[2] = 0.0;
    lgs[7] -= lgs[5]; lgs[5] = 0.0;
    lgs[8] -= lgs[6]; lgs[6] = 0.0;
  }
  // transpose of the pull
  const int xl = (x == 0) ? V.nx - 1 : x - 1;
  const int xr = (x == V.nx - 1) ? 0 : x + 1;
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    const int xs = icx(k) == 1 ? xl : (icx(k) == -1 ? xr : x);
    const int js = j - icy(k);
    if (js < 0 || js >= V.ny) {
      V.lf_in[(size_t)opp(k) * V.plane + o] = lfs[k];  // bounce-back source
      V.lg_in[(size_t)opp(k) * V.plane + o] = 0.0;     // streams out, never read
    } else {
      const size_t os = (size_t)js * V.pitch + xs;
      V.lf_in[(size_t)k * V.plane + os] = lfs[k];
      V.lg_in[(size_t)k * V.plane + os] = lgs[k];
    }
  }
  V.lF[o] = lFin;
}

// observation adjoint of step n: lambda T += 2 r_p w_corner, fixed point
__global__ void adj_obs_scatter_kernel(const double* __restrict__ ox, const double* __restrict__ oy,
                                       const double* __restrict__ res, int nobs, int nx, int ny,
                                       int pitch, unsigned long long* __restrict__ acc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nobs) return;
  const double xx = ox[p], yy = oy[p];
  if (!(xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0)) return;
  const int x1 = (int)xx, y1 = (int)yy, x2 = x1 + 1, y2 = y1 + 1;
  int ix1 = (x1 - 1) % nx; if (ix1 < 0) ix1 += nx;
  int ix2 = (x2 - 1) % nx; if (ix2 < 0) ix2 += nx;
  int jy1 = (y1 - 1) % ny; if (jy1 < 0) jy1 += ny;
  int jy2 = (y2 - 1) % ny; if (jy2 < 0) jy2 += ny;
  const double g = 2.0 * res[p];
  const double wx1 = (double)x2 - xx, wx2 = xx - (double)x1;
  const double wy1 = (double)y2 - yy, wy2 = yy - (double)y1;
  atomicAdd(&acc[(size_t)jy1 * pitch + ix1], (unsigned long long)__double2ll_rn(g * wx1 * wy1 * ADJ_FIX));
  atomicAdd(&acc[(size_t)jy1 * pitch + ix2], (unsigned long long)__double2ll_rn(g * wx2 * wy1 * ADJ_FIX));
  atomicAdd(&acc[(size_t)jy2 * pitch + ix1], (unsigned long long)__double2ll_rn(g * wx1 * wy2 * ADJ_FIX));
  atomicAdd(&acc[(size_t)jy2 * pitch + ix2], (unsigned long long)__double2ll_rn(g * wx2 * wy2 * ADJ_FIX));
}

// residuals r_p = T(x_p) - T_obs,p of one observation step (forward)
template <typename Real>
__global__ void obs_residual_kernel(const Real* __restrict__ T, int nx, int ny, int pitch,
                                    const double* __restrict__ ox, const double* __restrict__ oy,
                                    const double* __restrict__ oT, int nobs, double* __restrict__ res) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nobs) return;
  const double xx = ox[p], yy = oy[p];
  if (!(xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0)) { res[p] = 0.0; return; }
  const int x1 = (int)xx, y1 = (int)yy, x2 = x1 + 1, y2 = y1 + 1;
  int ix1 = (x1 - 1) % nx; if (ix1 < 0) ix1 += nx;
  int ix2 = (x2 - 1) % nx; if (ix2 < 0) ix2 += nx;
  int jy1 = (y1 - 1) % ny; if (jy1 < 0) jy1 += ny;
  int jy2 = (y2 - 1) % ny; if (jy2 < 0) jy2 += ny;
  const double u11 = (double)T[(size_t)jy1 * pitch + ix1], u12 = (double)T[(size_t)jy2 * pitch + ix1];
  const double u21 = (double)T[(size_t)jy1 * pitch + ix2], u22 = (double)T[(size_t)jy2 * pitch + ix2];
  const double tm = u11 * ((double)x2 - xx) * ((double)y2 - yy) + u21 * (xx - (double)x1) * ((double)y2 - yy) +
                    u12 * ((double)x2 - xx) * (yy - (double)y1) + u22 * (xx - (double)x1) * (yy - (double)y1);
  res[p] = tm - oT[p];
}

// initial state from a temperature field T0 (f = feq(1,0), g = geq(T0,0),
// moments by the restart route), as lbrb_init_conduction without the profile
template <typename Real>
__global__ void init_from_T0_kernel(const double* __restrict__ T0f, Real* __restrict__ pops,
                                    Real* __restrict__ rho, Real* __restrict__ u, Real* __restrict__ v,
                                    Real* __restrict__ T, Real* __restrict__ F, int nx, int ny,
                                    int pitch, size_t plane, double Tref, double neg_gravity) {
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const size_t o = (size_t)j * pitch + i;
    const double t = T0f[q];
    double feq[NPOP], geq[NPOP];
    equil_ref(1.0, 0.0, 0.0, feq);
    equil_ref(t, 0.0, 0.0, geq);
    double r = 0.0, tt = 0.0;
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      r = r + feq[k];
      if constexpr (std::is_same<Real, double>::value) {
        pops[(size_t)k * plane + o] = feq[k];
        pops[(size_t)(k + NPOP) * plane + o] = geq[k];
      } else {
        pops[(size_t)k * plane + o] = (float)(feq[k] - w_of(k));
        pops[(size_t)(k + NPOP) * plane + o] = (float)(geq[k] - w_of(k) * Tref);
      }
    }
#pragma unroll
    for (int k = 0; k < NPOP; k++) tt = tt + geq[k];
    const double rhoi = 1. / r;
    double fl[NPOP];
#pragma unroll
    for (int k = 0; k < NPOP; k++) fl[k] = feq[k] * rhoi;
    rho[o] = (Real)r;
    T[o] = (Real)tt;
    u[o] = (Real)(fl[1] - fl[3] + fl[5] - fl[6] - fl[7] + fl[8]);
    v[o] = (Real)(fl[5] + fl[2] + fl[6] - fl[7] - fl[4] - fl[8] + (0.5 * neg_gravity * tt));
    if constexpr (std::is_same<Real, double>::value) F[o] = neg_gravity * r * (tt - 0.0);
    else F[o] = (float)neg_gravity * (float)r * (float)tt;
  }
}

// gradient with respect to T0: sum_k w_k lambda g_k^0 + g*beta rho^0 (sum_k w_k) lambda F^1
__global__ void adj_initial_kernel(const double* __restrict__ lg, const double* __restrict__ lF,
                                   int nx, int ny, int pitch, size_t plane, double gbeta,
                                   double* __restrict__ out) {
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const size_t o = (size_t)j * pitch + i;
    double s = 0.0, sw = 0.0, r0 = 0.0, feq[NPOP];
    equil_ref(1.0, 0.0, 0.0, feq);
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      s += w_of(k) * lg[(size_t)k * plane + o];
      sw += w_of(k);
      r0 = r0 + feq[k];
    }
    out[q] = s + gbeta * r0 * sw * lF[o];
  }
}

// ---------------------------------------------------------------- launchers
template <typename Real>
static cudaError_t launch_adj_t(const AdjView<Real>& V, cudaStream_t s) {
  dim3 grid((V.nx + 127) / 128, V.ny);
  adjoint_step_kernel<Real><<<grid, 128, 0, s>>>(V);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_step(bool fp32, const void* fsrc, const void* gsrc, const void* Fin,
                                const double* lf_out, const double* lg_out, double* lf_in,
                                double* lg_in, double* lF, long long* lT, int nx, int ny, int pitch,
                                size_t plane, double omega, double omegag, double gbeta, double T0,
                                double Tup, double Tdown, cudaStream_t s) {
  if (fp32) {
    AdjView<float> V{(const float*)fsrc, (const float*)gsrc, (const float*)Fin, lf_out, lg_out, lf_in,
                     lg_in, lF, lT, nx, ny, pitch, plane, omega, omegag, gbeta, T0, Tup, Tdown};
    return launch_adj_t(V, s);
  }
  AdjView<double> V{(const double*)fsrc, (const double*)gsrc, (const double*)Fin, lf_out, lg_out, lf_in,
                    lg_in, lF, lT, nx, ny, pitch, plane, omega, omegag, gbeta, T0, Tup, Tdown};
  return launch_adj_t(V, s);
}

cudaError_t launch_adj_obs_scatter(const double* ox, const double* oy, const double* res, int nobs,
                                   int nx, int ny, int pitch, long long* acc, cudaStream_t s) {
  if (nobs <= 0) return cudaSuccess;
  adj_obs_scatter_kernel<<<(nobs + 127) / 128, 128, 0, s>>>(ox, oy, res, nobs, nx, ny, pitch,
                                                            reinterpret_cast<unsigned long long*>(acc));
  return cudaGetLastError();
}

cudaError_t launch_obs_residual(const void* T, bool fp32, int nx, int ny, int pitch, const double* ox,
                                const double* oy, const double* oT, int nobs, double* res,
                                cudaStream_t s) {
  if (nobs <= 0) return cudaSuccess;
  if (fp32)
    obs_residual_kernel<float><<<(nobs + 127) / 128, 128, 0, s>>>((const float*)T, nx, ny, pitch, ox, oy, oT, nobs, res);
  else
    obs_residual_kernel<double><<<(nobs + 127) / 128, 128, 0, s>>>((const double*)T, nx, ny, pitch, ox, oy, oT, nobs, res);
  return cudaGetLastError();
}

cudaError_t launch_init_from_T0(const double* T0f, void* pops, void* rho, void* u, void* v, void* T,
                                void* F, bool fp32, int nx, int ny, int pitch, size_t plane,
                                double Tref, double neg_gravity, cudaStream_t s) {
  const int g = 148 * 8;
  if (fp32)
    init_from_T0_kernel<float><<<g, 256, 0, s>>>(T0f, (float*)pops, (float*)rho, (float*)u, (float*)v,
                                                 (float*)T, (float*)F, nx, ny, pitch, plane, Tref, neg_gravity);
  else
    init_from_T0_kernel<double><<<g, 256, 0, s>>>(T0f, (double*)pops, (double*)rho, (double*)u, (double*)v,
                                                  (double*)T, (double*)F, nx, ny, pitch, plane, Tref, neg_gravity);
  return cudaGetLastError();
}

cudaError_t launch_adj_initial(const double* lg, const double* lF, int nx, int ny, int pitch,
                               size_t plane, double gbeta, double* out, cudaStream_t s) {
  adj_initial_kernel<<<148 * 8, 256, 0, s>>>(lg, lF, nx, ny, pitch, plane, gbeta, out);
  return cudaGetLastError();
}

}  // namespace lbrb
