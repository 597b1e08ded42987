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
