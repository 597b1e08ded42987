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
// A domain held as y-slabs: every slab holds all particles.  Each step, the
// slab whose rows hold a particle's cell (its position before the step)
// advances it, reading the fields through the view's row tables; every slab
// notes that owner.  The merge then copies each particle it did not own (and,
// on record steps, its record) from its owner.  (The reference keeps each
// rank's particles in that rank and sends those that leave its rows to the
// neighbour, toggle_prtcl in Trajectories/code/mympi2.h:568-760; replicated
// arrays need no compaction and keep the whole domain's particle order.)
__device__ __forceinline__ int cell_row(double yy, int ny) {
  if (!(yy > -2.0 && yy < ny + 2.0)) return 0;  // (flagged by make_cell)
  return wrapi((int)yy - 1, ny);
}

template <typename Real, bool DERIVS>
__global__ void __launch_bounds__(128)
    particle_slab_kernel(const PView<Real> V, const int* __restrict__ slab_of_row, int me, int* __restrict__ own) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= V.np) return;
  const int o = slab_of_row[cell_row(V.P[V.np + p], V.ny)];
  own[p] = o;
  if (o != me) return;
  particle_update<Real, DERIVS, true>(V, p);
}

__global__ void __launch_bounds__(128)
    particle_merge_kernel(double* __restrict__ P, int np, const int* __restrict__ own, int me,
                          const double* const* __restrict__ Ps, double* __restrict__ rec,
                          const double* const* __restrict__ recs, size_t rec_off, int nrec) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int o = own[p];
  if (o == me) return;
  const double* Q = Ps[o];
#pragma unroll
  for (int k = 0; k < 8; k++) P[(size_t)k * np + p] = Q[(size_t)k * np + p];
  if (rec) {
    const double* R = recs[o] + rec_off;
    for (int f = 0; f < nrec; f++) rec[(size_t)f * np + p] = R[(size_t)f * np + p];
  }
}

cudaError_t launch_particles_slab(const void* u, const void* v, const void* ub, const void* vb, const void* T,
                                  const void* const* rows5, bool fp32, int nx, int ny_total, int pitch,
                                  double* P, const int* ptype, int np, double beta, int record, int full,
                                  double* rec, unsigned* dflags, const int* slab_of_row, int me, int* own,
                                  cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  const int g = (np + 127) / 128;
  auto go = [&](auto zero) -> cudaError_t {
    using Real = decltype(zero);
    using Rows = const Real* const*;
    PView<Real> V{(const Real*)u, (const Real*)v, (const Real*)ub, (const Real*)vb, (const Real*)T, nx, ny_total,
                  pitch, P, ptype, np, beta, record, full, rec, dflags, (Rows)rows5[0], (Rows)rows5[1],
                  (Rows)rows5[2], (Rows)rows5[3], (Rows)rows5[4]};
    if (beta != 0.0 || full) particle_slab_kernel<Real, true><<<g, 128, 0, s>>>(V, slab_of_row, me, own);
    else particle_slab_kernel<Real, false><<<g, 128, 0, s>>>(V, slab_of_row, me, own);
    return cudaGetLastError();
  };
  return fp32 ? go(0.f) : go(0.0);
}

cudaError_t launch_particles_merge(double* P, int np, const int* own, int me, const double* const* Ps,
                                   double* rec, const double* const* recs, size_t rec_off, int nrec,
                                   cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  particle_merge_kernel<<<(np + 127) / 128, 128, 0, s>>>(P, np, own, me, Ps, rec, recs, rec_off, nrec);
  return cudaGetLastError();
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
