// noalloc.cu -- lbrb_stats_noalloc: the field statistics (mean kinetic
// energy, mean temperature, Nusselt number) of caller-owned device fields,
// computed without allocating any memory.
//
// Why it exists: some callers cannot allocate device memory when they need
// these numbers.  A host framework that owns all device memory through its
// own pool, or a long-running loop that must not allocate after start-up
// (cudaMalloc synchronises the device and may fail under memory pressure),
// still wants the diagnostics of lbrb_energy()/lbrb_nusselt() on fields it
// holds itself.  This entry point takes their device pointers and keeps its
// only scratch -- one partial-sum record per grid row -- in the file-scope
// array below.
//
// Limits and sharing:
//  - at most LBRB_STATS_NOALLOC_MAX_ROWS rows (ny); larger grids are rejected;
//  - the array lives in every GPU that loads the library until the process
//    exits (LBRB_STATS_NOALLOC_MAX_ROWS * 6 doubles, 768 KiB);
//  - all calls share it: two calls whose work overlaps on the GPU (different
//    streams, no ordering between them) race on it and give wrong results;
//  - each call rewrites every row record it reads, so nothing needs clearing;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current.  Under CUDA's default
//    lazy module loading that lookup loads this library's device code, and
//    the array with it, onto the device: the one moment the entry point
//    takes device memory.  Make that first call at start-up, before memory
//    runs short and before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/lbrb.h"

namespace {

constexpr int MAX_ROWS = LBRB_STATS_NOALLOC_MAX_ROWS;
constexpr int NQ = 3;  // kinetic energy, T, v*T
constexpr int MAX_DEVICES = 64;

// [row][quantity][sum, compensation]
static __device__ __align__(256) double g_row_partials[MAX_ROWS * NQ * 2];

double* g_scratch_ptr[MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mu;

struct Neumaier {
  double s = 0.0, c = 0.0;
  __device__ void add(double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
  }
};

// one block per row: compensated sums of 0.5 rho |u|^2, T and v T
template <typename Real>
__global__ void __launch_bounds__(256) row_stats_kernel(const Real* __restrict__ rho,
                                                        const Real* __restrict__ u,
                                                        const Real* __restrict__ v,
                                                        const Real* __restrict__ T, int nx,
                                                        int pitch, double* __restrict__ rows) {
  const int j = blockIdx.x;
  Neumaier a[NQ];
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    const size_t o = (size_t)j * pitch + i;
    const double r = rho[o], uu = u[o], vv = v[o], t = T[o];
    a[0].add(0.5 * r * (uu * uu + vv * vv));
    a[1].add(t);
    a[2].add(vv * t);
  }
  __shared__ double sh[NQ][2][256];
  for (int q = 0; q < NQ; q++) {
    sh[q][0][threadIdx.x] = a[q].s;
    sh[q][1][threadIdx.x] = a[q].c;
  }
  __syncthreads();
  if (threadIdx.x < NQ) {
    Neumaier b;
    for (int t = 0; t < (int)blockDim.x; t++) {
      b.add(sh[threadIdx.x][0][t]);
      b.add(sh[threadIdx.x][1][t]);
    }
    rows[((size_t)j * NQ + threadIdx.x) * 2] = b.s;
    rows[((size_t)j * NQ + threadIdx.x) * 2 + 1] = b.c;
  }
}

// one warp: fold the row records into the three totals, kept in the first
// row record (read back by the host)
__global__ void rows_final_kernel(double* __restrict__ rows, int ny) {
  if (threadIdx.x >= NQ) return;
  Neumaier b;
  for (int j = 0; j < ny; j++) {
    b.add(rows[((size_t)j * NQ + threadIdx.x) * 2]);
    b.add(rows[((size_t)j * NQ + threadIdx.x) * 2 + 1]);
  }
  __syncwarp(0x7u);
  rows[threadIdx.x * 2] = b.s + b.c;
}

// device address of the scratch array for the current device (set up once)
cudaError_t scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_row_partials);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int lbrb_stats_noalloc(const void* rho, const void* u, const void* v, const void* T,
                                  int precision, int nx, int ny, int pitch, double relaxg,
                                  double Tup, double Tdown, void* cuda_stream, double* out3) {
  if (!rho || !u || !v || !T || !out3 || nx < 1 || ny < 1 || pitch < nx ||
      (precision != LBRB_PREC_FP64 && precision != LBRB_PREC_FP32_SHIFTED) || !(relaxg > 0.5) ||
      !(Tdown != Tup))
    return LBRB_ERR_ARG;
  if (ny > MAX_ROWS) return LBRB_ERR_RANGE;  // more rows than the scratch array holds
  double* rows = nullptr;
  if (scratch_for_current_device(&rows) != cudaSuccess) return LBRB_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  if (precision == LBRB_PREC_FP32_SHIFTED)
    row_stats_kernel<float><<<ny, 256, 0, s>>>((const float*)rho, (const float*)u, (const float*)v,
                                               (const float*)T, nx, pitch, rows);
  else
    row_stats_kernel<double><<<ny, 256, 0, s>>>((const double*)rho, (const double*)u,
                                                (const double*)v, (const double*)T, nx, pitch, rows);
  rows_final_kernel<<<1, 32, 0, s>>>(rows, ny);
  if (cudaGetLastError() != cudaSuccess) return LBRB_ERR_CUDA;
  double tot[NQ * 2];
  if (cudaMemcpyAsync(tot, rows, sizeof(tot), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return LBRB_ERR_CUDA;
  const double nn = (double)nx * (double)ny;
  const double kappa = (relaxg - 0.5) / 3.0;
  out3[0] = tot[0] / nn;
  out3[1] = tot[2] / nn;
  out3[2] = 1.0 + (tot[4] / nn) * (double)ny / (kappa * (Tdown - Tup));
  return LBRB_OK;
}
