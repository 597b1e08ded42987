// capi_internal.cuh -- the handle type behind the C-ABI and the host-side
// helpers shared by the translation units that implement it (capi.cu,
// ensemble.cu), plus the launchers the kernel files export.
#pragma once

#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "lbrb_internal.cuh"
#include "slab_parts.cuh"

namespace lbrb {
// an NVTX range over a C-ABI call (free when no tool is attached)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};
}  // namespace lbrb

namespace lbrb {
cudaError_t launch_lb_fp64(const LBView<double>& V, int twall, bool refnudge, int shape,
                           cudaStream_t s, bool pdl = false);
cudaError_t launch_lb_fp32(const LBView<float>& V, int twall, int shape, cudaStream_t s, bool pdl = false);
int tune_lb_fp64(const LBView<double>& V, int twall, cudaStream_t s, float* best_ms);
cudaError_t launch_pull_fp64(const LBView<double>& V, int twall, void* outf, void* outg, cudaStream_t s);
cudaError_t launch_pull_fp32(const LBView<float>& V, int twall, void* outf, void* outg, cudaStream_t s);
int tune_lb_fp32(const LBView<float>& V, int twall, cudaStream_t s, float* best_ms);
// two steps per launch (Dirichlet walls, no ghost rows): V1 = step n, V2 = step n+1
cudaError_t launch_pair_fp32(const LBView<float>& V1, const LBView<float>& V2, int shape, cudaStream_t s, bool pdl);
cudaError_t launch_pair_fp64(const LBView<double>& V1, const LBView<double>& V2, int shape, cudaStream_t s, bool pdl);
int tune_pair_fp32(const LBView<float>& V1, const LBView<float>& V2, cudaStream_t s, float* best_ms);
int tune_pair_fp64(const LBView<double>& V1, const LBView<double>& V2, cudaStream_t s, float* best_ms);
cudaError_t launch_particles(const void* u, const void* v, const void* ub, const void* vb,
                             const void* T, bool fp32, int nx, int ny, int pitch, double* P,
                             const int* ptype, int np, double beta, int record, int full,
                             double* rec, unsigned* dflags, cudaStream_t s, bool pdl = false);
// two steps of every particle (after a two-step fused launch): fields_a and
// fields_b = {u, v, ub, vb, T} of steps n and n+1; rec_a / rec_b: the ring
// slots of a record step, else null
cudaError_t launch_particles_pair(const void* const* fields_a, const void* const* fields_b, bool fp32, int nx,
                                  int ny, int pitch, double* P, const int* ptype, int np, double beta, int full,
                                  double* rec_a, double* rec_b, unsigned* dflags, cudaStream_t s, bool pdl);
// y-slabs: rows5 = device tables of row pointers (u, v, ub, vb, T), one
// entry per global row
// y-slabs holding their own particles (particle_kernels.cu): the moment
// messages of a slab; one particle step (advance, classify, compact, pack
// the hand-off lists) through the 5 field tables rows5; the append of the
// received lists
cudaError_t launch_slab_mom_pack(const void* u, const void* v, const void* ub, const void* vb, const void* T,
                                 bool fp32, int nx, int nyl, int pitch, void* mup, void* mdown, size_t pstride,
                                 int istep, int j0, cudaStream_t s, bool pdl);
cudaError_t launch_own_particles(const void* const* rows5, bool fp32, int nx, int ny_total, const SlabParts& S,
                                 void* hand_up, void* hand_down, int j0, int nyl, int istep, double beta, int record,
                                 int full, double* rec, int* rid, int* rcnt, unsigned* dflags, cudaStream_t s,
                                 bool pdl);
cudaError_t launch_own_recv(const SlabParts& S, int j0, int nyl, int nyT, int istep, unsigned* dflags,
                            cudaStream_t s, bool pdl);
// y-slabs: Trows = device table of T row pointers, one per global row
cudaError_t launch_bilinear_nudge_slab(const void* Trows, void* g, bool fp32, size_t plane, int nx, int ny_total,
                                       int j0, int nyl, int pitch, const double* ox, const double* oy,
                                       const double* oT, int nobs, double alpha, long long* acc, unsigned* dflags,
                                       cudaStream_t s);
cudaError_t launch_box_nudge(double* nb, int* nbi, int n, int nx, int ny, int ny_total, int j0, int nt, int istep,
                             int ncx, int ncy, int* cell_count, int* cell_start, int* cell_fill,
                             int* cell_dirty, int* items, int* nudge_vol, double* tempreadint,
                             int pitch, unsigned* dflags, cudaStream_t s);
cudaError_t launch_bilinear_nudge(void* T, void* g, bool fp32, size_t plane, int nx, int ny,
                                  int pitch, const double* ox, const double* oy, const double* oT,
                                  int nobs, double alpha, long long* acc, unsigned* dflags,
                                  cudaStream_t s, bool pdl = false);
// two-step launches of a bilinear-nudged run (nudge_kernels.cu)
cudaError_t launch_obs_pre_fp32(const LBView<float>& V, const double* ox, const double* oy, const double* oT,
                                int nobs, double alpha, long long* acc, unsigned* mask, unsigned* dflags,
                                cudaStream_t s, bool pdl);
cudaError_t launch_obs_pre_fp64(const LBView<double>& V, const double* ox, const double* oy, const double* oT,
                                int nobs, double alpha, long long* acc, unsigned* mask, unsigned* dflags,
                                cudaStream_t s, bool pdl);
// after a nudged two-step launch: step n+1's scatter and apply pass, and
// the clearing of step n's in-launch sums (acc2) and mask bits
cudaError_t launch_bilinear_nudge_clear(void* T, void* g, bool fp32, size_t plane, int nx, int ny, int pitch,
                                        const double* ox, const double* oy, const double* oT, int nobs, double alpha,
                                        long long* acc, const double* ox1, const double* oy1, long long* acc2,
                                        unsigned* mask, unsigned* dflags, cudaStream_t s, bool pdl);
cudaError_t launch_pops_in(const double* h, int layout, void* d, bool fp32, int nx, int ny,
                           int pitch, size_t plane, double base, cudaStream_t s);
cudaError_t launch_pops_out(const void* d, int layout, double* h, bool fp32, int nx, int ny,
                            int pitch, size_t plane, double base, cudaStream_t s);
cudaError_t launch_scalar_in(const double* h, int layout, void* d, bool fp32, int nx, int ny,
                             int pitch, cudaStream_t s);
// units [u0, u1) of a host-layout array between a staging slot and the device
// (in: slot -> device; out: device -> slot); aux_kernels.cu describes units
cudaError_t launch_units(bool in, const void* src, void* dst, int layout, int npop, bool fp32, int nx, int ny,
                         int pitch, size_t plane, double base, int u0, int u1, cudaStream_t s);
cudaError_t launch_scalar_out(const void* d, int layout, double* h, bool fp32, int nx, int ny,
                              int pitch, cudaStream_t s);
cudaError_t launch_force(const void* rho, const void* T, void* F, bool fp32, int nx, int ny,
                         int pitch, double neg_gravity, cudaStream_t s);
cudaError_t launch_moments_from_pre(const double* fpre, const double* gpre, int layout, void* rho,
                                    void* u, void* v, void* T, bool fp32, int nx, int ny, int pitch,
                                    double neg_gravity, cudaStream_t s);
cudaError_t launch_init_conduction(void* pops, void* rho, void* u, void* v, void* T, bool fp32,
                                   int nx, int ny, int pitch, size_t plane, double Tup,
                                   double Tdown, double T0, double neg_gravity, uint64_t seed,
                                   double noise, int j0, int ny_total, cudaStream_t s);
// ghost blocks of SLAB_GH2_PLANES rows for two steps per launch
cudaError_t launch_slab_pack2(const void* pops, const void* F, bool fp32, int nx, int ny, int pitch, size_t plane,
                              void* up, void* down, cudaStream_t s);
cudaError_t launch_slab_pack(const void* pops, bool fp32, int nx, int ny, int pitch, size_t plane, void* up,
                             void* down, cudaStream_t s);
cudaError_t launch_stats(const void* rho, const void* u, const void* v, const void* T, bool fp32,
                         int nx, int ny, int pitch, double* part, double* out, cudaStream_t s);
cudaError_t launch_profile(const void* rho, const void* u, const void* v, const void* T, bool fp32,
                           int nx, int ny, int pitch, const double* Ttop, double* out, cudaStream_t s);
cudaError_t launch_finite(const void* a, size_t n, bool fp32, unsigned* flags, cudaStream_t s);
int red_blocks();
cudaError_t launch_adjoint_step(bool fp32, const void* after, const void* state, const double* lf_out,
                                const double* lg_out, double* lf_in, double* lg_in, double* lF,
                                long long* lT, int nx, int ny, int pitch, size_t plane, double omega,
                                double omegag, double gbeta, double T0, double Tup, double Tdown,
                                cudaStream_t s);
int adjoint_pair_variants();
cudaError_t launch_misfit(const double* res, long n, double* out, cudaStream_t s);
cudaError_t launch_adjoint_pair(bool fp32, int variant, const void* after_a, const void* state_a,
                                const void* state_b, const double* lf_out, const double* lg_out,
                                double* lf_in, double* lg_in, double* lF_in, double* lF_out,
                                const long long* lT_a, const long long* lT_b, int nx, int ny, int pitch,
                                size_t plane, double omega, double omegag, double gbeta, double T0,
                                double Tup, double Tdown, cudaStream_t s);
cudaError_t launch_adj_obs_clear(const double* ox, const double* oy, int nobs, int nx, int ny, int pitch,
                                 long long* acc, cudaStream_t s);
cudaError_t launch_adj_obs_scatter(const double* ox, const double* oy, const double* res, int nobs,
                                   int nx, int ny, int pitch, long long* acc, cudaStream_t s);
cudaError_t launch_obs_residual(const void* T, bool fp32, int nx, int ny, int pitch, const double* ox,
                                const double* oy, const double* oT, int nobs, double* res,
                                cudaStream_t s);
cudaError_t launch_init_from_T0(const double* T0f, void* pops, void* rho, void* u, void* v, void* T,
                                void* F, bool fp32, int nx, int ny, int pitch, size_t plane,
                                double Tref, double neg_gravity, cudaStream_t s);
cudaError_t launch_adj_initial(const double* lg, const double* lF, int nx, int ny, int pitch,
                               size_t plane, double gbeta, double* out, cudaStream_t s);
}  // namespace lbrb

using namespace lbrb;

struct lbrb_s : public Handle {
  std::vector<int> h_ids;
  // timing: event pool and the (class, begin, end) marks of this window
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct Mark { int cls; cudaEvent_t a, b; };
  std::vector<Mark> marks;
};

inline cudaEvent_t pool_event(lbrb_t* h) {
  if (h->ev_used == h->ev_pool.size()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    h->ev_pool.push_back(e);
  }
  return h->ev_pool[h->ev_used++];
}

// begin/end of a timed launch on `s` (no-ops unless timing is enabled)
inline int tmark_begin(lbrb_t* h, int cls, cudaStream_t s) {
  if (!h->timing) return -1;
  cudaEvent_t a = pool_event(h), b = pool_event(h);
  if (!a || !b) return -1;
  cudaEventRecord(a, s);
  h->marks.push_back({cls, a, b});
  return (int)h->marks.size() - 1;
}
inline void tmark_end(lbrb_t* h, int m, cudaStream_t s) {
  if (m >= 0) cudaEventRecord(h->marks[m].b, s);
}

// per-observation arrays of the box mode (see nudge_kernels.cu)
enum { NB_OX = 0, NB_OY, NB_OT, NB_FX, NB_FY, NB_FT, NB_XINT, NB_YINT, NB_TINT, NB_DX, NB_DY,
       NB_DT, NB_COUNT };
enum { NBI_CHK = 0, NBI_BC, NBI_XIDX, NBI_YIDX, NBI_COUNT };

inline int fail(lbrb_t* h, int code, const std::string& msg, cudaError_t e = cudaSuccess) {
  if (h) {
    h->err = msg;
    if (e != cudaSuccess) h->err += std::string(": ") + cudaGetErrorString(e);
  }
  return code;
}

#define CK(h, call)                                                   \
  do {                                                                \
    cudaError_t e_ = (call);                                          \
    if (e_ != cudaSuccess) return fail((h), LBRB_ERR_CUDA, #call, e_); \
  } while (0)

inline bool fp32(const lbrb_t* h) { return h->p.precision == LBRB_PREC_FP32_SHIFTED; }
inline double T0_of(const lbrb_t* h) { return 0.5 * (h->p.Tup + h->p.Tdown); }

inline char* pop_base(const lbrb_t* h, int buf, int which /*0 f, 1 g*/) {
  return (char*)h->pops[buf] + (size_t)which * NPOP * h->plane * h->esize;
}

// view of one step of the handle: populations src -> dst, u/v into slot uvslot
template <typename Real>
inline LBView<Real> make_view(lbrb_t* h, int src, int dst, int uvslot, int write_uv, int write_rt) {
  LBView<Real> V{};
  V.fsrc = (const Real*)pop_base(h, src, 0);
  V.gsrc = (const Real*)pop_base(h, src, 1);
  V.fdst = (Real*)pop_base(h, dst, 0);
  V.gdst = (Real*)pop_base(h, dst, 1);
  V.Fin = (const Real*)h->F[src];
  V.Fout = (Real*)h->F[dst];
  V.rho = (Real*)h->rho[dst];
  V.T = (Real*)h->T[dst];
  V.u = (Real*)h->uv[uvslot][0];
  V.v = (Real*)h->uv[uvslot][1];
  V.nx = h->p.nx;
  V.ny = h->p.ny;
  V.pitch = h->pitch;
  V.plane = h->plane;
  V.omega = 1. / h->p.relax;
  V.omegag = 1. / h->p.relaxg;
  V.neg_gravity = -h->p.gravity;
  V.Tup = h->p.Tup;
  V.Tdown = h->p.Tdown;
  V.T0 = T0_of(h);
  V.omega_f = (float)V.omega;
  V.omegag_f = (float)V.omegag;
  V.neg_gravity_f = (float)V.neg_gravity;
  V.T0_f = (float)V.T0;

  V.nudge_vol = h->nudge_vol;
  V.tempreadint = h->tempreadint;
  V.nud_term = h->nud_term;
  V.tsum0 = h->tsum0;
  V.alpha = h->p.alpha;
  V.write_uv = write_uv;
  V.write_rt = write_rt;
  V.ghost_lo = (const Real*)h->slab_ghost_lo;
  V.ghost_hi = (const Real*)h->slab_ghost_hi;
  return V;
}
