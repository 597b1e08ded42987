// capi.cu -- the C-ABI declared in include/lbrb.h.
//
// One handle = one whole-domain run on one device.  lbrb_step() queues, per
// time step, on the handle's stream:
//   [box nudging: observation interpolation + ordered box means]
//   fused stream/collide kernel (reads buffer cur, writes cur^1)
//   [bilinear nudging: innovation scatter + apply on the new g]
//   particle kernel (+ record into the device ring; a copy stream moves each
//   finished record into pinned host memory while the next steps run)
// and returns without waiting; lbrb_sync() waits and reports device flags.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "capi_internal.cuh"

template <typename T>
static cudaError_t dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e == cudaSuccess) e = cudaMemset(*p, 0, count * sizeof(T));
  return e;
}

static size_t host_pops_count(const lbrb_t* h, int layout) {
  return layout == LBRB_LAYOUT_REF_AOS_HALO ? (size_t)(h->p.nx + 2) * (h->p.ny + 2) * NPOP
                                            : (size_t)NPOP * h->p.nx * h->p.ny;
}
static size_t host_scalar_count(const lbrb_t* h, int layout) {
  return layout == LBRB_LAYOUT_REF_AOS_HALO ? (size_t)(h->p.nx + 2) * (h->p.ny + 2)
                                            : (size_t)h->p.nx * h->p.ny;
}

// Launch shapes timed once per process: a handle on the same device with the
// same grid, precision, walls, nudging mode, particle use and slab ghost rows
// starts with the shapes an earlier handle timed, without trial launches.
struct TuneKey {
  int dev, nx, ny, pitch, esize, twall, nudge, parts, ghosts;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, nx, ny, pitch, esize, twall, nudge, parts, ghosts) <
           std::tie(o.dev, o.nx, o.ny, o.pitch, o.esize, o.twall, o.nudge, o.parts, o.ghosts);
  }
};
struct TuneVal {
  int shape;
  float ms;
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneVal> g_tuned_single, g_tuned_pair;
// the steps store u, v every step (and T on record steps) for particles:
// the whole domain's, or a slab's own (lbrb_slab_particles_set)
static bool moves_particles(const lbrb_t* h) { return h->np > 0 || (h->sp && h->sp->cap > 0); }
static TuneKey tune_key(const lbrb_t* h) {
  return {h->dev, h->p.nx, h->p.ny, h->pitch, (int)h->esize, h->p.twall, h->p.nudge, moves_particles(h) ? 1 : 0,
          (h->slab_gh2_lo ? 1 : 0) | (h->slab_gh2_hi ? 2 : 0) | (h->slab ? 4 : 0)};
}
static bool tuned_get(std::map<TuneKey, TuneVal>& m, const lbrb_t* h, int* shape, float* ms) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = m.find(tune_key(h));
  if (it == m.end()) return false;
  *shape = it->second.shape;
  *ms = it->second.ms;
  return true;
}
static void tuned_put(std::map<TuneKey, TuneVal>& m, const lbrb_t* h, int shape, float ms) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  m[tune_key(h)] = {shape, ms};
}

// the full-size scratch of the rare paths (restart-route moments, post-stream
// dump), allocated on first use
static int ensure_big(lbrb_t* h, size_t bytes) {
  if (h->big_bytes >= bytes) return LBRB_OK;
  if (h->big) cudaFree(h->big);
  h->big = nullptr;
  h->big_bytes = 0;
  cudaError_t e = cudaMalloc(&h->big, bytes);
  if (e != cudaSuccess) return fail(h, LBRB_ERR_NOMEM, "scratch allocation", e);
  h->big_bytes = bytes;
  return LBRB_OK;
}

// bytes per staging slot: 64 MB, or the largest host array if smaller, and
// at least one transfer unit (a halo column of populations or a row)
constexpr size_t STAGE_SLOT_DOUBLES = (size_t)8 << 20;
static size_t stage_slot_doubles(const lbrb_params& p) {
  const size_t full = (size_t)(p.nx + 2) * (p.ny + 2) * NPOP;
  const size_t unit = std::max((size_t)(p.ny + 2) * NPOP, (size_t)p.nx);
  return std::max(unit, std::min(full, STAGE_SLOT_DOUBLES));
}

// Host <-> device transfer of units [ub, ue) of a host array in `layout`
// (unit u = `unit` doubles at host element u * unit; aux_kernels.cu, units_*),
// chunk by chunk through the two staging slots; conv(slot, u0, u1) converts a
// chunk on the handle's stream.  Upload: the copy of the next chunk (copy
// stream) overlaps the conversion of this one; download: the conversion of
// the next chunk overlaps the copy of this one.  A slot is reused only after
// the last work that read it (events), also across calls; the caller
// synchronises at the end.  One cudaMemcpyAsync per chunk.
template <typename Conv>
static int xfer_units(lbrb_t* h, bool in, double* host, size_t unit, int ub, int ue, Conv&& conv) {
  const int per = (int)std::max<size_t>(1, h->stage_slot / unit);
  double* slot[2] = {(double*)h->staging, (double*)h->staging + h->stage_slot};
  cudaEvent_t* copied = h->xfer_ev;
  cudaEvent_t* converted = h->xfer_ev + 2;
  int c = 0;
  for (int u0 = ub; u0 < ue; u0 += per, c++) {
    const int u1 = std::min(ue, u0 + per), sl = c & 1;
    const size_t bytes = (size_t)(u1 - u0) * unit * sizeof(double);
    double* hp = host + (size_t)u0 * unit;
    if (in) {
      CK(h, cudaStreamWaitEvent(h->copy_stream, converted[sl], 0));  // the slot's last conversion read it
      CK(h, cudaMemcpyAsync(slot[sl], hp, bytes, cudaMemcpyHostToDevice, h->copy_stream));
      CK(h, cudaEventRecord(copied[sl], h->copy_stream));
      CK(h, cudaStreamWaitEvent(h->stream, copied[sl], 0));
      CK(h, conv(slot[sl], u0, u1));
      CK(h, cudaEventRecord(converted[sl], h->stream));
    } else {
      CK(h, cudaStreamWaitEvent(h->stream, copied[sl], 0));  // the slot's last copy read it
      CK(h, conv(slot[sl], u0, u1));
      CK(h, cudaEventRecord(converted[sl], h->stream));
      CK(h, cudaStreamWaitEvent(h->copy_stream, converted[sl], 0));
      CK(h, cudaMemcpyAsync(hp, slot[sl], bytes, cudaMemcpyDeviceToHost, h->copy_stream));
      CK(h, cudaEventRecord(copied[sl], h->copy_stream));
    }
  }
  return LBRB_OK;
}

// units of a host array: populations (npop = 9) or a scalar field (npop = 1);
// uploads skip the reference layout's halo columns (units 0 and nx + 1)
static size_t unit_doubles(const lbrb_t* h, int layout, int npop) {
  return layout == LBRB_LAYOUT_REF_AOS_HALO ? (size_t)(h->p.ny + 2) * npop : (size_t)h->p.nx;
}
static void unit_range(const lbrb_t* h, int layout, int npop, bool in, int* ub, int* ue) {
  if (layout == LBRB_LAYOUT_REF_AOS_HALO) {
    *ub = in ? 1 : 0;
    *ue = in ? h->p.nx + 1 : h->p.nx + 2;
  } else {
    *ub = 0;
    *ue = npop * h->p.ny;
  }
}
static int xfer_array(lbrb_t* h, bool in, double* host, void* dev, int layout, int npop, double base) {
  int ub, ue;
  unit_range(h, layout, npop, in, &ub, &ue);
  return xfer_units(h, in, host, unit_doubles(h, layout, npop), ub, ue, [&](double* st, int u0, int u1) {
    return launch_units(in, in ? (const void*)st : dev, in ? dev : (void*)st, layout, npop, fp32(h), h->p.nx,
                        h->p.ny, h->pitch, h->plane, base, u0, u1, h->stream);
  });
}

// Host copies out of the pinned record ring.  A large drain (hundreds of MB
// at the production size) is split over host threads: one thread's memcpy
// runs at a fraction of the host memory bandwidth.
struct CopyJob {
  void* dst;
  const void* src;
  size_t bytes;
};

static void parallel_copy(const std::vector<CopyJob>& jobs) {
  size_t total = 0;
  for (const CopyJob& j : jobs) total += j.bytes;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nt = std::min(hw, 16u);
  if (total < ((size_t)32 << 20) || nt == 1) {
    for (const CopyJob& j : jobs) std::memcpy(j.dst, j.src, j.bytes);
    return;
  }
  // pieces of about total / (4 nt) bytes, at least 1 MB, handed out in order
  const size_t piece = std::max(total / (4 * nt), (size_t)1 << 20);
  std::vector<CopyJob> pieces;
  for (const CopyJob& j : jobs)
    for (size_t o = 0; o < j.bytes; o += piece)
      pieces.push_back({(char*)j.dst + o, (const char*)j.src + o, std::min(piece, j.bytes - o)});
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (size_t i; (i = next.fetch_add(1)) < pieces.size();)
      std::memcpy(pieces[i].dst, pieces[i].src, pieces[i].bytes);
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < nt; t++) pool.emplace_back(work);
  work();
  for (std::thread& t : pool) t.join();
}

extern "C" {

int lbrb_abi_version(void) { return LBRB_ABI_VERSION; }

void lbrb_params_default(lbrb_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  // reference values: temppart_dump.c:16-28, Trajectories/code/mympi2.h:14-19,
  // tempvel_nudge.c:13, 23
  p->nx = 1680;
  p->ny = 840;
  p->relax = 0.502;
  p->relaxg = 0.502;
  p->Tup = -0.01;
  p->Tdown = 0.01;
  p->gravity = -0.00004;
  p->precision = LBRB_PREC_FP64;
  p->twall = LBRB_TWALL_DIRICHLET;
  p->nudge = LBRB_NUDGE_NONE;
  p->alpha = 0.01;
  p->ntempread = 250;
  p->nobs = 0;
  p->beta = 0.1;
  p->nprtcl = 0;
  p->noutconfig = 0;
  p->record_full = 0;
  p->record_slots = 16;
  p->device = 0;
  p->autotune = 1;
}

const char* lbrb_last_error(const lbrb_t* h) { return h ? h->err.c_str() : "null handle"; }

static void free_sp(SlabParts* S) {
  if (!S) return;
  auto F = [](void* q) { if (q) cudaFree(q); };
  for (int b = 0; b < 2; b++) {
    F(S->P[b]); F(S->id[b]); F(S->type[b]);
  }
  F(S->cnt); F(S->cls); F(S->bcnt); F(S->done); F(S->rows); F(S->zrow); F(S->d_rec); F(S->d_rid); F(S->d_rcnt);
  for (void* q : S->mom) F(q);
  for (void* q : S->hand) F(q);
  if (S->h_rec) cudaFreeHost(S->h_rec);
  if (S->h_rid) cudaFreeHost(S->h_rid);
  if (S->h_rcnt) cudaFreeHost(S->h_rcnt);
  for (cudaEvent_t e : S->rev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : {S->ev_mom, S->ev_part, S->ev_hand})
    if (e) cudaEventDestroy(e);
  delete S;
}

static void free_all(lbrb_t* h) {
  auto F = [](void* q) { if (q) cudaFree(q); };
  F(h->pops[0]); F(h->pops[1]); F(h->F[0]); F(h->F[1]);
  F(h->rho[0]); F(h->rho[1]); F(h->T[0]); F(h->T[1]);
  for (int a = 0; a < 3; a++) for (int b = 0; b < 2; b++) F(h->uv[a][b]);
  F(h->px); F(h->pid); F(h->ptype); F(h->d_ring);
  if (h->h_ring) cudaFreeHost(h->h_ring);
  delete[] h->h_ring_step;
  if (h->ring_ev) {
    for (int s = 0; s < h->p.record_slots; s++) if (h->ring_ev[s]) cudaEventDestroy(h->ring_ev[s]);
    delete[] h->ring_ev;
  }
  F(h->nb); F(h->nbi); F(h->nudge_vol); F(h->tempreadint); F(h->nud_term); F(h->tsum0);
  F(h->cell_count); F(h->cell_start); F(h->cell_fill); F(h->cell_dirty); F(h->cell_items);
  delete[] h->h_chk; delete[] h->h_oid;
  F(h->obs); F(h->acc); F(h->acc2); F(h->nmask); F(h->staging); F(h->big); F(h->red); F(h->dflags);
  F(h->adj_obs); F(h->adj_res); F(h->adj_chk); F(h->adj_seg); F(h->adj_lam); F(h->adj_lT); F(h->adj_T0);
  F(h->adj_store);
  F(h->slab_ghost_lo); F(h->slab_ghost_hi); F(h->slab_up); F(h->slab_down); F(h->slab_tab);
  free_sp(h->sp);
  h->sp = nullptr;
  F(h->slab_gh2_lo); F(h->slab_gh2_hi); F(h->slab_up2); F(h->slab_down2);
  for (cudaGraphExec_t& g : h->graph_exec)
    if (g) cudaGraphExecDestroy(g);
  if (h->slab_ev_xfer) cudaEventDestroy(h->slab_ev_xfer);
  if (h->slab_ev_done) cudaEventDestroy(h->slab_ev_done);
  delete[] h->adj_steps;
  if (h->h_flags) cudaFreeHost(h->h_flags);
  if (h->h_scalar) cudaFreeHost(h->h_scalar);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->join_ev) cudaEventDestroy(h->join_ev);
  for (cudaEvent_t e : h->xfer_ev)
    if (e) cudaEventDestroy(e);
  if (h->pstream) cudaStreamDestroy(h->pstream);
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
}

int lbrb_create(const lbrb_params* pin, lbrb_t** out) {
  if (!pin || !out) return LBRB_ERR_ARG;
  *out = nullptr;
  const lbrb_params& p = *pin;
  auto bad = [](double x) { return !(x == x) || x > 1e300 || x < -1e300; };
  if (p.nx < 4 || p.nx % 4 != 0 || p.ny < 3 || bad(p.relax) || bad(p.relaxg) || p.relax <= 0.5 ||
      p.relaxg <= 0.5 || bad(p.Tup) || bad(p.Tdown) || bad(p.gravity) || bad(p.alpha) ||
      bad(p.beta) || p.nprtcl < 0 || p.noutconfig < 0 || p.nobs < 0 ||
      (p.precision != LBRB_PREC_FP64 && p.precision != LBRB_PREC_FP32_SHIFTED) ||
      (p.twall != LBRB_TWALL_DIRICHLET && p.twall != LBRB_TWALL_ADIABATIC) ||
      (p.nudge < LBRB_NUDGE_NONE || p.nudge > LBRB_NUDGE_BILINEAR))
    return LBRB_ERR_ARG;
  if (p.nudge != LBRB_NUDGE_NONE && p.nobs <= 0) return LBRB_ERR_ARG;
  if (p.nudge == LBRB_NUDGE_REFBOX && p.ntempread < 2) return LBRB_ERR_ARG;
  if (p.nudge == LBRB_NUDGE_REFBOX && p.precision != LBRB_PREC_FP64) return LBRB_ERR_UNSUPPORTED;
  if (p.nprtcl > 0 && p.noutconfig > 0 && p.record_slots < 1) return LBRB_ERR_ARG;
  if (p.launch_shape < 0 || p.launch_shape > 9) return LBRB_ERR_ARG;
  if ((long)p.nx * p.ny > (1L << 31) - 1) return LBRB_ERR_ARG;

  lbrb_t* h = new lbrb_t();
  h->p = p;
  if (h->p.record_slots < 1) h->p.record_slots = 1;
  h->dev = p.device;
  auto done = [&](int code) -> int {
    if (code != LBRB_OK) {
      free_all(h);
      delete h;
      return code;
    }
    *out = h;
    return (int)LBRB_OK;
  };
  cudaError_t e = cudaSetDevice(p.device);
  if (e != cudaSuccess) return done(LBRB_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->join_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->pstream, cudaStreamNonBlocking) != cudaSuccess)
    return done(LBRB_ERR_CUDA);
  h->stream = h->own_stream;
  h->pitch = (p.nx + 31) / 32 * 32;
  h->plane = (size_t)p.ny * h->pitch;
  h->esize = fp32(h) ? 4 : 8;
  const size_t pb = 2 * NPOP * h->plane * h->esize;
  for (int b = 0; b < 2; b++) {
    if (cudaMalloc(&h->pops[b], pb) != cudaSuccess) return done(LBRB_ERR_NOMEM);
    cudaMemset(h->pops[b], 0, pb);
  }
  void** scal[] = {&h->F[0], &h->F[1], &h->rho[0], &h->rho[1], &h->T[0], &h->T[1],
                   &h->uv[0][0], &h->uv[0][1], &h->uv[1][0], &h->uv[1][1], &h->uv[2][0], &h->uv[2][1]};
  for (void** s : scal) {
    if (cudaMalloc(s, h->plane * h->esize) != cudaSuccess) return done(LBRB_ERR_NOMEM);
    cudaMemset(*s, 0, h->plane * h->esize);
  }
  h->np = p.nprtcl;
  if (h->np > 0) {
    if (dalloc(&h->px, (size_t)9 * h->np) || dalloc(&h->pid, h->np) || dalloc(&h->ptype, h->np))
      return done(LBRB_ERR_NOMEM);
    h->nrec_fields = p.record_full ? LBRB_REC_NFULL : LBRB_REC_NBASIC;
    if (p.noutconfig > 0) {
      const size_t rb = (size_t)h->p.record_slots * h->nrec_fields * h->np;
      if (dalloc(&h->d_ring, rb)) return done(LBRB_ERR_NOMEM);
      if (cudaMallocHost(&h->h_ring, rb * sizeof(double)) != cudaSuccess) return done(LBRB_ERR_NOMEM);
      h->h_ring_step = new int[h->p.record_slots]();
      h->ring_ev = new cudaEvent_t[h->p.record_slots]();
      for (int s = 0; s < h->p.record_slots; s++)
        if (cudaEventCreateWithFlags(&h->ring_ev[s], cudaEventDisableTiming) != cudaSuccess)
          return done(LBRB_ERR_CUDA);
    }
  }
  h->nobs = p.nobs;
  if (p.nudge == LBRB_NUDGE_REFBOX) {
    const int n = h->nobs;
    h->ncx = (p.nx + 7) / 8;
    h->ncy = (p.ny + 7) / 8;
    const size_t nc = (size_t)h->ncx * h->ncy;
    if (dalloc(&h->nb, (size_t)NB_COUNT * n) || dalloc(&h->nbi, (size_t)NBI_COUNT * n) ||
        dalloc(&h->nudge_vol, h->plane) || dalloc(&h->tempreadint, h->plane) ||
        dalloc(&h->nud_term, h->plane) || dalloc(&h->tsum0, (size_t)h->pitch) || dalloc(&h->cell_count, nc) ||
        dalloc(&h->cell_start, nc) || dalloc(&h->cell_fill, nc) || dalloc(&h->cell_dirty, nc) ||
        dalloc(&h->cell_items, (size_t)2 * 12 * n))
      return done(LBRB_ERR_NOMEM);
    h->h_chk = new int[n]();
    h->h_oid = new int[n]();
  }
  if (p.nudge == LBRB_NUDGE_BILINEAR) {
    if (dalloc(&h->acc, h->plane) || dalloc(&h->acc2, h->plane) ||
        dalloc(&h->nmask, (size_t)p.ny * (h->pitch / 32)))
      return done(LBRB_ERR_NOMEM);
  }
  h->stage_slot = stage_slot_doubles(p);
  h->staging_bytes = 2 * h->stage_slot * sizeof(double);
  if (cudaMalloc(&h->staging, h->staging_bytes) != cudaSuccess) return done(LBRB_ERR_NOMEM);
  for (cudaEvent_t& ev : h->xfer_ev)
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return done(LBRB_ERR_CUDA);
  if (dalloc(&h->red, (size_t)red_blocks() * 6 + 8 + (size_t)p.ny * 9)) return done(LBRB_ERR_NOMEM);
  if (dalloc(&h->dflags, 1)) return done(LBRB_ERR_NOMEM);
  if (cudaMallocHost(&h->h_flags, sizeof(unsigned)) != cudaSuccess) return done(LBRB_ERR_NOMEM);
  if (cudaMallocHost(&h->h_scalar, sizeof(double)) != cudaSuccess) return done(LBRB_ERR_NOMEM);
  if (cudaDeviceSynchronize() != cudaSuccess) return done(LBRB_ERR_CUDA);
  return done(LBRB_OK);
}

int lbrb_destroy(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  cudaSetDevice(h->dev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->pstream) cudaStreamSynchronize(h->pstream);
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  free_all(h);
  delete h;
  return LBRB_OK;
}

int lbrb_get_istep(const lbrb_t* h, int* istep) {
  if (!h || !istep) return LBRB_ERR_ARG;
  *istep = h->istep;
  return LBRB_OK;
}

int lbrb_set_istep(lbrb_t* h, int istep) {
  if (!h || istep < 0) return LBRB_ERR_ARG;
  h->istep = istep;
  return LBRB_OK;
}

// ------------------------------------------------------------- state I/O
int lbrb_set_populations(lbrb_t* h, const double* f, const double* g, int layout) {
  if (!h || !f || !g || (layout != LBRB_LAYOUT_REF_AOS_HALO && layout != LBRB_LAYOUT_SOA))
    return fail(h, LBRB_ERR_ARG, "set_populations: bad arguments");
  CK(h, cudaSetDevice(h->dev));
  const double* src[2] = {f, g};
  for (int a = 0; a < 2; a++) {
    const int rc = xfer_array(h, true, const_cast<double*>(src[a]), pop_base(h, h->cur, a), layout, NPOP,
                              a ? T0_of(h) : 1.0);
    if (rc) return rc;
  }
  CK(h, cudaStreamSynchronize(h->stream));
  h->prev_valid = false;
  h->prev_pair = false;
  return LBRB_OK;
}

int lbrb_get_populations(lbrb_t* h, double* f, double* g, int layout) {
  if (!h || (layout != LBRB_LAYOUT_REF_AOS_HALO && layout != LBRB_LAYOUT_SOA))
    return fail(h, LBRB_ERR_ARG, "get_populations: bad arguments");
  CK(h, cudaSetDevice(h->dev));
  double* dst[2] = {f, g};
  for (int a = 0; a < 2; a++) {
    if (!dst[a]) continue;
    const int rc = xfer_array(h, false, dst[a], pop_base(h, h->cur, a), layout, NPOP, a ? T0_of(h) : 1.0);
    if (rc) return rc;
  }
  CK(h, cudaStreamSynchronize(h->copy_stream));
  return LBRB_OK;
}

int lbrb_set_moments(lbrb_t* h, const double* rho, const double* u, const double* v,
                     const double* T, int layout) {
  if (!h || !rho || !u || !v || !T || (layout != LBRB_LAYOUT_REF_AOS_HALO && layout != LBRB_LAYOUT_SOA))
    return fail(h, LBRB_ERR_ARG, "set_moments: bad arguments");
  CK(h, cudaSetDevice(h->dev));
  const double* src[4] = {rho, u, v, T};
  void* dst[4] = {h->rho[h->cur], h->uv[h->uvcur][0], h->uv[h->uvcur][1], h->T[h->cur]};
  for (int a = 0; a < 4; a++) {
    const int rc = xfer_array(h, true, const_cast<double*>(src[a]), dst[a], layout, 1, 0.0);
    if (rc) return rc;
  }
  CK(h, launch_force(h->rho[h->cur], h->T[h->cur], h->F[h->cur], fp32(h), h->p.nx, h->p.ny, h->pitch, -h->p.gravity, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->moments_valid = true;
  return LBRB_OK;
}

int lbrb_get_moments(lbrb_t* h, double* rho, double* u, double* v, double* T, int layout) {
  if (!h || (layout != LBRB_LAYOUT_REF_AOS_HALO && layout != LBRB_LAYOUT_SOA))
    return fail(h, LBRB_ERR_ARG, "get_moments: bad arguments");
  CK(h, cudaSetDevice(h->dev));
  double* dst[4] = {rho, u, v, T};
  const void* src[4] = {h->rho[h->cur], h->uv[h->uvcur][0], h->uv[h->uvcur][1], h->T[h->cur]};
  for (int a = 0; a < 4; a++) {
    if (!dst[a]) continue;
    const int rc = xfer_array(h, false, dst[a], const_cast<void*>(src[a]), layout, 1, 0.0);
    if (rc) return rc;
  }
  CK(h, cudaStreamSynchronize(h->copy_stream));
  return LBRB_OK;
}

int lbrb_moments_from_pre(lbrb_t* h, const double* fpre, const double* gpre, int layout) {
  if (!h || !fpre || !gpre || (layout != LBRB_LAYOUT_REF_AOS_HALO && layout != LBRB_LAYOUT_SOA))
    return fail(h, LBRB_ERR_ARG, "moments_from_pre: bad arguments");
  CK(h, cudaSetDevice(h->dev));
  const size_t cnt = host_pops_count(h, layout), bytes = cnt * sizeof(double);
  int rc = ensure_big(h, 2 * bytes);
  if (rc) return rc;
  double* st = (double*)h->big;
  CK(h, cudaMemcpyAsync(st, fpre, bytes, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(st + cnt, gpre, bytes, cudaMemcpyHostToDevice, h->stream));
  CK(h, launch_moments_from_pre(st, st + cnt, layout, h->rho[h->cur], h->uv[h->uvcur][0],
                                h->uv[h->uvcur][1], h->T[h->cur], fp32(h), h->p.nx, h->p.ny, h->pitch,
                                -h->p.gravity, h->stream));
  CK(h, launch_force(h->rho[h->cur], h->T[h->cur], h->F[h->cur], fp32(h), h->p.nx, h->p.ny, h->pitch, -h->p.gravity, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->moments_valid = true;
  return LBRB_OK;
}

int lbrb_init_conduction(lbrb_t* h, uint64_t seed, double noise) {
  if (!h || !(noise == noise)) return fail(h, LBRB_ERR_ARG, "init_conduction: bad arguments");
  CK(h, cudaSetDevice(h->dev));
  CK(h, launch_init_conduction(h->pops[h->cur], h->rho[h->cur], h->uv[h->uvcur][0],
                               h->uv[h->uvcur][1], h->T[h->cur], fp32(h), h->p.nx, h->p.ny, h->pitch, h->plane, h->p.Tup,
                               h->p.Tdown, T0_of(h), -h->p.gravity, seed, noise, h->slab ? h->slab_j0 : 0,
                               h->slab ? h->slab_ny_total : h->p.ny, h->stream));
  CK(h, launch_force(h->rho[h->cur], h->T[h->cur], h->F[h->cur], fp32(h), h->p.nx, h->p.ny, h->pitch, -h->p.gravity, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->moments_valid = true;
  return LBRB_OK;
}

// ------------------------------------------------------------- particles
int lbrb_particles_set(lbrb_t* h, int n, const int* ids, const double* x, const double* y,
                       const double* u, const double* v, const int* ptype, const double* invtau) {
  if (!h || n != h->np || n <= 0 || !ids || !x || !y || !u || !v || !ptype || !invtau)
    return fail(h, LBRB_ERR_ARG, "particles_set: arguments must cover all nprtcl particles");
  const int nyd = h->slab ? h->slab_ny_total : h->p.ny;  // (a y-slab: the whole domain's rows)
  for (int q = 0; q < n; q++) {
    if (!(x[q] > -1.0 && x[q] < h->p.nx + 1.0 && y[q] >= 0.0 && y[q] <= nyd + 1.0))
      return fail(h, LBRB_ERR_RANGE, "particles_set: position outside the domain");
    if (!(u[q] == u[q]) || !(v[q] == v[q]) || !(invtau[q] >= 0.0) ||
        (ptype[q] != LBRB_PTYPE_TRACER && ptype[q] != LBRB_PTYPE_INERTIAL))
      return fail(h, LBRB_ERR_ARG, "particles_set: bad velocity, type or 1/tau");
  }
  CK(h, cudaSetDevice(h->dev));
  std::vector<double> P((size_t)9 * n);
  std::memcpy(&P[0 * (size_t)n], x, n * sizeof(double));
  std::memcpy(&P[1 * (size_t)n], y, n * sizeof(double));
  std::memcpy(&P[2 * (size_t)n], u, n * sizeof(double));
  std::memcpy(&P[3 * (size_t)n], v, n * sizeof(double));
  std::memcpy(&P[4 * (size_t)n], x, n * sizeof(double));
  std::memcpy(&P[5 * (size_t)n], y, n * sizeof(double));
  std::memcpy(&P[6 * (size_t)n], u, n * sizeof(double));
  std::memcpy(&P[7 * (size_t)n], v, n * sizeof(double));
  std::memcpy(&P[8 * (size_t)n], invtau, n * sizeof(double));
  CK(h, cudaMemcpyAsync(h->px, P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->pid, ids, n * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->ptype, ptype, n * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->h_ids.assign(ids, ids + n);
  h->particles_set = true;
  return LBRB_OK;
}

int lbrb_particles_get(lbrb_t* h, int n, int* ids, double* x, double* y, double* u, double* v,
                       double* xo, double* yo, double* uo, double* vo) {
  if (!h || n != h->np || n <= 0) return fail(h, LBRB_ERR_ARG, "particles_get: n must be nprtcl");
  CK(h, cudaSetDevice(h->dev));
  std::vector<double> P((size_t)9 * n);
  CK(h, cudaMemcpyAsync(P.data(), h->px, P.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  double* outs[8] = {x, y, u, v, xo, yo, uo, vo};
  for (int a = 0; a < 8; a++)
    if (outs[a]) std::memcpy(outs[a], &P[(size_t)a * n], n * sizeof(double));
  if (ids) std::memcpy(ids, h->h_ids.data(), n * sizeof(int));
  return LBRB_OK;
}

// --------------------------------------------------------------- records
int lbrb_record_pending(lbrb_t* h, int* count) {
  if (!h || !count) return LBRB_ERR_ARG;
  *count = (int)(h->rec_head - h->rec_tail);
  return LBRB_OK;
}

int lbrb_record_drain(lbrb_t* h, int max_records, int* steps, double* buf, int* ids, int* n_drained) {
  if (!h || max_records < 0 || (max_records > 0 && (!steps || !buf)))
    return fail(h, LBRB_ERR_ARG, "record_drain: bad arguments");
  CK(h, cudaSetDevice(h->dev));
  const size_t per = (size_t)h->nrec_fields * h->np;
  int k = 0;
  std::vector<CopyJob> jobs;
  while (k < max_records && h->rec_tail < h->rec_head) {
    const int slot = (int)(h->rec_tail % h->p.record_slots);
    CK(h, cudaEventSynchronize(h->ring_ev[slot]));
    jobs.push_back({buf + (size_t)k * per, h->h_ring + (size_t)slot * per, per * sizeof(double)});
    steps[k] = h->h_ring_step[slot];
    h->rec_tail++;
    k++;
  }
  parallel_copy(jobs);
  if (ids && h->np > 0) std::memcpy(ids, h->h_ids.data(), h->np * sizeof(int));
  if (n_drained) *n_drained = k;
  return LBRB_OK;
}

// --------------------------------------------------------------- nudging
int lbrb_nudge_init(lbrb_t* h, int n, const double* x, const double* y, const double* T,
                    const int* ids) {
  if (!h || h->p.nudge != LBRB_NUDGE_REFBOX || n != h->nobs || !x || !y || !T || !ids)
    return fail(h, LBRB_ERR_ARG, "nudge_init: box nudging with n == nobs required");
  CK(h, cudaSetDevice(h->dev));
  const size_t b = n * sizeof(double);
  double* nb = h->nb;
  const double* src[6] = {x, y, T, x, y, T};
  const int dst[6] = {NB_OX, NB_OY, NB_OT, NB_XINT, NB_YINT, NB_TINT};
  for (int a = 0; a < 6; a++)
    CK(h, cudaMemcpyAsync(nb + (size_t)dst[a] * n, src[a], b, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemsetAsync(h->nbi, 0, sizeof(int) * NBI_COUNT * (size_t)n, h->stream));
  CK(h, cudaMemsetAsync(h->nud_term, 0, sizeof(double) * h->plane, h->stream));
  CK(h, cudaMemsetAsync(h->tsum0, 0, sizeof(double) * h->pitch, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  std::memcpy(h->h_oid, ids, n * sizeof(int));
  std::memset(h->h_chk, 0, n * sizeof(int));
  h->nudge_init_done = true;
  return LBRB_OK;
}

int lbrb_nudge_load(lbrb_t* h, int n, const double* x, const double* y, const int* ids,
                    const double* T) {
  if (!h || h->p.nudge != LBRB_NUDGE_REFBOX || n != h->nobs || !x || !y || !T || !ids)
    return fail(h, LBRB_ERR_ARG, "nudge_load: box nudging with n == nobs required");
  if (!h->nudge_init_done) return fail(h, LBRB_ERR_STATE, "nudge_load before nudge_init");
  // read_prtcl matches ids by a first-hit search (tempvel_nudge.c:1480-1487);
  // the same first occurrence through a hash map
  std::unordered_map<int, int> first;
  first.reserve((size_t)n * 2);
  for (int j = 0; j < n; j++) first.emplace(ids[j], j);
  for (int i = 0; i < n; i++) {
    auto it = first.find(h->h_oid[i]);
    if (it == first.end()) return fail(h, LBRB_ERR_IDS, "nudge_load: an observed id is missing from the file");
    h->h_chk[i] = it->second;
  }
  CK(h, cudaSetDevice(h->dev));
  const size_t b = n * sizeof(double);
  CK(h, cudaMemcpyAsync(h->nb + (size_t)NB_FX * n, x, b, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->nb + (size_t)NB_FY * n, y, b, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->nb + (size_t)NB_FT * n, T, b, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->nbi + (size_t)NBI_CHK * n, h->h_chk, n * sizeof(int),
                        cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->nudge_file_loaded = true;
  return LBRB_OK;
}

int lbrb_nudge_obs(lbrb_t* h, int first_step, int nsteps, const double* x, const double* y,
                   const double* T) {
  if (!h || h->p.nudge != LBRB_NUDGE_BILINEAR || nsteps < 1 || !x || !y || !T)
    return fail(h, LBRB_ERR_ARG, "nudge_obs: bilinear nudging required");
  CK(h, cudaSetDevice(h->dev));
  const int n = h->nobs;
  if (nsteps > h->obs_cap_steps) {
    if (h->obs) cudaFree(h->obs);
    h->obs = nullptr;
    h->obs_cap_steps = 0;
    cudaError_t e = cudaMalloc(&h->obs, (size_t)nsteps * 3 * n * sizeof(double));
    if (e != cudaSuccess) return fail(h, LBRB_ERR_NOMEM, "nudge_obs allocation", e);
    h->obs_cap_steps = nsteps;
  }
  CK(h, cudaStreamSynchronize(h->stream));  // the previous series may still be in use
  for (int s = 0; s < nsteps; s++) {
    double* base = h->obs + (size_t)s * 3 * n;
    CK(h, cudaMemcpyAsync(base, x + (size_t)s * n, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(base + n, y + (size_t)s * n, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(base + 2 * n, T + (size_t)s * n, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }
  CK(h, cudaStreamSynchronize(h->stream));
  h->obs_first = first_step;
  h->obs_nsteps = nsteps;
  return LBRB_OK;
}

// ------------------------------------------------------------- time loop
}  // extern "C"

// view of one step from one state slot (SLOT_PLANES planes: pops, F,
// moments) to another; with `mom` the step's moments go to the destination
// slot's moment planes
template <typename Real>
static LBView<Real> seg_view(lbrb_t* h, const char* src, char* dst, int mom) {
  LBView<Real> V = make_view<Real>(h, 0, 1, h->uvcur, mom, mom ? 3 : 0);
  const size_t pl = h->plane;
  const Real* a = (const Real*)src;
  Real* b = (Real*)dst;
  V.fsrc = a;
  V.gsrc = a + NPOP * pl;
  V.Fin = a + SLOT_F * pl;
  V.fdst = b;
  V.gdst = b + NPOP * pl;
  V.Fout = b + SLOT_F * pl;
  V.rho = b + SLOT_MOM * pl;
  V.u = b + (SLOT_MOM + 1) * pl;
  V.v = b + (SLOT_MOM + 2) * pl;
  V.T = b + (SLOT_MOM + 3) * pl;
  return V;
}

static const int SHAPE_BS[] = {256, 256, 256, 128, 128, 512, 512, 256, 128, 128};
static const int SHAPE_MB[] = {1, 2, 3, 4, 6, 1, 2, 3, 4, 6};

extern "C" {

int lbrb_get_launch_shape(const lbrb_t* h, int* shape, int* block, int* min_blocks, float* ms) {
  if (!h) return LBRB_ERR_ARG;
  const int sh = h->lb_shape < 0 ? h->p.launch_shape : h->lb_shape;
  if (shape) *shape = sh;
  if (block) *block = SHAPE_BS[sh];
  if (min_blocks) *min_blocks = SHAPE_MB[sh];
  if (ms) *ms = h->lb_shape_ms;
  return LBRB_OK;
}

int lbrb_get_poststream(lbrb_t* h, double* f, double* g, int layout) {
  if (!h || (layout != LBRB_LAYOUT_REF_AOS_HALO && layout != LBRB_LAYOUT_SOA))
    return fail(h, LBRB_ERR_ARG, "get_poststream: bad arguments");
  if (!h->prev_valid && !h->prev_pair)
    return fail(h, LBRB_ERR_STATE, "get_poststream: no step since the populations were set");
  CK(h, cudaSetDevice(h->dev));
  const size_t tmp = 2 * NPOP * h->plane * h->esize;
  const size_t cnt = host_pops_count(h, layout), bytes = cnt * sizeof(double);
  // (a call that ended with a two-step launch: room for the rebuilt state
  // before its last step and that step's F)
  const size_t extra = h->prev_valid ? 0 : tmp + h->plane * h->esize;
  int rc = ensure_big(h, tmp + 2 * bytes + extra);
  if (rc) return rc;
  char* t = (char*)h->big;
  double* st = (double*)(t + tmp);
  const int prev = h->cur ^ 1;
  if (h->prev_valid) {
    if (fp32(h)) CK(h, launch_pull_fp32(make_view<float>(h, prev, h->cur, h->uvcur, 0, 0), h->p.twall, t, t + tmp / 2, h->stream));
    else CK(h, launch_pull_fp64(make_view<double>(h, prev, h->cur, h->uvcur, 0, 0), h->p.twall, t, t + tmp / 2, h->stream));
  } else {
    // the state before the last step is the first step of the last launch,
    // taken again from the state before that launch (its populations and F
    // are still in the other buffer): one single step into scratch, which
    // equals the two-step launch's first step bit for bit, then the pull
    char* scr = t + tmp + 2 * bytes;
    char* scrF = scr + tmp;
    const int shape = h->lb_shape >= 0 ? h->lb_shape : h->p.launch_shape;
    auto rebuild = [&](auto zero) -> cudaError_t {
      using Real = decltype(zero);
      LBView<Real> V = make_view<Real>(h, prev, h->cur, h->uvcur, 0, 0);
      V.fdst = (Real*)scr;
      V.gdst = (Real*)scr + NPOP * h->plane;
      V.Fout = (Real*)scrF;
      cudaError_t e;
      if constexpr (std::is_same<Real, float>::value) e = launch_lb_fp32(V, h->p.twall, shape, h->stream, false);
      else e = launch_lb_fp64(V, h->p.twall, false, shape, h->stream, false);
      if (e != cudaSuccess) return e;
      LBView<Real> P = make_view<Real>(h, prev, h->cur, h->uvcur, 0, 0);
      P.fsrc = (const Real*)scr;
      P.gsrc = (const Real*)scr + NPOP * h->plane;
      if constexpr (std::is_same<Real, float>::value) return launch_pull_fp32(P, h->p.twall, t, t + tmp / 2, h->stream);
      else return launch_pull_fp64(P, h->p.twall, t, t + tmp / 2, h->stream);
    };
    if (fp32(h)) CK(h, rebuild(0.f));
    else CK(h, rebuild(0.0));
  }
  if (f) {
    CK(h, launch_pops_out(t, layout, st, fp32(h), h->p.nx, h->p.ny, h->pitch, h->plane, 1.0, h->stream));
    CK(h, cudaMemcpyAsync(f, st, bytes, cudaMemcpyDeviceToHost, h->stream));
  }
  if (g) {
    CK(h, launch_pops_out(t + tmp / 2, layout, st + cnt, fp32(h), h->p.nx, h->p.ny, h->pitch, h->plane,
                          T0_of(h), h->stream));
    CK(h, cudaMemcpyAsync(g, st + cnt, bytes, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(h, cudaStreamSynchronize(h->stream));
  return LBRB_OK;
}

static bool step_pairs_ok(const lbrb_t* h);  // (below)

// CUDA-graph replay of plain steps: forced (graph_mode 1), or automatic on
// grids up to GRAPH_MAX_NODES nodes where two steps per launch do not apply
// (two-step launches beat graph replays of single steps there: at 512x256
// 25-26k against 18k MLUPS in FP32, 16k against 14.4k in FP64); a
// capturable stream (not the legacy default stream), no nudging, no
// per-kernel timing, particle kernels on the step stream, not a y-slab
constexpr int GRAPH_STEPS = 3;
constexpr long GRAPH_MAX_NODES = 1L << 20;
static bool graph_ok(const lbrb_t* h) {
  return h->graph_mode != 0 &&
         (h->graph_mode == 1 || ((long)h->p.nx * h->p.ny <= GRAPH_MAX_NODES && !step_pairs_ok(h))) &&
         h->stream != nullptr && h->p.nudge == LBRB_NUDGE_NONE && !h->timing && !h->slab;
}

// two steps per launch: Dirichlet walls, no nudging (it acts between the
// steps), not a y-slab (ghost rows are exchanged every step)
static bool pairs_ok(const lbrb_t* h) {
  return h->pair_mode != 0 && h->p.twall == LBRB_TWALL_DIRICHLET && h->p.nudge == LBRB_NUDGE_NONE && !h->slab;
}

// lbrb_step's two steps per launch: as pairs_ok, and also with bilinear
// nudging (step n's innovations are formed before the launch and added to g
// inside it; step n+1's are applied after it, as a single step applies them)
static bool step_pairs_ok(const lbrb_t* h) {
  return h->pair_mode != 0 && h->p.twall == LBRB_TWALL_DIRICHLET &&
         (h->p.nudge == LBRB_NUDGE_NONE || h->p.nudge == LBRB_NUDGE_BILINEAR) && !h->slab;
}

static int slab_pair_launch(lbrb_t* h, bool rec1, bool rec2, bool last);  // (y-slabs, below)

int lbrb_step(lbrb_t* h, int n) {
  if (!h || n < 0) return fail(h, LBRB_ERR_ARG, "step: bad arguments");
  NvtxRange nvtx("lbrb_step");
  if (n == 0) return LBRB_OK;
  if (h->slab && !h->slab_stepping && n == 2 && h->p.nudge == LBRB_NUDGE_NONE &&
      h->p.twall == LBRB_TWALL_DIRICHLET && h->pair_mode != 0) {
    // one process per GPU: two steps from the two-row ghost blocks
    // (lbrb_slab_pack2 and the exchange of lbrb_slab_buffers2 done)
    if (!h->moments_valid)
      return fail(h, LBRB_ERR_STATE, "step: set the moments (set_moments, moments_from_pre or init_conduction) first");
    if (!h->slab_gh2_packed)
      return fail(h, LBRB_ERR_STATE,
                  "step: two steps on a y-slab need lbrb_slab_pack2 and the ghost-block exchange first");
    const bool own = moves_particles(h);  // (the slab holds its own particles)
    if (own && (h->sp->part_step != h->istep || h->sp->recv_step != h->istep))
      return fail(h, LBRB_ERR_STATE,
                  "step: a slab with particles steps after lbrb_slab_particles_step and lbrb_slab_particles_recv "
                  "of its last step");
    CK(h, cudaSetDevice(h->dev));
    const int i1 = h->istep + 1, i2 = h->istep + 2;
    const bool rec1 = own && h->p.noutconfig > 0 && i1 % h->p.noutconfig == 0;
    const bool rec2 = own && h->p.noutconfig > 0 && i2 % h->p.noutconfig == 0;
    const int rc = slab_pair_launch(h, rec1, rec2, true);
    if (rc) return rc;
    h->slab_gh2_packed = false;
    h->prev_valid = false;
    h->prev_pair = false;
    if (!own) {
      h->cur ^= 1;
      h->istep += 2;
      return LBRB_OK;
    }
    // the first step's state (u^n in the free slot, T^n in the source
    // buffer): its particle exchange runs next, and its
    // lbrb_slab_particles_recv moves the handle on to the second step's
    h->pair_save[0] = h->cur, h->pair_save[1] = h->uvcur, h->pair_save[2] = h->uvprev;
    const int A = 3 - h->uvcur - h->uvprev;
    h->uvprev = h->uvcur;
    h->uvcur = A;
    h->istep = i1;
    h->sp->pair_pending = true;
    return LBRB_OK;
  }
  if (h->slab && (n != 1 || (h->p.nudge == LBRB_NUDGE_BILINEAR && !h->slab_stepping && !h->sp)))
    return fail(h, LBRB_ERR_ARG,
                "step: a y-slab takes one step per boundary exchange, or two after lbrb_slab_pack2 (lbrb_slab_step); "
                "a nudged slab stepped alone needs the moment messages (lbrb_slab_particles_set)");
  if (h->sp && !h->slab_stepping && h->sp->cap > 0 &&
      (h->sp->part_step != h->istep || h->sp->recv_step != h->istep))
    return fail(h, LBRB_ERR_STATE,
                "step: a slab with particles steps after lbrb_slab_particles_step and lbrb_slab_particles_recv "
                "of its last step");
  if (h->sp && !h->slab_stepping && h->p.nudge == LBRB_NUDGE_BILINEAR && h->sp->nudge_step != h->istep)
    return fail(h, LBRB_ERR_STATE, "step: a nudged slab applies lbrb_slab_nudge after each step");
  if (!h->moments_valid)
    return fail(h, LBRB_ERR_STATE, "step: set the moments (set_moments, moments_from_pre or init_conduction) first");
  if (h->np > 0 && !h->particles_set) return fail(h, LBRB_ERR_STATE, "step: particles not set");
  if (h->p.nudge == LBRB_NUDGE_REFBOX && !h->nudge_init_done)
    return fail(h, LBRB_ERR_STATE, "step: nudge_init not called");
  CK(h, cudaSetDevice(h->dev));
  const bool f32 = fp32(h);
  const bool refbox = h->p.nudge == LBRB_NUDGE_REFBOX;
  const int nx = h->p.nx, ny = h->p.ny;
  if (h->lb_shape < 0) {
    // autotune the fused kernel's launch shape on this grid (trial launches
    // write only the buffers the real step overwrites)
    int sh = h->p.launch_shape;
    float ms = 0.f;
    if (h->p.autotune && !refbox && !tuned_get(g_tuned_single, h, &sh, &ms)) {
      // trials store u, v as the steps will (particles need them every step),
      // into the slot the first step overwrites
      const bool mp = moves_particles(h);
      const int tuv = mp ? 3 - h->uvcur - h->uvprev : h->uvcur;
      if (f32) sh = tune_lb_fp32(make_view<float>(h, h->cur, h->cur ^ 1, tuv, mp, 0), h->p.twall, h->stream, &ms);
      else sh = tune_lb_fp64(make_view<double>(h, h->cur, h->cur ^ 1, tuv, mp, 0), h->p.twall, h->stream, &ms);
      CK(h, cudaGetLastError());
      tuned_put(g_tuned_single, h, sh, ms);
    }
    CK(h, cudaGetLastError());
    h->lb_shape = sh;
    h->lb_shape_ms = ms;
  }
  // the record of step istep in ring slot `slot`, written by a particle
  // kernel on stream ps: copied to the host ring on the copy stream
  auto record_copy = [&](int istep, int slot, double* rslot, cudaStream_t ps) -> int {
    h->h_ring_step[slot] = istep;
    CK(h, cudaEventRecord(h->ring_ev[slot], ps));
    CK(h, cudaStreamWaitEvent(h->copy_stream, h->ring_ev[slot], 0));
    const size_t per = (size_t)h->nrec_fields * h->np;
    const int tc = tmark_begin(h, 3, h->copy_stream);
    CK(h, cudaMemcpyAsync(h->h_ring + (size_t)slot * per, rslot, per * sizeof(double), cudaMemcpyDeviceToHost,
                          h->copy_stream));
    tmark_end(h, tc, h->copy_stream);
    CK(h, cudaEventRecord(h->ring_ev[slot], h->copy_stream));
    h->rec_head++;
    h->join_pending = true;
    return LBRB_OK;
  };
  // one step's launches; `last` writes the moments
  const bool pdl_ok = !h->timing;  // (per-kernel timing keeps plain launches)
  // the bilinear observations of step `istep` (rows [x][y][T] of nobs), or null
  auto obs_row = [&](int istep) -> const double* {
    if (!h->obs || istep < h->obs_first || (!h->p.obs_cycle && istep >= h->obs_first + h->obs_nsteps))
      return nullptr;
    int row = istep - h->obs_first;
    if (h->p.obs_cycle) row %= h->obs_nsteps;
    return h->obs + (size_t)row * 3 * h->nobs;
  };
  auto one = [&](bool last) -> int {
    const int istep = h->istep + 1;
    const bool rec = h->np > 0 && h->p.noutconfig > 0 && istep % h->p.noutconfig == 0;
    if (rec && !h->slab && (h->rec_head - h->rec_tail) >= h->p.record_slots)
      return fail(h, LBRB_ERR_OVERFLOW, "step: record ring full, drain records first");
    const double* obs = nullptr;
    if (h->p.nudge == LBRB_NUDGE_BILINEAR) {
      obs = obs_row(istep);
      if (!obs) return fail(h, LBRB_ERR_STATE, "step: no bilinear observations for this step");
    }
    if (refbox) {
      const int nt = h->p.ntempread;
      if (istep % nt == 1 && !h->nudge_file_loaded)
        return fail(h, LBRB_ERR_STATE, "step: observation file for this interval not loaded");
      const int tm = tmark_begin(h, 2, h->stream);
      CK(h, launch_box_nudge(h->nb, h->nbi, h->nobs, nx, ny, h->slab ? h->slab_ny_total : ny, h->slab ? h->slab_j0 : 0,
                             nt, istep, h->ncx, h->ncy,
                             h->cell_count, h->cell_start, h->cell_fill, h->cell_dirty,
                             h->cell_items, h->nudge_vol, h->tempreadint, h->pitch, h->dflags,
                             h->stream));
      tmark_end(h, tm, h->stream);
      if (istep % nt == 1) h->nudge_file_loaded = false;
    }
    const int write_uv = moves_particles(h) || last;
    // T for the records (a slab's own too) and the nudging scatter; rho only
    // for the call's end
    const bool rec_own = h->sp && h->p.noutconfig > 0 && istep % h->p.noutconfig == 0;
    const int write_rt = last ? 3 : ((rec || rec_own || h->p.nudge == LBRB_NUDGE_BILINEAR) ? 1 : 0);
    const int src = h->cur, dst = h->cur ^ 1;
    const int uvn = write_uv ? 3 - h->uvcur - h->uvprev : h->uvcur;
    {
      const int tm = tmark_begin(h, 0, h->stream);
      // programmatic dependent launch when the kernel before it is this
      // loop's own (the fused kernel waits for it before touching memory)
      if (f32) CK(h, launch_lb_fp32(make_view<float>(h, src, dst, uvn, write_uv, write_rt), h->p.twall, h->lb_shape, h->stream, pdl_ok));
      else CK(h, launch_lb_fp64(make_view<double>(h, src, dst, uvn, write_uv, write_rt), h->p.twall, refbox, h->lb_shape, h->stream, pdl_ok));
      tmark_end(h, tm, h->stream);
    }
    if (h->slab) h->slab_obs = obs;  // (y-slabs: lbrb_slab_step nudges once every slab has stepped)
    if (obs && !h->slab) {
      const int tm = tmark_begin(h, 2, h->stream);
      CK(h, launch_bilinear_nudge(h->T[dst], pop_base(h, dst, 1), f32, h->plane, nx, ny, h->pitch, obs,
                                  obs + h->nobs, obs + 2 * (size_t)h->nobs, h->nobs, h->p.alpha,
                                  h->acc, h->dflags, h->stream, pdl_ok));
      tmark_end(h, tm, h->stream);
    }
    if (h->np > 0 && !h->slab) {  // (y-slabs: lbrb_slab_step moves the particles)
      // Particles of step n, in order on the step stream.  (Run on a second
      // stream beside the next fused kernel, with events ordering the u, v
      // slots and T buffers, they slowed the fused kernel by about their own
      // time on B200, so they stay in order.)
      const int ub = write_uv ? h->uvcur : h->uvprev;
      const int slot = rec ? (int)(h->rec_head % h->p.record_slots) : 0;
      double* rslot = rec ? h->d_ring + (size_t)slot * h->nrec_fields * h->np : nullptr;
      const int tm = tmark_begin(h, 1, h->stream);
      CK(h, launch_particles(h->uv[uvn][0], h->uv[uvn][1], h->uv[ub][0], h->uv[ub][1],
                             h->T[dst], f32, nx, ny, h->pitch, h->px, h->ptype, h->np, h->p.beta,
                             rec ? 1 : 0, h->p.record_full, rslot, h->dflags, h->stream, pdl_ok));
      tmark_end(h, tm, h->stream);
      if (rec) {
        const int rc = record_copy(istep, slot, rslot, h->stream);
        if (rc) return rc;
      }
    }
    h->cur = dst;
    h->prev_valid = true;
    h->prev_pair = false;
    if (write_uv) {
      h->uvprev = h->uvcur;
      h->uvcur = uvn;
    }
    h->istep = istep;
    return LBRB_OK;
  };
  // Two plain steps n, n+1 in one launch (lb_pair_kernel), then the particles
  // of each.  Step n's T goes to the source buffer T[cur] (its particle
  // records read it there), step n+1's to T[cur ^ 1]; u, v of step n go to
  // the free slot and of step n+1 to the slot of u^{n-2}, as two `one` calls
  // would rotate them.  `last`: step n+1 ends the call and also stores rho
  // and u, v, as `one(true)` does.  The intermediate populations stay in
  // shared memory; the source buffer and F keep the state before the launch,
  // from which get_poststream rebuilds step n.
  auto two = [&](bool last) -> int {
    const int i1 = h->istep + 1, i2 = h->istep + 2;
    const bool parts = h->np > 0;
    const bool rec1 = parts && h->p.noutconfig > 0 && i1 % h->p.noutconfig == 0;
    const bool rec2 = parts && h->p.noutconfig > 0 && i2 % h->p.noutconfig == 0;
    const int src = h->cur, dst = h->cur ^ 1;
    const int A = parts ? 3 - h->uvcur - h->uvprev : h->uvcur;  // u^n
    // u^{n+1}: the slot of u^{n-2}; without particles only the call's last
    // step stores u, v, in the free slot as one(true) would
    const int B = parts ? h->uvprev : (last ? 3 - h->uvcur - h->uvprev : h->uvcur);
    const int wuv = parts ? 1 : 0;
    // bilinear nudging: step n's innovations before the launch (into acc2 and
    // the node mask, read inside it), step n+1's after it (T^{n+1} stored)
    const bool nud = h->p.nudge == LBRB_NUDGE_BILINEAR;
    const double* o1 = nud ? obs_row(i1) : nullptr;
    const double* o2 = nud ? obs_row(i2) : nullptr;
    const size_t no = (size_t)h->nobs;
    if (nud) {
      const int tm = tmark_begin(h, 2, h->stream);
      if (f32)
        CK(h, launch_obs_pre_fp32(make_view<float>(h, src, dst, A, 0, 0), o1, o1 + no, o1 + 2 * no, h->nobs,
                                  h->p.alpha, h->acc2, h->nmask, h->dflags, h->stream, pdl_ok));
      else
        CK(h, launch_obs_pre_fp64(make_view<double>(h, src, dst, A, 0, 0), o1, o1 + no, o1 + 2 * no, h->nobs,
                                  h->p.alpha, h->acc2, h->nmask, h->dflags, h->stream, pdl_ok));
      tmark_end(h, tm, h->stream);
    }
    {
      const int tm = tmark_begin(h, 0, h->stream);
      const int rt2 = last ? 3 : ((rec2 || nud) ? 1 : 0);
      if (f32) {
        LBView<float> V1 = make_view<float>(h, src, dst, A, wuv, rec1 ? 1 : 0);
        V1.T = (float*)h->T[src];
        V1.rho = (float*)h->rho[src];
        if (nud) {
          V1.nmask = h->nmask;
          V1.nacc = reinterpret_cast<const unsigned long long*>(h->acc2);
        }
        CK(h, launch_pair_fp32(V1, make_view<float>(h, dst, dst, B, wuv || last, rt2), h->pair_shape, h->stream,
                               pdl_ok));
      } else {
        LBView<double> V1 = make_view<double>(h, src, dst, A, wuv, rec1 ? 1 : 0);
        V1.T = (double*)h->T[src];
        V1.rho = (double*)h->rho[src];
        if (nud) {
          V1.nmask = h->nmask;
          V1.nacc = reinterpret_cast<const unsigned long long*>(h->acc2);
        }
        CK(h, launch_pair_fp64(V1, make_view<double>(h, dst, dst, B, wuv || last, rt2), h->pair_shape, h->stream,
                               pdl_ok));
      }
      tmark_end(h, tm, h->stream);
    }
    if (nud) {
      const int tm = tmark_begin(h, 2, h->stream);
      // step n+1's scatter, then its apply pass together with the clearing
      // of step n's in-launch sums
      CK(h, launch_bilinear_nudge_clear(h->T[dst], pop_base(h, dst, 1), f32, h->plane, nx, ny, h->pitch, o2, o2 + no,
                                        o2 + 2 * no, h->nobs, h->p.alpha, h->acc, o1, o1 + no, h->acc2, h->nmask,
                                        h->dflags, h->stream, pdl_ok));
      tmark_end(h, tm, h->stream);
    }
    if (parts) {
      // both steps of every particle in one launch; the ring slots in step order
      long head = h->rec_head;
      const int slot1 = rec1 ? (int)(head++ % h->p.record_slots) : 0;
      const int slot2 = rec2 ? (int)(head % h->p.record_slots) : 0;
      const size_t per = (size_t)h->nrec_fields * h->np;
      double* r1 = rec1 ? h->d_ring + (size_t)slot1 * per : nullptr;
      double* r2 = rec2 ? h->d_ring + (size_t)slot2 * per : nullptr;
      const void* fa[5] = {h->uv[A][0], h->uv[A][1], h->uv[h->uvcur][0], h->uv[h->uvcur][1], h->T[src]};
      const void* fb[5] = {h->uv[B][0], h->uv[B][1], h->uv[A][0], h->uv[A][1], h->T[dst]};
      const int tm = tmark_begin(h, 1, h->stream);
      CK(h, launch_particles_pair(fa, fb, f32, nx, ny, h->pitch, h->px, h->ptype, h->np, h->p.beta,
                                  h->p.record_full, r1, r2, h->dflags, h->stream, pdl_ok));
      tmark_end(h, tm, h->stream);
      if (rec1) {
        const int rc = record_copy(i1, slot1, r1, h->stream);
        if (rc) return rc;
      }
      if (rec2) {
        const int rc = record_copy(i2, slot2, r2, h->stream);
        if (rc) return rc;
      }
      h->uvprev = A;
      h->uvcur = B;
    } else if (last) {
      h->uvprev = h->uvcur;
      h->uvcur = B;
    }
    h->cur = dst;
    h->prev_valid = false;
    h->prev_pair = !nud;
    h->istep = i2;
    return LBRB_OK;
  };
  auto tune_pairs = [&]() -> int {
    const int src = h->cur, dst = h->cur ^ 1;
    const bool parts = h->np > 0;
    const int A = parts ? 3 - h->uvcur - h->uvprev : h->uvcur;
    const int B = parts ? h->uvprev : h->uvcur;
    const int wuv = parts ? 1 : 0;
    {
      float ms = 0.f;
      int sh = 0;
      if (!tuned_get(g_tuned_pair, h, &sh, &ms)) {
        if (f32) {
          LBView<float> t1 = make_view<float>(h, src, dst, A, wuv, 0), t2 = make_view<float>(h, dst, dst, B, wuv, 0);
          sh = tune_pair_fp32(t1, t2, h->stream, &ms);
        } else {
          LBView<double> t1 = make_view<double>(h, src, dst, A, wuv, 0), t2 = make_view<double>(h, dst, dst, B, wuv, 0);
          sh = tune_pair_fp64(t1, t2, h->stream, &ms);
        }
        CK(h, cudaGetLastError());
        tuned_put(g_tuned_pair, h, sh, ms);
      }
      h->pair_shape = sh;
      h->pair_ms = ms;
      // automatic mode keeps pairs only where one beats two tuned single launches
      if (h->pair_mode < 0 && h->lb_shape_ms > 0.f && ms >= 2.f * h->lb_shape_ms) h->pair_mode = 0;
    }
    return LBRB_OK;
  };
  bool graphs_on = graph_ok(h);  // (refined below for a caller's capture)
  if (step_pairs_ok(h) && h->pair_shape < 0 && n >= 3) {
    // the pair shape is timed on the first call that can use pairs (trial
    // launches write only what the steps overwrite)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(h, cudaStreamIsCapturing(h->stream, &cs));
    if (cs == cudaStreamCaptureStatusNone && !(graphs_on && n - 1 >= GRAPH_STEPS)) {
      const int rc = tune_pairs();
      if (rc) return rc;
    }
  }
  // Small grids: a run of GRAPH_STEPS plain steps (no record, not the call's
  // last step) replays a CUDA graph of exactly the launches `one` would
  // issue.  Those launches depend only on the buffer phase (cur, uvcur,
  // uvprev), so one graph per phase is captured on first use.
  bool graphs = graph_ok(h);
  if (graphs) {
    // a caller capturing this stream gets the launches themselves
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(h, cudaStreamIsCapturing(h->stream, &cs));
    graphs = cs == cudaStreamCaptureStatusNone;
  }
  int s = 0;
  while (s < n) {
    if (graphs && n - 1 - s >= GRAPH_STEPS) {
      bool plain = true;
      if (h->np > 0 && h->p.noutconfig > 0)
        for (int q = 1; q <= GRAPH_STEPS; q++) plain = plain && (h->istep + q) % h->p.noutconfig != 0;
      if (plain) {
        const int key = h->cur * 9 + h->uvcur * 3 + h->uvprev;
        if (!h->graph_exec[key]) {
          const int cur0 = h->cur, uvc0 = h->uvcur, uvp0 = h->uvprev, ist0 = h->istep;
          cudaGraph_t g = nullptr;
          CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
          int rc = LBRB_OK;
          for (int q = 0; q < GRAPH_STEPS && rc == LBRB_OK; q++) rc = one(false);
          const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
          h->cur = cur0, h->uvcur = uvc0, h->uvprev = uvp0, h->istep = ist0;  // captured, not run
          if (rc != LBRB_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
          }
          if (ec != cudaSuccess) return fail(h, LBRB_ERR_CUDA, "step: graph capture", ec);
          const cudaError_t ei = cudaGraphInstantiate(&h->graph_exec[key], g, 0);
          cudaGraphDestroy(g);
          if (ei != cudaSuccess) {
            h->graph_exec[key] = nullptr;
            return fail(h, LBRB_ERR_CUDA, "step: graph instantiate", ei);
          }
        }
        CK(h, cudaGraphLaunch(h->graph_exec[key], h->stream));
        // the state after the replayed steps, as `one` leaves it
        for (int q = 0; q < GRAPH_STEPS; q++) {
          h->cur ^= 1;
          if (h->np > 0) {
            const int uvn = 3 - h->uvcur - h->uvprev;
            h->uvprev = h->uvcur;
            h->uvcur = uvn;
          }
        }
        h->prev_valid = true;
        h->prev_pair = false;
        h->istep += GRAPH_STEPS;
        s += GRAPH_STEPS;
        continue;
      }
    }
    // the call's last step joins a pair when the call's remaining steps
    // are exactly two and no nudging acts between them (get_poststream
    // rebuilds it from the state before the pair)
    const bool last_pair = n - s == 2 && h->p.nudge == LBRB_NUDGE_NONE;
    if (!graphs && h->pair_shape >= 0 && step_pairs_ok(h) && (n - 1 - s >= 2 || last_pair)) {
      // two steps per launch; a pair whose records would not fit in the
      // ring, or whose observations are missing, runs as single steps (which
      // report the error at the same step)
      int need = 0;
      for (int q = 1; q <= 2; q++)
        need += h->np > 0 && h->p.noutconfig > 0 && (h->istep + q) % h->p.noutconfig == 0;
      const bool obs_ok = h->p.nudge != LBRB_NUDGE_BILINEAR || (obs_row(h->istep + 1) && obs_row(h->istep + 2));
      if (h->rec_head - h->rec_tail + need <= h->p.record_slots && obs_ok) {
        const int rc = two(n - s == 2);
        if (rc) return rc;
        s += 2;
        continue;
      }
    }
    const int rc = one(s == n - 1 && !h->slab_defer_moments);
    if (rc) return rc;
    s++;
  }
  // the caller's stream sees the record copies as part of the steps
  if (h->join_pending) {
    CK(h, cudaEventRecord(h->join_ev, h->copy_stream));
    CK(h, cudaStreamWaitEvent(h->stream, h->join_ev, 0));
    h->join_pending = false;
  }
  h->slab_gh2_packed = false;  // (a y-slab's two-row ghost blocks now lag its state)
  return LBRB_OK;
}

int lbrb_adjoint_set_obs(lbrb_t* h, int nobs_steps, const int* steps, int nobs, const double* x,
                         const double* y, const double* T) {
  if (!h || nobs_steps < 1 || nobs < 1 || !steps || !x || !y || !T)
    return fail(h, LBRB_ERR_ARG, "adjoint_set_obs: bad arguments");
  for (int a = 0; a < nobs_steps; a++)
    if (steps[a] < 1 || (a > 0 && steps[a] <= steps[a - 1]))
      return fail(h, LBRB_ERR_ARG, "adjoint_set_obs: steps must be >= 1 and increasing");
  CK(h, cudaSetDevice(h->dev));
  if (h->adj_obs) cudaFree(h->adj_obs);
  if (h->adj_res) cudaFree(h->adj_res);
  h->adj_obs = nullptr;
  h->adj_res = nullptr;
  delete[] h->adj_steps;
  h->adj_steps = nullptr;
  const size_t n = (size_t)nobs_steps * nobs;
  if (cudaMalloc(&h->adj_obs, 3 * n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->adj_res, n * sizeof(double)) != cudaSuccess)
    return fail(h, LBRB_ERR_NOMEM, "adjoint_set_obs: allocation");
  for (int a = 0; a < nobs_steps; a++) {
    double* b = h->adj_obs + (size_t)a * 3 * nobs;
    CK(h, cudaMemcpyAsync(b, x + (size_t)a * nobs, nobs * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(b + nobs, y + (size_t)a * nobs, nobs * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(b + 2 * nobs, T + (size_t)a * nobs, nobs * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }
  CK(h, cudaStreamSynchronize(h->stream));
  h->adj_steps = new int[nobs_steps];
  std::memcpy(h->adj_steps, steps, nobs_steps * sizeof(int));
  h->adj_nobs = nobs;
  h->adj_nsteps_obs = nobs_steps;
  return LBRB_OK;
}

static int grow(lbrb_t* h, void** p, size_t* have, size_t need) {
  if (*have >= need) return LBRB_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc(p, need);
  if (e != cudaSuccess) return fail(h, LBRB_ERR_NOMEM, "adjoint buffers", e);
  *have = need;
  return LBRB_OK;
}

// Assimilation window, in one of two forms that give the same J and gradient
// bit for bit.
// Store (a gradient window whose moment blocks fit, or lbrb_adjoint_set_store
// 1): the forward pass writes every state's moment block (F and the
// moments, MB_PLANES planes) to the store, two steps per launch, the
// populations alternating between two slots; the backward pass reads the
// store and recomputes nothing.
// Checkpoints every K steps (otherwise): step i of segment c reads its input
// state from checkpoint c (i = 0) or segment slot i, and writes its output to
// slot i+1 -- or, for the segment's last step, to checkpoint c+1 (the
// window's end state: slot K).  The last segment's states are therefore still
// in the slots when the backward pass starts and need no recompute.
// Backward: segments last to first; each is recomputed into the slots (all
// but the last), then its steps run in reverse, two at a time through the
// pair kernel (lambda crosses HBM once per two steps) and one at a time for
// an odd leftover.  Results do not depend on K.
int lbrb_adjoint_window(lbrb_t* h, const double* T0, int nsteps, int K, double* J, double* dJdT0) {
  if (!h || !T0 || nsteps < 1 || K < 1 || !J) return fail(h, LBRB_ERR_ARG, "adjoint_window: bad arguments");
  NvtxRange nvtx("lbrb_adjoint_window");
  if (h->p.twall != LBRB_TWALL_DIRICHLET || h->p.nudge != LBRB_NUDGE_NONE)
    return fail(h, LBRB_ERR_UNSUPPORTED, "adjoint_window: Dirichlet walls without nudging only");
  if (h->slab) return fail(h, LBRB_ERR_UNSUPPORTED, "adjoint_window: whole domains only, not a y-slab");
  if (!h->adj_obs) return fail(h, LBRB_ERR_STATE, "adjoint_window: no observations set");
  CK(h, cudaSetDevice(h->dev));
  const bool f32 = fp32(h);
  const int nx = h->p.nx, ny = h->p.ny, pitch = h->pitch;
  const size_t plane = h->plane, es = h->esize;
  const size_t sb = SLOT_PLANES * plane * es;  // one state slot: pops, F, moments
  const size_t mbb = MB_PLANES * plane * es;    // one moment block: F, moments
  const size_t nn = (size_t)nx * ny;
  int rc;
  // store mode: every state's moment block, when asked or when it fits in
  // half of the free device memory (the store of an earlier window counts
  // as free: it is released before a larger one is allocated)
  bool store = false;
  if (dJdT0 && h->adj_store_mode != 0) {
    const size_t need = (size_t)(nsteps + 1) * mbb;
    store = h->adj_store_mode == 1 || h->adj_store_bytes >= need;
    if (!store) {
      size_t fr = 0, tot = 0;
      CK(h, cudaMemGetInfo(&fr, &tot));
      store = need <= (fr + h->adj_store_bytes) / 2;
    }
    if (store && (rc = grow(h, &h->adj_store, &h->adj_store_bytes, need))) return rc;
  }
  if (dJdT0 && !store && h->adj_store) {
    // a window too long for the store: release an earlier window's store
    // before the checkpoint buffers are allocated
    cudaFree(h->adj_store);
    h->adj_store = nullptr;
    h->adj_store_bytes = 0;
  }
  h->adj_store_used = store ? 1 : 0;
  // store mode: one segment of the whole window (no checkpoints), the
  // populations alternating between checkpoint slots 0 and 1 (slot 2 takes
  // the pair tuner's second output)
  if (K > nsteps || store) K = nsteps;
  const int nchk = (nsteps + K - 1) / K;
  if ((rc = grow(h, &h->adj_chk, &h->adj_chk_bytes, (size_t)(store ? 3 : nchk) * sb))) return rc;
  // two segment buffers: the backward sweep of one segment reads one while
  // the recompute of the segment before it fills the other
  if (!store && (rc = grow(h, &h->adj_seg, &h->adj_seg_bytes, 2 * (size_t)(K + 1) * sb))) return rc;
  if (!h->adj_T0 && cudaMalloc(&h->adj_T0, nn * sizeof(double)) != cudaSuccess)
    return fail(h, LBRB_ERR_NOMEM, "adjoint T0");
  CK(h, cudaMemcpyAsync(h->adj_T0, T0, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const double T0ref = T0_of(h), ng = -h->p.gravity;
  const double om = 1. / h->p.relax, omg = 1. / h->p.relaxg;
  // observation step lookup
  std::vector<int> obs_at(nsteps + 1, -1);
  for (int a = 0; a < h->adj_nsteps_obs; a++)
    if (h->adj_steps[a] <= nsteps) obs_at[h->adj_steps[a]] = a;
  const int nob = h->adj_nobs;
  char* chk = (char*)h->adj_chk;
  char* seg = (char*)h->adj_seg;
  char* const mstore = (char*)h->adj_store;
  // where the tuners' trial launches write (overwritten by the forward pass)
  char* const trial1 = store ? chk + sb : seg + sb;
  char* const trial2 = store ? chk + 2 * sb : seg + 2 * sb;
  // segment c's states live in buffer (nchk-1-c) % 2: the last segment, which
  // the forward pass leaves in place, in buffer 0
  auto segbuf = [&](int c) -> char* { return seg + (size_t)((nchk - 1 - c) & 1) * (K + 1) * sb; };
  auto state_in = [&](int c, int i) -> char* { return i == 0 ? chk + (size_t)c * sb : segbuf(c) + (size_t)i * sb; };
  // the state after i steps of segment c (its last step writes the next
  // checkpoint; the last segment's, slot K)
  auto after = [&](int c, int i) -> char* {
    if (i < std::min(K, nsteps - c * K)) return state_in(c, i);
    return c + 1 < nchk ? chk + (size_t)(c + 1) * sb : segbuf(c) + (size_t)K * sb;
  };
  // the moment block of a slot, and of state s in the store
  auto mb = [&](char* slot) -> char* { return slot + (size_t)SLOT_F * plane * es; };
  auto mblk = [&](int s) -> char* { return mstore + (size_t)s * mbb; };
  // the window's initial state in checkpoint 0 (pops + F), moments in
  // buffer 0; in store mode F also in the store's block 0
  CK(h, launch_init_from_T0(h->adj_T0, chk, h->rho[0], h->uv[h->uvcur][0], h->uv[h->uvcur][1],
                            h->T[0], mb(chk), f32, nx, ny, pitch, plane, T0ref, ng, h->stream));
  if (store) CK(h, cudaMemcpyAsync(mblk(0), mb(chk), plane * es, cudaMemcpyDeviceToDevice, h->stream));
  if (h->lb_shape < 0) {
    // the fused kernel's launch shape, timed on this window's initial state
    int sh = h->p.launch_shape;
    float ms = 0.f;
    if (h->p.autotune) {
      if (f32) sh = tune_lb_fp32(seg_view<float>(h, chk, trial1, 0), h->p.twall, h->stream, &ms);
      else sh = tune_lb_fp64(seg_view<double>(h, chk, trial1, 0), h->p.twall, h->stream, &ms);
    }
    CK(h, cudaGetLastError());
    h->lb_shape = sh;
    h->lb_shape_ms = ms;
  }
  const int shape = h->lb_shape;
  auto launch_fwd_on = [&](const char* src, char* dst, int mom, cudaStream_t st) -> cudaError_t {
    // programmatic dependent launch: each step may start while the one
    // before it in the stream finishes (the kernel waits for it first)
    if (f32) return launch_lb_fp32(seg_view<float>(h, src, dst, mom), h->p.twall, shape, st, true);
    return launch_lb_fp64(seg_view<double>(h, src, dst, mom), h->p.twall, false, shape, st, true);
  };
  auto launch_fwd = [&](const char* src, char* dst, int mom) { return launch_fwd_on(src, dst, mom, h->stream); };
  // two steps per launch where the state between them is not read: not an
  // observation step, not in a segment whose states the backward pass keeps
  const bool fwd_pairs = pairs_ok(h) && nsteps >= 2;
  if (fwd_pairs && h->pair_shape < 0) {
    // the pair tile shape, timed on the window's initial state (trial
    // launches write two slots that the forward pass overwrites)
    float ms = 0.f;
    int sh = 0;
    if (f32) sh = tune_pair_fp32(seg_view<float>(h, chk, trial1, 0), seg_view<float>(h, chk, trial2, 0), h->stream, &ms);
    else sh = tune_pair_fp64(seg_view<double>(h, chk, trial1, 0), seg_view<double>(h, chk, trial2, 0), h->stream, &ms);
    CK(h, cudaGetLastError());
    h->pair_shape = sh;
    h->pair_ms = ms;
    if (h->pair_mode < 0 && h->lb_shape_ms > 0.f && ms >= 2.f * h->lb_shape_ms) h->pair_mode = 0;
  }
  // residual of observation step oi from a moment block's T
  auto residual = [&](int oi, const char* mblock) -> cudaError_t {
    const double* ob = h->adj_obs + (size_t)oi * 3 * nob;
    return launch_obs_residual(mblock + 4 * plane * es, f32, nx, ny, pitch, ob, ob + nob, ob + 2 * nob,
                               nob, h->adj_res + (size_t)oi * nob, h->stream);
  };
  // ---- forward pass: checkpoints (or the store), residuals
  char* end_state = nullptr;  // populations of the window's end state
  char* end_F = nullptr;      // its F
  if (store) {
    // every state's moment block into the store; two steps per launch, the
    // first step's F and moments stored too, so observation steps need not
    // end a launch
    char* pop[2] = {chk, chk + sb};
    int pc = 0;
    // one step's view: populations pop[pc] -> pop[pc ^ 1], F of state s in,
    // F and moments of state s + 1 out
    auto sview = [&](auto zero, int s) {
      using Real = decltype(zero);
      LBView<Real> V = make_view<Real>(h, 0, 1, h->uvcur, 1, 3);
      const Real* a = (const Real*)pop[pc];
      Real* b = (Real*)pop[pc ^ 1];
      const Real* mi = (const Real*)mblk(s);
      Real* mo = (Real*)mblk(s + 1);
      V.fsrc = a;
      V.gsrc = a + NPOP * plane;
      V.fdst = b;
      V.gdst = b + NPOP * plane;
      V.Fin = mi;
      V.Fout = mo;
      V.rho = mo + plane;
      V.u = mo + 2 * plane;
      V.v = mo + 3 * plane;
      V.T = mo + 4 * plane;
      return V;
    };
    for (int s = 0; s < nsteps;) {
      if (fwd_pairs && h->pair_mode != 0 && s + 2 <= nsteps) {
        if (f32) {
          LBView<float> V1 = sview(0.f, s);
          V1.write_F = 1;
          CK(h, launch_pair_fp32(V1, sview(0.f, s + 1), h->pair_shape, h->stream, true));
        } else {
          LBView<double> V1 = sview(0.0, s);
          V1.write_F = 1;
          CK(h, launch_pair_fp64(V1, sview(0.0, s + 1), h->pair_shape, h->stream, true));
        }
        for (int q = 1; q <= 2; q++)
          if (obs_at[s + q] >= 0) CK(h, residual(obs_at[s + q], mblk(s + q)));
        s += 2;
      } else {
        if (f32) CK(h, launch_lb_fp32(sview(0.f, s), h->p.twall, shape, h->stream, true));
        else CK(h, launch_lb_fp64(sview(0.0, s), h->p.twall, false, shape, h->stream, true));
        if (obs_at[s + 1] >= 0) CK(h, residual(obs_at[s + 1], mblk(s + 1)));
        s += 1;
      }
      pc ^= 1;
    }
    end_state = pop[pc];
    end_F = mblk(nsteps);
  }
  for (int c = 0; c < nchk && !store; c++) {
    const int s0 = c * K, len = std::min(K, nsteps - s0);
    const bool last = c + 1 == nchk;
    // the last two segments keep every state for the backward pass (one in
    // each segment buffer); inside a segment that the backward pass
    // recomputes, the states alternate between slots 1 and 2 (a footprint
    // that stays in L2)
    const bool keep = dJdT0 && c + 2 >= nchk;
    char* const slot1 = segbuf(c) + sb;
    char* cur_state = state_in(c, 0);
    for (int i = 0; i < len;) {
      const int s = s0 + i + 1;
      // where the state after step i + q goes
      auto out = [&](int q) -> char* {
        if (i + q < len) return keep ? segbuf(c) + (size_t)(i + q) * sb : (cur_state == slot1 ? slot1 + sb : slot1);
        return last ? segbuf(c) + (size_t)K * sb : chk + (size_t)(c + 1) * sb;
      };
      if (fwd_pairs && h->pair_mode != 0 && !keep && i + 1 < len && obs_at[s] < 0) {
        char* dst = out(2);
        const int oi = obs_at[s + 1];
        const int mom = (dJdT0 && i + 2 == len) || oi >= 0;
        if (f32)
          CK(h, launch_pair_fp32(seg_view<float>(h, cur_state, dst, 0), seg_view<float>(h, cur_state, dst, mom),
                                 h->pair_shape, h->stream, true));
        else
          CK(h, launch_pair_fp64(seg_view<double>(h, cur_state, dst, 0), seg_view<double>(h, cur_state, dst, mom),
                                 h->pair_shape, h->stream, true));
        if (oi >= 0) CK(h, residual(oi, mb(dst)));
        cur_state = dst;
        i += 2;
        continue;
      }
      char* dst = out(1);
      const int oi = obs_at[s];
      // moments into every state the backward pass reads (and at observation
      // steps, for the residual's T)
      CK(h, launch_fwd(cur_state, dst, (dJdT0 && (keep || i + 1 == len)) || oi >= 0));
      if (oi >= 0) CK(h, residual(oi, mb(dst)));
      cur_state = dst;
      i++;
    }
    end_state = cur_state;
    end_F = mb(cur_state);
  }
  // misfit on the device (observation steps inside the window: a prefix)
  int nused = 0;
  while (nused < h->adj_nsteps_obs && h->adj_steps[nused] <= nsteps) nused++;
  double* dJ = h->red;  // reduction scratch of the handle
  CK(h, launch_misfit(h->adj_res, (long)nused * nob, dJ, h->stream));
  CK(h, cudaMemcpyAsync(h->h_scalar, dJ, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  // the handle's state: end of the window
  {
    const size_t popb = 2 * NPOP * plane * es;
    CK(h, cudaMemcpyAsync(h->pops[h->cur], end_state, popb, cudaMemcpyDeviceToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->F[h->cur], end_F, plane * es, cudaMemcpyDeviceToDevice, h->stream));
    h->prev_valid = false;
    h->prev_pair = false;
  }
  if (!dJdT0) {
    CK(h, cudaStreamSynchronize(h->stream));
    *J = *h->h_scalar;
    return LBRB_OK;
  }
  // ---- backward pass
  const size_t lp = NPOP * plane;  // one lambda population set (doubles)
  if (!h->adj_lam && cudaMalloc((void**)&h->adj_lam, (4 * lp + 2 * plane) * sizeof(double)) != cudaSuccess)
    return fail(h, LBRB_ERR_NOMEM, "adjoint lambda");
  if (!h->adj_lT && cudaMalloc((void**)&h->adj_lT, 2 * plane * sizeof(long long)) != cudaSuccess)
    return fail(h, LBRB_ERR_NOMEM, "adjoint lambda T");
  double* lam[2][2] = {{h->adj_lam, h->adj_lam + lp}, {h->adj_lam + 2 * lp, h->adj_lam + 3 * lp}};
  double* lF[2] = {h->adj_lam + 4 * lp, h->adj_lam + 4 * lp + plane};
  long long* lT[2] = {h->adj_lT, h->adj_lT + plane};
  CK(h, cudaMemsetAsync(h->adj_lam, 0, (4 * lp + 2 * plane) * sizeof(double), h->stream));
  CK(h, cudaMemsetAsync(h->adj_lT, 0, 2 * plane * sizeof(long long), h->stream));
  int lc = 0, fc = 0;  // lam[lc]: adjoint of the current state; lF[fc]: lambda F of the next step
  // the moment blocks the backward pass reads: state i of segment c, and the
  // state after i steps of segment c (in store mode, one segment: state i)
  auto m_in = [&](int c, int i) -> char* { return store ? mblk(c * K + i) : mb(state_in(c, i)); };
  auto m_after = [&](int c, int i) -> char* { return store ? mblk(c * K + i) : mb(after(c, i)); };
  auto scatter = [&](int s, long long* acc) -> cudaError_t {
    const int oi = obs_at[s];
    if (oi < 0) return cudaSuccess;
    const double* ob = h->adj_obs + (size_t)oi * 3 * nob;
    return launch_adj_obs_scatter(ob, ob + nob, h->adj_res + (size_t)oi * nob, nob, nx, ny, pitch, acc, h->stream);
  };
  auto unscatter = [&](int s, long long* acc) -> cudaError_t {
    const int oi = obs_at[s];
    if (oi < 0) return cudaSuccess;
    const double* ob = h->adj_obs + (size_t)oi * 3 * nob;
    return launch_adj_obs_clear(ob, ob + nob, nob, nx, ny, pitch, acc, h->stream);
  };
  if (h->adj_pair_variant < 0) {
    // launch variants of the pair kernel, timed on the window's last pair
    // before anything runs beside it; every trial writes all of its outputs
    // from unchanged inputs, and the real launch later overwrites them
    int bv = 0;
    const int sl = nsteps, il = sl - (nchk - 1) * K - 1;
    if (il >= 1) {
      cudaEvent_t ea, eb;
      CK(h, cudaEventCreate(&ea));
      CK(h, cudaEventCreate(&eb));
      float best = 1e30f;
      for (int v = 0; v < adjoint_pair_variants(); v++) {
        auto trial = [&]() {
          return launch_adjoint_pair(f32, v, m_after(nchk - 1, il + 1), m_in(nchk - 1, il),
                                     m_in(nchk - 1, il - 1),
                                     lam[lc][0], lam[lc][1], lam[lc ^ 1][0], lam[lc ^ 1][1], lF[fc],
                                     lF[fc ^ 1], nullptr, nullptr, nx, ny, pitch, plane, om, omg, ng, T0ref,
                                     h->p.Tup, h->p.Tdown, h->stream);
        };
        CK(h, trial());
        CK(h, cudaEventRecord(ea, h->stream));
        CK(h, trial());
        CK(h, trial());
        CK(h, cudaEventRecord(eb, h->stream));
        CK(h, cudaEventSynchronize(eb));
        float ms = 0.f;
        CK(h, cudaEventElapsedTime(&ms, ea, eb));
        if (ms < best) best = ms, bv = v;
      }
      cudaEventDestroy(ea);
      cudaEventDestroy(eb);
    }
    h->adj_pair_variant = bv;
  }
  // The recompute of segment c-1 runs on the second stream while the
  // backward sweep of segment c runs on the handle's stream: the sweep is
  // latency-bound and leaves HBM bandwidth for the recompute.  Events order
  // each buffer's reuse (a recompute waits for the sweep that last read its
  // buffer; a sweep waits for its recompute).
  cudaEvent_t ev_fwd = nullptr, ev_rec[2] = {nullptr, nullptr}, ev_bwd[2] = {nullptr, nullptr};
  struct EvGuard {
    cudaEvent_t* e[5];
    ~EvGuard() {
      for (cudaEvent_t* p : e)
        if (*p) cudaEventDestroy(*p);
    }
  } ev_guard{{&ev_fwd, &ev_rec[0], &ev_rec[1], &ev_bwd[0], &ev_bwd[1]}};
  for (cudaEvent_t* p : ev_guard.e) CK(h, cudaEventCreateWithFlags(p, cudaEventDisableTiming));
  cudaStream_t rs = h->pstream;
  CK(h, cudaEventRecord(ev_fwd, h->stream));
  CK(h, cudaStreamWaitEvent(rs, ev_fwd, 0));
  for (int c = nchk - 1; c >= 0; c--) {
    const int s0 = c * K, len = std::min(K, nsteps - s0), s1 = s0 + len;
    const int b = (nchk - 1 - c) & 1;
    if (c >= 1 && c + 1 < nchk) {
      // recompute segment c-1 into the other buffer, after the sweep that
      // read it (segment nchk-2 is still there from the forward pass)
      const int cp = c - 1, lenp = std::min(K, nsteps - cp * K);
      CK(h, cudaStreamWaitEvent(rs, ev_bwd[b ^ 1], 0));
      // the sweep reads each state's moments and F, never its populations,
      // so two steps go in one launch whose first step stores only those
      for (int i = 0; i + 1 < lenp;) {
        char* s1p = segbuf(cp) + (size_t)(i + 1) * sb;
        if (fwd_pairs && h->pair_mode != 0 && i + 2 < lenp) {
          char* s2p = s1p + sb;
          if (f32) {
            LBView<float> V1 = seg_view<float>(h, state_in(cp, i), s1p, 1);
            V1.write_F = 1;
            CK(h, launch_pair_fp32(V1, seg_view<float>(h, s1p, s2p, 1), h->pair_shape, rs, true));
          } else {
            LBView<double> V1 = seg_view<double>(h, state_in(cp, i), s1p, 1);
            V1.write_F = 1;
            CK(h, launch_pair_fp64(V1, seg_view<double>(h, s1p, s2p, 1), h->pair_shape, rs, true));
          }
          i += 2;
        } else {
          CK(h, launch_fwd_on(state_in(cp, i), s1p, 1, rs));
          i++;
        }
      }
      CK(h, cudaEventRecord(ev_rec[b ^ 1], rs));
    }
    if (c + 2 < nchk) CK(h, cudaStreamWaitEvent(h->stream, ev_rec[b], 0));
    int s = s1;
    while (s > s0) {
      const int i = s - s0 - 1;
      if (s - 1 > s0) {
        // steps s and s-1 in one launch
        CK(h, scatter(s, lT[0]));
        CK(h, scatter(s - 1, lT[1]));
        auto pair = [&](int variant) {
          return launch_adjoint_pair(f32, variant, m_after(c, i + 1), m_in(c, i), m_in(c, i - 1),
                                     lam[lc][0], lam[lc][1],
                                     lam[lc ^ 1][0], lam[lc ^ 1][1], lF[fc], lF[fc ^ 1],
                                     obs_at[s] >= 0 ? lT[0] : nullptr, obs_at[s - 1] >= 0 ? lT[1] : nullptr,
                                     nx, ny, pitch, plane, om, omg, ng, T0ref, h->p.Tup, h->p.Tdown,
                                     h->stream);
        };
        CK(h, pair(h->adj_pair_variant));
        CK(h, unscatter(s, lT[0]));
        CK(h, unscatter(s - 1, lT[1]));
        lc ^= 1;
        fc ^= 1;
        s -= 2;
      } else {
        CK(h, scatter(s, lT[0]));
        CK(h, launch_adjoint_step(f32, m_after(c, i + 1), m_in(c, i),
                                  lam[lc][0], lam[lc][1], lam[lc ^ 1][0], lam[lc ^ 1][1], lF[fc],
                                  obs_at[s] >= 0 ? lT[0] : nullptr, nx, ny, pitch, plane, om, omg, ng,
                                  T0ref, h->p.Tup, h->p.Tdown, h->stream));
        CK(h, unscatter(s, lT[0]));
        lc ^= 1;
        s -= 1;
      }
    }
    CK(h, cudaEventRecord(ev_bwd[b], h->stream));
  }
  CK(h, launch_adj_initial(lam[lc][1], lF[fc], nx, ny, pitch, plane, ng, h->adj_T0, h->stream));
  CK(h, cudaMemcpyAsync(dJdT0, h->adj_T0, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  *J = *h->h_scalar;
  return LBRB_OK;
}

int lbrb_adjoint_variants(void) { return adjoint_pair_variants(); }

int lbrb_adjoint_set_variant(lbrb_t* h, int variant) {
  if (!h || variant < -1 || variant >= adjoint_pair_variants())
    return fail(h, LBRB_ERR_ARG, "adjoint_set_variant: variant out of range");
  h->adj_pair_variant = variant;
  return LBRB_OK;
}

int lbrb_adjoint_get_variant(const lbrb_t* h, int* variant) {
  if (!h || !variant) return LBRB_ERR_ARG;
  *variant = h->adj_pair_variant;
  return LBRB_OK;
}

int lbrb_adjoint_set_store(lbrb_t* h, int mode) {
  if (!h || mode < -1 || mode > 1) return fail(h, LBRB_ERR_ARG, "adjoint_set_store: mode must be -1, 0 or 1");
  h->adj_store_mode = mode;
  if (mode == 0 && h->adj_store) {
    CK(h, cudaSetDevice(h->dev));
    CK(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->adj_store);
    h->adj_store = nullptr;
    h->adj_store_bytes = 0;
  }
  return LBRB_OK;
}

int lbrb_adjoint_get_store(const lbrb_t* h, int* mode, int* used_last, size_t* bytes) {
  if (!h) return LBRB_ERR_ARG;
  if (mode) *mode = h->adj_store_mode;
  if (used_last) *used_last = h->adj_store_used;
  if (bytes) *bytes = h->adj_store_bytes;
  return LBRB_OK;
}

// ------------------------------------------------------------ y-slabs
// One domain over several GPUs, cut into slabs of rows.  The reference cuts
// its domain over MPI ranks and refreshes halo rows of the populations by
// message passing (pbc, temppart_dump.c:234-250, called around the stream in
// the loop, temppart_dump.c:1674-1759); here a slab's step pulls
// the three f and three g populations that cross an inner boundary from
// ghost rows filled from the neighbour's boundary row (lbrb_slab_pack), and
// the walls apply only at the domain's own bottom and top.
int lbrb_slab_set(lbrb_t* h, int j0, int ny_total) {
  if (!h) return LBRB_ERR_ARG;
  if (j0 < 0 || ny_total < 2 || j0 + h->p.ny > ny_total)
    return fail(h, LBRB_ERR_ARG, "slab_set: rows [j0, j0 + ny) must lie in [0, ny_total)");
  if (h->np > 0)
    return fail(h, LBRB_ERR_UNSUPPORTED,
                "slab_set: a slab's particles are set by lbrb_slab_particles_set (create it with nprtcl = 0)");
  CK(h, cudaSetDevice(h->dev));
  free_sp(h->sp);  // (its rows change)
  h->sp = nullptr;
  const size_t gb = lbrb_slab_ghost_bytes(h);
  const size_t gb2 = (size_t)SLAB_GH2_PLANES * h->p.nx * h->esize;
  void** bufs[] = {&h->slab_ghost_lo, &h->slab_ghost_hi, &h->slab_up, &h->slab_down,
                   &h->slab_gh2_lo, &h->slab_gh2_hi, &h->slab_up2, &h->slab_down2};
  for (void** b : bufs) {
    if (*b) cudaFree(*b);
    *b = nullptr;
  }
  // ghost rows only across inner boundaries (none at a wall of the domain)
  const bool lo = j0 > 0, hi = j0 + h->p.ny < ny_total;
  if ((lo && (cudaMalloc(&h->slab_ghost_lo, gb) != cudaSuccess || cudaMalloc(&h->slab_gh2_lo, gb2) != cudaSuccess)) ||
      (hi && (cudaMalloc(&h->slab_ghost_hi, gb) != cudaSuccess || cudaMalloc(&h->slab_gh2_hi, gb2) != cudaSuccess)))
    return fail(h, LBRB_ERR_NOMEM, "slab ghosts");
  if (cudaMalloc(&h->slab_up, gb) != cudaSuccess || cudaMalloc(&h->slab_down, gb) != cudaSuccess ||
      cudaMalloc(&h->slab_up2, gb2) != cudaSuccess || cudaMalloc(&h->slab_down2, gb2) != cudaSuccess)
    return fail(h, LBRB_ERR_NOMEM, "slab boundary rows");
  for (void* b : {h->slab_ghost_lo, h->slab_ghost_hi, h->slab_up, h->slab_down})
    if (b) CK(h, cudaMemsetAsync(b, 0, gb, h->stream));
  for (void* b : {h->slab_gh2_lo, h->slab_gh2_hi, h->slab_up2, h->slab_down2})
    if (b) CK(h, cudaMemsetAsync(b, 0, gb2, h->stream));
  if (!h->slab_ev_xfer) CK(h, cudaEventCreateWithFlags(&h->slab_ev_xfer, cudaEventDisableTiming));
  if (!h->slab_ev_done) CK(h, cudaEventCreateWithFlags(&h->slab_ev_done, cudaEventDisableTiming));
  h->slab_sig.clear();  // (tables rebuilt on the next slab step)
  CK(h, cudaStreamSynchronize(h->stream));
  h->slab = true;
  h->slab_j0 = j0;
  h->slab_ny_total = ny_total;
  return LBRB_OK;
}

size_t lbrb_slab_ghost_bytes(const lbrb_t* h) { return h ? 6 * (size_t)h->p.nx * h->esize : 0; }

size_t lbrb_slab_ghost2_bytes(const lbrb_t* h) { return h ? (size_t)SLAB_GH2_PLANES * h->p.nx * h->esize : 0; }

int lbrb_slab_buffers2(lbrb_t* h, void** up, void** down, void** ghost_lo, void** ghost_hi) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->slab) return fail(h, LBRB_ERR_STATE, "slab_buffers2: not a y-slab (lbrb_slab_set)");
  if (up) *up = h->slab_up2;
  if (down) *down = h->slab_down2;
  if (ghost_lo) *ghost_lo = h->slab_gh2_lo;
  if (ghost_hi) *ghost_hi = h->slab_gh2_hi;
  return LBRB_OK;
}

int lbrb_slab_pack2(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->slab) return fail(h, LBRB_ERR_STATE, "slab_pack2: not a y-slab (lbrb_slab_set)");
  CK(h, cudaSetDevice(h->dev));
  CK(h, launch_slab_pack2(h->pops[h->cur], h->F[h->cur], fp32(h), h->p.nx, h->p.ny, h->pitch, h->plane, h->slab_up2,
                          h->slab_down2, h->stream));
  h->slab_gh2_packed = true;
  return LBRB_OK;
}

int lbrb_slab_buffers(lbrb_t* h, void** up, void** down, void** ghost_lo, void** ghost_hi) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->slab) return fail(h, LBRB_ERR_STATE, "slab_buffers: not a y-slab (lbrb_slab_set)");
  if (up) *up = h->slab_up;
  if (down) *down = h->slab_down;
  if (ghost_lo) *ghost_lo = h->slab_ghost_lo;
  if (ghost_hi) *ghost_hi = h->slab_ghost_hi;
  return LBRB_OK;
}

int lbrb_slab_pack(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->slab) return fail(h, LBRB_ERR_STATE, "slab_pack: not a y-slab (lbrb_slab_set)");
  CK(h, cudaSetDevice(h->dev));
  CK(h, launch_slab_pack(h->pops[h->cur], fp32(h), h->p.nx, h->p.ny, h->pitch, h->plane, h->slab_up,
                         h->slab_down, h->stream));
  h->slab_gh2_packed = false;
  return LBRB_OK;
}

// ------------------------------------------------- owner-slab particles
// The particles of a y-slab held by the slab whose rows hold their cell, as
// the reference's ranks hold them (init_prtcl keeps a rank's particles,
// Trajectories/code/mympi2.h:116-290; toggle_prtcl hands the leavers to the
// neighbour, :568-760).  Per step, after the slab's lbrb_step(h, 1):
// lbrb_slab_moments_pack, the exchange of the moment messages,
// lbrb_slab_particles_step, the exchange of the hand-off lists and
// lbrb_slab_particles_recv (own_*_kernel, particle_kernels.cu).

// the cell row of a position as the device computes it (cell_row)
static int host_cell_row(double yy, int ny) {
  if (!(yy > -2.0 && yy < ny + 2.0)) return 0;
  int r = ((int)yy - 1) % ny;
  return r < 0 ? r + ny : r;
}

// the 14 field tables of the particle kernels: for every row of the domain,
// the row in this slab's planes, in a received moment message (one row below
// the slab, two above, periodic in y) or the zero row
static std::vector<const void*> own_tables(const lbrb_t* h) {
  const SlabParts& S = *h->sp;
  const int nyT = h->slab_ny_total, j0 = h->slab_j0, nyl = h->p.ny;
  const size_t rowb = (size_t)h->pitch * h->esize;
  auto mplane = [&](int which, int q) -> const void* {
    return (const char*)S.mom[which] + MOM_PLANES_OFF + (size_t)q * S.mom_pstride;
  };
  // per role (u, v, u^{n-1}, v^{n-1}, T): the planes of the lo message and of
  // the hi message's two rows (-1: not sent, the zero row)
  const int lo_q[5] = {0, 1, -1, -1, 2}, hi0_q[5] = {0, 1, 2, 3, 4}, hi1_q[5] = {5, 6, -1, -1, 7};
  std::vector<const void*> t((size_t)OWN_TABLES * nyT, S.zrow);
  for (int j = 0; j < nyT; j++) {
    const int d = ((j - j0) % nyT + nyT) % nyT;
    const bool below = j == ((j0 - 1) % nyT + nyT) % nyT;
    for (int tab = 0; tab < OWN_TABLES; tab++) {
      const int role = tab < 3 ? 0 : tab < 6 ? 1 : tab < 9 ? 2 : tab < 12 ? 3 : 4;
      const void* own = role == 4 ? h->T[tab - 12] : h->uv[tab % 3][role & 1];
      const void* r = S.zrow;
      if (d < nyl) r = (const char*)own + (size_t)d * rowb;
      else if (d == nyl) r = mplane(3, hi0_q[role]);
      else if (below) r = lo_q[role] >= 0 ? mplane(2, lo_q[role]) : S.zrow;
      else if (d == nyl + 1) r = hi1_q[role] >= 0 ? mplane(3, hi1_q[role]) : S.zrow;
      t[(size_t)tab * nyT + j] = r;
    }
  }
  return t;
}

int lbrb_slab_particle_format(int* msg_header_bytes, int* record_bytes, int* mom_planes_offset) {
  if (msg_header_bytes) *msg_header_bytes = (int)sizeof(SlabMsg);
  if (record_bytes) *record_bytes = (int)sizeof(HandoffRec);
  if (mom_planes_offset) *mom_planes_offset = (int)MOM_PLANES_OFF;
  return LBRB_OK;
}

int lbrb_slab_particles_set(lbrb_t* h, int n, const int* ids, const double* x, const double* y, const double* u,
                            const double* v, const int* ptype, const double* invtau, int capacity,
                            int handoff_capacity) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->slab) return fail(h, LBRB_ERR_STATE, "slab_particles_set: not a y-slab (lbrb_slab_set)");
  // capacity -1: no particles, the moment messages only (bilinear nudging)
  const bool msg_only = capacity == -1;
  if (n < 0 || (n > 0 && (!ids || !x || !y || !u || !v || !ptype || !invtau)) || capacity < -1 ||
      handoff_capacity < 0 || (msg_only && n > 0))
    return fail(h, LBRB_ERR_ARG, "slab_particles_set: bad arguments");
  const int nyT = h->slab_ny_total, j0 = h->slab_j0, nyl = h->p.ny;
  std::vector<int> keep;
  for (int q = 0; q < n; q++) {
    if (!(x[q] > -1.0 && x[q] < h->p.nx + 1.0 && y[q] >= 0.0 && y[q] <= nyT + 1.0))
      return fail(h, LBRB_ERR_RANGE, "slab_particles_set: position outside the domain");
    if (!(u[q] == u[q]) || !(v[q] == v[q]) || !(invtau[q] >= 0.0) ||
        (ptype[q] != LBRB_PTYPE_TRACER && ptype[q] != LBRB_PTYPE_INERTIAL))
      return fail(h, LBRB_ERR_ARG, "slab_particles_set: bad velocity, type or 1/tau");
    const int cr = host_cell_row(y[q], nyT);
    if (cr >= j0 && cr < j0 + nyl) keep.push_back(q);
  }
  long cap = msg_only ? 0 : (capacity > 0 ? capacity : std::max(n, 1));
  cap = (cap + 127) / 128 * 128;
  if ((long)keep.size() > cap || cap > (1L << 22))
    return fail(h, LBRB_ERR_ARG, "slab_particles_set: capacity below the slab's particles or too large");
  const int xcap = msg_only ? 0 : (handoff_capacity > 0 ? handoff_capacity : (int)std::min(cap, 1024L));
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaStreamSynchronize(h->stream));
  free_sp(h->sp);
  h->sp = new SlabParts();
  SlabParts& S = *h->sp;
  S.cap = (int)cap;
  S.xcap = xcap;
  const size_t C = (size_t)cap;
  S.mom_pstride = ((size_t)h->p.nx * h->esize + 255) / 256 * 256;
  S.mom_up_bytes = MOM_PLANES_OFF + MOM_UP_PLANES * S.mom_pstride;
  S.mom_down_bytes = MOM_PLANES_OFF + MOM_DOWN_PLANES * S.mom_pstride;
  S.hand_bytes = msg_only ? 0 : HAND_RECS_OFF + (size_t)xcap * sizeof(HandoffRec);
  bool bad = false;
  if (!msg_only) {
    for (int b = 0; b < 2; b++)
      bad = bad || dalloc(&S.P[b], 9 * C) || dalloc(&S.id[b], C) || dalloc(&S.type[b], C);
    bad = bad || dalloc(&S.cnt, 2) || dalloc(&S.cls, C) || dalloc(&S.bcnt, 3 * (C / 128)) || dalloc(&S.done, 1);
  }
  bad = bad || cudaMalloc(&S.rows, (size_t)OWN_TABLES * nyT * sizeof(void*)) != cudaSuccess ||
        cudaMalloc(&S.zrow, (size_t)h->pitch * h->esize) != cudaSuccess;
  for (int m = 0; m < 4 && !bad; m++)
    bad = cudaMalloc(&S.mom[m], (m & 1) ? S.mom_down_bytes : S.mom_up_bytes) != cudaSuccess ||
          (!msg_only && cudaMalloc(&S.hand[m], S.hand_bytes) != cudaSuccess);
  const int slots = h->p.record_slots;
  const int nrec = h->p.record_full ? LBRB_REC_NFULL : LBRB_REC_NBASIC;
  if (!bad && !msg_only && h->p.noutconfig > 0) {
    bad = dalloc(&S.d_rec, (size_t)slots * nrec * C) || dalloc(&S.d_rid, (size_t)slots * C) ||
          dalloc(&S.d_rcnt, (size_t)slots) ||
          cudaMallocHost(&S.h_rec, (size_t)slots * nrec * C * sizeof(double)) != cudaSuccess ||
          cudaMallocHost(&S.h_rid, (size_t)slots * C * sizeof(int)) != cudaSuccess ||
          cudaMallocHost(&S.h_rcnt, (size_t)slots * sizeof(int)) != cudaSuccess;
    S.rstep.assign(slots, 0);
    S.rev.assign(slots, nullptr);
    for (int q = 0; q < slots && !bad; q++)
      bad = cudaEventCreateWithFlags(&S.rev[q], cudaEventDisableTiming) != cudaSuccess;
  }
  for (cudaEvent_t* e : {&S.ev_mom, &S.ev_part, &S.ev_hand})
    bad = bad || cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess;
  if (bad) {
    free_sp(h->sp);
    h->sp = nullptr;
    return fail(h, LBRB_ERR_NOMEM, "slab_particles_set: buffers");
  }
  h->nrec_fields = nrec;
  CK(h, cudaMemsetAsync(S.zrow, 0, (size_t)h->pitch * h->esize, h->stream));
  for (int m = 0; m < 4; m++) {
    CK(h, cudaMemsetAsync(S.mom[m], 0, (m & 1) ? S.mom_down_bytes : S.mom_up_bytes, h->stream));
    if (!msg_only) CK(h, cudaMemsetAsync(S.hand[m], 0, S.hand_bytes, h->stream));
  }
  const std::vector<const void*> tab = own_tables(h);
  CK(h, cudaMemcpyAsync(S.rows, tab.data(), tab.size() * sizeof(void*), cudaMemcpyHostToDevice, h->stream));
  S.part_step = S.recv_step = S.nudge_step = h->istep;
  S.mom_step = -1;
  if (msg_only) {
    CK(h, cudaStreamSynchronize(h->stream));
    return LBRB_OK;
  }
  CK(h, cudaMemsetAsync(S.cls, 3, C, h->stream));
  CK(h, cudaMemsetAsync(S.done, 0, sizeof(unsigned), h->stream));
  // the kept particles, in the order given
  const size_t k = keep.size();
  std::vector<double> P(9 * C, 0.0);
  std::vector<int> I(C, 0), T(C, 0);
  for (size_t a = 0; a < k; a++) {
    const int q = keep[a];
    const double vals[9] = {x[q], y[q], u[q], v[q], x[q], y[q], u[q], v[q], invtau[q]};
    for (int f = 0; f < 9; f++) P[(size_t)f * C + a] = vals[f];
    I[a] = ids[q];
    T[a] = ptype[q];
  }
  const int cnt[2] = {(int)k, (int)k};
  CK(h, cudaMemcpyAsync(S.P[0], P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(S.id[0], I.data(), C * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(S.type[0], T.data(), C * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(S.cnt, cnt, sizeof(cnt), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return LBRB_OK;
}

int lbrb_slab_particle_bytes(const lbrb_t* h, size_t* mom_up, size_t* mom_down, size_t* handoff) {
  if (!h || !h->sp) return LBRB_ERR_ARG;
  if (mom_up) *mom_up = h->sp->mom_up_bytes;
  if (mom_down) *mom_down = h->sp->mom_down_bytes;
  if (handoff) *handoff = h->sp->hand_bytes;
  return LBRB_OK;
}

int lbrb_slab_particle_buffers(lbrb_t* h, void** mom_up, void** mom_down, void** mom_lo, void** mom_hi,
                               void** hand_up, void** hand_down, void** hand_lo, void** hand_hi) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->sp) return fail(h, LBRB_ERR_STATE, "slab_particle_buffers: no slab particles (lbrb_slab_particles_set)");
  void** out[8] = {mom_up, mom_down, mom_lo, mom_hi, hand_up, hand_down, hand_lo, hand_hi};
  for (int m = 0; m < 4; m++) {
    if (out[m]) *out[m] = h->sp->mom[m];
    if (out[4 + m]) *out[4 + m] = h->sp->hand[m];
  }
  return LBRB_OK;
}

int lbrb_slab_moments_pack(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->sp) return fail(h, LBRB_ERR_STATE, "slab_moments_pack: no slab particles (lbrb_slab_particles_set)");
  SlabParts& S = *h->sp;
  if (S.cap > 0 ? h->istep != S.part_step + 1 : S.mom_step == h->istep)
    return fail(h, LBRB_ERR_STATE, "slab_moments_pack: once per step, after lbrb_step(h, 1)");
  CK(h, cudaSetDevice(h->dev));
  CK(h, launch_slab_mom_pack(h->uv[h->uvcur][0], h->uv[h->uvcur][1], h->uv[h->uvprev][0], h->uv[h->uvprev][1],
                             h->T[h->cur], fp32(h), h->p.nx, h->p.ny, h->pitch, S.dst_mom[0] ? S.dst_mom[0] : S.mom[0],
                             S.dst_mom[1] ? S.dst_mom[1] : S.mom[1], S.mom_pstride, h->istep, h->slab_j0, h->stream,
                             !h->timing));
  S.mom_step = h->istep;
  return LBRB_OK;
}

int lbrb_slab_particles_step(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->sp) return fail(h, LBRB_ERR_STATE, "slab_particles_step: no slab particles (lbrb_slab_particles_set)");
  SlabParts& S = *h->sp;
  if (S.cap == 0) return fail(h, LBRB_ERR_STATE, "slab_particles_step: the slab holds no particles (capacity -1)");
  if (h->istep != S.part_step + 1 || S.recv_step != S.part_step || S.mom_step != h->istep)
    return fail(h, LBRB_ERR_STATE,
                "slab_particles_step: once per step, after lbrb_step(h, 1), lbrb_slab_moments_pack and the "
                "moment exchange");
  const int istep = h->istep, nyT = h->slab_ny_total;
  const bool rec = h->p.noutconfig > 0 && istep % h->p.noutconfig == 0;
  const int slots = h->p.record_slots;
  if (rec && S.rhead - S.rtail >= slots)
    return fail(h, LBRB_ERR_OVERFLOW, "slab_particles_step: record ring full, drain records first");
  CK(h, cudaSetDevice(h->dev));
  const int slot = rec ? (int)(S.rhead % slots) : 0;
  const size_t per = (size_t)h->nrec_fields * S.cap;
  const void* const* tab = (const void* const*)S.rows;
  // after the step: u, v in slot uvcur, the step's input in uvprev, T in cur
  const void* rows5[5] = {tab + (size_t)h->uvcur * nyT, tab + (size_t)(3 + h->uvcur) * nyT,
                          tab + (size_t)(6 + h->uvprev) * nyT, tab + (size_t)(9 + h->uvprev) * nyT,
                          tab + (size_t)(12 + h->cur) * nyT};
  const int tm = tmark_begin(h, 1, h->stream);
  CK(h, launch_own_particles(rows5, fp32(h), h->p.nx, nyT, S, S.dst_hand[0] ? S.dst_hand[0] : S.hand[0],
                             S.dst_hand[1] ? S.dst_hand[1] : S.hand[1], h->slab_j0, h->p.ny, istep, h->p.beta,
                             rec ? 1 : 0, h->p.record_full, rec ? S.d_rec + (size_t)slot * per : nullptr,
                             rec ? S.d_rid + (size_t)slot * S.cap : nullptr, rec ? S.d_rcnt + slot : nullptr,
                             h->dflags, h->stream, !h->timing));
  tmark_end(h, tm, h->stream);
  S.pc ^= 1;
  if (rec) {
    // the record to the host ring on the copy stream
    S.rstep[slot] = istep;
    CK(h, cudaEventRecord(S.rev[slot], h->stream));
    CK(h, cudaStreamWaitEvent(h->copy_stream, S.rev[slot], 0));
    const int tc = tmark_begin(h, 3, h->copy_stream);
    CK(h, cudaMemcpyAsync(S.h_rec + (size_t)slot * per, S.d_rec + (size_t)slot * per, per * sizeof(double),
                          cudaMemcpyDeviceToHost, h->copy_stream));
    CK(h, cudaMemcpyAsync(S.h_rid + (size_t)slot * S.cap, S.d_rid + (size_t)slot * S.cap, S.cap * sizeof(int),
                          cudaMemcpyDeviceToHost, h->copy_stream));
    CK(h, cudaMemcpyAsync(S.h_rcnt + slot, S.d_rcnt + slot, sizeof(int), cudaMemcpyDeviceToHost, h->copy_stream));
    tmark_end(h, tc, h->copy_stream);
    CK(h, cudaEventRecord(S.rev[slot], h->copy_stream));
    S.rhead++;
    h->join_pending = true;
  }
  S.part_step = istep;
  return LBRB_OK;
}

int lbrb_slab_particles_recv(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->sp) return fail(h, LBRB_ERR_STATE, "slab_particles_recv: no slab particles (lbrb_slab_particles_set)");
  SlabParts& S = *h->sp;
  if (S.cap == 0) return fail(h, LBRB_ERR_STATE, "slab_particles_recv: the slab holds no particles (capacity -1)");
  if (S.part_step != h->istep || S.part_step == S.recv_step)
    return fail(h, LBRB_ERR_STATE, "slab_particles_recv: once per step, after lbrb_slab_particles_step");
  CK(h, cudaSetDevice(h->dev));
  const int tm = tmark_begin(h, 1, h->stream);
  CK(h, launch_own_recv(S, h->slab_j0, h->p.ny, h->slab_ny_total, h->istep, h->dflags, h->stream, !h->timing));
  tmark_end(h, tm, h->stream);
  S.recv_step = h->istep;
  if (S.pair_pending) {
    // the second step of lbrb_step(h, 2): populations and T in the other
    // buffer, u^{n+1} in the slot of u^{n-2}
    h->cur = h->pair_save[0] ^ 1;
    h->uvprev = h->uvcur;
    h->uvcur = h->pair_save[2];
    h->istep += 1;
    S.pair_pending = false;
  }
  return LBRB_OK;
}

// Bilinear nudging of a y-slab stepped by its own process (the in-process
// lbrb_slab_step reads T through peer tables instead): the step's
// observations whose cell has a corner in the slab's rows are interpolated
// from T^n -- the slab's own rows and the received moment messages' T rows,
// which hold every corner row within one of the slab -- and their shares
// are scattered to, and applied at, the corners in the slab's rows.  The
// integer sums do not depend on which slab adds them, so g equals the whole
// domain's bit for bit.
int lbrb_slab_nudge(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  if (!h->slab || !h->sp)
    return fail(h, LBRB_ERR_STATE, "slab_nudge: a y-slab with the moment messages (lbrb_slab_particles_set) only");
  if (h->p.nudge != LBRB_NUDGE_BILINEAR) return fail(h, LBRB_ERR_STATE, "slab_nudge: bilinear nudging only");
  SlabParts& S = *h->sp;
  if (S.mom_step != h->istep || S.nudge_step == h->istep || !h->slab_obs)
    return fail(h, LBRB_ERR_STATE,
                "slab_nudge: once per step, after lbrb_step(h, 1), lbrb_slab_moments_pack and the moment exchange");
  CK(h, cudaSetDevice(h->dev));
  const int nyT = h->slab_ny_total;
  const double* obs = h->slab_obs;
  const void* const* Trows = (const void* const*)S.rows + (size_t)(12 + h->cur) * nyT;
  const int tm = tmark_begin(h, 2, h->stream);
  CK(h, launch_bilinear_nudge_slab(Trows, pop_base(h, h->cur, 1), fp32(h), h->plane, h->p.nx, nyT, h->slab_j0,
                                   h->p.ny, h->pitch, obs, obs + h->nobs, obs + 2 * (size_t)h->nobs, h->nobs,
                                   h->p.alpha, h->acc, h->dflags, h->stream));
  tmark_end(h, tm, h->stream);
  S.nudge_step = h->istep;
  return LBRB_OK;
}

int lbrb_slab_particles_count(lbrb_t* h, int* n) {
  if (!h || !n) return LBRB_ERR_ARG;
  if (!h->sp) return fail(h, LBRB_ERR_STATE, "slab_particles_count: no slab particles (lbrb_slab_particles_set)");
  CK(h, cudaSetDevice(h->dev));
  int c = 0;
  if (h->sp->cap == 0) {
    *n = 0;
    return LBRB_OK;
  }
  CK(h, cudaMemcpyAsync(&c, h->sp->cnt + 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  *n = c;
  return LBRB_OK;
}

int lbrb_slab_particles_get(lbrb_t* h, int max_n, int* n, int* ids, double* x, double* y, double* u, double* v,
                            double* xo, double* yo, double* uo, double* vo) {
  if (!h || !n || max_n < 0) return LBRB_ERR_ARG;
  int cnt = 0;
  const int rc = lbrb_slab_particles_count(h, &cnt);
  if (rc) return rc;
  if (cnt > max_n) return fail(h, LBRB_ERR_ARG, "slab_particles_get: max_n below the slab's particle count");
  const SlabParts& S = *h->sp;
  std::vector<double> P((size_t)8 * cnt);
  for (int a = 0; a < 8 && cnt > 0; a++)
    CK(h, cudaMemcpyAsync(P.data() + (size_t)a * cnt, S.P[S.pc] + (size_t)a * S.cap, cnt * sizeof(double),
                          cudaMemcpyDeviceToHost, h->stream));
  std::vector<int> I(cnt);
  if (cnt > 0) CK(h, cudaMemcpyAsync(I.data(), S.id[S.pc], cnt * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  double* outs[8] = {x, y, u, v, xo, yo, uo, vo};
  for (int a = 0; a < 8; a++)
    if (outs[a] && cnt > 0) std::memcpy(outs[a], &P[(size_t)a * cnt], cnt * sizeof(double));
  if (ids && cnt > 0) std::memcpy(ids, I.data(), cnt * sizeof(int));
  *n = cnt;
  return LBRB_OK;
}

int lbrb_slab_record_pending(lbrb_t* h, int* count) {
  if (!h || !count) return LBRB_ERR_ARG;
  *count = h->sp ? (int)(h->sp->rhead - h->sp->rtail) : 0;
  return LBRB_OK;
}

int lbrb_slab_record_drain(lbrb_t* h, int max_n, int* step, int* count, int* ids, double* buf) {
  if (!h || !step || !count || max_n < 0) return LBRB_ERR_ARG;
  *step = -1;
  *count = 0;
  if (!h->sp || h->sp->rtail == h->sp->rhead) return LBRB_OK;
  SlabParts& S = *h->sp;
  const int slot = (int)(S.rtail % h->p.record_slots);
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaEventSynchronize(S.rev[slot]));
  const int c = S.h_rcnt[slot];
  if (c > max_n) return fail(h, LBRB_ERR_ARG, "slab_record_drain: max_n below the record's particle count");
  const size_t per = (size_t)h->nrec_fields * S.cap;
  if (buf)
    for (int f = 0; f < h->nrec_fields; f++)
      std::memcpy(buf + (size_t)f * c, S.h_rec + (size_t)slot * per + (size_t)f * S.cap, c * sizeof(double));
  if (ids) std::memcpy(ids, S.h_rid + (size_t)slot * S.cap, c * sizeof(int));
  *step = S.rstep[slot];
  *count = c;
  S.rtail++;
  return LBRB_OK;
}

// One two-step launch of a y-slab from its two-row ghost blocks (filled by
// the neighbours' lbrb_slab_pack2), records of the steps as flagged; `last`:
// the second step writes the moments (it ends the call).  Buffers as two
// one-step launches leave them; the caller updates the handle's state.
static int slab_pair_launch(lbrb_t* h, bool rec1, bool rec2, bool last) {
  const bool parts = moves_particles(h);
  const int src = h->cur, dst = h->cur ^ 1;
  const int A = parts ? 3 - h->uvcur - h->uvprev : h->uvcur;
  const int B = parts ? h->uvprev : h->uvcur;
  const int wuv = parts ? 1 : 0;
  auto views = [&](auto zero, int r1, int r2, int w2) {
    using Real = decltype(zero);
    LBView<Real> V1 = make_view<Real>(h, src, dst, A, wuv, r1), V2 = make_view<Real>(h, dst, dst, B, w2, r2);
    V1.T = (Real*)h->T[src];
    V1.rho = (Real*)h->rho[src];
    for (LBView<Real>* V : {&V1, &V2}) {
      V->ghost_lo = V->gh2_lo = (const Real*)h->slab_gh2_lo;
      V->ghost_hi = V->gh2_hi = (const Real*)h->slab_gh2_hi;
    }
    return std::make_pair(V1, V2);
  };
  if (h->pair_shape < 0) {
    // the tile shape, timed on first use (trial launches write only what the
    // two steps overwrite)
    float ms = 0.f;
    int sh = 0;
    if (!tuned_get(g_tuned_pair, h, &sh, &ms)) {
      if (fp32(h)) {
        auto v = views(0.f, 0, 0, wuv);
        sh = tune_pair_fp32(v.first, v.second, h->stream, &ms);
      } else {
        auto v = views(0.0, 0, 0, wuv);
        sh = tune_pair_fp64(v.first, v.second, h->stream, &ms);
      }
      CK(h, cudaGetLastError());
      tuned_put(g_tuned_pair, h, sh, ms);
    }
    h->pair_shape = sh;
    h->pair_ms = ms;
  }
  const int r2 = last ? 3 : (rec2 ? 1 : 0), w2 = last ? 1 : wuv;
  const int tm = tmark_begin(h, 0, h->stream);
  if (fp32(h)) {
    auto v = views(0.f, rec1 ? 1 : 0, r2, w2);
    CK(h, launch_pair_fp32(v.first, v.second, h->pair_shape, h->stream, false));
  } else {
    auto v = views(0.0, rec1 ? 1 : 0, r2, w2);
    CK(h, launch_pair_fp64(v.first, v.second, h->pair_shape, h->stream, false));
  }
  tmark_end(h, tm, h->stream);
  return LBRB_OK;
}

// Tables for the bilinear nudging of a slab domain in one process, one copy
// on each slab's device (addresses are unified, so the copies are equal): for
// every row of the domain a pointer to that row of T (2 buffers) in the slab
// that holds it.  Kernels on one device read the other slabs' rows through
// peer access.
// peer access between every pair of the slabs' GPUs (kernels of one slab
// then read or write another slab's memory); false if a pair cannot have it
static bool peers_on(lbrb_t* const* slabs, int n) {
  for (int s = 0; s < n; s++)
    for (int t = 0; t < n; t++) {
      const int a = slabs[s]->dev, b = slabs[t]->dev;
      if (a == b) continue;
      int ok = 0;
      if (cudaDeviceCanAccessPeer(&ok, a, b) != cudaSuccess || !ok) return false;
      if (cudaSetDevice(a) != cudaSuccess) return false;
      const cudaError_t e = cudaDeviceEnablePeerAccess(b, 0);
      if (e == cudaErrorPeerAccessAlreadyEnabled) (void)cudaGetLastError();
      else if (e != cudaSuccess) return false;
    }
  return true;
}

static int slab_nudge_tables(lbrb_t* const* slabs, int n) {
  lbrb_t* h0 = slabs[0];
  std::vector<const void*> sig(slabs, slabs + n);
  bool fresh = true;
  for (int s = 0; s < n; s++) fresh = fresh && slabs[s]->slab_sig == sig;
  if (fresh) return LBRB_OK;
  if (!peers_on(slabs, n))
    return fail(slabs[0], LBRB_ERR_UNSUPPORTED, "slab_step: nudging needs peer access between the slabs' GPUs");
  const int nyT = h0->slab_ny_total;
  std::vector<const void*> tab((size_t)2 * nyT);
  for (int t = 0; t < n; t++) {
    const lbrb_t* h = slabs[t];
    const size_t rowb = (size_t)h->pitch * h->esize;
    for (int jl = 0; jl < h->p.ny; jl++)
      for (int b = 0; b < 2; b++) tab[(size_t)b * nyT + h->slab_j0 + jl] = (const char*)h->T[b] + jl * rowb;
  }
  const size_t bytes = tab.size() * sizeof(void*);
  for (int s = 0; s < n; s++) {
    lbrb_t* h = slabs[s];
    CK(h, cudaSetDevice(h->dev));
    if (h->slab_tab_bytes < bytes) {
      if (h->slab_tab) cudaFree(h->slab_tab);
      h->slab_tab = nullptr;
      h->slab_tab_bytes = 0;
      if (cudaMalloc(&h->slab_tab, bytes) != cudaSuccess) return fail(h, LBRB_ERR_NOMEM, "slab nudging tables");
      h->slab_tab_bytes = bytes;
    }
    CK(h, cudaMemcpyAsync(h->slab_tab, tab.data(), bytes, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    h->slab_sig = sig;
  }
  return LBRB_OK;
}

// The particles of one step of a slab domain in one process, after every
// slab's fused kernel: the exchange a process per GPU does over NCCL, around
// the ring of slabs (up to s + 1, down to s - 1, periodic).  `direct` (the
// slabs' GPUs reach each other's memory): the moment-row pack and the
// particle step write straight into the neighbours' receive buffers; else
// each slab's messages are peer-copied there.  A write into a neighbour's
// buffer waits for the neighbour's last read of it: the moment messages were
// last read by its previous particle step (ev_part), the hand-off lists by
// its previous receive, which comes before its moment pack (ev_mom).
static int slab_owner_particles(lbrb_t* const* slabs, int n, bool direct) {
  auto up = [&](int s) { return slabs[(s + 1) % n]; };
  auto dn = [&](int s) { return slabs[(s + n - 1) % n]; };
  auto wait_nb = [&](lbrb_t* h, int s, auto ev) -> int {
    CK(h, cudaStreamWaitEvent(h->stream, ev(up(s)), 0));
    CK(h, cudaStreamWaitEvent(h->stream, ev(dn(s)), 0));
    return LBRB_OK;
  };
  auto ev_part = [](lbrb_t* t) { return t->sp->ev_part; };
  auto ev_mom = [](lbrb_t* t) { return t->sp->ev_mom; };
  auto ev_hand = [](lbrb_t* t) { return t->sp->ev_hand; };
  // 1. moment messages
  for (int s = 0; s < n; s++) {
    lbrb_t* h = slabs[s];
    SlabParts& S = *h->sp;
    CK(h, cudaSetDevice(h->dev));
    int rc = wait_nb(h, s, ev_part);
    if (rc) return rc;
    if (direct) {
      S.dst_mom[0] = up(s)->sp->mom[2];
      S.dst_mom[1] = dn(s)->sp->mom[3];
    }
    rc = lbrb_slab_moments_pack(h);
    S.dst_mom[0] = S.dst_mom[1] = nullptr;
    if (rc) return rc;
    if (!direct) {
      CK(h, cudaMemcpyPeerAsync(up(s)->sp->mom[2], up(s)->dev, S.mom[0], h->dev, S.mom_up_bytes, h->stream));
      CK(h, cudaMemcpyPeerAsync(dn(s)->sp->mom[3], dn(s)->dev, S.mom[1], h->dev, S.mom_down_bytes, h->stream));
    }
    CK(h, cudaEventRecord(S.ev_mom, h->stream));
  }
  // 2. each slab's particles (and, direct, its hand-off lists into the neighbours)
  for (int s = 0; s < n; s++) {
    lbrb_t* h = slabs[s];
    SlabParts& S = *h->sp;
    CK(h, cudaSetDevice(h->dev));
    int rc = wait_nb(h, s, ev_mom);
    if (rc) return rc;
    if (direct) {
      S.dst_hand[0] = up(s)->sp->hand[2];
      S.dst_hand[1] = dn(s)->sp->hand[3];
    }
    rc = lbrb_slab_particles_step(h);
    S.dst_hand[0] = S.dst_hand[1] = nullptr;
    if (rc) return rc;
    CK(h, cudaEventRecord(S.ev_part, h->stream));
  }
  // 3. hand-off lists (copies)
  if (!direct)
    for (int s = 0; s < n; s++) {
      lbrb_t* h = slabs[s];
      CK(h, cudaSetDevice(h->dev));
      const int rc = wait_nb(h, s, ev_part);
      if (rc) return rc;
      CK(h, cudaMemcpyPeerAsync(up(s)->sp->hand[2], up(s)->dev, h->sp->hand[0], h->dev, h->sp->hand_bytes,
                                h->stream));
      CK(h, cudaMemcpyPeerAsync(dn(s)->sp->hand[3], dn(s)->dev, h->sp->hand[1], h->dev, h->sp->hand_bytes,
                                h->stream));
      CK(h, cudaEventRecord(h->sp->ev_hand, h->stream));
    }
  // 4. each slab appends what it received
  for (int s = 0; s < n; s++) {
    lbrb_t* h = slabs[s];
    CK(h, cudaSetDevice(h->dev));
    int rc = wait_nb(h, s, direct ? ev_part : ev_hand);
    if (!rc) rc = lbrb_slab_particles_recv(h);
    if (rc) return rc;
  }
  return LBRB_OK;
}

int lbrb_slab_step(lbrb_t* const* slabs, int n, int nsteps) {
  if (!slabs || n < 1 || nsteps < 0) return LBRB_ERR_ARG;
  for (int s = 0; s < n; s++) {
    const lbrb_t* h = slabs[s];
    if (!h || !h->slab) return LBRB_ERR_ARG;
    const lbrb_t* h0 = slabs[0];
    if (h->p.nx != h0->p.nx || h->esize != h0->esize || h->slab_ny_total != h0->slab_ny_total)
      return LBRB_ERR_ARG;
    // slabs in order, each starting where the previous ends
    if (h->slab_j0 != (s == 0 ? 0 : slabs[s - 1]->slab_j0 + slabs[s - 1]->p.ny)) return LBRB_ERR_ARG;
  }
  if (slabs[n - 1]->slab_j0 + slabs[n - 1]->p.ny != slabs[0]->slab_ny_total) return LBRB_ERR_ARG;
  lbrb_t* h0 = slabs[0];
  auto holds = [](const lbrb_t* h) { return h->sp != nullptr && h->sp->cap > 0; };
  const bool parts = holds(h0);
  const bool nudge = h0->p.nudge == LBRB_NUDGE_BILINEAR;
  for (int s = 0; s < n; s++) {
    lbrb_t* h = slabs[s];
    if (holds(h) != parts)
      return fail(h, LBRB_ERR_ARG, "slab_step: every slab or none holds particles (lbrb_slab_particles_set)");
    if (h->p.nudge != h0->p.nudge || h->p.alpha != h0->p.alpha || h->nobs != h0->nobs)
      return fail(h, LBRB_ERR_ARG, "slab_step: slabs differ in nudging");
    if (!parts) continue;
    if (h->p.noutconfig != h0->p.noutconfig || h->p.record_full != h0->p.record_full || h->p.beta != h0->p.beta ||
        h->istep != h0->istep || h->cur != h0->cur || h->uvcur != h0->uvcur || h->uvprev != h0->uvprev)
      return fail(h, LBRB_ERR_ARG, "slab_step: slabs differ in particle settings or step");
    if (h->sp->part_step != h->istep || h->sp->recv_step != h->istep)
      return fail(h, LBRB_ERR_STATE, "slab_step: a slab's particle exchange of its last step is unfinished");
  }
  if (nudge) {
    const int rc = slab_nudge_tables(slabs, n);
    if (rc) return rc;
  }
  // particle messages written straight into the neighbours' buffers when
  // every slab's GPU reaches the others' memory (one GPU: always)
  const bool direct = parts && peers_on(slabs, n);
  // records pending in the fullest slab ring (every slab records the same steps)
  auto ring_used = [&]() -> long {
    long m = 0;
    for (int s = 0; s < n; s++) m = std::max(m, slabs[s]->sp->rhead - slabs[s]->sp->rtail);
    return m;
  };
  const size_t gb = lbrb_slab_ghost_bytes(h0);
  const size_t gb2 = (size_t)SLAB_GH2_PLANES * h0->p.nx * h0->esize;
  // two steps per launch: Dirichlet walls, no nudging, never the call's last
  // step (which writes the moments)
  bool slab_pairs = !nudge && h0->p.twall == LBRB_TWALL_DIRICHLET;
  for (int s = 0; s < n; s++) slab_pairs = slab_pairs && slabs[s]->pair_mode != 0;
  // Two steps of every slab: the ghost blocks (two rows deep) go across each
  // inner boundary, then each slab runs lb_pair_kernel, whose ring rows beyond
  // an inner boundary come from them; then the particles, step by step.
  auto pair_iteration = [&]() -> int {
    const int i1 = h0->istep + 1, i2 = h0->istep + 2;
    const bool rec1 = parts && h0->p.noutconfig > 0 && i1 % h0->p.noutconfig == 0;
    const bool rec2 = parts && h0->p.noutconfig > 0 && i2 % h0->p.noutconfig == 0;
    for (int s = 0; s < n; s++) {
      lbrb_t* h = slabs[s];
      CK(h, cudaSetDevice(h->dev));
      if (s > 0) CK(h, cudaStreamWaitEvent(h->stream, slabs[s - 1]->slab_ev_done, 0));
      if (s + 1 < n) CK(h, cudaStreamWaitEvent(h->stream, slabs[s + 1]->slab_ev_done, 0));
      int rc = lbrb_slab_pack2(h);
      if (rc) return rc;
      if (s + 1 < n)
        CK(h, cudaMemcpyPeerAsync(slabs[s + 1]->slab_gh2_lo, slabs[s + 1]->dev, h->slab_up2, h->dev, gb2, h->stream));
      if (s > 0)
        CK(h, cudaMemcpyPeerAsync(slabs[s - 1]->slab_gh2_hi, slabs[s - 1]->dev, h->slab_down2, h->dev, gb2, h->stream));
      CK(h, cudaEventRecord(h->slab_ev_xfer, h->stream));
    }
    for (int s = 0; s < n; s++) {
      lbrb_t* h = slabs[s];
      CK(h, cudaSetDevice(h->dev));
      if (s > 0) CK(h, cudaStreamWaitEvent(h->stream, slabs[s - 1]->slab_ev_xfer, 0));
      if (s + 1 < n) CK(h, cudaStreamWaitEvent(h->stream, slabs[s + 1]->slab_ev_xfer, 0));
      const int rc = slab_pair_launch(h, rec1, rec2, false);
      if (rc) return rc;
      CK(h, cudaEventRecord(h->slab_ev_done, h->stream));
    }
    // the particles of each step, with each handle's buffer state set to that
    // step's (u^n in slot A, T^n in the source buffer)
    for (int q = 0; q < 2; q++) {
      for (int s = 0; s < n; s++) {
        lbrb_t* h = slabs[s];
        if (q == 0) {
          // after step n: T^n in the source buffer, u^n in the free slot
          h->pair_save[0] = h->cur, h->pair_save[1] = h->uvcur, h->pair_save[2] = h->uvprev;
          if (parts) {
            const int A = 3 - h->uvcur - h->uvprev;
            h->uvprev = h->uvcur;
            h->uvcur = A;
          }
          h->istep = i1;
        } else {
          // after step n+1: populations and T in the other buffer, u^{n+1}
          // in the slot of u^{n-2}
          h->cur = h->pair_save[0] ^ 1;
          if (parts) {
            h->uvprev = h->uvcur;
            h->uvcur = h->pair_save[2];
          }
          h->istep = i2;
        }
      }
      if (parts) {
        const int rc = slab_owner_particles(slabs, n, direct);
        if (rc) return rc;
      }
    }
    for (int s = 0; s < n; s++) slabs[s]->prev_valid = false, slabs[s]->prev_pair = false;
    return LBRB_OK;
  };
  for (int it = 0; it < nsteps; it++) {
    if (slab_pairs && nsteps - it >= 3) {
      int need = 0;
      for (int q = 1; q <= 2; q++) need += parts && h0->p.noutconfig > 0 && (h0->istep + q) % h0->p.noutconfig == 0;
      if (!parts || ring_used() + need <= h0->p.record_slots) {
        const int rc = pair_iteration();
        if (rc) return rc;
        it++;  // (and the loop's own increment)
        continue;
      }
    }
    if (parts && h0->p.noutconfig > 0 && (h0->istep + 1) % h0->p.noutconfig == 0 &&
        ring_used() >= h0->p.record_slots)
      return fail(h0, LBRB_ERR_OVERFLOW, "slab_step: record ring full, drain records first");
    // 1. each slab packs its boundary rows and copies them into its
    //    neighbours' ghost rows, once the neighbours' previous step (which
    //    read those ghost rows, possibly in an earlier call) is done
    for (int s = 0; s < n; s++) {
      lbrb_t* h = slabs[s];
      CK(h, cudaSetDevice(h->dev));
      if (s > 0) CK(h, cudaStreamWaitEvent(h->stream, slabs[s - 1]->slab_ev_done, 0));
      if (s + 1 < n) CK(h, cudaStreamWaitEvent(h->stream, slabs[s + 1]->slab_ev_done, 0));
      int rc = lbrb_slab_pack(h);
      if (rc) return rc;
      if (s + 1 < n)
        CK(h, cudaMemcpyPeerAsync(slabs[s + 1]->slab_ghost_lo, slabs[s + 1]->dev, h->slab_up, h->dev, gb, h->stream));
      if (s > 0)
        CK(h, cudaMemcpyPeerAsync(slabs[s - 1]->slab_ghost_hi, slabs[s - 1]->dev, h->slab_down, h->dev, gb, h->stream));
      CK(h, cudaEventRecord(h->slab_ev_xfer, h->stream));
    }
    // 2. each slab steps once its ghost rows are filled
    for (int s = 0; s < n; s++) {
      lbrb_t* h = slabs[s];
      CK(h, cudaSetDevice(h->dev));
      if (s > 0) CK(h, cudaStreamWaitEvent(h->stream, slabs[s - 1]->slab_ev_xfer, 0));
      if (s + 1 < n) CK(h, cudaStreamWaitEvent(h->stream, slabs[s + 1]->slab_ev_xfer, 0));
      // the moments (rho, u, v, T) are written on the last step only
      h->slab_defer_moments = it + 1 < nsteps;
      h->slab_stepping = true;
      int rc = lbrb_step(h, 1);
      h->slab_defer_moments = false;
      h->slab_stepping = false;
      if (rc) return rc;
      CK(h, cudaEventRecord(h->slab_ev_done, h->stream));
    }
    // 3. bilinear nudging: each slab's innovations read T of every slab and
    //    go to the corners in its own rows (g of the step's output)
    if (nudge) {
      for (int s = 0; s < n; s++) {
        lbrb_t* h = slabs[s];
        CK(h, cudaSetDevice(h->dev));
        for (int t = 0; t < n; t++)
          if (t != s) CK(h, cudaStreamWaitEvent(h->stream, slabs[t]->slab_ev_done, 0));
        const double* obs = h->slab_obs;
        const void* const* Trows = (const void* const*)h->slab_tab + (size_t)h->cur * h->slab_ny_total;
        const int tm = tmark_begin(h, 2, h->stream);
        CK(h, launch_bilinear_nudge_slab(Trows, pop_base(h, h->cur, 1), fp32(h), h->plane, h->p.nx, h->slab_ny_total,
                                         h->slab_j0, h->p.ny, h->pitch, obs, obs + h->nobs, obs + 2 * (size_t)h->nobs,
                                         h->nobs, h->p.alpha, h->acc, h->dflags, h->stream));
        tmark_end(h, tm, h->stream);
        if (h->sp) h->sp->nudge_step = h->istep;
      }
    }
    // 4. the particles of the step (each slab's next fused kernel runs after
    //    its receive on its stream)
    if (parts) {
      const int rc = slab_owner_particles(slabs, n, direct);
      if (rc) return rc;
    }
  }
  for (int s = 0; s < n; s++) {
    lbrb_t* h = slabs[s];
    if (!h->join_pending) continue;
    // the record copies are part of the steps for each slab's stream
    CK(h, cudaSetDevice(h->dev));
    CK(h, cudaEventRecord(h->join_ev, h->copy_stream));
    CK(h, cudaStreamWaitEvent(h->stream, h->join_ev, 0));
    h->join_pending = false;
  }
  return LBRB_OK;
}

int lbrb_set_graph(lbrb_t* h, int mode) {
  if (!h || mode < -1 || mode > 1) return fail(h, LBRB_ERR_ARG, "set_graph: mode must be -1, 0 or 1");
  h->graph_mode = mode;
  return LBRB_OK;
}

int lbrb_set_pairs(lbrb_t* h, int mode) {
  if (!h || mode < -1 || mode > 1) return fail(h, LBRB_ERR_ARG, "set_pairs: mode must be -1, 0 or 1");
  h->pair_mode = mode;
  return LBRB_OK;
}

int lbrb_pair_shapes(void) { return NUM_PAIR_SHAPES; }

int lbrb_set_pair_shape(lbrb_t* h, int shape) {
  if (!h || shape < -1 || shape >= NUM_PAIR_SHAPES)
    return fail(h, LBRB_ERR_ARG, "set_pair_shape: shape must be -1 (tune) or a shape index");
  h->pair_shape = shape;
  h->pair_ms = 0.f;
  return LBRB_OK;
}

int lbrb_get_pair_shape(const lbrb_t* h, int* shape, int* tile_x, int* tile_y, float* ms) {
  if (!h) return LBRB_ERR_ARG;
  // (lb_kernels.cu: PAIR_SHAPES, then MARCH_SHAPES: a strip of 32 columns
  // walked in groups of tile_y rows)
  static const int TXS[] = {32, 32, 32, 64, 32, 30, 32, 32, 64, 32, 32, 32, 32, 32, 32},
                   TYS[] = {8, 4, 16, 4, 8, 8, 8, 6, 8, 8, 8, 8, 6, 4, 6};
  static_assert(sizeof(TXS) / sizeof(int) == NUM_PAIR_SHAPES, "pair shape table");
  const int sh = h->pair_shape;
  if (shape) *shape = sh;
  if (tile_x) *tile_x = sh < 0 ? 0 : TXS[sh];
  if (tile_y) *tile_y = sh < 0 ? 0 : TYS[sh];
  if (ms) *ms = h->pair_ms;
  return LBRB_OK;
}

int lbrb_set_stream(lbrb_t* h, void* cuda_stream) {
  if (!h) return LBRB_ERR_ARG;
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaStreamSynchronize(h->stream));
  h->stream = cuda_stream ? (cudaStream_t)cuda_stream : h->own_stream;
  return LBRB_OK;
}

int lbrb_set_timing(lbrb_t* h, int enable) {
  if (!h) return LBRB_ERR_ARG;
  h->timing = enable != 0;
  return LBRB_OK;
}

int lbrb_get_timing(lbrb_t* h, double* ms, int* launches, int n) {
  if (!h || n < 0 || n > 4) return fail(h, LBRB_ERR_ARG, "get_timing: n must be 0..4");
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaStreamSynchronize(h->stream));
  CK(h, cudaStreamSynchronize(h->pstream));
  CK(h, cudaStreamSynchronize(h->copy_stream));
  double acc[4] = {0, 0, 0, 0};
  int cnt[4] = {0, 0, 0, 0};
  for (const auto& m : h->marks) {
    float t = 0.f;
    CK(h, cudaEventElapsedTime(&t, m.a, m.b));
    acc[m.cls] += t;
    cnt[m.cls]++;
  }
  for (int c = 0; c < n; c++) {
    if (ms) ms[c] = acc[c];
    if (launches) launches[c] = cnt[c];
  }
  h->marks.clear();
  h->ev_used = 0;
  return LBRB_OK;
}

int lbrb_sync(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaStreamSynchronize(h->stream));
  CK(h, cudaStreamSynchronize(h->pstream));
  CK(h, cudaStreamSynchronize(h->copy_stream));
  CK(h, cudaMemcpy(h->h_flags, h->dflags, sizeof(unsigned), cudaMemcpyDeviceToHost));
  const unsigned f = *h->h_flags;
  if (f & DFLAG_NONFINITE) return fail(h, LBRB_ERR_NONFINITE, "device: non-finite value seen");
  if (f & DFLAG_RANGE) return fail(h, LBRB_ERR_RANGE, "device: particle or observation outside the domain");
  if (f & DFLAG_BOXCAP) return fail(h, LBRB_ERR_STATE, "device: box nudging list inconsistent");
  if (f & DFLAG_XCAP)
    return fail(h, LBRB_ERR_OVERFLOW, "device: a slab's particles or a hand-off list over its capacity");
  if (f & DFLAG_XMSG)
    return fail(h, LBRB_ERR_STATE, "device: a slab message from the wrong step or neighbour (exchange missing?)");
  return LBRB_OK;
}

int lbrb_check_finite(lbrb_t* h) {
  if (!h) return LBRB_ERR_ARG;
  CK(h, cudaSetDevice(h->dev));
  CK(h, launch_finite(h->pops[h->cur], 2 * NPOP * h->plane, fp32(h), h->dflags, h->stream));
  return lbrb_sync(h);
}

// ------------------------------------------------------------ diagnostics
static int stats(lbrb_t* h, double out[3]) {
  if (!h->moments_valid) return fail(h, LBRB_ERR_STATE, "diagnostics: no moments yet");
  CK(h, cudaSetDevice(h->dev));
  double* part = h->red;
  double* res = h->red + (size_t)red_blocks() * 6;
  CK(h, launch_stats(h->rho[h->cur], h->uv[h->uvcur][0], h->uv[h->uvcur][1], h->T[h->cur], fp32(h), h->p.nx,
                     h->p.ny, h->pitch, part, res, h->stream));
  CK(h, cudaMemcpyAsync(out, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return LBRB_OK;
}

int lbrb_energy(lbrb_t* h, double* ke_mean, double* t_mean) {
  if (!h) return LBRB_ERR_ARG;
  double s[3];
  int rc = stats(h, s);
  if (rc) return rc;
  const double nn = (double)h->p.nx * (double)h->p.ny;
  if (ke_mean) *ke_mean = s[0] / nn;
  if (t_mean) *t_mean = s[1] / nn;
  return LBRB_OK;
}

int lbrb_nusselt(lbrb_t* h, double* nu) {
  if (!h || !nu) return LBRB_ERR_ARG;
  double s[3];
  int rc = stats(h, s);
  if (rc) return rc;
  const double nn = (double)h->p.nx * (double)h->p.ny;
  const double kappa = (h->p.relaxg - 0.5) / 3.0;
  // (a y-slab: its mean of v T at the whole domain's height; the domain's Nu
  // is the slabs' values weighted by their heights)
  const double H = h->slab ? (double)h->slab_ny_total : (double)h->p.ny;
  *nu = 1.0 + (s[2] / nn) * H / (kappa * (h->p.Tdown - h->p.Tup));
  return LBRB_OK;
}

int lbrb_profile(lbrb_t* h, double* out) {
  if (!h || !out) return LBRB_ERR_ARG;
  if (!h->moments_valid) return fail(h, LBRB_ERR_STATE, "profile: no moments yet");
  CK(h, cudaSetDevice(h->dev));
  double* dout = h->red + (size_t)red_blocks() * 6 + 8;
  // box nudging: the row above the top row is the reference's periodic halo
  // row, row 0's sum of g without the 1/2 nud_term (kept by the fused step)
  const double* Ttop = (h->p.nudge == LBRB_NUDGE_REFBOX && h->istep > 0) ? h->tsum0 : nullptr;
  CK(h, launch_profile(h->rho[h->cur], h->uv[h->uvcur][0], h->uv[h->uvcur][1], h->T[h->cur], fp32(h), h->p.nx,
                       h->p.ny, h->pitch, Ttop, dout, h->stream));
  CK(h, cudaMemcpyAsync(out, dout, (size_t)h->p.ny * 9 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  const double kappa = (h->p.relaxg - 0.5) / 3.0;
  const double dTw = h->p.Tdown - h->p.Tup;
  for (int j = 0; j < h->p.ny; j++)
    out[(size_t)j * 9 + 8] = (out[(size_t)j * 9 + 6] - kappa * out[(size_t)j * 9 + 7]) / (kappa * dTw / (double)h->p.ny);
  return LBRB_OK;
}

}  // extern "C"
