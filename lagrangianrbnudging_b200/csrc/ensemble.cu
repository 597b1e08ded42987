// ensemble.cu -- C-ABI of the ensemble: many independent runs (handles made by
// lbrb_create) advanced together, one launch per phase of the step for all
// of them, replayed from a CUDA graph.  No counterpart in the reference.
//
// A member's state stays in its handle.  Every call of lbrb_ensemble_step
// rebuilds the members' step views for the six phases of the buffer cycle
// (populations and F alternate over 2 buffers, u and v over 3 slots, so the
// buffer assignment repeats every 6 steps) and one view set for the last
// step (which also writes the moments, as lbrb_step does), uploads them,
// and queues the steps: 6-step graph replays, then single steps.  The views
// follow lbrb_step's own buffer bookkeeping step by step, so a member
// advanced by the ensemble ends bit-identical to the same handle advanced by
// lbrb_step.
#include <algorithm>
#include <cstring>
#include <vector>

#include "capi_internal.cuh"
#include "ensemble.cuh"

using namespace lbrb;

struct lbrb_ensemble_s {
  std::vector<lbrb_t*> m;
  std::string err;
  int dev = 0, nsm = 148;
  bool f32 = true;
  int twall = LBRB_TWALL_DIRICHLET;
  bool off32 = true;            // 32-bit element offsets for every member
  size_t vsize = 0, asize = 0;  // bytes of one LBView / EnsAux
  cudaStream_t stream = nullptr, own_stream = nullptr;
  cudaEvent_t ev = nullptr;
  void* d_views = nullptr;      // [9][n]: phases 0..5, the last step; with pairs: tail steps 7, 8
  void* d_aux = nullptr;        // [9][n]
  int4* d_items = nullptr;
  int nitems = 0, items_variant = -1;
  int2* d_pch = nullptr;
  int npch = 0;
  int2* d_och = nullptr;
  int noch = 0;
  int* d_ctr = nullptr;
  int variant = -1;             // -1: tune at the next step
  float variant_ms = 0.f;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int graph_variant = -1;
  // two steps per launch: pair_mode -1 (default) / 1 on, 0 off; pair views
  // [6 phases][2 steps][n] and their EnsAux, items of the marching kernel
  // (member, first column, first row, rows) and of each tile variant
  // (member, first column, first row, 0), the variant (-1: tune), a graph
  // of 6 pairs (12 steps, the period of the buffer cycle)
  int pair_mode = -1;
  int pair_variant = -1;
  float pair_ms = 0.f;
  void* d_pviews = nullptr;
  void* d_paux = nullptr;
  int4* d_pitems = nullptr;
  int npitems = 0;
  int4* d_titems[ENS_PAIR_VARIANTS - ENS_MARCH_VARIANTS] = {};
  int ntitems[ENS_PAIR_VARIANTS - ENS_MARCH_VARIANTS] = {};
  cudaGraph_t pgraph = nullptr;
  cudaGraphExec_t pgexec = nullptr;
  int pgraph_variant = -1;
  bool timing = false;
  std::vector<cudaEvent_t> evpool;
  size_t evused = 0;
  struct Mark { int cls; cudaEvent_t a, b; };
  std::vector<Mark> marks;
};

static int efail(lbrb_ensemble_t* e, int code, const std::string& msg, cudaError_t ce = cudaSuccess) {
  if (e) {
    e->err = msg;
    if (ce != cudaSuccess) e->err += std::string(": ") + cudaGetErrorString(ce);
  }
  return code;
}

#define EK(e, call)                                                     \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) return efail((e), LBRB_ERR_CUDA, #call, e_); \
  } while (0)

namespace {

// buffer bookkeeping of one member, as lbrb_step advances it
struct MState {
  int cur, uvcur, uvprev;
};

struct StepBufs {
  int src, dst, uvn, ub, write_uv, write_rt;
};

StepBufs step_bufs(const lbrb_t* h, MState& s, bool last) {
  StepBufs b;
  b.write_uv = (h->np > 0) || last;
  b.write_rt = last ? 3 : (h->p.nudge == LBRB_NUDGE_BILINEAR ? 1 : 0);  // (as lbrb_step)
  b.src = s.cur;
  b.dst = s.cur ^ 1;
  b.uvn = b.write_uv ? 3 - s.uvcur - s.uvprev : s.uvcur;
  b.ub = b.write_uv ? s.uvcur : s.uvprev;
  s.cur = b.dst;
  if (b.write_uv) {
    s.uvprev = s.uvcur;
    s.uvcur = b.uvn;
  }
  return b;
}

// two steps of one launch, as lbrb_step's pairs advance the buffers
struct PairBufs {
  int src, dst, A, B, uvcur0, wuv;
};

PairBufs pair_bufs(const lbrb_t* h, MState& s) {
  const bool parts = h->np > 0;
  PairBufs b;
  b.src = s.cur;
  b.dst = s.cur ^ 1;
  b.A = parts ? 3 - s.uvcur - s.uvprev : s.uvcur;  // u^n
  b.B = parts ? s.uvprev : s.uvcur;                // u^{n+1}
  b.uvcur0 = s.uvcur;                              // u^{n-1}
  b.wuv = parts ? 1 : 0;
  s.cur = b.dst;
  if (parts) {
    s.uvprev = b.A;
    s.uvcur = b.B;
  }
  return b;
}

// a member's EnsAux for one step: particles read u (slot un), u^{n-1}
// (slot ub) and T (buffer tb); nudging reads T and applies to g of buffer tb
template <typename Real>
EnsAux<Real> make_aux(lbrb_t* h, int un, int ub, int tb) {
  EnsAux<Real> a{};
  a.P = PView<Real>{(const Real*)h->uv[un][0], (const Real*)h->uv[un][1],
                    (const Real*)h->uv[ub][0], (const Real*)h->uv[ub][1],
                    (const Real*)h->T[tb], h->p.nx, h->p.ny, h->pitch, h->px, h->ptype, h->np,
                    h->p.beta, 0, 0, nullptr, h->dflags};
  a.T = (const Real*)h->T[tb];
  a.g = (Real*)pop_base(h, tb, 1);
  a.plane = h->plane;
  a.nx = h->p.nx;
  a.ny = h->p.ny;
  a.pitch = h->pitch;
  if (h->p.nudge == LBRB_NUDGE_BILINEAR) {
    a.obs = h->obs;
    a.nobs = h->nobs;
    a.obs_first = h->obs_first;
    a.obs_nsteps = h->obs_nsteps;
    a.obs_cycle = h->p.obs_cycle;
    a.alpha = h->p.alpha;
    a.acc = reinterpret_cast<unsigned long long*>(h->acc);
    a.acc2 = reinterpret_cast<unsigned long long*>(h->acc2);
    a.nmask = h->nmask;
  }
  a.istep0 = h->istep;
  a.dflags = h->dflags;
  return a;
}

// the two views and EnsAux of a pair (lbrb_step's two(): step n's T into
// the source buffer's T, its innovations added inside the launch)
template <typename Real>
void fill_pair(lbrb_t* h, const PairBufs& b, LBView<Real>* V1, LBView<Real>* V2, EnsAux<Real>* A1, EnsAux<Real>* A2) {
  const bool nud = h->p.nudge == LBRB_NUDGE_BILINEAR;
  *V1 = make_view<Real>(h, b.src, b.dst, b.A, b.wuv, 0);
  V1->T = (Real*)h->T[b.src];
  V1->rho = (Real*)h->rho[b.src];
  if (nud) {
    V1->nmask = h->nmask;
    V1->nacc = reinterpret_cast<const unsigned long long*>(h->acc2);
  }
  *V2 = make_view<Real>(h, b.dst, b.dst, b.B, b.wuv, nud ? 1 : 0);
  *A1 = make_aux<Real>(h, b.A, b.uvcur0, b.src);
  *A2 = make_aux<Real>(h, b.B, b.A, b.dst);
}

template <typename Real>
void fill_views(lbrb_t* h, const StepBufs& b, LBView<Real>* V, EnsAux<Real>* A) {
  *V = make_view<Real>(h, b.src, b.dst, b.uvn, b.write_uv, b.write_rt);
  EnsAux<Real> a{};
  a.P = PView<Real>{(const Real*)h->uv[b.uvn][0], (const Real*)h->uv[b.uvn][1],
                    (const Real*)h->uv[b.ub][0], (const Real*)h->uv[b.ub][1],
                    (const Real*)h->T[b.dst], h->p.nx, h->p.ny, h->pitch, h->px, h->ptype, h->np,
                    h->p.beta, 0, 0, nullptr, h->dflags};
  a.T = (const Real*)h->T[b.dst];
  a.g = (Real*)pop_base(h, b.dst, 1);
  a.plane = h->plane;
  a.nx = h->p.nx;
  a.ny = h->p.ny;
  a.pitch = h->pitch;
  if (h->p.nudge == LBRB_NUDGE_BILINEAR) {
    a.obs = h->obs;
    a.nobs = h->nobs;
    a.obs_first = h->obs_first;
    a.obs_nsteps = h->obs_nsteps;
    a.obs_cycle = h->p.obs_cycle;
    a.alpha = h->p.alpha;
    a.acc = reinterpret_cast<unsigned long long*>(h->acc);
  }
  a.istep0 = h->istep;
  a.dflags = h->dflags;
  *A = a;
}

// Views of one call of n steps.  Single steps: phases 0..5 from the current
// state and the last step (slot 6).  With npairs > 0 pairs first: the pair
// views of 6 phases from the current state (pv, pa: [6][2][n]), then the
// tail's single steps from the state after the pairs (slot 7: an extra step
// when two remain, slot 8: the last step); slots 0..5 stay those of the
// current state (the single-step tuner's trials read slot 0).
template <typename Real>
void build_views(lbrb_ensemble_t* e, int n, int npairs, std::vector<char>& vbuf, std::vector<char>& abuf,
                 std::vector<char>& pvbuf, std::vector<char>& pabuf) {
  const size_t nm = e->m.size();
  vbuf.assign(9 * nm * sizeof(LBView<Real>), 0);
  abuf.assign(9 * nm * sizeof(EnsAux<Real>), 0);
  pvbuf.assign(12 * nm * sizeof(LBView<Real>), 0);
  pabuf.assign(12 * nm * sizeof(EnsAux<Real>), 0);
  LBView<Real>* V = reinterpret_cast<LBView<Real>*>(vbuf.data());
  EnsAux<Real>* A = reinterpret_cast<EnsAux<Real>*>(abuf.data());
  LBView<Real>* PV = reinterpret_cast<LBView<Real>*>(pvbuf.data());
  EnsAux<Real>* PA = reinterpret_cast<EnsAux<Real>*>(pabuf.data());
  for (size_t i = 0; i < nm; i++) {
    lbrb_t* h = e->m[i];
    MState s{h->cur, h->uvcur, h->uvprev};
    for (int ph = 0; ph < 6; ph++) {
      StepBufs b = step_bufs(h, s, false);
      fill_views<Real>(h, b, V + ph * nm + i, A + ph * nm + i);
    }
    MState l{h->cur, h->uvcur, h->uvprev};
    if (npairs == 0) {
      for (int t = 0; t < (n - 1) % 6; t++) step_bufs(h, l, false);
      StepBufs b = step_bufs(h, l, true);
      fill_views<Real>(h, b, V + 6 * nm + i, A + 6 * nm + i);
      continue;
    }
    MState q{h->cur, h->uvcur, h->uvprev};
    for (int ph = 0; ph < 6; ph++) {
      PairBufs b = pair_bufs(h, q);
      fill_pair<Real>(h, b, PV + (2 * ph) * nm + i, PV + (2 * ph + 1) * nm + i, PA + (2 * ph) * nm + i,
                      PA + (2 * ph + 1) * nm + i);
    }
    for (int t = 0; t < npairs % 6; t++) pair_bufs(h, l);
    if (n - 2 * npairs == 2) {
      StepBufs b = step_bufs(h, l, false);
      fill_views<Real>(h, b, V + 7 * nm + i, A + 7 * nm + i);
    }
    StepBufs b = step_bufs(h, l, true);
    fill_views<Real>(h, b, V + 8 * nm + i, A + 8 * nm + i);
  }
}

// the handle state lbrb_step(n) would leave (npairs pairs, then singles)
void advance_members(lbrb_ensemble_t* e, int n, int npairs) {
  for (lbrb_t* h : e->m) {
    MState s{h->cur, h->uvcur, h->uvprev};
    for (int t = 0; t < npairs % 6; t++) pair_bufs(h, s);
    const int singles = n - 2 * npairs;
    const int lead = npairs > 0 ? singles - 1 : (n - 1) % 6;
    for (int t = 0; t < lead; t++) step_bufs(h, s, false);
    step_bufs(h, s, true);
    h->cur = s.cur;
    h->uvcur = s.uvcur;
    h->uvprev = s.uvprev;
    h->istep += n;
    h->prev_valid = true;
    h->prev_pair = false;
  }
}

std::vector<int4> make_items(const lbrb_ensemble_t* e, int bs, int rows) {
  std::vector<int4> it;
  for (size_t i = 0; i < e->m.size(); i++) {
    const lbrb_t* h = e->m[i];
    for (int j = 0; j < h->p.ny; j += rows)
      for (int x = 0; x < h->p.nx; x += bs) it.push_back(make_int4((int)i, j, x, 0));
  }
  return it;
}

cudaEvent_t pool_ev(lbrb_ensemble_t* e) {
  if (e->evused == e->evpool.size()) {
    cudaEvent_t ev = nullptr;
    if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
    e->evpool.push_back(ev);
  }
  return e->evpool[e->evused++];
}

int mark_begin(lbrb_ensemble_t* e, int cls) {
  if (!e->timing) return -1;
  cudaEvent_t a = pool_ev(e), b = pool_ev(e);
  if (!a || !b) return -1;
  cudaEventRecord(a, e->stream);
  e->marks.push_back({cls, a, b});
  return (int)e->marks.size() - 1;
}
void mark_end(lbrb_ensemble_t* e, int k) {
  if (k >= 0) cudaEventRecord(e->marks[k].b, e->stream);
}

const char* view_at(const lbrb_ensemble_t* e, int ph) {
  return (const char*)e->d_views + (size_t)ph * e->m.size() * e->vsize;
}
const char* aux_at(const lbrb_ensemble_t* e, int ph) {
  return (const char*)e->d_aux + (size_t)ph * e->m.size() * e->asize;
}

// one step of every member, phase ph (0..5) or the last step (6)
cudaError_t launch_step(lbrb_ensemble_t* e, int ph) {
  int k = mark_begin(e, 0);
  cudaError_t c = launch_ens_lb(e->f32, e->off32, e->twall, e->variant, view_at(e, ph), e->d_items, e->nitems,
                                e->d_ctr, e->nsm, e->stream);
  mark_end(e, k);
  if (c != cudaSuccess) return c;
  k = mark_begin(e, 1);
  c = launch_ens_aux(e->f32, aux_at(e, ph), e->d_pch, e->npch, e->d_och, e->noch, e->d_ctr, e->stream);
  mark_end(e, k);
  if (c != cudaSuccess) return c;
  if (e->noch > 0) {
    k = mark_begin(e, 2);
    c = launch_ens_apply(e->f32, aux_at(e, ph), e->d_och, e->noch, e->d_ctr, e->stream);
    mark_end(e, k);
  }
  return c;
}

const char* pview_at(const lbrb_ensemble_t* e, int ph, int step) {
  return (const char*)e->d_pviews + (size_t)(2 * ph + step) * e->m.size() * e->vsize;
}
const char* paux_at(const lbrb_ensemble_t* e, int ph, int step) {
  return (const char*)e->d_paux + (size_t)(2 * ph + step) * e->m.size() * e->asize;
}

// the two-step LB launch of variant v over every member, pair phase ph
static cudaError_t launch_pair_lb(lbrb_ensemble_t* e, int v, int ph) {
  const bool tile = v >= ENS_MARCH_VARIANTS;
  return launch_ens_march(e->f32, e->off32, v, pview_at(e, ph, 0), pview_at(e, ph, 1),
                          tile ? e->d_titems[v - ENS_MARCH_VARIANTS] : e->d_pitems,
                          tile ? e->ntitems[v - ENS_MARCH_VARIANTS] : e->npitems, e->d_ctr, e->stream);
}

// two steps of every member, pair phase ph (0..5)
cudaError_t launch_pair(lbrb_ensemble_t* e, int ph) {
  cudaError_t c = cudaSuccess;
  int k;
  if (e->noch > 0) {
    k = mark_begin(e, 2);
    c = launch_ens_pre(e->f32, pview_at(e, ph, 0), paux_at(e, ph, 0), e->d_och, e->noch, e->d_ctr, e->stream);
    mark_end(e, k);
    if (c != cudaSuccess) return c;
  }
  k = mark_begin(e, 0);
  c = launch_pair_lb(e, e->pair_variant, ph);
  mark_end(e, k);
  if (c != cudaSuccess) return c;
  k = mark_begin(e, 1);
  c = launch_ens_aux2(e->f32, paux_at(e, ph, 0), paux_at(e, ph, 1), e->d_pch, e->npch, e->d_och, e->noch, e->d_ctr,
                      e->stream);
  mark_end(e, k);
  if (c != cudaSuccess) return c;
  if (e->noch > 0) {
    k = mark_begin(e, 2);
    c = launch_ens_apply2(e->f32, paux_at(e, ph, 0), paux_at(e, ph, 1), e->d_och, e->noch, e->d_ctr, e->stream);
    mark_end(e, k);
  }
  return c;
}

// work items of the marching kernel: every member's strips of 32 columns x
// chunks of PAIR_CHUNK rows (whole groups of 6 or 8 rows with the two ring
// rows); of a tile variant: every member's tiles, row by row
constexpr int PAIR_CHUNK = 62;
static int upload_items(lbrb_ensemble_t* e, const std::vector<int4>& it, int4** d, int* n) {
  EK(e, cudaMalloc(d, it.size() * sizeof(int4)));
  EK(e, cudaMemcpyAsync(*d, it.data(), it.size() * sizeof(int4), cudaMemcpyHostToDevice, e->stream));
  EK(e, cudaStreamSynchronize(e->stream));
  *n = (int)it.size();
  return LBRB_OK;
}

int set_pair_items(lbrb_ensemble_t* e) {
  if (e->d_pitems) return LBRB_OK;
  std::vector<int4> it;
  for (size_t i = 0; i < e->m.size(); i++) {
    const lbrb_t* h = e->m[i];
    for (int y = 0; y < h->p.ny; y += PAIR_CHUNK)
      for (int x = 0; x < h->p.nx; x += 32) it.push_back(make_int4((int)i, x, y, std::min(PAIR_CHUNK, h->p.ny - y)));
  }
  int rc = upload_items(e, it, &e->d_pitems, &e->npitems);
  for (int v = ENS_MARCH_VARIANTS; v < ENS_PAIR_VARIANTS && rc == LBRB_OK; v++) {
    const int tx = ens_pair_tile_cols(v), ty = ens_pair_rows(v);
    it.clear();
    for (size_t i = 0; i < e->m.size(); i++) {
      const lbrb_t* h = e->m[i];
      for (int y = 0; y < h->p.ny; y += ty)
        for (int x = 0; x < h->p.nx; x += tx) it.push_back(make_int4((int)i, x, y, 0));
    }
    rc = upload_items(e, it, &e->d_titems[v - ENS_MARCH_VARIANTS], &e->ntitems[v - ENS_MARCH_VARIANTS]);
  }
  return rc;
}

// Pair autotuner: each variant's marching launch on pair phase 0 (trials
// write only buffers the real pair overwrites), 3 timed launches after a
// warm-up; the fastest is kept
int tune_pairs(lbrb_ensemble_t* e) {
  int rc = set_pair_items(e);
  if (rc) return rc;
  cudaEvent_t a, b;
  EK(e, cudaEventCreate(&a));
  EK(e, cudaEventCreate(&b));
  int best = 0;
  float bt = 1e30f;
  for (int v = 0; v < ENS_PAIR_VARIANTS; v++) {
    float tot = 0.f;
    bool ok = true;
    for (int r = 0; r < 4 && ok; r++) {
      EK(e, cudaEventRecord(a, e->stream));
      cudaError_t c = launch_pair_lb(e, v, 0);
      if (c != cudaSuccess) {
        cudaGetLastError();
        ok = false;
        break;
      }
      EK(e, cudaEventRecord(b, e->stream));
      EK(e, cudaEventSynchronize(b));
      float ms = 0.f;
      EK(e, cudaEventElapsedTime(&ms, a, b));
      if (r > 0) tot += ms;
    }
    if (ok && tot / 3 < bt) {
      bt = tot / 3;
      best = v;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  EK(e, cudaMemsetAsync(e->d_ctr, 0, 2 * sizeof(int), e->stream));
  e->pair_variant = best;
  e->pair_ms = bt;
  return LBRB_OK;
}

int ensure_pair_graph(lbrb_ensemble_t* e) {
  if (e->pgexec && e->pgraph_variant == e->pair_variant) return LBRB_OK;
  if (e->pgexec) cudaGraphExecDestroy(e->pgexec);
  if (e->pgraph) cudaGraphDestroy(e->pgraph);
  e->pgexec = nullptr;
  e->pgraph = nullptr;
  EK(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t c = cudaSuccess;
  for (int ph = 0; ph < 6 && c == cudaSuccess; ph++) c = launch_pair(e, ph);
  cudaGraph_t g = nullptr;
  cudaError_t c2 = cudaStreamEndCapture(e->stream, &g);
  if (c != cudaSuccess) return efail(e, LBRB_ERR_CUDA, "ensemble pair graph capture", c);
  if (c2 != cudaSuccess) return efail(e, LBRB_ERR_CUDA, "ensemble pair graph capture", c2);
  e->pgraph = g;
  EK(e, cudaGraphInstantiate(&e->pgexec, g, 0));
  e->pgraph_variant = e->pair_variant;
  return LBRB_OK;
}

int set_items(lbrb_ensemble_t* e, int variant) {
  if (e->items_variant >= 0 && ENS_TABLE[e->items_variant].bs == ENS_TABLE[variant].bs &&
      ENS_TABLE[e->items_variant].rows == ENS_TABLE[variant].rows) {
    e->items_variant = variant;
    EK(e, launch_ens_lb(e->f32, e->off32, e->twall, variant, e->d_views, e->d_items, 0, e->d_ctr, e->nsm, e->stream));
    return LBRB_OK;
  }
  std::vector<int4> it = make_items(e, ENS_TABLE[variant].bs, ENS_TABLE[variant].rows);
  if (e->d_items) cudaFree(e->d_items);
  e->d_items = nullptr;
  EK(e, cudaMalloc(&e->d_items, it.size() * sizeof(int4)));
  EK(e, cudaMemcpyAsync(e->d_items, it.data(), it.size() * sizeof(int4), cudaMemcpyHostToDevice, e->stream));
  EK(e, cudaStreamSynchronize(e->stream));
  e->nitems = (int)it.size();
  e->items_variant = variant;
  // the variant's occupancy query runs here, never inside a graph capture
  EK(e, launch_ens_lb(e->f32, e->off32, e->twall, variant, e->d_views, e->d_items, 0, e->d_ctr, e->nsm, e->stream));
  return LBRB_OK;
}

// Autotuner: time each variant's phase-A launch on the members' current state
// (a trial reads the current buffers and writes only buffers the real step
// overwrites), 3 timed launches after a warm-up, and keep the fastest.
int tune(lbrb_ensemble_t* e) {
  cudaEvent_t a, b;
  EK(e, cudaEventCreate(&a));
  EK(e, cudaEventCreate(&b));
  int best = 0;
  float bt = 1e30f;
  for (int v = 0; v < ENS_NVARIANTS; v++) {
    int rc = set_items(e, v);
    if (rc) return rc;
    float tot = 0.f;
    bool ok = true;
    for (int r = 0; r < 4 && ok; r++) {
      EK(e, cudaMemsetAsync(e->d_ctr, 0, 2 * sizeof(int), e->stream));
      EK(e, cudaEventRecord(a, e->stream));
      cudaError_t c = launch_ens_lb(e->f32, e->off32, e->twall, v, view_at(e, 0), e->d_items, e->nitems, e->d_ctr,
                                    e->nsm, e->stream);
      if (c != cudaSuccess) {
        cudaGetLastError();
        ok = false;
        break;
      }
      EK(e, cudaEventRecord(b, e->stream));
      EK(e, cudaEventSynchronize(b));
      float ms = 0.f;
      EK(e, cudaEventElapsedTime(&ms, a, b));
      if (r > 0) tot += ms;
    }
    if (ok && tot / 3 < bt) {
      bt = tot / 3;
      best = v;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  EK(e, cudaMemsetAsync(e->d_ctr, 0, 2 * sizeof(int), e->stream));
  e->variant = best;
  e->variant_ms = bt;
  return set_items(e, best);
}

int ensure_graph(lbrb_ensemble_t* e) {
  if (e->gexec && e->graph_variant == e->variant) return LBRB_OK;
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->gexec = nullptr;
  e->graph = nullptr;
  EK(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t c = cudaSuccess;
  for (int ph = 0; ph < 6 && c == cudaSuccess; ph++) c = launch_step(e, ph);
  cudaGraph_t g = nullptr;
  cudaError_t c2 = cudaStreamEndCapture(e->stream, &g);
  if (c != cudaSuccess) return efail(e, LBRB_ERR_CUDA, "ensemble graph capture", c);
  if (c2 != cudaSuccess) return efail(e, LBRB_ERR_CUDA, "ensemble graph capture", c2);
  e->graph = g;
  EK(e, cudaGraphInstantiate(&e->gexec, g, 0));
  e->graph_variant = e->variant;
  return LBRB_OK;
}

}  // namespace

extern "C" {

int lbrb_ensemble_nvariants(void) { return ENS_NVARIANTS; }

int lbrb_ensemble_create(lbrb_t* const* members, int n, lbrb_ensemble_t** out) {
  if (!out) return LBRB_ERR_ARG;
  *out = nullptr;
  if (!members || n < 1) return LBRB_ERR_ARG;
  for (int i = 0; i < n; i++) {
    const lbrb_t* h = members[i];
    if (!h) return LBRB_ERR_ARG;
    for (int k = 0; k < i; k++)
      if (members[k] == h) return LBRB_ERR_ARG;  // a handle appears once
    const lbrb_t* h0 = members[0];
    if (h->dev != h0->dev || h->p.precision != h0->p.precision || h->p.twall != h0->p.twall)
      return LBRB_ERR_ARG;
    if (h->p.nudge == LBRB_NUDGE_REFBOX) return LBRB_ERR_UNSUPPORTED;
    if (h->np > 0 && h->p.noutconfig > 0) return LBRB_ERR_UNSUPPORTED;
    if (h->slab) return LBRB_ERR_UNSUPPORTED;  // members are whole domains
  }
  lbrb_ensemble_t* e = new lbrb_ensemble_t();
  e->m.assign(members, members + n);
  e->dev = members[0]->dev;
  e->f32 = fp32(members[0]);
  e->twall = members[0]->p.twall;
  for (int i = 0; i < n; i++) e->off32 = e->off32 && off32_ok(members[i]->plane);
  e->vsize = e->f32 ? sizeof(LBView<float>) : sizeof(LBView<double>);
  e->asize = e->f32 ? sizeof(EnsAux<float>) : sizeof(EnsAux<double>);
  auto bad = [&](cudaError_t c) {
    lbrb_ensemble_destroy(e);
    return c == cudaErrorMemoryAllocation ? LBRB_ERR_NOMEM : LBRB_ERR_CUDA;
  };
  cudaError_t c = cudaSetDevice(e->dev);
  if (c == cudaSuccess) c = cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, e->dev);
  if (c == cudaSuccess) c = cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking);
  if (c == cudaSuccess) c = cudaEventCreateWithFlags(&e->ev, cudaEventDisableTiming);
  if (c == cudaSuccess) c = cudaMalloc(&e->d_views, 9 * (size_t)n * e->vsize);
  if (c == cudaSuccess) c = cudaMalloc(&e->d_aux, 9 * (size_t)n * e->asize);
  if (c == cudaSuccess) c = cudaMalloc(&e->d_pviews, 12 * (size_t)n * e->vsize);
  if (c == cudaSuccess) c = cudaMalloc(&e->d_paux, 12 * (size_t)n * e->asize);
  if (c == cudaSuccess) c = cudaMalloc((void**)&e->d_ctr, 4 * sizeof(int));
  if (c != cudaSuccess) return bad(c);
  e->stream = e->own_stream;
  std::vector<int2> pch, och;
  for (int i = 0; i < n; i++) {
    const lbrb_t* h = members[i];
    for (int p = 0; p < h->np; p += ENS_PCHUNK) pch.push_back(make_int2(i, p));
    if (h->p.nudge == LBRB_NUDGE_BILINEAR)
      for (int o = 0; o < h->nobs; o += ENS_OCHUNK) och.push_back(make_int2(i, o));
  }
  e->npch = (int)pch.size();
  e->noch = (int)och.size();
  c = cudaMalloc((void**)&e->d_pch, std::max<size_t>(1, pch.size()) * sizeof(int2));
  if (c == cudaSuccess) c = cudaMalloc((void**)&e->d_och, std::max<size_t>(1, och.size()) * sizeof(int2));
  if (c == cudaSuccess && !pch.empty())
    c = cudaMemcpy(e->d_pch, pch.data(), pch.size() * sizeof(int2), cudaMemcpyHostToDevice);
  if (c == cudaSuccess && !och.empty())
    c = cudaMemcpy(e->d_och, och.data(), och.size() * sizeof(int2), cudaMemcpyHostToDevice);
  if (c == cudaSuccess) c = cudaMemset(e->d_ctr, 0, 4 * sizeof(int));
  if (c != cudaSuccess) return bad(c);
  *out = e;
  return LBRB_OK;
}

int lbrb_ensemble_destroy(lbrb_ensemble_t* e) {
  if (!e) return LBRB_ERR_ARG;
  cudaSetDevice(e->dev);
  if (e->own_stream) cudaStreamSynchronize(e->own_stream);
  if (e->stream && e->stream != e->own_stream) cudaStreamSynchronize(e->stream);
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->pgexec) cudaGraphExecDestroy(e->pgexec);
  if (e->pgraph) cudaGraphDestroy(e->pgraph);
  for (void* p : {(void*)e->d_views, (void*)e->d_aux, (void*)e->d_items, (void*)e->d_pch, (void*)e->d_och,
                  (void*)e->d_ctr, (void*)e->d_pviews, (void*)e->d_paux, (void*)e->d_pitems})
    if (p) cudaFree(p);
  for (int4* p : e->d_titems)
    if (p) cudaFree(p);
  for (cudaEvent_t ev : e->evpool) cudaEventDestroy(ev);
  if (e->ev) cudaEventDestroy(e->ev);
  if (e->own_stream) cudaStreamDestroy(e->own_stream);
  delete e;
  return LBRB_OK;
}

const char* lbrb_ensemble_last_error(const lbrb_ensemble_t* e) { return e ? e->err.c_str() : "null ensemble"; }

int lbrb_ensemble_set_stream(lbrb_ensemble_t* e, void* cuda_stream) {
  if (!e) return LBRB_ERR_ARG;
  EK(e, cudaSetDevice(e->dev));
  EK(e, cudaStreamSynchronize(e->stream));
  e->stream = cuda_stream ? (cudaStream_t)cuda_stream : e->own_stream;
  return LBRB_OK;
}

int lbrb_ensemble_set_schedule(lbrb_ensemble_t* e, int variant) {
  if (!e || variant < -1 || variant >= ENS_NVARIANTS)
    return efail(e, LBRB_ERR_ARG, "ensemble_set_schedule: variant out of range");
  EK(e, cudaSetDevice(e->dev));
  e->variant = variant;
  e->variant_ms = 0.f;
  if (variant >= 0) return set_items(e, variant);
  return LBRB_OK;
}

int lbrb_ensemble_get_schedule(const lbrb_ensemble_t* e, int* variant, int* block, int* rows,
                               int* schedule, int* fast_pull, float* ms) {
  if (!e) return LBRB_ERR_ARG;
  const int v = e->variant;
  if (variant) *variant = v;
  if (block) *block = v >= 0 ? ENS_TABLE[v].bs : 0;
  if (rows) *rows = v >= 0 ? ENS_TABLE[v].rows : 0;
  if (schedule) *schedule = v >= 0 ? ENS_TABLE[v].sched : -1;
  if (fast_pull) *fast_pull = v >= 0 ? ENS_TABLE[v].fast : -1;
  if (ms) *ms = e->variant_ms;
  return LBRB_OK;
}

int lbrb_ensemble_set_pairs(lbrb_ensemble_t* e, int mode) {
  if (!e || mode < -1 || mode > 1) return efail(e, LBRB_ERR_ARG, "ensemble_set_pairs: mode must be -1, 0 or 1");
  e->pair_mode = mode;
  return LBRB_OK;
}

int lbrb_ensemble_pair_variants(void) { return ENS_PAIR_VARIANTS; }

int lbrb_ensemble_set_pair_variant(lbrb_ensemble_t* e, int variant) {
  if (!e || variant < -1 || variant >= ENS_PAIR_VARIANTS)
    return efail(e, LBRB_ERR_ARG, "ensemble_set_pair_variant: variant out of range");
  e->pair_variant = variant;
  e->pair_ms = 0.f;
  return LBRB_OK;
}

int lbrb_ensemble_get_pair_variant(const lbrb_ensemble_t* e, int* variant, int* tile_cols) {
  if (!e) return LBRB_ERR_ARG;
  if (variant) *variant = e->pair_variant;
  if (tile_cols) *tile_cols = e->pair_variant >= 0 ? ens_pair_tile_cols(e->pair_variant) : 0;
  return LBRB_OK;
}

int lbrb_ensemble_get_pairs(const lbrb_ensemble_t* e, int* mode, int* rows, float* ms) {
  if (!e) return LBRB_ERR_ARG;
  if (mode) *mode = e->pair_mode;
  if (rows) *rows = e->pair_variant >= 0 ? ens_pair_rows(e->pair_variant) : 0;
  if (ms) *ms = e->pair_ms;
  return LBRB_OK;
}

int lbrb_ensemble_set_timing(lbrb_ensemble_t* e, int enable) {
  if (!e) return LBRB_ERR_ARG;
  e->timing = enable != 0;
  return LBRB_OK;
}

int lbrb_ensemble_get_timing(lbrb_ensemble_t* e, double* ms, int* launches, int n) {
  if (!e || n < 0 || n > 3) return efail(e, LBRB_ERR_ARG, "ensemble_get_timing: n must be 0..3");
  EK(e, cudaSetDevice(e->dev));
  EK(e, cudaStreamSynchronize(e->stream));
  double acc[3] = {0, 0, 0};
  int cnt[3] = {0, 0, 0};
  for (const auto& mk : e->marks) {
    float t = 0.f;
    EK(e, cudaEventElapsedTime(&t, mk.a, mk.b));
    acc[mk.cls] += t;
    cnt[mk.cls]++;
  }
  for (int c = 0; c < n; c++) {
    if (ms) ms[c] = acc[c];
    if (launches) launches[c] = cnt[c];
  }
  e->marks.clear();
  e->evused = 0;
  return LBRB_OK;
}

int lbrb_ensemble_step(lbrb_ensemble_t* e, int n) {
  if (!e || n < 0) return efail(e, LBRB_ERR_ARG, "ensemble_step: bad arguments");
  NvtxRange nvtx("lbrb_ensemble_step");
  if (n == 0) return LBRB_OK;
  for (size_t i = 0; i < e->m.size(); i++) {
    const lbrb_t* h = e->m[i];
    const std::string who = "ensemble_step: member " + std::to_string(i) + ": ";
    if (!h->moments_valid) return efail(e, LBRB_ERR_STATE, who + "moments not set");
    if (h->np > 0 && !h->particles_set) return efail(e, LBRB_ERR_STATE, who + "particles not set");
    if (h->p.nudge == LBRB_NUDGE_BILINEAR) {
      const int first = h->istep + 1, last = h->istep + n;
      if (!h->obs || first < h->obs_first ||
          (!h->p.obs_cycle && last >= h->obs_first + h->obs_nsteps))
        return efail(e, LBRB_ERR_STATE, who + "no bilinear observations for every step");
    }
  }
  EK(e, cudaSetDevice(e->dev));
  // after the work already queued on the members' own streams
  for (lbrb_t* h : e->m) {
    EK(e, cudaEventRecord(e->ev, h->stream));
    EK(e, cudaStreamWaitEvent(e->stream, e->ev, 0));
  }
  // two steps per launch for all but the call's last step (lbrb_step's
  // rule: a pair never takes a call's last step)
  const bool pairs = e->pair_mode != 0 && e->twall == LBRB_TWALL_DIRICHLET && n >= 3;
  const int npairs = pairs ? (n - 1) / 2 : 0;
  std::vector<char> vb, ab, pvb, pab;
  if (e->f32) build_views<float>(e, n, npairs, vb, ab, pvb, pab);
  else build_views<double>(e, n, npairs, vb, ab, pvb, pab);
  EK(e, cudaMemcpyAsync(e->d_views, vb.data(), vb.size(), cudaMemcpyHostToDevice, e->stream));
  EK(e, cudaMemcpyAsync(e->d_aux, ab.data(), ab.size(), cudaMemcpyHostToDevice, e->stream));
  if (npairs > 0) {
    EK(e, cudaMemcpyAsync(e->d_pviews, pvb.data(), pvb.size(), cudaMemcpyHostToDevice, e->stream));
    EK(e, cudaMemcpyAsync(e->d_paux, pab.data(), pab.size(), cudaMemcpyHostToDevice, e->stream));
  }
  EK(e, cudaMemsetAsync(e->d_ctr, 0, 2 * sizeof(int), e->stream));
  if (e->variant < 0) {
    int rc = tune(e);
    if (rc) return rc;
  } else if (e->items_variant != e->variant) {
    int rc = set_items(e, e->variant);
    if (rc) return rc;
  }
  if (npairs > 0) {
    if (e->pair_variant < 0) {
      int rc = tune_pairs(e);
      if (rc) return rc;
    }
    int rc = set_pair_items(e);
    if (rc) return rc;
    int q = 0;
    if (!e->timing && npairs >= 6) {
      rc = ensure_pair_graph(e);
      if (rc) return rc;
      for (; q + 6 <= npairs; q += 6) EK(e, cudaGraphLaunch(e->pgexec, e->stream));
    }
    for (; q < npairs; q++) EK(e, launch_pair(e, q % 6));
    if (n - 2 * npairs == 2) EK(e, launch_step(e, 7));
    EK(e, launch_step(e, 8));
  } else {
    int t = 0;
    if (!e->timing && n - 1 >= 6) {
      int rc = ensure_graph(e);
      if (rc) return rc;
      for (; t + 6 <= n - 1; t += 6) EK(e, cudaGraphLaunch(e->gexec, e->stream));
    }
    for (; t < n - 1; t++) EK(e, launch_step(e, t % 6));
    EK(e, launch_step(e, 6));
  }
  advance_members(e, n, npairs);
  // the members' own streams see the ensemble's steps
  EK(e, cudaEventRecord(e->ev, e->stream));
  for (lbrb_t* h : e->m) EK(e, cudaStreamWaitEvent(h->stream, e->ev, 0));
  return LBRB_OK;
}

int lbrb_ensemble_sync(lbrb_ensemble_t* e) {
  if (!e) return LBRB_ERR_ARG;
  EK(e, cudaSetDevice(e->dev));
  EK(e, cudaStreamSynchronize(e->stream));
  for (size_t i = 0; i < e->m.size(); i++) {
    const int rc = lbrb_sync(e->m[i]);
    if (rc != LBRB_OK)
      return efail(e, rc, "member " + std::to_string(i) + ": " + lbrb_last_error(e->m[i]));
  }
  return LBRB_OK;
}

}  // extern "C"
