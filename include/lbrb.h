/*
 * lbrb.h -- C-ABI of the B200 thermal lattice-Boltzmann Rayleigh-Benard step
 * loop with Lagrangian particles and temperature nudging.
 *
 * The reference drives its time loop from main() through plain C functions on
 * host arrays (Trajectories/code/temppart_dump.c:1674-1759,
 * Nudging/code/tempvel_nudge.c:2346-2411).  This library replaces that loop
 * body: one opaque handle owns the whole domain in device memory; the caller
 * hands state in and out through host buffers in the reference's own layouts.
 *
 * Conventions
 *  - Every call returns an int status: LBRB_OK (0) or a negative LBRB_ERR_*;
 *    lbrb_last_error() returns a message for the last failure on a handle.
 *  - Host buffers are borrowed for the duration of the call only.
 *  - A handle has one CUDA stream and must be used from one host thread.
 *  - Grid: nx, ny interior nodes (the reference's nx, ny); nx % 4 == 0.
 *  - Reference node (i, j), 1 <= i <= nx, 1 <= j <= ny, has position (i, j):
 *    particle coordinates use the same frame (walls half-way at y = 0.5 and
 *    y = ny + 0.5, x periodic with period nx).
 *
 * Layouts for populations (9 per node, D2Q9 order of the reference's dellar(),
 * temppart_dump.c:1363-1401) and scalar fields:
 *  - LBRB_LAYOUT_REF_AOS_HALO: the reference's own arrays, pop_type[(nx+2)*(ny+2)]
 *    with node index idx = j + (ny+2)*i (temppart_dump.c:38-40, 1598-1601);
 *    scalars REAL[(nx+2)*(ny+2)].  On output the halo is filled periodically
 *    in x and y as pbc() and communication() leave it.
 *  - LBRB_LAYOUT_SOA: interior only, pops [9][ny][nx], scalars [ny][nx], x fastest.
 */
#ifndef LBRB_H
#define LBRB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBRB_ABI_VERSION 1

#if defined(__GNUC__)
#define LBRB_API __attribute__((visibility("default")))
#else
#define LBRB_API
#endif

typedef struct lbrb_s lbrb_t;

enum lbrb_status {
  LBRB_OK = 0,
  LBRB_ERR_ARG = -1,        /* invalid argument (reference: silent UB or exit(8)) */
  LBRB_ERR_CUDA = -2,       /* CUDA runtime failure */
  LBRB_ERR_NOMEM = -3,      /* device or pinned allocation failed */
  LBRB_ERR_STATE = -4,      /* call out of order (e.g. nudging data missing) */
  LBRB_ERR_NONFINITE = -5,  /* NaN/Inf found in the state */
  LBRB_ERR_RANGE = -6,      /* particle or observation outside the domain */
  LBRB_ERR_OVERFLOW = -7,   /* record ring full: drain before stepping on */
  LBRB_ERR_IDS = -8,        /* observation ids do not match particle ids */
  LBRB_ERR_UNSUPPORTED = -9 /* combination not built */
};

enum { LBRB_PREC_FP64 = 0, LBRB_PREC_FP32_SHIFTED = 1 };
enum { LBRB_TWALL_DIRICHLET = 0, LBRB_TWALL_ADIABATIC = 1 };
enum { LBRB_NUDGE_NONE = 0, LBRB_NUDGE_REFBOX = 1, LBRB_NUDGE_BILINEAR = 2 };
enum { LBRB_LAYOUT_REF_AOS_HALO = 0, LBRB_LAYOUT_SOA = 1 };
enum { LBRB_PTYPE_TRACER = 0, LBRB_PTYPE_INERTIAL = 1 };

/* record fields, in the order of the reference's Particles%d.h5 datasets
 * (temppart_dump.c:1553-1562, then the Prtcl_Writefull block mympi2.h:549-556) */
enum {
  LBRB_REC_X = 0, LBRB_REC_Y, LBRB_REC_U, LBRB_REC_V, LBRB_REC_XO, LBRB_REC_YO,
  LBRB_REC_UO, LBRB_REC_VO, LBRB_REC_TEMP,
  LBRB_REC_DTU, LBRB_REC_DTV, LBRB_REC_DXU, LBRB_REC_DXV, LBRB_REC_DYU, LBRB_REC_DYV,
  LBRB_REC_FU, LBRB_REC_FV,
  LBRB_REC_NBASIC = 9, LBRB_REC_NFULL = 17
};

/* Run parameters.  Names follow the reference's compile-time #defines
 * (temppart_dump.c:15-31, Trajectories/code/mympi2.h:14-21,
 * tempvel_nudge.c:13-31); here they are runtime values. */
typedef struct {
  int nx, ny;             /* nx, ny */
  double relax, relaxg;   /* relax, relaxg (tau of f and g) */
  double Tup, Tdown;      /* Tup, Tdown */
  double gravity;         /* gravity (negative; F_y = -gravity*rho*T) */
  int precision;          /* LBRB_PREC_* */
  int twall;              /* LBRB_TWALL_*: Trajectories = Dirichlet, Nudging = adiabatic */
  int nudge;              /* LBRB_NUDGE_* */
  double alpha;           /* alpha: nudging coefficient */
  int ntempread;          /* ntempread: observation file interval (box mode) */
  int nobs;               /* observations per step (box: Nprtcl; bilinear: any) */
  double beta;            /* beta: Maxey-Riley coefficient */
  int nprtcl;             /* Nprtcl: Lagrangian particles advanced by the run */
  int noutconfig;         /* noutconfig: record interval (0 = no records) */
  int record_full;        /* Prtcl_Writefull: also record the 8 Maxey-Riley terms */
  int record_slots;       /* records held before lbrb_record_drain() must run */
  int device;             /* CUDA device ordinal */
  int autotune;           /* 1: time the fused kernel's launch shapes on the first step
                           * (once per process for handles on the same device with
                           * the same grid, precision, walls, nudging mode, particle
                           * use and slab position: later handles reuse the result) */
  int launch_shape;       /* with autotune 0: the shape used, an index into
                           * (threads per block, min blocks per SM) =
                           * (256,1) (256,2) (256,3) (128,4) (128,6) (512,1) (512,2)
                           * with interior rows pulled without wall logic, then
                           * (256,3) (128,4) (128,6) with the general pull on every row */
  int obs_cycle;          /* bilinear nudging: 1 = the series given to lbrb_nudge_obs repeats
                           * (step s uses row (s - first_step) mod nsteps); 0 = a step
                           * outside the series is an error (LBRB_ERR_STATE) */
} lbrb_params;

/* Fill *p with defaults (reference values where it has them). */
LBRB_API void lbrb_params_default(lbrb_params *p);

/* Create / destroy a run.  Replaces myInit + the mallocs of main()
 * (Trajectories/code/mympi2.h:41-108, temppart_dump.c:1589-1641). */
LBRB_API int lbrb_create(const lbrb_params *p, lbrb_t **out);
LBRB_API int lbrb_destroy(lbrb_t *h);
LBRB_API const char *lbrb_last_error(const lbrb_t *h);
LBRB_API int lbrb_abi_version(void);

/* ---- state in / out ------------------------------------------------------ */
/* Post-collision populations f, g.  Replaces restoref/restoreg
 * (temppart_dump.c:348-507) and dumpf/dumpg (temppart_dump.c:52-141). */
LBRB_API int lbrb_set_populations(lbrb_t *h, const double *f, const double *g, int layout);
LBRB_API int lbrb_get_populations(lbrb_t *h, double *f, double *g, int layout);
/* Post-stream (pre-collision) populations of the last step, walls applied:
 * what dumpfpre/dumpgpre write (temppart_dump.c:143-232, called at
 * :1702-1710).  Rebuilt from the state before the last step, which the
 * ping-pong layout keeps; when the call's last two steps ran in one two-step
 * launch, that state is first formed again by one step from the state before
 * the launch (bit-identical).  Any pointer may be NULL. */
LBRB_API int lbrb_get_poststream(lbrb_t *h, double *f, double *g, int layout);
/* Moments of the last step (rhopre, upre, vpre, temppre); any pointer may be
 * NULL on get.  The next step's buoyancy uses rho and T (forcingconstructWW,
 * temppart_dump.c:744-755). */
LBRB_API int lbrb_set_moments(lbrb_t *h, const double *rho, const double *u, const double *v,
                     const double *T, int layout);
LBRB_API int lbrb_get_moments(lbrb_t *h, double *rho, double *u, double *v, double *T, int layout);
/* Restart route: moments from the "pre" populations confpre/congpre
 * (inithydro scratch==0, temppart_dump.c:703-726). */
LBRB_API int lbrb_moments_from_pre(lbrb_t *h, const double *fpre, const double *gpre, int layout);
/* Seeded initial state: linear conduction T plus uniform noise of amplitude
 * `noise` (splitmix64 of seed and node index), f = feq(1,0), g = geq(T,0),
 * moments by the restart route.  No reference counterpart (the reference's
 * scratch state uses rand(), inithydro temppart_dump.c:686-701). */
LBRB_API int lbrb_init_conduction(lbrb_t *h, uint64_t seed, double noise);

/* ---- time loop ----------------------------------------------------------- */
/* Advance n steps: the loop body temppart_dump.c:1675-1757 (stream, walls,
 * force, moments, particles, records, collision) or tempvel_nudge.c:2349-2377
 * (observation update, stream, walls, moments, nudged collision). */
LBRB_API int lbrb_step(lbrb_t *h, int n);
/* Wait for all queued work and report device-side status (LBRB_ERR_RANGE,
 * LBRB_ERR_NONFINITE, ...). */
LBRB_API int lbrb_sync(lbrb_t *h);
LBRB_API int lbrb_get_istep(const lbrb_t *h, int *istep);
LBRB_API int lbrb_set_istep(lbrb_t *h, int istep);
/* Scan the populations for NaN/Inf (LBRB_ERR_NONFINITE if any). */
LBRB_API int lbrb_check_finite(lbrb_t *h);
/* Queue all work of this handle on `cuda_stream` (a cudaStream_t of the
 * handle's device; NULL restores the handle's own stream).  lbrb_step() joins
 * its record copies back into this stream before returning, so an event
 * recorded on it after lbrb_step() covers the whole step. */
LBRB_API int lbrb_set_stream(lbrb_t *h, void *cuda_stream);
/* CUDA-graph replay inside lbrb_step: runs of 3 steps without a record
 * replay a graph of the same launches (one graph per buffer phase, captured
 * on first use), so small grids are not bound by the host's per-launch
 * enqueue.  Results are identical either way.  -1 (the default): grids of
 * at most 2^20 nodes where two steps per launch do not apply (lbrb_set_pairs;
 * a two-step launch is faster than a replay of two single steps); 0: off;
 * 1: every grid, ahead of two-step launches.  Not used with nudging,
 * per-kernel timing, a y-slab, the legacy default stream, or while the
 * caller captures the handle's stream.  No counterpart in the reference. */
LBRB_API int lbrb_set_graph(lbrb_t *h, int mode);
/* Two steps per launch inside lbrb_step: the fused kernel computes step n
 * at a tile and a one-node ring into shared memory and step n+1 from there,
 * so populations and F cross HBM once per two steps (u, v, and T on record
 * steps, are still stored for every step; the particle kernels run after
 * the launch for each step).  Results are identical to single steps.
 * -1 (the default): pairs where a timed pair launch beats two single ones;
 * 1: always; 0: off (pairs give way to graph replays forced by
 * lbrb_set_graph(h, 1)).
 * Used with Dirichlet walls, without nudging or with bilinear nudging, not
 * on a y-slab, and never for the last step of a call (so
 * lbrb_get_poststream keeps its meaning).  With bilinear nudging, step n's
 * innovations are formed before the launch from T^n -- the moment of the
 * populations streaming into each observation's cell corners, summed as the
 * step sums it -- and added to g inside the launch right after the
 * collision; step n+1's are applied after the launch, as for one step.
 * The launch shape is timed on first use (once per process for handles
 * of the same kind, as for autotune); lbrb_get_pair_shape reports it
 * (shape index, tile columns and rows, ms per launch; shape -1 before).
 * Replaces, for two steps at a time, the reference's per-step sweeps
 * (stream, moments, collide: temppart_dump.c:1674-1759). */
LBRB_API int lbrb_set_pairs(lbrb_t *h, int mode);
/* fix the launch shape of the two-step kernel instead of timing the shapes
 * on first use (-1).  Tiles with a one-node ring recomputed around each:
 * 0: 32x8, 1: 32x4, 2: 32x16, 3: 64x4, 4: 32x8 with a thread per node of
 * the tile and its ring, 5: 30x8 likewise, 6: 32x8 at 5 blocks per SM,
 * 7: 32x6, 8: 64x8.  Strips of 32 columns walked down a chunk of rows,
 * recomputing only two halo columns and two rows per chunk (tile_y: rows
 * per group): 9: 8 rows, 3 blocks per SM; 10: 8 rows, 3 blocks, the next
 * group's loads issued before this group's second step (software
 * pipelining); 11: likewise, 2 blocks; 12: 6 rows, 4 blocks, pipelined;
 * 13: 4 rows, 6 blocks, pipelined; 14: 6 rows, 3 blocks, pipelined. */
LBRB_API int lbrb_set_pair_shape(lbrb_t *h, int shape);
/* the number of launch shapes of the two-step kernel (0 .. n-1) */
LBRB_API int lbrb_pair_shapes(void);
LBRB_API int lbrb_get_pair_shape(const lbrb_t *h, int *shape, int *tile_x, int *tile_y, float *ms);
/* Per-kernel device timing with CUDA events around each launch.  Classes:
 * 0 fused stream/collide, 1 particles, 2 nudging, 3 record copies.
 * lbrb_get_timing() waits, returns total milliseconds and launch counts per
 * class (arrays of length n <= 4) and resets the accumulators. */
LBRB_API int lbrb_set_timing(lbrb_t *h, int enable);
LBRB_API int lbrb_get_timing(lbrb_t *h, double *ms, int *launches, int n);
/* Launch shape of the fused kernel (index into the launch_shape list,
 * threads per block, min blocks per SM) and its timed milliseconds per
 * launch when the autotuner picked it (0 before the first step or with
 * autotune off). */
LBRB_API int lbrb_get_launch_shape(const lbrb_t *h, int *shape, int *block, int *min_blocks,
                                   float *ms);

/* ---- particles ------------------------------------------------------------ */
/* Replaces init_prtcl/restore_prtcl (Trajectories/code/mympi2.h:116-290,
 * temppart_dump.c:252-346).  Arrays of length n == nprtcl; positions in the
 * global frame; ptype LBRB_PTYPE_*; invtau = onebytaulag per particle. */
LBRB_API int lbrb_particles_set(lbrb_t *h, int n, const int *ids, const double *x, const double *y,
                       const double *u, const double *v, const int *ptype, const double *invtau);
/* Current particle state (after wrap/reflect, toggle_prtcl mympi2.h:568-760);
 * any pointer may be NULL. */
LBRB_API int lbrb_particles_get(lbrb_t *h, int n, int *ids, double *x, double *y, double *u, double *v,
                       double *xo, double *yo, double *uo, double *vo);

/* ---- trajectory records (prtcl_write, temppart_dump.c:1467-1571) ----------- */
/* Records are kept on the device and copied to pinned host memory as they
 * complete.  Drain up to max_records of them, oldest first: steps[r] is the
 * step of record r and buf holds [r][field][nprtcl] doubles with
 * LBRB_REC_NBASIC or LBRB_REC_NFULL fields; ids (may be NULL) gets the
 * particle ids in record order. */
LBRB_API int lbrb_record_pending(lbrb_t *h, int *count);
LBRB_API int lbrb_record_drain(lbrb_t *h, int max_records, int *steps, double *buf, int *ids,
                      int *n_drained);

/* ---- nudging --------------------------------------------------------------- */
/* Box mode (tempvel_nudge.c): initial observations (set_nudge_vol contin==0,
 * :2080-2122) and the observation file for step istep+ntempread-1 read by
 * read_prtcl (:1380-1476), arrays of length nobs in file order. */
LBRB_API int lbrb_nudge_init(lbrb_t *h, int n, const double *x, const double *y, const double *T,
                    const int *ids);
LBRB_API int lbrb_nudge_load(lbrb_t *h, int n, const double *x, const double *y, const int *ids,
                    const double *T);
/* Bilinear mode (no reference counterpart): observations for nsteps
 * consecutive steps starting at step first_step, arrays [nsteps][nobs]. */
LBRB_API int lbrb_nudge_obs(lbrb_t *h, int first_step, int nsteps, const double *x, const double *y,
                   const double *T);

/* ---- diagnostics ----------------------------------------------------------- */
/* Mean kinetic energy and mean temperature over the interior (evolution.dat,
 * temppart_dump.c:1739-1757), compensated FP64 sums. */
LBRB_API int lbrb_energy(lbrb_t *h, double *ke_mean, double *t_mean);
/* Volume Nusselt number 1 + <vT> ny / (kappa (Tdown-Tup)), kappa = (relaxg-1/2)/3. */
LBRB_API int lbrb_nusselt(lbrb_t *h, double *nu);
/* Per-row profile [ny][9]: rho, u, v, u^2, v^2, T, vT, dT/dy (profile(),
 * tempvel_nudge.c:1104-1260), and the row Nusselt number.  Means are the
 * reference's row sums scaled by 1/nx (taken here as compensated sums);
 * dT/dy is T(j+1) - T(j), periodic at the top row as the reference's halo
 * row there is, and with box nudging that halo value is row 0's sum of g
 * without the 1/2 nud_term (hydrovar forms halo rows whose nudge_vol is 0).
 * The reference run on several ranks in y treats the last row of every rank
 * that way; this whole-domain profile does so at the top row only. */
LBRB_API int lbrb_profile(lbrb_t *h, double *out);

/* ---- adjoint (no counterpart in the reference) ----------------------------- */
/* Observations of an assimilation window: nobs_steps window steps
 * (1-based, increasing), each with nobs observations -- positions x, y in
 * the reference frame and temperatures T, arrays [nobs_steps][nobs]. */
LBRB_API int lbrb_adjoint_set_obs(lbrb_t *h, int nobs_steps, const int *steps, int nobs,
                                  const double *x, const double *y, const double *T);
/* Run the window from the initial temperature field T0 ([ny][nx]: f =
 * feq(1,0), g = geq(T0,0), moments by the restart route) for nsteps steps and
 * return the misfit J = sum over the observations of (T(x,t) - T_obs)^2,
 * T(x,t) the bilinear interpolation of the step's temperature.  If dJdT0 is
 * not NULL, also its gradient with respect to T0 ([ny][nx]) by the adjoint
 * of the time step.  The backward pass reads each forward state's F and
 * moments: from a store of all of them (see lbrb_adjoint_set_store), or by
 * recomputing the forward from checkpoints taken every `checkpoint_every`
 * steps (`checkpoint_every` is unused in store mode).  Dirichlet walls, no
 * nudging; the handle's state ends at the end of the window; particles are
 * not advanced. */
LBRB_API int lbrb_adjoint_window(lbrb_t *h, const double *T0, int nsteps, int checkpoint_every,
                                 double *J, double *dJdT0);
/* Launch variant of the two-step adjoint kernel, 0 .. lbrb_adjoint_variants()-1:
 * 0-3 the tiled kernel (tile shape, threads, blocks per SM), 4 and up the
 * marching kernel (rows per group, blocks per SM, register prefetch, waves).
 * -1 (the default): timed on the first step pair of the next window and the
 * fastest kept.  Every variant gives the same gradient, bit for bit. */
LBRB_API int lbrb_adjoint_variants(void);
LBRB_API int lbrb_adjoint_set_variant(lbrb_t *h, int variant);
LBRB_API int lbrb_adjoint_get_variant(const lbrb_t *h, int *variant);
/* How a gradient window keeps the forward states for its backward pass.
 * 1: a store of every state's F and moments, 5 planes per step, (nsteps+1) x
 *    5 x pitch x ny elements of the handle's precision (21 GB at 1024x512 over
 *    2000 steps in FP32), allocated by the window and kept by the handle for
 *    the next one; nothing is recomputed.  LBRB_ERR_NOMEM if it cannot be
 *    allocated.
 * 0: checkpoints every checkpoint_every steps, each segment recomputed during
 *    the backward pass (memory of two segments); frees a store.
 * -1 (the default): the store when it fits in half of the device's free
 *    memory (an earlier window's store counted as free), else checkpoints,
 *    releasing an earlier window's store first.
 * Both give the same J and gradient, bit for bit.  get_store: the mode, whether
 * the last gradient window stored (1) or recomputed (0), and the store's size. */
LBRB_API int lbrb_adjoint_set_store(lbrb_t *h, int mode);
LBRB_API int lbrb_adjoint_get_store(const lbrb_t *h, int *mode, int *used_last, size_t *bytes);

/* ---- ensemble (no counterpart in the reference) ---------------------------
 * Independent runs ("members": handles made by lbrb_create, of any grid size
 * and closure) advanced together.  Per time step one launch covers the fused
 * stream/collide step of every member (a persistent kernel over a work list
 * of equal tiles), one advances every member's particles and scatters its
 * bilinear observations, and one applies the nudging of all members; the
 * steps are replayed from a CUDA graph.  A member's state stays in its
 * handle: every per-handle call (get_moments, particles_get, energy, ...)
 * works between ensemble steps, and a member advanced by the ensemble ends
 * bit-identical to the same handle advanced by lbrb_step.
 * Members: one device, one precision, one wall mode, nudging none or
 * bilinear, no trajectory records (noutconfig 0 when nprtcl > 0).  The
 * ensemble borrows the handles: destroy it before them. */
typedef struct lbrb_ensemble_s lbrb_ensemble_t;
LBRB_API int lbrb_ensemble_create(lbrb_t *const *members, int n, lbrb_ensemble_t **out);
LBRB_API int lbrb_ensemble_destroy(lbrb_ensemble_t *e);
LBRB_API const char *lbrb_ensemble_last_error(const lbrb_ensemble_t *e);
/* Advance every member by n steps (queued, like lbrb_step). */
LBRB_API int lbrb_ensemble_step(lbrb_ensemble_t *e, int n);
/* Wait; return the first member status that is not LBRB_OK. */
LBRB_API int lbrb_ensemble_sync(lbrb_ensemble_t *e);
LBRB_API int lbrb_ensemble_set_stream(lbrb_ensemble_t *e, void *cuda_stream);
/* Launch variant of the fused phase (threads per tile row, rows per tile,
 * schedule: 0 one block per tile, 1 persistent grid stride, 2 persistent
 * atomic tile counter; pull form: 1 interior rows without wall logic, 0 the
 * general pull).  -1 (the default): the autotuner times every variant on
 * the members' state at the next step and keeps the fastest. */
LBRB_API int lbrb_ensemble_nvariants(void);
LBRB_API int lbrb_ensemble_set_schedule(lbrb_ensemble_t *e, int variant);
LBRB_API int lbrb_ensemble_get_schedule(const lbrb_ensemble_t *e, int *variant, int *block,
                                        int *rows, int *schedule, int *fast_pull, float *ms);
/* Two steps per launch for every member (as lbrb_set_pairs, with Dirichlet
 * walls; bilinear-nudged members too): every step of a call but its last
 * (and one more when an even count remains) goes in pairs, each pair one
 * launch over all members -- marching over strips of 32 columns x chunks of
 * rows (lb_march_kernel's block) or over tiles (lb_pair_kernel's block), the
 * members' views in shared memory -- with the nudged members' step-n
 * innovations formed before it and every member's particles, step n+1
 * innovations and nudging apply after it; 12 steps are replayed from a CUDA
 * graph.  Members end bit-identical to lbrb_step.
 * mode -1 (the default) and 1: on; 0: one step per launch.  The launch
 * variant (lbrb_ensemble_pair_variants() of them: marching with 6 or 8 rows
 * per group, tiles of 32 x 8 or 30 x 8 nodes) is timed at the first paired
 * call unless set; lbrb_ensemble_get_pairs reports its rows per group or per
 * tile (0 before) and ms per launch (0 when set rather than timed). */
LBRB_API int lbrb_ensemble_set_pairs(lbrb_ensemble_t *e, int mode);
LBRB_API int lbrb_ensemble_get_pairs(const lbrb_ensemble_t *e, int *mode, int *rows, float *ms);
LBRB_API int lbrb_ensemble_pair_variants(void);
/* variant -1: time the variants at the next paired call (the default);
 * 0 .. lbrb_ensemble_pair_variants() - 1: use that one.  get: the variant
 * (-1 before timing) and its tile columns (0 for a marching variant). */
LBRB_API int lbrb_ensemble_set_pair_variant(lbrb_ensemble_t *e, int variant);
LBRB_API int lbrb_ensemble_get_pair_variant(const lbrb_ensemble_t *e, int *variant, int *tile_cols);
/* Per-launch device timing (steps then launch directly, without the graph).
 * Classes: 0 fused step (one or two steps), 1 particles + innovation
 * scatter, 2 nudging (apply; with pairs also the innovations before the
 * launch). */
LBRB_API int lbrb_ensemble_set_timing(lbrb_ensemble_t *e, int enable);
LBRB_API int lbrb_ensemble_get_timing(lbrb_ensemble_t *e, double *ms, int *launches, int n);

/* ---- diagnostics without allocation ----------------------------------------
 * No counterpart in the reference.  lbrb_stats_noalloc computes what
 * lbrb_energy() and lbrb_nusselt() give (out3 = mean kinetic energy, mean T,
 * Nusselt number) from device fields the caller owns -- rho, u, v, T, each
 * ny rows of `pitch` elements of `precision` (LBRB_PREC_FP64: double,
 * LBRB_PREC_FP32_SHIFTED: float) -- for callers that cannot allocate device
 * memory at that point (a framework that keeps all device memory in its own
 * pool, a loop that must not allocate after start-up).  It allocates
 * nothing: its scratch is a fixed device array of LBRB_STATS_NOALLOC_MAX_ROWS
 * row records, so ny above that is rejected with LBRB_ERR_RANGE.  Work runs
 * on `cuda_stream` (NULL: the default stream) and the call returns after it
 * finishes.  Calls share the scratch array: calls that overlap on the GPU
 * race.  The first call on a device looks up the array's address, which
 * loads this library's device code on that device (with CUDA's default lazy
 * module loading) and with it the 768 KiB array: make that first call at
 * start-up, before memory runs short and before any stream capture; later
 * calls take no device memory.  Only nx <= pitch is checked: each field must
 * hold ny * pitch elements, which a device pointer does not reveal. */
#define LBRB_STATS_NOALLOC_MAX_ROWS 16384
LBRB_API int lbrb_stats_noalloc(const void *rho, const void *u, const void *v, const void *T,
                                int precision, int nx, int ny, int pitch, double relaxg,
                                double Tup, double Tdown, void *cuda_stream, double *out3);

/* ---- One domain over several GPUs: y-slabs ------------------------------
 * Replaces the reference's domain decomposition over MPI ranks and its halo
 * refresh of the populations around the stream (pbc, temppart_dump.c:234-250,
 * called in the loop at temppart_dump.c:1674-1759) for a split in y.
 * A handle created with ny rows becomes rows [j0, j0 + ny) of a domain of
 * ny_total rows.  Only the slab at j0 = 0 has the bottom wall and only the
 * slab ending at ny_total the top wall.  Across an inner boundary a step
 * pulls the three f and three g populations that cross it from the
 * handle's ghost rows, which must hold the neighbour slab's boundary row
 * after its previous step.  The slabs of one domain then advance exactly as
 * the whole domain in one handle would, bit for bit.
 * lbrb_init_conduction on a slab gives the whole domain's profile and noise
 * at its rows; lbrb_nusselt gives the slab's mean of v T at the whole
 * domain's height (the domain's Nu is the slabs' values weighted by ny).
 * Supported: Dirichlet and adiabatic walls (the walls of the domain only);
 * particles (held by their owner slab, below); bilinear nudging: every slab
 * holds all observations (lbrb_nudge_obs on each, in the whole domain's
 * coordinates) and lbrb_slab_step applies them (one process per GPU:
 * lbrb_slab_nudge); box nudging (FP64): every slab takes all observations
 * (lbrb_nudge_init / lbrb_nudge_load on each) and keeps the running means
 * of the boxes' nodes in its own rows, inside its lbrb_step, as the
 * reference's ranks in y do.  Two steps per launch need Dirichlet walls and
 * no nudging.
 * Create slab handles with nprtcl = 0 (lbrb_slab_set rejects a handle with
 * whole-domain particles). */
LBRB_API int lbrb_slab_set(lbrb_t *h, int j0, int ny_total);
/* bytes of one packed boundary row set: 6 rows (f then g) of nx values */
LBRB_API size_t lbrb_slab_ghost_bytes(const lbrb_t *h);
/* device buffers of a slab: `up` and `down` receive lbrb_slab_pack's output
 * (the top row's upward populations f2 f5 f6 g2 g5 g6 for the slab above;
 * the bottom row's downward f4 f7 f8 g4 g7 g8 for the slab below);
 * `ghost_lo` / `ghost_hi` are the rows below row 0 / above row ny-1 (NULL at
 * a wall).  One process per GPU: after lbrb_slab_pack, send `up` to the slab
 * above's ghost_lo and `down` to the slab below's ghost_hi (NCCL send/recv
 * of lbrb_slab_ghost_bytes on the handle's stream), then lbrb_step(h, 1). */
LBRB_API int lbrb_slab_buffers(lbrb_t *h, void **up, void **down, void **ghost_lo, void **ghost_hi);
LBRB_API int lbrb_slab_pack(lbrb_t *h);
/* Two steps per exchange (one process per GPU; no particles, no nudging):
 * lbrb_slab_pack2 packs two-row ghost blocks of lbrb_slab_ghost2_bytes
 * (the boundary row: its three f and three g populations that cross, its
 * k = 0, 1, 3 f and g, its F; then the three f and three g crossing
 * populations of the next row in); send `up` to the slab above's ghost_lo
 * and `down` to the slab below's ghost_hi (lbrb_slab_buffers2), then
 * lbrb_step(h, 2) advances two steps in one launch, bit-identical to two
 * one-step exchanges.  Its second step writes the moments; the post-stream
 * populations of the first are not kept (lbrb_get_poststream).
 * lbrb_step(h, 2) returns LBRB_ERR_STATE unless lbrb_slab_pack2 ran on the
 * slab since its last step (a one-step lbrb_slab_pack clears that mark); the
 * exchange itself is the caller's and cannot be checked here. */
LBRB_API size_t lbrb_slab_ghost2_bytes(const lbrb_t *h);
LBRB_API int lbrb_slab_buffers2(lbrb_t *h, void **up, void **down, void **ghost_lo, void **ghost_hi);
LBRB_API int lbrb_slab_pack2(lbrb_t *h);
/* nsteps steps of a whole domain whose slabs this process holds (one or
 * several GPUs), slabs in order of j0: per step, every slab packs and copies
 * its boundary rows into its neighbours' ghost rows (peer copies across
 * GPUs), then steps; events order the copies against the neighbours' steps.
 * Without nudging, steps go two per launch (as lbrb_set_pairs describes;
 * a slab's lbrb_set_pairs(h, 0) turns it off): the exchange is then two rows
 * deep and goes every two steps; results are the same bit for bit.
 * The moments (rho, u, v, T) are written on the last of the nsteps.
 * With particles (lbrb_slab_particles_set on every slab): after every
 * slab's step, the particle exchange below, its messages copied between the
 * slabs around the ring (peer copies across GPUs); each slab keeps its own
 * particles and records (lbrb_slab_particles_get, lbrb_slab_record_drain).
 * With bilinear nudging, after every slab's step each slab scatters the
 * innovations of the observations to the cell corners in its own rows
 * (order-free fixed-point sums, so g is the whole domain's bit for bit). */
/* Errors: a bad slab list is rejected before any launch; an error during
 * the steps (a full record ring is checked first, so it is not one) leaves
 * the slabs possibly at different steps: set their state again. */
LBRB_API int lbrb_slab_step(lbrb_t *const *slabs, int nslabs, int nsteps);

/* ---- particles of a y-slab, held by their owner slab ----------------------
 * (no reference counterpart as an API; the reference's ranks keep the
 * particles in their block, init_prtcl at Trajectories/code/mympi2.h:116-290,
 * and hand those that leave it to the neighbour rank each step,
 * toggle_prtcl at mympi2.h:568-760.)
 * lbrb_slab_particles_set keeps, of the n particles given (the whole
 * domain's, arguments as lbrb_particles_set), those whose cell lies in the
 * slab's rows, in the order given.  capacity: particles the slab can hold
 * (0: n); handoff_capacity: particles that may leave it per step and
 * direction (0: min(capacity, 1024)).  A step of a slab with particles, one
 * process per GPU (s+1 / s-1: the slabs above / below, around the ring:
 * the top slab's "up" goes to slab 0 and slab 0's "down" to the top slab):
 *   lbrb_slab_pack; send up -> s+1 ghost_lo, down -> s-1 ghost_hi;
 *   lbrb_step(h, 1);
 *   lbrb_slab_moments_pack; send mom_up -> s+1 mom_lo, mom_down -> s-1 mom_hi;
 *   lbrb_slab_particles_step;
 *   send hand_up -> s+1 hand_lo, hand_down -> s-1 hand_hi;
 *   lbrb_slab_particles_recv.
 * (The hand-off exchange may go with the next step's ghost exchange, with
 * lbrb_slab_particles_recv before the next lbrb_step.)  Two steps per
 * launch: lbrb_slab_pack2 and its exchange, lbrb_step(h, 2), then the
 * moment pack / exchange / particle step / hand-off exchange / receive of
 * the first step, whose receive moves the handle on to the second step,
 * and the same again for the second (no nudging).  Sizes are
 * lbrb_slab_particle_bytes (mom_up, mom_down, and each hand-off list); all
 * work and copies on the handle's stream, so a caller's NCCL send/recv on
 * that stream orders itself.  The moment messages carry the fields one row
 * below the slab and two above (u, v, T of the sender's top row; u, v,
 * u^{n-1}, v^{n-1}, T of its row 0 and u, v, T of its row 1), which is all
 * a particle stencil of the slab reads while no particle moves more than a
 * row per step; a hand-off list carries the particles that left the slab's
 * rows (their whole state, 80 bytes each).  Each message has a header with
 * the sender's step and rows: a message from the wrong step or neighbour,
 * a particle outside the slab's reach, or a full slab or list is reported
 * by lbrb_sync (LBRB_ERR_STATE, LBRB_ERR_RANGE, LBRB_ERR_OVERFLOW).  Calls
 * out of this order return LBRB_ERR_STATE.  A particle's state equals the
 * whole domain's bit for bit; its record goes into the ring of the slab
 * that advanced it.
 * capacity -1 (with n = 0): no particles, only the moment messages, for a
 * nudged slab without particles (lbrb_slab_particles_step and _recv are
 * then not called; the other calls of the step stay). */
LBRB_API int lbrb_slab_particles_set(lbrb_t *h, int n, const int *ids, const double *x, const double *y,
                                     const double *u, const double *v, const int *ptype, const double *invtau,
                                     int capacity, int handoff_capacity);
LBRB_API int lbrb_slab_particle_bytes(const lbrb_t *h, size_t *mom_up, size_t *mom_down, size_t *handoff);
LBRB_API int lbrb_slab_particle_buffers(lbrb_t *h, void **mom_up, void **mom_down, void **mom_lo, void **mom_hi,
                                        void **hand_up, void **hand_down, void **hand_lo, void **hand_hi);
LBRB_API int lbrb_slab_moments_pack(lbrb_t *h);
LBRB_API int lbrb_slab_particles_step(lbrb_t *h);
LBRB_API int lbrb_slab_particles_recv(lbrb_t *h);
/* Bilinear nudging of a y-slab stepped by its own process: after
 * lbrb_step(h, 1), lbrb_slab_moments_pack and the moment exchange, the
 * step's observations (lbrb_nudge_obs with the whole domain's
 * coordinates) whose cell has a corner in the slab's rows are interpolated
 * from T of the slab's rows and of the received moment rows, and their
 * shares added at the corners in the slab's rows; the slab's g then equals
 * the whole domain's bit for bit.  Once per step; lbrb_step refuses the next
 * step of a nudged slab until it ran.  (No reference counterpart as an API:
 * the reference's nudged run is not decomposed in y in this way.) */
LBRB_API int lbrb_slab_nudge(lbrb_t *h);
/* the slab's particle count and state (waits; arrays of at least max_n) */
LBRB_API int lbrb_slab_particles_count(lbrb_t *h, int *n);
LBRB_API int lbrb_slab_particles_get(lbrb_t *h, int max_n, int *n, int *ids, double *x, double *y, double *u,
                                     double *v, double *xo, double *yo, double *uo, double *vo);
/* Records of the particles the slab advanced, oldest first, one per call:
 * step (-1 when none is pending), count, ids[count] and buf[field][count]
 * (LBRB_REC_NBASIC or LBRB_REC_NFULL fields), arrays of at least max_n. */
LBRB_API int lbrb_slab_record_pending(lbrb_t *h, int *count);
LBRB_API int lbrb_slab_record_drain(lbrb_t *h, int max_n, int *step, int *count, int *ids, double *buf);
/* byte layout of the messages (needs no device): header bytes of each
 * message (int count, step, j0, j1, kind, 3 pad), bytes of a hand-off
 * record (9 doubles x y u v xo yo uo vo invtau, int id, int type; after the
 * header), offset of the first moment plane (planes of nx values, each
 * mom plane stride = nx * element size rounded up to 256 bytes) */
LBRB_API int lbrb_slab_particle_format(int *msg_header_bytes, int *record_bytes, int *mom_planes_offset);

#ifdef __cplusplus
}
#endif
#endif
