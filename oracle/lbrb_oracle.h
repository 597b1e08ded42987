/*
 * lbrb_oracle.h -- CPU restatement of the reference time-step loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it.  The product (liblbrb.so) never links or calls it.
 *
 * One whole domain, FP64, interior arrays only (no halo); the reference's
 * periodic halos become index wrap.  Every arithmetic expression follows the
 * reference's operation order so that results are bit-identical to the
 * reference compiled with gcc -O2 on x86-64 (no FMA contraction).
 *
 * Layouts (0-based interior indices, i = x in [0,nx), j = y in [0,ny)):
 *   populations  f[k][j][i]  ->  f[(k*ny + j)*nx + i]
 *   scalars      s[j][i]     ->  s[j*nx + i]
 * Reference node (i_ref, j_ref) with 1 <= i_ref <= NX maps to (i_ref-1, j_ref-1).
 */
#ifndef LBRB_ORACLE_H
#define LBRB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_TWALL_DIRICHLET = 0, ORC_TWALL_ADIABATIC = 1 };
enum { ORC_NUDGE_NONE = 0, ORC_NUDGE_REFBOX = 1, ORC_NUDGE_BILINEAR = 2 };
enum { ORC_PTYPE_TRACER = 0, ORC_PTYPE_INERTIAL = 1 };

typedef struct {
  int nx, ny;
  double relax, relaxg;     /* tau, tau_g */
  double Tup, Tdown;        /* top / bottom wall temperature */
  double gravity;           /* reference sign convention: negative, F_y = -gravity*rho*T */
  int twall;                /* ORC_TWALL_* */
  int nudge;                /* ORC_NUDGE_* */
  double alpha;             /* nudging coefficient */
  int ntempread;            /* observation file interval (reference box mode) */
  double beta;              /* Maxey-Riley added-mass coefficient */
  int noutconfig;           /* record interval, 0 = never */
  int record_full;          /* also record the 8 Maxey-Riley terms at (xo,yo) */
} orc_params;

typedef struct orc_s orc_t;

/* field ids for orc_field() */
enum {
  ORC_F = 0, ORC_G, ORC_RHO, ORC_U, ORC_V, ORC_T, ORC_UBEF, ORC_VBEF,
  ORC_FY, ORC_TEMPREADINT, ORC_NUDTERM, ORC_NUDGE_SRC,
  ORC_TSUM, /* sum of g of the step, before box nudging's 1/2 nud_term */
  ORC_NFIELDS
};
/* particle array ids for orc_prtcl() */
enum {
  ORC_PX = 0, ORC_PY, ORC_PU, ORC_PV, ORC_PXO, ORC_PYO, ORC_PUO, ORC_PVO,
  ORC_PINVTAU, ORC_NPARR
};
/* record field ids (rows of the record block) */
enum {
  ORC_R_X = 0, ORC_R_Y, ORC_R_U, ORC_R_V, ORC_R_XO, ORC_R_YO, ORC_R_UO, ORC_R_VO,
  ORC_R_TEMP, ORC_R_DTU, ORC_R_DTV, ORC_R_DXU, ORC_R_DXV, ORC_R_DYU, ORC_R_DYV,
  ORC_R_FU, ORC_R_FV, ORC_NREC
};

orc_t *orc_create(const orc_params *p, int nprtcl);
void orc_destroy(orc_t *s);

double *orc_field(orc_t *s, int which);
int *orc_nudge_vol(orc_t *s);
double *orc_prtcl(orc_t *s, int which);
int *orc_prtcl_ids(orc_t *s);
int *orc_prtcl_type(orc_t *s);
/* record block [ORC_NREC][nprtcl]; *istep_out = step of the last record or -1 */
double *orc_record(orc_t *s, int *istep_out);

/* one full reference step number `istep` (1-based, like the reference loop) */
void orc_step(orc_t *s, int istep);

/* Reference restart route (temppart_dump.c:703-726): moments from the "pre"
 * populations; v gets +0.5*(-gravity)*T without a rho factor. */
void orc_moments_from_pre(orc_t *s, const double *fpre, const double *gpre);

/* The benchmark configurations' initial state: linear conduction T plus seeded uniform noise,
 * f = feq(1,0), g = geq(T,0); moments by the restart route. */
void orc_init_conduction(orc_t *s, unsigned long long seed, double noise_amp);
double orc_splitmix_uniform(unsigned long long seed, unsigned long long index);

/* Reference box nudging (tempvel_nudge.c): initial observation arrays
 * (set_nudge_vol, contin==0, :2080-2122) and the file read every ntempread
 * steps (read_prtcl :1432-1476).  Arrays have length nprtcl, file order. */
void orc_nudge_init(orc_t *s, const double *x, const double *y,
                    const double *T, const int *id);
void orc_nudge_load(orc_t *s, const double *x, const double *y,
                    const int *id, const double *T);
/* bilinear nudging: observations valid for the next step (positions, T) */
void orc_nudge_obs(orc_t *s, int nobs, const double *x, const double *y,
                   const double *T);

/* diagnostics over the interior, reference summation order */
void orc_energy(orc_t *s, double *ke_mean, double *t_mean);
/* per-row profile: out[9*ny]: rho,u,v,u2,v2,T,vT,dyT (reference profile())
 * plus row Nusselt ingredients; rows j=0..ny-1 */
void orc_profile(orc_t *s, double *out);
/* the same as the reference prints it from a run on `ranks_y` ranks in y
 * (only dT/dy at the last row of each rank depends on that) */
void orc_profile_ranks(orc_t *s, int ranks_y, double *out);
double orc_nusselt(orc_t *s);

/* FP64 tangent-linear model of an assimilation window (no counterpart in the
 * reference): from the initial temperature T0 ([ny][nx]; f = feq(1,0),
 * g = geq(T0,0), moments by the restart route) and a direction dT0, run
 * nsteps reference steps (Dirichlet walls, no particles, no nudging) and
 * return the misfit J = sum over observations of (T(x,t) - T_obs)^2 and its
 * directional derivative dJ = <grad J, dT0>.  Observations: nobs_steps steps
 * (1-based, increasing), nobs each, arrays [nobs_steps][nobs]. */
void orc_tlm_window(orc_t *s, const double *T0, const double *dT0, int nsteps, int nobs_steps,
                    const int *steps, int nobs, const double *ox, const double *oy,
                    const double *oT, double *J, double *dJ);

#ifdef __cplusplus
}
#endif
#endif
