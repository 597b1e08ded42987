/*
 * lbrb_oracle.c -- CPU restatement of the reference time-step loop (FP64).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 *
 * What is restated, and where it comes from (reference paths, file:line):
 *   lattice tables             Trajectories/code/temppart_dump.c:1363-1401 (dellar)
 *   pull streaming             temppart_dump.c:781-854 (8 in-place sweeps; here a
 *                              per-node pull, which moves the same values)
 *   force from step n-1        temppart_dump.c:744-755 (forcingconstructWW)
 *   f half-way bounce-back     temppart_dump.c:763-777, 859-894
 *   g anti-bounce-back (T)     temppart_dump.c:896-921
 *   g adiabatic walls (N)      Nudging/code/tempvel_nudge.c:684-702, 783-962
 *   moments                    temppart_dump.c:957-987; tempvel_nudge.c:1069-1102
 *   equilibria                 temppart_dump.c:1097-1180
 *   collision                  temppart_dump.c:1314-1341; nudged g
 *                              tempvel_nudge.c:1917-1945
 *   bilinear interpolation     Trajectories/code/mympi2.h:292-311
 *   particle advance           mympi2.h:350-433; record mympi2.h:434-565 and
 *                              temppart_dump.c:1467-1571; wrap/reflect
 *                              mympi2.h:589-635, 681-723
 *   box nudging observations   tempvel_nudge.c:1380-1781 (read_prtcl)
 *   energy diagnostics         temppart_dump.c:1739-1757
 *   restart-route moments      temppart_dump.c:703-726 (inithydro, scratch==0)
 *
 * The reference's periodic halos (pbc + communication, periodic in x AND y)
 * become index wrap on a single whole-domain layout.  Expressions keep the
 * reference's operation order: compiled with gcc -O2 on x86-64 (no FMA) the
 * field results are bit-identical to the reference run at NPX=1.
 */
#include "lbrb_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NPOP 9

/* D2Q9 constants as the reference builds them (temppart_dump.c:9-12, 1363-1401).
 * Note cy[3] = -cy[1] and cx[4] = -cx[2] are negative zeros there. */
static const double CS2 = 1.0 / 3.0;
static const double WW[NPOP] = {16. / 36., 4. / 36., 4. / 36., 4. / 36., 4. / 36.,
                                1. / 36.,  1. / 36., 1. / 36., 1. / 36.};
static const double CX[NPOP] = {0., 1., 0., -1., -0., 1., -1., -1., 1.};
static const double CY[NPOP] = {0., 0., 1., -0., -1., 1., 1., -1., -1.};
static const int ICX[NPOP] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int ICY[NPOP] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
/* opposite direction */
static const int OPP[NPOP] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

struct orc_s {
  orc_params p;
  int np;
  double *fld[ORC_NFIELDS];
  double *fs, *gs;               /* post-stream populations of the current step */
  double *d[6];                  /* dtu dtv dxu dxv dyu dyv */
  int *nudge_vol;
  /* particles */
  double *pa[ORC_NPARR];
  int *pid, *ptype;
  double *rec;
  int rec_step;
  /* reference box nudging state (tempvel_nudge.c main :2294-2306) */
  double *ox, *oy, *oT;          /* prtcl_x/y/T: last file, file order */
  int *oid;                      /* prtcl_ids: initial order */
  double *fx, *fy, *fT;          /* prtcl2_*: the file just loaded */
  int *fid;
  double *xint, *yint, *Tint, *dxs, *dys, *dTs;
  int *chk_id, *bc_chky, *xidx, *yidx;
  /* bilinear nudging observations */
  int nobs;
  double *bx, *by, *bT;
  int64_t *acc;
};

static inline int wrap(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}
static inline size_t sidx(const orc_t *s, int i, int j) { return (size_t)j * s->p.nx + i; }
static inline size_t pidx(const orc_t *s, int k, int i, int j) {
  return ((size_t)k * s->p.ny + j) * s->p.nx + i;
}

orc_t *orc_create(const orc_params *p, int nprtcl) {
  orc_t *s = (orc_t *)calloc(1, sizeof(orc_t));
  if (!s) return NULL;
  s->p = *p;
  s->np = nprtcl;
  size_t n = (size_t)p->nx * p->ny;
  for (int w = 0; w < ORC_NFIELDS; w++) {
    size_t len = (w == ORC_F || w == ORC_G) ? NPOP * n : n;
    s->fld[w] = (double *)calloc(len, sizeof(double));
  }
  s->fs = (double *)calloc(NPOP * n, sizeof(double));
  s->gs = (double *)calloc(NPOP * n, sizeof(double));
  for (int w = 0; w < 6; w++) s->d[w] = (double *)calloc(n, sizeof(double));
  s->nudge_vol = (int *)calloc(n, sizeof(int));
  size_t m = nprtcl > 0 ? (size_t)nprtcl : 1;
  for (int w = 0; w < ORC_NPARR; w++) s->pa[w] = (double *)calloc(m, sizeof(double));
  s->pid = (int *)calloc(m, sizeof(int));
  s->ptype = (int *)calloc(m, sizeof(int));
  s->rec = (double *)calloc(ORC_NREC * m, sizeof(double));
  s->rec_step = -1;
  double **dd[] = {&s->ox, &s->oy, &s->oT, &s->fx, &s->fy, &s->fT,
                   &s->xint, &s->yint, &s->Tint, &s->dxs, &s->dys, &s->dTs};
  for (unsigned w = 0; w < sizeof(dd) / sizeof(dd[0]); w++)
    *dd[w] = (double *)calloc(m, sizeof(double));
  int **ii[] = {&s->oid, &s->fid, &s->chk_id, &s->bc_chky, &s->xidx, &s->yidx};
  for (unsigned w = 0; w < sizeof(ii) / sizeof(ii[0]); w++) *ii[w] = (int *)calloc(m, sizeof(int));
  s->acc = (int64_t *)calloc(n, sizeof(int64_t));
  return s;
}

void orc_destroy(orc_t *s) {
  if (!s) return;
  for (int w = 0; w < ORC_NFIELDS; w++) free(s->fld[w]);
  free(s->fs); free(s->gs);
  for (int w = 0; w < 6; w++) free(s->d[w]);
  free(s->nudge_vol);
  for (int w = 0; w < ORC_NPARR; w++) free(s->pa[w]);
  free(s->pid); free(s->ptype); free(s->rec);
  free(s->ox); free(s->oy); free(s->oT); free(s->fx); free(s->fy); free(s->fT);
  free(s->xint); free(s->yint); free(s->Tint); free(s->dxs); free(s->dys); free(s->dTs);
  free(s->oid); free(s->fid); free(s->chk_id); free(s->bc_chky); free(s->xidx); free(s->yidx);
  free(s->bx); free(s->by); free(s->bT); free(s->acc);
  free(s);
}

double *orc_field(orc_t *s, int which) { return (which >= 0 && which < ORC_NFIELDS) ? s->fld[which] : NULL; }
int *orc_nudge_vol(orc_t *s) { return s->nudge_vol; }
double *orc_prtcl(orc_t *s, int which) { return (which >= 0 && which < ORC_NPARR) ? s->pa[which] : NULL; }
int *orc_prtcl_ids(orc_t *s) { return s->pid; }
int *orc_prtcl_type(orc_t *s) { return s->ptype; }
double *orc_record(orc_t *s, int *istep_out) {
  if (istep_out) *istep_out = s->rec_step;
  return s->rec;
}

/* ---------------------------------------------------------------- equilibria */
/* equilif/equilig, temppart_dump.c:1097-1180: r1 is rho (f) or T (g). */
static void equil(double r1, double u, double v, double feq[NPOP]) {
  double usq = u * u;
  double vsq = v * v;
  double sumsq = (usq + vsq) / (2. * CS2);
  double sumsq2 = sumsq * (1. - CS2) / CS2;
  double u2 = usq / (2. / 9.);
  double v2 = vsq / (2. / 9.);
  double ui = u / CS2;
  double vi = v / CS2;
  double uv = ui * vi;
  feq[0] = r1 * WW[0] * (1. - sumsq);
  feq[1] = r1 * WW[1] * (1. - sumsq + u2 + ui);
  feq[2] = r1 * WW[2] * (1. - sumsq + v2 + vi);
  feq[3] = r1 * WW[3] * (1. - sumsq + u2 - ui);
  feq[4] = r1 * WW[4] * (1. - sumsq + v2 - vi);
  feq[5] = r1 * WW[5] * (1. + sumsq2 + ui + vi + uv);
  feq[6] = r1 * WW[6] * (1. + sumsq2 - ui + vi - uv);
  feq[7] = r1 * WW[7] * (1. + sumsq2 - ui - vi + uv);
  feq[8] = r1 * WW[8] * (1. + sumsq2 + ui - vi - uv);
}

/* -------------------------------------------------------------- interpolation */
/* bilinear, mympi2.h:292-311.  (xx,yy) are reference node coordinates
 * (interior nodes at 1..NX, 1..NY); the cell index truncates toward zero and
 * the halo rows/columns 0 and N+1 wrap periodically (communication(),
 * mympi2.h:313-348, is periodic in x and in y). */
static double bilinear(const orc_t *s, const double *fld, double xx, double yy) {
  int nx = s->p.nx, ny = s->p.ny;
  int x1 = (int)xx;
  int x2 = x1 + 1;
  int y1 = (int)yy;
  int y2 = y1 + 1;
  int ix1 = wrap(x1 - 1, nx), ix2 = wrap(x2 - 1, nx);
  int jy1 = wrap(y1 - 1, ny), jy2 = wrap(y2 - 1, ny);
  double u11 = fld[(size_t)jy1 * nx + ix1];
  double u12 = fld[(size_t)jy2 * nx + ix1];
  double u21 = fld[(size_t)jy1 * nx + ix2];
  double u22 = fld[(size_t)jy2 * nx + ix2];
  double val1 = u11 * ((double)x2 - xx) * ((double)y2 - yy);
  double val2 = u21 * (xx - (double)x1) * ((double)y2 - yy);
  double val3 = u12 * ((double)x2 - xx) * (yy - (double)y1);
  double val4 = u22 * (xx - (double)x1) * (yy - (double)y1);
  return val1 + val2 + val3 + val4;
}

/* ------------------------------------------------------------------ stream */
/* Pull streaming plus wall rules.  Reference: temppart_dump.c:757-922
 * (Dirichlet T walls) and tempvel_nudge.c:677-1004 (adiabatic T walls, the
 * NPY>=2 behaviour: f streamed once everywhere, g rows 1 and NY held as
 * pre-stream copies of rows 2 and NY-1). */
static void stream(orc_t *s) {
  const int nx = s->p.nx, ny = s->p.ny;
  const double *f = s->fld[ORC_F], *g = s->fld[ORC_G];
  double *fs = s->fs, *gs = s->gs;
  const int adiabatic = (s->p.twall == ORC_TWALL_ADIABATIC);
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) {
      for (int k = 0; k < NPOP; k++) {
        int js = j - ICY[k];
        int is = wrap(i - ICX[k], nx);
        double fv;
        if (js < 0 || js >= ny) {
          /* half-way bounce-back with the pre-stream wall row:
           * f2,f5,f6(row 1) <- f4,f7,f8 ; f4,f7,f8(row NY) <- f2,f5,f6 */
          fv = f[pidx(s, OPP[k], i, j)];
        } else {
          fv = f[pidx(s, k, is, js)];
        }
        fs[pidx(s, k, i, j)] = fv;
        if (!adiabatic) {
          /* wall-crossing g values are replaced below; read in range */
          gs[pidx(s, k, i, j)] = (js < 0 || js >= ny) ? 0.0 : g[pidx(s, k, is, js)];
        } else {
          int jd = j;
          if (j == 0 || j == ny - 1) {
            /* rows 1 and NY are not streamed; they hold copies of rows 2 / NY-1 */
            int jc = (j == 0) ? 1 : ny - 2;
            gs[pidx(s, k, i, jd)] = g[pidx(s, k, i, jc)];
          } else {
            int jsrc = js;
            if (jsrc == 0) jsrc = 1;            /* row 1 holds row 2's copy */
            else if (jsrc == ny - 1) jsrc = ny - 2;
            gs[pidx(s, k, i, jd)] = g[pidx(s, k, is, jsrc)];
          }
        }
      }
    }
  }
  if (!adiabatic) {
    /* anti-bounce-back with the post-stream opposite population
     * (temppart_dump.c:896-921): top wall first, then bottom. */
    const double Tup = s->p.Tup, Tdown = s->p.Tdown;
    for (int i = 0; i < nx; i++) {
      int j = ny - 1;
      gs[pidx(s, 4, i, j)] = -gs[pidx(s, 2, i, j)] + 2.0 * WW[2] * Tup;
      gs[pidx(s, 7, i, j)] = -gs[pidx(s, 5, i, j)] + 2.0 * WW[5] * Tup;
      gs[pidx(s, 8, i, j)] = -gs[pidx(s, 6, i, j)] + 2.0 * WW[6] * Tup;
    }
    for (int i = 0; i < nx; i++) {
      int j = 0;
      gs[pidx(s, 2, i, j)] = -gs[pidx(s, 4, i, j)] + 2.0 * WW[4] * Tdown;
      gs[pidx(s, 5, i, j)] = -gs[pidx(s, 7, i, j)] + 2.0 * WW[7] * Tdown;
      gs[pidx(s, 6, i, j)] = -gs[pidx(s, 8, i, j)] + 2.0 * WW[8] * Tdown;
    }
  }
}

/* ------------------------------------------------- reference box nudging */
static void box_add(orc_t *s, int i, int j, double T) {
  /* reference node (i,j), 1-based; running mean of tempreadint (N:1580) */
  size_t q = sidx(s, i - 1, j - 1);
  double *tri = s->fld[ORC_TEMPREADINT];
  int nv = s->nudge_vol[q];
  tri[q] = (tri[q] * (double)nv + T) / ((double)nv + 1.0);
  s->nudge_vol[q] = nv + 1;
}

/* 7x7 box scatter around round(x), round(y), single domain (NPX=NPY=1
 * semantics of tempvel_nudge.c:1568-1616 / 1641-1686 / 1734-1779). */
static void box_scatter(orc_t *s) {
  const int nx = s->p.nx, ny = s->p.ny;
  memset(s->nudge_vol, 0, sizeof(int) * (size_t)nx * ny);
  memset(s->fld[ORC_TEMPREADINT], 0, sizeof(double) * (size_t)nx * ny);
  for (int k = 0; k < s->np; k++) {
    int x_now = s->xidx[k], y_now = s->yidx[k];
    for (int i1 = -3; i1 < 4; i1++)
      for (int j1 = -3; j1 < 4; j1++) {
        int i = x_now + i1, j = y_now + j1;
        if (i > 0 && i <= nx && j > 0 && j <= ny) box_add(s, i, j, s->Tint[k]);
      }
    if (s->xidx[k] < 4) {
      int tmp = nx + x_now;
      for (int i1 = -3; i1 < 1; i1++)
        for (int j1 = -3; j1 < 4; j1++) {
          int i = tmp + i1, j = y_now + j1;
          if (i > 0 && i <= nx && j > 0 && j <= ny) box_add(s, i, j, s->Tint[k]);
        }
    }
    if (s->xidx[k] > nx - 2) {
      int tmp = x_now - nx;
      for (int i1 = 0; i1 < 4; i1++)
        for (int j1 = -3; j1 < 4; j1++) {
          int i = tmp + i1, j = y_now + j1;
          if (i > 0 && i <= nx && j > 0 && j <= ny) box_add(s, i, j, s->Tint[k]);
        }
    }
  }
}

/* read_prtcl, tempvel_nudge.c:1380-1781, with the file contents already
 * loaded by orc_nudge_load (fx, fy, fT, fid). */
static void box_update(orc_t *s, int istep) {
  const int nx = s->p.nx, ny = s->p.ny, N = s->np, nt = s->p.ntempread;
  if (istep % nt == 1) {
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++)
        if (s->fid[j] == s->oid[i]) { s->chk_id[i] = j; break; }
    for (int i = 0; i < N; i++) {
      s->bc_chky[i] = 0;
      double xread = s->fx[s->chk_id[i]];
      double yread = s->fy[s->chk_id[i]];
      s->dxs[i] = (xread - s->xint[i]) / ((double)nt);
      if (abs((int)(xread - s->xint[i])) > ((double)nx / 2.0)) {
        if (xread > s->xint[i]) {
          xread = xread - (double)nx;
          s->dxs[i] = (xread - s->xint[i]) / ((double)nt);
        } else {
          xread = xread + (double)nx;
          s->dxs[i] = (xread - s->xint[i]) / ((double)nt);
        }
      }
      double xposnow = s->xint[i] + s->dxs[i];
      if (xposnow > (double)nx) xposnow = xposnow - (double)nx;
      if (xposnow < 0.0) xposnow = xposnow + (double)nx;
      s->xint[i] = xposnow;
      s->dys[i] = (yread - s->yint[i]) / ((double)nt);
      if (abs((int)(yread - s->yint[i])) > ((double)ny / 2.0)) {
        s->bc_chky[i] = 1;
        if (yread > s->yint[i]) {
          yread = yread - (double)ny + 1.0;
          s->dys[i] = (yread - s->yint[i]) / ((double)nt);
        } else {
          yread = yread + (double)ny - 1.0;
          s->dys[i] = (yread - s->yint[i]) / ((double)nt);
        }
      }
      double yposnow = s->yint[i] + s->dys[i];
      if (yposnow > (double)ny) { yposnow = yposnow - (double)ny + 1.0; s->bc_chky[i] = 2; }
      if (yposnow < 1.0) { yposnow = yposnow + (double)ny - 1.0; s->bc_chky[i] = 2; }
      s->yint[i] = yposnow;
      s->xidx[i] = (int)round(xposnow);
      s->yidx[i] = (int)round(yposnow);
      double Tread = s->fT[s->chk_id[i]];
      s->dTs[i] = (Tread - s->Tint[i]) / ((double)nt);
      double Tnow = s->Tint[i] + s->dTs[i];
      if (s->bc_chky[i] == 1) Tnow = s->Tint[i];
      if (s->bc_chky[i] == 2) { Tnow = s->fT[s->chk_id[i]]; s->bc_chky[i] = 1; }
      s->Tint[i] = Tnow;
    }
    box_scatter(s);
    for (int k = 0; k < N; k++) { s->ox[k] = s->fx[k]; s->oy[k] = s->fy[k]; s->oT[k] = s->fT[k]; }
  } else if (istep % nt == 0) {
    for (int i = 0; i < N; i++) {
      s->xint[i] = s->ox[s->chk_id[i]];
      s->yint[i] = s->oy[s->chk_id[i]];
      s->Tint[i] = s->oT[s->chk_id[i]];
      s->xidx[i] = (int)round(s->ox[s->chk_id[i]]);
      s->yidx[i] = (int)round(s->oy[s->chk_id[i]]);
    }
    box_scatter(s);
  } else {
    for (int i = 0; i < N; i++) {
      double xposnow = s->xint[i] + s->dxs[i];
      if (xposnow > (double)nx) xposnow = xposnow - (double)nx;
      if (xposnow < 0.0) xposnow = xposnow + (double)nx;
      s->xint[i] = xposnow;
      double yposnow = s->yint[i] + s->dys[i];
      if (yposnow > (double)ny) { yposnow = yposnow - (double)ny + 1.0; s->bc_chky[i] = 2; }
      if (yposnow < 1.0) { yposnow = yposnow + (double)ny - 1.0; s->bc_chky[i] = 2; }
      s->yint[i] = yposnow;
      s->xidx[i] = (int)round(xposnow);
      s->yidx[i] = (int)round(yposnow);
      double Tnow = s->Tint[i] + s->dTs[i];
      if (s->bc_chky[i] == 1) Tnow = s->Tint[i];
      if (s->bc_chky[i] == 2) { Tnow = s->oT[s->chk_id[i]]; s->bc_chky[i] = 1; }
      s->Tint[i] = Tnow;
    }
    box_scatter(s);
  }
}

void orc_nudge_init(orc_t *s, const double *x, const double *y, const double *T, const int *id) {
  /* set_nudge_vol, contin==0 (tempvel_nudge.c:2114-2122); nud_term = 0 */
  for (int i = 0; i < s->np; i++) {
    s->ox[i] = x[i]; s->oy[i] = y[i]; s->oT[i] = T[i]; s->oid[i] = id[i];
    s->xint[i] = x[i]; s->yint[i] = y[i]; s->Tint[i] = T[i];
    s->chk_id[i] = 0; s->bc_chky[i] = 0;
  }
  memset(s->fld[ORC_NUDTERM], 0, sizeof(double) * (size_t)s->p.nx * s->p.ny);
}

void orc_nudge_load(orc_t *s, const double *x, const double *y, const int *id, const double *T) {
  for (int i = 0; i < s->np; i++) { s->fx[i] = x[i]; s->fy[i] = y[i]; s->fid[i] = id[i]; s->fT[i] = T[i]; }
}

void orc_nudge_obs(orc_t *s, int nobs, const double *x, const double *y, const double *T) {
  free(s->bx); free(s->by); free(s->bT);
  s->nobs = nobs;
  s->bx = (double *)malloc(sizeof(double) * (nobs > 0 ? nobs : 1));
  s->by = (double *)malloc(sizeof(double) * (nobs > 0 ? nobs : 1));
  s->bT = (double *)malloc(sizeof(double) * (nobs > 0 ? nobs : 1));
  for (int p = 0; p < nobs; p++) { s->bx[p] = x[p]; s->by[p] = y[p]; s->bT[p] = T[p]; }
}

/* Bilinear nudging (no counterpart in the reference): the innovation
 * d = alpha*(T_obs - T(x_p)) is spread to the 4 cell corners with the
 * bilinear weights, accumulated in 2^-40 fixed point so that the sum does
 * not depend on the order of the contributions, and added to the
 * post-collision g as w_k * S. */
#define NUDGE_FIX_SCALE 1099511627776.0 /* 2^40 */
static void bilinear_nudge(orc_t *s) {
  const int nx = s->p.nx, ny = s->p.ny;
  const double *T = s->fld[ORC_T];
  double *src = s->fld[ORC_NUDGE_SRC];
  memset(s->acc, 0, sizeof(int64_t) * (size_t)nx * ny);
  for (int p = 0; p < s->nobs; p++) {
    double xx = s->bx[p], yy = s->by[p];
    double tm = bilinear(s, T, xx, yy);
    double dlt = s->p.alpha * (s->bT[p] - tm);
    int x1 = (int)xx, y1 = (int)yy;
    int x2 = x1 + 1, y2 = y1 + 1;
    double wx1 = (double)x2 - xx, wx2 = xx - (double)x1;
    double wy1 = (double)y2 - yy, wy2 = yy - (double)y1;
    int ix1 = wrap(x1 - 1, nx), ix2 = wrap(x2 - 1, nx);
    int jy1 = wrap(y1 - 1, ny), jy2 = wrap(y2 - 1, ny);
    s->acc[(size_t)jy1 * nx + ix1] += llrint(dlt * (wx1 * wy1) * NUDGE_FIX_SCALE);
    s->acc[(size_t)jy1 * nx + ix2] += llrint(dlt * (wx2 * wy1) * NUDGE_FIX_SCALE);
    s->acc[(size_t)jy2 * nx + ix1] += llrint(dlt * (wx1 * wy2) * NUDGE_FIX_SCALE);
    s->acc[(size_t)jy2 * nx + ix2] += llrint(dlt * (wx2 * wy2) * NUDGE_FIX_SCALE);
  }
  double *g = s->fld[ORC_G];
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      size_t q = sidx(s, i, j);
      double sv = (double)s->acc[q] * (1.0 / NUDGE_FIX_SCALE);
      src[q] = sv;
      if (s->acc[q] != 0)
        for (int k = 0; k < NPOP; k++) g[pidx(s, k, i, j)] = g[pidx(s, k, i, j)] + WW[k] * sv;
    }
}

/* ------------------------------------------------------------- particles */
/* derivative fields of the Maxey-Riley update (mympi2.h:374-411): central
 * differences, one-sided at the wall rows, periodic halos afterwards */
static void deriv_fields(orc_t *s) {
  const int nx = s->p.nx, ny = s->p.ny;
  const double *u = s->fld[ORC_U], *v = s->fld[ORC_V];
  const double *ub = s->fld[ORC_UBEF], *vb = s->fld[ORC_VBEF];
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      size_t q = sidx(s, i, j);
      size_t qr = sidx(s, wrap(i + 1, nx), j), ql = sidx(s, wrap(i - 1, nx), j);
      size_t qt = sidx(s, i, wrap(j + 1, ny)), qb = sidx(s, i, wrap(j - 1, ny));
      s->d[0][q] = u[q] - ub[q];
      s->d[1][q] = v[q] - vb[q];
      s->d[2][q] = (u[qr] - u[ql]) * 0.5;
      s->d[3][q] = (v[qr] - v[ql]) * 0.5;
      if (j == 0) {
        s->d[4][q] = (u[qt] - u[q]);
        s->d[5][q] = (v[qt] - v[q]);
      } else if (j == ny - 1) {
        s->d[4][q] = (u[q] - u[qb]);
        s->d[5][q] = (v[q] - v[qb]);
      } else {
        s->d[4][q] = (u[qt] - u[qb]) * 0.5;
        s->d[5][q] = (v[qt] - v[qb]) * 0.5;
      }
    }
}

static void particles(orc_t *s, int istep) {
  const double delta_t = 1.0;
  const double beta = s->p.beta;
  const double *u = s->fld[ORC_U], *v = s->fld[ORC_V], *T = s->fld[ORC_T];
  int need_d = s->p.record_full && s->p.noutconfig > 0 && istep % s->p.noutconfig == 0;
  for (int q = 0; q < s->np && !need_d; q++) need_d = (s->ptype[q] == ORC_PTYPE_INERTIAL);
  if (need_d) deriv_fields(s);
  double *px = s->pa[ORC_PX], *py = s->pa[ORC_PY], *pu = s->pa[ORC_PU], *pv = s->pa[ORC_PV];
  double *pxo = s->pa[ORC_PXO], *pyo = s->pa[ORC_PYO], *puo = s->pa[ORC_PUO], *pvo = s->pa[ORC_PVO];
  const double *pinv = s->pa[ORC_PINVTAU];
  for (int i = 0; i < s->np; i++) {
    double xx = px[i], yy = py[i];
    puo[i] = pu[i];
    pvo[i] = pv[i];
    double tempup = bilinear(s, u, xx, yy);
    double tempvp = bilinear(s, v, xx, yy);
    pxo[i] = xx;
    pyo[i] = yy;
    if (s->ptype[i] == ORC_PTYPE_TRACER) {
      /* Adams-Bashforth 2, mympi2.h:358-372 */
      px[i] = xx + 1.5 * delta_t * tempup - 0.5 * delta_t * puo[i];
      py[i] = yy + 1.5 * delta_t * tempvp - 0.5 * delta_t * pvo[i];
      pu[i] = tempup;
      pv[i] = tempvp;
    } else {
      /* Maxey-Riley explicit Euler, mympi2.h:413-432 */
      double tdtu = bilinear(s, s->d[0], xx, yy), tdtv = bilinear(s, s->d[1], xx, yy);
      double tdxu = bilinear(s, s->d[2], xx, yy), tdxv = bilinear(s, s->d[3], xx, yy);
      double tdyu = bilinear(s, s->d[4], xx, yy), tdyv = bilinear(s, s->d[5], xx, yy);
      double inv = pinv[i];
      pu[i] = pu[i] + delta_t * (beta * (tdtu + tempup * tdxu + tempvp * tdyu) - inv * (pu[i] - tempup));
      pv[i] = pv[i] + delta_t * (beta * (tdtv + tempup * tdxv + tempvp * tdyv) - inv * (pv[i] - tempvp));
      px[i] = xx + delta_t * pu[i];
      py[i] = yy + delta_t * pv[i];
    }
  }
  if (s->p.noutconfig > 0 && istep % s->p.noutconfig == 0) {
    /* prtcl_write (temppart_dump.c:1467-1571): T at the pre-toggle position */
    const int N = s->np;
    double *r = s->rec;
    for (int i = 0; i < N; i++) {
      r[ORC_R_X * N + i] = 0.0 + px[i];
      r[ORC_R_Y * N + i] = 0.0 + py[i];
      r[ORC_R_U * N + i] = pu[i];
      r[ORC_R_V * N + i] = pv[i];
      r[ORC_R_XO * N + i] = 0.0 + pxo[i];
      r[ORC_R_YO * N + i] = 0.0 + pyo[i];
      r[ORC_R_UO * N + i] = puo[i];
      r[ORC_R_VO * N + i] = pvo[i];
      r[ORC_R_TEMP * N + i] = bilinear(s, T, px[i], py[i]);
      if (s->p.record_full) {
        /* Prtcl_Writefull block, mympi2.h:484-503, evaluated at (xo,yo) */
        double xo = pxo[i], yo = pyo[i];
        r[ORC_R_FU * N + i] = bilinear(s, u, xo, yo);
        r[ORC_R_FV * N + i] = bilinear(s, v, xo, yo);
        r[ORC_R_DTU * N + i] = bilinear(s, s->d[0], xo, yo);
        r[ORC_R_DTV * N + i] = bilinear(s, s->d[1], xo, yo);
        r[ORC_R_DXU * N + i] = bilinear(s, s->d[2], xo, yo);
        r[ORC_R_DXV * N + i] = bilinear(s, s->d[3], xo, yo);
        r[ORC_R_DYU * N + i] = bilinear(s, s->d[4], xo, yo);
        r[ORC_R_DYV * N + i] = bilinear(s, s->d[5], xo, yo);
      }
    }
    s->rec_step = istep;
  }
  /* toggle_prtcl wrap/reflect, mympi2.h:589-635 and 681-723 (one domain) */
  const double NXd = (double)s->p.nx, NYd = (double)s->p.ny;
  for (int i = 0; i < s->np; i++) {
    if (px[i] >= NXd) px[i] = px[i] - NXd;
    else if (px[i] <= 0.0) px[i] = px[i] + NXd;
    if (py[i] < 1.0) {
      py[i] = py[i] + 2.0 * (1.0 - py[i]);
      pv[i] = -pv[i];
    } else if (py[i] >= NYd) {
      py[i] = py[i] + 2.0 * (NYd - py[i]);
      pv[i] = -pv[i];
    }
  }
}

/* -------------------------------------------------------------------- step */
void orc_step(orc_t *s, int istep) {
  const int nx = s->p.nx, ny = s->p.ny;
  const size_t n = (size_t)nx * ny;
  double *rho = s->fld[ORC_RHO], *u = s->fld[ORC_U], *v = s->fld[ORC_V], *T = s->fld[ORC_T];
  double *Fy = s->fld[ORC_FY];
  const int refbox = (s->p.nudge == ORC_NUDGE_REFBOX);

  if (refbox) box_update(s, istep);
  stream(s);
  /* forcingconstructWW: previous step's rho and T (temppart_dump.c:744-755) */
  for (size_t q = 0; q < n; q++) Fy[q] = -s->p.gravity * rho[q] * (T[q] - 0.0);
  /* mirror: keep u^{n-1} for the Maxey-Riley time derivative */
  memcpy(s->fld[ORC_UBEF], u, n * sizeof(double));
  memcpy(s->fld[ORC_VBEF], v, n * sizeof(double));
  /* hydrovar (temppart_dump.c:957-987 / tempvel_nudge.c:1069-1102) */
  const double *fs = s->fs, *gs = s->gs;
  const double *nud = s->fld[ORC_NUDTERM];
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      size_t q = sidx(s, i, j);
      double fl[NPOP];
      double r = 0.0, t = 0.0;
      for (int k = 0; k < NPOP; k++) r = r + fs[pidx(s, k, i, j)];
      for (int k = 0; k < NPOP; k++) t = t + gs[pidx(s, k, i, j)];
      s->fld[ORC_TSUM][q] = t;
      if (refbox && s->nudge_vol[q] > 0) t = (t + 0.5 * nud[q]);
      rho[q] = r;
      T[q] = t;
      double rhoi = 1. / r;
      for (int k = 0; k < NPOP; k++) fl[k] = fs[pidx(s, k, i, j)] * rhoi;
      const double Fx = 0.0;
      u[q] = fl[1] - fl[3] + fl[5] - fl[6] - fl[7] + fl[8] + 0.5 * rhoi * Fx;
      v[q] = fl[5] + fl[2] + fl[6] - fl[7] - fl[4] - fl[8] + 0.5 * rhoi * Fy[q];
    }
  if (s->np > 0) particles(s, istep);
  /* collision (computetau/equilif/collisf/equilig/collisg), reference loop
   * order i-major, j-minor (matters only for the carried Q of collisg) */
  const double omega = 1. / s->p.relax;
  const double omegag = 1. / s->p.relaxg;
  double *f = s->fld[ORC_F], *g = s->fld[ORC_G];
  double *tri = s->fld[ORC_TEMPREADINT], *nudt = s->fld[ORC_NUDTERM];
  double Q = 0.0;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) {
      size_t q = sidx(s, i, j);
      double feq[NPOP], geq[NPOP];
      equil(rho[q], u[q], v[q], feq);
      const double Fx = 0.0, Fyq = Fy[q];
      for (int k = 0; k < NPOP; k++) {
        double source = (1.0 - 0.5 * omega) * WW[k];
        double factor = ((CX[k] - u[q]) * Fx + (CY[k] - v[q]) * Fyq) / CS2;
        factor = factor + ((CX[k] * u[q] + CY[k] * v[q]) * (CX[k] * Fx + CY[k] * Fyq)) / (CS2 * CS2);
        f[pidx(s, k, i, j)] = fs[pidx(s, k, i, j)] * (1. - omega) + omega * feq[k] + source * factor;
      }
      equil(T[q], u[q], v[q], geq);
      if (refbox && s->nudge_vol[q] > 0) {
        double B = 1.0 - 0.5 * omegag;
        Q = s->p.alpha * (T[q] - tri[q]);
        for (int k = 0; k < NPOP; k++)
          g[pidx(s, k, i, j)] = gs[pidx(s, k, i, j)] * (1. - omegag) + omegag * geq[k] - B * WW[k] * Q;
        nudt[q] = -1. * Q;
      } else {
        double B = 0.0;
        for (int k = 0; k < NPOP; k++)
          g[pidx(s, k, i, j)] = gs[pidx(s, k, i, j)] * (1. - omegag) + omegag * geq[k] + B * WW[k] * Q;
      }
    }
  if (s->p.nudge == ORC_NUDGE_BILINEAR) bilinear_nudge(s);
}

/* ------------------------------------------------------------ initial state */
void orc_moments_from_pre(orc_t *s, const double *fpre, const double *gpre) {
  const int nx = s->p.nx, ny = s->p.ny;
  double *rho = s->fld[ORC_RHO], *u = s->fld[ORC_U], *v = s->fld[ORC_V], *T = s->fld[ORC_T];
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      size_t q = sidx(s, i, j);
      double r = 0.0, t = 0.0, fl[NPOP];
      for (int k = 0; k < NPOP; k++) r = r + fpre[pidx(s, k, i, j)];
      for (int k = 0; k < NPOP; k++) t = t + gpre[pidx(s, k, i, j)];
      double rhoi = 1. / r;
      for (int k = 0; k < NPOP; k++) fl[k] = fpre[pidx(s, k, i, j)] * rhoi;
      rho[q] = r;
      T[q] = t;
      u[q] = fl[1] - fl[3] + fl[5] - fl[6] - fl[7] + fl[8];
      v[q] = fl[5] + fl[2] + fl[6] - fl[7] - fl[4] - fl[8] + (0.5 * (-s->p.gravity) * t);
    }
}

static uint64_t splitmix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* uniform double in [0,1) from (seed, index): splitmix64 of
 * seed + (index+1)*golden, top 53 bits */
double orc_splitmix_uniform(unsigned long long seed, unsigned long long index) {
  uint64_t z = splitmix64((uint64_t)seed + ((uint64_t)index + 1ULL) * 0x9E3779B97F4A7C15ULL);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

void orc_init_conduction(orc_t *s, unsigned long long seed, double noise_amp) {
  const int nx = s->p.nx, ny = s->p.ny;
  double *f = s->fld[ORC_F], *g = s->fld[ORC_G];
  const double dT = s->p.Tup - s->p.Tdown;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      size_t q = sidx(s, i, j);
      double un = orc_splitmix_uniform(seed, q);
      double t = s->p.Tdown + dT * (((double)j + 0.5) / (double)ny) + noise_amp * (2.0 * un - 1.0);
      double feq[NPOP], geq[NPOP];
      equil(1.0, 0.0, 0.0, feq);
      equil(t, 0.0, 0.0, geq);
      for (int k = 0; k < NPOP; k++) {
        f[pidx(s, k, i, j)] = feq[k];
        g[pidx(s, k, i, j)] = geq[k];
      }
    }
  orc_moments_from_pre(s, f, g);
}

/* ------------------------------------------------------------- diagnostics */
void orc_energy(orc_t *s, double *ke_mean, double *t_mean) {
  const int nx = s->p.nx, ny = s->p.ny;
  const double *rho = s->fld[ORC_RHO], *u = s->fld[ORC_U], *v = s->fld[ORC_V], *T = s->fld[ORC_T];
  double te = 0.0, tt = 0.0;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) {
      size_t q = sidx(s, i, j);
      te += 0.5 * rho[q] * (u[q] * u[q] + v[q] * v[q]);
      tt += T[q];
    }
  te /= (((double)nx) * ((double)ny));
  tt /= (((double)nx) * ((double)ny));
  if (ke_mean) *ke_mean = te;
  if (t_mean) *t_mean = tt;
}

/* per-row averages (tempvel_nudge.c profile(), :1186-1232): columns
 * rho, u, v, u^2, v^2, T, vT, dT/dy (T(j+1)-T(j)), each scaled by 1/nx;
 * plus column 8 = row Nusselt (vT - kappa dT/dy) / (kappa dT_walls / ny).
 * At the last row of each of the reference's `ranks_y` ranks in y, T(j+1)
 * is the halo row: hydrovar (tempvel_nudge.c:1069-1102) forms it from the
 * halo populations that pbc copied from the next rank's first row (periodic
 * at the top), and the halo's nudge_vol is 0, so it is that row's sum of g
 * without box nudging's 1/2 nud_term. */
void orc_profile(orc_t *s, double *out) { orc_profile_ranks(s, 1, out); }

void orc_profile_ranks(orc_t *s, int ranks_y, double *out) {
  const int nx = s->p.nx, ny = s->p.ny;
  const double *rho = s->fld[ORC_RHO], *u = s->fld[ORC_U], *v = s->fld[ORC_V], *T = s->fld[ORC_T];
  const double *Thalo = s->p.nudge == ORC_NUDGE_REFBOX ? s->fld[ORC_TSUM] : T;
  const double kappa = (s->p.relaxg - 0.5) / 3.0;
  const double dTw = s->p.Tdown - s->p.Tup;
  const int NYr = ny / (ranks_y > 0 ? ranks_y : 1);
  for (int j = 0; j < ny; j++) {
    double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const double *Tup_row = ((j + 1) % NYr == 0) ? Thalo : T;
    for (int i = 0; i < nx; i++) {
      size_t q = sidx(s, i, j), qt = sidx(s, i, wrap(j + 1, ny));
      a[0] += rho[q]; a[1] += u[q]; a[2] += v[q];
      a[3] += u[q] * u[q]; a[4] += v[q] * v[q]; a[5] += T[q];
      a[6] += v[q] * T[q]; a[7] += Tup_row[qt] - T[q];
    }
    const double norma = 1 / ((double)nx); /* the reference scales by 1/nx (:1225-1229) */
    for (int c = 0; c < 8; c++) out[(size_t)j * 9 + c] = a[c] * norma;
    out[(size_t)j * 9 + 8] = (out[(size_t)j * 9 + 6] - kappa * out[(size_t)j * 9 + 7]) / (kappa * dTw / (double)ny);
  }
}

/* volume Nusselt number 1 + <vT> H / (kappa dT), H = ny (half-way walls) */
double orc_nusselt(orc_t *s) {
  const int nx = s->p.nx, ny = s->p.ny;
  const double *v = s->fld[ORC_V], *T = s->fld[ORC_T];
  const double kappa = (s->p.relaxg - 0.5) / 3.0;
  const double dTw = s->p.Tdown - s->p.Tup;
  double sum = 0.0, c = 0.0;
  for (size_t q = 0; q < (size_t)nx * ny; q++) {
    double y = v[q] * T[q] - c;
    double t = sum + y;
    c = (t - sum) - y;
    sum = t;
  }
  double mean = sum / ((double)nx * (double)ny);
  return 1.0 + mean * (double)ny / (kappa * dTw);
}

/* ------------------------------------------------- tangent-linear model */
/* Tangent of one step, applied after orc_step() computed the values: the
 * post-stream values fs, gs, the buoyancy Fy used and the moments are in
 * the state.  Tangents: tf, tg (post-collision, 9 planes each), tF (the
 * buoyancy of the next step); updated in place through the scratch tfs/tgs.
 * Differentiates the shifted-form mathematics of the step (see the CUDA
 * adjoint for the formulas); the pull moves tangents like values, and the
 * anti-bounce-back drops its constant. */
static void tlm_step(orc_t *s, double *tf, double *tg, double *tF, double *tfs, double *tgs,
                     double *tT) {
  const int nx = s->p.nx, ny = s->p.ny;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
      for (int k = 0; k < NPOP; k++) {
        int js = j - ICY[k], is = wrap(i - ICX[k], nx);
        tfs[pidx(s, k, i, j)] = (js < 0 || js >= ny) ? tf[pidx(s, OPP[k], i, j)] : tf[pidx(s, k, is, js)];
        tgs[pidx(s, k, i, j)] = (js < 0 || js >= ny) ? 0.0 : tg[pidx(s, k, is, js)];
      }
  for (int i = 0; i < nx; i++) {
    int j = ny - 1;
    tgs[pidx(s, 4, i, j)] = -tgs[pidx(s, 2, i, j)];
    tgs[pidx(s, 7, i, j)] = -tgs[pidx(s, 5, i, j)];
    tgs[pidx(s, 8, i, j)] = -tgs[pidx(s, 6, i, j)];
    j = 0;
    tgs[pidx(s, 2, i, j)] = -tgs[pidx(s, 4, i, j)];
    tgs[pidx(s, 5, i, j)] = -tgs[pidx(s, 7, i, j)];
    tgs[pidx(s, 6, i, j)] = -tgs[pidx(s, 8, i, j)];
  }
  const double om = 1. / s->p.relax, omg = 1. / s->p.relaxg, srcf = 1.0 - 0.5 * om;
  const double gb = -s->p.gravity;
  const double *rho = s->fld[ORC_RHO], *u = s->fld[ORC_U], *v = s->fld[ORC_V], *T = s->fld[ORC_T];
  const double *Fy = s->fld[ORC_FY];
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      size_t q = sidx(s, i, j);
      double r = rho[q], uu = u[q], vv = v[q], t = T[q], F = Fy[q];
      double rd = 0, jxd = 0, jyd = 0, td = 0;
      for (int k = 0; k < NPOP; k++) {
        double a = tfs[pidx(s, k, i, j)];
        rd += a;
        jxd += ICX[k] * a;
        jyd += ICY[k] * a;
        td += tgs[pidx(s, k, i, j)];
      }
      double Fd = tF[q];
      double ud = (jxd - uu * rd) / r, vd = (jyd + 0.5 * Fd - vv * rd) / r;
      for (int k = 0; k < NPOP; k++) {
        double w = WW[k], cx = ICX[k], cy = ICY[k];
        double cu = cx * uu + cy * vv, cud = cx * ud + cy * vd;
        double P = 3.0 * cu + 4.5 * cu * cu - 1.5 * (uu * uu + vv * vv);
        double Pd = (3.0 + 9.0 * cu) * cud - 3.0 * (uu * ud + vv * vd);
        double feqd = w * (rd + rd * P + r * Pd);
        double Sd = srcf * w * (Fd * (3.0 * (cy - vv) + 9.0 * cu * cy) + F * (-3.0 * vd + 9.0 * cud * cy));
        tf[pidx(s, k, i, j)] = (1.0 - om) * tfs[pidx(s, k, i, j)] + om * feqd + Sd;
        double geqd = w * (td + td * P + t * Pd);
        tg[pidx(s, k, i, j)] = (1.0 - omg) * tgs[pidx(s, k, i, j)] + omg * geqd;
      }
      tF[q] = gb * (rd * t + r * td);
      tT[q] = td;
    }
}

void orc_tlm_window(orc_t *s, const double *T0, const double *dT0, int nsteps, int nobs_steps,
                    const int *steps, int nobs, const double *ox, const double *oy,
                    const double *oT, double *J, double *dJ) {
  const int nx = s->p.nx, ny = s->p.ny;
  const size_t n = (size_t)nx * ny;
  double *f = s->fld[ORC_F], *g = s->fld[ORC_G];
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      double feq[NPOP], geq[NPOP];
      equil(1.0, 0.0, 0.0, feq);
      equil(T0[sidx(s, i, j)], 0.0, 0.0, geq);
      for (int k = 0; k < NPOP; k++) {
        f[pidx(s, k, i, j)] = feq[k];
        g[pidx(s, k, i, j)] = geq[k];
      }
    }
  orc_moments_from_pre(s, f, g);
  double *tf = (double *)calloc(NPOP * n, sizeof(double)), *tg = (double *)calloc(NPOP * n, sizeof(double));
  double *tfs = (double *)calloc(NPOP * n, sizeof(double)), *tgs = (double *)calloc(NPOP * n, sizeof(double));
  double *tF = (double *)calloc(n, sizeof(double)), *tT = (double *)calloc(n, sizeof(double));
  double sw = 0.0;
  for (int k = 0; k < NPOP; k++) sw += WW[k];
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      size_t q = sidx(s, i, j);
      for (int k = 0; k < NPOP; k++) tg[pidx(s, k, i, j)] = WW[k] * dT0[q];
      tF[q] = -s->p.gravity * s->fld[ORC_RHO][q] * sw * dT0[q];
    }
  double Js = 0.0, dJs = 0.0;
  int a = 0;
  for (int st = 1; st <= nsteps; st++) {
    orc_step(s, st);
    tlm_step(s, tf, tg, tF, tfs, tgs, tT);
    while (a < nobs_steps && steps[a] < st) a++;
    if (a < nobs_steps && steps[a] == st) {
      for (int p = 0; p < nobs; p++) {
        size_t o = (size_t)a * nobs + p;
        double r = bilinear(s, s->fld[ORC_T], ox[o], oy[o]) - oT[o];
        Js += r * r;
        dJs += 2.0 * r * bilinear(s, tT, ox[o], oy[o]);
      }
    }
  }
  *J = Js;
  *dJ = dJs;
  free(tf); free(tg); free(tfs); free(tgs); free(tF); free(tT);
}
