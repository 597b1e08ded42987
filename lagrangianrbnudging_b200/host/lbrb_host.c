/*
 * lbrb_host.c -- host program for the B200 step loop, a drop-in for the
 * reference's two main() programs:
 *
 *   lbrb_host trajectories [name=value ...]   (Trajectories/code/temppart_dump.c:1573-1769)
 *   lbrb_host nudging      [name=value ...]   (Nudging/code/tempvel_nudge.c:2254-2419)
 *
 * Parameters keep the reference's #define names (temppart_dump.c:15-31,
 * Trajectories/code/mympi2.h:14-21, tempvel_nudge.c:13-31) and defaults;
 * here they are read at run time.  Extra names: precision=fp64|fp32,
 * Ra/Pr/U (closure: relax = 3 nu + 1/2, relaxg = 3 kappa + 1/2,
 * gravity = -U^2/ny, Tup/Tdown = -/+ 1/2), ic=conduction with seed/noise,
 * prtcl=uniform with seed, device, dir (working directory).
 *
 * Input and output files follow the reference's names and dataset layouts:
 *   restart   conf.h5:/f cong.h5:/g confpre.h5:/f congpre.h5:/g  [nx][ny][9]
 *             (restoref..restoregpre, temppart_dump.c:348-668)
 *   particles Prtcl_Veldata1/Particles<nstart>.h5:/id + prtcl_dump<nstart>.in
 *             (restore_prtcl, temppart_dump.c:252-346)
 *   records   Prtcl_Veldata1/Particles<istep>.h5: /id /x /y /u /v /xo /yo /uo
 *             /vo /temp (+ /dtu /dtv /dxu /dxv /dyu /dyv /fu /fv with
 *             Prtcl_Writefull) (temppart_dump.c:1545-1562, mympi2.h:549-556)
 *   dumps     confnew/congnew<istep>.h5 (post-collision), confpre/congpre
 *             (post-stream, last step) [nx][ny][9]; prtcl_dump<istep>.in
 *   fields    Tempfolder/snaptemp<istep>.h5: /T /u /v [nx][ny]
 *   text      evolution.dat "istep KE T"; profiles.<istep>.dat
 *   nudging   obs/init_prtcl{x,y,T,_id}0.in, obs/Prtcl_Veldata1/Particles<k>.h5
 * HDF5 is not part of this build: a dataset "/x" of file NAME.h5 is the raw
 * little-endian file NAME.h5.d/x.bin in C order (the layout of the reference
 * built against this repository's HDF5 stand-in).
 *
 * Records hold the particles in id order (the reference writes them in its
 * ranks' local order, which changes as particles migrate; the /id dataset
 * identifies them in both).
 */
#define _GNU_SOURCE
#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <nvtx3/nvToolsExt.h>

#include "../../include/lbrb.h"

#define NPOP 9

typedef struct {
  int program;  /* 0 trajectories, 1 nudging */
  int nx, ny, scratch, nstart, nsteps, nout, noutconfig;
  double relax, relaxg, Tup, Tdown, gravity;
  int Particle, Particle_scratch, Nprtcl, tracer, heavyprtcl, Prtcl_Writefull;
  double taulag, beta;
  double alpha;
  int contin, ntempread;
  int precision, device;
  int ic_conduction;
  unsigned long long seed;
  double noise;
  int prtcl_uniform;
  char dir[1024];
} cfg_t;

static const double WW[NPOP] = {16. / 36., 4. / 36., 4. / 36., 4. / 36., 4. / 36.,
                                1. / 36.,  1. / 36., 1. / 36., 1. / 36.};

static void die(const char *msg, lbrb_t *h) {
  fprintf(stderr, "lbrb_host: %s%s%s\n", msg, h ? ": " : "", h ? lbrb_last_error(h) : "");
  exit(8);
}

#define CALL(h, x)                              \
  do {                                          \
    int rc_ = (x);                              \
    if (rc_ != LBRB_OK) die(#x, (h));           \
  } while (0)

/* ------------------------------------------------------------- parameters */
static void defaults(cfg_t *c, int program) {
  memset(c, 0, sizeof(*c));
  c->program = program;
  /* temppart_dump.c:16-28 / tempvel_nudge.c:15-29 */
  c->nx = 1680;
  c->ny = 840;
  c->scratch = program ? 1 : 0;
  c->nstart = 0;
  c->nsteps = program ? 3000000 : 5000000;
  c->nout = 20000;
  c->noutconfig = program ? 20000 : 250;
  c->relax = 0.502;
  c->relaxg = 0.502;
  c->Tup = -0.01;
  c->Tdown = 0.01;
  c->gravity = -0.00004;
  c->Particle = 1;
  c->Particle_scratch = 1;
  /* Trajectories/code/mympi2.h:14-21, Nudging/code/mympi2.h:15 */
  c->Nprtcl = 1600;
  c->tracer = 0;
  c->heavyprtcl = 1;
  c->taulag = 2150.0;
  c->beta = 0.1;
  c->Prtcl_Writefull = 1;
  c->alpha = 0.01; /* tempvel_nudge.c:13 */
  c->contin = 0;
  c->ntempread = 250;
  c->precision = LBRB_PREC_FP64;
  c->device = 0;
  c->seed = 1;
  c->noise = 1e-3;
  strcpy(c->dir, ".");
}

static int set_param(cfg_t *c, const char *k, const char *v, double *Ra, double *Pr, double *U) {
#define IP(name) if (!strcmp(k, #name)) { c->name = atoi(v); return 1; }
#define DP(name) if (!strcmp(k, #name)) { c->name = atof(v); return 1; }
  IP(nx) IP(ny) IP(scratch) IP(nstart) IP(nsteps) IP(nout) IP(noutconfig)
  DP(relax) DP(relaxg) DP(Tup) DP(Tdown) DP(gravity)
  IP(Particle) IP(Particle_scratch) IP(Nprtcl) IP(tracer) IP(heavyprtcl) IP(Prtcl_Writefull)
  DP(taulag) DP(beta) DP(alpha) IP(contin) IP(ntempread) IP(device) DP(noise)
#undef IP
#undef DP
  if (!strcmp(k, "rhom1")) return atof(v) == 1.0 ? 1 : -1;
  if (!strcmp(k, "precision")) { c->precision = !strcmp(v, "fp32") ? LBRB_PREC_FP32_SHIFTED : LBRB_PREC_FP64; return 1; }
  if (!strcmp(k, "ic")) { c->ic_conduction = !strcmp(v, "conduction"); return 1; }
  if (!strcmp(k, "prtcl")) { c->prtcl_uniform = !strcmp(v, "uniform"); return 1; }
  if (!strcmp(k, "seed")) { c->seed = strtoull(v, NULL, 10); return 1; }
  if (!strcmp(k, "dir")) { snprintf(c->dir, sizeof(c->dir), "%s", v); return 1; }
  if (!strcmp(k, "Ra")) { *Ra = atof(v); return 1; }
  if (!strcmp(k, "Pr")) { *Pr = atof(v); return 1; }
  if (!strcmp(k, "U")) { *U = atof(v); return 1; }
  return 0;
}

/* ---------------------------------------------------------- raw datasets */
static void ensure_dir(const char *d) {
  if (mkdir(d, 0755) != 0 && errno != EEXIST) {
    fprintf(stderr, "lbrb_host: cannot create %s\n", d);
    exit(8);
  }
}

static void write_ds(const char *file, const char *name, const void *data, size_t bytes) {
  char dir[1200], path[1400];
  snprintf(dir, sizeof(dir), "%s.d", file);
  ensure_dir(dir);
  snprintf(path, sizeof(path), "%s/%s.bin", dir, name);
  FILE *f = fopen(path, "wb");
  if (!f || fwrite(data, 1, bytes, f) != bytes) {
    fprintf(stderr, "lbrb_host: cannot write %s\n", path);
    exit(8);
  }
  fclose(f);
}

static int read_ds(const char *file, const char *name, void *data, size_t bytes) {
  char path[1400];
  snprintf(path, sizeof(path), "%s.d/%s.bin", file, name);
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  size_t got = fread(data, 1, bytes, f);
  fclose(f);
  return got == bytes ? 0 : -1;
}

static int read_raw(const char *path, void *data, size_t bytes) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  size_t got = fread(data, 1, bytes, f);
  fclose(f);
  return got == bytes ? 0 : -1;
}

static void write_raw(const char *path, const void *data, size_t bytes) {
  FILE *f = fopen(path, "wb");
  if (!f || fwrite(data, 1, bytes, f) != bytes) {
    fprintf(stderr, "lbrb_host: cannot write %s\n", path);
    exit(8);
  }
  fclose(f);
}

/* reference haloed AoS (idx = j + (ny+2) i) <-> dataset [nx][ny][9] */
static void pops_halo_to_ds(const cfg_t *c, const double *halo, double *ds) {
  for (int i = 1; i <= c->nx; i++)
    for (int j = 1; j <= c->ny; j++)
      memcpy(ds + ((size_t)(i - 1) * c->ny + (j - 1)) * NPOP,
             halo + ((size_t)j + (size_t)(c->ny + 2) * i) * NPOP, NPOP * sizeof(double));
}

static void pops_ds_to_halo(const cfg_t *c, const double *ds, double *halo) {
  memset(halo, 0, sizeof(double) * NPOP * (size_t)(c->nx + 2) * (c->ny + 2));
  for (int i = 1; i <= c->nx; i++)
    for (int j = 1; j <= c->ny; j++)
      memcpy(halo + ((size_t)j + (size_t)(c->ny + 2) * i) * NPOP,
             ds + ((size_t)(i - 1) * c->ny + (j - 1)) * NPOP, NPOP * sizeof(double));
}

static void scalar_halo_to_ds(const cfg_t *c, const double *halo, double *ds) {
  for (int i = 1; i <= c->nx; i++)
    for (int j = 1; j <= c->ny; j++)
      ds[(size_t)(i - 1) * c->ny + (j - 1)] = halo[(size_t)j + (size_t)(c->ny + 2) * i];
}

/* ----------------------------------------------------------- interpolation */
/* bilinear on a haloed field (Trajectories/code/mympi2.h:292-311) */
static double bilinear(const cfg_t *c, const double *u, double xx, double yy) {
  int x1 = (int)xx, x2 = x1 + 1, y1 = (int)yy, y2 = y1 + 1;
  int NY2 = c->ny + 2;
  double u11 = u[y1 + NY2 * x1], u12 = u[y2 + NY2 * x1];
  double u21 = u[y1 + NY2 * x2], u22 = u[y2 + NY2 * x2];
  double val1 = u11 * ((double)x2 - xx) * ((double)y2 - yy);
  double val2 = u21 * (xx - (double)x1) * ((double)y2 - yy);
  double val3 = u12 * ((double)x2 - xx) * (yy - (double)y1);
  double val4 = u22 * (xx - (double)x1) * (yy - (double)y1);
  return val1 + val2 + val3 + val4;
}

/* ------------------------------------------------------------ initial state */
/* the reference's scratch state (inithydro, temppart_dump.c:686-701) for one
 * rank: srand(0), one rand() per haloed node in i-major order */
static void scratch_state(const cfg_t *c, double *f, double *g, double *rho, double *u, double *v,
                          double *T) {
  const double randnorm = 1.0 / RAND_MAX;
  const double epstan = 10.;
  srand(0);
  size_t nh = (size_t)(c->nx + 2) * (c->ny + 2);
  for (int i = 0; i < c->nx + 2; i++)
    for (int j = 0; j < c->ny + 2; j++) {
      size_t q = (size_t)j + (size_t)(c->ny + 2) * i;
      double yyytemp = ((double)(j - 1 + (c->ny) * 0));
      double y_c = (double)c->ny * (1) / 2. + (randnorm * rand() - 0.5) * 2. * epstan;
      rho[q] = 1.0;
      T[q] = c->Tdown + (c->Tup - c->Tdown) * (tanh((yyytemp - y_c) / epstan) + 1.0) / 2.0;
      u[q] = 0;
      v[q] = 0;
    }
  /* feq(rho=1,u=0) and geq(T,u=0) as equilif/equilig evaluate them */
  for (size_t q = 0; q < nh; q++)
    for (int k = 0; k < NPOP; k++) {
      f[q * NPOP + k] = rho[q] * WW[k] * (1. - 0.0);
      g[q * NPOP + k] = T[q] * WW[k] * (1. - 0.0);
    }
}

/* 40x40 particle lattice of init_prtcl (Trajectories/code/mympi2.h:116-168),
 * one rank; returns the number placed */
static int lattice_particles(const cfg_t *c, double *x, double *y, int nmax) {
  int nsqx = 40, nsqy = 40, xs[40], ys[40], n = 0;
  xs[0] = 5;
  for (int i = 1; i < nsqx; i++) xs[i] = xs[i - 1] + 42 + (i % 2);
  xs[nsqx - 1] += 2;
  xs[nsqx - 1] += 1;
  ys[0] = 10;
  for (int i = 1; i < nsqy; i++) ys[i] = ys[i - 1] + 21;
  const double del = 0.000001;
  for (int i1 = 0; i1 < nsqx; i1++)
    for (int j1 = 0; j1 < nsqy; j1++)
      for (int i = 1; i < c->nx + 1; i++)
        for (int j = 1; j < c->ny + 1; j++)
          if (abs(i - xs[i1]) < 1 && abs(j - ys[j1]) < 1 && n < nmax) {
            x[n] = (double)i;
            y[n] = (double)j;
            if (i == 1) x[n] = (double)i + del;
            if (j == 1) y[n] = (double)j + del;
            if (i == c->nx) x[n] = (double)i - del;
            if (j == c->ny) y[n] = (double)j - del;
            n++;
          }
  return n;
}

static double splitmix_uniform(unsigned long long seed, unsigned long long index) {
  uint64_t z = (uint64_t)seed + ((uint64_t)index + 1ULL) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------ output */
static const char *REC_NAMES[LBRB_REC_NFULL] = {"x", "y", "u", "v", "xo", "yo", "uo", "vo",
                                                "temp", "dtu", "dtv", "dxu", "dxv", "dyu",
                                                "dyv", "fu", "fv"};

static void write_records(lbrb_t *h, const cfg_t *c, int nrec_fields) {
  int pending = 0;
  CALL(h, lbrb_record_pending(h, &pending));
  if (pending == 0) return;
  size_t per = (size_t)nrec_fields * c->Nprtcl;
  double *buf = (double *)malloc(per * sizeof(double) * (size_t)pending);
  int *steps = (int *)malloc(sizeof(int) * (size_t)pending);
  int *ids = (int *)malloc(sizeof(int) * (size_t)c->Nprtcl);
  int got = 0;
  CALL(h, lbrb_record_drain(h, pending, steps, buf, ids, &got));
  for (int r = 0; r < got; r++) {
    char fname[256];
    snprintf(fname, sizeof(fname), "Prtcl_Veldata1/Particles%d.h5", steps[r]);
    if (steps[r] > 10000000) snprintf(fname, sizeof(fname), "Prtcl_Veldata2/Particles%d.h5", steps[r]);
    write_ds(fname, "id", ids, sizeof(int) * (size_t)c->Nprtcl);
    for (int k = 0; k < nrec_fields; k++)
      write_ds(fname, REC_NAMES[k], buf + (size_t)r * per + (size_t)k * c->Nprtcl,
               sizeof(double) * (size_t)c->Nprtcl);
  }
  free(buf);
  free(steps);
  free(ids);
}

static void dump_pops(lbrb_t *h, const cfg_t *c, const char *fprefix, const char *gprefix, int istep) {
  size_t nh = (size_t)(c->nx + 2) * (c->ny + 2) * NPOP, nd = (size_t)c->nx * c->ny * NPOP;
  double *fh = (double *)malloc(nh * sizeof(double)), *gh = (double *)malloc(nh * sizeof(double));
  double *ds = (double *)malloc(nd * sizeof(double));
  CALL(h, lbrb_get_populations(h, fh, gh, LBRB_LAYOUT_REF_AOS_HALO));
  char fname[256];
  snprintf(fname, sizeof(fname), "%s%d.h5", fprefix, istep);
  pops_halo_to_ds(c, fh, ds);
  write_ds(fname, "f", ds, nd * sizeof(double));
  snprintf(fname, sizeof(fname), "%s%d.h5", gprefix, istep);
  pops_halo_to_ds(c, gh, ds);
  write_ds(fname, "g", ds, nd * sizeof(double));
  free(fh);
  free(gh);
  free(ds);
}

static void snapshot(lbrb_t *h, const cfg_t *c, int istep) {
  size_t nh = (size_t)(c->nx + 2) * (c->ny + 2), nd = (size_t)c->nx * c->ny;
  double *m[3], *ds = (double *)malloc(nd * sizeof(double));
  for (int a = 0; a < 3; a++) m[a] = (double *)malloc(nh * sizeof(double));
  CALL(h, lbrb_get_moments(h, NULL, m[1], m[2], m[0], LBRB_LAYOUT_REF_AOS_HALO));
  char fname[256];
  snprintf(fname, sizeof(fname), "Tempfolder/snaptemp%d.h5", istep);
  const char *names[3] = {"T", "u", "v"};
  for (int a = 0; a < 3; a++) {
    scalar_halo_to_ds(c, m[a], ds);
    write_ds(fname, names[a], ds, nd * sizeof(double));
    free(m[a]);
  }
  free(ds);
}

static void profile_out(lbrb_t *h, const cfg_t *c, int istep) {
  double *pr = (double *)malloc(sizeof(double) * 9 * (size_t)c->ny);
  CALL(h, lbrb_profile(h, pr));
  char fname[256];
  snprintf(fname, sizeof(fname), "profiles.%d.dat", istep);
  FILE *f = fopen(fname, "w");
  for (int j = 0; j < c->ny; j++) {
    fprintf(f, "%d", j + 1);
    for (int k = 0; k < 8; k++) fprintf(f, " %e", pr[(size_t)j * 9 + k]);
    fprintf(f, " \n");
  }
  fclose(f);
  free(pr);
}

static void prtcl_dump(lbrb_t *h, const cfg_t *c, int istep) {
  int n = c->Nprtcl;
  double *a[8];
  for (int k = 0; k < 8; k++) a[k] = (double *)malloc(sizeof(double) * (size_t)n);
  CALL(h, lbrb_particles_get(h, n, NULL, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7]));
  /* prtcl_type records; prtcl_dump fills x, y, u, v (temppart_dump.c:1419-1424) */
  double *rec = (double *)calloc((size_t)n * 8, sizeof(double));
  for (int p = 0; p < n; p++)
    for (int k = 0; k < 4; k++) rec[(size_t)p * 8 + k] = a[k][p];
  char fname[256];
  snprintf(fname, sizeof(fname), "prtcl_dump%d.in", istep);
  write_raw(fname, rec, sizeof(double) * 8 * (size_t)n);
  free(rec);
  for (int k = 0; k < 8; k++) free(a[k]);
}

static void evolution(lbrb_t *h, const cfg_t *c, FILE *f, int istep) {
  double ke = 0, tm = 0;
  (void)c;
  /* NaN/Inf sentinel over the populations at every evolution line */
  const int fin = lbrb_check_finite(h);
  if (fin == LBRB_ERR_NONFINITE) {
    fprintf(stderr, "lbrb_host: non-finite populations at step %d\n", istep);
    exit(7);
  }
  if (fin != LBRB_OK) die("lbrb_check_finite", h);
  CALL(h, lbrb_energy(h, &ke, &tm));
  fprintf(f, "%d %e %e\n", istep, ke, tm);
  fflush(f);
}

/* -------------------------------------------------------------------- main */
static int min_int(int a, int b) { return a < b ? a : b; }

/* next step > istep at which the host has work: records / snapshots
 * (noutconfig), evolution and profiles (nout; 5000 for nudging), dumps
 * (2000000, last), and for nudging the step before each observation file */
static int next_event(const cfg_t *c, int istep, int last) {
  int nx = last;
  int every[5] = {c->noutconfig, c->nout, c->program == 1 ? 5000 : 0, 2000000,
                  c->program == 1 ? c->ntempread : 0};
  if (c->program == 0 && !c->Particle) every[0] = 0;
  for (int e = 0; e < 5; e++)
    if (every[e] > 0) nx = min_int(nx, (istep / every[e] + 1) * every[e]);
  return nx;
}

int main(int argc, char **argv) {
  if (argc < 2 || (strcmp(argv[1], "trajectories") && strcmp(argv[1], "nudging"))) {
    fprintf(stderr, "usage: %s trajectories|nudging [name=value ...]\n", argv[0]);
    return 2;
  }
  cfg_t c;
  defaults(&c, !strcmp(argv[1], "nudging"));
  double Ra = 0, Pr = 1, U = 0;
  for (int a = 2; a < argc; a++) {
    char *eq = strchr(argv[a], '=');
    if (!eq) { fprintf(stderr, "bad argument %s\n", argv[a]); return 2; }
    *eq = 0;
    int r = set_param(&c, argv[a], eq + 1, &Ra, &Pr, &U);
    if (r <= 0) { fprintf(stderr, "unknown or unsupported parameter %s\n", argv[a]); return 2; }
  }
  if (Ra > 0 && U > 0) {
    double nu = U * c.ny * sqrt(Pr / Ra), kappa = U * c.ny / sqrt(Ra * Pr);
    c.relax = 3.0 * nu + 0.5;
    c.relaxg = 3.0 * kappa + 0.5;
    c.gravity = -(U * U) / c.ny;
    c.Tup = -0.5;
    c.Tdown = 0.5;
  }
  if (c.program == 1 && c.contin != 0) {
    /* the reference's contin==1 restart reads an uninitialised rhoi
     * (tempvel_nudge.c:636-639); only contin==0 is supported */
    fprintf(stderr, "contin=1 is not supported\n");
    return 2;
  }
  /* the run directory and its missing parents are created (mkdir -p) */
  {
    char path[1024];
    snprintf(path, sizeof(path), "%s", c.dir);
    for (char *q = path + 1; *q; q++)
      if (*q == '/') {
        *q = '\0';
        if (mkdir(path, 0755) != 0 && errno != EEXIST) break;
        *q = '/';
      }
    if (mkdir(path, 0755) != 0 && errno != EEXIST) { /* chdir below reports it */ }
  }
  if (chdir(c.dir) != 0) { fprintf(stderr, "cannot enter %s\n", c.dir); return 2; }
  ensure_dir("Prtcl_Veldata1");
  ensure_dir("Tempfolder");
  const int traj = c.program == 0;
  const int np = traj && c.Particle ? c.Nprtcl : 0;
  const int nrec_fields = c.Prtcl_Writefull ? LBRB_REC_NFULL : LBRB_REC_NBASIC;

  lbrb_params p;
  lbrb_params_default(&p);
  p.nx = c.nx;
  p.ny = c.ny;
  p.relax = c.relax;
  p.relaxg = c.relaxg;
  p.Tup = c.Tup;
  p.Tdown = c.Tdown;
  p.gravity = c.gravity;
  p.precision = c.precision;
  p.twall = traj ? LBRB_TWALL_DIRICHLET : LBRB_TWALL_ADIABATIC;
  p.nudge = traj ? LBRB_NUDGE_NONE : LBRB_NUDGE_REFBOX;
  p.alpha = c.alpha;
  p.ntempread = c.ntempread;
  p.nobs = traj ? 0 : c.Nprtcl;
  p.beta = c.beta;
  p.nprtcl = np;
  p.noutconfig = traj ? c.noutconfig : 0;
  p.record_full = c.Prtcl_Writefull;
  p.record_slots = 4;
  p.device = c.device;
  lbrb_t *h = NULL;
  int rc = lbrb_create(&p, &h);
  if (rc != LBRB_OK) { fprintf(stderr, "lbrb_create failed (%d)\n", rc); return 8; }

  size_t nh = (size_t)(c.nx + 2) * (c.ny + 2);
  size_t nd = (size_t)c.nx * c.ny * NPOP;
  double *f = (double *)malloc(nh * NPOP * sizeof(double));
  double *g = (double *)malloc(nh * NPOP * sizeof(double));
  double *rho = (double *)malloc(nh * sizeof(double)), *u = (double *)malloc(nh * sizeof(double));
  double *v = (double *)malloc(nh * sizeof(double)), *T = (double *)malloc(nh * sizeof(double));
  /* ---- initial state */
  if (c.ic_conduction) {
    CALL(h, lbrb_init_conduction(h, c.seed, c.noise));
  } else if (c.scratch) {
    scratch_state(&c, f, g, rho, u, v, T);
    CALL(h, lbrb_set_populations(h, f, g, LBRB_LAYOUT_REF_AOS_HALO));
    CALL(h, lbrb_set_moments(h, rho, u, v, T, LBRB_LAYOUT_REF_AOS_HALO));
  } else if (!traj) {
    /* nudging restart, contin==0 (tempvel_nudge.c:2319-2327 with inithydro
     * :596-618): g from cong, f = feq(1,0), rho = 1, u = v = 0, and T the sum
     * of congpre only inside the initial nudging boxes of set_nudge_vol
     * (:2054-2079), zero elsewhere */
    double *ds = (double *)malloc(nd * sizeof(double));
    if (read_ds("cong.h5", "g", ds, nd * sizeof(double))) die("cong not found", NULL);
    pops_ds_to_halo(&c, ds, g);
    if (read_ds("congpre.h5", "g", ds, nd * sizeof(double))) die("cong not found", NULL);
    int xs[40], ys[40];
    xs[0] = 5;
    for (int i = 1; i < 40; i++) xs[i] = xs[i - 1] + 42 + (i % 2);
    xs[39] += 3;
    ys[0] = 10;
    for (int i = 1; i < 40; i++) ys[i] = ys[i - 1] + 21;
    for (size_t q = 0; q < nh; q++) {
      rho[q] = 1.0;
      u[q] = 0.0;
      v[q] = 0.0;
      T[q] = 0.0;
      for (int k = 0; k < NPOP; k++) f[q * NPOP + k] = WW[k] * (1. - 0.0);
    }
    for (int i = 1; i <= c.nx; i++)
      for (int j = 1; j <= c.ny; j++) {
        int in = 0;
        for (int a = 0; a < 40 && !in; a++)
          for (int b = 0; b < 40 && !in; b++) in = abs(i - xs[a]) < 4 && abs(j - ys[b]) < 4;
        size_t q = (size_t)j + (size_t)(c.ny + 2) * i;
        if (in) {
          double t = 0.0;
          for (int k = 0; k < NPOP; k++) t += ds[((size_t)(i - 1) * c.ny + (j - 1)) * NPOP + k];
          T[q] = t;
        }
      }
    CALL(h, lbrb_set_populations(h, f, g, LBRB_LAYOUT_REF_AOS_HALO));
    CALL(h, lbrb_set_moments(h, rho, u, v, T, LBRB_LAYOUT_REF_AOS_HALO));
    free(ds);
  } else {
    double *ds = (double *)malloc(nd * sizeof(double));
    double *fp = (double *)malloc(nh * NPOP * sizeof(double)), *gp = (double *)malloc(nh * NPOP * sizeof(double));
    if (read_ds("conf.h5", "f", ds, nd * sizeof(double))) die("conf not found", NULL);
    pops_ds_to_halo(&c, ds, f);
    if (read_ds("cong.h5", "g", ds, nd * sizeof(double))) die("cong not found", NULL);
    pops_ds_to_halo(&c, ds, g);
    if (read_ds("confpre.h5", "f", ds, nd * sizeof(double))) die("confpre not found", NULL);
    pops_ds_to_halo(&c, ds, fp);
    if (read_ds("congpre.h5", "g", ds, nd * sizeof(double))) die("congpre not found", NULL);
    pops_ds_to_halo(&c, ds, gp);
    /* restore* abort on a population that is exactly zero (temppart_dump.c:414-425) */
    for (size_t q = 0; q < nd; q++)
      if (ds[q] == 0.0) die("a restored population is exactly zero", NULL);
    CALL(h, lbrb_set_populations(h, f, g, LBRB_LAYOUT_REF_AOS_HALO));
    CALL(h, lbrb_moments_from_pre(h, fp, gp, LBRB_LAYOUT_REF_AOS_HALO));
    free(ds);
    free(fp);
    free(gp);
  }
  CALL(h, lbrb_set_istep(h, c.nstart));
  /* ---- particles */
  if (np > 0) {
    int *ids = (int *)malloc(sizeof(int) * (size_t)np), *pt = (int *)malloc(sizeof(int) * (size_t)np);
    double *px = (double *)calloc((size_t)np, sizeof(double)), *py = (double *)calloc((size_t)np, sizeof(double));
    double *pu = (double *)calloc((size_t)np, sizeof(double)), *pv = (double *)calloc((size_t)np, sizeof(double));
    double *inv = (double *)malloc(sizeof(double) * (size_t)np);
    CALL(h, lbrb_get_moments(h, rho, u, v, T, LBRB_LAYOUT_REF_AOS_HALO));
    const double fac = c.tracer ? 1.0 : 0.98; /* init_prtcl: v = u or 0.98 u */
    if (!c.Particle_scratch) {
      /* restore_prtcl: ids from Particles<nstart>.h5, state from prtcl_dump<nstart>.in */
      char fname[256];
      snprintf(fname, sizeof(fname), "Prtcl_Veldata1/Particles%d.h5", c.nstart);
      if (read_ds(fname, "id", ids, sizeof(int) * (size_t)np)) die("Particle file not opened", NULL);
      double *rec = (double *)malloc(sizeof(double) * 8 * (size_t)np);
      snprintf(fname, sizeof(fname), "prtcl_dump%d.in", c.nstart);
      if (read_raw(fname, rec, sizeof(double) * 8 * (size_t)np)) die("prtcl_dump file not read", NULL);
      for (int q = 0; q < np; q++) {
        px[q] = rec[q * 8 + 0];
        py[q] = rec[q * 8 + 1];
        pu[q] = rec[q * 8 + 2];
        pv[q] = rec[q * 8 + 3];
      }
      free(rec);
    } else {
      int placed = 0;
      if (c.prtcl_uniform) {
        for (int q = 0; q < np; q++) {
          px[q] = c.nx * splitmix_uniform(c.seed + 7, 2 * (unsigned long long)q);
          py[q] = 1.0 + (c.ny - 1) * splitmix_uniform(c.seed + 7, 2 * (unsigned long long)q + 1);
          if (px[q] <= 0.0) px[q] = 0.5;
        }
        placed = np;
      } else {
        placed = lattice_particles(&c, px, py, np);
      }
      if (placed != np) {
        fprintf(stderr, "lbrb_host: the particle lattice placed %d of Nprtcl=%d particles\n", placed, np);
        return 8;
      }
      double *Tp = (double *)malloc(sizeof(double) * (size_t)np);
      for (int q = 0; q < np; q++) {
        ids[q] = q;
        pu[q] = fac * bilinear(&c, u, px[q], py[q]);
        pv[q] = fac * bilinear(&c, v, px[q], py[q]);
        Tp[q] = bilinear(&c, T, px[q], py[q]);
      }
      /* init_prtcl writes its initial state (mympi2.h:256-289) */
      char fname[64];
      snprintf(fname, sizeof(fname), "init_prtclx%d.in", c.nstart); write_raw(fname, px, sizeof(double) * np);
      snprintf(fname, sizeof(fname), "init_prtcly%d.in", c.nstart); write_raw(fname, py, sizeof(double) * np);
      snprintf(fname, sizeof(fname), "init_prtclT%d.in", c.nstart); write_raw(fname, Tp, sizeof(double) * np);
      snprintf(fname, sizeof(fname), "init_prtclu%d.in", c.nstart); write_raw(fname, pu, sizeof(double) * np);
      snprintf(fname, sizeof(fname), "init_prtclv%d.in", c.nstart); write_raw(fname, pv, sizeof(double) * np);
      snprintf(fname, sizeof(fname), "init_prtcl_id%d.in", c.nstart); write_raw(fname, ids, sizeof(int) * np);
      free(Tp);
    }
    for (int q = 0; q < np; q++) {
      pt[q] = c.tracer ? LBRB_PTYPE_TRACER : LBRB_PTYPE_INERTIAL;
      inv[q] = 1.0 / c.taulag;
    }
    CALL(h, lbrb_particles_set(h, np, ids, px, py, pu, pv, pt, inv));
    free(ids); free(pt); free(px); free(py); free(pu); free(pv); free(inv);
  }
  /* ---- nudging observations (set_nudge_vol contin==0, tempvel_nudge.c:2080-2122) */
  int nobs = c.Nprtcl;
  double *ox = NULL, *oy = NULL, *oT = NULL;
  int *oid = NULL;
  if (!traj) {
    ox = (double *)malloc(sizeof(double) * nobs);
    oy = (double *)malloc(sizeof(double) * nobs);
    oT = (double *)malloc(sizeof(double) * nobs);
    oid = (int *)malloc(sizeof(int) * nobs);
    if (read_raw("obs/init_prtclx0.in", ox, sizeof(double) * nobs) ||
        read_raw("obs/init_prtcly0.in", oy, sizeof(double) * nobs) ||
        read_raw("obs/init_prtclT0.in", oT, sizeof(double) * nobs) ||
        read_raw("obs/init_prtcl_id0.in", oid, sizeof(int) * nobs))
      die("initial observation files obs/init_prtcl*0.in not readable", NULL);
    CALL(h, lbrb_nudge_init(h, nobs, ox, oy, oT, oid));
  }
  FILE *fevo = fopen("evolution.dat", "w");
  /* ---- time loop (temppart_dump.c:1674-1759, tempvel_nudge.c:2346-2411) */
  int istep = c.nstart;
  const int last = c.nstart + c.nsteps;
  while (istep < last) {
    if (!traj && (istep + 1) % c.ntempread == 1) {
      /* read_prtcl: the file of step istep+ntempread-1 (tempvel_nudge.c:1415) */
      char fname[256];
      snprintf(fname, sizeof(fname), "obs/Prtcl_Veldata1/Particles%d.h5", istep + c.ntempread);
      if (read_ds(fname, "x", ox, sizeof(double) * nobs) || read_ds(fname, "y", oy, sizeof(double) * nobs) ||
          read_ds(fname, "id", oid, sizeof(int) * nobs) || read_ds(fname, "temp", oT, sizeof(double) * nobs))
        die("Particle file not opened", NULL);
      CALL(h, lbrb_nudge_load(h, nobs, ox, oy, oid, oT));
    }
    int target = next_event(&c, istep, last);
    if (target <= istep) target = istep + 1;
    nvtxRangePushA("lbrb_host steps");
    CALL(h, lbrb_step(h, target - istep));
    istep = target;
    CALL(h, lbrb_sync(h));
    nvtxRangePop();
    nvtxRangePushA("lbrb_host output");
    if (np > 0) write_records(h, &c, nrec_fields);
    /* post-stream populations of this step (dumpfpre/dumpgpre) */
    if (istep == last || istep % 2000000 == 0) {
      double *fh = (double *)malloc(nh * NPOP * sizeof(double)), *gh = (double *)malloc(nh * NPOP * sizeof(double));
      double *ds = (double *)malloc(nd * sizeof(double));
      CALL(h, lbrb_get_poststream(h, fh, gh, LBRB_LAYOUT_REF_AOS_HALO));
      char fname[256];
      snprintf(fname, sizeof(fname), "confpre%d.h5", istep);
      pops_halo_to_ds(&c, fh, ds);
      write_ds(fname, "f", ds, nd * sizeof(double));
      snprintf(fname, sizeof(fname), "congpre%d.h5", istep);
      pops_halo_to_ds(&c, gh, ds);
      write_ds(fname, "g", ds, nd * sizeof(double));
      free(fh); free(gh); free(ds);
    }
    if (traj) {
      if (istep % c.nout == 0) evolution(h, &c, fevo, istep);
    } else {
      if (istep % c.noutconfig == 0) snapshot(h, &c, istep);
      if (istep % c.nout == 0) profile_out(h, &c, istep);
      if (istep % 5000 == 0) evolution(h, &c, fevo, istep);
    }
    if (istep % 2000000 == 0) {
      dump_pops(h, &c, "confnew", "congnew", istep);
      if (np > 0) prtcl_dump(h, &c, istep);
    }
    nvtxRangePop();
  }
  fclose(fevo);
  /* final dumps (temppart_dump.c:1763-1767): the reference's loop counter is
   * nsteps+nstart+1 after the loop */
  dump_pops(h, &c, "confnew", "congnew", last + 1);
  if (np > 0) prtcl_dump(h, &c, last + 1);
  lbrb_destroy(h);
  free(f); free(g); free(rho); free(u); free(v); free(T);
  free(ox); free(oy); free(oT); free(oid);
  return 0;
}
