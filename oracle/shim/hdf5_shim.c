/*
 * hdf5_shim.c -- implementation of the minimal HDF5 stand-in (see hdf5.h).
 * TEST INFRASTRUCTURE: used only to run the reference's own sources.
 */
#define _GNU_SOURCE
#include "hdf5.h"

#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#define MAXOBJ 4096
#define MAXRANK 4

typedef struct {
  int used, rank;
  hsize_t dims[MAXRANK], start[MAXRANK], block[MAXRANK];
  int selected;
} space_t;
typedef struct {
  int used;
  char dir[1024];
} file_t;
typedef struct {
  int used, fd;
} dset_t;

static space_t g_s[MAXOBJ];
static file_t g_f[MAXOBJ];
static dset_t g_d[MAXOBJ];
static hid_t g_plist = 100;

herr_t H5Eset_current_stack(hid_t s) { (void)s; return 0; }
hid_t H5Pcreate(hid_t c) { (void)c; return g_plist++; }
herr_t H5Pset_fapl_mpio(hid_t p, MPI_Comm c, MPI_Info i) { (void)p; (void)c; (void)i; return 0; }
herr_t H5Pset_dxpl_mpio(hid_t p, int m) { (void)p; (void)m; return 0; }
herr_t H5Pclose(hid_t p) { (void)p; return 0; }

hid_t H5Screate_simple(int rank, const hsize_t dims[], const hsize_t maxdims[]) {
  (void)maxdims;
  for (int i = 1; i < MAXOBJ; i++)
    if (!g_s[i].used) {
      space_t *s = &g_s[i];
      memset(s, 0, sizeof(*s));
      s->used = 1;
      s->rank = rank;
      for (int d = 0; d < rank; d++) { s->dims[d] = dims[d]; s->block[d] = dims[d]; }
      return i;
    }
  return -1;
}

herr_t H5Sselect_hyperslab(hid_t sp, int op, const hsize_t start[], const hsize_t stride[],
                           const hsize_t count[], const hsize_t block[]) {
  (void)op;
  space_t *s = &g_s[sp];
  for (int d = 0; d < s->rank; d++) {
    if ((stride && stride[d] != 1) || (count && count[d] != 1)) {
      fprintf(stderr, "hdf5 shim: only stride 1, count 1 hyperslabs\n");
      exit(95);
    }
    s->start[d] = start[d];
    s->block[d] = block ? block[d] : 1;
  }
  s->selected = 1;
  return 0;
}

herr_t H5Sclose(hid_t sp) { g_s[sp].used = 0; return 0; }

static hid_t new_file(const char *name) {
  for (int i = 1; i < MAXOBJ; i++)
    if (!g_f[i].used) {
      g_f[i].used = 1;
      snprintf(g_f[i].dir, sizeof(g_f[i].dir), "%s.d", name);
      return i;
    }
  return -1;
}

hid_t H5Fcreate(const char *name, unsigned flags, hid_t fcpl, hid_t fapl) {
  (void)flags; (void)fcpl; (void)fapl;
  char dir[1100];
  snprintf(dir, sizeof(dir), "%s.d", name);
  if (mkdir(dir, 0755) != 0 && errno != EEXIST) return -1;
  return new_file(name);
}

hid_t H5Fopen(const char *name, unsigned flags, hid_t fapl) {
  (void)flags; (void)fapl;
  char dir[1100];
  struct stat st;
  snprintf(dir, sizeof(dir), "%s.d", name);
  if (stat(dir, &st) != 0 || !S_ISDIR(st.st_mode)) return -1;
  return new_file(name);
}

herr_t H5Fclose(hid_t f) { g_f[f].used = 0; return 0; }

static long tsize(hid_t t) { return t == H5T_NATIVE_INT ? 4 : 8; }

static void dpath(hid_t f, const char *name, char *out, size_t n) {
  char nm[512];
  const char *p = name[0] == '/' ? name + 1 : name;
  size_t k = 0;
  for (; p[k] && k + 1 < sizeof(nm); k++) nm[k] = p[k] == '/' ? '_' : p[k];
  nm[k] = 0;
  snprintf(out, n, "%s/%s.bin", g_f[f].dir, nm);
}

static hid_t new_dset(int fd) {
  for (int i = 1; i < MAXOBJ; i++)
    if (!g_d[i].used) { g_d[i].used = 1; g_d[i].fd = fd; return i; }
  return -1;
}

hid_t H5Dcreate(hid_t f, const char *name, hid_t type, hid_t space, hid_t a, hid_t b, hid_t c) {
  (void)a; (void)b; (void)c;
  char path[1400];
  dpath(f, name, path, sizeof(path));
  int fd = open(path, O_RDWR | O_CREAT, 0644);
  if (fd < 0) return -1;
  const space_t *s = &g_s[space];
  off_t total = tsize(type);
  for (int d = 0; d < s->rank; d++) total *= (off_t)s->dims[d];
  struct stat st;
  if (fstat(fd, &st) == 0 && st.st_size < total) {
    if (ftruncate(fd, total) != 0) { close(fd); return -1; }
  }
  return new_dset(fd);
}

hid_t H5Dopen(hid_t f, const char *name, hid_t a) {
  (void)a;
  char path[1400];
  dpath(f, name, path, sizeof(path));
  int fd = open(path, O_RDWR);
  if (fd < 0) return -1;
  return new_dset(fd);
}

herr_t H5Dclose(hid_t d) {
  close(g_d[d].fd);
  g_d[d].used = 0;
  return 0;
}

/* walk the selected box of memspace and filespace together, one innermost
 * contiguous run at a time */
static herr_t xfer(hid_t d, hid_t type, hid_t ms, hid_t fs, void *buf, int writing) {
  const space_t *m = &g_s[ms], *f = &g_s[fs];
  long es = tsize(type);
  int rm = m->rank, rf = f->rank;
  hsize_t nm = 1, nf = 1;
  for (int k = 0; k < rm; k++) nm *= m->block[k];
  for (int k = 0; k < rf; k++) nf *= f->block[k];
  if (nm != nf) { fprintf(stderr, "hdf5 shim: selection sizes differ\n"); exit(95); }
  if (nm == 0) return 0;
  if (rm != rf) { fprintf(stderr, "hdf5 shim: selection ranks differ\n"); exit(95); }
  int r = rm;
  hsize_t run = m->block[r - 1];
  if (f->block[r - 1] != run) { fprintf(stderr, "hdf5 shim: selection shapes differ\n"); exit(95); }
  hsize_t idx[MAXRANK] = {0, 0, 0, 0};
  hsize_t nruns = nm / run;
  for (hsize_t q = 0; q < nruns; q++) {
    hsize_t mo = 0, fo = 0;
    for (int k = 0; k < r; k++) {
      mo = mo * m->dims[k] + (m->start[k] + idx[k]);
      fo = fo * f->dims[k] + (f->start[k] + idx[k]);
    }
    char *mp = (char *)buf + mo * es;
    ssize_t nb = (ssize_t)(run * es);
    ssize_t done = writing ? pwrite(g_d[d].fd, mp, (size_t)nb, (off_t)(fo * es))
                           : pread(g_d[d].fd, mp, (size_t)nb, (off_t)(fo * es));
    if (done != nb) { fprintf(stderr, "hdf5 shim: short %s\n", writing ? "write" : "read"); exit(95); }
    for (int k = r - 2; k >= 0; k--) {
      if (++idx[k] < m->block[k]) break;
      idx[k] = 0;
    }
  }
  return 0;
}

herr_t H5Dwrite(hid_t d, hid_t t, hid_t ms, hid_t fs, hid_t x, const void *buf) {
  (void)x;
  return xfer(d, t, ms, fs, (void *)buf, 1);
}

herr_t H5Dread(hid_t d, hid_t t, hid_t ms, hid_t fs, hid_t x, void *buf) {
  (void)x;
  return xfer(d, t, ms, fs, buf, 0);
}
