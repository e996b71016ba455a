/*
 * fb_host.c -- host side of the B200 hydro step (C99 + CUDA runtime API).
 *
 * Owns a disk's device memory, the mesh tables, the planetary system and the
 * order of the stage kernels within one hydro step (main.c:361-448 of the
 * reference).  The scalar work of a step -- the CFL minimum's clipping to the
 * DT interval, the planets' RK5 orbit, the frame rotation -- runs here in
 * FP64, as it does in the reference (potential.c:10-49); everything per cell
 * runs on the GPU.  There is no CPU path for the per-cell work.
 */
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "fargo_b200.h"
#include "fb_dev.h"
#include "fb_psys.h"

#define NG 3
#define G 1.0
#define MSTAR 1.0
#define R0 1.0
#define SMALLTIME (1e-10 * sqrt(R0 * R0 * R0 / (G * MSTAR)))
#define MAXALLOC 1024  /* device allocations per disk: geometry, tables, 8 fluids x 30 fields */

static __thread char g_err[512];

const char *fb_last_error(void) { return g_err; }

static int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

/* error text for the batch and server translation units */
int fb_internal_fail(int code, const char *what, int cuda_err) {
  if (cuda_err) return fail(code, "%s: %s", what, cudaGetErrorString((cudaError_t)cuda_err));
  return fail(code, "%s", what);
}

#define CU(call)                                                                 \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess)                                                       \
      return fail(FB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
  } while (0)

#define LCH(call)                                                                \
  do {                                                                           \
    int e_ = (call);                                                             \
    if (e_ != 0)                                                                 \
      return fail(FB_ERR_CUDA, "%s failed: %s", #call,                           \
                  cudaGetErrorString((cudaError_t)e_));                          \
  } while (0)

struct fb_disk {
  fb_params p;
  fb_disk_dev d;
  int device;
  cudaStream_t stream;
  size_t esz;                   /* element size of the fields */
  long long ncell;              /* stored cells per field */
  /* host geometry (double) */
  double *xmin, *ymin, *zmin, *xmed, *ymed, *zmed, *invdiffxmed;
  double *sxi, *sxj, *syj, *szj, *sxk, *syk, *szk, *invvj;
  double mindx;
  /* planetary system, frame and time (fb_psys.h) */
  fb_psys ps;
  fb_scalars sc;
  double *h_dtmin;              /* pinned: [0..1] CFL minimum + flag, [8..] disk accelerations */
  double *d_ring3, *d_facc;     /* disk-force scratch: ring sums, accelerations (3 per planet) */
  int feeldisk;                 /* some planet feels the disk */
  void *allocs[MAXALLOC];
  int nalloc;
  size_t bytes;                 /* device bytes requested by this disk */
  /* one device arena per disk, sized by fb_params_bytes and zeroed once:
     the fields and tables are carved from it (creation costs one
     cudaMalloc + one memset instead of one of each per array) */
  char *arena;
  size_t arena_size, arena_used;
  int arena_owned, stream_owned;  /* 0: lent by a batch (fb_disk_internal_provide) */
  char *hstage;                 /* host image of the arena's table region, sent in one copy */
  size_t hstage_size, hstage_hi;
  /* optional per-launch timing (fb_disk_profile) */
  int prof;
  int nev;
  cudaEvent_t ev[32];
  const char *evname[32];
  float prof_ms[32];
  int prof_n;
};

/* record an event after a launch when profiling; names label the interval
 * that ends at this event */
static void mark(fb_disk *D, const char *name) {
  if (!D->prof || D->nev >= 32) return;
  if (!D->ev[D->nev]) cudaEventCreate(&D->ev[D->nev]);
  cudaEventRecord(D->ev[D->nev], D->stream);
  D->evname[D->nev] = name;
  D->nev++;
}

/* ------------------------------------------------------------------------ */
static int dalloc(fb_disk *D, void **p, size_t bytes) {
  cudaError_t e;
  size_t need = ((bytes ? bytes : 16) + 255) & ~(size_t)255;
  if (D->arena && D->arena_used + need <= D->arena_size) {
    *p = D->arena + D->arena_used;   /* 256-byte aligned, already zero */
    D->arena_used += need;
    D->bytes += bytes ? bytes : 16;
    return FB_OK;
  }
  if (D->nalloc >= MAXALLOC) return fail(FB_ERR_NOMEM, "too many device allocations");
  e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) return fail(FB_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  D->allocs[D->nalloc++] = *p;
  D->bytes += bytes ? bytes : 16;
  cudaMemset(*p, 0, bytes ? bytes : 16);
  return FB_OK;
}

/* Pinned 256-byte slots for the per-step readback (CFL minimum, flag, disk
 * accelerations), carved from 64 KiB pinned blocks and recycled through a
 * free list: creating a disk pins no memory of its own. */
#define PIN_SLOT 256
#define PIN_BLOCK (64 * 1024)
static pthread_mutex_t g_pin_mu = PTHREAD_MUTEX_INITIALIZER;
static void *g_pin_free = NULL;             /* singly linked through the slots */
static char *g_pin_block = NULL;
static size_t g_pin_used = PIN_BLOCK;

static double *pinned_slot(void) {
  void *p = NULL;
  pthread_mutex_lock(&g_pin_mu);
  if (g_pin_free) {
    p = g_pin_free;
    g_pin_free = *(void **)p;
  } else {
    if (g_pin_used + PIN_SLOT > PIN_BLOCK) {
      char *b = NULL;
      if (cudaMallocHost((void **)&b, PIN_BLOCK) == cudaSuccess) {
        g_pin_block = b;
        g_pin_used = 0;
      }
    }
    if (g_pin_block && g_pin_used + PIN_SLOT <= PIN_BLOCK) {
      p = g_pin_block + g_pin_used;
      g_pin_used += PIN_SLOT;
    }
  }
  pthread_mutex_unlock(&g_pin_mu);
  if (p) memset(p, 0, PIN_SLOT);
  return (double *)p;
}

static void pinned_release(double *p) {
  pthread_mutex_lock(&g_pin_mu);
  *(void **)p = g_pin_free;
  g_pin_free = p;
  pthread_mutex_unlock(&g_pin_mu);
}

/* upload a double table, converted to the disk's precision when asked */
static int upload(fb_disk *D, const void **dst, const double *src, int n, int as_float) {
  void *p;
  int rc, i;
  const size_t bytes = (as_float ? sizeof(float) : sizeof(double)) * (size_t)n;
  rc = dalloc(D, &p, bytes);
  if (rc) return rc;
  if (D->hstage && (char *)p >= D->arena && (size_t)((char *)p - D->arena) + bytes <= D->hstage_size) {
    char *h = D->hstage + ((char *)p - D->arena);   /* staged: sent with the others */
    if (as_float)
      for (i = 0; i < n; i++) ((float *)h)[i] = (float)src[i];
    else
      memcpy(h, src, bytes);
    if ((size_t)((char *)p - D->arena) + bytes > D->hstage_hi) D->hstage_hi = (size_t)((char *)p - D->arena) + bytes;
    *dst = p;
    return FB_OK;
  }
  if (as_float) {
    float *tmp = (float *)malloc(sizeof(float) * (n ? n : 1));
    for (i = 0; i < n; i++) tmp[i] = (float)src[i];
    cudaMemcpy(p, tmp, sizeof(float) * n, cudaMemcpyHostToDevice);
    free(tmp);
  } else {
    cudaMemcpy(p, src, sizeof(double) * n, cudaMemcpyHostToDevice);
  }
  *dst = p;
  return FB_OK;
}

/* ------------------------------------------------------------------------ */
/* Mesh: InitSpace (LowTasks.c:300-383) and InitSurfaces (LowTasks.c:466-563) */
static void mesh(fb_disk *D) {
  const fb_params *p = &D->p;
  int i, j, k, sx = p->nx, sy = D->d.sy, sz = D->d.sz, is3d = D->d.is3d;
  /* a slab's rows are rows y0 .. y0 + ny - 1 of the whole mesh: its edges
     are the whole mesh's, from the global index (split.c / InitSpace) */
  const int nyg = p->slab_ny_global > 0 ? p->slab_ny_global : p->ny, y0 = p->slab_ny_global > 0 ? p->slab_y0 : 0;
  double dx = (p->xmax - p->xmin) / p->nx, dy = (p->ymax - p->ymin) / nyg;
  double dz = is3d ? (p->zmax - p->zmin) / p->nz : 0.0;
  if (p->log_spacing) {
    dy = (log(p->ymax) - log(p->ymin)) / nyg;
    for (j = 0; j < sy + 1; j++) D->ymin[j] = exp(log(p->ymin) + dy * (j + y0 - NG));
  } else {
    for (j = 0; j < sy + 1; j++) D->ymin[j] = p->ymin + dy * (j + y0 - NG);
  }
  for (k = 0; k < sz + 1; k++) D->zmin[k] = is3d ? p->zmin + dz * (k - NG) : 0.0;
  for (i = 0; i < sx + 1; i++) D->xmin[i] = p->xmin + dx * i;
  for (i = 0; i < sx; i++) D->xmed[i] = 0.5 * (D->xmin[i + 1] + D->xmin[i]);
  for (j = 0; j < sy; j++) D->ymed[j] = 0.5 * (D->ymin[j + 1] + D->ymin[j]);
  for (k = 0; k < sz; k++) D->zmed[k] = 0.5 * (D->zmin[k + 1] + D->zmin[k]);
  for (i = 1; i < sx; i++) D->invdiffxmed[i] = 1. / (D->xmed[i] - D->xmed[i - 1]);
  D->invdiffxmed[0] = 1. / (D->xmed[0] - (D->xmed[p->nx - 1] - (p->xmax - p->xmin)));
  for (i = 0; i < sx; i++) D->sxi[i] = D->xmin[i + 1] - D->xmin[i];
  D->mindx = D->sxi[0];
  for (i = 1; i < sx; i++)
    if (D->sxi[i] < D->mindx) D->mindx = D->sxi[i];
  if (!p->spherical) {
    for (j = 0; j < sy; j++) {
      D->sxj[j] = D->ymin[j + 1] - D->ymin[j];
      D->syj[j] = D->ymin[j];
      D->szj[j] = 0.5 * (D->ymin[j + 1] * D->ymin[j + 1] - D->ymin[j] * D->ymin[j]);
      D->invvj[j] = 1.0 / D->szj[j];
    }
    for (k = 0; k < sz; k++) {
      D->sxk[k] = is3d ? D->zmin[k + 1] - D->zmin[k] : 1.0;
      D->syk[k] = D->sxk[k];
      D->szk[k] = 1.0;
    }
  } else {
    for (j = 0; j < sy; j++) {
      D->sxj[j] = 0.5 * (D->ymin[j + 1] * D->ymin[j + 1] - D->ymin[j] * D->ymin[j]);
      D->syj[j] = D->ymin[j] * D->ymin[j];
      D->szj[j] = 0.5 * (D->ymin[j + 1] * D->ymin[j + 1] - D->ymin[j] * D->ymin[j]);
      D->invvj[j] = 3. / ((D->ymin[j + 1] * D->ymin[j + 1] * D->ymin[j + 1] - D->ymin[j] * D->ymin[j] * D->ymin[j]));
    }
    for (k = 0; k < sz; k++) {
      D->sxk[k] = D->zmin[k + 1] - D->zmin[k];
      D->syk[k] = cos(D->zmin[k]) - cos(D->zmin[k + 1]);
      D->szk[k] = sin(D->zmin[k]);
    }
  }
}

/* Upload the mesh and every libm-derived table the kernels read. */
static int upload_geometry(fb_disk *D) {
  const fb_params *p = &D->p;
  int sx = p->nx, sy = D->d.sy, sz = D->d.sz, i, j, k, pass, rc;
  double *t_szmed = malloc(sizeof(double) * (sz + 1)), *t_czmed = malloc(sizeof(double) * (sz + 1));
  double *t_szmin = malloc(sizeof(double) * (sz + 1)), *t_czmin = malloc(sizeof(double) * (sz + 1));
  double *t_cx = malloc(sizeof(double) * sx), *t_sx = malloc(sizeof(double) * sx);
  double *t_visc = malloc(sizeof(double) * sy), *t_viscm = malloc(sizeof(double) * sy), *t_tau = malloc(sizeof(double) * sy);
  double *t_r2 = malloc(sizeof(double) * sy), *t_dr2 = malloc(sizeof(double) * sy);
  double *t_s2 = malloc(sizeof(double) * (sz + 1)), *t_ds2 = malloc(sizeof(double) * (sz + 1));
  double *t_iym = malloc(sizeof(double) * sy), *t_iyi = malloc(sizeof(double) * sy);
  double *t_idy = malloc(sizeof(double) * sy), *t_pst = malloc(sizeof(double) * sy);
  for (k = 0; k < sz; k++) { t_szmed[k] = sin(D->zmed[k]); t_czmed[k] = cos(D->zmed[k]); }
  for (k = 0; k < sz + 1; k++) { t_szmin[k] = sin(D->zmin[k]); t_czmin[k] = cos(D->zmin[k]); }
  t_szmed[sz] = t_czmed[sz] = 0.0;
  for (i = 0; i < sx; i++) { t_cx[i] = cos(D->xmed[i]); t_sx[i] = sin(D->xmed[i]); }
  for (j = 0; j < sy; j++) {
    t_visc[j] = sqrt(D->ymed[j] * D->ymed[j] * D->ymed[j] / (G * MSTAR));   /* visctensor_*.c alpha-nu */
    t_viscm[j] = sqrt(D->ymin[j] * D->ymin[j] * D->ymin[j] / (G * MSTAR));
    t_tau[j] = p->tau_damp * sqrt(D->ymed[j] * D->ymed[j] * D->ymed[j] / G / MSTAR); /* stockholm.c:134 */
  }
  /* R^2 = (r sin(theta))^2 factors of the frame rotation and their
     neighbour differences, each difference taken in double so that the
     FP32 sweeps never subtract two large R^2 values themselves */
  for (j = 0; j < sy; j++) {
    t_r2[j] = D->ymed[j] * D->ymed[j];
    t_dr2[j] = j > 0 ? D->ymed[j] * D->ymed[j] - D->ymed[j - 1] * D->ymed[j - 1] : 0.0;
  }
  for (j = 0; j < sy; j++) {
    t_iym[j] = 1.0 / D->ymed[j];
    t_iyi[j] = 1.0 / D->ymin[j];
    t_idy[j] = j > 0 ? 1.0 / (D->ymed[j] - D->ymed[j - 1]) : 0.0;
    /* potential.c:101-106: the star's term, -G M / r (r = Ymed in spherical
       meshes, sqrt(Ymed^2 + Zmed^2) with Zmed = 0 in 2D cylindrical ones) */
    t_pst[j] = D->d.spherical ? -G * MSTAR / D->ymed[j] : -G * MSTAR / sqrt(D->ymed[j] * D->ymed[j]);
  }
  for (k = 0; k < sz + 1; k++) t_s2[k] = t_szmed[k] * t_szmed[k];
  for (k = 0; k < sz + 1; k++) t_ds2[k] = k > 0 && k < sz ? t_s2[k] - t_s2[k - 1] : 0.0;
  for (pass = 0; pass < 2; pass++) {
    /* pass 0: double tables; pass 1: the disk's precision (skipped in FP64) */
    fb_geom_dev *g = pass == 0 ? &D->d.geomd : &D->d.geom;
    int f = pass == 1 && D->d.precision == FB_FP32;
    if (pass == 1 && !f) { D->d.geom = D->d.geomd; break; }
#define UP(field, arr, n) if ((rc = upload(D, &g->field, arr, n, f))) goto out
    UP(xmin, D->xmin, sx + 1); UP(ymin, D->ymin, sy + 1); UP(zmin, D->zmin, sz + 1);
    UP(xmed, D->xmed, sx); UP(ymed, D->ymed, sy); UP(zmed, D->zmed, sz);
    UP(invdiffxmed, D->invdiffxmed, sx); UP(sxi, D->sxi, sx);
    UP(sxj, D->sxj, sy); UP(syj, D->syj, sy); UP(szj, D->szj, sy); UP(invvj, D->invvj, sy);
    UP(sxk, D->sxk, sz); UP(syk, D->syk, sz); UP(szk, D->szk, sz);
    UP(sin_zmed, t_szmed, sz + 1); UP(cos_zmed, t_czmed, sz + 1);
    UP(sin_zmin, t_szmin, sz + 1); UP(cos_zmin, t_czmin, sz + 1);
    UP(cos_xmed, t_cx, sx); UP(sin_xmed, t_sx, sx);
    UP(visc_j, t_visc, sy); UP(viscm_j, t_viscm, sy); UP(tau_j, t_tau, sy);
    UP(r2_j, t_r2, sy); UP(dr2_j, t_dr2, sy); UP(s2_k, t_s2, sz + 1); UP(ds2_k, t_ds2, sz + 1);
    UP(inv_ymed, t_iym, sy); UP(inv_ymin, t_iyi, sy); UP(inv_dymed, t_idy, sy); UP(pot_star, t_pst, sy);
#undef UP
  }
  rc = FB_OK;
out:
  free(t_szmed); free(t_czmed); free(t_szmin); free(t_czmin); free(t_cx); free(t_sx);
  free(t_visc); free(t_viscm); free(t_tau);
  free(t_r2); free(t_dr2); free(t_s2); free(t_ds2);
  free(t_iym); free(t_iyi); free(t_idy); free(t_pst);
  return rc;
}

/* Boundary-template factors (std/boundaries.txt) and Stockholm ramps
 * (stockholm.c:113-129), tabulated with the host libm. */
static int upload_tables(fb_disk *D) {
  const fb_params *p = &D->p;
  int sy = D->d.sy, sz = D->d.sz, ny = p->ny, nz = D->d.nz, s, jj, j, k, kk, rc;
  int n = 18 + 6 * sz + 6 * sy + 6;
  double *t = calloc(n, sizeof(double));
  double ss = p->sigmaslope, fi = p->flaringindex, ar = p->aspectratio;
  double *ramps;
  for (s = 0; s < 2; s++)
    for (jj = 0; jj < 3; jj++) {
      int jgh = s == 0 ? jj : ny + NG + jj, jact = s == 0 ? 2 * NG - jj - 1 : ny + NG - 1 - jj;
      double ya = D->ymed[jact], yg = D->ymed[jgh];
      if (!D->d.is3d) {
        t[s * 3 + jj] = pow(ya / yg, ss);                 /* KEPLERIAN2DDENS */
        t[6 + s * 3 + jj] = sqrt(ya / yg);                /* KEPLERIAN2DVAZIM */
        t[12 + s * 3 + jj] = 1.0;
      } else {
        t[s * 3 + jj] = pow(ya / yg, ss + fi + 1.);      /* KEPLERIAN3DSPHDENSRAD */
        t[6 + s * 3 + jj] = sqrt(ya / yg);                /* KEPLERIAN3DSPHVAZIMRAD */
        t[12 + s * 3 + jj] = (1. + (2. + ss - fi) * (ya - yg) / R0 * fi * ar * ar * pow((yg + ya) / (2. * R0), 2. * fi - 1.));
        for (k = 0; k < sz; k++)
          t[18 + (s * 3 + jj) * sz + k] =
              exp(-pow(cos(D->zmed[k]), 2.) / (ar * ar) * (1. - yg / (.5 * (ya + yg))) * fi * pow(.5 * (yg + ya) / R0, -2. * fi - 1.));
      }
    }
  if (D->d.is3d)
    for (s = 0; s < 2; s++)
      for (kk = 0; kk < 3; kk++) {
        int kgh = s == 0 ? kk : nz + NG + kk, kact = s == 0 ? 2 * NG - kk - 1 : nz + NG - 1 - kk;
        for (j = 0; j < sy; j++)   /* KEPLERIAN3DSPHDENSCOL */
          t[18 + 6 * sz + (s * 3 + kk) * sy + j] =
              pow(sin(D->zmed[kgh]) / sin(D->zmed[kact]), fi - 2. - ss + 1. / (ar * ar) * pow(D->ymed[j] / R0, -2. * fi));
        /* KEPLERIAN3DSPHVAZIMCOL */
        t[18 + 6 * sz + 6 * sy + s * 3 + kk] =
            (1. + fi * cos(.5 * (D->zmed[kgh] + D->zmed[kact])) * (D->zmed[kact] - D->zmed[kgh]));
      }
  rc = upload(D, (const void **)&D->d.bnd_tab, t, n, 0);
  D->d.bnd_tab_n = n;
  free(t);
  if (rc) return rc;
  /* Stockholm ramps */
  ramps = calloc(sy + 2 * sz, sizeof(double));
  {
    double y_inf = p->ymin * pow(p->damping_zone, 2.0 / 3.0), y_sup = p->ymax * pow(p->damping_zone, -2.0 / 3.0);
    double z_inf, z_sup;
    if (!p->spherical) {
      z_inf = p->zmin + (p->zmax - p->zmin) * 0.1;
      z_sup = p->zmax - (p->zmax - p->zmin) * 0.1;
    } else {
      z_inf = M_PI / 2.0 - (M_PI / 2.0 - p->zmin) * (1.0 - p->killing_bc_colatitude);
      z_sup = M_PI / 2.0 + (M_PI / 2.0 - p->zmin) * (1.0 - p->killing_bc_colatitude);
    }
    for (j = 0; j < sy; j++) {
      double r = 0.0, y = D->ymed[j];
      if (y > y_sup) r = (y - y_sup) / (p->ymax - y_sup);
      if (y < y_inf) r = (y_inf - y) / (y_inf - p->ymin);
      ramps[j] = r * r;
    }
    for (k = 0; k < sz && D->d.is3d; k++) {
      double rz = 0.0, rzz = 0.0, z = D->zmed[k], zm = D->zmin[k];
      if (z > z_sup) rz = (z - z_sup) / (p->zmax - z_sup);
      if (z < z_inf) rz = (z_inf - z) / (z_inf - p->zmin);
      if (zm > z_sup) rzz = (zm - z_sup) / (p->zmax - z_sup);
      if (zm < z_inf) rzz = (z_inf - zm) / (z_inf - p->zmin);
      ramps[sy + k] = rz * rz;
      ramps[sy + sz + k] = rzz * rzz;
    }
  }
  rc = upload(D, (const void **)&D->d.ramps, ramps, sy + 2 * sz, 0);
  free(ramps);
  return rc;
}

/* Upper bound of the device bytes fb_disk_create requests for a mesh: the
 * fields (exact) plus the per-row / per-layer tables (bounded). */
int fb_params_bytes(const fb_params *p, int precision, size_t *out) {
  size_t esz, sy, sz, nc, rings, fields, b;
  int is3d;
  if (!p || !out || p->nx < 1 || p->ny < 1 || p->nfluids < 1) return fail(FB_ERR_ARG, "invalid parameters");
  is3d = p->nz > 1;
  esz = precision == FB_FP64 ? sizeof(double) : sizeof(float);
  sy = (size_t)p->ny + 2 * NG;
  sz = is3d ? (size_t)p->nz + 2 * NG : 1;
  nc = (size_t)p->nx * sy * sz;
  rings = sy * sz;
  fields = (is3d ? 15 + 7 : 11) + (p->adiabatic ? 2 : 0);
  b = (size_t)p->nfluids * (fields * nc * esz + 2 * rings * sizeof(double) + rings * sizeof(int) + 4 * rings * esz);
  /* FP32: per-ring azimuthal background and its y / z differences */
  if (precision != FB_FP64) b += (size_t)p->nfluids * rings * (sizeof(double) + 3 * esz);
  b += 2 * sizeof(double) * (6 * ((size_t)p->nx + 1) + 20 * (sy + 1) + 16 * (sz + 1));
  b += sizeof(double) * (18 + 6 * sz + 6 * sy + 6) + sizeof(double) * (sy + 2 * sz);
  b += 64 + sizeof(fb_scalars) + 64 * 16 + sizeof(double) * (2 * rings + 2);
  *out = b;
  return FB_OK;
}

/* Tile choices: azimuthal sweep cells per thread (1, 2, 4, 8, 16 dividing
 * Nx with at most 256 threads per ring; 0 restores the default) and column
 * sweep segment length (4, 8, 16; 0 restores 8). */
#define FB_SMEM_MAX (227 * 1024)

static int default_cx(int nx) {
  const int cs[5] = {4, 8, 16, 2, 1};
  int t;
  for (t = 0; t < 5; t++)
    if (nx % cs[t] == 0 && nx / cs[t] <= 256) return cs[t];
  return 0;
}

int fb_disk_set_tiles(fb_disk *D, int cx, int ns) {
  if (!D) return fail(FB_ERR_ARG, "null disk");
  if (cx != 0 && !((cx == 1 || cx == 2 || cx == 4 || cx == 8 || cx == 16) && D->d.nx % cx == 0 && D->d.nx / cx <= 256))
    return fail(FB_ERR_ARG, "azimuthal chunk %d does not tile Nx = %d in 256 threads", cx, D->d.nx);
  if (cx != 0) {
    /* whole rings per CTA of 256 threads, two buffers of (1 + nq) fields
     * plus the velocity ring, in the sweep's element size: at most 227 KiB */
    size_t rpc = 256 / (D->d.nx / cx), nq = D->d.is3d ? 6 : (D->d.adiabatic ? 5 : 4);
    size_t nxp = (size_t)D->d.nx + 16 / D->esz; /* padded ring row */
    size_t bytes = rpc * nxp * (2 * (1 + nq) + 1) * D->esz;
    if (bytes > FB_SMEM_MAX)
      return fail(FB_ERR_ARG, "azimuthal chunk %d on Nx = %d needs %zu bytes of shared memory", cx, D->d.nx, bytes);
  }
  if (ns != 0 && ns != 4 && ns != 8 && ns != 16) return fail(FB_ERR_ARG, "column segment %d not in {4, 8, 16}", ns);
  D->d.tile_cx = cx;
  D->d.tile_ns = ns;
  return FB_OK;
}

/* Polls of the bounded wait on the azimuthal sweep's staged ring loads
 * before the disk is flagged (failure detection): 0 restores the default,
 * a negative value polls not at all (the wait gives up at once; for tests). */
int fb_disk_set_wait_limit(fb_disk *D, long long polls) {
  if (!D) return fail(FB_ERR_ARG, "null disk");
  D->d.wait_limit = polls;
  return FB_OK;
}

int fb_disk_get_tiles(fb_disk *D, int *cx, int *ns) {
  if (!D) return fail(FB_ERR_ARG, "null disk");
  if (cx) *cx = D->d.tile_cx ? D->d.tile_cx : default_cx(D->d.nx);
  if (ns) *ns = D->d.tile_ns ? D->d.tile_ns : (D->d.precision == FB_FP64 ? 4 : 8);
  return FB_OK;
}

int fb_disk_bytes(fb_disk *D, size_t *out) {
  if (!D || !out) return fail(FB_ERR_ARG, "null argument");
  *out = D->bytes;
  return FB_OK;
}

/* ------------------------------------------------------------------------ */
#define LAUNCH(name, ...) \
  (D->d.precision == FB_FP64 ? fb_launch_##name##_f64(__VA_ARGS__) : fb_launch_##name##_f32(__VA_ARGS__))

/* A batch creating all its members at once lends each one a zeroed region of
 * one batch-wide allocation and the batch's stream: the next fb_disk_create
 * on this thread uses them instead of its own cudaMalloc / stream. */
static __thread char *g_lent_arena = NULL;
static __thread size_t g_lent_size = 0;
static __thread cudaStream_t g_lent_stream = NULL;

void fb_disk_internal_provide(void *arena, size_t size, void *stream) {
  g_lent_arena = (char *)arena;
  g_lent_size = size;
  g_lent_stream = (cudaStream_t)stream;
}

/* device bytes one disk's arena takes: the fields and tables bound plus
 * 256-byte alignment of every carved array */
size_t fb_disk_internal_arena_bytes(const fb_params *p, int precision) {
  size_t est = 0;
  if (fb_params_bytes(p, precision, &est) != FB_OK) return 0;
  return est + (size_t)MAXALLOC * 256;
}

int fb_disk_create(const fb_params *p, int precision, int device, fb_disk **out) {
  fb_disk *D;
  int f, rc, ndev = 0;
  long long nc;
  cudaError_t e;
  *out = NULL;
  if (!p || p->nx < 4 || p->ny < 4) return fail(FB_ERR_ARG, "invalid mesh size");
  if (p->nz > 1 && !p->spherical) return fail(FB_ERR_ARG, "3D meshes are spherical in this library");
  if (p->nz <= 1 && p->spherical) return fail(FB_ERR_ARG, "2D meshes are cylindrical in this library");
  if (p->nplanets < 0 || p->nplanets > FB_MAXPLANETS) return fail(FB_ERR_ARG, "nplanets out of range");
  if (p->nfluids < 1 || p->nfluids > FB_MAXFLUIDS) return fail(FB_ERR_ARG, "nfluids out of range");
  if (p->frame != FB_FRAME_FIXED && p->nplanets < 1) return fail(FB_ERR_ARG, "rotating frame needs a planet");
  if (precision != FB_FP64 && precision != FB_FP32) return fail(FB_ERR_ARG, "precision");
  if (p->adiabatic && (precision != FB_FP64 || p->nz > 1 || p->nfluids != 1 || !(p->gamma > 1.0)))
    return fail(FB_ERR_ARG, "adiabatic disks are FP64, 2D cylindrical, one fluid, with GAMMA > 1");
  if (p->dust_diffusion && (precision != FB_FP64 || p->nz > 1 || p->nfluids < 2))
    return fail(FB_ERR_ARG, "dust diffusion runs on FP64 2D cylindrical disks with dust fluids");
  if (p->slab_ny_global > 0) {
    int n;
    if (p->slab_y0 < 0 || p->slab_y0 + p->ny > p->slab_ny_global || precision != FB_FP64 || p->nfluids != 1)
      return fail(FB_ERR_ARG, "a slab is FP64, one fluid, rows inside [0, slab_ny_global)");
    for (n = 0; n < p->nplanets; n++)
      if (p->pl_feeldisk[n]) return fail(FB_ERR_ARG, "planets that feel the disk need the whole disk");
  }
  e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev <= device || device < 0)
    return fail(FB_ERR_CUDA, "no CUDA device %d available (%s)", device, cudaGetErrorString(e));
  CU(cudaSetDevice(device));
  D = (fb_disk *)calloc(1, sizeof(fb_disk));
  D->p = *p;
  D->device = device;
  D->esz = precision == FB_FP64 ? sizeof(double) : sizeof(float);
  D->d.precision = precision;
  D->d.nx = p->nx; D->d.ny = p->ny;
  D->d.is3d = p->nz > 1;
  D->d.nz = D->d.is3d ? p->nz : 1;
  D->d.sy = p->ny + 2 * NG;
  D->d.sz = D->d.is3d ? p->nz + 2 * NG : 1;
  D->d.pitch = p->nx;
  D->d.stride = (long long)p->nx * D->d.sy;
  D->d.spherical = p->spherical;
  D->d.alpha_visc = p->alpha_visc;
  D->d.xlen = p->xmax - p->xmin;
  D->d.cfl = p->cfl;
  D->d.stockholm = p->stockholm;
  D->d.nfluids = p->nfluids;
  /* collision rates (ColRate with feedback, setups/fargo_multifluid/condinit.c:88-94) */
  for (f = 1; f < p->nfluids; f++) {
    D->d.alpha[0 + f * p->nfluids] = p->invstokes[f - 1];
    D->d.alpha[f + 0 * p->nfluids] = p->invstokes[f - 1];
  }
  D->d.aspectratio = p->aspectratio; D->d.sigmaslope = p->sigmaslope; D->d.flaringindex = p->flaringindex;
  D->d.adiabatic = p->adiabatic;
  D->d.dust_diffusion = p->dust_diffusion;
  D->d.bc_lo = p->slab_ny_global <= 0 || p->slab_y0 == 0;
  D->d.bc_hi = p->slab_ny_global <= 0 || p->slab_y0 + p->ny == p->slab_ny_global;
  D->d.gamma = p->gamma;
  D->ncell = nc = D->d.stride * D->d.sz;
  D->xmin = calloc(p->nx + 1, 8); D->ymin = calloc(D->d.sy + 1, 8); D->zmin = calloc(D->d.sz + 1, 8);
  D->xmed = calloc(p->nx, 8); D->ymed = calloc(D->d.sy, 8); D->zmed = calloc(D->d.sz, 8);
  D->invdiffxmed = calloc(p->nx, 8); D->sxi = calloc(p->nx, 8);
  D->sxj = calloc(D->d.sy, 8); D->syj = calloc(D->d.sy, 8); D->szj = calloc(D->d.sy, 8); D->invvj = calloc(D->d.sy, 8);
  D->sxk = calloc(D->d.sz, 8); D->syk = calloc(D->d.sz, 8); D->szk = calloc(D->d.sz, 8);
  mesh(D);
  D->d.mindx = D->mindx;
  if (g_lent_stream) {
    D->stream = g_lent_stream;
    D->stream_owned = 0;
  } else {
    if (cudaStreamCreateWithFlags(&D->stream, cudaStreamNonBlocking) != cudaSuccess) {
      D->stream = NULL;
      fb_disk_destroy(D);
      return fail(FB_ERR_CUDA, "cudaStreamCreate failed");
    }
    D->stream_owned = 1;
  }
  if (g_lent_arena && g_lent_size >= fb_disk_internal_arena_bytes(p, precision)) {
    D->arena = g_lent_arena;   /* zeroed by the lender */
    D->arena_size = g_lent_size;
    D->arena_owned = 0;
  } else {
    size_t est = fb_disk_internal_arena_bytes(p, precision);
    if (est && cudaMalloc((void **)&D->arena, est) == cudaSuccess && cudaMemsetAsync(D->arena, 0, est, D->stream) == cudaSuccess &&
        cudaStreamSynchronize(D->stream) == cudaSuccess) {
      D->arena_size = est;
      D->arena_owned = 1;
    } else {
      if (D->arena && D->arena_owned) cudaFree(D->arena);
      D->arena = NULL;     /* fall back to one allocation per array */
      cudaGetLastError();
    }
  }
  g_lent_arena = NULL;
  g_lent_size = 0;
  g_lent_stream = NULL;
  if (D->arena) {  /* host image of the table region (tables are carved first) */
    size_t sy = (size_t)D->d.sy, sz = (size_t)D->d.sz;
    D->hstage_size = 2 * sizeof(double) * (6 * ((size_t)p->nx + 1) + 32 * (sy + 1) + 24 * (sz + 1)) +
                     sizeof(double) * (18 + 6 * sz + 6 * sy + 6 + sy + 2 * sz) + (size_t)128 * 256;
    if (D->hstage_size > D->arena_size) D->hstage_size = D->arena_size;
    D->hstage = (char *)calloc(1, D->hstage_size);
    if (!D->hstage) D->hstage_size = 0;
  }
  rc = upload_geometry(D);
  if (!rc) rc = upload_tables(D);
  /* an asynchronous copy from pageable memory has taken the bytes when it
     returns (the image can be freed); a disk on its own stream waits for
     the copy here, a batch's member once for all members (fb_batch_create) */
  if (!rc && D->hstage && D->hstage_hi > 0 &&
      (cudaMemcpyAsync(D->arena, D->hstage, D->hstage_hi, cudaMemcpyHostToDevice, D->stream) != cudaSuccess ||
       (D->stream_owned && cudaStreamSynchronize(D->stream) != cudaSuccess)))
    rc = fail(FB_ERR_CUDA, "table upload");
  free(D->hstage);
  D->hstage = NULL;
  if (rc) { fb_disk_destroy(D); return rc; }
  for (f = 0; f < p->nfluids; f++) {
    fb_fluid_dev *F = &D->d.fl[f];
    size_t fb = D->esz * nc, f2 = sizeof(double) * D->d.sy * D->d.sz, e2 = D->esz * D->d.sy * D->d.sz;
    void **fields[] = {&F->rho, &F->cs, &F->vx, &F->vy, &F->vz, &F->vxt, &F->vyt, &F->vzt,
                       &F->mpx, &F->mmx, &F->mpy, &F->mmy, &F->mpz, &F->mmz, &F->rho_a};
    int i;
    for (i = 0; i < 15; i++) {
      if (!D->d.is3d && (i == 4 || i == 7 || i == 12 || i == 13)) { *fields[i] = NULL; continue; }
      if ((rc = dalloc(D, fields[i], fb))) { fb_disk_destroy(D); return rc; }
    }
    if (D->d.is3d) {
      void **b[] = {&F->mpx_b, &F->mmx_b, &F->mpy_b, &F->mmy_b, &F->mpz_b, &F->mmz_b, &F->rho_b};
      for (i = 0; i < 7; i++)
        if ((rc = dalloc(D, b[i], fb))) { fb_disk_destroy(D); return rc; }
    }
    if ((rc = dalloc(D, (void **)&F->vxmed, f2)) || (rc = dalloc(D, (void **)&F->vxmed_t, f2)) ||
        (rc = dalloc(D, (void **)&F->nshift, sizeof(int) * D->d.sy * D->d.sz)) ||
        (rc = dalloc(D, &F->rho0, e2)) || (rc = dalloc(D, &F->vx0, e2)) || (rc = dalloc(D, &F->vy0, e2)) ||
        (rc = dalloc(D, &F->vz0, e2))) {
      fb_disk_destroy(D);
      return rc;
    }
    if (p->adiabatic && ((rc = dalloc(D, &F->et, fb)) || (rc = dalloc(D, &F->e_a, fb)))) {
      fb_disk_destroy(D);
      return rc;
    }
    if (precision == FB_FP32 &&   /* zero until the first vx arrives (fb_disk_set_state) */
        ((rc = dalloc(D, (void **)&F->vbg, f2)) || (rc = dalloc(D, &F->dlb_y, e2)) || (rc = dalloc(D, &F->dlb_z, e2)) ||
         (rc = dalloc(D, &F->shear_bg, e2)))) {
      fb_disk_destroy(D);
      return rc;
    }
    F->dust = f > 0;
  }
  if ((rc = dalloc(D, (void **)&D->d.dtmin, 64)) || (rc = dalloc(D, (void **)&D->d.scal_dev, sizeof(fb_scalars))) ||
      (rc = dalloc(D, (void **)&D->d.ringsum, sizeof(double) * (2 * (size_t)D->d.sy * D->d.sz + 2)))) {
    fb_disk_destroy(D);
    return rc;
  }
  if (!(D->h_dtmin = pinned_slot())) {
    fb_disk_destroy(D);
    return fail(FB_ERR_CUDA, "pinned host memory");
  }
  for (f = 0; f < p->nplanets; f++) D->feeldisk |= p->pl_feeldisk[f] != 0;
  if (D->feeldisk &&
      ((rc = dalloc(D, (void **)&D->d_ring3, sizeof(double) * 3 * D->d.sy * D->d.sz)) ||
       (rc = dalloc(D, (void **)&D->d_facc, sizeof(double) * 3 * FB_MAXPLANETS)))) {
    fb_disk_destroy(D);
    return rc;
  }
  D->d.feeldisk = D->feeldisk;
  D->d.ring3 = D->d_ring3;
  D->d.facc = D->d_facc;
  fb_psys_init(&D->ps, p->nplanets, p->pl_dist, p->pl_mass, p->pl_feeldisk, p->pl_feelothers, p->eccentricity, p->inclination,
               p->frame, p->omegaframe, p->indirect_term, p->roche_smoothing, p->aspectratio, p->flaringindex,
               p->thickness_smoothing);
  D->sc.nu = p->nu; D->sc.alpha = p->alpha; D->sc.cfl = p->cfl;
  D->sc.omegaframe = D->ps.omegaframe; D->sc.omegaframe0 = D->ps.omegaframe0;
  fb_psys_fill_scalars(&D->ps, &D->sc);
  *out = D;
  return FB_OK;
}

int fb_disk_destroy(fb_disk *D) {
  int i;
  if (!D) return FB_OK;
  if (D->device >= 0) cudaSetDevice(D->device);
  if (D->stream) cudaStreamSynchronize(D->stream);
  for (i = 0; i < D->nalloc; i++) cudaFree(D->allocs[i]);
  if (D->arena && D->arena_owned) cudaFree(D->arena);
  if (D->h_dtmin) pinned_release(D->h_dtmin);
  for (i = 0; i < 32; i++)
    if (D->ev[i]) cudaEventDestroy(D->ev[i]);
  if (D->stream && D->stream_owned) cudaStreamDestroy(D->stream);
  free(D->xmin); free(D->ymin); free(D->zmin); free(D->xmed); free(D->ymed); free(D->zmed);
  free(D->invdiffxmed); free(D->sxi); free(D->sxj); free(D->syj); free(D->szj); free(D->invvj);
  free(D->sxk); free(D->syk); free(D->szk);
  free(D);
  return FB_OK;
}

static int put(fb_disk *D, void *dst, const double *src) {
  size_t n = (size_t)D->ncell;
  if (!src || !dst) return FB_OK;
  if (D->d.precision == FB_FP64) {
    CU(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, D->stream));
  } else {
    float *tmp = (float *)malloc(n * sizeof(float));
    size_t i;
    for (i = 0; i < n; i++) tmp[i] = (float)src[i];
    CU(cudaMemcpyAsync(dst, tmp, n * sizeof(float), cudaMemcpyHostToDevice, D->stream));
    CU(cudaStreamSynchronize(D->stream));
    free(tmp);
  }
  return FB_OK;
}

static int get(fb_disk *D, double *dst, const void *src) {
  size_t n = (size_t)D->ncell;
  if (!src || !dst) return FB_OK;
  if (D->d.precision == FB_FP64) {
    CU(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, D->stream));
    CU(cudaStreamSynchronize(D->stream));
  } else {
    float *tmp = (float *)malloc(n * sizeof(float));
    size_t i;
    CU(cudaMemcpyAsync(tmp, src, n * sizeof(float), cudaMemcpyDeviceToHost, D->stream));
    CU(cudaStreamSynchronize(D->stream));
    for (i = 0; i < n; i++) dst[i] = tmp[i];
    free(tmp);
  }
  return FB_OK;
}

/* Device staging for the state transfers of FP32 disks: one chunk buffer
 * per device (made on first use, kept for the life of the process, guarded
 * by a lock; outside the disks' own arenas).  The caller's doubles are
 * copied into it as they are, a chunk at a time, and rounded to the FP32
 * field by a kernel on the disk's stream (and the reverse for reads), so a
 * page-locked caller buffer moves by DMA with no host-side conversion. */
#define FB_MAXDEV 64
#ifndef DSTAGE_N
#define DSTAGE_N ((size_t)4 << 20) /* doubles per chunk (32 MB) */
#endif
static pthread_mutex_t g_stage_mu = PTHREAD_MUTEX_INITIALIZER;
static double *g_dstage[FB_MAXDEV];

static double *dstage_lock(int device) {
  pthread_mutex_lock(&g_stage_mu);
  if (device < 0 || device >= FB_MAXDEV) {
    pthread_mutex_unlock(&g_stage_mu);
    return NULL;
  }
  if (!g_dstage[device] && cudaMalloc((void **)&g_dstage[device], DSTAGE_N * sizeof(double)) != cudaSuccess) {
    g_dstage[device] = NULL;
    cudaGetLastError();
    pthread_mutex_unlock(&g_stage_mu);
    return NULL;
  }
  return g_dstage[device];
}
static void stage_unlock(void) { pthread_mutex_unlock(&g_stage_mu); }

/* host doubles -> FP32 field (to_f32) or FP32 field -> host doubles */
static int stage_move(fb_disk *D, double *st, double *host, void *field, size_t n, int to_f32) {
  size_t o;
  for (o = 0; o < n; o += DSTAGE_N) {
    size_t c = n - o < DSTAGE_N ? n - o : DSTAGE_N;
    if (to_f32) {
      if (cudaMemcpyAsync(st, host + o, c * sizeof(double), cudaMemcpyHostToDevice, D->stream) != cudaSuccess ||
          fb_launch_convert((float *)field + o, st, c, 1, D->stream) != cudaSuccess)
        return 1;
    } else {
      if (fb_launch_convert(st, (float *)field + o, c, 0, D->stream) != cudaSuccess ||
          cudaMemcpyAsync(host + o, st, c * sizeof(double), cudaMemcpyDeviceToHost, D->stream) != cudaSuccess)
        return 1;
    }
  }
  return 0;
}

int fb_disk_set_state(fb_disk *D, int f, const double *rho, const double *vx, const double *vy, const double *vz,
                      const double *cs) {
  fb_fluid_dev *F;
  int rc = FB_OK, q;
  if (!D || f < 0 || f >= D->p.nfluids) return fail(FB_ERR_ARG, "bad disk/fluid");
  CU(cudaSetDevice(D->device));
  F = &D->d.fl[f];
  if (D->d.precision == FB_FP32) {
    (void)F;
    (void)q;
    return fb_disks_set_state(&D, 1, f, &rho, &vx, &vy, &vz, &cs);
  }
  if ((rc = put(D, F->rho, rho)) || (rc = put(D, F->vx, vx)) || (rc = put(D, F->vy, vy)) ||
      (rc = put(D, F->cs, cs)))
    return rc;
  if (D->d.is3d && (rc = put(D, F->vz, vz))) return rc;
  CU(cudaStreamSynchronize(D->stream));
  return FB_OK;
}

/* Chunked transfers for FP32 disks: the host doubles of many fields (of
 * many disks) are packed back to back into the device staging chunk and
 * converted by one launch per chunk (and the reverse for reads: one launch,
 * then the chunk's copies).  Pieces of a field with a per-ring background
 * end at ring boundaries.  Pieces that lie back to back both in host memory
 * and in the chunk (the fields of disks kept in one host buffer, in the
 * order they are passed) cross in one copy: a DMA costs some microseconds
 * besides its bytes, which dominate for the small fields of small disks. */
typedef struct {
  fb_segs s;
  size_t fill;
  double *st;
  cudaStream_t stream;
  int to_f32;
  double *host[FB_MAXSEG];   /* reads: where each segment's doubles go */
  const double *pend_h;      /* uploads: the host->chunk copy not issued yet */
  size_t pend_off, pend_n;
  /* uploads: ring means of first backgrounds, formed from the chunk at the
     flush (after its copy, before its conversion) */
  struct { double *out; size_t off; int nx, nrings; } rm[FB_MAXSEG];
  int nrm;
} seg_chunk;

static int pend_issue(seg_chunk *c) {
  cudaError_t e;
  if (!c->pend_n) return 0;
  e = cudaMemcpyAsync(c->st + c->pend_off, c->pend_h, c->pend_n * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  c->pend_n = 0;
  return e != cudaSuccess;
}

/* queue n host doubles for chunk offset off, joining the pending copy when
 * both sides continue it */
static int pend_add(seg_chunk *c, const double *h, size_t off, size_t n) {
  if (c->pend_n && c->pend_h + c->pend_n == h && c->pend_off + c->pend_n == off) {
    c->pend_n += n;
    return 0;
  }
  if (pend_issue(c)) return 1;
  c->pend_h = h;
  c->pend_off = off;
  c->pend_n = n;
  return 0;
}

static int chunk_flush(seg_chunk *c) {
  int k, e;
  if (!c->s.n) return 0;
  if (c->to_f32 && pend_issue(c)) return 1;
  for (k = 0; k < c->nrm; k++)
    if (fb_launch_ring_mean(c->rm[k].out, c->st + c->rm[k].off, c->rm[k].nx, c->rm[k].nrings, c->stream)) return 1;
  c->nrm = 0;
  if (fb_launch_convert_segs(c->st, &c->s, c->to_f32, c->stream) != 0) return 1;
  if (!c->to_f32)
    for (k = 0; k < c->s.n; k = e + 1) {
      size_t len = (size_t)c->s.s[k].n;
      for (e = k; e + 1 < c->s.n && c->host[e] + c->s.s[e].n == c->host[e + 1] &&
                  c->s.s[e].off + c->s.s[e].n == c->s.s[e + 1].off;
           e++)
        len += (size_t)c->s.s[e + 1].n;
      if (cudaMemcpyAsync(c->host[k], c->st + c->s.s[k].off, len * sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream) != cudaSuccess)
        return 1;
    }
  c->s.n = 0;
  c->fill = 0;
  return 0;
}

/* n values of one field between host and the FP32 field f; bg: the field's
 * per-ring background (rings of nx values), first_bg: where the ring means of
 * this first upload go (the background is then bg itself) */
static int chunk_add(seg_chunk *c, float *f, double *host, size_t n, const double *bg, int nx, double *first_bg) {
  const size_t unit = bg ? (size_t)nx : 1;
  size_t o = 0;
  if (unit == 0 || unit > DSTAGE_N) return 1;
  while (o < n) {
    size_t room = DSTAGE_N - c->fill, take;
    fb_seg *g;
    room -= room % unit;
    if (room == 0 || c->s.n == FB_MAXSEG) {
      if (chunk_flush(c)) return 1;
      continue;
    }
    take = n - o < room ? n - o : room;
    if (c->to_f32) {
      if (pend_add(c, host + o, c->fill, take)) return 1;
      if (first_bg) {   /* one piece is one segment: the list cannot overflow */
        c->rm[c->nrm].out = first_bg + o / unit;
        c->rm[c->nrm].off = c->fill;
        c->rm[c->nrm].nx = nx;
        c->rm[c->nrm].nrings = (int)(take / unit);
        c->nrm++;
      }
    } else {
      c->host[c->s.n] = host + o;
    }
    g = &c->s.s[c->s.n++];
    g->f = f + o;
    g->bg = bg ? bg + o / unit : NULL;
    g->off = (long long)c->fill;
    g->n = (long long)take;
    g->nx = nx;
    c->fill += take;
    o += take;
  }
  return 0;
}

/* Fluid f's state of n disks that share one stream (the members of a batch):
 * every disk's transfers are queued on that stream (through the one device
 * staging chunk for FP32 disks: the stream orders its reuse) and waited for
 * once, instead of once per disk.  Arrays of n host pointers; a NULL array
 * or entry leaves that field or disk as it is. */
int fb_disks_set_state(fb_disk **ds, int n, int f, const double *const *rho, const double *const *vx,
                       const double *const *vy, const double *const *vz, const double *const *cs) {
  int i, q, rc = FB_OK;
  double *st = NULL;
  if (n <= 0) return FB_OK;
  for (i = 0; i < n; i++)
    if (!ds[i] || f < 0 || f >= ds[i]->p.nfluids || ds[i]->stream != ds[0]->stream ||
        ds[i]->device != ds[0]->device || ds[i]->d.precision != ds[0]->d.precision)
      return fail(FB_ERR_ARG, "disks of one stream, device and precision with fluid %d", f);
  CU(cudaSetDevice(ds[0]->device));
  if (ds[0]->d.precision == FB_FP32 && !(st = dstage_lock(ds[0]->device))) return fail(FB_ERR_CUDA, "device staging");
  {
    seg_chunk c;
    memset(&c, 0, sizeof c);
    c.st = st;
    c.stream = ds[0]->stream;
    c.to_f32 = 1;
    for (i = 0; i < n && !rc; i++) {
      fb_disk *D = ds[i];
      fb_fluid_dev *F = &D->d.fl[f];
      const double *src[5] = {rho ? rho[i] : NULL, vx ? vx[i] : NULL, vy ? vy[i] : NULL,
                              vz && D->d.is3d ? vz[i] : NULL, cs ? cs[i] : NULL};
      void *dst[5] = {F->rho, F->vx, F->vy, F->vz, F->cs};
      for (q = 0; q < 5 && !rc; q++) {
        if (!src[q] || !dst[q]) continue;
        if (st) {
          /* the azimuthal velocity crosses as vx - vbg(ring); the first vx
             given sets the background (its rings' FP64 means) */
          const int bgq = q == 1, first = bgq && !F->has_bg;
          if (bgq && !F->vbg) { rc = fail(FB_ERR_CUDA, "state upload"); break; }
          if (chunk_add(&c, (float *)dst[q], (double *)src[q], (size_t)D->ncell, bgq ? F->vbg : NULL, D->d.nx,
                        first ? F->vbg : NULL))
            rc = fail(FB_ERR_CUDA, "state upload");
          else if (first) {
            F->has_bg = 2;   /* its differences follow the last flush */
          }
        } else if (cudaMemcpyAsync(dst[q], src[q], (size_t)D->ncell * sizeof(double), cudaMemcpyHostToDevice,
                                   D->stream) != cudaSuccess) {
          rc = fail(FB_ERR_CUDA, "state upload");
        }
      }
    }
    if (st && !rc && chunk_flush(&c)) rc = fail(FB_ERR_CUDA, "state upload");
    /* the neighbour differences of the new backgrounds (every ring mean of
       a background is formed by now) */
    for (i = 0; i < n; i++) {
      fb_fluid_dev *F = &ds[i]->d.fl[f];
      if (F->has_bg != 2) continue;
      F->has_bg = 1;
      if (!rc && fb_launch_bg_diffs(&ds[i]->d, f, ds[i]->stream) != cudaSuccess) rc = fail(FB_ERR_CUDA, "state upload");
    }
  }
  if (cudaStreamSynchronize(ds[0]->stream) != cudaSuccess && !rc) rc = fail(FB_ERR_CUDA, "state upload");
  if (st) stage_unlock();
  return rc;
}

int fb_disks_get_state(fb_disk **ds, int n, int f, double *const *rho, double *const *vx, double *const *vy,
                       double *const *vz) {
  int i, q, rc = FB_OK;
  double *st = NULL;
  if (n <= 0) return FB_OK;
  for (i = 0; i < n; i++)
    if (!ds[i] || f < 0 || f >= ds[i]->p.nfluids || ds[i]->stream != ds[0]->stream ||
        ds[i]->device != ds[0]->device || ds[i]->d.precision != ds[0]->d.precision)
      return fail(FB_ERR_ARG, "disks of one stream, device and precision with fluid %d", f);
  CU(cudaSetDevice(ds[0]->device));
  if (ds[0]->d.precision == FB_FP32 && !(st = dstage_lock(ds[0]->device))) return fail(FB_ERR_CUDA, "device staging");
  {
    seg_chunk c;
    memset(&c, 0, sizeof c);
    c.st = st;
    c.stream = ds[0]->stream;
    c.to_f32 = 0;
    for (i = 0; i < n && !rc; i++) {
      fb_disk *D = ds[i];
      fb_fluid_dev *F = &D->d.fl[f];
      double *dst[4] = {rho ? rho[i] : NULL, vx ? vx[i] : NULL, vy ? vy[i] : NULL, vz && D->d.is3d ? vz[i] : NULL};
      void *src[4] = {F->rho, F->vx, F->vy, F->vz};
      for (q = 0; q < 4 && !rc; q++) {
        if (!src[q] || !dst[q]) continue;
        if (st) {
          if (q == 1 && !F->vbg) { rc = fail(FB_ERR_CUDA, "state download"); break; }
          if (chunk_add(&c, (float *)src[q], dst[q], (size_t)D->ncell, q == 1 ? F->vbg : NULL, D->d.nx, NULL))
            rc = fail(FB_ERR_CUDA, "state download");
        } else if (cudaMemcpyAsync(dst[q], src[q], (size_t)D->ncell * sizeof(double), cudaMemcpyDeviceToHost,
                                   D->stream) != cudaSuccess) {
          rc = fail(FB_ERR_CUDA, "state download");
        }
      }
    }
    if (st && !rc && chunk_flush(&c)) rc = fail(FB_ERR_CUDA, "state download");
  }
  if (cudaStreamSynchronize(ds[0]->stream) != cudaSuccess && !rc) rc = fail(FB_ERR_CUDA, "state download");
  if (st) stage_unlock();
  for (i = 0; i < n; i++)
    if (!ds[i]->d.is3d && vz && vz[i]) memset(vz[i], 0, sizeof(double) * ds[i]->ncell);
  return rc;
}

int fb_disk_get_energy(fb_disk *D, int f, double *e) {
  if (!D || !e || f < 0 || f >= D->p.nfluids) return fail(FB_ERR_ARG, "bad disk/fluid");
  CU(cudaSetDevice(D->device));
  if (D->d.precision == FB_FP32) {
    double *st = dstage_lock(D->device);
    int rc = FB_OK;
    if (!st) return fail(FB_ERR_CUDA, "device staging");
    if (stage_move(D, st, e, D->d.fl[f].cs, (size_t)D->ncell, 0) || cudaStreamSynchronize(D->stream) != cudaSuccess)
      rc = fail(FB_ERR_CUDA, "energy download");
    stage_unlock();
    return rc;
  }
  return get(D, e, D->d.fl[f].cs);
}

int fb_disk_get_state(fb_disk *D, int f, double *rho, double *vx, double *vy, double *vz) {
  fb_fluid_dev *F;
  int rc = FB_OK, q;
  if (!D || f < 0 || f >= D->p.nfluids) return fail(FB_ERR_ARG, "bad disk/fluid");
  CU(cudaSetDevice(D->device));
  F = &D->d.fl[f];
  if (D->d.precision == FB_FP32) {
    (void)F;
    (void)q;
    return fb_disks_get_state(&D, 1, f, &rho, &vx, &vy, &vz);
  }
  if ((rc = get(D, rho, F->rho)) || (rc = get(D, vx, F->vx)) || (rc = get(D, vy, F->vy))) return rc;
  if (D->d.is3d && (rc = get(D, vz, F->vz))) return rc;
  if (!D->d.is3d && vz) memset(vz, 0, sizeof(double) * D->ncell);
  return FB_OK;
}

/* ---- FARGO3D output files (output.c) ------------------------------------
 * Merged field files <dir>/<fluid><field><n>.dat (WriteMerging,
 * output.c:283-315): the active cells only, as raw doubles, x fastest, then
 * y, then z; fields dens, energy (the isothermal sound speed, as FARGO3D
 * stores it), vx, vy and, in 3D, vz.  The reader is the inverse (the
 * restart path of LowTasks.c:816-1049 with merged files); it replaces the
 * active cells of the fluid's state and keeps its ghosts. */
static int dat_path(char *buf, size_t n, const char *dir, const char *fluid, const char *field, int num) {
  int k = snprintf(buf, n, "%s%s%s%s%d.dat", dir, (*dir && dir[strlen(dir) - 1] != '/') ? "/" : "", fluid, field, num);
  return k > 0 && (size_t)k < n ? FB_OK : FB_ERR_ARG;
}

static int dat_write(fb_disk *D, const char *path, const double *full) {
  FILE *fo = fopen(path, "wb");
  int j, k, k0 = D->d.is3d ? NG : 0, k1 = D->d.is3d ? D->d.nz + NG : 1;
  if (!fo) return fail(FB_ERR_ARG, "cannot write %s", path);
  for (k = k0; k < k1; k++)
    for (j = NG; j < D->d.ny + NG; j++)
      if (fwrite(full + (size_t)k * D->d.stride + (size_t)j * D->d.pitch, sizeof(double), D->d.nx, fo) != (size_t)D->d.nx) {
        fclose(fo);
        return fail(FB_ERR_ARG, "short write to %s", path);
      }
  fclose(fo);
  return FB_OK;
}

static int dat_read(fb_disk *D, const char *path, double *full) {
  FILE *fi = fopen(path, "rb");
  int j, k, k0 = D->d.is3d ? NG : 0, k1 = D->d.is3d ? D->d.nz + NG : 1;
  if (!fi) return fail(FB_ERR_ARG, "cannot read %s", path);
  for (k = k0; k < k1; k++)
    for (j = NG; j < D->d.ny + NG; j++)
      if (fread(full + (size_t)k * D->d.stride + (size_t)j * D->d.pitch, sizeof(double), D->d.nx, fi) != (size_t)D->d.nx) {
        fclose(fi);
        return fail(FB_ERR_ARG, "%s is shorter than the mesh", path);
      }
  fclose(fi);
  return FB_OK;
}

int fb_disk_write_dat(fb_disk *D, int f, const char *dir, const char *fluid, int num) {
  static const char *names[5] = {"dens", "vx", "vy", "vz", "energy"};
  double *a[5];
  char path[1024];
  int q, rc = FB_OK;
  if (!D || !dir || !fluid || f < 0 || f >= D->p.nfluids) return fail(FB_ERR_ARG, "bad arguments");
  CU(cudaSetDevice(D->device));
  for (q = 0; q < 5; q++) a[q] = (double *)malloc(sizeof(double) * (size_t)D->ncell);
  rc = fb_disk_get_state(D, f, a[0], a[1], a[2], a[3]);
  if (!rc) rc = get(D, a[4], D->d.fl[f].cs);
  for (q = 0; q < 5 && !rc; q++) {
    if (q == 3 && !D->d.is3d) continue;
    if (!(rc = dat_path(path, sizeof path, dir, fluid, names[q], num))) rc = dat_write(D, path, a[q]);
  }
  for (q = 0; q < 5; q++) free(a[q]);
  return rc;
}

int fb_disk_read_dat(fb_disk *D, int f, const char *dir, const char *fluid, int num) {
  static const char *names[5] = {"dens", "vx", "vy", "vz", "energy"};
  double *a[5];
  char path[1024];
  int q, rc = FB_OK;
  if (!D || !dir || !fluid || f < 0 || f >= D->p.nfluids) return fail(FB_ERR_ARG, "bad arguments");
  CU(cudaSetDevice(D->device));
  for (q = 0; q < 5; q++) a[q] = (double *)malloc(sizeof(double) * (size_t)D->ncell);
  rc = fb_disk_get_state(D, f, a[0], a[1], a[2], a[3]);   /* ghosts kept */
  if (!rc) rc = get(D, a[4], D->d.fl[f].cs);
  for (q = 0; q < 5 && !rc; q++) {
    if (q == 3 && !D->d.is3d) continue;
    if (!(rc = dat_path(path, sizeof path, dir, fluid, names[q], num))) rc = dat_read(D, path, a[q]);
  }
  if (!rc) rc = fb_disk_set_state(D, f, a[0], a[1], a[2], D->d.is3d ? a[3] : NULL, a[4]);
  for (q = 0; q < 5; q++) free(a[q]);
  return rc;
}

/* planet<k>.dat lines (WritePlanetFile, output.c:46-75): output number,
 * x, y, z, vx, vy, vz, mass, physical time, OMEGAFRAME. */
int fb_disk_write_planets(fb_disk *D, const char *dir, int num) {
  char path[1024];
  int n;
  if (!D || !dir) return fail(FB_ERR_ARG, "bad arguments");
  for (n = 0; n < D->ps.np; n++) {
    FILE *fo;
    int k = snprintf(path, sizeof path, "%s%splanet%d.dat", dir, (*dir && dir[strlen(dir) - 1] != '/') ? "/" : "", n);
    if (k <= 0 || (size_t)k >= sizeof path) return fail(FB_ERR_ARG, "path too long");
    if (!(fo = fopen(path, "a"))) return fail(FB_ERR_ARG, "cannot append to %s", path);
    fprintf(fo, "%d\t%#.18g\t%#.18g\t%#.18g\t%#.18g\t%#.18g\t%#.18g\t%#.18g\t%#.18g\t%#.18g\n", num, D->ps.px[n],
            D->ps.py[n], D->ps.pz[n], D->ps.pvx[n], D->ps.pvy[n], D->ps.pvz[n], D->ps.pmass[n], D->ps.phys_time,
            D->ps.omegaframe);
    fclose(fo);
  }
  return FB_OK;
}

static int push_scalars(fb_disk *D) {
  D->sc.omegaframe = D->ps.omegaframe;
  D->sc.omegaframe0 = D->ps.omegaframe0;
  CU(cudaMemcpyAsync(D->d.scal_dev, &D->sc, sizeof(fb_scalars), cudaMemcpyHostToDevice, D->stream));
  return FB_OK;
}

/* fb_disk_initialize's work queued on the disk's stream without waiting (a
 * batch initialises all its members this way and waits once) */
int fb_disk_internal_initialize_async(fb_disk *D) {
  int f, rc;
  if (!D) return fail(FB_ERR_ARG, "null disk");
  CU(cudaSetDevice(D->device));
  if ((rc = push_scalars(D))) return rc;
  for (f = 0; f < D->p.nfluids; f++) LCH(LAUNCH(bnd, &D->d, f, 0, D->stream));
  /* init_stockholm (init_stockholm.c:56-105): 2D profiles from column i = 0 */
  for (f = 0; f < D->p.nfluids; f++) {
    fb_fluid_dev *F = &D->d.fl[f];
    void *src[4] = {F->rho, F->vx, F->vy, F->vz}, *dst[4] = {F->rho0, F->vx0, F->vy0, F->vz0};
    int q;
    for (q = 0; q < 4; q++) {
      if (!src[q]) continue;
      CU(cudaMemcpy2DAsync(dst[q], D->esz, src[q], D->esz * D->d.pitch, D->esz, (size_t)D->d.sy * D->d.sz,
                           cudaMemcpyDeviceToDevice, D->stream));
    }
  }
  return FB_OK;
}

int fb_disk_initialize(fb_disk *D) {
  int rc = fb_disk_internal_initialize_async(D);
  if (rc) return rc;
  CU(cudaStreamSynchronize(D->stream));
  return FB_OK;
}

/* Part 1 of a step: ComputeVmed(Vx) + cfl (main.c:366-388), and the disk's
 * pull on the planets that feel it (AdvanceSystemFromDisk's accelerations,
 * planets.c:86-114), from the state at the step's start; the CFL minimum
 * and the failure flags come back to the host. */
int fb_disk_step_begin(fb_disk *D, double *cfl_min) {
  int f, rc;
  const uint64_t start_bits = 0x4415AF1D78B58C40ULL; /* 1e20, the MIN reduction start (define.h:165) */
  if (!D) return fail(FB_ERR_ARG, "null disk");
  CU(cudaSetDevice(D->device));
  CU(cudaMemcpyAsync(D->d.dtmin, &start_bits, 8, cudaMemcpyHostToDevice, D->stream));
  if ((rc = push_scalars(D))) return rc;
  D->nev = 0;
  mark(D, "start");
  for (f = 0; f < D->p.nfluids; f++) LCH(LAUNCH(rowsum, &D->d, f, 0, D->stream));
  mark(D, "rowsum");
  for (f = 0; f < D->p.nfluids; f++) LCH(LAUNCH(cfl, &D->d, f, D->stream));
  mark(D, "cfl");
  if (D->feeldisk) {
    int n;
    for (n = 0; n < D->ps.np; n++) {
      double m = D->ps.pmass[n], x = D->ps.px[n], y = D->ps.py[n], z = D->ps.pz[n], r, sm;
      if (!D->ps.feeldisk[n]) continue;
      r = sqrt(x * x + y * y + z * z);
      if (D->p.roche_smoothing != 0) sm = r * pow(m / 3. / MSTAR, 1. / 3.) * D->p.roche_smoothing;
      else sm = D->p.aspectratio * pow(r / R0, D->p.flaringindex) * r * D->p.thickness_smoothing;
      LCH(LAUNCH(disk_force, &D->d, x, y, z, sm, D->d_ring3, D->d_facc + 3 * n, D->stream));
    }
    CU(cudaMemcpyAsync(D->h_dtmin + 8, D->d_facc, sizeof(double) * 3 * D->ps.np, cudaMemcpyDeviceToHost, D->stream));
    mark(D, "disk_force");
  }
  CU(cudaMemcpyAsync(D->h_dtmin, D->d.dtmin, 16, cudaMemcpyDeviceToHost, D->stream));
  CU(cudaStreamSynchronize(D->stream));
  if (((const uint64_t *)D->h_dtmin)[1] & 2)
    return fail(FB_ERR_NONFINITE, "a staged ring load of the azimuthal sweep did not complete in time");
  if (((const uint64_t *)D->h_dtmin)[1] != 0)
    return fail(FB_ERR_NONFINITE, "non-finite time step or non-positive density in the state");
  if (cfl_min) *cfl_min = D->h_dtmin[0];
  return FB_OK;
}

/* Part 2: CflFluidsMin with the (global) CFL minimum, the DT clip
 * (main.c:388-395) and compute_potential's planetary update
 * (potential.c:10-49), then Sources (algogas.c:30-120) with SubStep3 and the
 * ghost fill of V_temp on the mesh's own edges, the implicit drag
 * (main.c:412-414) and the dust diffusion (main.c:417-419). */
int fb_disk_step_advance(fb_disk *D, double DT, double cfl_min, double *dt_out) {
  int f, rc;
  double dt;
  if (!D) return fail(FB_ERR_ARG, "null disk");
  CU(cudaSetDevice(D->device));
  dt = fb_psys_step(&D->ps, cfl_min, DT, &D->sc, D->feeldisk ? D->h_dtmin + 8 : NULL);
  if (dt < 0.0) return fail(FB_ERR_NULL_DT, "null time step (CFL minimum %g)", cfl_min);
  if ((rc = push_scalars(D))) return rc;
  mark(D, "host_scalars");
  for (f = 0; f < D->p.nfluids; f++) {
    LCH(LAUNCH(sources, &D->d, f, D->stream));
    mark(D, "sources");
    if (D->d.adiabatic) {   /* SubStep3 (algogas.c:82-84), before the ghost fill */
      LCH(LAUNCH(substep3, &D->d, f, D->stream));
      mark(D, "substep3");
    }
    LCH(LAUNCH(bnd, &D->d, f, 1, D->stream));
    mark(D, "bnd_vtemp");
  }
  if (D->p.nfluids > 1) {
    LCH(LAUNCH(collisions, &D->d, D->stream));
    mark(D, "collisions");
  }
  if (D->d.dust_diffusion) {
    for (f = 1; f < D->p.nfluids; f++) LCH(LAUNCH(dust_diffusion, &D->d, f, D->stream));
    mark(D, "dust_diffusion");
  }
  if (dt_out) *dt_out = dt;
  if (D->p.slab_ny_global > 0) CU(cudaStreamSynchronize(D->stream));   /* V_temp is read for the halos */
  return FB_OK;
}

/* Part 3: Transport (algogas.c:135-159), NewVelocity + StockholmBoundary and
 * the ghost fill on the mesh's own edges (main.c:427-431). */
int fb_disk_step_transport(fb_disk *D) {
  int f;
  if (!D) return fail(FB_ERR_ARG, "null disk");
  CU(cudaSetDevice(D->device));
  for (f = 0; f < D->p.nfluids; f++) {
    LCH(LAUNCH(rowsum, &D->d, f, 1, D->stream));
    mark(D, "rowsum_vtemp");
    LCH(LAUNCH(sweep_cols, &D->d, f, D->stream));
    mark(D, "sweep_cols");
    LCH(LAUNCH(sweep_x, &D->d, f, D->stream));
    mark(D, "sweep_x");
  }
  for (f = 0; f < D->p.nfluids; f++) {
    LCH(LAUNCH(newvel, &D->d, f, D->stream));
    mark(D, "newvel");
    LCH(LAUNCH(bnd, &D->d, f, 0, D->stream));
    mark(D, "bnd");
  }
  if (D->prof && D->nev > 1) {
    int i;
    CU(cudaEventSynchronize(D->ev[D->nev - 1]));
    D->prof_n = D->nev - 1;
    for (i = 1; i < D->nev; i++) cudaEventElapsedTime(&D->prof_ms[i - 1], D->ev[i - 1], D->ev[i]);
  }
  if (D->p.slab_ny_global > 0) CU(cudaStreamSynchronize(D->stream));   /* the state is read for the halos */
  return FB_OK;
}

int fb_disk_step(fb_disk *D, double DT, double *dt_out) {
  double cflmin = 0.0;
  int rc = fb_disk_step_begin(D, &cflmin);
  if (!rc) rc = fb_disk_step_advance(D, DT, cflmin, dt_out);
  if (!rc) rc = fb_disk_step_transport(D);
  return rc;
}

/* The fields a halo carries: state (rho, vx, vy[, vz][, energy]) or V_temp
 * (rho, vx_temp, vy_temp[, vz_temp][, energy]) of the disk's one fluid. */
static int halo_fields(fb_disk *D, int which, void **out) {
  const fb_fluid_dev *F = &D->d.fl[0];
  int n = 0;
  out[n++] = F->rho;
  out[n++] = which == FB_HALO_VTEMP ? F->vxt : F->vx;
  out[n++] = which == FB_HALO_VTEMP ? F->vyt : F->vy;
  if (D->d.is3d) out[n++] = which == FB_HALO_VTEMP ? F->vzt : F->vz;
  if (D->d.adiabatic) out[n++] = F->cs;
  return n;
}

int fb_disk_halo_bytes(fb_disk *D, int which, size_t *bytes) {
  void *fl[8];
  if (!D || !bytes || (which != FB_HALO_STATE && which != FB_HALO_VTEMP)) return fail(FB_ERR_ARG, "bad arguments");
  *bytes = (size_t)halo_fields(D, which, fl) * D->d.sz * NG * D->d.nx * D->esz;
  return FB_OK;
}

/* NGHY rows of every halo field, per layer, between the disk and a
 * contiguous buffer [field][layer][3][Nx] (comm.c:197-363 sends the same
 * rows of the primitive fields to the neighbouring domains). */
int fb_disk_halo(fb_disk *D, int which, int side, int unpack, void *buf, int host) {
  void *fl[8];
  int n, q;
  size_t rowb, lay;
  int j0;
  if (!D || !buf || (which != FB_HALO_STATE && which != FB_HALO_VTEMP) || side < 0 || side > 1)
    return fail(FB_ERR_ARG, "bad arguments");
  CU(cudaSetDevice(D->device));
  n = halo_fields(D, which, fl);
  rowb = (size_t)NG * D->d.nx * D->esz;              /* three rows of one layer */
  lay = (size_t)D->d.stride * D->esz;                 /* one layer */
  if (!unpack) j0 = side == 0 ? NG : D->d.ny;         /* the first / last three active rows */
  else j0 = side == 0 ? 0 : D->d.ny + NG;             /* the ghost rows */
  for (q = 0; q < n; q++) {
    char *field = (char *)fl[q] + (size_t)j0 * D->d.pitch * D->esz;
    char *b = (char *)buf + (size_t)q * D->d.sz * rowb;
    enum cudaMemcpyKind kind = unpack ? (host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice)
                                      : (host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice);
    if (unpack) CU(cudaMemcpy2DAsync(field, lay, b, rowb, rowb, D->d.sz, kind, D->stream));
    else CU(cudaMemcpy2DAsync(b, rowb, field, lay, rowb, D->d.sz, kind, D->stream));
  }
  CU(cudaStreamSynchronize(D->stream));
  return FB_OK;
}

int fb_disk_get_scalars(fb_disk *D, double o[8]) {
  if (!D || !o) return fail(FB_ERR_ARG, "null");
  const fb_psys *S = &D->ps;
  o[0] = S->phys_time; o[1] = S->omegaframe; o[2] = S->last_dt;
  o[3] = S->np ? S->px[0] : 0; o[4] = S->np ? S->py[0] : 0;
  o[5] = S->np ? S->pvx[0] : 0; o[6] = S->np ? S->pvy[0] : 0; o[7] = S->domega;
  return FB_OK;
}

/* The planetary system (Sys of psys.c): positions, velocities and masses of
 * the n planets, and the frame rotation.  Setting it replaces the circular
 * orbits built from pl_dist at creation, e.g. when a running simulation hands
 * its state over; getting it keeps the caller's copy current for outputs. */
int fb_disk_set_planets(fb_disk *D, int n, const double *x, const double *y, const double *z, const double *vx,
                        const double *vy, const double *vz, const double *mass, double omegaframe,
                        double omegaframe0) {
  int i;
  if (!D || n != D->ps.np || (n > 0 && (!x || !y || !z || !vx || !vy || !vz || !mass)))
    return fail(FB_ERR_ARG, "planet count %d does not match the disk's %d", n, D ? D->ps.np : -1);
  for (i = 0; i < n; i++) {
    D->ps.px[i] = x[i]; D->ps.py[i] = y[i]; D->ps.pz[i] = z[i];
    D->ps.pvx[i] = vx[i]; D->ps.pvy[i] = vy[i]; D->ps.pvz[i] = vz[i];
    D->ps.pmass[i] = mass[i];
  }
  D->ps.omegaframe = omegaframe;
  D->ps.omegaframe0 = omegaframe0;
  fb_psys_fill_scalars(&D->ps, &D->sc);
  D->sc.omegaframe = omegaframe;
  D->sc.omegaframe0 = omegaframe0;
  return FB_OK;
}

int fb_disk_get_planets(fb_disk *D, int n, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                        double *mass, double *omegaframe) {
  int i;
  if (!D || n != D->ps.np) return fail(FB_ERR_ARG, "planet count mismatch");
  for (i = 0; i < n; i++) {
    if (x) x[i] = D->ps.px[i];
    if (y) y[i] = D->ps.py[i];
    if (z) z[i] = D->ps.pz[i];
    if (vx) vx[i] = D->ps.pvx[i];
    if (vy) vy[i] = D->ps.pvy[i];
    if (vz) vz[i] = D->ps.pvz[i];
    if (mass) mass[i] = D->ps.pmass[i];
  }
  if (omegaframe) *omegaframe = D->ps.omegaframe;
  return FB_OK;
}

int fb_disk_device_fields(fb_disk *D, int f, void *ptrs[5], size_t *esz) {
  if (!D || f < 0 || f >= D->p.nfluids) return fail(FB_ERR_ARG, "bad disk/fluid");
  ptrs[0] = D->d.fl[f].rho; ptrs[1] = D->d.fl[f].vx; ptrs[2] = D->d.fl[f].vy;
  ptrs[3] = D->d.fl[f].vz; ptrs[4] = D->d.fl[f].cs;
  if (esz) *esz = D->esz;
  return FB_OK;
}

/* Total mass of one fluid (ComputeMass, LowTasks.c:709-748): the sum of
 * rho * Vol over the active cells, FP64 with compensation, on the device.
 * Synchronous; a batch member's caller calls fb_batch_sync first. */
int fb_disk_mass(fb_disk *D, int f, double *mass) {
  double *part, *out;
  if (!D || !mass || f < 0 || f >= D->p.nfluids) return fail(FB_ERR_ARG, "bad disk/fluid");
  CU(cudaSetDevice(D->device));
  part = D->d.ringsum;
  out = part + 2 * (size_t)D->d.sy * D->d.sz;
  LCH(LAUNCH(mass, &D->d, f, part, out, D->stream));
  CU(cudaMemcpyAsync(mass, out, sizeof(double), cudaMemcpyDeviceToHost, D->stream));
  CU(cudaStreamSynchronize(D->stream));
  return FB_OK;
}

/* The per-ring azimuthal background of an FP32 fluid ((Nz+6 or 1) x (Ny+6)
 * doubles; zeros for FP64 disks and before the first vx was given). */
int fb_disk_get_background(fb_disk *D, int f, double *out) {
  size_t n;
  if (!D || !out || f < 0 || f >= D->p.nfluids) return fail(FB_ERR_ARG, "bad disk/fluid");
  n = (size_t)D->d.sy * D->d.sz;
  if (!D->d.fl[f].vbg) {
    memset(out, 0, n * sizeof(double));
    return FB_OK;
  }
  CU(cudaSetDevice(D->device));
  CU(cudaMemcpyAsync(out, D->d.fl[f].vbg, n * sizeof(double), cudaMemcpyDeviceToHost, D->stream));
  CU(cudaStreamSynchronize(D->stream));
  return FB_OK;
}

void *fb_disk_stream(fb_disk *D) { return D ? (void *)D->stream : NULL; }

int fb_disk_profile(fb_disk *D, int enable) {
  if (!D) return fail(FB_ERR_ARG, "null disk");
  D->prof = enable;
  return FB_OK;
}

int fb_disk_profile_read(fb_disk *D, float *ms, const char **names, int max) {
  int i, n;
  if (!D) return fail(FB_ERR_ARG, "null disk");
  n = D->prof_n < max ? D->prof_n : max;
  for (i = 0; i < n; i++) {
    ms[i] = D->prof_ms[i];
    names[i] = D->evname[i + 1];
  }
  return n;
}

fb_disk_dev *fb_disk_internal_dev(fb_disk *D) { return &D->d; }
struct fb_psys_s *fb_disk_internal_psys(fb_disk *D) { return &D->ps; }
void *fb_disk_internal_scalars(fb_disk *D) { return &D->sc; }
size_t fb_disk_internal_esz(fb_disk *D) { return D->esz; }
