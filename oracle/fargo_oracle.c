/*
 * fargo_oracle.c -- TEST INFRASTRUCTURE ONLY (see fargo_oracle.h).
 *
 * A CPU restatement of FARGO3D's hydro step (isothermal 2D cylindrical and
 * 3D spherical disks, several fluids with implicit drag, planets feeling the
 * disk; the ADIABATIC equation of state and DUSTDIFFUSION on 2D cylindrical
 * disks), written from the equations and loop bounds of the reference
 * sources.  Each function names the reference
 * file:line it follows (paths relative to the reference's src/ directory).
 * Floating-point expressions keep the reference's evaluation order, including
 * the order implied by its un-parenthesised geometry macros (define.h:226-260),
 * so that the restatement agrees with the reference to the last bit wherever
 * libm agrees with itself.
 */
#include "fargo_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NG FO_NGH
#define CVNR 1.41            /* define.h:9 */
#define G 1.0                /* fondam.h:14,33 (scale-free units) */
#define MSTAR 1.0            /* fondam.h:15,34 */
#define R0 1.0               /* fondam.h:16,35 */
#define SMALLTIME (1e-10 * sqrt(R0 * R0 * R0 / (G * MSTAR))) /* define.h:617 */
#define MAX1D 16384

typedef struct {
  double *rho, *cs, *vx, *vy, *vz;       /* Density, Energy(=cs), Vx, Vy, Vz */
  double *vxt, *vyt, *vzt;               /* Vx_temp, Vy_temp, Vz_temp        */
  double *vxmed;                         /* VxMed (2D)                        */
  double *rho0, *vx0, *vy0, *vz0;        /* Stockholm references (2D)         */
  int dust;                              /* Fluidtype == DUST                 */
} fo_fluid;

struct fo_disk {
  fo_params p;
  int nx, ny, nz, sx, sy, sz, is3d;
  long pitch, stride, ncell;
  /* geometry (LowTasks.c:198-563) */
  double *xmin, *ymin, *zmin, *xmed, *ymed, *zmed, *invdiffxmed;
  double *sxi, *sxj, *syj, *szj, *sxk, *syk, *szk, *invvj;
  double mindx;
  fo_fluid fl[FO_MAXFLUIDS];
  int cur;                               /* FluidIndex                        */
  /* shared scratch fields (LowTasks.c:595-640) */
  double *pres, *pot, *mpx, *mmx, *mpy, *mmy, *mpz, *mmz;
  double *slope, *divrho, *densstar, *qs, *ql, *qr, *totdens;
  double *red2d; int *nshift;
  double *sdiff_c, *sdiff_f;              /* Sdiffyczc, Sdiffyfzc (DUSTDIFFUSION) */
  /* scalars */
  double omegaframe, omegaframe0, phys_time, domega, dtemp, last_dt;
  double minstep[FO_MAXFLUIDS];
  long timestep_count;
  int potential_done_at;
  /* planetary system (psys.c) */
  int np;
  double px[FO_MAXPLANETS], py[FO_MAXPLANETS], pz[FO_MAXPLANETS];
  double pvx[FO_MAXPLANETS], pvy[FO_MAXPLANETS], pvz[FO_MAXPLANETS];
  double pmass[FO_MAXPLANETS];
  int pfeeldisk[FO_MAXPLANETS], pfeelothers[FO_MAXPLANETS];
  double xplanet_mark, yplanet_mark;
  double xaxis_rotation;
  double indirect_x, indirect_y, indirect_z;
};

/* ------------------------------------------------------------------------- */
/* index helpers: define.h:391-458 (NGHX = 0, periodic x inside the kernels) */
#define L(i, j, k) ((long)(i) + (long)(j) * d->pitch + (long)(k) * d->stride)
#define L2D(j, k) ((j) + (k) * d->sy)
static inline long lxp_(const fo_disk *d, int i, long l) { return (i < d->nx - 1) ? l + 1 : l - (d->nx - 1); }
static inline long lxm_(const fo_disk *d, int i, long l) { return (i > 0) ? l - 1 : l + (d->nx - 1); }
static inline int ixm_(const fo_disk *d, int i) { return i > 0 ? i - 1 : d->nx - 1; }
static inline int ixp_(const fo_disk *d, int i) { return i < d->nx - 1 ? i + 1 : 0; }
#define LXP lxp_(d, i, l)
#define LXM lxm_(d, i, l)
#define LYP (l + d->pitch)
#define LYM (l - d->pitch)
#define LZP (l + d->stride)
#define LZM (l - d->stride)

/* geometry macros, CPU flavour (define.h:226-350) */
#define Xmin(i) d->xmin[i]
#define Ymin(j) d->ymin[j]
#define Zmin(k) d->zmin[k]
#define Xmed(i) d->xmed[i]
#define Ymed(j) d->ymed[j]
#define Zmed(k) d->zmed[k]
#define Sxi(i) d->sxi[i]
#define Sxj(j) d->sxj[j]
#define Syj(j) d->syj[j]
#define Szj(j) d->szj[j]
#define Sxk(k) d->sxk[k]
#define Syk(k) d->syk[k]
#define Szk(k) d->szk[k]
#define InvVj(j) d->invvj[j]
#define InvDiffXmed(i) d->invdiffxmed[i]
/* The reference's un-parenthesised macros are expanded in place below
 * wherever evaluation order matters (InvVol, Vol, SurfX/Y/Z). */
static inline double zone_size_x(const fo_disk *d, int i, int j, int k) {
  if (d->p.spherical) return (Sxi(i) * Ymed(j) * sin(Zmed(k)));
  return (Sxi(i) * Ymed(j));
}
static inline double inv_zone_size_xmed(const fo_disk *d, int i, int j, int k) {
  if (d->p.spherical) return (InvDiffXmed(i) / Ymed(j) / sin(Zmed(k)));
  return (InvDiffXmed(i) / Ymed(j));
}
static inline double zone_size_y(const fo_disk *d, int j) { return (Ymin(j + 1) - Ymin(j)); }
static inline double zone_size_z(const fo_disk *d, int j, int k) {
  if (d->p.spherical) return ((Zmin(k + 1) - Zmin(k)) * Ymed(j));
  return (Zmin(k + 1) - Zmin(k));
}
static inline double edge_size_x_middley_lowz(const fo_disk *d, int i, int j, int k) {
  return (Sxi(i) * Ymed(j) * sin(Zmin(k)));
}

static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s);
  if (!p) abort();
  return p;
}

/* ------------------------------------------------------------------------- */
/* InitSpace (LowTasks.c:300-383) and InitSurfaces (LowTasks.c:466-563).      */
static void init_space(fo_disk *d) {
  const fo_params *p = &d->p;
  int i, j, k;
  double dx = (p->xmax - p->xmin) / p->nx;
  double dy = (p->ymax - p->ymin) / p->ny;
  double dz = d->is3d ? (p->zmax - p->zmin) / p->nz : 0.0;
  if (p->log_spacing) {
    dy = (log(p->ymax) - log(p->ymin)) / p->ny;
    for (j = 0; j < d->sy + 1; j++) Ymin(j) = exp(log(p->ymin) + dy * (j - NG));
  } else {
    for (j = 0; j < d->sy + 1; j++) Ymin(j) = p->ymin + dy * (j - NG);
  }
  for (k = 0; k < d->sz + 1; k++) Zmin(k) = d->is3d ? p->zmin + dz * (k - NG) : 0.0;
  for (i = 0; i < d->sx + 1; i++) Xmin(i) = p->xmin + dx * i;
  for (i = 0; i < d->sx; i++) Xmed(i) = 0.5 * (Xmin(i + 1) + Xmin(i));
  for (j = 0; j < d->sy; j++) Ymed(j) = 0.5 * (Ymin(j + 1) + Ymin(j));
  for (k = 0; k < d->sz; k++) Zmed(k) = 0.5 * (Zmin(k + 1) + Zmin(k));
  for (i = 1; i < d->sx; i++) InvDiffXmed(i) = 1. / (Xmed(i) - Xmed(i - 1));
  InvDiffXmed(0) = 1. / (Xmed(0) - (Xmed(d->nx - 1) - (p->xmax - p->xmin)));

  for (i = 0; i < d->sx; i++) Sxi(i) = Xmin(i + 1) - Xmin(i);
  d->mindx = Sxi(0);
  for (i = 1; i < d->sx; i++)
    if (Sxi(i) < d->mindx) d->mindx = Sxi(i);
  if (!p->spherical) { /* CYLINDRICAL */
    for (j = 0; j < d->sy; j++) {
      Sxj(j) = Ymin(j + 1) - Ymin(j);
      Syj(j) = Ymin(j);
      Szj(j) = 0.5 * (Ymin(j + 1) * Ymin(j + 1) - Ymin(j) * Ymin(j));
      InvVj(j) = 1.0 / Szj(j);
    }
    for (k = 0; k < d->sz; k++) {
      Sxk(k) = d->is3d ? Zmin(k + 1) - Zmin(k) : 1.0;
      Syk(k) = Sxk(k);
      Szk(k) = 1.0;
    }
  } else { /* SPHERICAL */
    for (j = 0; j < d->sy; j++) {
      Sxj(j) = 0.5 * (Ymin(j + 1) * Ymin(j + 1) - Ymin(j) * Ymin(j));
      Syj(j) = Ymin(j) * Ymin(j);
      Szj(j) = 0.5 * (Ymin(j + 1) * Ymin(j + 1) - Ymin(j) * Ymin(j));
      InvVj(j) = 3. / ((Ymin(j + 1) * Ymin(j + 1) * Ymin(j + 1) - Ymin(j) * Ymin(j) * Ymin(j)));
    }
    for (k = 0; k < d->sz; k++) {
      Sxk(k) = Zmin(k + 1) - Zmin(k);
      Syk(k) = cos(Zmin(k)) - cos(Zmin(k + 1));
      Szk(k) = sin(Zmin(k));
    }
  }
}

/* ------------------------------------------------------------------------- */
/* Planetary system: InitPlanetarySystem (psys.c:141-225), GetPsysInfo
 * (psys.c:362-415), RotatePsys (psys.c:417-440), RK5 (runge_kutta.c).       */
typedef struct { double e, a, M, E, ta, per, i, an, phi; } orb_t;

static orb_t sv2oe(double x, double y, double z, double vx, double vy, double vz, double m) {
  /* planets.c:116-190 */
  orb_t o;
  double d = sqrt(x * x + y * y + z * z);
  double hx = y * vz - z * vy, hy = z * vx - x * vz, hz = x * vy - y * vx;
  double hhor = sqrt(hx * hx + hy * hy);
  double h2 = hx * hx + hy * hy + hz * hz, h = sqrt(h2);
  double Ax, Ay, Az, e, a, E, V, an, per;
  o.i = asin(hhor / h);
  Ax = vy * hz - vz * hy - G * m * x / d;
  Ay = vz * hx - vx * hz - G * m * y / d;
  Az = vx * hy - vy * hx - G * m * z / d;
  o.e = e = sqrt(Ax * Ax + Ay * Ay + Az * Az) / (G * m);
  o.a = a = h * h / (G * m * (1. - e * e));
  if (e != 0.0) E = acos((1.0 - d / a) / e);
  else E = 0.0;
  if (x * vx + y * vy + z * vz < 0) E = -E;
  if (isnan(E)) E = (d < a) ? 0.0 : M_PI;
  o.M = E - e * sin(E);
  o.E = E;
  if (e > 1.e-14) V = acos((a * (1.0 - e * e) / d - 1.0) / e);
  else V = 0.0;
  if (E < 0.0) V = -V;
  o.ta = V;
  if (fabs(o.i) > 1e-5) {
    an = atan2(hy, hx) + M_PI * .5;
    if (an > 2.0 * M_PI) an -= 2.0 * M_PI;
  } else an = 0.0;
  o.an = an;
  per = acos((Ax * cos(an) + Ay * sin(an)) / sqrt(Ax * Ax + Ay * Ay + Az * Az));
  if ((-hz * sin(an) * Ax + hz * cos(an) * Ay + (hx * sin(an) - hy * cos(an)) * Az) < 0.0)
    per = 2.0 * M_PI - per;
  o.per = per;
  if (Ax * Ax + Ay * Ay > 0.0) o.phi = atan2(Ay, Ax);
  else o.phi = atan2(y, x);
  return o;
}

enum { PS_GET = 0, PS_MARK = 1, PS_FREQUENCY = 2 };
static double get_psys_info(fo_disk *d, int action) {
  double x = d->px[0], y = d->py[0], z = d->pz[0];
  double vx = d->pvx[0], vy = d->pvy[0], vz = d->pvz[0];
  double m = d->pmass[0] + MSTAR, xc = x, yc = y, d1, d2, cross;
  orb_t o = sv2oe(x, y, z, vx, vy, vz, m);
  if (d->p.frame == FO_FRAME_GUIDING) {
    xc = o.a * cos(o.M + o.phi) * cos(o.i);
    yc = o.a * sin(o.M + o.phi) * cos(o.i);
  }
  if (o.e < 1e-8) { xc = x; yc = y; }
  switch (action) {
  case PS_MARK:
    d->xplanet_mark = xc; d->yplanet_mark = yc;
    return 0.;
  case PS_GET:
    x = xc; y = yc;
    d2 = sqrt(x * x + y * y);
    d1 = sqrt(d->xplanet_mark * d->xplanet_mark + d->yplanet_mark * d->yplanet_mark);
    cross = d->xplanet_mark * y - x * d->yplanet_mark;
    d->xplanet_mark = x; d->yplanet_mark = y;
    return asin(cross / (d1 * d2));
  case PS_FREQUENCY:
    if (d->p.frame == FO_FRAME_GUIDING) return sqrt(G * m / pow(o.a, 3.0));
    return (x * vy - y * vx) / (x * x + y * y);
  }
  return 0.0;
}

static void rotate_psys(fo_disk *d, double angle) {
  int i;
  double sint = sin(angle), cost = cos(angle), xt, yt;
  d->xaxis_rotation += angle;
  if (d->xaxis_rotation >= 2.0 * M_PI) d->xaxis_rotation -= 2.0 * M_PI;
  if (d->xaxis_rotation < 0.0) d->xaxis_rotation += 2.0 * M_PI;
  for (i = 0; i < d->np; i++) {
    xt = d->px[i]; yt = d->py[i];
    d->px[i] = xt * cost + yt * sint;
    d->py[i] = -xt * sint + yt * cost;
    xt = d->pvx[i]; yt = d->pvy[i];
    d->pvx[i] = xt * cost + yt * sint;
    d->pvy[i] = -xt * sint + yt * cost;
  }
}

static void rk5_deriv(const fo_disk *d, const double *q, const double *masses, double *der,
                      int n, double dt) {
  /* runge_kutta.c:14-79 */
  const double *x = q, *y = q + n, *z = q + 2 * n, *vx = q + 3 * n, *vy = q + 4 * n, *vz = q + 5 * n;
  double *dx = der, *dy = der + n, *dz = der + 2 * n, *dvx = der + 3 * n, *dvy = der + 4 * n,
         *dvz = der + 5 * n;
  double dist[FO_MAXPLANETS], coef, dd;
  int i, j;
  for (i = 0; i < n; i++) dist[i] = sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
  for (i = 0; i < n; i++) {
    dx[i] = vx[i]; dy[i] = vy[i]; dz[i] = vz[i];
    coef = -G * MSTAR / dist[i] / dist[i] / dist[i];
    dvx[i] = coef * x[i]; dvy[i] = coef * y[i]; dvz[i] = coef * z[i];
    for (j = 0; j < n; j++) {
      if (d->p.indirect_term) {
        coef = G * masses[j] / dist[j] / dist[j] / dist[j];
        dvx[i] -= coef * x[j]; dvy[i] -= coef * y[j]; dvz[i] -= coef * z[j];
      }
      if ((j != i) && d->pfeelothers[i]) {
        dd = (x[i] - x[j]) * (x[i] - x[j]) + (y[i] - y[j]) * (y[i] - y[j]) + (z[i] - z[j]) * (z[i] - z[j]);
        dd = sqrt(dd);
        coef = G * masses[j] / dd / dd / dd;
        dvx[i] += coef * (x[j] - x[i]); dvy[i] += coef * (y[j] - y[i]); dvz[i] += coef * (z[j] - z[i]);
      }
    }
  }
  for (i = 0; i < 6 * n; i++) der[i] *= dt;
}

static void advance_rk5(fo_disk *d, double dt) {
  /* runge_kutta.c:81-145: Cash-Karp fifth-order step */
  int n = d->np, i;
  double q0[6 * FO_MAXPLANETS] = {0}, q1[6 * FO_MAXPLANETS] = {0}, m[FO_MAXPLANETS] = {0};
  double k1[6 * FO_MAXPLANETS], k2[6 * FO_MAXPLANETS], k3[6 * FO_MAXPLANETS];
  double k4[6 * FO_MAXPLANETS], k5[6 * FO_MAXPLANETS], k6[6 * FO_MAXPLANETS];
  if (n == 0) return;
  for (i = 0; i < n; i++) {
    q0[i] = d->px[i]; q0[i + n] = d->py[i]; q0[i + 2 * n] = d->pz[i];
    q0[i + 3 * n] = d->pvx[i]; q0[i + 4 * n] = d->pvy[i]; q0[i + 5 * n] = d->pvz[i];
    m[i] = d->pmass[i];
  }
#define TR(c1, c2, c3, c4, c5) \
  for (i = 0; i < 6 * n; i++) q1[i] = q0[i] + c1 * k1[i] + c2 * k2[i] + c3 * k3[i] + c4 * k4[i] + c5 * k5[i];
  memset(k1, 0, sizeof k1); memset(k2, 0, sizeof k2); memset(k3, 0, sizeof k3);
  memset(k4, 0, sizeof k4); memset(k5, 0, sizeof k5);
  rk5_deriv(d, q0, m, k1, n, dt);
  TR(0.2, 0.0, 0.0, 0.0, 0.0);
  rk5_deriv(d, q1, m, k2, n, dt);
  TR(0.075, 0.225, 0.0, 0.0, 0.0);
  rk5_deriv(d, q1, m, k3, n, dt);
  TR(0.3, -0.9, 1.2, 0.0, 0.0);
  rk5_deriv(d, q1, m, k4, n, dt);
  TR(-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0.0);
  rk5_deriv(d, q1, m, k5, n, dt);
  TR(1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0);
  rk5_deriv(d, q1, m, k6, n, dt);
#undef TR
  for (i = 0; i < 6 * n; i++)
    q1[i] = (q0[i] + 37.0 / 378.0 * k1[i] + 250.0 / 621.0 * k3[i] + 125.0 / 594.0 * k4[i] + 512.0 / 1771.0 * k6[i]);
  /* RELEASEDATE = 0 and PhysicalTime >= 0: every planet is updated. */
  for (i = 0; i < n; i++) {
    d->px[i] = q1[i]; d->py[i] = q1[i + n]; d->pz[i] = q1[i + 2 * n];
    d->pvx[i] = q1[i + 3 * n]; d->pvy[i] = q1[i + 4 * n]; d->pvz[i] = q1[i + 5 * n];
  }
}

/* ------------------------------------------------------------------------- */
/* Reductions: reduction_generic.c:5-23 and reduction_full_generic.c:1-18.   */
static void reduction_sum_rows(fo_disk *d, const double *f, int ymin, int ymax, int zmin, int zmax) {
  int i, j, k;
  for (k = zmin; k < zmax; k++)
    for (j = ymin; j < ymax; j++) {
      d->red2d[L2D(j, k)] = 0.0;
      for (i = 0; i < d->nx; i++) d->red2d[L2D(j, k)] = d->red2d[L2D(j, k)] + f[L(i, j, k)];
    }
}
static double reduction_full_sum(fo_disk *d, const double *f, int ymin, int ymax, int zmin, int zmax) {
  int j, k;
  double r = 0.0;
  reduction_sum_rows(d, f, ymin, ymax, zmin, zmax);
  for (k = zmin; k < zmax; k++)
    for (j = ymin; j < ymax; j++) r = d->red2d[L2D(j, k)] + r;
  return r;
}
static double reduction_full_min(fo_disk *d, const double *f, int ymin, int ymax, int zmin, int zmax) {
  int i, j, k;
  double r = 1e20;
  for (k = zmin; k < zmax; k++)
    for (j = ymin; j < ymax; j++) {
      double m = 1e20;
      for (i = 0; i < d->nx; i++) m = (m < f[L(i, j, k)]) ? m : f[L(i, j, k)];
      d->red2d[L2D(j, k)] = m;
    }
  for (k = zmin; k < zmax; k++)
    for (j = ymin; j < ymax; j++) r = (d->red2d[L2D(j, k)] < r) ? d->red2d[L2D(j, k)] : r;
  return r;
}

/* ComputeVmed (compute_vmed.c:10-39) with ComputeVweight (:42-97). */
static void compute_vmed(fo_disk *d, const double *v) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->sx; i++) d->qs[L(i, j, k)] = v[L(i, j, k)] * (Xmin(i + 1) - Xmin(i));
  reduction_sum_rows(d, d->qs, 0, d->sy, 0, d->sz);
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++) F->vxmed[L2D(j, k)] = d->red2d[L2D(j, k)] / (d->p.xmax - d->p.xmin);
}

/* cfl (cfl.c:10-270), cfl_b (cfl_b.c:3-41). */
static double max2(double a, double b) { return a > b ? a : b; }
static double max3(double a, double b, double c) { return (((a) > (b) ? (a) : (b)) > (c) ? ((a) > (b) ? (a) : (b)) : (c)); }
static void cfl(fo_disk *d) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  int k0 = d->is3d ? NG : 0, k1 = d->is3d ? d->nz + NG : 1;
  for (k = k0; k < k1; k++)
    for (j = NG; j < d->ny + NG; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double vxx = F->vx[l] - F->vxmed[L2D(j, k)];
        double vxxp = F->vx[LXP] - F->vxmed[L2D(j, k)];
        double ss2 = F->cs[l] * F->cs[l], ss, visc, c1a, c1b, c1c = 0.0, c1, c2, c3, c4 = 0.0;
        double c5a, c5b, c5c = 0.0, c5, c7a, c7b, c7c = 0.0, c7;
        const double gm = d->p.gamma;
        if (d->p.alpha_visc && d->p.adiabatic)   /* cfl.c:162-164: cs holds the internal energy */
          visc = d->p.alpha * gm * (gm - 1.0) * F->cs[l] / F->rho[l] * sqrt(Ymed(j) * Ymed(j) * Ymed(j) / (G * MSTAR));
        else if (d->p.alpha_visc)
          visc = d->p.alpha * F->cs[l] * F->cs[l] * sqrt(Ymed(j) * Ymed(j) * Ymed(j) / (G * MSTAR));
        else
          visc = d->p.nu;
        if (d->p.adiabatic) ss2 = gm * (gm - 1) * F->cs[l] / F->rho[l];   /* cfl.c:170-172 */
        ss = sqrt(ss2);
        c1a = ss / zone_size_x(d, i, j, k);
        c1b = ss / zone_size_y(d, j);
        if (d->is3d) c1c = ss / zone_size_z(d, j, k);
        c1 = max3(c1a, c1b, c1c);
        c2 = (max2(fabs(vxx), fabs(vxxp))) / zone_size_x(d, i, j, k);
        c3 = (max2(fabs(F->vy[l]), fabs(F->vy[LYP]))) / zone_size_y(d, j);
        if (d->is3d) c4 = (max2(fabs(F->vz[l]), fabs(F->vz[LZP]))) / zone_size_z(d, j, k);
        c5a = fabs(F->vx[LXP] - F->vx[l]) / zone_size_x(d, i, j, k);
        c5b = fabs(F->vy[LYP] - F->vy[l]) / zone_size_y(d, j);
        if (d->is3d) c5c = fabs(F->vz[LZP] - F->vz[l]) / zone_size_z(d, j, k);
        c5 = max3(c5a, c5b, c5c) * 4.0 * CVNR;
        c7a = 1.0 / zone_size_x(d, i, j, k);
        c7b = 1.0 / zone_size_y(d, j);
        if (d->is3d) c7c = 1.0 / zone_size_z(d, j, k);
        c7 = 4.0 * visc * pow(max3(c7a, c7b, c7c), 2);
        d->densstar[l] = d->p.cfl / sqrt(c1 * c1 + c2 * c2 + c3 * c3 + c4 * c4 + c5 * c5 + 0.0 * 0.0 +
                                          c7 * c7 + 0.0 * 0.0 + 0.0 * 0.0 + 0.0 * 0.0);
      }
  /* cfl_b.c:7-39 */
  d->minstep[d->cur] = reduction_full_min(d, d->densstar, NG, d->ny + NG, k0, k1);
  for (k = k0; k < k1; k++)
    for (j = NG; j < d->ny + NG; j++) {
      double shear = d->p.cfl * d->mindx /
                     fabs(F->vxmed[L2D(j, k)] / Ymed(j) - F->vxmed[L2D(j, k) + 1] / Ymed(j + 1));
      if (shear < d->minstep[d->cur]) d->minstep[d->cur] = shear;
    }
}

/* ComputePressureFieldIso (CompPresIso.c:10-64) or, ADIABATIC,
 * ComputePressureFieldAd (CompPresAd.c:52-53): P = (gamma - 1) e. */
static void pressure(fo_disk *d) {
  fo_fluid *F = &d->fl[d->cur];
  long l;
  if (d->p.adiabatic)
    for (l = 0; l < d->ncell; l++) d->pres[l] = (d->p.gamma - 1.0) * F->cs[l];
  else
    for (l = 0; l < d->ncell; l++) d->pres[l] = F->rho[l] * F->cs[l] * F->cs[l];
}

/* _ComputeForce_cpu (compute_force.c:16-219) for x=y=z=0 (the star): only the
 * "outer" partial sums survive (index < NGHY), which ComputeAccel adds. */
/* ComputeAccel (planets.c:62-84) with _ComputeForce_cpu (compute_force.c:16-219):
 * the gravitational acceleration the disk (Total_Density) exerts at the
 * point (x, y, z) with smoothing rs, as the sum of the inner and outer
 * contributions split at the point's radius (HILLCUT and EXCLUDEHILL off). */
static void compute_accel(fo_disk *d, double x, double y, double z, double rs, double *ax, double *ay, double *az) {
  int i, j, k, k0 = d->is3d ? NG : 0, k1 = d->is3d ? d->nz + NG : 1, index;
  const double *dens = d->totdens;
  double aa, fin[3] = {0.0, 0.0, 0.0}, fout[3] = {0.0, 0.0, 0.0};
  for (k = k0; k < k1; k++)
    for (j = NG; j < d->ny + NG; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double cellmass = Syk(k) * Sxi(i) / InvVj(j) * dens[l];
        double dx, dy, dz, dist2, distance, inv3;
        if (d->p.spherical) {
          dx = Ymed(j) * cos(Xmed(i)) * sin(Zmed(k)) - x;
          dy = Ymed(j) * sin(Xmed(i)) * sin(Zmed(k)) - y;
          dz = Ymed(j) * cos(Zmed(k)) - z;
        } else {
          dx = Ymed(j) * cos(Xmed(i)) - x;
          dy = Ymed(j) * sin(Xmed(i)) - y;
          dz = Zmed(k) - z;
        }
        dist2 = dx * dx + dy * dy + dz * dz;
        dist2 += rs * rs;
        distance = sqrt(dist2);
        inv3 = 1.0 / (dist2 * distance);
        inv3 *= G * cellmass;
        d->mmx[l] = dx * inv3;
        d->mpx[l] = dy * inv3;
        d->mmy[l] = dz * inv3;
        d->mpy[l] = 0.0;            /* fxhi: HILLCUT is not defined */
        d->fl[d->cur].vxt[l] = 0.0; /* fyhi */
        d->fl[d->cur].vyt[l] = 0.0; /* fzhi */
      }
  /* compute_force.c:161-214: inner rings up to the point's radius index */
  aa = sqrt(x * x + y * y + z * z);
  index = (int)(((aa - Ymin(NG)) / (Ymin(d->ny + NG + 1) - Ymin(NG))) * (double)d->ny) + NG;
  if (index >= NG) {
    if (index < d->ny + NG) {
      fin[0] = reduction_full_sum(d, d->mmx, NG, index, k0, k1);
      fin[1] = reduction_full_sum(d, d->mpx, NG, index, k0, k1);
      fin[2] = reduction_full_sum(d, d->mmy, NG, index, k0, k1);
      fout[0] = reduction_full_sum(d, d->mmx, index, d->ny + NG, k0, k1);
      fout[1] = reduction_full_sum(d, d->mpx, index, d->ny + NG, k0, k1);
      fout[2] = reduction_full_sum(d, d->mmy, index, d->ny + NG, k0, k1);
    } else {
      fin[0] = reduction_full_sum(d, d->mmx, NG, d->ny + NG, k0, k1);
      fin[1] = reduction_full_sum(d, d->mpx, NG, d->ny + NG, k0, k1);
      fin[2] = reduction_full_sum(d, d->mmy, NG, d->ny + NG, k0, k1);
    }
  } else {
    fout[0] = reduction_full_sum(d, d->mmx, NG, d->ny + NG, k0, k1);
    fout[1] = reduction_full_sum(d, d->mpx, NG, d->ny + NG, k0, k1);
    fout[2] = reduction_full_sum(d, d->mmy, NG, d->ny + NG, k0, k1);
  }
  *ax = fin[0] + fout[0];
  *ay = fin[1] + fout[1];
  *az = fin[2] + fout[2];
}

/* DiskOnPrimaryAcceleration = ComputeAccel(0, 0, 0, 0, 0) (potential.c:29). */
static void compute_star_accel(fo_disk *d, double *ax, double *ay, double *az) {
  compute_accel(d, 0.0, 0.0, 0.0, 0.0, ax, ay, az);
}

/* AdvanceSystemFromDisk (planets.c:86-114): a planet that feels the disk
 * gets dt times the disk's acceleration at its position (GASINDIRECTTERM
 * off). */
static void advance_system_from_disk(fo_disk *d, double dt) {
  int n;
  for (n = 0; n < d->np; n++) {
    double m, x, y, z, r, smoothing, gx, gy, gz;
    if (!d->pfeeldisk[n]) continue;
    m = d->pmass[n]; x = d->px[n]; y = d->py[n]; z = d->pz[n];
    r = sqrt(x * x + y * y + z * z);
    if (d->p.roche_smoothing != 0) smoothing = r * pow(m / 3. / MSTAR, 1. / 3.) * d->p.roche_smoothing;
    else smoothing = d->p.aspectratio * pow(r / R0, d->p.flaringindex) * r * d->p.thickness_smoothing;
    compute_accel(d, x, y, z, smoothing, &gx, &gy, &gz);
    d->pvx[n] += dt * gx;
    d->pvy[n] += dt * gy;
    d->pvz[n] += dt * gz;
  }
}

/* Potential_cpu (potential.c:51-208), taper = 1 (MASSTAPER = 0). */
static void potential(fo_disk *d) {
  int i, j, k, n;
  double smooth[FO_MAXPLANETS], pdist[FO_MAXPLANETS];
  for (n = 0; n < d->np; n++) {
    double mp = d->pmass[n] * 1.0, rroche, s;
    pdist[n] = sqrt(d->px[n] * d->px[n] + d->py[n] * d->py[n] + d->pz[n] * d->pz[n]);
    rroche = pdist[n] * pow((1.0 / 3.0 * mp / MSTAR), 1.0 / 3.0);
    if (d->p.roche_smoothing != 0) s = rroche * d->p.roche_smoothing;
    else s = d->p.aspectratio * pow(pdist[n] / R0, d->p.flaringindex) * pdist[n] * d->p.thickness_smoothing;
    smooth[n] = s * s;
  }
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->sx; i++) {
        long l = L(i, j, k);
        double XC, YC, ZC, pot;
        if (d->p.spherical) {
          XC = Ymed(j) * cos(Xmed(i)) * sin(Zmed(k));
          YC = Ymed(j) * sin(Xmed(i)) * sin(Zmed(k));
          ZC = Ymed(j) * cos(Zmed(k));
          pot = -G * MSTAR / Ymed(j);
        } else {
          XC = Ymed(j) * cos(Xmed(i));
          YC = Ymed(j) * sin(Xmed(i));
          ZC = Zmed(k);
          pot = -G * MSTAR / sqrt(Ymed(j) * Ymed(j) + ZC * ZC);
        }
        for (n = 0; n < d->np; n++) {
          double mp = d->pmass[n] * 1.0;
          double dist = ((XC - d->px[n]) * (XC - d->px[n]) + (YC - d->py[n]) * (YC - d->py[n]) +
                         (ZC - d->pz[n]) * (ZC - d->pz[n]));
          if (d->p.indirect_term)
            pot += G * mp * (XC * d->px[n] + YC * d->py[n] + ZC * d->pz[n]) / (pdist[n] * pdist[n] * pdist[n]);
          pot += -G * mp / sqrt(dist + smooth[n]);
        }
        d->pot[l] = pot;
      }
}

/* compute_potential (potential.c:10-49). */
static void compute_potential(fo_disk *d, double dt) {
  int i;
  if (d->potential_done_at == d->timestep_count) return;
  if (d->p.frame != FO_FRAME_FIXED) get_psys_info(d, PS_MARK);
  {
    double ax, ay, az;
    compute_star_accel(d, &ax, &ay, &az); /* DiskOnPrimaryAcceleration */
    if (d->p.indirect_term) { d->indirect_x = -ax; d->indirect_y = -ay; d->indirect_z = -az; }
    else { d->indirect_x = d->indirect_y = d->indirect_z = 0.0; }
  }
  potential(d);
  advance_system_from_disk(d, dt);
  for (i = 0; i < 5; i++) advance_rk5(d, 1.0 / ((double)(5)) * dt);
  d->potential_done_at = (int)d->timestep_count;
  if (d->p.frame != FO_FRAME_FIXED) {
    double omeganew = get_psys_info(d, PS_GET) / dt;
    d->domega = omeganew - d->omegaframe;
    d->omegaframe = omeganew;
  }
  rotate_psys(d, d->omegaframe * dt);
}

/* CorrectVtheta_cpu (correct_vtheta.c:10-68). */
static void correct_vtheta(fo_disk *d, double domega) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->sx; i++) {
        if (d->p.spherical) F->vx[L(i, j, k)] -= domega * Ymed(j) * sin(Zmed(k));
        else F->vx[L(i, j, k)] -= domega * Ymed(j);
      }
}

/* SubStep1_x_cpu (substep1_x.c:87-150). */
static void substep1_x(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k, k0 = d->is3d ? 1 : 0, k1 = d->is3d ? d->sz - 1 : 1;
  for (k = k0; k < k1; k++)
    for (j = 1; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxm = LXM;
        double dxmed = 0.5 * (Sxi(i) + Sxi(ixm_(d, i)));
        double dtOVERrhom = 2. * dt / (F->rho[l] * Sxi(i) + F->rho[lxm] * Sxi(ixm_(d, i))) * dxmed;
        F->vxt[l] = F->vx[l];
        if (!F->dust) F->vxt[l] -= dtOVERrhom * (d->pres[l] - d->pres[lxm]) * inv_zone_size_xmed(d, i, j, k);
        F->vxt[l] -= (d->pot[l] - d->pot[lxm]) * dt * inv_zone_size_xmed(d, i, j, k);
      }
}

/* SubStep1_y_cpu (substep1_y.c:123-250). */
static void substep1_y(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k, k0 = d->is3d ? 1 : 0, k1 = d->is3d ? d->sz - 1 : 1;
  for (k = k0; k < k1; k++)
    for (j = 1; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxp = LXP, lym = LYM;
        double dtOVERrhom = 2.0 * dt / (F->rho[l] * (Ymin(j + 1) - Ymin(j)) + F->rho[lym] * (Ymin(j) - Ymin(j - 1))) *
                            (Ymed(j) - Ymed(j - 1));
        double vphi;
        F->vyt[l] = F->vy[l];
        if (!F->dust) F->vyt[l] -= dtOVERrhom * (d->pres[l] - d->pres[lym]) / (Ymed(j) - Ymed(j - 1));
        if (!d->p.spherical) {
          vphi = .25 * (F->vx[l] + F->vx[lxp] + F->vx[lym] + F->vx[lxp - d->pitch]);
          vphi += Ymin(j) * d->omegaframe;
          F->vyt[l] += vphi * vphi / Ymin(j) * dt;
        } else {
          double vzz;
          vphi = .25 * (F->vx[l] + F->vx[lxp] + F->vx[lym] + F->vx[lxp - d->pitch]);
          vphi += Ymin(j) * sin(Zmed(k)) * d->omegaframe;
          vzz = .25 * (F->vz[l] + F->vz[l + d->stride] + F->vz[lym] + F->vz[l + d->stride - d->pitch]);
          F->vyt[l] += (vphi * vphi + vzz * vzz) / Ymin(j) * dt;
        }
        F->vyt[l] -= (d->pot[l] - d->pot[lym]) * dt / (Ymed(j) - Ymed(j - 1));
      }
}

/* SubStep1_z_cpu (substep1_z.c:117-185), SPHERICAL branch. */
static void substep1_z(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 1; k < d->sz - 1; k++)
    for (j = 1; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxp = LXP, lzm = LZM;
        double dtOVERrhom = 2.0 * dt / (F->rho[l] * (Zmin(k + 1) - Zmin(k)) + F->rho[lzm] * (Zmin(k) - Zmin(k - 1))) *
                            (Zmed(k) - Zmed(k - 1));
        double vphi = .25 * (F->vx[l] + F->vx[lxp] + F->vx[lzm] + F->vx[lxp - d->stride]);
        vphi += Ymed(j) * sin(Zmin(k)) * d->omegaframe;
        F->vzt[l] = F->vz[l];
        if (!F->dust) F->vzt[l] -= dtOVERrhom * (d->pres[l] - d->pres[lzm]) / (Ymed(j) * (Zmed(k) - Zmed(k - 1)));
        F->vzt[l] += vphi * vphi * cos(Zmin(k)) / (sin(Zmin(k)) * Ymed(j)) * dt;
        F->vzt[l] -= (d->pot[l] - d->pot[lzm]) * dt / (Ymed(j) * (Zmed(k) - Zmed(k - 1)));
      }
}

/* Viscosity coefficients (visctensor_cyl.c:140-151; visctensor_sph.c). */
static void visc_coeffs(const fo_disk *d, const fo_fluid *F, int i, int j, int k, long l,
                        double *v, double *vm, double *vzm, double *vzmym) {
  if (d->p.alpha_visc && d->p.adiabatic) {
    /* visctensor_cyl.c:146-150: gamma (gamma - 1) e / rho in place of cs^2 */
    const double *e = F->cs, *r = F->rho;
    long lxm = LXM, lym = LYM, lzm = l, lxm_s = lxm, lym_s = lym;
    double a = d->p.alpha, gm = d->p.gamma;
    (void)i;
    (void)k;
    *v = a * gm * (gm - 1.0) * e[l] / r[l] * sqrt(Ymed(j) * Ymed(j) * Ymed(j) / (G * MSTAR));
    *vm = a * gm * (gm - 1.0) * (e[l] + e[lxm] + e[lym] + e[lxm - d->pitch]) /
          (r[l] + r[lxm] + r[lym] + r[lxm - d->pitch]) * sqrt(Ymin(j) * Ymin(j) * Ymin(j) / (G * MSTAR));
    *vzmym = a * gm * (gm - 1.0) * (e[l] + e[lym] + e[lzm] + e[lym_s]) / (r[l] + r[lym] + r[lzm] + r[lym_s]) *
             sqrt(Ymin(j) * Ymin(j) * Ymin(j) / (G * MSTAR));
    *vzm = a * gm * (gm - 1.0) * (e[l] + e[lzm] + e[lxm] + e[lxm_s]) / (r[l] + r[lzm] + r[lxm] + r[lxm_s]) *
           sqrt(Ymed(j) * Ymed(j) * Ymed(j) / (G * MSTAR));
  } else if (d->p.alpha_visc) {
    const double *e = F->cs;
    long lxm = LXM, lym = LYM, lzm = d->is3d ? LZM : l;
    long lxm_s = d->is3d ? lxm - d->stride : lxm, lym_s = d->is3d ? lym - d->stride : lym;
    double a = d->p.alpha;
    (void)i;
    *v = a * e[l] * e[l] * sqrt(Ymed(j) * Ymed(j) * Ymed(j) / (G * MSTAR));
    *vm = a * 0.0625 * (e[l] + e[lxm] + e[lym] + e[lxm - d->pitch]) * (e[l] + e[lxm] + e[lym] + e[lxm - d->pitch]) *
          sqrt(Ymin(j) * Ymin(j) * Ymin(j) / (G * MSTAR));
    if (!d->p.spherical) {
      *vzmym = a * 0.0625 * (e[l] + e[lym] + e[lzm] + e[lym_s]) * (e[l] + e[lym] + e[lzm] + e[lym_s]) *
               sqrt(Ymin(j) * Ymin(j) * Ymin(j) / (G * MSTAR));
      *vzm = a * 0.0625 * (e[l] + e[lzm] + e[lxm] + e[lxm_s]) * (e[l] + e[lzm] + e[lxm] + e[lxm_s]) *
             sqrt(Ymed(j) * Ymed(j) * Ymed(j) / (G * MSTAR));
    } else {
      *vzm = a * 0.0625 * (e[l] + e[lzm] + e[lxm] + e[lxm_s]) * (e[l] + e[lzm] + e[lxm] + e[lxm_s]) *
             sqrt(Ymed(j) * Ymed(j) * Ymed(j) / (G * MSTAR));
      *vzmym = a * 0.0625 * (e[l] + e[lzm] + e[lym] + e[lym_s]) * (e[l] + e[lzm] + e[lym] + e[lym_s]) *
               sqrt(Ymin(j) * Ymin(j) * Ymin(j) / (G * MSTAR));
    }
    (void)k;
  } else {
    *vzmym = *vzm = *vm = *v = d->p.nu;
  }
}

/* visctensor_cyl_cpu (visctensor_cyl.c:134-203) and
 * visctensor_sph_cpu (visctensor_sph.c:131-216). Taus go to Mmx (xx), Mmy (yy),
 * Mmz (zz), Mpx (xz), Mpy (yx), Mpz (zy). */
static void visctensor(fo_disk *d) {
  fo_fluid *F = &d->fl[d->cur];
  const double *rho = F->rho, *vx = F->vx, *vy = F->vy, *vz = F->vz;
  int i, j, k, k0 = d->is3d ? 1 : 0, k1 = d->is3d ? d->sz - 1 : 1;
  for (k = k0; k < k1; k++)
    for (j = 1; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxp = LXP, lxm = LXM, lyp = LYP, lym = LYM;
        double visc, viscm, visczm, visczmym, div_v;
        visc_coeffs(d, F, i, j, k, l, &visc, &viscm, &visczm, &visczmym);
        div_v = 0.0;
        div_v += (vx[lxp] - vx[l]) * Sxj(j) * Sxk(k);
        div_v += (vy[lyp] * Syj(j + 1) * Syk(k) * Sxi(i) - vy[l] * Syj(j) * Syk(k) * Sxi(i));
        if (d->is3d)
          div_v += (vz[LZP] * Szj(j) * Szk(k + 1) * Sxi(i) - vz[l] * Szj(j) * Szk(k) * Sxi(i));
        div_v *= 2.0 / 3.0 * InvVj(j) / (Syk(k) * Sxi(i));
        if (!d->p.spherical) {
          d->mmx[l] = visc * rho[l] * (2.0 * (vx[lxp] - vx[l]) / zone_size_x(d, i, j, k) - div_v);
          d->mmx[l] += visc * rho[l] * (vy[lyp] + vy[l]) / Ymed(j);
          d->mmy[l] = visc * rho[l] * (2.0 * (vy[lyp] - vy[l]) / (Ymin(j + 1) - Ymin(j)) - div_v);
          d->mpy[l] = viscm * .25 * (rho[l] + rho[lxm] + rho[lym] + rho[lxm - d->pitch]) *
                      ((vy[l] - vy[lxm]) * InvDiffXmed(i) / Ymin(j) + (vx[l] - vx[lym]) / (Ymed(j) - Ymed(j - 1)) -
                       .5 * (vx[l] + vx[lym]) / Ymin(j));
        } else {
          long lzp = LZP, lzm = LZM;
          d->mmx[l] = visc * rho[l] * (2.0 * (vx[lxp] - vx[l]) / zone_size_x(d, i, j, k) - div_v);
          d->mmx[l] += visc * rho[l] * (vy[lyp] + vy[l]) / Ymed(j);
          d->mmx[l] += visc * rho[l] * (vz[lzp] + vz[l]) * cos(Zmed(k)) / (sin(Zmed(k)) * Ymed(j));
          d->mmy[l] = visc * rho[l] * (2.0 * (vy[lyp] - vy[l]) / (Ymin(j + 1) - Ymin(j)) - div_v);
          d->mmz[l] = visc * rho[l] * (2.0 * (vz[lzp] - vz[l]) / (Ymed(j) * (Zmin(k + 1) - Zmin(k))) - div_v);
          d->mmz[l] += visc * rho[l] * (vy[l] + vy[lyp]) / Ymed(j);
          d->mpx[l] = visczm * .25 * (rho[l] + rho[lzm] + rho[lxm] + rho[lxm - d->stride]) *
                      ((vx[l] / sin(Zmed(k)) - vx[lzm] / sin(Zmed(k - 1))) * sin(Zmin(k)) / (Ymed(j) * (Zmed(k) - Zmed(k - 1))) +
                       ((vz[l] - vz[lxm]) * InvDiffXmed(i) / (sin(Zmin(k)) * Ymed(j))));
          d->mpy[l] = viscm * .25 * (rho[l] + rho[lxm] + rho[lym] + rho[lxm - d->pitch]) *
                      ((vy[l] - vy[lxm]) * InvDiffXmed(i) / (Ymin(j) * sin(Zmed(k))) +
                       (vx[l] - vx[lym]) / (Ymed(j) - Ymed(j - 1)) - .5 * (vx[l] + vx[lym]) / Ymin(j));
          d->mpz[l] = visczmym * .25 * (rho[l] + rho[lym] + rho[lzm] + rho[lym - d->stride]) *
                      ((vz[l] - vz[lym]) / (Ymed(j) - Ymed(j - 1)) - .5 * (vz[l] + vz[lym]) / Ymin(j) +
                       (vy[l] - vy[lzm]) / (Ymin(j) * (Zmed(k) - Zmed(k - 1))));
        }
      }
}

/* addviscosity_cyl_cpu (addviscosity_cyl.c:74-140),
 * addviscosity_sph_cpu (addviscosity_sph.c). */
static void addviscosity(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  const double *rho = F->rho;
  double *vx = F->vxt, *vy = F->vyt, *vz = F->vzt;
  const double *txx = d->mmx, *tyy = d->mmy, *tzz = d->mmz, *txz = d->mpx, *tyx = d->mpy, *tzy = d->mpz;
  int i, j, k, k0 = d->is3d ? 1 : 0, k1 = d->is3d ? d->sz - 2 : 1;
  for (k = k0; k < k1; k++)
    for (j = 1; j < d->sy - 2; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxp = LXP, lxm = LXM, lyp = LYP, lym = LYM;
        if (!d->p.spherical) {
          vx[l] += 2.0 * (txx[l] - txx[lxm]) * inv_zone_size_xmed(d, i, j, k) / ((rho[l] + rho[lxm])) * dt;
          vx[l] += 2.0 * (Ymin(j + 1) * Ymin(j + 1) * tyx[lyp] - Ymin(j) * Ymin(j) * tyx[l]) /
                   ((Ymin(j + 1) - Ymin(j)) * Ymed(j) * Ymed(j) * (rho[lxm] + rho[l])) * dt;
          vy[l] += 2.0 * (Ymed(j) * tyy[l] - Ymed(j - 1) * tyy[lym]) /
                   ((Ymed(j) - Ymed(j - 1)) * (rho[l] + rho[lym]) * Ymin(j)) * dt;
          vy[l] += 2.0 * (tyx[lxp] - tyx[l]) / ((Xmin(i + 1) - Xmin(i)) * Ymin(j) * (rho[l] + rho[lym])) * dt;
          vy[l] -= (txx[l] + txx[lym]) / (Ymin(j) * (rho[l] + rho[lym])) * dt;
        } else {
          long lzp = LZP, lzm = LZM;
          vx[l] += 2.0 * (txx[l] - txx[lxm]) * inv_zone_size_xmed(d, i, j, k) / ((rho[l] + rho[lxm])) * dt;
          vx[l] += 2.0 * (Ymin(j + 1) * Ymin(j + 1) * tyx[lyp] - Ymin(j) * Ymin(j) * tyx[l]) /
                   ((Ymin(j + 1) - Ymin(j)) * Ymed(j) * Ymed(j) * (rho[lxm] + rho[l])) * dt;
          vx[l] += (tyx[lyp] + tyx[l]) / ((rho[lxm] + rho[l]) * Ymed(j)) * dt;
          vx[l] += 2.0 * (txz[lzp] - txz[l]) / (zone_size_z(d, j, k) * (rho[lxm] + rho[l])) * dt;
          vx[l] += 2.0 * (txz[lzp] + txz[l]) * cos(Zmed(k)) / (sin(Zmed(k)) * Ymed(j) * (rho[lxm] + rho[l])) * dt;

          vy[l] += 2.0 * (Ymed(j) * Ymed(j) * tyy[l] - Ymed(j - 1) * Ymed(j - 1) * tyy[lym]) /
                   ((Ymed(j) - Ymed(j - 1)) * (rho[l] + rho[lym]) * Ymin(j) * Ymin(j)) * dt;
          vy[l] += 2.0 * (tyx[lxp] - tyx[l]) /
                   ((Xmin(i + 1) - Xmin(i)) * Ymin(j) * sin(Zmed(k)) * (rho[l] + rho[lym])) * dt;
          vy[l] -= (txx[l] + txx[lym]) / (Ymin(j) * (rho[l] + rho[lym])) * dt;
          vy[l] -= (tzz[l] + tzz[lym]) / (Ymin(j) * (rho[l] + rho[lym])) * dt;
          vy[l] += 2.0 * (tzy[lzp] * sin(Zmin(k + 1)) - tzy[l] * sin(Zmin(k))) /
                   ((Zmin(k + 1) - Zmin(k)) * Ymin(j) * sin(Zmed(k)) * (rho[l] + rho[lym])) * dt;

          vz[l] += 2.0 * (tzz[l] * sin(Zmed(k)) - tzz[lzm] * sin(Zmed(k - 1))) /
                   ((Zmed(k) - Zmed(k - 1)) * Ymed(j) * sin(Zmin(k)) * (rho[l] + rho[lzm])) * dt;
          vz[l] += 2.0 * (txz[lxp] - txz[l]) / (edge_size_x_middley_lowz(d, i, j, k) * (rho[l] + rho[lzm])) * dt;
          vz[l] += 2.0 * (Ymin(j + 1) * Ymin(j + 1) * Ymin(j + 1) * tzy[lyp] - Ymin(j) * Ymin(j) * Ymin(j) * tzy[l]) /
                   ((Ymin(j + 1) - Ymin(j)) * Ymed(j) * Ymed(j) * Ymed(j) * (rho[l] + rho[lzm])) * dt;
          vz[l] -= (txx[l] + txx[lzm]) * cos(Zmin(k)) / (Ymed(j) * sin(Zmin(k)) * (rho[l] + rho[lzm])) * dt;
        }
      }
}

/* SubStep2_a_cpu (substep2_a.c:90-165): artificial viscous pressure q into
 * Mpx, Mpy, Mpz, computed from the velocity at the start of the step. */
static void substep2_a(fo_disk *d) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k, k1 = d->is3d ? d->sz - 1 : 1;
  const double c2 = CVNR * CVNR;
  for (k = 0; k < k1; k++)
    for (j = 0; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double dvx = F->vx[LXP] - F->vx[l], dvy = F->vy[LYP] - F->vy[l];
        (void)c2;
        d->mpx[l] = (dvx < 0.0) ? CVNR * CVNR * F->rho[l] * dvx * dvx : 0.0;
        d->mpy[l] = (dvy < 0.0) ? CVNR * CVNR * F->rho[l] * dvy * dvy : 0.0;
        if (d->is3d) {
          double dvz = F->vz[LZP] - F->vz[l];
          d->mpz[l] = (dvz < 0.0) ? CVNR * CVNR * F->rho[l] * dvz * dvz : 0.0;
        }
      }
}

/* SubStep2_b_cpu (substep2_b.c:130-200). */
static void substep2_b(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k, k0 = d->is3d ? 1 : 0, k1 = d->is3d ? d->sz - 1 : 1;
  for (k = k0; k < k1; k++)
    for (j = 1; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxm = LXM, lym = LYM;
        double dxrho1 = Sxi(i), dxrho2 = Sxi(ixm_(d, i)), dxmed = 0.5 * (Sxi(i) + Sxi(ixm_(d, i)));
        double dyrho1 = Ymin(j + 1) - Ymin(j), dyrho2 = Ymin(j) - Ymin(j - 1);
        F->vxt[l] += -2.0 * dt * dxmed * (d->mpx[l] - d->mpx[lxm]) / (F->rho[l] * dxrho1 + F->rho[lxm] * dxrho2) *
                     inv_zone_size_xmed(d, i, j, k);
        if (d->p.adiabatic)   /* substep2_b.c:161-163: the artificial viscosity's heating */
          F->cs[l] += -dt * (d->mpx[l] * (F->vx[LXP] - F->vx[l]) / zone_size_x(d, i, j, k));
        F->vyt[l] += -2.0 * (d->mpy[l] - d->mpy[lym]) / (F->rho[l] * dyrho1 + F->rho[lym] * dyrho2) * dt;
        if (d->p.adiabatic)   /* substep2_b.c:176-178 */
          F->cs[l] += -dt * (d->mpy[l] * (F->vy[LYP] - F->vy[l]) / zone_size_y(d, j));
        if (d->is3d) {
          long lzm = LZM;
          double dzmed = Zmed(k) - Zmed(k - 1), dzrho1 = Zmin(k + 1) - Zmin(k), dzrho2 = Zmin(k) - Zmin(k - 1);
          F->vzt[l] += -2.0 * dzmed * (d->mpz[l] - d->mpz[lzm]) / (F->rho[l] * dzrho1 + F->rho[lzm] * dzrho2) * dt /
                       (Ymed(j) * (Zmed(k) - Zmed(k - 1)));
        }
      }
}

/* SubStep3_cpu (substep3.c:79-118), ADIABATIC: the compressional heating
 * -P div v, implicit in e, with the velocities after the source terms. */
static void substep3(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  const double *vx = F->vxt, *vy = F->vyt;
  const double gm = d->p.gamma;
  int i, j, k = 0;
  for (j = 0; j < d->sy - 1; j++)
    for (i = 0; i < d->nx; i++) {
      long l = L(i, j, k);
      double div_v = 0.0, term;
      div_v += (vx[LXP] - vx[l]) * Sxj(j) * Sxk(k);
      div_v += (vy[LYP] * Syj(j + 1) * Syk(k) * Sxi(i) - vy[l] * Syj(j) * Syk(k) * Sxi(i));
      term = 0.5 * dt * (gm - 1.) * div_v * InvVj(j) / (Syk(k) * Sxi(i));
      F->cs[l] *= (1.0 - term) / (1.0 + term);
    }
}

/* ------------------------------------------------------------------------- */
/* Ghost boundaries: the code FARGO3D generates from std/boundaries.txt and
 * the setups' .bound files (scripts/boundparser.py:360-398 index rules):
 *   2D: fargo.bound (KEPLERIAN2DDENS, KEPLERIAN2DVAZIM, ANTISYMMETRIC vr)
 *   3D: p3disof.bound (KEPLERIAN3DSPH*, SYMMETRIC / ANTISYMMETRIC)         */
static void boundary_z(fo_disk *d, int up) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k, nz = d->nz, nghz = NG;
  double fi = d->p.flaringindex, ss = d->p.sigmaslope, ar = d->p.aspectratio, of = d->omegaframe;
  for (k = 0; k < nghz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->sx; i++) {
        long lgh, lghs, lact, lacts, lnull;
        int kgh, kact;
        if (!up) {
          lgh = L(i, j, k); lghs = lgh;
          lact = L(i, j, 2 * nghz - k - 1); lacts = L(i, j, 2 * nghz - k);
          lnull = L(i, j, nghz);
          kgh = k; kact = 2 * nghz - k - 1;
        } else {
          lgh = L(i, j, nz + nghz + k); lghs = L(i, j, nz + nghz + 1 + k);
          lact = L(i, j, nz + nghz - 1 - k); lacts = lact;
          lnull = L(i, j, nz + nghz);
          kgh = nz + nghz + k; kact = nz + nghz - 1 - k;
        }
        /* Density: KEPLERIAN3DSPHDENSCOL */
        F->rho[lgh] = F->rho[lact] * pow(sin(Zmed(kgh)) / sin(Zmed(kact)),
                                        fi - 2. - ss + 1. / (ar * ar) * pow(Ymed(j) / R0, -2. * fi));
        /* Vx: KEPLERIAN3DSPHVAZIMCOL */
        F->vx[lgh] = (F->vx[lact] + of * Ymed(j) * sin(Zmed(kact))) *
                         (1. + fi * cos(.5 * (Zmed(kgh) + Zmed(kact))) * (Zmed(kact) - Zmed(kgh))) -
                     Ymed(j) * of * sin(Zmed(kgh));
        /* Vy: SYMMETRIC (centred in z) */
        F->vy[lgh] = F->vy[lact];
        /* Vz: ANTISYMMETRIC (staggered in z) */
        if (!up) F->vz[lghs] = -F->vz[lacts];
        else if (k < nghz - 1) F->vz[lghs] = -F->vz[lacts];
        F->vz[lnull] = 0;
      }
}

static void boundary_y(fo_disk *d, int right) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k, ny = d->ny, nghy = NG;
  double ss = d->p.sigmaslope, fi = d->p.flaringindex, ar = d->p.aspectratio, of = d->omegaframe;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < nghy; j++)
      for (i = 0; i < d->sx; i++) {
        long lgh, lghs, lact, lacts, lnull;
        int jgh, jact;
        if (!right) {
          lgh = L(i, j, k); lghs = lgh;
          lact = L(i, 2 * nghy - j - 1, k); lacts = L(i, 2 * nghy - j, k);
          lnull = L(i, nghy, k);
          jgh = j; jact = 2 * nghy - j - 1;
        } else {
          lgh = L(i, ny + nghy + j, k); lghs = L(i, ny + nghy + 1 + j, k);
          lact = L(i, ny + nghy - 1 - j, k); lacts = lact;
          lnull = L(i, ny + nghy, k);
          jgh = ny + nghy + j; jact = ny + nghy - 1 - j;
        }
        if (!d->is3d) {
          /* KEPLERIAN2DDENS, KEPLERIAN2DVAZIM, ANTISYMMETRIC */
          F->rho[lgh] = F->rho[lact] * pow(Ymed(jact) / Ymed(jgh), ss);
          F->vx[lgh] = (F->vx[lact] + Ymed(jact) * of) * sqrt(Ymed(jact) / Ymed(jgh)) - Ymed(jgh) * of;
          /* ADIABATIC: the energy's ghosts mirror the active cells (SYMMETRIC,
             std/boundaries.txt), the oracle's adiabatic variant of fargo.bound */
          if (d->p.adiabatic) F->cs[lgh] = F->cs[lact];
        } else {
          /* KEPLERIAN3DSPHDENSRAD, KEPLERIAN3DSPHVAZIMRAD */
          F->rho[lgh] = F->rho[lact] * pow(Ymed(jact) / Ymed(jgh), ss + fi + 1.) *
                        exp(-pow(cos(Zmed(k)), 2.) / (ar * ar) * (1. - Ymed(jgh) / (.5 * (Ymed(jact) + Ymed(jgh)))) * fi *
                            pow(.5 * (Ymed(jgh) + Ymed(jact)) / R0, -2. * fi - 1.));
          F->vx[lgh] = (F->vx[lact] + of * Ymed(jact) * sin(Zmed(k))) * sqrt(Ymed(jact) / Ymed(jgh)) *
                           (1. + (2. + ss - fi) * (Ymed(jact) - Ymed(jgh)) / R0 * fi * ar * ar *
                                     pow((Ymed(jgh) + Ymed(jact)) / (2. * R0), 2. * fi - 1.)) -
                       Ymed(jgh) * of * sin(Zmed(k));
          /* Vz: SYMMETRIC (centred in y) */
          F->vz[lgh] = F->vz[lact];
        }
        if (!right) F->vy[lghs] = -F->vy[lacts];
        else if (j < nghy - 1) F->vy[lghs] = -F->vy[lacts];
        F->vy[lnull] = 0;
      }
}

/* FillGhosts (algogas.c:11-27) -> boundaries() (boundary.c:2-22). */
static void fill_ghosts(fo_disk *d) {
  if (d->is3d) { boundary_z(d, 0); boundary_z(d, 1); }
  boundary_y(d, 0);
  boundary_y(d, 1);
}

/* ------------------------------------------------------------------------- */
/* Transport (transport.c) */
static void momenta_x(fo_disk *d) { /* momenta_x.c:55-90 */
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxp = LXP;
        if (!d->p.spherical) {
          d->mmx[l] = (F->vxt[l] + Ymed(j) * d->omegaframe) * Ymed(j) * F->rho[l];
          d->mpx[l] = (F->vxt[lxp] + Ymed(j) * d->omegaframe) * Ymed(j) * F->rho[l];
        } else {
          double rcyl = Ymed(j) * sin(Zmed(k));
          d->mmx[l] = (F->vxt[l] + rcyl * d->omegaframe) * rcyl * F->rho[l];
          d->mpx[l] = (F->vxt[lxp] + rcyl * d->omegaframe) * rcyl * F->rho[l];
        }
      }
}
static void momenta_y(fo_disk *d) { /* momenta_y.c:49-69 */
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        d->mmy[l] = F->vyt[l] * F->rho[l];
        d->mpy[l] = F->vyt[LYP] * F->rho[l];
      }
}
static void momenta_z(fo_disk *d) { /* momenta_z.c:51-70 */
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 0; k < d->sz - 1; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        d->mpz[l] = F->vzt[LZP] * F->rho[l];
        d->mmz[l] = F->vzt[l] * F->rho[l];
        if (d->p.spherical) { d->mpz[l] *= Ymed(j); d->mmz[l] *= Ymed(j); }
      }
}
static void divide_by_rho(fo_disk *d, const double *q) { /* divrho.c:37-60 */
  fo_fluid *F = &d->fl[d->cur];
  long l;
  for (l = 0; l < d->ncell; l++) d->divrho[l] = q[l] / F->rho[l];
}

static void vanleer_y_a(fo_disk *d, const double *q) { /* vanleer_y_a.c:49-74 */
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 1; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double dqm = (q[l] - q[LYM]) / zone_size_y(d, j);
        double dqp = (q[LYP] - q[l]) / zone_size_y(d, j + 1);
        if (dqp * dqm <= 0) d->slope[l] = 0;
        else d->slope[l] = 2. * dqp * dqm / (dqm + dqp);
      }
}
static void vanleer_y_b(fo_disk *d, double dt, const double *q, double *qs) { /* vanleer_y_b.c:50-73 */
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 1; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        if (F->vyt[l] > 0.)
          qs[l] = q[LYM] + 0.5 * (zone_size_y(d, j - 1) - F->vyt[l] * dt) * d->slope[LYM];
        else
          qs[l] = q[l] - 0.5 * (zone_size_y(d, j) + F->vyt[l] * dt) * d->slope[l];
      }
}
static void update_y(fo_disk *d, double dt, double *qb, const double *qs, int density) {
  /* update_y.c:56-80, update_density_y.c:54-78 */
  fo_fluid *F = &d->fl[d->cur];
  const double *vy = F->vyt, *rs = d->densstar;
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lyp = LYP;
        if (!density)
          qb[l] += (vy[l] * qs[l] * rs[l] * Syj(j) * Syk(k) * Sxi(i) -
                    vy[lyp] * qs[lyp] * rs[lyp] * Syj(j + 1) * Syk(k) * Sxi(i)) *
                   dt * InvVj(j) / (Syk(k) * Sxi(i));
        else
          qb[l] += (vy[l] * rs[l] * Syj(j) * Syk(k) * Sxi(i) - vy[lyp] * rs[lyp] * Syj(j + 1) * Syk(k) * Sxi(i)) *
                   dt * InvVj(j) / (Syk(k) * Sxi(i));
      }
}
static void transport_y(fo_disk *d, double *q, double dt) { /* transport.c:24-34 */
  fo_fluid *F = &d->fl[d->cur];
  if (q != F->rho) {
    divide_by_rho(d, q);
    vanleer_y_a(d, d->divrho);
    vanleer_y_b(d, dt, d->divrho, d->qs);
    update_y(d, dt, q, d->qs, 0);
  } else {
    update_y(d, dt, q, NULL, 1);
  }
}

static void vanleer_z_a(fo_disk *d, const double *q) { /* vanleer_z_a.c:49-74 */
  int i, j, k;
  for (k = 1; k < d->sz - 1; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double dqm = (q[l] - q[LZM]) / zone_size_z(d, j, k);
        double dqp = (q[LZP] - q[l]) / zone_size_z(d, j, k + 1);
        if (dqp * dqm <= 0) d->slope[l] = 0;
        else d->slope[l] = 2. * dqp * dqm / (dqm + dqp);
      }
}
static void vanleer_z_b(fo_disk *d, double dt, const double *q, double *qs) { /* vanleer_z_b.c:50-73 */
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 1; k < d->sz - 1; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        if (F->vzt[l] > 0.)
          qs[l] = q[LZM] + 0.5 * (zone_size_z(d, j, k - 1) - F->vzt[l] * dt) * d->slope[LZM];
        else
          qs[l] = q[l] - 0.5 * (zone_size_z(d, j, k) + F->vzt[l] * dt) * d->slope[l];
      }
}
static void update_z(fo_disk *d, double dt, double *qb, const double *qs, int density) {
  /* update_z.c:56-80, update_density_z.c:54-78 */
  fo_fluid *F = &d->fl[d->cur];
  const double *vz = F->vzt, *rs = d->densstar;
  int i, j, k;
  for (k = 0; k < d->sz - 1; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lzp = LZP;
        if (!density)
          qb[l] += (vz[l] * qs[l] * rs[l] * Szj(j) * Szk(k) * Sxi(i) -
                    vz[lzp] * qs[lzp] * rs[lzp] * Szj(j) * Szk(k + 1) * Sxi(i)) *
                   dt * InvVj(j) / (Syk(k) * Sxi(i));
        else
          qb[l] += (vz[l] * rs[l] * Szj(j) * Szk(k) * Sxi(i) - vz[lzp] * rs[lzp] * Szj(j) * Szk(k + 1) * Sxi(i)) *
                   dt * InvVj(j) / (Syk(k) * Sxi(i));
      }
}
static void transport_z(fo_disk *d, double *q, double dt) { /* transport.c:36-46 */
  fo_fluid *F = &d->fl[d->cur];
  if (q != F->rho) {
    divide_by_rho(d, q);
    vanleer_z_a(d, d->divrho);
    vanleer_z_b(d, dt, d->divrho, d->qs);
    update_z(d, dt, q, d->qs, 0);
  } else {
    update_z(d, dt, q, NULL, 1);
  }
}

/* X sweep: van Leer (vanleer_x_a.c:55-71, vanleer_x_b.c:56-66) */
static void vanleer_x_a(fo_disk *d, const double *q) {
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double dqm = (q[l] - q[LXM]) / zone_size_x(d, i, j, k);
        double dqp = (q[LXP] - q[l]) / zone_size_x(d, ixp_(d, i), j, k);
        if (dqp * dqm <= 0.0) d->slope[l] = 0.0;
        else d->slope[l] = (2. * dqp * dqm) / (dqm + dqp);
      }
}
static void vanleer_x_b(fo_disk *d, double dt, const double *q, double *qs, const double *vx) {
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        if (vx[l] > 0.0)
          qs[l] = q[LXM] + 0.5 * (zone_size_x(d, ixm_(d, i), j, k) - vx[l] * dt) * d->slope[LXM];
        else
          qs[l] = q[l] - 0.5 * (zone_size_x(d, i, j, k) + vx[l] * dt) * d->slope[l];
      }
}
/* PPA (fargo_ppa_a.c:55-76, _b.c:52-64, _c.c:50-69, _d.c:55-78) */
static void ppa_a(fo_disk *d, const double *q) {
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double dqm = (q[l] - q[LXM]), dqp = (q[LXP] - q[l]), work;
        if (dqp * dqm <= 0.0) d->slope[l] = 0.0;
        else {
          d->slope[l] = 0.5 * (q[LXP] - q[LXM]);
          work = fabs(d->slope[l]);
          if (2.0 * fabs(dqm) < work) work = 2.0 * fabs(dqm);
          if (2.0 * fabs(dqp) < work) work = 2.0 * fabs(dqp);
          if (d->slope[l] < 0) d->slope[l] = -work;
          else d->slope[l] = work;
        }
      }
}
static void ppa_b(fo_disk *d, const double *q) {
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxp = LXP;
        double temp = q[l] + 0.5 * (q[lxp] - q[l]) - 1.0 / 6.0 * (d->slope[lxp] - d->slope[l]);
        d->qr[l] = temp;
        d->ql[lxp] = temp;
      }
}
static void ppa_c(fo_disk *d, const double *q) {
  long l;
  for (l = 0; l < d->ncell; l++) {
    double diff, cord;
    if ((d->qr[l] - q[l]) * (q[l] - d->ql[l]) < 0.0) { d->ql[l] = q[l]; d->qr[l] = q[l]; }
    diff = d->qr[l] - d->ql[l];
    cord = q[l] - 0.5 * (d->ql[l] + d->qr[l]);
    if (6.0 * diff * cord > diff * diff) d->ql[l] = 3.0 * q[l] - 2.0 * d->qr[l];
    if (-diff * diff > 6.0 * diff * cord) d->qr[l] = 3.0 * q[l] - 2.0 * d->ql[l];
  }
}
static void ppa_d(fo_disk *d, double dt, const double *q, double *qs, const double *vx) {
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxm = LXM;
        double ksi;
        if (vx[l] > 0.0) {
          ksi = vx[l] * dt / zone_size_x(d, i, j, k);
          qs[l] = d->qr[lxm] + ksi * (q[lxm] - d->qr[lxm]);
          qs[l] += ksi * (1.0 - ksi) * (2.0 * q[lxm] - d->qr[lxm] - d->ql[lxm]);
        } else {
          ksi = -vx[l] * dt / zone_size_x(d, i, j, k);
          qs[l] = d->ql[l] + ksi * (q[l] - d->ql[l]);
          qs[l] += ksi * (1.0 - ksi) * (2.0 * q[l] - d->qr[l] - d->ql[l]);
        }
      }
}
static void vanleer_x(fo_disk *d, int ppa, const double *q, double *qs, const double *vx, double dt) {
  /* transport.c:5-8 and vanleerx_ppa.c:3-12 */
  if (!ppa) { vanleer_x_a(d, q); vanleer_x_b(d, dt, q, qs, vx); }
  else { ppa_a(d, q); ppa_b(d, q); ppa_c(d, q); ppa_d(d, dt, q, qs, vx); }
}
static void update_x(fo_disk *d, double dt, double *qb, const double *qs, const double *vx, int density) {
  /* update_x.c:56-78, update_density_x.c:54-76 */
  const double *rs = d->densstar;
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxp = LXP;
        if (!density)
          qb[l] += ((vx[l] * qs[l] * rs[l] - vx[lxp] * qs[lxp] * rs[lxp]) * Sxj(j) * Sxk(k) * dt * InvVj(j) /
                    (Syk(k) * Sxi(i)));
        else
          qb[l] += ((vx[l] * rs[l] - vx[lxp] * rs[lxp]) * Sxj(j) * Sxk(k) * dt * InvVj(j) / (Syk(k) * Sxi(i)));
      }
}
static void transport_x(fo_disk *d, int ppa, double *q, const double *vx, double dt) { /* transport.c:11-22 */
  fo_fluid *F = &d->fl[d->cur];
  if (q != F->rho) {
    divide_by_rho(d, q);
    vanleer_x(d, ppa, d->divrho, d->qs, vx, dt);
    update_x(d, dt, q, d->qs, vx, 0);
  } else {
    update_x(d, dt, q, NULL, vx, 1);
  }
}
static void x_advection(fo_disk *d, int ppa, const double *vx, double dt) { /* transport.c:49-67 */
  fo_fluid *F = &d->fl[d->cur];
  vanleer_x(d, ppa, F->rho, d->densstar, vx, dt);
  transport_x(d, ppa, d->mpx, vx, dt);
  transport_x(d, ppa, d->mmx, vx, dt);
  transport_x(d, ppa, d->mpy, vx, dt);
  transport_x(d, ppa, d->mmy, vx, dt);
  if (d->is3d) { transport_x(d, ppa, d->mpz, vx, dt); transport_x(d, ppa, d->mmz, vx, dt); }
  if (d->p.adiabatic) transport_x(d, ppa, F->cs, vx, dt);   /* transport.c:63-65 */
  transport_x(d, ppa, F->rho, vx, dt);
}

/* ComputeResidual_cpu (compute_residual.c:55-80). */
static void compute_residual(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double vm = F->vxmed[L2D(j, k)];
        double ntilde = vm * dt / zone_size_x(d, i, j, k);
        double nround = floor(ntilde + 0.5);
        if (i == 0) d->nshift[L2D(j, k)] = (int)nround;
        F->vx[l] = F->vxt[l] - vm;
        F->vxt[l] = (ntilde - nround) * zone_size_x(d, i, j, k) / dt;
      }
}

/* AdvectSHIFT_cpu (advect_shift.c:45-66); Pressure is the auxiliary array. */
static void advect_shift(fo_disk *d, double *f) {
  int i, j, k;
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        int it = i - d->nshift[L2D(j, k)];
        while (it < 0) it += d->nx;
        while (it >= d->nx) it -= d->nx;
        d->pres[l] = f[l - i + it];
      }
  memcpy(f, d->pres, sizeof(double) * d->ncell);
}

/* NewVelocity_x/y/z (newvel_x.c:61-95, newvel_y.c:55-75, newvel_z.c:56-78). */
static void new_velocity(fo_disk *d) {
  fo_fluid *F = &d->fl[d->cur];
  const double *rho = F->rho;
  int i, j, k, k0 = d->is3d ? 1 : 0;
  for (k = k0; k < d->sz; k++)
    for (j = 1; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxm = LXM;
        int im = ixm_(d, i);
        if (!d->p.spherical) {
          F->vx[l] = (d->mmx[l] * Syk(k) * Sxi(i) / InvVj(j) + d->mpx[lxm] * Syk(k) * Sxi(im) / InvVj(j)) /
                         ((rho[l] * Syk(k) * Sxi(i) / InvVj(j) + rho[lxm] * Syk(k) * Sxi(im) / InvVj(j)) * Ymed(j)) -
                     d->omegaframe * Ymed(j);
        } else {
          double rcyl = Ymed(j) * sin(Zmed(k));
          F->vx[l] = (d->mmx[l] * Syk(k) * Sxi(i) / InvVj(j) + d->mpx[lxm] * Syk(k) * Sxi(im) / InvVj(j)) /
                         ((rho[l] * Syk(k) * Sxi(i) / InvVj(j) + rho[lxm] * Syk(k) * Sxi(im) / InvVj(j)) * rcyl) -
                     d->omegaframe * rcyl;
        }
      }
  for (k = k0; k < d->sz; k++)
    for (j = 1; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lym = LYM;
        F->vy[l] = (d->mmy[l] * Syk(k) * Sxi(i) / InvVj(j) + d->mpy[lym] * Syk(k) * Sxi(i) / InvVj(j - 1)) /
                   (rho[l] * Syk(k) * Sxi(i) / InvVj(j) + rho[lym] * Syk(k) * Sxi(i) / InvVj(j - 1));
      }
  if (d->is3d)
    for (k = 1; k < d->sz; k++)
      for (j = 1; j < d->sy; j++)
        for (i = 0; i < d->nx; i++) {
          long l = L(i, j, k), lzm = LZM;
          F->vz[l] = (d->mmz[l] * Syk(k) * Sxi(i) / InvVj(j) + d->mpz[lzm] * Syk(k - 1) * Sxi(i) / InvVj(j)) /
                     (rho[l] * Syk(k) * Sxi(i) / InvVj(j) + rho[lzm] * Syk(k - 1) * Sxi(i) / InvVj(j));
          if (d->p.spherical) F->vz[l] /= Ymed(j);
        }
}

/* transport (transport.c:69-193), FARGO flavour (neither STANDARD nor RAM). */
static void transport(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  momenta_x(d);
  momenta_y(d);
  if (d->is3d) momenta_z(d);
  if (d->is3d && d->nz > 1) {
    vanleer_z_a(d, F->rho);
    vanleer_z_b(d, dt, F->rho, d->densstar);
    transport_z(d, d->mpx, dt); transport_z(d, d->mmx, dt);
    transport_z(d, d->mpy, dt); transport_z(d, d->mmy, dt);
    transport_z(d, d->mpz, dt); transport_z(d, d->mmz, dt);
    transport_z(d, F->rho, dt);
  }
  if (d->ny > 1) {
    vanleer_y_a(d, F->rho);
    vanleer_y_b(d, dt, F->rho, d->densstar);
    transport_y(d, d->mpx, dt); transport_y(d, d->mmx, dt);
    transport_y(d, d->mpy, dt); transport_y(d, d->mmy, dt);
    if (d->is3d) { transport_y(d, d->mpz, dt); transport_y(d, d->mmz, dt); }
    if (d->p.adiabatic) transport_y(d, F->cs, dt);   /* transport.c:122-124 */
    transport_y(d, F->rho, dt);
  }
  if (d->nx > 1) {
    compute_residual(d, dt);
    x_advection(d, 0, F->vx, dt);
    x_advection(d, 1, F->vxt, dt);
    advect_shift(d, d->mpx); advect_shift(d, d->mmx);
    advect_shift(d, d->mpy); advect_shift(d, d->mmy);
    if (d->is3d) { advect_shift(d, d->mpz); advect_shift(d, d->mmz); }
    if (d->p.adiabatic) advect_shift(d, F->cs);   /* transport.c:155-157 */
    advect_shift(d, F->rho);
  }
  new_velocity(d);
}

/* StockholmBoundary_cpu (stockholm.c:90-190). */
static void stockholm(fo_disk *d, double dt) {
  fo_fluid *F = &d->fl[d->cur];
  const fo_params *p = &d->p;
  int i, j, k;
  double Y_inf = p->ymin * pow(p->damping_zone, 2.0 / 3.0);
  double Y_sup = p->ymax * pow(p->damping_zone, -2.0 / 3.0);
  double Z_inf = p->zmin - (p->zmax - p->zmin), Z_sup = p->zmax + (p->zmax - p->zmin);
  if (!p->spherical) {
    Z_inf = p->zmin + (p->zmax - p->zmin) * 0.1;
    Z_sup = p->zmax - (p->zmax - p->zmin) * 0.1;
  } else {
    Z_inf = M_PI / 2.0 - (M_PI / 2.0 - p->zmin) * (1.0 - p->killing_bc_colatitude);
    Z_sup = M_PI / 2.0 + (M_PI / 2.0 - p->zmin) * (1.0 - p->killing_bc_colatitude);
  }
  for (k = 0; k < d->sz; k++)
    for (j = 0; j < d->sy; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k);
        double rampy = 0.0, rampz = 0.0, rampzz = 0.0, ramp, rampi, tau, taud;
        if (Ymed(j) > Y_sup) rampy = (Ymed(j) - Y_sup) / (p->ymax - Y_sup);
        if (Ymed(j) < Y_inf) rampy = (Y_inf - Ymed(j)) / (Y_inf - p->ymin);
        rampy *= rampy;
        if (d->is3d) {
          if (Zmed(k) > Z_sup) rampz = (Zmed(k) - Z_sup) / (p->zmax - Z_sup);
          if (Zmed(k) < Z_inf) rampz = (Z_inf - Zmed(k)) / (Z_inf - p->zmin);
          rampz = rampz * rampz;
          if (Zmin(k) > Z_sup) rampzz = (Zmin(k) - Z_sup) / (p->zmax - Z_sup);
          if (Zmin(k) < Z_inf) rampzz = (Z_inf - Zmin(k)) / (Z_inf - p->zmin);
          rampzz = rampzz * rampzz;
        }
        ramp = rampy + rampz;
        rampi = rampy + rampzz;
        tau = p->tau_damp * sqrt(Ymed(j) * Ymed(j) * Ymed(j) / G / MSTAR);
        if (ramp > 0.0) {
          double vx0_target = F->vx0[L2D(j, k)], radius = Ymed(j);
          taud = tau / ramp;
          F->rho[l] = (F->rho[l] * taud + F->rho0[L2D(j, k)] * dt) / (dt + taud);
          if (p->spherical) radius *= sin(Zmed(k));
          vx0_target -= (d->omegaframe - d->omegaframe0) * radius;
          F->vx[l] = (F->vx[l] * taud + vx0_target * dt) / (dt + taud);
          F->vy[l] = (F->vy[l] * taud + F->vy0[L2D(j, k)] * dt) / (dt + taud);
        }
        if (d->is3d && rampi > 0.0) {
          taud = tau / rampi;
          F->vz[l] = (F->vz[l] * taud + F->vz0[L2D(j, k)] * dt) / (dt + taud);
        }
      }
}

/* ------------------------------------------------------------------------- */
/* Multifluid implicit drag (collisions below). */
static void collisions(fo_disk *d, double dt);

/* ------------------------------------------------------------------------- */
fo_disk *fo_create(const fo_params *p) {
  fo_disk *d = (fo_disk *)xcalloc(1, sizeof(fo_disk));
  int f, n;
  d->p = *p;
  if (d->p.nfluids < 1) d->p.nfluids = 1;
  /* the adiabatic EOS and dust diffusion are restated for 2D cylindrical
     disks (each on its own: the dust coefficients of an adiabatic gas are not) */
  if ((p->adiabatic || p->dust_diffusion) && (p->nz > 1 || p->spherical || (p->adiabatic && p->dust_diffusion) ||
                                              (p->dust_diffusion && d->p.nfluids < 2))) {
    free(d);
    return NULL;
  }
  d->is3d = p->nz > 1;
  d->nx = p->nx; d->ny = p->ny; d->nz = d->is3d ? p->nz : 1;
  d->sx = d->nx; d->sy = d->ny + 2 * NG; d->sz = d->is3d ? d->nz + 2 * NG : 1;
  d->pitch = d->sx; d->stride = (long)d->sx * d->sy; d->ncell = d->stride * d->sz;
  d->xmin = xcalloc(d->sx + 1, 8); d->ymin = xcalloc(d->sy + 1, 8); d->zmin = xcalloc(d->sz + 1, 8);
  d->xmed = xcalloc(d->sx, 8); d->ymed = xcalloc(d->sy, 8); d->zmed = xcalloc(d->sz, 8);
  d->invdiffxmed = xcalloc(d->sx, 8); d->sxi = xcalloc(d->sx, 8);
  d->sxj = xcalloc(d->sy, 8); d->syj = xcalloc(d->sy, 8); d->szj = xcalloc(d->sy, 8); d->invvj = xcalloc(d->sy, 8);
  d->sxk = xcalloc(d->sz, 8); d->syk = xcalloc(d->sz, 8); d->szk = xcalloc(d->sz, 8);
  init_space(d);
  for (f = 0; f < d->p.nfluids; f++) {
    fo_fluid *F = &d->fl[f];
    F->rho = xcalloc(d->ncell, 8); F->cs = xcalloc(d->ncell, 8);
    F->vx = xcalloc(d->ncell, 8); F->vy = xcalloc(d->ncell, 8); F->vz = xcalloc(d->ncell, 8);
    F->vxt = xcalloc(d->ncell, 8); F->vyt = xcalloc(d->ncell, 8); F->vzt = xcalloc(d->ncell, 8);
    F->vxmed = xcalloc((size_t)d->sy * d->sz, 8);
    F->rho0 = xcalloc((size_t)d->sy * d->sz, 8); F->vx0 = xcalloc((size_t)d->sy * d->sz, 8);
    F->vy0 = xcalloc((size_t)d->sy * d->sz, 8); F->vz0 = xcalloc((size_t)d->sy * d->sz, 8);
    F->dust = f > 0;
  }
  d->pres = xcalloc(d->ncell, 8); d->pot = xcalloc(d->ncell, 8);
  d->mpx = xcalloc(d->ncell, 8); d->mmx = xcalloc(d->ncell, 8);
  d->mpy = xcalloc(d->ncell, 8); d->mmy = xcalloc(d->ncell, 8);
  d->mpz = xcalloc(d->ncell, 8); d->mmz = xcalloc(d->ncell, 8);
  d->slope = xcalloc(d->ncell, 8); d->divrho = xcalloc(d->ncell, 8);
  d->densstar = xcalloc(d->ncell, 8); d->qs = xcalloc(d->ncell, 8);
  d->ql = xcalloc(d->ncell, 8); d->qr = xcalloc(d->ncell, 8); d->totdens = xcalloc(d->ncell, 8);
  d->red2d = xcalloc((size_t)d->sy * d->sz, 8); d->nshift = xcalloc((size_t)d->sy * d->sz, sizeof(int));
  d->sdiff_c = xcalloc(d->ncell, 8); d->sdiff_f = xcalloc(d->ncell, 8);
  /* planets (psys.c:141-225) */
  d->np = p->nplanets;
  for (n = 0; n < d->np; n++) {
    double dist = p->pl_dist[n];
    d->pmass[n] = p->pl_mass[n];
    d->px[n] = dist * (1.0 + p->eccentricity);
    d->py[n] = 0.0; d->pz[n] = 0.0;
    d->pvy[n] = sqrt(G * (MSTAR + d->pmass[n]) / dist) * sqrt((1.0 - p->eccentricity) / (1.0 + p->eccentricity)) *
                cos(p->inclination);
    d->pvx[n] = -0.0000000000 * d->pvy[n];
    d->pvz[n] = d->pvy[n] * sin(p->inclination) / cos(p->inclination);
    d->pfeeldisk[n] = p->pl_feeldisk[n];
    d->pfeelothers[n] = p->pl_feelothers[n];
  }
  d->omegaframe = p->omegaframe;
  /* main.c:240-242 */
  if (p->frame != FO_FRAME_FIXED && d->np > 0) d->omegaframe = get_psys_info(d, PS_FREQUENCY);
  d->omegaframe0 = d->omegaframe;
  d->potential_done_at = -1;
  return d;
}

void fo_destroy(fo_disk *d) {
  int f;
  if (!d) return;
  for (f = 0; f < d->p.nfluids; f++) {
    fo_fluid *F = &d->fl[f];
    free(F->rho); free(F->cs); free(F->vx); free(F->vy); free(F->vz);
    free(F->vxt); free(F->vyt); free(F->vzt); free(F->vxmed);
    free(F->rho0); free(F->vx0); free(F->vy0); free(F->vz0);
  }
  free(d->pres); free(d->pot); free(d->mpx); free(d->mmx); free(d->mpy); free(d->mmy);
  free(d->mpz); free(d->mmz); free(d->slope); free(d->divrho); free(d->densstar); free(d->qs);
  free(d->ql); free(d->qr); free(d->totdens); free(d->red2d); free(d->nshift);
  free(d->sdiff_c); free(d->sdiff_f);
  free(d->xmin); free(d->ymin); free(d->zmin); free(d->xmed); free(d->ymed); free(d->zmed);
  free(d->invdiffxmed); free(d->sxi); free(d->sxj); free(d->syj); free(d->szj); free(d->invvj);
  free(d->sxk); free(d->syk); free(d->szk);
  free(d);
}

void fo_get_geometry(const fo_disk *d, double *xa, double *ya, double *za) {
  if (xa) memcpy(xa, d->xmin, sizeof(double) * (d->sx + 1));
  if (ya) memcpy(ya, d->ymin, sizeof(double) * (d->sy + 1));
  if (za) memcpy(za, d->zmin, sizeof(double) * (d->sz + 1));
}

void fo_set_state(fo_disk *d, int f, const double *rho, const double *vx, const double *vy,
                  const double *vz, const double *cs) {
  fo_fluid *F = &d->fl[f];
  size_t n = sizeof(double) * d->ncell;
  if (rho) memcpy(F->rho, rho, n);
  if (vx) memcpy(F->vx, vx, n);
  if (vy) memcpy(F->vy, vy, n);
  if (vz && d->is3d) memcpy(F->vz, vz, n);
  if (cs) memcpy(F->cs, cs, n);
}

void fo_get_energy(const fo_disk *d, int f, double *e) {
  memcpy(e, d->fl[f].cs, sizeof(double) * d->ncell);
}

void fo_get_state(const fo_disk *d, int f, double *rho, double *vx, double *vy, double *vz) {
  const fo_fluid *F = &d->fl[f];
  size_t n = sizeof(double) * d->ncell;
  if (rho) memcpy(rho, F->rho, n);
  if (vx) memcpy(vx, F->vx, n);
  if (vy) memcpy(vy, F->vy, n);
  if (vz && d->is3d) memcpy(vz, F->vz, n);
}

void fo_initialize(fo_disk *d) {
  int f, j, k;
  for (f = 0; f < d->p.nfluids; f++) { d->cur = f; fill_ghosts(d); }
  /* init_stockholm (init_stockholm.c:56-105): profiles taken at i = 0 */
  for (f = 0; f < d->p.nfluids; f++) {
    fo_fluid *F = &d->fl[f];
    for (k = 0; k < d->sz; k++)
      for (j = 0; j < d->sy; j++) {
        F->vx0[L2D(j, k)] = F->vx[L(0, j, k)];
        F->vy0[L2D(j, k)] = F->vy[L(0, j, k)];
        if (d->is3d) F->vz0[L2D(j, k)] = F->vz[L(0, j, k)];
        F->rho0[L2D(j, k)] = F->rho[L(0, j, k)];
      }
  }
  d->cur = 0;
}

/* DustDiffusion_Main (dust_diffusion_main.c:3-28): the diffusion
 * coefficients from the gas (DustDiffusion_Coefficients_cpu,
 * dust_diffusion_coefficients.c:56-118; 2D cylindrical), then for every dust
 * fluid the update of its density from the gradient of its concentration
 * rho_d / (rho_d + rho_g) (DustDiffusion_Core_cpu, dust_diffusion_core.c:
 * 97-170) into the Pressure scratch, copied to the density, and FillGhosts.
 * copy_field copies the whole field; its rows 0 and Ny+5, which the core
 * does not write, are ghost rows that FillGhosts rewrites, so only the rows
 * the core writes are copied here. */
static void dust_diffusion(fo_disk *d, double dt) {
  const fo_fluid *Gs = &d->fl[0];
  const double *cs = Gs->cs, *rhog = Gs->rho;
  double *sdc = d->sdiff_c, *sdf = d->sdiff_f, *temp = d->pres;
  int i, j, k = 0, f;
  for (j = 0; j < d->sy; j++)
    for (i = 0; i < d->nx; i++) {
      long l = L(i, j, k);
      if (d->p.alpha_visc) {
        double ss2 = cs[l] * cs[l], ssf2, r3c, r3f;
        if (j == 0) ssf2 = ss2;
        else ssf2 = 0.5 * (cs[l] + cs[LYM]) * 0.5 * (cs[l] + cs[LYM]);
        r3c = Ymed(j) * Ymed(j) * Ymed(j);
        r3f = Ymin(j) * Ymin(j) * Ymin(j);
        sdc[l] = d->p.alpha * ss2 / sqrt(G * MSTAR / r3c);
        sdf[l] = d->p.alpha * ssf2 / sqrt(G * MSTAR / r3f);
      } else {
        sdc[l] = d->p.nu;
        sdf[l] = d->p.nu;
      }
    }
  for (f = 1; f < d->p.nfluids; f++) {
    fo_fluid *F = &d->fl[f];
    const double *rhod = F->rho;
    d->cur = f;
    for (j = 1; j < d->sy - 1; j++)
      for (i = 0; i < d->nx; i++) {
        long l = L(i, j, k), lxp = LXP, lxm = LXM, lyp = LYP, lym = LYM;
        double c, update, d1, d2, d3, d4, cxp, cxm, cyp, cym, dxmin, dxmedp, dxmedm;
        update = 0.0;
        c = rhod[l] / (rhod[l] + rhog[l]);
        dxmin = Xmin(i + 1) - Xmin(i);
        dxmedp = 1.0 / d->invdiffxmed[ixp_(d, i)];
        dxmedm = 1.0 / d->invdiffxmed[i];
        d1 = 0.25 * (rhod[l] + rhog[l] + rhod[lxp] + rhog[lxp]) * (sdc[lxp] + sdc[l]);
        d2 = 0.25 * (rhod[l] + rhog[l] + rhod[lxm] + rhog[lxm]) * (sdc[lxm] + sdc[l]);
        cxp = rhod[lxp] / (rhod[lxp] + rhog[lxp]);
        cxm = rhod[lxm] / (rhod[lxm] + rhog[lxm]);
        update += 1.0 / Ymed(j) / Ymed(j) / (dxmin) * (d1 * (cxp - c) / (dxmedp) - (d2 * (c - cxm)) / (dxmedm));
        d3 = 0.5 * (rhod[l] + rhog[l] + rhod[lyp] + rhog[lyp]) * sdf[lyp];
        d4 = 0.5 * (rhod[l] + rhog[l] + rhod[lym] + rhog[lym]) * sdf[l];
        cyp = rhod[lyp] / (rhod[lyp] + rhog[lyp]);
        cym = rhod[lym] / (rhod[lym] + rhog[lym]);
        update += 1.0 / Ymed(j) / (Ymin(j + 1) - Ymin(j)) *
                  (Ymin(j + 1) * d3 * (cyp - c) / (Ymed(j + 1) - Ymed(j)) -
                   (Ymin(j) * d4 * (c - cym)) / (Ymed(j) - Ymed(j - 1)));
        temp[l] = rhod[l] + dt * update;
      }
    memcpy(F->rho + L(0, 1, 0), temp + L(0, 1, 0), sizeof(double) * (size_t)(d->sy - 2) * d->pitch);
    fill_ghosts(d);
  }
  d->cur = 0;
}

static void sources(fo_disk *d, double dt) { /* algogas.c:30-133 */
  fo_fluid *F = &d->fl[d->cur];
  pressure(d);
  compute_potential(d, dt);
  if (d->p.frame != FO_FRAME_FIXED) correct_vtheta(d, d->domega);
  substep1_x(d, dt);
  substep1_y(d, dt);
  if (d->is3d) substep1_z(d, dt);
  if (!F->dust && (d->p.nu != 0.0 || d->p.alpha_visc)) { visctensor(d); addviscosity(d, dt); }
  substep2_a(d);
  substep2_b(d, dt);
  if (d->p.adiabatic && !F->dust) substep3(d, dt);   /* algogas.c:82-84 */
  /* copy_velocities(VTEMP2V); FillGhosts; copy_velocities(V2VTEMP) */
  memcpy(F->vx, F->vxt, sizeof(double) * d->ncell);
  memcpy(F->vy, F->vyt, sizeof(double) * d->ncell);
  if (d->is3d) memcpy(F->vz, F->vzt, sizeof(double) * d->ncell);
  fill_ghosts(d);
  memcpy(F->vxt, F->vx, sizeof(double) * d->ncell);
  memcpy(F->vyt, F->vy, sizeof(double) * d->ncell);
  if (d->is3d) memcpy(F->vzt, F->vz, sizeof(double) * d->ncell);
}

double fo_step(fo_disk *d, double DT) {
  int f;
  double dt, step = 1e30;
  long l;
  if (d->dtemp >= DT) d->dtemp = 0.0;
  for (f = 0; f < d->p.nfluids; f++) { d->cur = f; compute_vmed(d, d->fl[f].vx); }
  for (f = 0; f < d->p.nfluids; f++) { d->cur = f; cfl(d); }
  for (f = 0; f < d->p.nfluids; f++)
    if (step > d->minstep[f]) step = d->minstep[f];
  if (step <= SMALLTIME) return -1.0;
  dt = step;
  d->dtemp += dt;
  if (d->dtemp > DT) dt = DT - (d->dtemp - dt);
  memset(d->totdens, 0, sizeof(double) * d->ncell);
  for (f = 0; f < d->p.nfluids; f++)
    for (l = 0; l < d->ncell; l++) d->totdens[l] += d->fl[f].rho[l];
  for (f = 0; f < d->p.nfluids; f++) { d->cur = f; sources(d, dt); }
  if (d->p.nfluids > 1) collisions(d, dt);
  if (d->p.dust_diffusion) dust_diffusion(d, dt);   /* main.c:417-419 */
  for (f = 0; f < d->p.nfluids; f++) {
    d->cur = f;
    compute_vmed(d, d->fl[f].vxt); /* algogas.c:141 */
    transport(d, dt);
  }
  d->phys_time += dt;
  d->timestep_count++;
  if (d->p.stockholm)
    for (f = 0; f < d->p.nfluids; f++) { d->cur = f; stockholm(d, dt); }
  for (f = 0; f < d->p.nfluids; f++) { d->cur = f; fill_ghosts(d); }
  d->cur = 0;
  d->last_dt = dt;
  return dt;
}

void fo_get_scalars(const fo_disk *d, double *o) {
  o[0] = d->phys_time; o[1] = d->omegaframe; o[2] = d->last_dt;
  o[3] = d->np ? d->px[0] : 0; o[4] = d->np ? d->py[0] : 0;
  o[5] = d->np ? d->pvx[0] : 0; o[6] = d->np ? d->pvy[0] : 0; o[7] = d->domega;
}

double fo_mass(const fo_disk *d, int f) {
  const fo_fluid *F = &d->fl[f];
  int i, j, k, k0 = d->is3d ? NG : 0, k1 = d->is3d ? d->nz + NG : 1;
  double s = 0.0, c = 0.0;
  for (k = k0; k < k1; k++)
    for (j = NG; j < d->ny + NG; j++)
      for (i = 0; i < d->nx; i++) {
        double v = F->rho[L(i, j, k)] * (Syk(k) * Sxi(i) / InvVj(j)) - c;
        double t = s + v;
        c = (t - s) - v;
        s = t;
      }
  return s;
}

/* Implicit drag between the fluids, STOKESNUMBER form (collisions.c:10-189,
 * collision_kernel.h:11-94, gauss.h:1-45), applied to V_temp after the
 * sources of every fluid.  For each direction in turn (x, then y, then z) and
 * each face l of the range j >= 1 (k >= 1 in 3D), the velocities b[o] of the
 * N fluids at that face solve M b_new = b_old with
 *   M[o][p] (o != p) = -dt W a[p][o] rho_p / rho_o   if p > o
 *                      -dt W a[p][o]                 otherwise
 *   M[p][p]          = 1 + dt W sum_{q != p} (q > p ? a[q][p] rho_q / rho_p : a[q][p])
 * where rho_* are face averages 0.5 (rho[l] + rho[l - 1 cell along the
 * direction]), W the Keplerian frequency at the face's radius (Ymed for the
 * x and z faces, Ymin for the y faces: collision_kernel.h:16-18) and
 * a[p][o] the collision-rate matrix (alpha[p + o N]),
 * filled as ColRate does (colrate.c:10-23): a[0][f] = a[f][0] = 1/St_f.  The
 * system is solved by Gaussian elimination with the reference's row pivoting
 * (the pivot search compares |m| with the signed value last kept, gauss.h:7-13)
 * and back substitution; the operation order is the reference's, so the
 * result is bit-identical. */
static void collisions(fo_disk *d, double dt) {
  const int N = d->p.nfluids;
  double alpha[FO_MAXFLUIDS * FO_MAXFLUIDS] = {0};
  double m[FO_MAXFLUIDS * FO_MAXFLUIDS], b[FO_MAXFLUIDS];
  double *rho[FO_MAXFLUIDS], *vel[FO_MAXFLUIDS];
  int dir, f, i, j, k, o, p, q, ir, ir2, ir_max = 0, ic;
  for (f = 1; f < N; f++) alpha[0 + f * N] = alpha[f + 0 * N] = d->p.invstokes[f - 1];
  for (f = 0; f < N; f++) rho[f] = d->fl[f].rho;
  for (dir = 0; dir < (d->is3d ? 3 : 2); dir++) {
    for (f = 0; f < N; f++) vel[f] = dir == 0 ? d->fl[f].vxt : (dir == 1 ? d->fl[f].vyt : d->fl[f].vzt);
    for (k = d->is3d ? 1 : 0; k < (d->is3d ? d->sz : 1); k++)
      for (j = 1; j < d->sy; j++)
        for (i = 0; i < d->nx; i++) {
          const long l = L(i, j, k);
          const long lm = dir == 0 ? lxm_(d, i, l) : (dir == 1 ? l - d->pitch : l - d->stride);
          const double y = dir == 1 ? Ymin(j) : Ymed(j);
          const double w = sqrt(G * MSTAR / (y * y * y));
          double rho_p, rho_o, rho_q, sum, mx, tmp, factor;
          for (o = 0; o < N; o++) {
            for (p = 0; p < N; p++) {
              rho_p = 0.5 * (rho[p][l] + rho[p][lm]);
              if (p != o) {
                rho_o = 0.5 * (rho[o][l] + rho[o][lm]);
                if (p > o) m[p + o * N] = -dt * w * alpha[p + o * N] * rho_p / rho_o;
                else m[p + o * N] = -dt * w * alpha[p + o * N];
              } else {
                sum = 0.0;
                for (q = 0; q < N; q++) {
                  if (q == p) continue;
                  rho_q = 0.5 * (rho[q][l] + rho[q][lm]);
                  if (q > p) sum += alpha[q + p * N] * rho_q / rho_p;
                  else sum += alpha[q + p * N];
                }
                m[p + p * N] = 1.0 + dt * w * sum;
              }
            }
            b[o] = vel[o][l];
          }
          for (ir = 0; ir < N - 1; ir++) {
            mx = -1;
            for (ir2 = ir; ir2 < N; ir2++)
              if (fabs(m[ir + ir2 * N]) >= mx) { mx = m[ir + ir2 * N]; ir_max = ir2; }
            if (ir_max != ir) {
              for (ic = 0; ic < N; ic++) {
                tmp = m[ic + ir * N]; m[ic + ir * N] = m[ic + ir_max * N]; m[ic + ir_max * N] = tmp;
              }
              tmp = b[ir]; b[ir] = b[ir_max]; b[ir_max] = tmp;
            }
            for (ir2 = ir + 1; ir2 < N; ir2++) {
              factor = m[ir + ir2 * N] / m[ir + ir * N];
              for (ic = 0; ic < N; ic++) m[ic + ir2 * N] -= m[ic + ir * N] * factor;
              b[ir2] -= b[ir] * factor;
            }
          }
          for (ir = N - 1; ir > -1; ir--) {
            for (ic = N - 1; ic > ir; ic--) b[ir] -= m[ic + ir * N] * b[ic];
            b[ir] /= m[ir + ir * N];
          }
          for (o = 0; o < N; o++) vel[o][l] = b[o];
        }
  }
}
