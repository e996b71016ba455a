/*
 * fb_psys.h -- the scalar part of a hydro step: time step from the CFL
 * minimum, planetary system and frame of reference, in FP64.
 *
 * Written once in C and compiled both for the host (fb_host.c, the
 * one-disk-at-a-time path, where it matches the reference's host code bit for
 * bit) and for the device (fb_batch.cu, where one thread per disk runs it
 * between the stage kernels of a captured step).
 *
 * Reference: InitPlanetarySystem (psys.c:141-225), SV2OE (planets.c:116-190),
 * GetPsysInfo (psys.c:362-415), RotatePsys (psys.c:417-440), the Cash-Karp
 * RK5 of runge_kutta.c, compute_potential (potential.c:10-49) and the DT-loop
 * clipping of main.c:388-395.
 */
#ifndef FB_PSYS_H
#define FB_PSYS_H

#include <math.h>
#include "fb_abi.h"
#include "fb_dev.h"

#ifdef __CUDACC__
#define FB_HD __host__ __device__
#define FB_FI __forceinline__
#else
#define FB_HD
#define FB_FI inline
#endif

#define FB_G 1.0
#define FB_MSTAR 1.0
#define FB_R0 1.0

typedef struct fb_psys_s {
  int np, frame, indirect_term;
  int feelothers[FB_MAXPLANETS];
  int feeldisk[FB_MAXPLANETS];   /* AdvanceSystemFromDisk applies (planets.c:93) */
  double px[FB_MAXPLANETS], py[FB_MAXPLANETS], pz[FB_MAXPLANETS];
  double pvx[FB_MAXPLANETS], pvy[FB_MAXPLANETS], pvz[FB_MAXPLANETS], pmass[FB_MAXPLANETS];
  double xmark, ymark, xaxis_rot;
  double omegaframe, omegaframe0, domega, phys_time, dtemp, last_dt;
  double roche_smoothing, aspectratio, flaringindex, thickness_smoothing;
  long long step_count;
  int status;     /* 0 ok, FB_ERR_NULL_DT after a null time step, FB_DONE */
  double t_end;   /* > 0: the disk stops at this physical time (batches) */
} fb_psys;

typedef struct { double e, a, M, i, phi; } fb_orbit;

static FB_HD inline fb_orbit fb_orbit_of(double x, double y, double z, double vx, double vy, double vz, double m) {
  fb_orbit o;
  double d = sqrt(x * x + y * y + z * z);
  double hx = y * vz - z * vy, hy = z * vx - x * vz, hz = x * vy - y * vx;
  double hhor = sqrt(hx * hx + hy * hy), h = sqrt(hx * hx + hy * hy + hz * hz);
  double Ax, Ay, Az, E;
  o.i = asin(hhor / h);
  Ax = vy * hz - vz * hy - FB_G * m * x / d;
  Ay = vz * hx - vx * hz - FB_G * m * y / d;
  Az = vx * hy - vy * hx - FB_G * m * z / d;
  o.e = sqrt(Ax * Ax + Ay * Ay + Az * Az) / (FB_G * m);
  o.a = h * h / (FB_G * m * (1. - o.e * o.e));
  E = (o.e != 0.0) ? acos((1.0 - d / o.a) / o.e) : 0.0;
  if (x * vx + y * vy + z * vz < 0) E = -E;
  if (isnan(E)) E = (d < o.a) ? 0.0 : M_PI;
  o.M = E - o.e * sin(E);
  o.phi = (Ax * Ax + Ay * Ay > 0.0) ? atan2(Ay, Ax) : atan2(y, x);
  return o;
}

enum { FB_PS_GET = 0, FB_PS_MARK = 1, FB_PS_FREQUENCY = 2 };

static FB_HD inline double fb_psys_info(fb_psys *S, int action) {
  double x = S->px[0], y = S->py[0], z = S->pz[0], vx = S->pvx[0], vy = S->pvy[0], vz = S->pvz[0];
  double m = S->pmass[0] + FB_MSTAR, xc = x, yc = y, d1, d2, cross;
  fb_orbit o = fb_orbit_of(x, y, z, vx, vy, vz, m);
  if (S->frame == FB_FRAME_GUIDING) {
    xc = o.a * cos(o.M + o.phi) * cos(o.i);
    yc = o.a * sin(o.M + o.phi) * cos(o.i);
  }
  if (o.e < 1e-8) { xc = x; yc = y; }
  if (action == FB_PS_MARK) { S->xmark = xc; S->ymark = yc; return 0.0; }
  if (action == FB_PS_GET) {
    x = xc; y = yc;
    d2 = sqrt(x * x + y * y);
    d1 = sqrt(S->xmark * S->xmark + S->ymark * S->ymark);
    cross = S->xmark * y - x * S->ymark;
    S->xmark = x; S->ymark = y;
    return asin(cross / (d1 * d2));
  }
  if (S->frame == FB_FRAME_GUIDING) return sqrt(FB_G * m / pow(o.a, 3.0));
  return (x * vy - y * vx) / (x * x + y * y);
}

static FB_HD inline void fb_psys_rotate(fb_psys *S, double angle) {
  int i;
  double s = sin(angle), c = cos(angle), xt, yt;
  S->xaxis_rot += angle;
  if (S->xaxis_rot >= 2.0 * M_PI) S->xaxis_rot -= 2.0 * M_PI;
  if (S->xaxis_rot < 0.0) S->xaxis_rot += 2.0 * M_PI;
  for (i = 0; i < S->np; i++) {
    xt = S->px[i]; yt = S->py[i];
    S->px[i] = xt * c + yt * s; S->py[i] = -xt * s + yt * c;
    xt = S->pvx[i]; yt = S->pvy[i];
    S->pvx[i] = xt * c + yt * s; S->pvy[i] = -xt * s + yt * c;
  }
}

static FB_HD FB_FI void fb_nbody_deriv(const fb_psys *S, const double *q, const double *ms, double *der, int n,
                                       double dt) {
  const double *x = q, *y = q + n, *z = q + 2 * n, *vx = q + 3 * n, *vy = q + 4 * n, *vz = q + 5 * n;
  double dist[FB_MAXPLANETS], coef, dd;
  int i, j;
  for (i = 0; i < n; i++) dist[i] = sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
#ifdef __CUDA_ARCH__
  /* on the device (batched steps): one reciprocal of d^3 per planet instead
     of the three chained divisions of runge_kutta.c -- the same quantity,
     rounded differently, in a step whose latency is this dependency chain */
  double id3[FB_MAXPLANETS];
  for (i = 0; i < n; i++) id3[i] = 1.0 / (dist[i] * dist[i] * dist[i]);
#define FB_INV_D3(k) (id3[k])
#else
#define FB_INV_D3(k) (1.0 / dist[k] / dist[k] / dist[k])
#endif
  for (i = 0; i < n; i++) {
    der[i] = vx[i]; der[i + n] = vy[i]; der[i + 2 * n] = vz[i];
#ifdef __CUDA_ARCH__
    coef = -FB_G * FB_MSTAR * FB_INV_D3(i);
#else
    coef = -FB_G * FB_MSTAR / dist[i] / dist[i] / dist[i];
#endif
    der[i + 3 * n] = coef * x[i]; der[i + 4 * n] = coef * y[i]; der[i + 5 * n] = coef * z[i];
    for (j = 0; j < n; j++) {
      if (S->indirect_term) {
#ifdef __CUDA_ARCH__
        coef = FB_G * ms[j] * FB_INV_D3(j);
#else
        coef = FB_G * ms[j] / dist[j] / dist[j] / dist[j];
#endif
        der[i + 3 * n] -= coef * x[j]; der[i + 4 * n] -= coef * y[j]; der[i + 5 * n] -= coef * z[j];
      }
      if (j != i && S->feelothers[i]) {
        dd = (x[i] - x[j]) * (x[i] - x[j]) + (y[i] - y[j]) * (y[i] - y[j]) + (z[i] - z[j]) * (z[i] - z[j]);
        dd = sqrt(dd);
        coef = FB_G * ms[j] / dd / dd / dd;
        der[i + 3 * n] += coef * (x[j] - x[i]); der[i + 4 * n] += coef * (y[j] - y[i]);
        der[i + 5 * n] += coef * (z[j] - z[i]);
      }
    }
  }
  for (i = 0; i < 6 * n; i++) der[i] *= dt;
#undef FB_INV_D3
}

static FB_HD FB_FI void fb_nbody_rk5_n(fb_psys *S, double dt, const int n) {
  enum { M6 = 6 * FB_MAXPLANETS };
  int i;
  double q0[M6], q1[M6], ms[FB_MAXPLANETS];
  double k1[M6], k2[M6], k3[M6], k4[M6], k5[M6], k6[M6];
  if (!n) return;
  /* the stages read k2..k5 (times 0.0) before writing them: zero the used part */
  for (i = 0; i < 6 * n; i++) { k2[i] = k3[i] = k4[i] = k5[i] = 0.0; }
  for (i = 0; i < n; i++) {
    q0[i] = S->px[i]; q0[i + n] = S->py[i]; q0[i + 2 * n] = S->pz[i];
    q0[i + 3 * n] = S->pvx[i]; q0[i + 4 * n] = S->pvy[i]; q0[i + 5 * n] = S->pvz[i];
    ms[i] = S->pmass[i];
  }
#define FB_STAGE(c1, c2, c3, c4, c5) \
  for (i = 0; i < 6 * n; i++) q1[i] = q0[i] + c1 * k1[i] + c2 * k2[i] + c3 * k3[i] + c4 * k4[i] + c5 * k5[i]
  fb_nbody_deriv(S, q0, ms, k1, n, dt);
  FB_STAGE(0.2, 0.0, 0.0, 0.0, 0.0);
  fb_nbody_deriv(S, q1, ms, k2, n, dt);
  FB_STAGE(0.075, 0.225, 0.0, 0.0, 0.0);
  fb_nbody_deriv(S, q1, ms, k3, n, dt);
  FB_STAGE(0.3, -0.9, 1.2, 0.0, 0.0);
  fb_nbody_deriv(S, q1, ms, k4, n, dt);
  FB_STAGE(-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0.0);
  fb_nbody_deriv(S, q1, ms, k5, n, dt);
  FB_STAGE(1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0);
  fb_nbody_deriv(S, q1, ms, k6, n, dt);
#undef FB_STAGE
  for (i = 0; i < 6 * n; i++)
    q1[i] = (q0[i] + 37.0 / 378.0 * k1[i] + 250.0 / 621.0 * k3[i] + 125.0 / 594.0 * k4[i] + 512.0 / 1771.0 * k6[i]);
  for (i = 0; i < n; i++) {
    S->px[i] = q1[i]; S->py[i] = q1[i + n]; S->pz[i] = q1[i + 2 * n];
    S->pvx[i] = q1[i + 3 * n]; S->pvy[i] = q1[i + 4 * n]; S->pvz[i] = q1[i + 5 * n];
  }
}

/* With one planet the count is a constant: the loops unroll and the stage
 * arrays stay in registers (the same operations in the same order). */
static FB_HD inline void fb_nbody_rk5(fb_psys *S, double dt) {
  if (S->np == 1) fb_nbody_rk5_n(S, dt, 1);
  else fb_nbody_rk5_n(S, dt, S->np);
}

/* Per-step scalars the kernels read (the planet terms of Potential_cpu that do
 * not depend on the cell, potential.c:137-160). */
static FB_HD inline void fb_psys_fill_scalars(const fb_psys *S, fb_scalars *sc) {
  int n;
  sc->nplanets = S->np;
  sc->indirect_term = S->indirect_term;
  for (n = 0; n < S->np; n++) {
    double mp = S->pmass[n] * 1.0, pd, rroche, s;
    pd = sqrt(S->px[n] * S->px[n] + S->py[n] * S->py[n] + S->pz[n] * S->pz[n]);
    rroche = pd * pow((1.0 / 3.0 * mp / FB_MSTAR), 1.0 / 3.0);
    if (S->roche_smoothing != 0) s = rroche * S->roche_smoothing;
    else s = S->aspectratio * pow(pd / FB_R0, S->flaringindex) * pd * S->thickness_smoothing;
    sc->px[n] = S->px[n]; sc->py[n] = S->py[n]; sc->pz[n] = S->pz[n];
    sc->pmass[n] = S->pmass[n];
    sc->psmooth2[n] = s * s;
    sc->pdist3[n] = pd * pd * pd;
  }
}

/* The scalar work of one hydro step, given the CFL minimum `cflmin` of the
 * disk (the MIN over fluids and shear limits): dt with the DT-interval clip,
 * then compute_potential's planetary update.  Returns dt, or -1 on a null
 * time step (cfl_fluids_min.c:18-21). */
/* One step of the planetary system (compute_potential, potential.c:10-49).
 * dacc: the disk's acceleration at each planet's position (3 per planet,
 * ComputeAccel), applied to the planets that feel the disk before the RK5
 * substeps (AdvanceSystemFromDisk, planets.c:86-114); NULL when none does. */
static FB_HD inline double fb_psys_step(fb_psys *S, double cflmin, double DT, fb_scalars *sc, const double *dacc) {
  double step = 1e30, dt;
  int f;
  if (S->dtemp >= DT) S->dtemp = 0.0;
  if (step > cflmin) step = cflmin;
  if (!(step > 1e-10 * sqrt(FB_R0 * FB_R0 * FB_R0 / (FB_G * FB_MSTAR)))) {
    S->status = FB_ERR_NULL_DT;
    return -1.0;
  }
  dt = step;
  S->dtemp += dt;
  if (S->dtemp > DT) dt = DT - (S->dtemp - dt);
  if (S->frame != FB_FRAME_FIXED) fb_psys_info(S, FB_PS_MARK);
  fb_psys_fill_scalars(S, sc);
  if (dacc)
    for (f = 0; f < S->np; f++)
      if (S->feeldisk[f]) {
        S->pvx[f] += dt * dacc[3 * f];
        S->pvy[f] += dt * dacc[3 * f + 1];
        S->pvz[f] += dt * dacc[3 * f + 2];
      }
  for (f = 0; f < 5; f++) fb_nbody_rk5(S, 1.0 / ((double)(5)) * dt);
  if (S->frame != FB_FRAME_FIXED) {
    double omeganew = fb_psys_info(S, FB_PS_GET) / dt;
    S->domega = omeganew - S->omegaframe;
    S->omegaframe = omeganew;
  }
  fb_psys_rotate(S, S->omegaframe * dt);
  sc->dt = dt;
  sc->domega = S->frame != FB_FRAME_FIXED ? S->domega : 0.0;
  sc->omegaframe = S->omegaframe;
  sc->omegaframe0 = S->omegaframe0;
  S->phys_time += dt;
  S->step_count++;
  S->last_dt = dt;
  return dt;
}

/* Initial planetary system (psys.c:190-210) and frame (main.c:240-242). */
static FB_HD inline void fb_psys_init(fb_psys *S, int np, const double *dist, const double *mass,
                                      const int *feeldisk, const int *feelothers, double ecc, double inc, int frame,
                                      double omegaframe, int indirect_term, double roche_smoothing,
                                      double aspectratio, double flaringindex, double thickness_smoothing) {
  int n;
  S->np = np;
  S->frame = frame;
  S->indirect_term = indirect_term;
  S->roche_smoothing = roche_smoothing; S->aspectratio = aspectratio;
  S->flaringindex = flaringindex; S->thickness_smoothing = thickness_smoothing;
  S->xmark = S->ymark = S->xaxis_rot = 0.0;
  S->domega = S->phys_time = S->dtemp = S->last_dt = 0.0;
  S->step_count = 0;
  S->status = 0;
  S->t_end = 0.0;
  for (n = 0; n < np; n++) {
    double d = dist[n];
    S->pmass[n] = mass[n];
    S->px[n] = d * (1.0 + ecc);
    S->py[n] = 0.0; S->pz[n] = 0.0;
    S->pvy[n] = sqrt(FB_G * (FB_MSTAR + S->pmass[n]) / d) * sqrt((1.0 - ecc) / (1.0 + ecc)) * cos(inc);
    S->pvx[n] = -0.0000000000 * S->pvy[n];
    S->pvz[n] = S->pvy[n] * sin(inc) / cos(inc);
    S->feelothers[n] = feelothers[n];
    S->feeldisk[n] = feeldisk[n];
  }
  S->omegaframe = omegaframe;
  if (frame != FB_FRAME_FIXED && np > 0) S->omegaframe = fb_psys_info(S, FB_PS_FREQUENCY);
  S->omegaframe0 = S->omegaframe;
}

#endif
