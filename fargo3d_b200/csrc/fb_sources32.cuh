// fb_sources32.cuh -- the source stage of FP32 2D cylindrical disks
// (algogas.c:30-120: ComputePressureFieldIso, the planets' potential,
// CorrectVtheta, SubStep1_x/y, visctensor_cyl + addviscosity_cyl, SubStep2_a/b)
// in FP32 arithmetic, without shared memory or CTA barriers.
//
// Layout of the work: a warp owns 32 consecutive columns (azimuthal cells) of
// a ring and marches down NS rows (radii), keeping the rows j-1, j, j+1 of its
// column in registers; the neighbours i-1 / i+1 come from the adjacent lanes
// by shuffle.  Lanes 0 and 31 are halo lanes: they compute what their
// neighbours need but write nothing, so a warp writes 30 columns.  Every
// quantity (pressure, planet potential, the three viscous stresses) is formed
// once per cell and row, none is staged or recomputed for a tile halo.
//
// Why FP32 is safe here: FP32 disks store v_phi relative to a per-ring
// background vbg (fb_fluid_dev), so no large velocity enters the arithmetic.
// What remains large is the background's own radial balance -- centrifugal
// (B^2 / r) against the star's gravity, with B = vbg + r OMEGAFRAME on the
// face -- two O(1) terms whose difference is O(h^2).  That difference is
// formed per row in FP64 (K_j below) and only the perturbation terms,
// (2 B + d) d / r with d the small relative velocity, the planets' potential
// and the pressure gradient, are formed in FP32.  Likewise the background's
// r-phi shear enters tau_r_phi as one per-row constant (fb_fluid_dev shear_bg,
// formed in FP64).  The planets' potential is the only potential evaluated
// per cell: the star's -GM/r cancels in the x differences and is part of
// K_j in the y difference.
#pragma once
#include "fb_kernels.cuh"

namespace fb {

constexpr int S32_WARPS = 4;                       // warps per CTA
constexpr int S32_OUT = 30;                        // columns written per warp (lanes 1..30)
constexpr int S32_COLS = S32_WARPS * S32_OUT;      // columns per CTA
constexpr int S32_NS = 16;                         // rows per CTA
// resident CTAs per SM the kernel is compiled for (register cap 64 at 8)
#ifndef FB_S32_MINB
#define FB_S32_MINB 8
#endif

// one row of a column: density, sound speed, relative azimuthal velocity
// (CorrectVtheta applied), radial velocity, pressure, planets' potential
struct Cell32 {
  float r, c, u, vy, p, pot;
};

__device__ __forceinline__ float lane_m(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }    // column i-1
__device__ __forceinline__ float lane_p(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }  // column i+1

// The planets of one step in FP32, formed once per CTA: position, mass,
// smoothing^2 + z^2 and the indirect-term factor m / d^3 (0 without it).
struct Planet32 {
  float x, y, m, s2z, ind;
};
__device__ __forceinline__ int planets32_load(const fb_scalars *__restrict__ sc, Planet32 *sp) {
  const int np = sc->nplanets;
  if ((int)threadIdx.x < np) {
    const int n = threadIdx.x;
    Planet32 p;
    p.x = (float)sc->px[n];
    p.y = (float)sc->py[n];
    p.m = (float)sc->pmass[n];
    p.s2z = (float)(sc->psmooth2[n] + sc->pz[n] * sc->pz[n]);
    p.ind = sc->indirect_term ? (float)(sc->pmass[n] / sc->pdist3[n]) : 0.0f;
    sp[n] = p;
  }
  __syncthreads();
  return np;
}

// planets' potential (potential.c:51-208 without the star's term), FP32
__device__ __forceinline__ float pot_planets32(const Planet32 *sp, int np, float XC, float YC) {
  float pot = 0.0f;
  for (int n = 0; n < np; n++) {
    const Planet32 p = sp[n];
    const float dx = XC - p.x, dy = YC - p.y;
    pot += p.ind * (XC * p.x + YC * p.y);
    pot -= p.m * rsqrtf(dx * dx + dy * dy + p.s2z);
  }
  return pot;
}

__device__ __forceinline__ Cell32 load_cell32(const Dims &m, const Geo<float> &g, const float *__restrict__ rho,
                                              const float *__restrict__ cs, const float *__restrict__ vx,
                                              const float *__restrict__ vy, const Planet32 *sp, int np,
                                              float domega, int i, int j) {
  const long long l = m.l(i, j, 0);
  Cell32 o;
  o.r = rho[l];
  o.c = cs[l];
  const float ym = ld(g.ymed + j);
  o.u = vx[l] - domega * ym;     // CorrectVtheta (correct_vtheta.c:55-60)
  o.vy = vy[l];
  o.p = o.r * o.c * o.c;         // ComputePressureFieldIso
  o.pot = pot_planets32(sp, np, ym * ld(g.cos_xmed + i), ym * ld(g.sin_xmed + i));
  return o;
}

// tau_phi_phi and tau_r_r of row j at column i (visctensor_cyl.c): R is row
// j, vyp the radial velocity of row j + 1, uxp the relative azimuthal
// velocity of column i + 1 (all lanes call it: it shuffles)
__device__ __forceinline__ void stress_diag32(const Geo<float> &g, const Cell32 &R, float vyp, int alpha_visc,
                                              float nu, float alpha, float sxi0, int j, float &txx, float &tyy) {
  const float uxp = lane_p(R.u);
  const float visc = alpha_visc ? alpha * R.c * R.c * ld(g.visc_j + j) : nu;
  const float dux = uxp - R.u;
  const float syj = ld(g.syj + j), syjp = ld(g.syj + j + 1), sxj = ld(g.sxj + j);
  float div_v = dux * sxj + (vyp * syjp * sxi0 - R.vy * syj * sxi0);
  div_v *= (2.0f / 3.0f) * ld(g.invvj + j) / sxi0;
  const float izx = ld(g.invdiffxmed + 0) * ld(g.inv_ymed + j);
  txx = visc * R.r * (2.0f * dux * izx - div_v) + visc * R.r * (vyp + R.vy) * ld(g.inv_ymed + j);
  tyy = visc * R.r * (2.0f * (vyp - R.vy) / sxj - div_v);
}

// tau_r_phi at the corner (i - 1/2, j - 1/2) from rows j (R) and j - 1 (Rm);
// the background's shear of this face is shb (shuffles)
__device__ __forceinline__ float stress_rphi32(const Geo<float> &g, const Cell32 &R, const Cell32 &Rm, int alpha_visc,
                                               float nu, float alpha, float shb, int j) {
  const float rxm = lane_m(R.r), rxym = lane_m(Rm.r), cxm = lane_m(R.c), cxym = lane_m(Rm.c), vyxm = lane_m(R.vy);
  float viscm = nu;
  if (alpha_visc) {
    const float s = R.c + cxm + Rm.c + cxym;
    viscm = alpha * 0.0625f * s * s * ld(g.viscm_j + j);
  }
  const float iyi = ld(g.inv_ymin + j);
  return viscm * 0.25f * (R.r + rxm + Rm.r + rxym) *
         ((R.vy - vyxm) * ld(g.invdiffxmed + 0) * iyi + (R.u - Rm.u) * ld(g.inv_dymed + j) -
          0.5f * (R.u + Rm.u) * iyi + shb);
}

__device__ __forceinline__ void b_sources_cyl32(const Dims m, const Geo<float> g, const Geo<double> gd,
    const float *__restrict__ rho, const float *__restrict__ cs, const float *__restrict__ vx,
    const float *__restrict__ vy, float *__restrict__ vxt, float *__restrict__ vyt,
    const fb_scalars *__restrict__ sc, int dust, int viscous, const double *__restrict__ vbg,
    const float *__restrict__ shear_bg, uint3 bid) {
  __shared__ Planet32 s_pl[FB_MAXPLANETS];
  const int np = planets32_load(sc, s_pl);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int iu = (int)(bid.x * S32_WARPS + w) * S32_OUT - 1 + lane;   // unwrapped column of this lane
  const int i = ((iu % m.nx) + m.nx) % m.nx;
  const bool writes = lane >= 1 && lane <= S32_OUT && iu < m.nx;
  const int j0 = FB_NGH + (int)bid.y * S32_NS, j1 = min(j0 + S32_NS, m.ny + FB_NGH);
  if (j0 >= j1) return;
  const double dtd = sc->dt, of = sc->omegaframe;
  const float dt = (float)dtd, domega = (float)sc->domega, nu = (float)sc->nu, alpha = (float)sc->alpha;
  const float sxi0 = ld(g.sxi + 0), idx0 = ld(g.invdiffxmed + 0);
  const float c2 = (float)FB_CVNR;
  // rows j0 - 1 and j0; the stresses of row j0 - 1 and the corner of row j0
  Cell32 A = load_cell32(m, g, rho, cs, vx, vy, s_pl, np, domega, i, j0 - 1);
  Cell32 C0 = load_cell32(m, g, rho, cs, vx, vy, s_pl, np, domega, i, j0);
  float txx_m = 0.f, tyy_m = 0.f, tyx_c = 0.f;
  if (viscous) {
    stress_diag32(g, A, C0.vy, m.alpha, nu, alpha, sxi0, j0 - 1, txx_m, tyy_m);
    tyx_c = stress_rphi32(g, C0, A, m.alpha, nu, alpha, ld(shear_bg + j0), j0);
  }
  for (int j = j0; j < j1; j++) {
    const Cell32 P = load_cell32(m, g, rho, cs, vx, vy, s_pl, np, domega, i, j + 1);
    float txx_c = 0.f, tyy_c = 0.f, tyx_p = 0.f;
    if (viscous) {
      stress_diag32(g, C0, P.vy, m.alpha, nu, alpha, sxi0, j, txx_c, tyy_c);
      tyx_p = stress_rphi32(g, P, C0, m.alpha, nu, alpha, ld(shear_bg + j + 1), j + 1);
    }
    // neighbours by shuffle (every lane takes part)
    const float rxm = lane_m(C0.r), pxm = lane_m(C0.p), potxm = lane_m(C0.pot);
    const float uxm = lane_m(C0.u), uxp = lane_p(C0.u), umxp = lane_p(A.u);
    const float txx_xm = lane_m(txx_c), tyx_xp = lane_p(tyx_c);
    // the background's balance on face j: K = B^2 / r - d(Phi_star)/dr,
    // B = (vbg(j) + vbg(j-1)) / 2 + Ymin(j) OMEGAFRAME, in FP64
    const double Bd = 0.5 * (bg_at(vbg, j) + bg_at(vbg, j - 1)) + ld(gd.ymin + j) * of;
    const float K = (float)(Bd * Bd * ld(gd.inv_ymin + j) -
                            (ld(gd.pot_star + j) - ld(gd.pot_star + j - 1)) * ld(gd.inv_dymed + j));
    const float B = (float)Bd;
    if (writes) {
      const float r = C0.r, rym = A.r;
      const float izx = idx0 * ld(g.inv_ymed + j);
      const float ym = ld(g.ymed + j), ymm = ld(g.ymed + j - 1), yi = ld(g.ymin + j), yip = ld(g.ymin + j + 1);
      const float iyi = ld(g.inv_ymin + j), idym = ld(g.inv_dymed + j);
      const float irx = 1.0f / (r + rxm);   // 1 / (rho + rho_{i-1}) (uniform azimuthal spacing)
      const float ideny = 1.0f / (r * ld(g.sxj + j) + rym * ld(g.sxj + j - 1));
      // SubStep1_x (substep1_x.c:107-117)
      float ax = C0.u;
      if (!dust) ax -= 2.0f * dt * irx * (C0.p - pxm) * izx;
      ax -= (C0.pot - potxm) * dt * izx;
      // SubStep1_y (substep1_y.c:146-192, cylindrical)
      float ay = C0.vy;
      if (!dust) ay -= 2.0f * dt * ideny * (C0.p - A.p);
      const float d = 0.25f * (C0.u + uxp + A.u + umxp);
      ay += (K + (2.0f * B + d) * d * iyi - (C0.pot - A.pot) * idym) * dt;
      if (viscous) {
        // addviscosity_cyl (addviscosity_cyl.c:106-124)
        ax += 2.0f * (txx_c - txx_xm) * izx * irx * dt;
        ax += 2.0f * (yip * yip * tyx_p - yi * yi * tyx_c) / ((yip - yi) * ym * ym * (rxm + r)) * dt;
        ay += 2.0f * (ym * tyy_c - ymm * tyy_m) / ((ym - ymm) * (r + rym) * yi) * dt;
        ay += 2.0f * (tyx_xp - tyx_c) / (sxi0 * yi * (r + rym)) * dt;
        ay -= (txx_c + txx_m) / (yi * (r + rym)) * dt;
      }
      // SubStep2_a / SubStep2_b (substep2_a.c:107-129, substep2_b.c:150-175)
      float dv = uxp - C0.u;
      const float qx = dv < 0.0f ? c2 * c2 * r * dv * dv : 0.0f;
      dv = C0.u - uxm;
      const float qxm = dv < 0.0f ? c2 * c2 * rxm * dv * dv : 0.0f;
      dv = P.vy - C0.vy;
      const float qy = dv < 0.0f ? c2 * c2 * r * dv * dv : 0.0f;
      dv = C0.vy - A.vy;
      const float qym = dv < 0.0f ? c2 * c2 * rym * dv * dv : 0.0f;
      ax += -2.0f * dt * (qx - qxm) * irx * izx;
      ay += -2.0f * (qy - qym) * ideny * dt;
      const long long l = m.l(i, j, 0);
      vxt[l] = ax;   // relative to the background, as the state
      vyt[l] = ay;
    }
    A = C0;
    C0 = P;
    txx_m = txx_c;
    tyy_m = tyy_c;
    tyx_c = tyx_p;
  }
}

// ---------------------------------------------------------------------------
// NewVelocity_x/y (newvel_x.c:81, newvel_y.c:70) and StockholmBoundary
// (stockholm.c:129-185) of FP32 2D disks.  A lane owns a column and marches
// over NV32_R rows: row j-1's transported density and upper-face radial
// momentum, which newvel_y reads for row j, are the previous iteration's own
// loads; the column i-1 values newvel_x reads come from the adjacent lane
// (lane 0 loads them).  The azimuthal spacing is uniform, so Sxi cancels from
// the x average; the momenta are relative to the frame and the ring
// background, and the velocity they give is the stored (relative) vx.  Each
// component is one correctly rounded division (see b_newvel).
constexpr int NV32_R = 8;

__device__ __forceinline__ void b_newvel_cyl32(const Dims m, const Geo<float> g, const float *__restrict__ rt,
    const float *__restrict__ mpx, const float *__restrict__ mmx, const float *__restrict__ mpy,
    const float *__restrict__ mmy, float *__restrict__ rho, float *__restrict__ vx, float *__restrict__ vy,
    const float *__restrict__ rho0, const float *__restrict__ vx0, const float *__restrict__ vy0,
    const double *__restrict__ ramps, int stockholm, const fb_scalars *__restrict__ sc, uint3 bid) {
  const int lane = threadIdx.x & 31;
  const int i = (int)bid.x * blockDim.x + threadIdx.x;
  const int j0 = FB_NGH + (int)bid.y * NV32_R, j1 = min(j0 + NV32_R, m.ny + FB_NGH);
  const bool act = i < m.nx;
  const int im = i > 0 ? i - 1 : m.nx - 1;
  const int ic = act ? i : m.nx - 1;   // lanes past the ring load a valid cell and write nothing
  const float dt = (float)sc->dt, dof = (float)(sc->omegaframe - sc->omegaframe0);
  // every load of the tile first (rows past j1 repeat the last row and are
  // not written): the kernel is bound by the loads in flight
  const int nr = j1 - j0;
  const bool edge = lane == 0 || i == 0;   // column i-1 outside this warp (or the wrap)
  float a_r[NV32_R], a_mmx[NV32_R], a_mpx[NV32_R], a_mmy[NV32_R], a_mpy[NV32_R], e_r[NV32_R], e_mpx[NV32_R];
#pragma unroll
  for (int q = 0; q < NV32_R; q++) {
    const int j = j0 + min(q, nr - 1);
    const long long l = m.l(ic, j, 0);
    a_r[q] = rt[l]; a_mmx[q] = mmx[l]; a_mpx[q] = mpx[l]; a_mmy[q] = mmy[l]; a_mpy[q] = mpy[l];
    if (edge) {
      const long long lxm = m.l(im, j, 0);
      e_r[q] = rt[lxm];
      e_mpx[q] = mpx[lxm];
    } else {
      e_r[q] = 0.0f;
      e_mpx[q] = 0.0f;
    }
  }
  // row j0 - 1: its density and upper-face radial momentum
  float r_m = rt[m.l(ic, j0 - 1, 0)], mpy_m = mpy[m.l(ic, j0 - 1, 0)];
#pragma unroll
  for (int q = 0; q < NV32_R; q++) {
    const int j = j0 + min(q, nr - 1);
    const long long l = m.l(ic, j, 0);
    const float r = a_r[q], mm_x = a_mmx[q], mp_x = a_mpx[q], mm_y = a_mmy[q], mp_y = a_mpy[q];
    float rxm = lane_m(r), mpxm = lane_m(mp_x);
    if (edge) {
      rxm = e_r[q];
      mpxm = e_mpx[q];
    }
    const float ivj = ld(g.invvj + j), ivjm = ld(g.invvj + j - 1), rc = ld(g.ymed + j);
    float nvx = __fdiv_rn(mm_x + mpxm, (r + rxm) * rc);
    float nvy = __fdiv_rn(mm_y * ivjm + mpy_m * ivj, r * ivjm + r_m * ivj);
    float nrho = r;
    if (stockholm) {
      const float ramp = (float)ramps[j];
      if (ramp > 0.0f) {
        const float taud = ld(g.tau_j + j) / ramp;
        const float vx0t = vx0[j] - dof * rc;
        nrho = (nrho * taud + rho0[j] * dt) / (dt + taud);
        nvx = (nvx * taud + vx0t * dt) / (dt + taud);
        nvy = (nvy * taud + vy0[j] * dt) / (dt + taud);
      }
    }
    if (act && q < nr) {
      rho[l] = nrho;
      vx[l] = nvx;
      vy[l] = nvy;
    }
    r_m = r;
    mpy_m = mp_y;
  }
}

static __global__ void __launch_bounds__(S32_WARPS * 32, FB_S32_MINB) k_sources_cyl32(Dims m, Geo<float> g, Geo<double> gd,
    const float *__restrict__ rho, const float *__restrict__ cs, const float *__restrict__ vx,
    const float *__restrict__ vy, float *__restrict__ vxt, float *__restrict__ vyt,
    const fb_scalars *__restrict__ scp, int dust, int viscous, const double *__restrict__ vbg,
    const float *__restrict__ shear_bg) {
  b_sources_cyl32(m, g, gd, rho, cs, vx, vy, vxt, vyt, scp, dust, viscous, vbg, shear_bg, blockIdx);
}

static __global__ void __launch_bounds__(128) k_newvel_cyl32(Dims m, Geo<float> g, const float *__restrict__ rt,
    const float *__restrict__ mpx, const float *__restrict__ mmx, const float *__restrict__ mpy,
    const float *__restrict__ mmy, float *__restrict__ rho, float *__restrict__ vx, float *__restrict__ vy,
    const float *__restrict__ rho0, const float *__restrict__ vx0, const float *__restrict__ vy0,
    const double *__restrict__ ramps, int stockholm, const fb_scalars *__restrict__ scp) {
  b_newvel_cyl32(m, g, rt, mpx, mmx, mpy, mmy, rho, vx, vy, rho0, vx0, vy0, ramps, stockholm, scp, blockIdx);
}

// ---------------------------------------------------------------------------
// The radial sweep of FP32 2D disks (TransportY, transport.c:24-46, for the
// density and the four momenta; vanleer_y_a/_b, divrho, update_y,
// update_density_y): b_sweep_col's work with the per-row factors formed from
// the row tables -- the zone sizes and their reciprocals, the face areas and
// the cell updates for the uniform azimuthal spacing -- and the specific
// momenta taken directly as v R or v (DivideByRho of rho v R is v R), so the
// only division per cell and quantity is the limiter's harmonic mean.  A
// thread marches down a segment of NS rows of one column.  The azimuthal
// momenta are frame- and background-relative as in b_sweep_col.
template <int NS>
__device__ __forceinline__ void b_sweep_col32(const Dims m, const Geo<float> g, const float *__restrict__ rho,
    const float *__restrict__ vxt, const float *__restrict__ vyt, const float *__restrict__ dlb, int clo, int chi,
    float *__restrict__ rho_out, float *__restrict__ o_mpx, float *__restrict__ o_mmx, float *__restrict__ o_mpy,
    float *__restrict__ o_mmy, const fb_scalars *__restrict__ scp, uint3 bid) {
  const int i = (int)bid.x * blockDim.x + threadIdx.x;
  if (i >= m.nx) return;
  const int c0 = clo + (int)bid.z * NS;
  if (c0 > chi) return;
  const float dt = (float)scp->dt, of = (float)scp->omegaframe;
  const int cmax = chi + 2;
  const int ixp = i < m.nx - 1 ? i + 1 : 0;
  const float sxi0 = ld(g.sxi + 0), isxi0 = 1.0f / sxi0;
  // The thread marches down its column from face c0 to face c0 + NS, holding
  // of every quantity only the cells around the current face: each cell is
  // loaded once, its van Leer slope formed once and each face's interface
  // value once (a window per segment would form them for the halo cells
  // again).  Quantities: 0 rho, 1 vxt(i+1) R, 2 vxt(i) R, 3 vyt(c+1), 4 vyt(c)
  // (momenta_x.c:76-85 relative, momenta_y.c:65-66, over rho); rows past
  // cmax are clamped like the field rows and only feed faces and cells that
  // are not stored.
  auto load = [&](int c, float *A) {
    const int rc = min(c, cmax);
    const long long l = m.l(i, rc, 0);
    const float ym = ld(g.ymed + rc);
    A[0] = rho[l];
    A[1] = vxt[m.l(ixp, rc, 0)] * ym;
    A[2] = vxt[l] * ym;
    A[3] = vyt[l + m.pitch];
    A[4] = vyt[l];
  };
  // OMEGAFRAME (R^2(c) - R^2(c-1)) + (vbg R)(c) - (vbg R)(c-1): the
  // neighbour difference of the offset the azimuthal momenta leave out
  auto offr = [&](int c) -> float { return c <= cmax ? of * ld(g.dr2_j + c) + (dlb ? ld(dlb + c) : 0.0f) : 0.0f; };
  auto zn = [&](int c) -> float { return ld(g.sxj + min(c, cmax)); };
  // vanleer_y_a: the slope of cell c from cells c-1, c, c+1, the zone
  // reciprocals of c and c+1 and (momenta 1, 2) the offsets of c and c+1
  auto slope = [&](int q, float am, float a0, float ap, float offc, float offp, float izc, float izp) -> float {
    float dqm = a0 - am, dqp = ap - a0;
    if (q == 1 || q == 2) { dqm += offc; dqp += offp; }
    dqm *= izc;
    dqp *= izp;
    return (dqp * dqm <= 0.0f) ? 0.0f : 2.0f * dqp * dqm / (dqm + dqp);
  };
  float Am[5], A0[5], Ap[5], slm[5], sl0[5], qsm[5], qs0[5];
  load(c0 - 2, Am);
  load(c0 - 1, A0);
  load(c0, Ap);
  float offm = offr(c0 - 1), off0 = offr(c0), offp;
  float znm = zn(c0 - 1), zn0 = zn(c0), znp;
  float iz0 = 1.0f / zn0, izp;
  {
    const float izm = 1.0f / znm;
#pragma unroll
    for (int q = 0; q < 5; q++) slm[q] = slope(q, Am[q], A0[q], Ap[q], offm, off0, izm, iz0);
  }
  // shift: cells c0-1, c0 become "previous" and "current"
#pragma unroll
  for (int q = 0; q < 5; q++) { Am[q] = A0[q]; A0[q] = Ap[q]; }
  // now Am = A(c0-1), A0 = A(c0), slm = slope(c0-1), znm = zn(c0-1), zn0 = zn(c0),
  // offm = off(c0-1), off0 = off(c0)
  float velm = 0.0f, sfm = 0.0f;
#pragma unroll
  for (int s2 = 0; s2 <= NS; s2++) {
    const int f = c0 + s2;   // the face between cells f-1 and f
    load(f + 1, Ap);
    offp = offr(f + 1);
    znp = zn(f + 1);
    izp = 1.0f / znp;
#pragma unroll
    for (int q = 0; q < 5; q++) sl0[q] = slope(q, Am[q], A0[q], Ap[q], off0, offp, iz0, izp);
    // vanleer_y_b: interface values at face f, upwind by the face velocity
    const float vel = A0[4];
#pragma unroll
    for (int q = 0; q < 5; q++) {
      if (vel > 0.0f) qs0[q] = Am[q] + 0.5f * (znm - vel * dt) * slm[q];
      else qs0[q] = A0[q] - 0.5f * (zn0 + vel * dt) * sl0[q];
    }
    const float sf0 = ld(g.syj + min(f, cmax)) * sxi0;
    if (s2 > 0) {   // update_y / update_density_y of cell c = f - 1
      const int c = f - 1;
      if (c <= chi) {
        const float fin = dt * ld(g.invvj + min(c, cmax)) * isxi0;
        const long long l = m.l(i, c, 0);
        float *qo[4] = {o_mpx, o_mmx, o_mpy, o_mmy};
#pragma unroll
        for (int q = 1; q < 5; q++) {
          float qin = qsm[q], qout = qs0[q];
          if (q <= 2) {
            if (velm > 0.0f) qin -= offm;          // upwind cell c-1
            if (!(vel > 0.0f)) qout += off0;       // upwind cell c+1
          }
          const float flux = velm * qin * qsm[0] * sfm - vel * qout * qs0[0] * sf0;
          qo[q - 1][l] = Am[q] * Am[0] + flux * fin;
        }
        const float flux = velm * qsm[0] * sfm - vel * qs0[0] * sf0;
        rho_out[l] = Am[0] + flux * fin;
      }
    }
#pragma unroll
    for (int q = 0; q < 5; q++) { Am[q] = A0[q]; A0[q] = Ap[q]; slm[q] = sl0[q]; qsm[q] = qs0[q]; }
    velm = vel; sfm = sf0;
    offm = off0; off0 = offp;
    znm = zn0; zn0 = znp; iz0 = izp;
  }
}

template <int NS>
static __global__ void __launch_bounds__(128, 8) k_sweep_col32(Dims m, Geo<float> g, const float *__restrict__ rho,
    const float *__restrict__ vxt, const float *__restrict__ vyt, const float *__restrict__ dlb, int clo, int chi,
    float *__restrict__ rho_out, float *__restrict__ o_mpx, float *__restrict__ o_mmx, float *__restrict__ o_mpy,
    float *__restrict__ o_mmy, const fb_scalars *__restrict__ scp) {
  b_sweep_col32<NS>(m, g, rho, vxt, vyt, dlb, clo, chi, rho_out, o_mpx, o_mmx, o_mpy, o_mmy, scp, blockIdx);
}

// ---------------------------------------------------------------------------
// CFL time step of FP32 2D disks (cfl.c:135-258, cfl_b.c:14-39): the limits
// of cfl_cell32 for a tile of 128 columns x CFL32_R rows, a lane per column
// marching over the rows with every load of the tile issued up front (the
// kernel is a stream of four fields; it is bound by how many loads are in
// flight), the x neighbour's vx by shuffle, the next row's vy reused.  The
// tile's minimum (with the shear limits of its rows) is folded into the
// disk's as in b_cfl; non-finite limits and non-positive densities set the
// disk's flag word.
constexpr int CFL32_R = 8;

__device__ __forceinline__ void b_cfl_cyl32(const Dims m, const Geo<float> g, const float *__restrict__ rho,
    const float *__restrict__ cs, const float *__restrict__ vx, const float *__restrict__ vy,
    const double *__restrict__ vxmed, const double *__restrict__ vbg, float nu, float alpha, double cfl_num,
    double mindx, unsigned long long *__restrict__ dtmin, uint3 bid) {
  const int lane = threadIdx.x & 31;
  const int i = (int)bid.x * blockDim.x + threadIdx.x;
  const int j0 = FB_NGH + (int)bid.y * CFL32_R;
  const int nr = min(CFL32_R, m.ny + FB_NGH - j0);
  const bool act = i < m.nx;
  const int ic = act ? i : m.nx - 1;
  const int ixp = ic < m.nx - 1 ? ic + 1 : 0;
  float r[CFL32_R], c[CFL32_R], u[CFL32_R], v[CFL32_R + 1], uxp_edge[CFL32_R];
#pragma unroll
  for (int q = 0; q < CFL32_R; q++) {
    const int j = j0 + min(q, nr - 1);
    const long long l = m.l(ic, j, 0);
    r[q] = rho[l];
    c[q] = cs[l];
    u[q] = vx[l];
    v[q] = vy[l];
    uxp_edge[q] = (lane == 31 || ic == m.nx - 1) ? vx[m.l(ixp, j, 0)] : 0.0f;
  }
  v[CFL32_R] = vy[m.l(ic, j0 + nr, 0)];
  const float cflf = (float)cfl_num;
  const float izx0 = ld(g.invdiffxmed + 0);
  float mn = 1e20f;
  bool bad = false;
#pragma unroll
  for (int q = 0; q < CFL32_R; q++) {
    const int j = j0 + min(q, nr - 1);
    float uxp = lane_p(u[q]);
    if (lane == 31 || ic == m.nx - 1) uxp = uxp_edge[q];
    const float vyp = q + 1 < nr ? v[q + 1] : v[CFL32_R];
    const float vmf = (float)(vxmed[j] - bg_at(vbg, j));
    const float izx = izx0 * ld(g.inv_ymed + j), izy = 1.0f / ld(g.sxj + j);
    const float visc = m.alpha ? alpha * c[q] * c[q] * ld(g.visc_j + j) : nu;
    const float mx7 = fmaxf(izx, izy);
    const float c1 = fabsf(c[q]) * mx7;
    const float c2 = fmaxf(fabsf(u[q] - vmf), fabsf(uxp - vmf)) * izx;
    const float c3 = fmaxf(fabsf(v[q]), fabsf(vyp)) * izy;
    const float c5 = fmaxf(fabsf(uxp - u[q]) * izx, fabsf(vyp - v[q]) * izy) * (4.0f * (float)FB_CVNR);
    const float c7 = 4.0f * visc * (mx7 * mx7);
    const float dtc = cflf * rsqrtf(c1 * c1 + c2 * c2 + c3 * c3 + c5 * c5 + c7 * c7);
    if (act && q < nr) {
      bad |= !(dtc == dtc) || !(r[q] > 0.0f);
      mn = fminf(mn, dtc);
    }
  }
  double mnd = (double)mn;
  if ((int)threadIdx.x < nr) {   // the shear limits of the tile's rows (a MIN: repeats are harmless)
    const int j = j0 + threadIdx.x;
    const double shear = cfl_shear(g, vxmed, cfl_num, mindx, j, j);
    if (shear < mnd) mnd = shear;
  }
  if (bad) atomicOr(dtmin + 1, 1ull);
  cfl_commit(mnd, dtmin);
}

// ---------------------------------------------------------------------------
// CFL limits and NewVelocity of FP32 2D disks whose rings hold a multiple of
// four cells: a thread takes four consecutive cells of a row with 16-byte
// loads (and stores), so the fields stream like a copy.  The x neighbour of
// its last (CFL) or first (NewVelocity) cell comes from the next or previous
// lane when that lane holds the adjacent four cells of the same row, else
// from one load; the row above (CFL: vy) or below (NewVelocity: density and
// radial momentum) by a second 16-byte load.  Per cell the arithmetic of
// b_cfl_cyl32 / b_newvel_cyl32; a CTA of Q32_T threads takes 4 Q32_T cells.
constexpr int Q32_T = 128;
__device__ __forceinline__ float4 ld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ float q4(const float4 &a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : (k == 2 ? a.z : a.w)); }

__device__ __forceinline__ void b_cfl_cyl32q(const Dims m, const Geo<float> g, const float *__restrict__ rho,
    const float *__restrict__ cs, const float *__restrict__ vx, const float *__restrict__ vy,
    const double *__restrict__ vxmed, const double *__restrict__ vbg, float nu, float alpha, double cfl_num,
    double mindx, unsigned long long *__restrict__ dtmin, int blk) {
  const int lane = threadIdx.x & 31;
  const int qpr = m.nx >> 2, nq = qpr * m.ny;
  const int t = blk * Q32_T + (int)threadIdx.x;
  const bool act = t < nq;
  const int tc = act ? t : nq - 1;
  const int j = FB_NGH + tc / qpr, q = tc - (j - FB_NGH) * qpr;
  const long long l = m.l(4 * q, j, 0);
  const float4 r4 = ld4(rho + l), c4 = ld4(cs + l), u4 = ld4(vx + l), v4 = ld4(vy + l), vp4 = ld4(vy + l + m.pitch);
  // vx of cell 4q + 4: the next lane's first cell, or a load (ring wrap, warp edge)
  float uxp3 = __shfl_down_sync(0xffffffffu, u4.x, 1);
  if (lane == 31 || q == qpr - 1) uxp3 = vx[q == qpr - 1 ? m.l(0, j, 0) : l + 4];
  const float cflf = (float)cfl_num;
  const float vmf = (float)(vxmed[j] - bg_at(vbg, j));
  const float izx = ld(g.invdiffxmed + 0) * ld(g.inv_ymed + j), izy = 1.0f / ld(g.sxj + j);
  const float vj = ld(g.visc_j + j);
  const float mx7 = fmaxf(izx, izy);
  float mn = 1e20f;
  bool bad = false;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float c = q4(c4, k), u = q4(u4, k), v = q4(v4, k), vyp = q4(vp4, k);
    const float uxp = k < 3 ? q4(u4, k + 1) : uxp3;
    const float visc = m.alpha ? alpha * c * c * vj : nu;
    const float c1 = fabsf(c) * mx7;
    const float c2 = fmaxf(fabsf(u - vmf), fabsf(uxp - vmf)) * izx;
    const float c3 = fmaxf(fabsf(v), fabsf(vyp)) * izy;
    const float c5 = fmaxf(fabsf(uxp - u) * izx, fabsf(vyp - v) * izy) * (4.0f * (float)FB_CVNR);
    const float c7 = 4.0f * visc * (mx7 * mx7);
    const float dtc = cflf * rsqrtf(c1 * c1 + c2 * c2 + c3 * c3 + c5 * c5 + c7 * c7);
    bad |= !(dtc == dtc) || !(q4(r4, k) > 0.0f);
    mn = fminf(mn, dtc);
  }
  double mnd = act ? (double)mn : 1e20;
  if (!act) bad = false;
  if (act && q == 0) {   // the shear limit of row j (once per row)
    const double shear = cfl_shear(g, vxmed, cfl_num, mindx, j, j);
    if (shear < mnd) mnd = shear;
  }
  if (bad) atomicOr(dtmin + 1, 1ull);
  cfl_commit(mnd, dtmin);
}

__device__ __forceinline__ void b_newvel_cyl32q(const Dims m, const Geo<float> g, const float *__restrict__ rt,
    const float *__restrict__ mpx, const float *__restrict__ mmx, const float *__restrict__ mpy,
    const float *__restrict__ mmy, float *__restrict__ rho, float *__restrict__ vx, float *__restrict__ vy,
    const float *__restrict__ rho0, const float *__restrict__ vx0, const float *__restrict__ vy0,
    const double *__restrict__ ramps, int stockholm, const fb_scalars *__restrict__ sc, int blk) {
  const int lane = threadIdx.x & 31;
  const int qpr = m.nx >> 2, nq = qpr * m.ny;
  const int t = blk * Q32_T + (int)threadIdx.x;
  const bool act = t < nq;
  const int tc = act ? t : nq - 1;
  const int j = FB_NGH + tc / qpr, q = tc - (j - FB_NGH) * qpr;
  const long long l = m.l(4 * q, j, 0);
  const float4 r4 = ld4(rt + l), mmx4 = ld4(mmx + l), mpx4 = ld4(mpx + l), mmy4 = ld4(mmy + l), mpy4 = ld4(mpy + l);
  const float4 rm4 = ld4(rt + l - m.pitch), pym4 = ld4(mpy + l - m.pitch);
  // cell 4q - 1: the previous lane's last cell, or a load (ring wrap, warp edge)
  float rxm0 = __shfl_up_sync(0xffffffffu, r4.w, 1), pxm0 = __shfl_up_sync(0xffffffffu, mpx4.w, 1);
  if (lane == 0 || q == 0) {
    const long long lm = q > 0 ? l - 1 : m.l(m.nx - 1, j, 0);
    rxm0 = rt[lm];
    pxm0 = mpx[lm];
  }
  const float dt = (float)sc->dt, dof = (float)(sc->omegaframe - sc->omegaframe0);
  const float ivj = ld(g.invvj + j), ivjm = ld(g.invvj + j - 1), rc = ld(g.ymed + j);
  float ramp = 0.0f, taud = 0.0f, vx0t = 0.0f, r0 = 0.0f, vy0j = 0.0f;
  if (stockholm) {
    ramp = (float)ramps[j];
    if (ramp > 0.0f) {
      taud = ld(g.tau_j + j) / ramp;
      vx0t = vx0[j] - dof * rc;
      r0 = rho0[j];
      vy0j = vy0[j];
    }
  }
  float o_r[4], o_u[4], o_v[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float r = q4(r4, k);
    const float rxm = k > 0 ? q4(r4, k - 1) : rxm0, mpxm = k > 0 ? q4(mpx4, k - 1) : pxm0;
    float nvx = __fdiv_rn(q4(mmx4, k) + mpxm, (r + rxm) * rc);
    float nvy = __fdiv_rn(q4(mmy4, k) * ivjm + q4(pym4, k) * ivj, r * ivjm + q4(rm4, k) * ivj);
    float nrho = r;
    if (stockholm && ramp > 0.0f) {
      nrho = (nrho * taud + r0 * dt) / (dt + taud);
      nvx = (nvx * taud + vx0t * dt) / (dt + taud);
      nvy = (nvy * taud + vy0j * dt) / (dt + taud);
    }
    o_r[k] = nrho;
    o_u[k] = nvx;
    o_v[k] = nvy;
  }
  if (act) {
    reinterpret_cast<float4 *>(rho + l)[0] = make_float4(o_r[0], o_r[1], o_r[2], o_r[3]);
    reinterpret_cast<float4 *>(vx + l)[0] = make_float4(o_u[0], o_u[1], o_u[2], o_u[3]);
    reinterpret_cast<float4 *>(vy + l)[0] = make_float4(o_v[0], o_v[1], o_v[2], o_v[3]);
  }
}

}  // namespace fb
