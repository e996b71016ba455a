// fb_kernels.cuh -- the hydro-step kernels, templated on the field precision.
//
// Stage kernels of one hydro step (FARGO3D main.c:361-448):
//   rowsum      ring sums of v_phi * dphi (ComputeVmed, compute_vmed.c:10-39)
//   cfl         per-cell time step, CFL minimum and shear limit (cfl.c, cfl_b.c)
//   sources     pressure, potential, SubStep1, viscous stress, SubStep2 fused in a
//               shared-memory tile (algogas.c:30-120)
//   bnd         ghost rows / layers (generated boundaries, algogas.c:11-27)
//   sweep_z/y   conservative upwind van Leer transport along a column, one thread
//               per column marching in its direction (transport.c:24-46, 84-127)
//   sweep_x     one CTA per ring: FARGO residual, van Leer, PPA and integer shift
//               in shared memory (transport.c:129-158)
//   newvel      new velocities and Stockholm damping (newvel_*.c, stockholm.c)
//
// Floating-point expressions follow the reference's evaluation order exactly
// (including the order implied by its geometry macros), so the FP64
// instantiation, compiled without FMA contraction, reproduces the CPU build.
#pragma once
#include <type_traits>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "fb_dev.h"

#define FB_CVNR 1.41
#define FB_NGH 3

namespace fb {

template <typename T>
struct Geo {
  const T *xmin, *ymin, *zmin, *xmed, *ymed, *zmed, *invdiffxmed;
  const T *sxi, *sxj, *syj, *szj, *sxk, *syk, *szk, *invvj;
  const T *sin_zmed, *cos_zmed, *sin_zmin, *cos_zmin;
  const T *cos_xmed, *sin_xmed;
  const T *visc_j, *viscm_j, *tau_j;
  const T *r2_j, *dr2_j, *s2_k, *ds2_k;
  const T *inv_ymed, *inv_ymin, *inv_dymed, *pot_star;
};

template <typename T>
__host__ __device__ inline Geo<T> geo_of(const fb_geom_dev &g) {
  Geo<T> o;
  o.xmin = (const T *)g.xmin; o.ymin = (const T *)g.ymin; o.zmin = (const T *)g.zmin;
  o.xmed = (const T *)g.xmed; o.ymed = (const T *)g.ymed; o.zmed = (const T *)g.zmed;
  o.invdiffxmed = (const T *)g.invdiffxmed; o.sxi = (const T *)g.sxi;
  o.sxj = (const T *)g.sxj; o.syj = (const T *)g.syj; o.szj = (const T *)g.szj;
  o.sxk = (const T *)g.sxk; o.syk = (const T *)g.syk; o.szk = (const T *)g.szk;
  o.invvj = (const T *)g.invvj;
  o.sin_zmed = (const T *)g.sin_zmed; o.cos_zmed = (const T *)g.cos_zmed;
  o.sin_zmin = (const T *)g.sin_zmin; o.cos_zmin = (const T *)g.cos_zmin;
  o.cos_xmed = (const T *)g.cos_xmed; o.sin_xmed = (const T *)g.sin_xmed;
  o.visc_j = (const T *)g.visc_j; o.viscm_j = (const T *)g.viscm_j; o.tau_j = (const T *)g.tau_j;
  o.r2_j = (const T *)g.r2_j; o.dr2_j = (const T *)g.dr2_j; o.s2_k = (const T *)g.s2_k; o.ds2_k = (const T *)g.ds2_k;
  o.inv_ymed = (const T *)g.inv_ymed; o.inv_ymin = (const T *)g.inv_ymin; o.inv_dymed = (const T *)g.inv_dymed;
  o.pot_star = (const T *)g.pot_star;
  return o;
}

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

struct Dims {
  int nx, ny, nz, sy, sz, pitch;
  long long stride;
  int is3d, sph, alpha;
  int adiab;        // ADIABATIC: the cs field holds the internal energy e
  double gam;       // GAMMA
  int bclo, bchi;   // the radial edges are the mesh's own (boundary templates) or a slab's
  __device__ __forceinline__ long long l(int i, int j, int k) const {
    return (long long)i + (long long)j * pitch + (long long)k * stride;
  }
};

__host__ __device__ inline Dims dims_of(const fb_disk_dev &d) {
  Dims m;
  m.nx = d.nx; m.ny = d.ny; m.nz = d.nz; m.sy = d.sy; m.sz = d.sz; m.pitch = d.pitch;
  m.stride = d.stride; m.is3d = d.is3d; m.sph = d.spherical; m.alpha = d.alpha_visc;
  m.adiab = d.adiabatic; m.gam = d.gamma;
  m.bclo = d.bc_lo; m.bchi = d.bc_hi;
  return m;
}

__device__ __forceinline__ int wrapx(int i, int nx) { return i < 0 ? i + nx : (i >= nx ? i - nx : i); }

// ---------------------------------------------------------------------------
// Ordered ring sums (ComputeVweight + reduction_SUM, compute_vmed.c:42-97,
// reduction_generic.c:5-23): vmed[j,k] = (sum_i v[i] * (xmin[i+1]-xmin[i])) /
// (XMAX - XMIN), accumulated sequentially in i as the reference does, one
// lane per ring; the rings' rows are staged through shared memory so that
// global loads stay coalesced.  32 rings per CTA of 256 threads.
template <typename T, bool ORDERED, typename S = T, int R = 32>
__device__ __forceinline__ void b_rowsum(Dims m, Geo<double> gd, const S *__restrict__ v,
                                                 double *__restrict__ out, double xlen, uint3 bid) {
  // R rings per CTA of 256 threads: 32 for meshes with many rings, 8 where
  // the rings are few (2D) and 32 per CTA would leave most SMs idle
  constexpr int CH = 128;
  __shared__ double buf[R][CH + 1];
  const int nring = m.sy * m.sz;
  const int r0 = bid.x * R;
  const int tid = threadIdx.x;
  double acc = 0.0;
  const int myring = r0 + (tid & (R - 1));
  for (int c0 = 0; c0 < m.nx; c0 += CH) {
    const int cw = min(CH, m.nx - c0);
    for (int e = tid; e < R * CH; e += blockDim.x) {
      const int rr = e / CH, ii = e - rr * CH;
      const int ring = r0 + rr;
      double val = 0.0;
      if (ring < nring && ii < cw) {
        const int j = ring % m.sy, k = ring / m.sy;
        const int i = c0 + ii;
        val = (double)v[m.l(i, j, k)] * (ld(gd.xmin + i + 1) - ld(gd.xmin + i));
      }
      buf[rr][ii] = val;
    }
    __syncthreads();
    if (ORDERED) {
      if (tid < R) {
        for (int ii = 0; ii < cw; ii++) acc = acc + buf[tid][ii];
      }
    } else {
      // warp w sums rings (R/8)w .. (R/8)(w+1)-1 with a shuffle tree (order-free path)
      const int w = tid >> 5, lane = tid & 31;
      for (int q = 0; q < R / 8; q++) {
        const int rr = w * (R / 8) + q;
        double s = 0.0;
        for (int ii = lane; ii < cw; ii += 32) s += buf[rr][ii];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) buf[rr][CH] = (c0 == 0 ? 0.0 : buf[rr][CH]) + s;
      }
    }
    __syncthreads();
  }
  if (tid < R && myring < nring) {
    double tot = ORDERED ? acc : buf[tid][CH];
    out[myring] = tot / xlen;
  }
}
// Order-free ring sums (FP32 storage): one warp per ring, lanes striding
// over the ring with an FP64 accumulator, then a shuffle tree; 8 rings per
// CTA of 256 threads, no shared memory and no barrier.  vbg: the ring's
// background azimuthal velocity (FP32 disks store v - vbg), added back so
// the mean is that of the full velocity.
template <typename S>
__device__ __forceinline__ void b_rowsum_warp(Dims m, Geo<double> gd, const S *__restrict__ v,
                                              double *__restrict__ out, double xlen, const double *__restrict__ vbg,
                                              uint3 bid) {
  const int ring = bid.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (ring >= m.sy * m.sz) return;
  const int j = ring % m.sy, k = ring / m.sy;
  const S *row = v + m.l(0, j, k);
  double acc = 0.0;
  if constexpr (sizeof(S) == 4) {
    if ((m.nx & 127) == 0 && (((uintptr_t)row) & 15) == 0) {
      // FP32 rings of a multiple of 128 cells: float4 loads, the uniform
      // azimuthal spacing factored out of the sum
      const float4 *r4 = reinterpret_cast<const float4 *>(row);
#pragma unroll 4
      for (int q = lane; q < (m.nx >> 2); q += 32) {
        const float4 x = r4[q];
        acc += ((double)x.x + (double)x.y) + ((double)x.z + (double)x.w);
      }
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) out[ring] = acc * (ld(gd.xmin + 1) - ld(gd.xmin + 0)) / xlen + (vbg ? vbg[ring] : 0.0);
      return;
    }
  }
  for (int i = lane; i < m.nx; i += 32) acc += (double)row[i] * (ld(gd.xmin + i + 1) - ld(gd.xmin + i));
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[ring] = acc / xlen + (vbg ? vbg[ring] : 0.0);
}

template <typename S>
__global__ void __launch_bounds__(256) k_rowsum_warp(Dims m, Geo<double> gd, const S *__restrict__ v,
                                                      double *__restrict__ out, double xlen,
                                                      const double *__restrict__ vbg) {
  b_rowsum_warp<S>(m, gd, v, out, xlen, vbg, blockIdx);
}

// The background of an FP32 fluid at ring (j, k) (0 without one).
__device__ __forceinline__ double bg_at(const double *__restrict__ vbg, int ring) {
  return vbg ? vbg[ring] : 0.0;
}

template <typename T, bool ORDERED, typename S = T, int R = 32>
__global__ void __launch_bounds__(256) k_rowsum(Dims m, Geo<double> gd, const S *__restrict__ v,
                                                 double *__restrict__ out, double xlen) {
  b_rowsum<T, ORDERED, S, R>(m, gd, v, out, xlen, blockIdx);
}

// ---------------------------------------------------------------------------
// CFL (cfl.c:135-258) and cfl_b's shear limit (cfl_b.c:14-39).  One CTA per
// active ring; the ring minimum (including its shear limit) is folded into a
// device-wide minimum held as the bit pattern of a positive double.
__device__ __forceinline__ double dmax2(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmax3(double a, double b, double c) {
  return (((a) > (b) ? (a) : (b)) > (c) ? ((a) > (b) ? (a) : (b)) : (c));
}
__device__ __forceinline__ float dmax2(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float dmax3(float a, float b, float c) {
  return (((a) > (b) ? (a) : (b)) > (c) ? ((a) > (b) ? (a) : (b)) : (c));
}

template <typename T>
__device__ __forceinline__ T zsx(const Dims &m, const Geo<T> &g, int i, int j, int k) {
  // zone_size_x (define.h:262-273)
  if (m.sph) return (ld(g.sxi + i) * ld(g.ymed + j) * ld(g.sin_zmed + k));
  return (ld(g.sxi + i) * ld(g.ymed + j));
}
template <typename T>
__device__ __forceinline__ T izsxmed(const Dims &m, const Geo<T> &g, int i, int j, int k) {
  // Inv_zone_size_xmed
  if (m.sph) return (ld(g.invdiffxmed + i) / ld(g.ymed + j) / ld(g.sin_zmed + k));
  return (ld(g.invdiffxmed + i) / ld(g.ymed + j));
}
template <typename T>
__device__ __forceinline__ T zsy(const Geo<T> &g, int j) { return (ld(g.ymin + j + 1) - ld(g.ymin + j)); }
template <typename T>
__device__ __forceinline__ T zsz(const Dims &m, const Geo<T> &g, int j, int k) {
  if (m.sph) return ((ld(g.zmin + k + 1) - ld(g.zmin + k)) * ld(g.ymed + j));
  return (ld(g.zmin + k + 1) - ld(g.zmin + k));
}

// This thread's share of ring (j, k): the minimum of its cells' limits (and,
// for thread 0, the ring's shear limit); non-finite steps or non-positive
// densities raise the flag word dtmin[1].
// Time-step limit of one cell (cfl.c:142-250); `bad` collects the failure
// flags (a non-finite limit or a non-positive density) without a memory
// operation, so the loads of consecutive cells can overlap.
template <typename T, typename S>
__device__ __forceinline__ T cfl_cell(const Dims &m, const Geo<T> &g, const S *__restrict__ rho,
                                      const S *__restrict__ cs, const S *__restrict__ vx,
                                      const S *__restrict__ vy, const S *__restrict__ vz, double vm, T nu,
                                      T alpha, double cfl_num, int i, int j, int k, bool &bad) {
  const long long l = m.l(i, j, k);
  const long long lxp = (i < m.nx - 1) ? l + 1 : l - (m.nx - 1);
  const T vxx = vx[l] - (T)vm, vxxp = vx[lxp] - (T)vm;
  const T c = cs[l];
  T ss2 = c * c;
  T visc;
  if (m.alpha) visc = alpha * c * c * ld(g.visc_j + j);
  else visc = nu;
  if (m.adiab) {   // cs holds the internal energy (cfl.c:164-172)
    const T gm = (T)m.gam;
    ss2 = gm * (gm - (T)1) * c / (T)rho[l];
    if (m.alpha) visc = alpha * gm * (gm - (T)1.0) * c / (T)rho[l] * ld(g.visc_j + j);
  }
  const T ss = sqrt(ss2);
  const T zx = zsx(m, g, i, j, k), zy = zsy(g, j);
  T c1a = ss / zx, c1b = ss / zy, c1c = 0, c4 = 0, c5c = 0, c7c = 0;
  T zz = 1;
  if (m.is3d) { zz = zsz(m, g, j, k); c1c = ss / zz; }
  const T c1 = (T)dmax3(c1a, c1b, c1c);
  const T c2 = (T)(dmax2(fabs(vxx), fabs(vxxp))) / zx;
  const T c3 = (T)(dmax2(fabs(vy[l]), fabs(vy[l + m.pitch]))) / zy;
  if (m.is3d) c4 = (T)(dmax2(fabs(vz[l]), fabs(vz[l + m.stride]))) / zz;
  const T c5a = fabs(vx[lxp] - vx[l]) / zx;
  const T c5b = fabs(vy[l + m.pitch] - vy[l]) / zy;
  if (m.is3d) c5c = fabs(vz[l + m.stride] - vz[l]) / zz;
  const T c5 = (T)dmax3(c5a, c5b, c5c) * (T)4.0 * (T)FB_CVNR;
  const T c7a = (T)1.0 / zx, c7b = (T)1.0 / zy;
  if (m.is3d) c7c = (T)1.0 / zz;
  const T mx7 = (T)dmax3(c7a, c7b, c7c);
  const T c7 = (T)4.0 * visc * (mx7 * mx7);
  const T zero = 0;
  const T dtc = (T)cfl_num / sqrt(c1 * c1 + c2 * c2 + c3 * c3 + c4 * c4 + c5 * c5 + zero * zero + c7 * c7 +
                                  zero * zero + zero * zero + zero * zero);
  bad |= !(dtc == dtc) || !(rho[l] > (T)0);
  return dtc;
}

// The same limit for FP32 2D disks (uniform azimuthal spacing): the zone
// sizes enter as per-ring reciprocals, the maxima of quotients as maxima of
// products, and the square root and division at the end as one reciprocal
// square root -- algebraically cfl.c's expression, rounded differently.
__device__ __forceinline__ float cfl_cell32(const Dims &m, const Geo<float> &g, const float *__restrict__ rho,
                                            const float *__restrict__ cs, const float *__restrict__ vx,
                                            const float *__restrict__ vy, double vm, float nu, float alpha,
                                            float cfl_num, int i, int j, bool &bad) {
  const long long l = m.l(i, j, 0);
  const long long lxp = (i < m.nx - 1) ? l + 1 : l - (m.nx - 1);
  const float izx = ld(g.invdiffxmed + 0) * ld(g.inv_ymed + j), izy = 1.0f / ld(g.sxj + j);
  const float vxl = vx[l], vxp = vx[lxp], vyl = vy[l], vyp = vy[l + m.pitch], c = cs[l];
  const float vmf = (float)vm;
  const float visc = m.alpha ? alpha * c * c * ld(g.visc_j + j) : nu;
  const float ss = fabsf(c);
  const float mx7 = fmaxf(izx, izy);
  const float c1 = ss * mx7;
  const float c2 = fmaxf(fabsf(vxl - vmf), fabsf(vxp - vmf)) * izx;
  const float c3 = fmaxf(fabsf(vyl), fabsf(vyp)) * izy;
  const float c5 = fmaxf(fabsf(vxp - vxl) * izx, fabsf(vyp - vyl) * izy) * (4.0f * (float)FB_CVNR);
  const float c7 = 4.0f * visc * (mx7 * mx7);
  const float dtc = cfl_num * rsqrtf(c1 * c1 + c2 * c2 + c3 * c3 + c5 * c5 + c7 * c7);
  bad |= !(dtc == dtc) || !(rho[l] > 0.0f);
  return dtc;
}

// Shear limit of ring j (cfl_b.c:20-31).
template <typename T>
__device__ __forceinline__ double cfl_shear(const Geo<T> &g, const double *__restrict__ vxmed, double cfl_num,
                                            double mindx, int jk, int j) {
  return cfl_num * mindx / fabs(vxmed[jk] / (double)ld(g.ymed + j) - vxmed[jk + 1] / (double)ld(g.ymed + j + 1));
}

template <typename T, typename S = T>
__device__ __forceinline__ double cfl_ring(Dims m, Geo<T> g, const S *__restrict__ rho, const S *__restrict__ cs,
                                           const S *__restrict__ vx, const S *__restrict__ vy,
                                           const S *__restrict__ vz, const double *__restrict__ vxmed,
                                           const fb_scalars *__restrict__ sc, double cfl_num, double mindx,
                                           unsigned long long *__restrict__ dtmin, int j, int k,
                                           const double *__restrict__ vbg) {
  // FP32 disks hold vx less the ring's background: the mean less it too
  const double vm = vxmed[j + k * m.sy] - bg_at(vbg, j + k * m.sy);
  const T nu = (T)sc->nu, alpha = (T)sc->alpha;
  double mn = 1e20;
  bool bad = false;
  for (int i = threadIdx.x; i < m.nx; i += blockDim.x)
    mn = fmin(mn, (double)cfl_cell<T, S>(m, g, rho, cs, vx, vy, vz, vm, nu, alpha, cfl_num, i, j, k, bad));
  // failure detection: the host or the batch scalar kernel reacts to dtmin[1]
  if (bad) atomicOr(dtmin + 1, 1ull);
  if (threadIdx.x == 0) {
    const double shear = cfl_shear(g, vxmed, cfl_num, mindx, j + k * m.sy, j);
    if (shear < mn) mn = shear;
  }
  return mn;
}

// Block minimum of the threads' shares, folded into the device-wide minimum.
__device__ __forceinline__ void cfl_commit(double mn, unsigned long long *__restrict__ dtmin) {
  for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  __shared__ double wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = mn;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : 1e20;
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0 && v > 0.0) atomicMin(dtmin, (unsigned long long)__double_as_longlong(v));
  }
}

template <typename T, typename S = T>
__device__ __forceinline__ void b_cfl(Dims m, Geo<T> g, const S *__restrict__ rho, const S *__restrict__ cs,
                                             const S *__restrict__ vx, const S *__restrict__ vy,
                                             const S *__restrict__ vz, const double *__restrict__ vxmed,
                                             const fb_scalars *__restrict__ sc, double cfl_num,
                                             double mindx, unsigned long long *__restrict__ dtmin,
                                             const double *__restrict__ vbg, uint3 bid) {
  const int j = FB_NGH + bid.x;
  const int k = m.is3d ? FB_NGH + bid.y : 0;
  cfl_commit(cfl_ring<T, S>(m, g, rho, cs, vx, vy, vz, vxmed, sc, cfl_num, mindx, dtmin, j, k, vbg), dtmin);
}

template <typename T, typename S = T>
__global__ void __launch_bounds__(256) k_cfl(Dims m, Geo<T> g, const S *__restrict__ rho, const S *__restrict__ cs,
                                             const S *__restrict__ vx, const S *__restrict__ vy,
                                             const S *__restrict__ vz, const double *__restrict__ vxmed,
                                             const fb_scalars *__restrict__ sc, double cfl_num,
                                             double mindx, unsigned long long *__restrict__ dtmin,
                                             const double *__restrict__ vbg) {
  b_cfl<T, S>(m, g, rho, cs, vx, vy, vz, vxmed, sc, cfl_num, mindx, dtmin, vbg, blockIdx);
}

// ---------------------------------------------------------------------------
// Potential (potential.c:51-208), FP64, at one cell.
__device__ __forceinline__ double potential_at(const Dims &m, const Geo<double> &gd,
                                               const fb_scalars &sc, int i, int j, int k) {
  double XC, YC, ZC, pot;
  const double ym = ld(gd.ymed + j);
  if (m.sph) {
    XC = ym * ld(gd.cos_xmed + i) * ld(gd.sin_zmed + k);
    YC = ym * ld(gd.sin_xmed + i) * ld(gd.sin_zmed + k);
    ZC = ym * ld(gd.cos_zmed + k);
    pot = -1.0 * 1.0 / ym;
  } else {
    XC = ym * ld(gd.cos_xmed + i);
    YC = ym * ld(gd.sin_xmed + i);
    ZC = ld(gd.zmed + k);
    pot = -1.0 * 1.0 / sqrt(ym * ym + ZC * ZC);
  }
  for (int n = 0; n < sc.nplanets; n++) {
    const double mp = sc.pmass[n] * 1.0;
    const double xp = sc.px[n], yp = sc.py[n], zp = sc.pz[n];
    const double dist = ((XC - xp) * (XC - xp) + (YC - yp) * (YC - yp) + (ZC - zp) * (ZC - zp));
    if (sc.indirect_term) pot += 1.0 * mp * (XC * xp + YC * yp + ZC * zp) / sc.pdist3[n];
    pot += -1.0 * mp / sqrt(dist + sc.psmooth2[n]);
  }
  return pot;
}

// The same potential for FP32-storage disks: the star's term from the per-row
// table, the indirect term with the planets' m / d^3 precomputed (ind[n]),
// the planets' terms with an FP64 reciprocal square root.
__device__ __forceinline__ double potential_fast(const Dims &m, const Geo<double> &gd, const fb_scalars &sc,
                                                 const double *ind, int i, int j, int k) {
  double XC, YC, ZC;
  const double ym = ld(gd.ymed + j);
  if (m.sph) {
    XC = ym * ld(gd.cos_xmed + i) * ld(gd.sin_zmed + k);
    YC = ym * ld(gd.sin_xmed + i) * ld(gd.sin_zmed + k);
    ZC = ym * ld(gd.cos_zmed + k);
  } else {
    XC = ym * ld(gd.cos_xmed + i);
    YC = ym * ld(gd.sin_xmed + i);
    ZC = ld(gd.zmed + k);
  }
  double pot = ld(gd.pot_star + j);
  for (int n = 0; n < sc.nplanets; n++) {
    const double xp = sc.px[n], yp = sc.py[n], zp = sc.pz[n];
    const double dist = ((XC - xp) * (XC - xp) + (YC - yp) * (YC - yp) + (ZC - zp) * (ZC - zp));
    if (sc.indirect_term) pot += ind[n] * (XC * xp + YC * yp + ZC * zp);
    pot -= sc.pmass[n] * rsqrt(dist + sc.psmooth2[n]);
  }
  return pot;
}

}  // namespace fb

namespace fb {

// ---------------------------------------------------------------------------
// Sources, 2D cylindrical (algogas.c:30-120): ComputePressureFieldIso,
// compute_potential's Potential, CorrectVtheta, SubStep1_x/y, visctensor_cyl,
// addviscosity_cyl, SubStep2_a/b, fused over a TX x TY tile of active cells.
// Inputs (rho, cs, v, P, Pot) are staged with a one-cell halo; the stress
// tensor is computed once per point into shared memory.
template <typename T, int TX, int TY, typename S = T>
__device__ __forceinline__ void b_sources_cyl(Dims m, Geo<T> g, Geo<double> gd,
    const S *__restrict__ rho, const S *__restrict__ cs, const S *__restrict__ vx,
    const S *__restrict__ vy, S *__restrict__ vxt, S *__restrict__ vyt,
    const fb_scalars *__restrict__ scp, int dust, int viscous, const double *__restrict__ vbg,
    S *__restrict__ et, uint3 bid) {
  constexpr int W = TX + 2, H = TY + 2;
  __shared__ T s_rho[H][W], s_cs[H][W], s_vx[H][W], s_vy[H][W], s_p[H][W];
  __shared__ double s_pot[H][W];
  // viscous stresses: FP32 arithmetic for FP32 storage (they enter as small
  // increments; velocity differences are taken exactly in T first), T else
  using TV = typename std::conditional<(sizeof(S) < sizeof(T)), float, T>::type;
  __shared__ TV s_txx[H][W], s_tyy[H][W], s_tyx[H][W];
  __shared__ fb_scalars sc;
  __shared__ double s_ind[FB_MAXPLANETS];
  // FP32 storage: the FP64 balance with per-row reciprocals and the fast
  // potential (one division per density-dependent denominator, reused)
  constexpr bool FAST = sizeof(S) < sizeof(T);
  const int i0 = bid.x * TX, j0 = FB_NGH + bid.y * TY;
  const int tid = threadIdx.x + threadIdx.y * TX;
  if (tid == 0) {
    sc = *scp;
    for (int n = 0; n < sc.nplanets; n++) s_ind[n] = sc.pmass[n] / sc.pdist3[n];
  }
  __syncthreads();
  const double dt = sc.dt;
  const T domega = (T)sc.domega, of = (T)sc.omegaframe;
  // stage inputs; vx carries CorrectVtheta (correct_vtheta.c:55-60)
  for (int e = tid; e < H * W; e += TX * TY) {
    const int lj = e / W, li = e - lj * W;
    const int j = j0 - 1 + lj, i = wrapx(i0 - 1 + li, m.nx);
    if (j < m.sy && i0 - 1 + li <= m.nx) {
      const long long l = m.l(i, j, 0);
      const T r = rho[l], c = cs[l];
      s_rho[lj][li] = r;
      s_cs[lj][li] = c;
      // FP32 storage holds vx less the ring's background (added back here)
      if (FAST) s_vx[lj][li] = ((T)vx[l] + (T)bg_at(vbg, j)) - domega * ld(g.ymed + j);
      else s_vx[lj][li] = vx[l] - domega * ld(g.ymed + j);
      s_vy[lj][li] = vy[l];
      // ComputePressureFieldIso, or ComputePressureFieldAd (CompPresAd.c:54)
      // where cs holds the internal energy
      s_p[lj][li] = m.adiab ? ((T)m.gam - (T)1.0) * c : r * c * c;
      s_pot[lj][li] = FAST ? potential_fast(m, gd, sc, s_ind, i, j, 0) : potential_at(m, gd, sc, i, j, 0);
    }
  }
  __syncthreads();
  if (viscous) {
    const TV nu = (TV)sc.nu, alpha = (TV)sc.alpha;
    for (int e = tid; e < H * W; e += TX * TY) {
      const int lj = e / W, li = e - lj * W;
      const int j = j0 - 1 + lj, i = wrapx(i0 - 1 + li, m.nx);
      if (j >= m.sy - 1 || i0 - 1 + li > m.nx) continue;
      // tau_xx, tau_yy at (li in [0,TX], lj in [0,TY]); tau_yx at (li,lj >= 1)
      TV visc = nu, viscm = nu;
      if (m.alpha && lj >= 1 && li >= 1) {
        const TV e0 = (TV)s_cs[lj][li], ex = (TV)s_cs[lj][li - 1], ey = (TV)s_cs[lj - 1][li],
                 exy = (TV)s_cs[lj - 1][li - 1];
        if (m.adiab)   // visctensor_cyl.c:148 (cs = internal energy)
          viscm = alpha * (TV)m.gam * ((TV)m.gam - (TV)1.0) * (e0 + ex + ey + exy) /
                  ((TV)s_rho[lj][li] + (TV)s_rho[lj][li - 1] + (TV)s_rho[lj - 1][li] + (TV)s_rho[lj - 1][li - 1]) *
                  (TV)ld(g.viscm_j + j);
        else
          viscm = alpha * (TV)0.0625 * (e0 + ex + ey + exy) * (e0 + ex + ey + exy) * (TV)ld(g.viscm_j + j);
      }
      if (m.alpha) {
        if (m.adiab)   // visctensor_cyl.c:147
          visc = alpha * (TV)m.gam * ((TV)m.gam - (TV)1.0) * (TV)s_cs[lj][li] / (TV)s_rho[lj][li] * (TV)ld(g.visc_j + j);
        else
          visc = alpha * (TV)s_cs[lj][li] * (TV)s_cs[lj][li] * (TV)ld(g.visc_j + j);
      }
      if (li <= TX && lj <= TY) {
        const TV r = (TV)s_rho[lj][li];
        // FP32 storage: uniform azimuthal spacing, the x factors of cell 0
        const int ix = FAST ? 0 : i;
        const TV sxi = (TV)ld(g.sxi + ix), syk = (TV)ld(g.syk + 0), sxk = (TV)ld(g.sxk + 0);
        TV div_v = 0.0;
        div_v += (TV)(s_vx[lj][li + 1] - s_vx[lj][li]) * (TV)ld(g.sxj + j) * sxk;
        div_v += ((TV)s_vy[lj + 1][li] * (TV)ld(g.syj + j + 1) * syk * sxi - (TV)s_vy[lj][li] * (TV)ld(g.syj + j) * syk * sxi);
        div_v *= (TV)(2.0 / 3.0) * (TV)ld(g.invvj + j) / (syk * sxi);
        TV txx = visc * r * ((TV)2.0 * (TV)(s_vx[lj][li + 1] - s_vx[lj][li]) / (TV)zsx(m, g, ix, j, 0) - div_v);
        txx += visc * r * (TV)(s_vy[lj + 1][li] + s_vy[lj][li]) / (TV)ld(g.ymed + j);
        s_txx[lj][li] = txx;
        s_tyy[lj][li] = visc * r * ((TV)2.0 * (TV)(s_vy[lj + 1][li] - s_vy[lj][li]) /
                                    (TV)(ld(g.ymin + j + 1) - ld(g.ymin + j)) - div_v);
      }
      if (li >= 1 && lj >= 1) {
        s_tyx[lj][li] = viscm * (TV)0.25 *
                        (TV)(s_rho[lj][li] + s_rho[lj][li - 1] + s_rho[lj - 1][li] + s_rho[lj - 1][li - 1]) *
                        ((TV)(s_vy[lj][li] - s_vy[lj][li - 1]) * (TV)ld(g.invdiffxmed + (FAST ? 0 : i)) / (TV)ld(g.ymin + j) +
                         (TV)(s_vx[lj][li] - s_vx[lj - 1][li]) / (TV)(ld(g.ymed + j) - ld(g.ymed + j - 1)) -
                         (TV)0.5 * (TV)(s_vx[lj][li] + s_vx[lj - 1][li]) / (TV)ld(g.ymin + j));
      }
    }
    __syncthreads();
  }
  const int li = threadIdx.x + 1, lj = threadIdx.y + 1;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  // adiabatic disks also need V_temp of row Ny+3, the outer edge face, which
  // SubStep3 reads before the ghost fill (substep1_y.c: j < Ny+2*NGHY-1)
  if (i >= m.nx || j > m.ny + FB_NGH - 1 + m.adiab) return;
  const int im = wrapx(i - 1, m.nx);
  // FP32 storage: uniform azimuthal spacing, the x factors of cell 0
  const int ix = FAST ? 0 : i, ixm = FAST ? 0 : im;
  const long long l = m.l(i, j, 0);
  const T r = s_rho[lj][li], rxm = s_rho[lj][li - 1], rym = s_rho[lj - 1][li];
  const T izx = FAST ? ld(g.invdiffxmed + ix) * ld(g.inv_ymed + j) : izsxmed(m, g, i, j, 0);
  // SubStep1_x (substep1_x.c:107-117)
  const T dxmed = (T)0.5 * (ld(g.sxi + ix) + ld(g.sxi + ixm));
  T idenx = 0, ideny = 0;
  T dtorx;
  if (FAST) {
    idenx = (T)1.0 / (r * ld(g.sxi + ix) + rxm * ld(g.sxi + ixm));
    dtorx = (T)2. * (T)dt * idenx * dxmed;
  } else {
    dtorx = (T)2. * (T)dt / (r * ld(g.sxi + i) + rxm * ld(g.sxi + im)) * dxmed;
  }
  T ax = s_vx[lj][li];
  if (!dust) ax -= dtorx * (s_p[lj][li] - s_p[lj][li - 1]) * izx;
  ax -= (T)((s_pot[lj][li] - s_pot[lj][li - 1]) * dt) * izx;
  // SubStep1_y (substep1_y.c:146-192, cylindrical)
  const T ym = ld(g.ymed + j), ymm = ld(g.ymed + j - 1), yi = ld(g.ymin + j), yip = ld(g.ymin + j + 1),
          yim = ld(g.ymin + j - 1);
  T dtory;
  if (FAST) {
    ideny = (T)1.0 / (r * (yip - yi) + rym * (yi - yim));
    dtory = (T)2.0 * (T)dt * ideny * (ym - ymm);
  } else {
    dtory = (T)2.0 * (T)dt / (r * (yip - yi) + rym * (yi - yim)) * (ym - ymm);
  }
  T ay = s_vy[lj][li];
  if (!dust) {
    if (FAST) ay -= dtory * (s_p[lj][li] - s_p[lj - 1][li]) * ld(g.inv_dymed + j);
    else ay -= dtory * (s_p[lj][li] - s_p[lj - 1][li]) / (ym - ymm);
  }
  T vphi = (T)0.25 * (s_vx[lj][li] + s_vx[lj][li + 1] + s_vx[lj - 1][li] + s_vx[lj - 1][li + 1]);
  vphi += yi * of;
  if (FAST) {
    ay += vphi * vphi * ld(g.inv_ymin + j) * (T)dt;
    ay -= (T)((s_pot[lj][li] - s_pot[lj - 1][li]) * dt) * ld(g.inv_dymed + j);
  } else {
    ay += vphi * vphi / yi * (T)dt;
    ay -= (T)((s_pot[lj][li] - s_pot[lj - 1][li]) * dt / (double)(ym - ymm));
  }
  if (viscous) {
    // addviscosity_cyl (addviscosity_cyl.c:106-124)
    const TV vr = (TV)r, vrxm = (TV)rxm, vrym = (TV)rym, vizx = (TV)izx, vdt = (TV)dt;
    const TV vym = (TV)ym, vymm = (TV)ymm, vyi = (TV)yi, vyip = (TV)yip;
    ax += (T)((TV)2.0 * (s_txx[lj][li] - s_txx[lj][li - 1]) * vizx / ((vr + vrxm)) * vdt);
    ax += (T)((TV)2.0 * (vyip * vyip * s_tyx[lj + 1][li] - vyi * vyi * s_tyx[lj][li]) /
              ((vyip - vyi) * vym * vym * (vrxm + vr)) * vdt);
    ay += (T)((TV)2.0 * (vym * s_tyy[lj][li] - vymm * s_tyy[lj - 1][li]) / ((vym - vymm) * (vr + vrym) * vyi) * vdt);
    ay += (T)((TV)2.0 * (s_tyx[lj][li + 1] - s_tyx[lj][li]) /
              ((TV)(FAST ? ld(g.sxi + ix) : ld(g.xmin + i + 1) - ld(g.xmin + i)) * vyi * (vr + vrym)) * vdt);
    ay -= (T)((s_txx[lj][li] + s_txx[lj - 1][li]) / (vyi * (vr + vrym)) * vdt);
  }
  // SubStep2_a / SubStep2_b (substep2_a.c:107-129, substep2_b.c:150-175)
  const T c2 = (T)FB_CVNR;
  T dv = s_vx[lj][li + 1] - s_vx[lj][li];
  const T qx = dv < (T)0.0 ? c2 * c2 * r * dv * dv : (T)0.0;
  dv = s_vx[lj][li] - s_vx[lj][li - 1];
  const T qxm = dv < (T)0.0 ? c2 * c2 * rxm * dv * dv : (T)0.0;
  dv = s_vy[lj + 1][li] - s_vy[lj][li];
  const T qy = dv < (T)0.0 ? c2 * c2 * r * dv * dv : (T)0.0;
  dv = s_vy[lj][li] - s_vy[lj - 1][li];
  const T qym = dv < (T)0.0 ? c2 * c2 * rym * dv * dv : (T)0.0;
  if (FAST) {
    ax += -(T)2.0 * (T)dt * dxmed * (qx - qxm) * idenx * izx;
    ay += -(T)2.0 * (qy - qym) * ideny * (T)dt;
  } else {
    ax += -(T)2.0 * (T)dt * dxmed * (qx - qxm) / (r * ld(g.sxi + i) + rxm * ld(g.sxi + im)) * izx;
    ay += -(T)2.0 * (qy - qym) / (r * (yip - yi) + rym * (yi - yim)) * (T)dt;
  }
  vxt[l] = FAST ? ax - (T)bg_at(vbg, j) : ax;
  vyt[l] = ay;
  if (m.adiab && !dust && et) {
    // SubStep2_b (substep2_b.c:161-178): the artificial viscosity's heating,
    // with the velocities the step started from (after CorrectVtheta)
    T e = s_cs[lj][li];
    e += -(T)dt * (qx * (s_vx[lj][li + 1] - s_vx[lj][li]) / zsx(m, g, i, j, 0));
    e += -(T)dt * (qy * (s_vy[lj + 1][li] - s_vy[lj][li]) / (yip - yi));
    et[l] = e;
  }
}
// resident CTAs per SM of the FP64 3D source stage (96 registers; the
// shared-memory tiles allow 5): 1.36 -> 1.30 ms at 512x256x48
#ifndef FB_SPH64_MINB
#define FB_SPH64_MINB 5
#endif

template <typename T, int TX, int TY, typename S = T>
__global__ void __launch_bounds__(TX *TY) k_sources_cyl(Dims m, Geo<T> g, Geo<double> gd,
    const S *__restrict__ rho, const S *__restrict__ cs, const S *__restrict__ vx,
    const S *__restrict__ vy, S *__restrict__ vxt, S *__restrict__ vyt,
    const fb_scalars *__restrict__ scp, int dust, int viscous, const double *__restrict__ vbg,
    S *__restrict__ et) {
  b_sources_cyl<T, TX, TY, S>(m, g, gd, rho, cs, vx, vy, vxt, vyt, scp, dust, viscous, vbg, et, blockIdx);
}

}  // namespace fb

namespace fb {

// ---------------------------------------------------------------------------
// Dust diffusion (DustDiffusion_Main, dust_diffusion_main.c:3-28), 2D
// cylindrical: each dust fluid's density diffuses down the gradient of its
// concentration c = rho_d / (rho_d + rho_g) with the gas's diffusivity --
// Nu (VISCOSITY) or Alpha cs^2 / Omega_K (ALPHAVISCOSITY, isothermal), at cell
// centres and at the radial faces (dust_diffusion_coefficients.c:94-120) --
// rho_d += dt div(D grad c) in the reference's operation order
// (dust_diffusion_core.c:132-185), into a buffer, for the active rows.
template <typename T, typename S>
__global__ void __launch_bounds__(128) k_dust_diffusion(Dims m, Geo<T> g, const S *__restrict__ rd,
                                                        const S *__restrict__ rg, const S *__restrict__ csg,
                                                        S *__restrict__ out, const fb_scalars *__restrict__ scp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = FB_NGH + blockIdx.y;
  if (i >= m.nx) return;
  const T dt = (T)scp->dt, nu = (T)scp->nu, alpha = (T)scp->alpha;
  const long long l = m.l(i, j, 0);
  const int ixp = i < m.nx - 1 ? i + 1 : 0;
  const long long lxp = (i < m.nx - 1) ? l + 1 : l - (m.nx - 1), lxm = i > 0 ? l - 1 : l + (m.nx - 1);
  const long long lyp = l + m.pitch, lym = l - m.pitch;
  // Sdiffyczc at a cell of row jj, Sdiffyfzc at the lower face of row jj
  auto sdc = [&](long long ll, int jj) -> T {
    if (!m.alpha) return nu;
    const T ss2 = (T)csg[ll] * (T)csg[ll];
    const T r3 = ld(g.ymed + jj) * ld(g.ymed + jj) * ld(g.ymed + jj);
    return alpha * ss2 / sqrt((T)1.0 * (T)1.0 / r3);
  };
  auto sdf = [&](long long ll, int jj) -> T {
    if (!m.alpha) return nu;
    T ssf2;
    if (jj == 0) ssf2 = (T)csg[ll] * (T)csg[ll];
    else ssf2 = (T)0.5 * ((T)csg[ll] + (T)csg[ll - m.pitch]) * (T)0.5 * ((T)csg[ll] + (T)csg[ll - m.pitch]);
    const T r3 = ld(g.ymin + jj) * ld(g.ymin + jj) * ld(g.ymin + jj);
    return alpha * ssf2 / sqrt((T)1.0 * (T)1.0 / r3);
  };
  const T d0 = rd[l], g0 = rg[l];
  T update = 0.0;
  const T c = d0 / (d0 + g0);
  const T dxmin = ld(g.xmin + i + 1) - ld(g.xmin + i);
  const T dxmedp = (T)1.0 / ld(g.invdiffxmed + ixp), dxmedm = (T)1.0 / ld(g.invdiffxmed + i);
  const T dxp = rd[lxp], gxp = rg[lxp], dxm = rd[lxm], gxm = rg[lxm];
  const T d1 = (T)0.25 * (d0 + g0 + dxp + gxp) * (sdc(lxp, j) + sdc(l, j));
  const T d2 = (T)0.25 * (d0 + g0 + dxm + gxm) * (sdc(lxm, j) + sdc(l, j));
  const T cxp = dxp / (dxp + gxp), cxm = dxm / (dxm + gxm);
  const T ym = ld(g.ymed + j), ymp = ld(g.ymed + j + 1), ymm = ld(g.ymed + j - 1);
  const T yi = ld(g.ymin + j), yip = ld(g.ymin + j + 1);
  update += (T)1.0 / ym / ym / (dxmin) * (d1 * (cxp - c) / (dxmedp) - (d2 * (c - cxm)) / (dxmedm));
  const T dyp = rd[lyp], gyp = rg[lyp], dym = rd[lym], gym = rg[lym];
  const T d3 = (T)0.5 * (d0 + g0 + dyp + gyp) * sdf(lyp, j + 1);
  const T d4 = (T)0.5 * (d0 + g0 + dym + gym) * sdf(l, j);
  const T cyp = dyp / (dyp + gyp), cym = dym / (dym + gym);
  update += (T)1.0 / ym / (yip - yi) * (yip * d3 * (cyp - c) / (ymp - ym) - (yi * d4 * (c - cym)) / (ym - ymm));
  out[l] = d0 + dt * update;
}

// copy_field(Density, Pressure) of DustDiffusion_Main for the active rows
template <typename S>
__global__ void __launch_bounds__(128) k_copy_rows(Dims m, const S *__restrict__ src, S *__restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nx) return;
  const long long l = m.l(i, FB_NGH + blockIdx.y, 0);
  dst[l] = src[l];
}

// FillGhosts(DENS): the density's radial ghosts only (KEPLERIAN2DDENS)
template <typename T, typename S>
__global__ void k_bnd_rho_y(Dims m, Geo<T> g, const double *__restrict__ tab, S *__restrict__ rho) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y % 3, s = blockIdx.y / 3;
  if (i >= m.nx) return;
  const int jgh = s == 0 ? jj : m.ny + FB_NGH + jj, jact = s == 0 ? 2 * FB_NGH - jj - 1 : m.ny + FB_NGH - 1 - jj;
  rho[m.l(i, jgh, 0)] = rho[m.l(i, jact, 0)] * (T)tab[s * 3 + jj];
  (void)g;
}

// ---------------------------------------------------------------------------
// SubStep3 (substep3.c:79-118), adiabatic disks: the compression work of the
// source step, e *= (1 - theta) / (1 + theta) with theta = dt (GAMMA - 1)
// div(V_temp) / (2 Vol), on the energy after SubStep2_b (et) into the Energy
// field, for the active rows (the ghosts are refilled after it).  The
// divergence uses the macros' unparenthesised products (SurfX, SurfY,
// InvVol: define.h:228-235) in the reference's order.
template <typename T>
__global__ void __launch_bounds__(128) k_substep3(Dims m, Geo<T> g, const T *__restrict__ et,
                                                  const T *__restrict__ vxt, const T *__restrict__ vyt,
                                                  T *__restrict__ e, const fb_scalars *__restrict__ scp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = FB_NGH + blockIdx.y, k = 0;
  if (i >= m.nx) return;
  const T dt = (T)scp->dt;
  const long long l = m.l(i, j, k);
  const long long lxp = (i < m.nx - 1) ? l + 1 : l - (m.nx - 1);
  T div_v = 0.0;
  div_v += (vxt[lxp] - vxt[l]) * ld(g.sxj + j) * ld(g.sxk + k);
  div_v += (vyt[l + m.pitch] * ld(g.syj + j + 1) * ld(g.syk + k) * ld(g.sxi + i) -
            vyt[l] * ld(g.syj + j) * ld(g.syk + k) * ld(g.sxi + i));
  const T term = (T)0.5 * dt * ((T)m.gam - (T)1.) * div_v * ld(g.invvj + j) / (ld(g.syk + k) * ld(g.sxi + i));
  e[l] = et[l] * (((T)1.0 - term) / ((T)1.0 + term));
}

// ---------------------------------------------------------------------------
// Ghost cells from the setups' boundary templates (std/boundaries.txt with
// setups/fargo/fargo.bound in 2D and setups/p3disof/p3disof.bound in 3D;
// index rules of scripts/boundparser.py:360-398).  All libm factors of the
// templates are tabulated on the host.  Table layout (doubles):
//   [0,6)  rho power factor per (side, ghost row)   [6,12) sqrt factor
//   [12,18) 3D radial v_phi correction factor        [18,18+6*sz) 3D exp factor
//   then 6*sy colatitude density factors, then 6 colatitude v_phi factors.
struct BndTab {
  const double *t;
  int sy, sz;
  __device__ double rhof(int s, int jj) const { return t[s * 3 + jj]; }
  __device__ double sqf(int s, int jj) const { return t[6 + s * 3 + jj]; }
  __device__ double cf(int s, int jj) const { return t[12 + s * 3 + jj]; }
  __device__ double rhoe(int s, int jj, int k) const { return t[18 + (s * 3 + jj) * sz + k]; }
  __device__ double zrho(int s, int kk, int j) const { return t[18 + 6 * sz + (s * 3 + kk) * sy + j]; }
  __device__ double zw(int s, int kk) const { return t[18 + 6 * sz + 6 * sy + s * 3 + kk]; }
};

// Radial sides: one thread per (i, ghost row jj, side s, layer k).
template <typename T, typename S = T>
__device__ __forceinline__ void b_bnd_y(Dims m, Geo<T> g, BndTab tb, S *__restrict__ rho, S *__restrict__ vx,
                        S *__restrict__ vy, S *__restrict__ vz, const fb_scalars *__restrict__ scp,
                        int do_rho, const double *__restrict__ vbg, uint3 bid, S *__restrict__ energy = nullptr) {
  const int i = bid.x * blockDim.x + threadIdx.x;
  const int jj = bid.y % 3, s = bid.y / 3, k = bid.z;
  if (i >= m.nx) return;
  // a slab's inner edge takes its ghosts from the neighbouring slab
  if ((s == 0 && !m.bclo) || (s == 1 && !m.bchi)) return;
  const T of = (T)scp->omegaframe;
  const int nghy = FB_NGH, ny = m.ny;
  int jgh, jact, jlacts, jnull;
  if (s == 0) { jgh = jj; jact = 2 * nghy - jj - 1; jlacts = 2 * nghy - jj; jnull = nghy; }
  else { jgh = ny + nghy + jj; jact = ny + nghy - 1 - jj; jlacts = jact; jnull = ny + nghy; }
  const long long lgh = m.l(i, jgh, k), lact = m.l(i, jact, k);
  const T yact = ld(g.ymed + jact), ygh = ld(g.ymed + jgh);
  // FP32 storage: vx less the ring backgrounds of the active and ghost rows
  constexpr bool BG = sizeof(S) < sizeof(T);
  const T vact = BG ? (T)vx[lact] + (T)bg_at(vbg, jact + k * m.sy) : (T)vx[lact];
  const T bgh = BG ? (T)bg_at(vbg, jgh + k * m.sy) : (T)0;
  if (!m.is3d) {
    if (do_rho) rho[lgh] = rho[lact] * (T)tb.rhof(s, jj);
    if (BG) vx[lgh] = (vact + yact * of) * (T)tb.sqf(s, jj) - ygh * of - bgh;
    else vx[lgh] = (vx[lact] + yact * of) * (T)tb.sqf(s, jj) - ygh * of;
  } else {
    const T sz = ld(g.sin_zmed + k);
    if (do_rho) rho[lgh] = rho[lact] * (T)tb.rhof(s, jj) * (T)tb.rhoe(s, jj, k);
    if (BG) vx[lgh] = (vact + of * yact * sz) * (T)tb.sqf(s, jj) * (T)tb.cf(s, jj) - ygh * of * sz - bgh;
    else vx[lgh] = (vx[lact] + of * yact * sz) * (T)tb.sqf(s, jj) * (T)tb.cf(s, jj) - ygh * of * sz;
  }
  // Energy of adiabatic disks: SYMMETRIC (the ghost mirrors the active cell)
  if (energy) energy[lgh] = energy[lact];
  // Vy: ANTISYMMETRIC, staggered in y (|-a|0|a|)
  if (s == 0) vy[lgh] = -vy[m.l(i, jlacts, k)];
  else if (jj < nghy - 1) vy[m.l(i, ny + nghy + 1 + jj, k)] = -vy[m.l(i, jlacts, k)];
  vy[m.l(i, jnull, k)] = 0;
  // Vz: SYMMETRIC, centred in y
  if (m.is3d) vz[lgh] = vz[lact];
}
template <typename T, typename S = T>
__global__ void k_bnd_y(Dims m, Geo<T> g, BndTab tb, S *__restrict__ rho, S *__restrict__ vx,
                        S *__restrict__ vy, S *__restrict__ vz, const fb_scalars *__restrict__ scp,
                        int do_rho, const double *__restrict__ vbg, S *__restrict__ energy) {
  b_bnd_y<T, S>(m, g, tb, rho, vx, vy, vz, scp, do_rho, vbg, blockIdx, energy);
}

// Colatitude sides (3D): one thread per (i, j, ghost layer kk, side s).
template <typename T, typename S = T>
__device__ __forceinline__ void b_bnd_z(Dims m, Geo<T> g, BndTab tb, S *__restrict__ rho, S *__restrict__ vx,
                        S *__restrict__ vy, S *__restrict__ vz, const fb_scalars *__restrict__ scp,
                        int do_rho, const double *__restrict__ vbg, uint3 bid) {
  const int i = bid.x * blockDim.x + threadIdx.x;
  const int j = bid.y, kk = bid.z % 3, s = bid.z / 3;
  if (i >= m.nx) return;
  const T of = (T)scp->omegaframe;
  const int nghz = FB_NGH, nz = m.nz;
  int kgh, kact, klacts, knull;
  if (s == 0) { kgh = kk; kact = 2 * nghz - kk - 1; klacts = 2 * nghz - kk; knull = nghz; }
  else { kgh = nz + nghz + kk; kact = nz + nghz - 1 - kk; klacts = kact; knull = nz + nghz; }
  const long long lgh = m.l(i, j, kgh), lact = m.l(i, j, kact);
  const T ym = ld(g.ymed + j);
  if (do_rho) rho[lgh] = rho[lact] * (T)tb.zrho(s, kk, j);
  if (sizeof(S) < sizeof(T)) {  // FP32 storage: vx less the ring backgrounds
    const T vact = (T)vx[lact] + (T)bg_at(vbg, j + kact * m.sy);
    vx[lgh] = (vact + of * ym * ld(g.sin_zmed + kact)) * (T)tb.zw(s, kk) - ym * of * ld(g.sin_zmed + kgh) -
              (T)bg_at(vbg, j + kgh * m.sy);
  } else {
    vx[lgh] = (vx[lact] + of * ym * ld(g.sin_zmed + kact)) * (T)tb.zw(s, kk) - ym * of * ld(g.sin_zmed + kgh);
  }
  vy[lgh] = vy[lact];
  if (s == 0) vz[lgh] = -vz[m.l(i, j, klacts)];
  else if (kk < nghz - 1) vz[m.l(i, j, nz + nghz + 1 + kk)] = -vz[m.l(i, j, klacts)];
  vz[m.l(i, j, knull)] = 0;
}
template <typename T, typename S = T>
__global__ void k_bnd_z(Dims m, Geo<T> g, BndTab tb, S *__restrict__ rho, S *__restrict__ vx,
                        S *__restrict__ vy, S *__restrict__ vz, const fb_scalars *__restrict__ scp,
                        int do_rho, const double *__restrict__ vbg) {
  b_bnd_z<T, S>(m, g, tb, rho, vx, vy, vz, scp, do_rho, vbg, blockIdx);
}

// ---------------------------------------------------------------------------
// Column sweeps (Y and Z): TransportY/TransportZ (transport.c:24-46) for the
// density and every momentum, one thread per column marching over a segment
// of NS rows (layers) with its input window in registers.
//   VanLeer*_a (vanleer_y_a.c:62-70), VanLeer*_b (vanleer_y_b.c:62-68),
//   DivideByRho (divrho.c:52), Update* / UpdateDensity* (update_y.c:68-72).
// DIR 0 = Y (radius), 1 = Z (colatitude).
template <typename T, int DIR>
struct ColGeo {
  Dims m; Geo<T> g; int i, j, k;
  __device__ T zone(int c) const {  // zone size at cell c along DIR
    if (DIR == 0) return zsy(g, c);
    return zsz(m, g, j, c);
  }
  __device__ T surf(T v, int c) const {  // v * Surf(c) with the reference's association
    if (DIR == 0) return v * ld(g.syj + c) * ld(g.syk + k) * ld(g.sxi + i);
    return v * ld(g.szj + j) * ld(g.szk + c) * ld(g.sxi + i);
  }
  __device__ T finish(T flux, T dt, int c) const {  // flux * dt * InvVol(i,j,k)
    if (DIR == 0) return flux * dt * ld(g.invvj + c) / (ld(g.syk + k) * ld(g.sxi + i));
    return flux * dt * ld(g.invvj + j) / (ld(g.syk + c) * ld(g.sxi + i));
  }
};

template <typename T, int DIR, int NS, bool OFF = false>
__device__ __forceinline__ void col_sweep_q(const ColGeo<T, DIR> &cg, int c0, const T *a, const T *vel,
                                            const T *off, T dt, T *qs) {
  // a: NS+4 cell values (c0-2 .. c0+NS+1); vel: NS+1 faces (c0 .. c0+NS).
  // OFF: a holds the quantity less a cell-dependent offset whose neighbour
  // differences are off[w] = offset(a[w+1]) - offset(a[w]); the limiter sees
  // the differences of the full quantity and qs[] comes back less the offset
  // of its upwind cell.
  T slope[NS + 2];
#pragma unroll
  for (int s = 0; s < NS + 2; s++) {
    const int c = c0 - 1 + s;
    T dqm = a[s + 1] - a[s], dqp = a[s + 2] - a[s + 1];
    if (OFF) { dqm += off[s]; dqp += off[s + 1]; }
    dqm /= cg.zone(c);
    dqp /= cg.zone(c + 1);
    if (dqp * dqm <= 0) slope[s] = 0;
    else slope[s] = (T)2. * dqp * dqm / (dqm + dqp);
  }
#pragma unroll
  for (int f = 0; f < NS + 1; f++) {
    const int c = c0 + f;
    const T v = vel[f];
    if (v > (T)0.)
      qs[f] = a[f + 1] + (T)0.5 * (cg.zone(c - 1) - v * dt) * slope[f];
    else
      qs[f] = a[f + 2] - (T)0.5 * (cg.zone(c) + v * dt) * slope[f + 1];
  }
  (void)off;
}

// Quantity sources: 2D Y sweep and 3D Z sweep build the momenta from rho and
// V_temp (momenta_x.c:76-85, momenta_y.c:65-66, momenta_z.c:61-66); the 3D
// Y sweep reads them from the Z sweep's output buffers.
template <typename T, typename S = T>
struct QSrc {
  const S *rho, *vxt, *vyt, *vzt;
  const S *q[6];   // when from buffers: mpx, mmx, mpy, mmy, mpz, mmz
  int from_v;
  T of;
  // FP32 storage: neighbour differences along the sweep of the background's
  // vbg * R per ring (fb_fluid_dev dlb_y / dlb_z), or null
  const T *dl;
};

// REL: the azimuthal momenta relative to the frame's rotation (the
// OMEGAFRAME * R term of momenta_x.c:77-78 left out).
template <typename T, typename S, bool REL = false>
__device__ __forceinline__ T momentum(const Dims &m, const Geo<T> &g, const QSrc<T, S> &src, int q, int i, int j,
                                      int k, long long l, T r) {
  if (!src.from_v) return src.q[q][l];
  switch (q) {
    case 0: case 1: {  // Mpx, Mmx
      const long long lx = (q == 0) ? ((i < m.nx - 1) ? l + 1 : l - (m.nx - 1)) : l;
      if (!m.sph) {
        const T y = ld(g.ymed + j);
        if (REL) return src.vxt[lx] * y * r;
        return (src.vxt[lx] + y * src.of) * y * r;
      }
      const T rc = ld(g.ymed + j) * ld(g.sin_zmed + k);
      if (REL) return src.vxt[lx] * rc * r;
      return (src.vxt[lx] + rc * src.of) * rc * r;
    }
    case 2: return src.vyt[l + m.pitch] * r;  // Mpy
    case 3: return src.vyt[l] * r;            // Mmy
    case 4: {                                 // Mpz
      T v = src.vzt[l + m.stride] * r;
      if (m.sph) v *= ld(g.ymed + j);
      return v;
    }
    default: {                                // Mmz
      T v = src.vzt[l] * r;
      if (m.sph) v *= ld(g.ymed + j);
      return v;
    }
  }
}

// One launch covers cells [clo, chi] along DIR for every column in range.
// grid.x: columns along x (blockDim.x threads), grid.y: the other transverse
// index (row j for Z sweeps, layer k for Y sweeps), grid.z: segments along DIR.
template <typename T, int DIR, int NS, typename S = T>
__device__ __forceinline__ void b_sweep_col(Dims m, Geo<T> g, QSrc<T, S> src, int nq, int clo, int chi,
                                                   int t2lo, S *__restrict__ rho_out, S *q_out0, S *q_out1,
                                                   S *q_out2, S *q_out3, S *q_out4, S *q_out5,
                                                   const fb_scalars *__restrict__ scp, uint3 bid,
                                                   const S *__restrict__ e_in = nullptr, S *__restrict__ e_out = nullptr) {
  const int i = bid.x * blockDim.x + threadIdx.x;
  if (i >= m.nx) return;
  const int t2 = t2lo + bid.y;
  const int c0 = clo + bid.z * NS;
  if (c0 > chi) return;
  const int j = (DIR == 0) ? 0 : t2, k = (DIR == 0) ? t2 : 0;
  ColGeo<T, DIR> cg{m, g, i, j, k};
  const T dt = (T)scp->dt;
  src.of = (T)scp->omegaframe;  // momenta_x.c:77-78 read the current OMEGAFRAME
  auto cidx = [&](int c) -> long long { return (DIR == 0) ? m.l(i, c, k) : m.l(i, j, c); };
  // cells beyond chi + 2 (faces beyond chi + 1) never reach an output: clamp
  const int cmax = chi + 2;
  T r[NS + 4], vel[NS + 1], rs[NS + 1], a[NS + 4], qs[NS + 1];
  const S *vface = (DIR == 0) ? src.vyt : src.vzt;
#pragma unroll
  for (int w = 0; w < NS + 4; w++) r[w] = src.rho[cidx(min(c0 - 2 + w, cmax))];
#pragma unroll
  for (int f = 0; f < NS + 1; f++) vel[f] = vface[cidx(min(c0 + f, cmax - 1))];
  // density interface values (VanLeer*_a/_b on Density -> DensStar)
  col_sweep_q<T, DIR, NS>(cg, c0, r, vel, nullptr, dt, rs);
  // With FP32 storage the azimuthal momenta live in the buffers relative to
  // the frame's rotation, Mrel = M - OMEGAFRAME * R^2 * rho (R the
  // cylindrical radius), so that the stored numbers and their rounding are of
  // the size of the residual velocity.  The sweep then transports Mrel
  // directly: the limiter sees the differences of the full specific momentum
  // (a_rel differences plus OMEGAFRAME times the tabulated R^2 differences),
  // and a face flux carries OMEGAFRAME (R^2_upwind - R^2_cell) times the
  // density flux, which is M's flux less OMEGAFRAME R^2_cell times rho's.
  // No large momentum is formed and then cancelled, so the update loses no
  // digits in FP32 arithmetic.
  constexpr bool REL = sizeof(S) == 4;
  T rnew[NS];
#pragma unroll
  for (int u = 0; u < NS; u++) {
    const int c = c0 + u;
    const T flux = cg.surf(vel[u] * rs[u], c) - cg.surf(vel[u + 1] * rs[u + 1], c + 1);
    rnew[u] = r[u + 2] + cg.finish(flux, dt, c);
  }
  // OMEGAFRAME * (R^2(c) - R^2(c-1)), plus (vbg R)(c) - (vbg R)(c-1) where
  // the stored azimuthal velocities are relative to a ring background: the
  // difference of the offset l(c) = R (OMEGAFRAME R + vbg) that the relative
  // momenta leave out
  auto dlb = [&](int c) -> T {
    if (!src.dl) return (T)0;
    return ld(src.dl + ((DIR == 0) ? c + k * m.sy : j + c * m.sy));
  };
  auto dr2 = [&](int c) -> T {
    if (!m.sph) return src.of * ld(g.dr2_j + c) + dlb(c);
    if (DIR == 0) return src.of * (ld(g.dr2_j + c) * ld(g.s2_k + k)) + dlb(c);
    return src.of * (ld(g.r2_j + j) * ld(g.ds2_k + c)) + dlb(c);
  };
  S *qo[6] = {q_out0, q_out1, q_out2, q_out3, q_out4, q_out5};
#pragma unroll
  for (int q = 0; q < 6; q++) {
    if (q >= nq) break;
    T qv[NS + 4];
#pragma unroll
    for (int w = 0; w < NS + 4; w++) {
      const int c = min(c0 - 2 + w, cmax);
      const int jj = (DIR == 0) ? c : j, kk = (DIR == 0) ? k : c;
      qv[w] = momentum<T, S, REL>(m, g, src, q, i, jj, kk, cidx(c), r[w]);
      a[w] = qv[w] / r[w];
    }
    if (REL && q < 2) {
      T off[NS + 3];
#pragma unroll
      for (int w = 0; w < NS + 3; w++) {
        const int c = c0 - 1 + w;   // the cell of a[w + 1]
        off[w] = c <= cmax ? dr2(c) : (T)0;
      }
      col_sweep_q<T, DIR, NS, true>(cg, c0, a, vel, off, dt, qs);
    } else {
      col_sweep_q<T, DIR, NS>(cg, c0, a, vel, nullptr, dt, qs);
    }
#pragma unroll
    for (int u = 0; u < NS; u++) {
      const int c = c0 + u;
      if (c <= chi) {
        T qin = qs[u], qout = qs[u + 1];
        if (REL && q < 2) {
          if (vel[u] > (T)0.) qin -= dr2(c);              // upwind cell c-1
          if (!(vel[u + 1] > (T)0.)) qout += dr2(c + 1);  // upwind cell c+1
        }
        const T flux = cg.surf(vel[u] * qin * rs[u], c) - cg.surf(vel[u + 1] * qout * rs[u + 1], c + 1);
        qo[q][cidx(c)] = qv[u + 2] + cg.finish(flux, dt, c);
      }
    }
  }
  if (e_in) {
    // TransportY/Z of the Energy of an adiabatic disk (transport.c:97-98,
    // 122-123): DivideByRho, VanLeer a/b, Update, as for the momenta
    T qv[NS + 4];
#pragma unroll
    for (int w = 0; w < NS + 4; w++) {
      qv[w] = e_in[cidx(min(c0 - 2 + w, cmax))];
      a[w] = qv[w] / r[w];
    }
    col_sweep_q<T, DIR, NS>(cg, c0, a, vel, nullptr, dt, qs);
#pragma unroll
    for (int u = 0; u < NS; u++) {
      const int c = c0 + u;
      if (c <= chi) {
        const T flux = cg.surf(vel[u] * qs[u] * rs[u], c) - cg.surf(vel[u + 1] * qs[u + 1] * rs[u + 1], c + 1);
        e_out[cidx(c)] = qv[u + 2] + cg.finish(flux, dt, c);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < NS; u++) {
    const int c = c0 + u;
    if (c <= chi) rho_out[cidx(c)] = rnew[u];
  }
}

// resident CTAs per SM the FP64 sweeps are compiled for, i.e. their register
// cap: 4 column-sweep CTAs of 128 threads and 2 azimuthal-sweep CTAs of 256
// threads, 128 registers each.  Their FP64 arithmetic is latency-bound, so
// the occupancy gained outweighs the few spilled values (3D 512x256x48: Y+Z
// sweeps 2.98 -> 1.70 ms, azimuthal sweep 2.26 -> 1.72 ms with 2 cells per
// thread; identical results, the register allocation changes no operation)
#ifndef FB_COL64_MINB
#define FB_COL64_MINB 4
#endif
#ifndef FB_SX64_MINB
#define FB_SX64_MINB 2
#endif

template <typename T, int DIR, int NS, typename S = T>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 4 : FB_COL64_MINB) k_sweep_col(Dims m, Geo<T> g, QSrc<T, S> src, int nq, int clo, int chi,
                                                   int t2lo, S *__restrict__ rho_out, S *q_out0, S *q_out1,
                                                   S *q_out2, S *q_out3, S *q_out4, S *q_out5,
                                                   const fb_scalars *__restrict__ scp, const S *__restrict__ e_in,
                                                   S *__restrict__ e_out) {
  b_sweep_col<T, DIR, NS, S>(m, g, src, nq, clo, chi, t2lo, rho_out, q_out0, q_out1, q_out2, q_out3, q_out4, q_out5, scp,
                             blockIdx, e_in, e_out);
}

}  // namespace fb

namespace fb {

// ---------------------------------------------------------------------------
// NewVelocity_x/y/z (newvel_x.c:81, newvel_y.c:70, newvel_z.c:66-69) and
// StockholmBoundary (stockholm.c:129-185) on the active cells; writes the
// new state (rho, vx, vy, vz).
// Correctly rounded division in either precision (IEEE division even where
// the FP32 build approximates '/').
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return a / b; }

template <typename T, typename S = T>
__device__ __forceinline__ void b_newvel(Dims m, Geo<T> g, const S *__restrict__ rt, const S *__restrict__ mpx,
                                                const S *__restrict__ mmx, const S *__restrict__ mpy,
                                                const S *__restrict__ mmy, const S *__restrict__ mpz,
                                                const S *__restrict__ mmz, S *__restrict__ rho, S *__restrict__ vx,
                                                S *__restrict__ vy, S *__restrict__ vz, const S *__restrict__ rho0,
                                                const S *__restrict__ vx0, const S *__restrict__ vy0,
                                                const S *__restrict__ vz0, const double *__restrict__ ramps,
                                                int stockholm, const fb_scalars *__restrict__ scp, uint3 bid,
                                                const S *__restrict__ e_src = nullptr, S *__restrict__ e_dst = nullptr) {
  const int i = bid.x * blockDim.x + threadIdx.x;
  const int j = FB_NGH + bid.y;
  const int k = m.is3d ? FB_NGH + bid.z : 0;
  if (i >= m.nx) return;
  const long long l = m.l(i, j, k);
  // the transported energy of an adiabatic disk becomes its Energy field
  // (StockholmBoundary leaves the energy alone: stockholm.c:167-186)
  if (e_src) e_dst[l] = e_src[l];
  const int im = i > 0 ? i - 1 : m.nx - 1;
  const long long lxm = i > 0 ? l - 1 : l + (m.nx - 1);
  const T of = (T)scp->omegaframe;
  const T syk = ld(g.syk + k), sxi = ld(g.sxi + i), sxim = ld(g.sxi + im), ivj = ld(g.invvj + j);
  const T r = rt[l];
  T nvx, nvy, nvz = 0;
  if (sizeof(S) == 4) {
    // FP32 storage: the same averages with the factors common to numerator
    // and denominator (Syk, InvVj) cancelled, one correctly rounded division
    // per component (a biased division would add the same error to a cell
    // step after step); the azimuthal momenta are frame-relative, so the
    // OMEGAFRAME * R term is not subtracted.
    const T rc = m.sph ? ld(g.ymed + j) * ld(g.sin_zmed + k) : ld(g.ymed + j);
    nvx = div_rn((T)mmx[l] * sxi + (T)mpx[lxm] * sxim, (r * sxi + (T)rt[lxm] * sxim) * rc);
    const T ivjm = ld(g.invvj + j - 1);
    const long long lym = l - m.pitch;
    nvy = div_rn((T)mmy[l] * ivjm + (T)mpy[lym] * ivj, r * ivjm + (T)rt[lym] * ivj);
    if (m.is3d) {
      const T sykm = ld(g.syk + k - 1);
      const long long lzm = l - m.stride;
      nvz = div_rn((T)mmz[l] * syk + (T)mpz[lzm] * sykm, r * syk + (T)rt[lzm] * sykm);
      if (m.sph) nvz = div_rn(nvz, ld(g.ymed + j));
    }
  } else {
    {
      const T rc = m.sph ? ld(g.ymed + j) * ld(g.sin_zmed + k) : ld(g.ymed + j);
      nvx = (mmx[l] * syk * sxi / ivj + mpx[lxm] * syk * sxim / ivj) /
            ((r * syk * sxi / ivj + rt[lxm] * syk * sxim / ivj) * rc);
      nvx -= of * rc;
    }
    {
      const T ivjm = ld(g.invvj + j - 1);
      const long long lym = l - m.pitch;
      nvy = (mmy[l] * syk * sxi / ivj + mpy[lym] * syk * sxi / ivjm) / (r * syk * sxi / ivj + rt[lym] * syk * sxi / ivjm);
    }
    if (m.is3d) {
      const T sykm = ld(g.syk + k - 1);
      const long long lzm = l - m.stride;
      nvz = (mmz[l] * syk * sxi / ivj + mpz[lzm] * sykm * sxi / ivj) / (r * syk * sxi / ivj + rt[lzm] * sykm * sxi / ivj);
      if (m.sph) nvz /= ld(g.ymed + j);
    }
  }
  T nr = r;
  if (stockholm) {
    const double dtd = scp->dt;
    const T dt = (T)dtd;
    const double rampy = ramps[j], rampz = m.is3d ? ramps[m.sy + k] : 0.0, rampzz = m.is3d ? ramps[m.sy + m.sz + k] : 0.0;
    const T ramp = (T)(rampy + rampz), rampi = (T)(rampy + rampzz);
    const T tau = ld(g.tau_j + j);
    const int l2 = j + k * m.sy;
    if (ramp > (T)0.0) {
      const T taud = tau / ramp;
      nr = (nr * taud + rho0[l2] * dt) / (dt + taud);
      T radius = ld(g.ymed + j);
      if (m.sph) radius *= ld(g.sin_zmed + k);
      T vx0t = vx0[l2];
      vx0t -= (of - (T)scp->omegaframe0) * radius;
      nvx = (nvx * taud + vx0t * dt) / (dt + taud);
      nvy = (nvy * taud + vy0[l2] * dt) / (dt + taud);
    }
    if (m.is3d && rampi > (T)0.0) {
      const T taud = tau / rampi;
      nvz = (nvz * taud + vz0[l2] * dt) / (dt + taud);
    }
  }
  rho[l] = nr;
  vx[l] = nvx;
  vy[l] = nvy;
  if (m.is3d) vz[l] = nvz;
}
template <typename T, typename S = T>
__global__ void __launch_bounds__(256) k_newvel(Dims m, Geo<T> g, const S *__restrict__ rt, const S *__restrict__ mpx,
                                                const S *__restrict__ mmx, const S *__restrict__ mpy,
                                                const S *__restrict__ mmy, const S *__restrict__ mpz,
                                                const S *__restrict__ mmz, S *__restrict__ rho, S *__restrict__ vx,
                                                S *__restrict__ vy, S *__restrict__ vz, const S *__restrict__ rho0,
                                                const S *__restrict__ vx0, const S *__restrict__ vy0,
                                                const S *__restrict__ vz0, const double *__restrict__ ramps,
                                                int stockholm, const fb_scalars *__restrict__ scp,
                                                const S *__restrict__ e_src, S *__restrict__ e_dst) {
  b_newvel<T, S>(m, g, rt, mpx, mmx, mpy, mmy, mpz, mmz, rho, vx, vy, vz, rho0, vx0, vy0, vz0, ramps, stockholm, scp,
                 blockIdx, e_src, e_dst);
}

}  // namespace fb

namespace fb {

// ---------------------------------------------------------------------------
// Sources, 3D spherical: the same fusion as k_sources_cyl over a TX x TY tile
// of one colatitude layer, with the inputs of layers k-1..k+1 staged and the
// six stress components of visctensor_sph (visctensor_sph.c:141-213) computed
// where addviscosity_sph (addviscosity_sph.c:74-126) reads them.
template <typename T, int TX, int TY, typename S = T>
__device__ __forceinline__ void b_sources_sph(Dims m, Geo<T> g, Geo<double> gd,
    const S *__restrict__ rho, const S *__restrict__ cs, const S *__restrict__ vx, const S *__restrict__ vy,
    const S *__restrict__ vz, S *__restrict__ vxt, S *__restrict__ vyt, S *__restrict__ vzt,
    const fb_scalars *__restrict__ scp, int dust, int viscous, const double *__restrict__ vbg, uint3 bid) {
  constexpr int W = TX + 2, H = TY + 2;
  __shared__ T s_rho[3][H][W], s_cs[3][H][W], s_vx[3][H][W], s_vy[3][H][W], s_vz[3][H][W];
  __shared__ double s_pot[2][H][W];   // layers k-1, k
  __shared__ T t_xx[2][H][W], t_zz[2][H][W], t_yy[H][W];   // planes k-1, k
  __shared__ T t_xz[2][H][W], t_zy[2][H][W], t_yx[H][W];   // planes k, k+1
  __shared__ fb_scalars sc;
  __shared__ double s_ind[FB_MAXPLANETS];
  constexpr bool FAST = sizeof(S) < sizeof(T);  // FP32 storage: fast potential
  const int i0 = bid.x * TX, j0 = FB_NGH + bid.y * TY, kc = FB_NGH + bid.z;
  const int tid = threadIdx.x + threadIdx.y * TX;
  if (tid == 0) {
    sc = *scp;
    for (int n = 0; n < sc.nplanets; n++) s_ind[n] = sc.pmass[n] / sc.pdist3[n];
  }
  __syncthreads();
  const double dt = sc.dt;
  const T domega = (T)sc.domega, of = (T)sc.omegaframe;
  for (int e = tid; e < 3 * H * W; e += TX * TY) {
    const int lk = e / (H * W), rem = e - lk * H * W, lj = rem / W, li = rem - lj * W;
    const int j = j0 - 1 + lj, k = kc - 1 + lk, i = wrapx(i0 - 1 + li, m.nx);
    if (j < m.sy && i0 - 1 + li <= m.nx) {
      const long long l = m.l(i, j, k);
      const T r = rho[l], c = cs[l];
      s_rho[lk][lj][li] = r;
      s_cs[lk][lj][li] = c;
      if (sizeof(S) < sizeof(T))   // FP32 storage: vx less the ring's background
        s_vx[lk][lj][li] = ((T)vx[l] + (T)bg_at(vbg, j + k * m.sy)) - domega * ld(g.ymed + j) * ld(g.sin_zmed + k);
      else
        s_vx[lk][lj][li] = vx[l] - domega * ld(g.ymed + j) * ld(g.sin_zmed + k);
      s_vy[lk][lj][li] = vy[l];
      s_vz[lk][lj][li] = vz[l];
      if (lk < 2) s_pot[lk][lj][li] = FAST ? potential_fast(m, gd, sc, s_ind, i, j, k) : potential_at(m, gd, sc, i, j, k);
    }
  }
  __syncthreads();
  if (viscous) {
    const T nu = (T)sc.nu, alpha = (T)sc.alpha;
    for (int e = tid; e < 3 * H * W; e += TX * TY) {
      const int lk = e / (H * W), rem = e - lk * H * W, lj = rem / W, li = rem - lj * W;
      const int j = j0 - 1 + lj, k = kc - 1 + lk, i = wrapx(i0 - 1 + li, m.nx);
      if (j >= m.sy - 1 || i0 - 1 + li > m.nx) continue;
      const bool diag = (lk <= 1) && li <= TX && lj <= TY && (lk == 1 || (li >= 1 && lj >= 1));
      const bool offd = (lk >= 1) && li >= 1 && lj >= 1 && (lk == 1 || (li <= TX && lj <= TY));
      if (!diag && !offd) continue;
      T visc = nu, viscm = nu, visczm = nu, visczmym = nu;
      const T e0 = s_cs[lk][lj][li];
      if (m.alpha) {
        visc = alpha * e0 * e0 * ld(g.visc_j + j);
        if (li >= 1 && lj >= 1) {
          const T s1 = e0 + s_cs[lk][lj][li - 1] + s_cs[lk][lj - 1][li] + s_cs[lk][lj - 1][li - 1];
          viscm = alpha * (T)0.0625 * s1 * s1 * ld(g.viscm_j + j);
        }
        if (lk >= 1 && li >= 1) {
          const T s2 = e0 + s_cs[lk - 1][lj][li] + s_cs[lk][lj][li - 1] + s_cs[lk - 1][lj][li - 1];
          visczm = alpha * (T)0.0625 * s2 * s2 * ld(g.visc_j + j);
        }
        if (lk >= 1 && lj >= 1) {
          const T s3 = e0 + s_cs[lk - 1][lj][li] + s_cs[lk][lj - 1][li] + s_cs[lk - 1][lj - 1][li];
          visczmym = alpha * (T)0.0625 * s3 * s3 * ld(g.viscm_j + j);
        }
      }
      const T r = s_rho[lk][lj][li];
      const T sxi = ld(g.sxi + i), syk = ld(g.syk + k);
      const T ym = ld(g.ymed + j), yi = ld(g.ymin + j);
      const T szm = ld(g.sin_zmed + k), czm = ld(g.cos_zmed + k);
      if (diag) {
        const T dvx = s_vx[lk][lj][li + 1] - s_vx[lk][lj][li];
        T div_v = 0.0;
        div_v += dvx * ld(g.sxj + j) * ld(g.sxk + k);
        div_v += (s_vy[lk][lj + 1][li] * ld(g.syj + j + 1) * syk * sxi - s_vy[lk][lj][li] * ld(g.syj + j) * syk * sxi);
        div_v += (s_vz[lk + 1][lj][li] * ld(g.szj + j) * ld(g.szk + k + 1) * sxi -
                  s_vz[lk][lj][li] * ld(g.szj + j) * ld(g.szk + k) * sxi);
        div_v *= (T)(2.0 / 3.0) * ld(g.invvj + j) / (syk * sxi);
        T txx = visc * r * ((T)2.0 * dvx / zsx(m, g, i, j, k) - div_v);
        txx += visc * r * (s_vy[lk][lj + 1][li] + s_vy[lk][lj][li]) / ym;
        txx += visc * r * (s_vz[lk + 1][lj][li] + s_vz[lk][lj][li]) * czm / (szm * ym);
        T tzz = visc * r * ((T)2.0 * (s_vz[lk + 1][lj][li] - s_vz[lk][lj][li]) / (ym * (ld(g.zmin + k + 1) - ld(g.zmin + k))) - div_v);
        tzz += visc * r * (s_vy[lk][lj][li] + s_vy[lk][lj + 1][li]) / ym;
        t_xx[lk][lj][li] = txx;
        t_zz[lk][lj][li] = tzz;
        if (lk == 1)
          t_yy[lj][li] = visc * r * ((T)2.0 * (s_vy[lk][lj + 1][li] - s_vy[lk][lj][li]) / (ld(g.ymin + j + 1) - yi) - div_v);
      }
      if (offd) {
        const T dzm = ld(g.zmed + k) - ld(g.zmed + k - 1), szi = ld(g.sin_zmin + k);
        const T txz = visczm * (T)0.25 * (r + s_rho[lk - 1][lj][li] + s_rho[lk][lj][li - 1] + s_rho[lk - 1][lj][li - 1]) *
                      ((s_vx[lk][lj][li] / szm - s_vx[lk - 1][lj][li] / ld(g.sin_zmed + k - 1)) * szi / (ym * dzm) +
                       ((s_vz[lk][lj][li] - s_vz[lk][lj][li - 1]) * ld(g.invdiffxmed + i) / (szi * ym)));
        const T tzy = visczmym * (T)0.25 * (r + s_rho[lk][lj - 1][li] + s_rho[lk - 1][lj][li] + s_rho[lk - 1][lj - 1][li]) *
                      ((s_vz[lk][lj][li] - s_vz[lk][lj - 1][li]) / (ym - ld(g.ymed + j - 1)) -
                       (T)0.5 * (s_vz[lk][lj][li] + s_vz[lk][lj - 1][li]) / yi +
                       (s_vy[lk][lj][li] - s_vy[lk - 1][lj][li]) / (yi * dzm));
        t_xz[lk - 1][lj][li] = txz;
        t_zy[lk - 1][lj][li] = tzy;
        if (lk == 1)
          t_yx[lj][li] = viscm * (T)0.25 * (r + s_rho[lk][lj][li - 1] + s_rho[lk][lj - 1][li] + s_rho[lk][lj - 1][li - 1]) *
                         ((s_vy[lk][lj][li] - s_vy[lk][lj][li - 1]) * ld(g.invdiffxmed + i) / (yi * szm) +
                          (s_vx[lk][lj][li] - s_vx[lk][lj - 1][li]) / (ym - ld(g.ymed + j - 1)) -
                          (T)0.5 * (s_vx[lk][lj][li] + s_vx[lk][lj - 1][li]) / yi);
      }
    }
    __syncthreads();
  }
  const int li = threadIdx.x + 1, lj = threadIdx.y + 1;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y, k = kc;
  if (i >= m.nx || j > m.ny + FB_NGH - 1) return;
  const int im = wrapx(i - 1, m.nx);
  const long long l = m.l(i, j, k);
  auto P = [&](int a, int b, int c) -> T { return s_rho[a][b][c] * s_cs[a][b][c] * s_cs[a][b][c]; };
  const T r = s_rho[1][lj][li], rxm = s_rho[1][lj][li - 1], rym = s_rho[1][lj - 1][li], rzm = s_rho[0][lj][li];
  const T izx = izsxmed(m, g, i, j, k);
  const T ym = ld(g.ymed + j), ymm = ld(g.ymed + j - 1), yi = ld(g.ymin + j), yip = ld(g.ymin + j + 1),
          yim = ld(g.ymin + j - 1);
  const T zi = ld(g.zmin + k), zip = ld(g.zmin + k + 1), zim = ld(g.zmin + k - 1);
  const T zm = ld(g.zmed + k), zmm = ld(g.zmed + k - 1);
  const T szm = ld(g.sin_zmed + k), czm = ld(g.cos_zmed + k), szi = ld(g.sin_zmin + k), czi = ld(g.cos_zmin + k);
  // SubStep1_x
  const T dxmed = (T)0.5 * (ld(g.sxi + i) + ld(g.sxi + im));
  const T dtorx = (T)2. * (T)dt / (r * ld(g.sxi + i) + rxm * ld(g.sxi + im)) * dxmed;
  T ax = s_vx[1][lj][li];
  if (!dust) ax -= dtorx * (P(1, lj, li) - P(1, lj, li - 1)) * izx;
  ax -= (T)((s_pot[1][lj][li] - s_pot[1][lj][li - 1]) * dt) * izx;
  // SubStep1_y (spherical branch, substep1_y.c:212-217)
  const T dtory = (T)2.0 * (T)dt / (r * (yip - yi) + rym * (yi - yim)) * (ym - ymm);
  T ay = s_vy[1][lj][li];
  if (!dust) ay -= dtory * (P(1, lj, li) - P(1, lj - 1, li)) / (ym - ymm);
  {
    T vphi = (T)0.25 * (s_vx[1][lj][li] + s_vx[1][lj][li + 1] + s_vx[1][lj - 1][li] + s_vx[1][lj - 1][li + 1]);
    vphi += yi * szm * of;
    const T vzz = (T)0.25 * (s_vz[1][lj][li] + s_vz[2][lj][li] + s_vz[1][lj - 1][li] + s_vz[2][lj - 1][li]);
    ay += (vphi * vphi + vzz * vzz) / yi * (T)dt;
  }
  ay -= (T)((s_pot[1][lj][li] - s_pot[1][lj - 1][li]) * dt / (double)(ym - ymm));
  // SubStep1_z (spherical branch, substep1_z.c:172-180)
  const T dtorz = (T)2.0 * (T)dt / (r * (zip - zi) + rzm * (zi - zim)) * (zm - zmm);
  T vphz = (T)0.25 * (s_vx[1][lj][li] + s_vx[1][lj][li + 1] + s_vx[0][lj][li] + s_vx[0][lj][li + 1]);
  vphz += ym * szi * of;
  T az = s_vz[1][lj][li];
  if (!dust) az -= dtorz * (P(1, lj, li) - P(0, lj, li)) / (ym * (zm - zmm));
  az += vphz * vphz * czi / (szi * ym) * (T)dt;
  az -= (T)((s_pot[1][lj][li] - s_pot[0][lj][li]) * dt / (double)(ym * (zm - zmm)));
  if (viscous) {
    // addviscosity_sph
    const T txx = t_xx[1][lj][li];
    ax += (T)2.0 * (txx - t_xx[1][lj][li - 1]) * izx / ((r + rxm)) * (T)dt;
    ax += (T)2.0 * (yip * yip * t_yx[lj + 1][li] - yi * yi * t_yx[lj][li]) / ((yip - yi) * ym * ym * (rxm + r)) * (T)dt;
    ax += (t_yx[lj + 1][li] + t_yx[lj][li]) / ((rxm + r) * ym) * (T)dt;
    ax += (T)2.0 * (t_xz[1][lj][li] - t_xz[0][lj][li]) / (zsz(m, g, j, k) * (rxm + r)) * (T)dt;
    ax += (T)2.0 * (t_xz[1][lj][li] + t_xz[0][lj][li]) * czm / (szm * ym * (rxm + r)) * (T)dt;

    ay += (T)2.0 * (ym * ym * t_yy[lj][li] - ymm * ymm * t_yy[lj - 1][li]) / ((ym - ymm) * (r + rym) * yi * yi) * (T)dt;
    ay += (T)2.0 * (t_yx[lj][li + 1] - t_yx[lj][li]) / ((ld(g.xmin + i + 1) - ld(g.xmin + i)) * yi * szm * (r + rym)) * (T)dt;
    ay -= (txx + t_xx[1][lj - 1][li]) / (yi * (r + rym)) * (T)dt;
    ay -= (t_zz[1][lj][li] + t_zz[1][lj - 1][li]) / (yi * (r + rym)) * (T)dt;
    ay += (T)2.0 * (t_zy[1][lj][li] * ld(g.sin_zmin + k + 1) - t_zy[0][lj][li] * szi) / ((zip - zi) * yi * szm * (r + rym)) * (T)dt;

    az += (T)2.0 * (t_zz[1][lj][li] * szm - t_zz[0][lj][li] * ld(g.sin_zmed + k - 1)) / ((zm - zmm) * ym * szi * (r + rzm)) * (T)dt;
    az += (T)2.0 * (t_xz[0][lj][li + 1] - t_xz[0][lj][li]) / ((ld(g.sxi + i) * ym * szi) * (r + rzm)) * (T)dt;
    az += (T)2.0 * (yip * yip * yip * t_zy[0][lj + 1][li] - yi * yi * yi * t_zy[0][lj][li]) / ((yip - yi) * ym * ym * ym * (r + rzm)) * (T)dt;
    az -= (txx + t_xx[0][lj][li]) * czi / (ym * szi * (r + rzm)) * (T)dt;
  }
  // SubStep2_a / SubStep2_b
  const T c2 = (T)FB_CVNR;
  T dv = s_vx[1][lj][li + 1] - s_vx[1][lj][li];
  const T qx = dv < (T)0.0 ? c2 * c2 * r * dv * dv : (T)0.0;
  dv = s_vx[1][lj][li] - s_vx[1][lj][li - 1];
  const T qxm = dv < (T)0.0 ? c2 * c2 * rxm * dv * dv : (T)0.0;
  dv = s_vy[1][lj + 1][li] - s_vy[1][lj][li];
  const T qy = dv < (T)0.0 ? c2 * c2 * r * dv * dv : (T)0.0;
  dv = s_vy[1][lj][li] - s_vy[1][lj - 1][li];
  const T qym = dv < (T)0.0 ? c2 * c2 * rym * dv * dv : (T)0.0;
  dv = s_vz[2][lj][li] - s_vz[1][lj][li];
  const T qz = dv < (T)0.0 ? c2 * c2 * r * dv * dv : (T)0.0;
  dv = s_vz[1][lj][li] - s_vz[0][lj][li];
  const T qzm = dv < (T)0.0 ? c2 * c2 * rzm * dv * dv : (T)0.0;
  ax += -(T)2.0 * (T)dt * dxmed * (qx - qxm) / (r * ld(g.sxi + i) + rxm * ld(g.sxi + im)) * izx;
  ay += -(T)2.0 * (qy - qym) / (r * (yip - yi) + rym * (yi - yim)) * (T)dt;
  {
    const T dzmed = zm - zmm, dzrho1 = zip - zi, dzrho2 = zi - zim;
    az += -(T)2.0 * dzmed * (qz - qzm) / (r * dzrho1 + rzm * dzrho2) * (T)dt / (ym * (zm - zmm));
  }
  vxt[l] = sizeof(S) < sizeof(T) ? ax - (T)bg_at(vbg, j + k * m.sy) : ax;
  vyt[l] = ay;
  vzt[l] = az;
}
template <typename T, int TX, int TY, typename S = T>
__global__ void __launch_bounds__(TX *TY, sizeof(T) == 4 ? 1 : FB_SPH64_MINB) k_sources_sph(Dims m, Geo<T> g, Geo<double> gd,
    const S *__restrict__ rho, const S *__restrict__ cs, const S *__restrict__ vx, const S *__restrict__ vy,
    const S *__restrict__ vz, S *__restrict__ vxt, S *__restrict__ vyt, S *__restrict__ vzt,
    const fb_scalars *__restrict__ scp, int dust, int viscous, const double *__restrict__ vbg) {
  b_sources_sph<T, TX, TY, S>(m, g, gd, rho, cs, vx, vy, vz, vxt, vyt, vzt, scp, dust, viscous, vbg, blockIdx);
}

}  // namespace fb

namespace fb {

// ---------------------------------------------------------------------------
// Azimuthal sweep, chunked: each thread owns C consecutive cells of a ring
// and keeps them, with a halo of 3 cells each side, in registers; NT threads
// hold NT / (nx / C) whole rings.  A pass (van Leer on the residual velocity,
// or PPA on the uniform fractional velocity) reads the ring from shared
// memory once, updates every quantity in registers and writes it back, so a
// ring costs four barriers instead of one per sub-stage.  Per-cell
// arithmetic is that of vanleer_x_a/_b, fargo_ppa_a..d and update_x as in
// ring_vl_iface / ring_ppa_iface / upd_x above.
template <typename T>
__device__ __forceinline__ T vl_slope(T am, T a0, T ap, T zc, T zp) {
  const T dqm = (a0 - am) / zc;
  const T dqp = (ap - a0) / zp;
  if (dqp * dqm <= (T)0.0) return (T)0.0;
  return ((T)2. * dqp * dqm) / (dqm + dqp);
}
template <typename T>
__device__ __forceinline__ T mc_slope(T am, T a0, T ap) {
  const T dqm = (a0 - am), dqp = (ap - a0);
  if (dqp * dqm <= (T)0.0) return (T)0.0;
  T sl = (T)0.5 * (ap - am);
  T work = fabs(sl);
  if ((T)2.0 * fabs(dqm) < work) work = (T)2.0 * fabs(dqm);
  if ((T)2.0 * fabs(dqp) < work) work = (T)2.0 * fabs(dqp);
  return sl < 0 ? -work : work;
}
template <typename T>
__device__ __forceinline__ void ppa_lr(T am, T a0, T ap, T sm, T s0, T sp, T &L, T &R) {
  R = a0 + (T)0.5 * (ap - a0) - (T)(1.0 / 6.0) * (sp - s0);
  L = am + (T)0.5 * (a0 - am) - (T)(1.0 / 6.0) * (s0 - sm);
  if ((R - a0) * (a0 - L) < (T)0.0) { L = a0; R = a0; }
  const T diff = R - L;
  const T cord = a0 - (T)0.5 * (L + R);
  if ((T)6.0 * diff * cord > diff * diff) L = (T)3.0 * a0 - (T)2.0 * R;
  if (-diff * diff > (T)6.0 * diff * cord) R = (T)3.0 * a0 - (T)2.0 * L;
}

// Interface values qs(f) at the C+1 faces f = c0 .. c0+C of a window
// w[0..C+5] holding cells c0-3 .. c0+C+2.  zone(u) is zone_size_x of cell
// c0-2+u.
template <typename T, int C, typename Z>
__device__ __forceinline__ void chunk_iface(const T *w, const T *v, const Z &zone, T dt, bool ppa, T *qs) {
  if (!ppa) {
    T sl[C + 2];  // cells c0-1 .. c0+C
#pragma unroll
    for (int u = 0; u < C + 2; u++) sl[u] = vl_slope(w[u + 1], w[u + 2], w[u + 3], zone(u + 1), zone(u + 2));
#pragma unroll
    for (int f = 0; f <= C; f++) {  // face c0+f: upwind cell c0+f-1 (sl[f]) or c0+f (sl[f+1])
      if (v[f] > (T)0.0) qs[f] = w[f + 2] + (T)0.5 * (zone(f + 1) - v[f] * dt) * sl[f];
      else qs[f] = w[f + 3] - (T)0.5 * (zone(f + 2) + v[f] * dt) * sl[f + 1];
    }
  } else {
    T sl[C + 4];  // cells c0-2 .. c0+C+1
#pragma unroll
    for (int u = 0; u < C + 4; u++) sl[u] = mc_slope(w[u], w[u + 1], w[u + 2]);
#pragma unroll
    for (int f = 0; f <= C; f++) {
      T L, R, ksi, s;
      if (v[f] > (T)0.0) {  // upwind cell c0+f-1: window index f+2, slopes sl[f..f+2]
        ppa_lr(w[f + 1], w[f + 2], w[f + 3], sl[f], sl[f + 1], sl[f + 2], L, R);
        ksi = v[f] * dt / zone(f + 2);
        s = R + ksi * (w[f + 2] - R);
        s += ksi * ((T)1.0 - ksi) * ((T)2.0 * w[f + 2] - R - L);
      } else {              // cell c0+f: window index f+3, slopes sl[f+1..f+3]
        ppa_lr(w[f + 2], w[f + 3], w[f + 4], sl[f + 1], sl[f + 2], sl[f + 3], L, R);
        ksi = -v[f] * dt / zone(f + 2);
        s = L + ksi * (w[f + 3] - L);
        s += ksi * ((T)1.0 - ksi) * ((T)2.0 * w[f + 3] - R - L);
      }
      qs[f] = s;
    }
  }
}

// The same interfaces for FP32 rings, whose azimuthal zones are one size z:
// the van Leer slope's zone factors cancel into the Courant number v dt / z
// (dtz = dt / z), leaving one division (the harmonic mean) per cell, and the
// PPA's xi = v dt / z is one product.  Algebraically vanleer_x_a/_b and
// fargo_ppa_a..d; rounded differently.
template <int C>
__device__ __forceinline__ void chunk_iface32(const float *w, const float *v, float dtz, bool ppa, float *qs) {
  if (!ppa) {
    float sl[C + 2];  // cells c0-1 .. c0+C: 2 dq+ dq- / (dq- + dq+) of the unscaled differences
#pragma unroll
    for (int u = 0; u < C + 2; u++) {
      const float dqm = w[u + 2] - w[u + 1], dqp = w[u + 3] - w[u + 2];
      sl[u] = (dqp * dqm <= 0.0f) ? 0.0f : (2.0f * dqp * dqm) / (dqm + dqp);
    }
#pragma unroll
    for (int f = 0; f <= C; f++) {
      const float cr = v[f] * dtz;
      if (v[f] > 0.0f) qs[f] = w[f + 2] + 0.5f * (1.0f - cr) * sl[f];
      else qs[f] = w[f + 3] - 0.5f * (1.0f + cr) * sl[f + 1];
    }
  } else {
    float sl[C + 4];  // cells c0-2 .. c0+C+1
#pragma unroll
    for (int u = 0; u < C + 4; u++) sl[u] = mc_slope(w[u], w[u + 1], w[u + 2]);
#pragma unroll
    for (int f = 0; f <= C; f++) {
      float L, R, s;
      if (v[f] > 0.0f) {
        ppa_lr(w[f + 1], w[f + 2], w[f + 3], sl[f], sl[f + 1], sl[f + 2], L, R);
        const float ksi = v[f] * dtz;
        s = R + ksi * (w[f + 2] - R);
        s += ksi * (1.0f - ksi) * (2.0f * w[f + 2] - R - L);
      } else {
        ppa_lr(w[f + 2], w[f + 3], w[f + 4], sl[f + 1], sl[f + 2], sl[f + 3], L, R);
        const float ksi = -v[f] * dtz;
        s = L + ksi * (w[f + 3] - L);
        s += ksi * (1.0f - ksi) * (2.0f * w[f + 3] - R - L);
      }
      qs[f] = s;
    }
  }
}

// The PPA interfaces of an FP32 ring, whose fractional velocity vf is one
// value for the whole ring (compute_residual.c:68-73 with uniform spacing):
// every face has the same upwind side, so the raw interface values
// (fargo_ppa_b: a + (a+ - a)/2 - (s+ - s)/6, shared by a cell's right and its
// neighbour's left edge) are formed once per face, the monotonised edges
// (fargo_ppa_c) once per upwind cell, and the Courant number xi = |vf| dt / z
// once per ring (fargo_ppa_d).
template <int C, int D>
__device__ __forceinline__ void ppa_uniform32_dir(const float *w, float ksi, float *qs) {
  float sl[C + 4];                          // MC slopes of window cells 1 .. C+4
#pragma unroll
  for (int u = 0; u < C + 4; u++) sl[u] = mc_slope(w[u], w[u + 1], w[u + 2]);
  float e[C + 3];                           // raw edge between window cells k and k+1, k = 1 .. C+3
#pragma unroll
  for (int k = 1; k < C + 4; k++)
    e[k - 1] = w[k] + 0.5f * (w[k + 1] - w[k]) - (1.0f / 6.0f) * (sl[k] - sl[k - 1]);
  const float kk = ksi * (1.0f - ksi);
#pragma unroll
  for (int f = 0; f <= C; f++) {
    constexpr int d = D;
    const int k = f + 2 + d;                // upwind window cell of face f
    const float a0 = w[k];
    float L = e[k - 2], R = e[k - 1];       // edges k-1|k and k|k+1
    if ((R - a0) * (a0 - L) < 0.0f) { L = a0; R = a0; }
    const float diff = R - L;
    const float cord = a0 - 0.5f * (L + R);
    if (6.0f * diff * cord > diff * diff) L = 3.0f * a0 - 2.0f * R;
    if (-diff * diff > 6.0f * diff * cord) R = 3.0f * a0 - 2.0f * L;
    const float edge = d ? L : R;
    qs[f] = edge + ksi * (a0 - edge) + kk * (2.0f * a0 - R - L);
  }
}
template <int C>
__device__ __forceinline__ void chunk_ppa_uniform32(const float *w, float vf, float dtz, float *qs) {
  const float ksi = fabsf(vf) * dtz;
  if (vf > 0.0f) ppa_uniform32_dir<C, 0>(w, ksi, qs);   // upwind: the cell before each face
  else ppa_uniform32_dir<C, 1>(w, ksi, qs);             // the cell after it
}

template <typename T, int C, int NT, typename S = T>
__device__ __forceinline__ void b_sweep_x2(const Dims &m, const Geo<T> &g, const Geo<double> &gd, int nq, int jlo,
                                           int klo, int nj, int nrings, S *rho, S *q0, S *q1, S *q2, S *q3, S *q4,
                                           S *q5, const S *__restrict__ vxt, const double *__restrict__ vxmed_t,
                                           int *__restrict__ nshift_out, const fb_scalars *__restrict__ scp,
                                           unsigned long long *__restrict__ errflag, const double *__restrict__ vbg,
                                           long long wait_limit, uint3 bid) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long mbar;
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int nx = m.nx, tpr = nx / C, rpc = NT / tpr, nf = 1 + nq;
  // ring rows in shared memory, each padded by 16 bytes (rows stay 16-byte
  // aligned for the bulk copies and successive rows start in other banks)
  const int nxp = nx + 16 / (int)sizeof(T);
  auto P = [](int i) { return i; };
  const int slot = threadIdx.x / tpr, lt = threadIdx.x - slot * tpr, c0 = lt * C;
  const int r = bid.x * rpc + slot;
  const bool active = slot < rpc && r < nrings;
  const int j = jlo + (active ? r % nj : 0), k = m.is3d ? klo + (active ? r / nj : 0) : 0;
  S *qg[6] = {q0, q1, q2, q3, q4, q5};
  const double dtd = scp->dt;
  const T dt = (T)dtd;
  // shared layout: buffers A and B of [slot][field][nxp] (field 0 rho, 1.. the
  // momenta), then the residual-velocity source vxt [slot][nxp]
  const size_t bufsz = (size_t)rpc * nf * nxp;
  T *bufA = sm, *bufB = sm + bufsz, *svx = sm + 2 * bufsz;
  // Ring rows are contiguous in HBM: when storage and compute types agree and
  // every row is 16-byte aligned, one thread hands all rows of this CTA to the
  // bulk-copy (TMA) engine, completing on an mbarrier; otherwise (FP32
  // storage with FP64 arithmetic, odd ring lengths) the threads load them.
  bool bulk = sizeof(S) == sizeof(T) && ((size_t)nx * sizeof(T)) % 16 == 0;
  if (bulk) {
    uintptr_t a = (uintptr_t)rho | (uintptr_t)vxt;
    for (int q = 0; q < nq; q++) a |= (uintptr_t)qg[q];
    bulk = (a & 15) == 0;
  }
  if (bulk) {
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&mbar);
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t row = (uint32_t)(nx * sizeof(T));
      int nval = 0;
      for (int s2 = 0; s2 < rpc; s2++)
        if (bid.x * rpc + s2 < nrings) nval++;
      const uint32_t total = row * (uint32_t)(nf + 1) * (uint32_t)nval;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(total) : "memory");
      for (int s2 = 0; s2 < rpc; s2++) {
        const int rr = bid.x * rpc + s2;
        if (rr >= nrings) continue;
        const int jj = jlo + rr % nj, kk = m.is3d ? klo + rr / nj : 0;
        const long long l0 = m.l(0, jj, kk);
        for (int q = 0; q <= nf; q++) {   // rho, the momenta, vxt
          const S *src = q == 0 ? rho + l0 : (q < nf ? qg[q - 1] + l0 : vxt + l0);
          T *dstp = q < nf ? bufA + (size_t)s2 * nf * nxp + (size_t)q * nxp : svx + (size_t)s2 * nxp;
          asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                       ::"r"((uint32_t)__cvta_generic_to_shared(dstp)), "l"(src), "r"(row), "r"(bar)
                       : "memory");
        }
      }
    }
    // Bounded wait (wait_limit polls).  The decision is the block's: if any
    // thread gave up, the disk is flagged (its next step reports it; a batch
    // freezes it), every thread waits again -- boundedly -- for the copies in
    // flight, so the CTA does not leave while the copy engine still writes
    // its shared memory, and the block then returns without computing or
    // writing anything.  Past the second limit the block returns regardless.
    uint32_t done = 0;
    for (long long it = 0; it < wait_limit && !done; it++)
      asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                   : "=r"(done) : "r"(bar), "r"(0) : "memory");
    if (__syncthreads_or(!done)) {
      if (threadIdx.x == 0) atomicOr(errflag, 2ull);
      uint32_t drained = 0;
      for (long it = 0; it < (1l << 22) && !drained; it++)
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(drained) : "r"(bar), "r"(0) : "memory");
      __syncthreads();
      return;
    }
  } else {
    for (int e = threadIdx.x; e < rpc * nx; e += NT) {
      const int s = e / nx, i = e - s * nx, rr = bid.x * rpc + s;
      if (rr < nrings) {
        const int jj = jlo + rr % nj, kk = m.is3d ? klo + rr / nj : 0;
        const long long l = m.l(i, jj, kk);
        T *b = bufA + (size_t)s * nf * nxp;
        b[P(i)] = rho[l];
        for (int q = 0; q < nq; q++) b[(1 + q) * nxp + P(i)] = qg[q][l];
        svx[s * nxp + P(i)] = vxt[l];
      }
    }
  }
  __syncthreads();
  const int sl0 = slot < rpc ? slot : 0;
  const double vm = active ? vxmed_t[j + k * m.sy] : 0.0;
  // the residual velocity of the stored (background-relative, FP32 disks) vxt
  const double vm_rel = vm - (active ? bg_at(vbg, j + k * m.sy) : 0.0);
  auto wrap = [&](int i) { i += (i < 0) ? nx : 0; i -= (i >= nx) ? nx : 0; return i; };
  // FP32: the azimuthal spacing is uniform (FARGO's shift requires it), so a
  // ring's zone size is one value, formed once in FP64, instead of a table
  // load per window cell and quantity; FP64 keeps the reference's per-cell
  // zone_size_x
  const T zring = (T)((ld(gd.xmin + 1) - ld(gd.xmin + 0)) * ld(gd.ymed + j) * (m.sph ? ld(gd.sin_zmed + k) : 1.0));
  auto zone = [&](int u) -> T {
    if constexpr (sizeof(T) == 4) return zring;
    else return zsx(m, g, wrap(c0 - 2 + u), j, k);
  };
  const T sxj = ld(g.sxj + j), sxk = ld(g.sxk + k), ivj = ld(g.invvj + j), syk = ld(g.syk + k);
  // FP32: with uniform spacing the update factor dt Surf / Vol is one value
  // per ring (formed in FP64); FP64 keeps the reference's per-cell form
  const T upd_ring = (T)((double)ld(gd.sxj + j) * ld(gd.sxk + k) * dtd * ld(gd.invvj + j) /
                         ((double)ld(gd.syk + k) * ld(gd.sxi + 0)));
  auto upd = [&](int u) -> T {
    if constexpr (sizeof(T) == 4) return upd_ring;
    else return sxj * sxk * dt * ivj / (syk * ld(g.sxi + c0 + u));
  };
  for (int pass = 0; pass < 2; pass++) {
    const T *src = (pass == 0 ? bufA : bufB) + (size_t)sl0 * nf * nxp;
    T *dst = (pass == 0 ? bufB : bufA) + (size_t)sl0 * nf * nxp;
    if (active) {
      T v[C + 1];
      if (pass == 0) {
        if constexpr (sizeof(T) == 4) {
          // the residual of FP32 rings in FP32: vm_rel is the small mean of
          // the background-relative velocity
          const float vr = (float)vm_rel;
          if constexpr (C == 4) {   // aligned float4 reads (no bank conflicts)
            const int tpn = lt < tpr - 1 ? lt + 1 : 0;
            const float4 a4 = reinterpret_cast<const float4 *>(svx + sl0 * nxp)[lt];
            const float v4 = svx[sl0 * nxp + 4 * tpn];
            v[0] = a4.x - vr; v[1] = a4.y - vr; v[2] = a4.z - vr; v[3] = a4.w - vr; v[4] = v4 - vr;
          } else {
#pragma unroll
            for (int f = 0; f <= C; f++) v[f] = svx[sl0 * nxp + P(wrap(c0 + f))] - vr;
          }
        } else {
#pragma unroll
          for (int f = 0; f <= C; f++) v[f] = (T)((double)svx[sl0 * nxp + P(wrap(c0 + f))] - vm_rel);  // residual
        }
      } else if constexpr (sizeof(T) == 4) {
        // uniform fractional velocity (compute_residual.c:68-73), FP64; the
        // FP32 path's azimuthal spacing is uniform, so it is one value per ring
        const double zx = (double)zsx(m, gd, 0, j, k);
        const double ntilde = vm * dtd / zx;
        const T vf = (T)((ntilde - floor(ntilde + 0.5)) * zx / dtd);
#pragma unroll
        for (int f = 0; f <= C; f++) v[f] = vf;
      } else {
#pragma unroll
        for (int f = 0; f <= C; f++) {  // uniform fractional velocity (compute_residual.c:68-73), FP64
          const double zx = (double)zsx(m, gd, wrap(c0 + f), j, k);
          const double ntilde = vm * dtd / zx;
          const double nround = floor(ntilde + 0.5);
          v[f] = (T)((ntilde - nround) * zx / dtd);
        }
      }
      // the C + 6 values around this thread's cells (halo 3 by wrap); FP32
      // rings of 4 cells per thread read three aligned float4 blocks (the
      // left neighbour's, its own, the right neighbour's: conflict-free)
      constexpr bool VEC = C == 4 && sizeof(T) == 4;
      const int tm = lt > 0 ? lt - 1 : tpr - 1, tp = lt < tpr - 1 ? lt + 1 : 0;
      auto window = [&](const T *row, T *w) {
        if constexpr (VEC) {
          const float4 a = reinterpret_cast<const float4 *>(row)[tm];
          const float4 b = reinterpret_cast<const float4 *>(row)[lt];
          const float4 c = reinterpret_cast<const float4 *>(row)[tp];
          w[0] = a.y; w[1] = a.z; w[2] = a.w; w[3] = b.x; w[4] = b.y;
          w[5] = b.z; w[6] = b.w; w[7] = c.x; w[8] = c.y; w[9] = c.z;
        } else {
#pragma unroll
          for (int u = 0; u < C + 6; u++) w[u] = row[P(wrap(c0 - 3 + u))];
        }
      };
      auto store = [&](T *row, const T *o) {
        if constexpr (VEC) {
          reinterpret_cast<float4 *>(row)[lt] = make_float4(o[0], o[1], o[2], o[3]);
        } else {
#pragma unroll
          for (int u = 0; u < C; u++) row[P(c0 + u)] = o[u];
        }
      };
      T wr[C + 6], rs[C + 1], out[C];
      window(src, wr);
      // FP32: one reciprocal of each window density, shared by the momenta
      T irw[C + 6];
      if constexpr (sizeof(T) == 4) {
        if (pass == 1) chunk_ppa_uniform32<C>((const float *)wr, (float)v[0], (float)(dt / zring), (float *)rs);
        else chunk_iface32<C>((const float *)wr, (const float *)v, (float)(dt / zring), false, (float *)rs);
#pragma unroll
        for (int u = 0; u < C + 6; u++) irw[u] = (T)1.0 / wr[u];
      } else {
        chunk_iface<T, C>(wr, v, zone, dt, pass == 1, rs);
      }
      for (int q = 0; q < nq; q++) {
        const T *sq = src + (1 + q) * nxp;
        T raw[C + 6], wq[C + 6], qs[C + 1];
        window(sq, raw);
        if constexpr (sizeof(T) == 4) {
#pragma unroll
          for (int u = 0; u < C + 6; u++) wq[u] = raw[u] * irw[u];  // DivideByRho
          if (pass == 1) chunk_ppa_uniform32<C>((const float *)wq, (float)v[0], (float)(dt / zring), (float *)qs);
          else chunk_iface32<C>((const float *)wq, (const float *)v, (float)(dt / zring), false, (float *)qs);
        } else {
#pragma unroll
          for (int u = 0; u < C + 6; u++) wq[u] = raw[u] / wr[u];  // DivideByRho
          chunk_iface<T, C>(wq, v, zone, dt, pass == 1, qs);
        }
#pragma unroll
        for (int u = 0; u < C; u++) {
          const T fl = v[u] * qs[u] * rs[u] - v[u + 1] * qs[u + 1] * rs[u + 1];
          out[u] = raw[u + 3] + (sizeof(T) == 4 ? fl * upd(u) : fl * sxj * sxk * dt * ivj / (syk * ld(g.sxi + c0 + u)));
        }
        store(dst + (1 + q) * nxp, out);
      }
#pragma unroll
      for (int u = 0; u < C; u++) {
        const T fl = v[u] * rs[u] - v[u + 1] * rs[u + 1];
        out[u] = wr[u + 3] + (sizeof(T) == 4 ? fl * upd(u) : fl * sxj * sxk * dt * ivj / (syk * ld(g.sxi + c0 + u)));
      }
      store(dst, out);
    }
    __syncthreads();
  }
  // AdvectSHIFT (advect_shift.c:49-54): integer shift nround of cell 0, one
  // value per ring (formed by the ring's first thread)
  __shared__ int s_nsh[NT];
  if (active && lt == 0) {
    const double ntilde0 = vm * dtd / (double)zsx(m, gd, 0, j, k);
    const int nsh = (int)floor(ntilde0 + 0.5);
    s_nsh[slot] = nsh;
    if (nshift_out) nshift_out[j + k * m.sy] = nsh;
  }
  __syncthreads();
  if constexpr (sizeof(T) == 4 && sizeof(S) == 4 && C == 4) {
    // FP32 rings of 4 cells per thread: each thread writes its own cells,
    // one float4 per field (the ring rows are 16-byte aligned: nx % 4 == 0)
    if (active) {
      const int nsh = s_nsh[slot];
      int it0 = (c0 - nsh) % nx;
      if (it0 < 0) it0 += nx;
      // the four source cells it0 .. it0+3 (mod nx) lie in the aligned float4
      // blocks q0 = it0 / 4 and the next one (mod nx / 4); the offset
      // it0 % 4 is the same for the whole ring (c0 is a multiple of 4)
      const int q0 = it0 >> 2, q1 = (q0 + 1 < tpr) ? q0 + 1 : 0, sh = it0 & 3;
      const T *b = bufA + (size_t)slot * nf * nxp;
      const long long l = m.l(c0, j, k);
      auto realign = [&](const T *row) -> float4 {
        const float4 x = reinterpret_cast<const float4 *>(row)[q0], y = reinterpret_cast<const float4 *>(row)[q1];
        const float w[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
        return sh == 0 ? make_float4(w[0], w[1], w[2], w[3])
             : sh == 1 ? make_float4(w[1], w[2], w[3], w[4])
             : sh == 2 ? make_float4(w[2], w[3], w[4], w[5])
                       : make_float4(w[3], w[4], w[5], w[6]);
      };
      reinterpret_cast<float4 *>(rho + l)[0] = realign(b);
      for (int q = 0; q < nq; q++) reinterpret_cast<float4 *>(qg[q] + l)[0] = realign(b + (1 + q) * nxp);
    }
    return;
  }
  for (int e = threadIdx.x; e < rpc * nx; e += NT) {
    const int s = e / nx, i = e - s * nx, rr = bid.x * rpc + s;
    if (rr >= nrings) continue;
    const int jj = jlo + rr % nj, kk = m.is3d ? klo + rr / nj : 0;
    const int nsh = s_nsh[s];
    int it = (i - nsh) % nx;
    if (it < 0) it += nx;
    const T *b = bufA + (size_t)s * nf * nxp;
    const long long l = m.l(i, jj, kk);
    rho[l] = b[P(it)];
    for (int q = 0; q < nq; q++) qg[q][l] = b[(1 + q) * nxp + P(it)];
  }
}

// ---------------------------------------------------------------------------
// Implicit drag between the N fluids (Collisions(dt, 1): collisions.c:10-189,
// collision_kernel.h:11-94, gauss.h:1-45), on V_temp after every fluid's
// sources.  One thread per cell (i, j >= 1[, k >= 1]) solves, for each
// direction, the N x N system of the face between the cell and its lower
// neighbour along that direction:
//   M[o][p] (o != p) = -dt W a[p][o] rho_p / rho_o  (p > o),  -dt W a[p][o]  (p < o)
//   M[p][p]          = 1 + dt W sum_{q != p} (q > p ? a[q][p] rho_q / rho_p : a[q][p])
// with face-averaged densities, W = sqrt(G M / r^3) at Ymed (x, z faces) or
// Ymin (y faces), by Gaussian elimination with the reference's row pivoting
// (the search compares |m| with the signed value last kept) and back
// substitution, in the reference's operation order.  The directions touch
// different velocity fields, so solving them in one thread per cell gives the
// reference's direction-by-direction result.
template <typename T, int N, typename S>
__device__ __forceinline__ void b_collisions(const fb_disk_dev &D, Dims m, Geo<double> gd, const fb_scalars *scp,
                                             uint3 bid) {
  const int i = bid.x * blockDim.x + threadIdx.x;
  const int j = 1 + bid.y, k = m.is3d ? 1 + bid.z : 0;
  if (i >= m.nx) return;
  const T dt = (T)scp->dt;
  const long long l = m.l(i, j, k);
  const int ndir = m.is3d ? 3 : 2;
  for (int dir = 0; dir < ndir; dir++) {
    const long long lm = dir == 0 ? (i > 0 ? l - 1 : l + (m.nx - 1)) : (dir == 1 ? l - m.pitch : l - m.stride);
    const T y = (T)(dir == 1 ? ld(gd.ymin + j) : ld(gd.ymed + j));
    const T w = sqrt((T)1.0 / (y * y * y));  // G = MSTAR = 1 (fondam.h)
    T rf[N], M[N * N], b[N];
#pragma unroll
    for (int f = 0; f < N; f++) {
      const S *r = (const S *)D.fl[f].rho;
      rf[f] = (T)0.5 * ((T)r[l] + (T)r[lm]);
    }
#pragma unroll
    for (int o = 0; o < N; o++) {
#pragma unroll
      for (int p = 0; p < N; p++) {
        if (p != o) {
          if (p > o) M[p + o * N] = -dt * w * (T)D.alpha[p + o * N] * rf[p] / rf[o];
          else M[p + o * N] = -dt * w * (T)D.alpha[p + o * N];
        } else {
          T sum = (T)0.0;
#pragma unroll
          for (int q = 0; q < N; q++) {
            if (q == p) continue;
            if (q > p) sum += (T)D.alpha[q + p * N] * rf[q] / rf[p];
            else sum += (T)D.alpha[q + p * N];
          }
          M[p + p * N] = (T)1.0 + dt * w * sum;
        }
      }
      const S *v = (const S *)(dir == 0 ? D.fl[o].vxt : (dir == 1 ? D.fl[o].vyt : D.fl[o].vzt));
      b[o] = (T)v[l];
      // FP32 storage: the drag acts on the full azimuthal velocities
      if (sizeof(S) < sizeof(T) && dir == 0) b[o] += (T)bg_at(D.fl[o].vbg, j + k * m.sy);
    }
#pragma unroll
    for (int ir = 0; ir < N - 1; ir++) {
      T mx = (T)-1;
      int irm = ir;
#pragma unroll
      for (int ir2 = ir; ir2 < N; ir2++)
        if (fabs(M[ir + ir2 * N]) >= mx) { mx = M[ir + ir2 * N]; irm = ir2; }
      if (irm != ir) {
#pragma unroll
        for (int ic = 0; ic < N; ic++) {
          // row exchange by predicated copies keeps the matrix in registers
          T a = M[ic + ir * N];
#pragma unroll
          for (int r2 = ir + 1; r2 < N; r2++)
            if (r2 == irm) { M[ic + ir * N] = M[ic + r2 * N]; M[ic + r2 * N] = a; }
        }
        T a = b[ir];
#pragma unroll
        for (int r2 = ir + 1; r2 < N; r2++)
          if (r2 == irm) { b[ir] = b[r2]; b[r2] = a; }
      }
#pragma unroll
      for (int ir2 = ir + 1; ir2 < N; ir2++) {
        const T factor = M[ir + ir2 * N] / M[ir + ir * N];
#pragma unroll
        for (int ic = 0; ic < N; ic++) M[ic + ir2 * N] -= M[ic + ir * N] * factor;
        b[ir2] -= b[ir] * factor;
      }
    }
#pragma unroll
    for (int ir = N - 1; ir > -1; ir--) {
#pragma unroll
      for (int ic = N - 1; ic > ir; ic--) b[ir] -= M[ic + ir * N] * b[ic];
      b[ir] /= M[ir + ir * N];
    }
#pragma unroll
    for (int o = 0; o < N; o++) {
      S *v = (S *)(dir == 0 ? D.fl[o].vxt : (dir == 1 ? D.fl[o].vyt : D.fl[o].vzt));
      if (sizeof(S) < sizeof(T) && dir == 0) v[l] = (S)(b[o] - (T)bg_at(D.fl[o].vbg, j + k * m.sy));
      else v[l] = (S)b[o];
    }
  }
}

template <typename T, int N, typename S>
__global__ void __launch_bounds__(128) k_collisions(const fb_disk_dev D, Dims m, Geo<double> gd,
                                                    const fb_scalars *scp) {
  b_collisions<T, N, S>(D, m, gd, scp, blockIdx);
}

// ---------------------------------------------------------------------------
// The disk's gravitational acceleration at a point (x, y, z) with smoothing
// rs: ComputeAccel (planets.c:62-84) over _ComputeForce_cpu
// (compute_force.c:16-219), in FP64 and in the reference's summation order:
// each active ring's cells in order of i (reduction_SUM), then the rings in
// order of k then j (reduction_full_SUM), the inner rings (up to the point's
// radius) and the outer ones separately.  Density = the sum of the fluids'
// densities in fluid order (ComputeTotalDensity).
template <typename S>
__device__ __forceinline__ void b_disk_force_rings(const fb_disk_dev &D, double x, double y, double z, double rs,
                                                   double *__restrict__ ring3, int r) {
  const Dims m = dims_of(D);
  const Geo<double> gd = geo_of<double>(D.geomd);
  if (r >= m.ny * (m.is3d ? m.nz : 1)) return;
  const int j = FB_NGH + r % m.ny, k = m.is3d ? FB_NGH + r / m.ny : 0;
  const double ym = ld(gd.ymed + j), syk = ld(gd.syk + k), ivj = ld(gd.invvj + j);
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int i = 0; i < m.nx; i++) {
    const long long l = m.l(i, j, k);
    double dens = 0.0;
    for (int f = 0; f < D.nfluids; f++) dens += (double)((const S *)D.fl[f].rho)[l];
    const double cellmass = syk * ld(gd.sxi + i) / ivj * dens;
    double dx, dy, dz;
    if (m.sph) {
      dx = ym * ld(gd.cos_xmed + i) * ld(gd.sin_zmed + k) - x;
      dy = ym * ld(gd.sin_xmed + i) * ld(gd.sin_zmed + k) - y;
      dz = ym * ld(gd.cos_zmed + k) - z;
    } else {
      dx = ym * ld(gd.cos_xmed + i) - x;
      dy = ym * ld(gd.sin_xmed + i) - y;
      dz = ld(gd.zmed + k) - z;
    }
    double dist2 = dx * dx + dy * dy + dz * dz;
    dist2 += rs * rs;
    const double distance = sqrt(dist2);
    double inv3 = 1.0 / (dist2 * distance);
    inv3 *= 1.0 * cellmass;  // G = 1
    sx += dx * inv3;
    sy += dy * inv3;
    sz += dz * inv3;
  }
  const int n2 = m.sy * m.sz, q = j + k * m.sy;
  ring3[q] = sx;
  ring3[n2 + q] = sy;
  ring3[2 * n2 + q] = sz;
}
template <typename S>
__global__ void __launch_bounds__(128) k_disk_force_rings(const fb_disk_dev D, double x, double y, double z,
                                                          double rs, double *__restrict__ ring3) {
  b_disk_force_rings<S>(D, x, y, z, rs, ring3, blockIdx.x * blockDim.x + threadIdx.x);
}

// fold the ring sums into inner + outer (compute_force.c:161-214)
__device__ __forceinline__ void b_disk_force_fold(const fb_disk_dev &D, double x, double y, double z,
                                                  const double *__restrict__ ring3, double *__restrict__ out3) {
  const Dims m = dims_of(D);
  const Geo<double> gd = geo_of<double>(D.geomd);
  const int k0 = m.is3d ? FB_NGH : 0, k1 = m.is3d ? m.nz + FB_NGH : 1, n2 = m.sy * m.sz;
  const double aa = sqrt(x * x + y * y + z * z);
  const int index = (int)(((aa - ld(gd.ymin + FB_NGH)) / (ld(gd.ymin + m.ny + FB_NGH + 1) - ld(gd.ymin + FB_NGH))) *
                          (double)m.ny) + FB_NGH;
  int ilo = FB_NGH, ihi = FB_NGH, olo = FB_NGH, ohi = m.ny + FB_NGH;   // default: all outer
  if (index >= FB_NGH) {
    if (index < m.ny + FB_NGH) { ihi = index; olo = index; }
    else { ihi = m.ny + FB_NGH; olo = ohi; }
  }
  for (int c = 0; c < 3; c++) {
    double fin = 0.0, fout = 0.0;
    for (int k = k0; k < k1; k++)
      for (int j = ilo; j < ihi; j++) fin = ring3[c * n2 + j + k * m.sy] + fin;
    for (int k = k0; k < k1; k++)
      for (int j = olo; j < ohi; j++) fout = ring3[c * n2 + j + k * m.sy] + fout;
    out3[c] = fin + fout;
  }
}
// one thread
static __global__ void k_disk_force_fold(const fb_disk_dev D, double x, double y, double z,
                                         const double *__restrict__ ring3, double *__restrict__ out3) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  b_disk_force_fold(D, x, y, z, ring3, out3);
}

// ---------------------------------------------------------------------------
// Mass of one fluid, ComputeMass (LowTasks.c:709-748): the sum over the active
// cells of rho * Vol(i, j, k), Vol = Syk(k) * Sxi(i) / InvVj(j) (define.h:229),
// in FP64 with compensation (Neumaier), so its rounding error does not grow
// with the cell count and a change of the total at round-off level is
// visible.  One warp per active ring writes the ring's (sum, compensation);
// one CTA folds the rings in a fixed order.
__device__ __forceinline__ void neumaier_add(double &s, double &c, double v) {
  const double t = s + v;
  if (fabs(s) >= fabs(v)) c += (s - t) + v;
  else c += (v - t) + s;
  s = t;
}
// (s, c) += (s2, c2) with the rounding error of s + s2 kept
__device__ __forceinline__ void neumaier_merge(double &s, double &c, double s2, double c2) {
  neumaier_add(s, c, s2);
  c += c2;
}

template <typename S>
__global__ void __launch_bounds__(256) k_mass_rings(Dims m, Geo<double> gd, const S *__restrict__ rho,
                                                    double *__restrict__ part) {
  const int r = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (r >= m.ny * (m.is3d ? m.nz : 1)) return;
  const int j = FB_NGH + r % m.ny, k = m.is3d ? FB_NGH + r / m.ny : 0;
  const double syk = ld(gd.syk + k), ivj = ld(gd.invvj + j);
  double s = 0.0, c = 0.0;
  for (int i = lane; i < m.nx; i += 32) neumaier_add(s, c, (double)rho[m.l(i, j, k)] * (syk * ld(gd.sxi + i) / ivj));
  for (int o = 16; o > 0; o >>= 1) {
    const double s2 = __shfl_xor_sync(0xffffffffu, s, o), c2 = __shfl_xor_sync(0xffffffffu, c, o);
    // both lanes of a pair fold in the same order (lower lane first)
    if (lane & o) { double t = s2, tc = c2; neumaier_merge(t, tc, s, c); s = t; c = tc; }
    else neumaier_merge(s, c, s2, c2);
  }
  if (lane == 0) { part[2 * r] = s; part[2 * r + 1] = c; }
}

static __global__ void __launch_bounds__(256) k_mass_fold(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double ss[256], cc[256];
  double s = 0.0, c = 0.0;
  for (int r = threadIdx.x; r < n; r += 256) neumaier_merge(s, c, part[2 * r], part[2 * r + 1]);
  ss[threadIdx.x] = s;
  cc[threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double S = 0.0, Cc = 0.0;
    for (int t = 0; t < 256; t++) neumaier_merge(S, Cc, ss[t], cc[t]);
    *out = S + Cc;
  }
}

// shared memory of b_sweep_x2 for a ring of nx cells (rpc rings per CTA)
__host__ __device__ inline size_t sweep_x2_smem(int nx, int C, int nt, int nq, size_t esz) {
  const int rpc = nt / (nx / C);
  const size_t nxp = (size_t)nx + 16 / esz;  // padded ring row (b_sweep_x2)
  return (size_t)rpc * nxp * (2 * (1 + nq) + 1) * esz;
}

// the chunk width a ring of nx cells uses with NT threads per CTA (0: none fits)
__host__ __device__ inline int sweep_x_chunk(int nx, int nt) {
  // the smallest of 4, 8, 16 that fits a ring into nt threads; odd rings 2, 1
  const int cs[5] = {4, 8, 16, 2, 1};
  for (int t = 0; t < 5; t++)
    if (nx % cs[t] == 0 && nx / cs[t] <= nt) return cs[t];
  return 0;
}

// Tile choices of a disk: the set value (fb_disk_set_tiles, usually from the
// autotuner) or the default.
inline int disk_cx(const fb_disk_dev &d) { return d.tile_cx ? d.tile_cx : sweep_x_chunk(d.nx, 256); }
// FP64 column sweeps are compiled for 4 resident CTAs (128 registers), where
// the 4-row segment needs no local memory; FP32 ones default to 8 rows
inline int default_ns(int precision) { return precision == FB_FP64 ? 4 : 8; }
inline int disk_ns(const fb_disk_dev &d) { return d.tile_ns ? d.tile_ns : default_ns(d.precision); }
inline bool valid_cx(int nx, int c) { return (c == 1 || c == 2 || c == 4 || c == 8 || c == 16) && nx % c == 0 && nx / c <= 256; }
inline bool valid_ns(int ns) { return ns == 4 || ns == 8 || ns == 16; }
// polls of the staged-load wait before a disk is flagged (fb_disk_set_wait_limit)
__host__ __device__ inline long long wait_limit(const fb_disk_dev &d) {
  return d.wait_limit > 0 ? d.wait_limit : (d.wait_limit < 0 ? 0 : (1ll << 22));
}

template <typename T, int C, typename S = T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : FB_SX64_MINB) k_sweep_x2(Dims m, Geo<T> g, Geo<double> gd, int nq, int jlo, int klo,
                                                  int nj, int nrings, S *rho, S *q0, S *q1, S *q2, S *q3, S *q4,
                                                  S *q5, const S *__restrict__ vxt,
                                                  const double *__restrict__ vxmed_t, int *__restrict__ nshift_out,
                                                  const fb_scalars *__restrict__ scp,
                                                  unsigned long long *__restrict__ errflag,
                                                  const double *__restrict__ vbg, long long wait_limit) {
  b_sweep_x2<T, C, 256, S>(m, g, gd, nq, jlo, klo, nj, nrings, rho, q0, q1, q2, q3, q4, q5, vxt, vxmed_t, nshift_out,
                        scp, errflag, vbg, wait_limit, blockIdx);
}

}  // namespace fb

#include "fb_sources32.cuh"
