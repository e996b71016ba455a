// fb_batch.cuh -- batched stage kernels and the step launcher (see fb_batch.cu),
// included by the per-precision translation units fb_batch_f64.cu and
// fb_batch_f32.cu.
#pragma once
#include <cuda_runtime.h>


#include <stdlib.h>
#include <string.h>
#include <vector>

#include "fargo_b200.h"
#include "fb_kernels.cuh"
#include "fb_psys.h"

namespace fb {

// The azimuthal sweep has one work list per chunk width C (cells per thread;
// ST_X1 + log2 C): each disk uses the width its own ring length picks
// (sweep_x_chunk), so its arithmetic never depends on the other members.
// Likewise the column sweeps have one per segment length NS (ST_Z4 + k,
// ST_Y4 + k for NS = 4 << k).  Both are per-disk tile choices (disk_cx,
// disk_ns; the autotuner sets them).
enum { ST_ROWSUM, ST_CFL, ST_SOURCES, ST_BND_Z, ST_BND_Y, ST_COLL, ST_Z4, ST_Z8, ST_Z16, ST_Y4, ST_Y8, ST_Y16,
       ST_X1, ST_X2, ST_X4, ST_X8, ST_X16, ST_NEWVEL, ST_FORCE, ST_CFL4, ST_NEWVEL4, ST_N };
constexpr int NXC = 5, NNS = 3;

// tile shapes shared with the one-disk launchers (fb_launch.cuh)
// CFL_R rings per CFL CTA and NV_R rows per NewVelocity CTA: enough work per
// CTA to amortise its descriptor loads
constexpr int CFL_R = 4, NV_R = 4;
constexpr int SRC2_TX = 32, SRC2_TY = 8, SRC3_TX = 32, SRC3_TY = 4, COL_BX = 128, BND_BX = 128,
              NV_BX = 128;

// resident CTAs per SM the FP32-storage kernels are compiled for (register
// caps 40 / 64 / 128: measured on the batched 64-disk step, where the
// latency-bound kernels gain more from occupancy than they lose to spills)
#ifndef FB_SRC_MINB
#define FB_SRC_MINB 6
#endif
#ifndef FB_SX_MINB32
#define FB_SX_MINB32 4
#endif
// FP32 2D CFL, NewVelocity and column sweep (kb_cfl_cyl32, kb_newvel_cyl32,
// kb_sweep_col32): 6, 8 and 8 CTAs of 128 threads per SM (80, 64 and 64
// registers).  Measured on the batched 64-disk step against the unconstrained
// builds (147, 128 and 128 registers): CFL 0.090 -> 0.061 ms, NewVelocity
// 0.088 -> 0.078 ms, column sweep 0.164 -> 0.135 ms (segments of 4 rows).
#ifndef FB_CFL32_MINB
#define FB_CFL32_MINB 6
#endif
#ifndef FB_NV32_MINB
#define FB_NV32_MINB 8
#endif
#ifndef FB_COL32_MINB
#define FB_COL32_MINB 8
#endif
#ifndef FB_COL_MINB32
#define FB_COL_MINB32 4
#endif

#define FB_TILE                                        \
  const int4 w = items[blockIdx.x];                    \
  const fb_disk_dev &D = ds[w.x];                      \
  const fb_scalars *scp = D.scal_dev;                  \
  if (scp->skip) return;                               \
  const uint3 bid = make_uint3(w.y, w.z, w.w);         \
  const fb_fluid_dev &F = D.fl[f];                     \
  (void)F;

template <typename T, bool ORDERED, typename S>
__global__ void __launch_bounds__(256) kb_rowsum(const fb_disk_dev *ds, const int4 *items, int f, int which) {
  FB_TILE
  const S *v = (const S *)(which == 0 ? F.vx : F.vxt);
  double *out = which == 0 ? F.vxmed : F.vxmed_t;
  if (ORDERED) b_rowsum<T, true, S>(dims_of(D), geo_of<double>(D.geomd), v, out, D.xlen, bid);  // 32 rings / CTA
  else b_rowsum_warp<S>(dims_of(D), geo_of<double>(D.geomd), v, out, D.xlen, F.vbg, bid);    // 8 rings / CTA
}

template <typename T, typename S>
__global__ void __launch_bounds__(256) kb_cfl(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  // CFL_R rings per CTA, one minimum folded per CTA
  const Dims m = dims_of(D);
  const Geo<T> g = geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom);
  const int k = m.is3d ? FB_NGH + (int)bid.y : 0;
  const int j0 = FB_NGH + (int)bid.x * CFL_R;
  const int nr = min(CFL_R, m.ny + FB_NGH - j0);
  const T nu = (T)scp->nu, alpha = (T)scp->alpha;
  unsigned long long *dtmin = (unsigned long long *)D.dtmin;
  double mn = 1e20;
  bool bad = false;
  // the CTA's cells, ring after ring, spread over all its threads (rings of
  // 128 cells keep all 256 busy); min and OR do not depend on the order
  int r = 0, i = threadIdx.x;
  while (i >= m.nx) { i -= m.nx; r++; }
  if constexpr (sizeof(T) == 4 && sizeof(S) == 4) {
    if (!m.is3d) {   // FP32 2D: per-ring reciprocals, no division per cell
#pragma unroll 2
      for (; r < nr;) {
        const int j = j0 + r;
        mn = fmin(mn, (double)cfl_cell32(m, g, (const float *)F.rho, (const float *)F.cs, (const float *)F.vx,
                                         (const float *)F.vy, F.vxmed[j] - bg_at(F.vbg, j), nu, alpha, (float)D.cfl,
                                         i, j, bad));
        i += blockDim.x;
        while (i >= m.nx) { i -= m.nx; r++; }
      }
      r = nr;
    }
  }
#pragma unroll 2
  for (; r < nr;) {
    const int j = j0 + r;
    mn = fmin(mn, (double)cfl_cell<T, S>(m, g, (const S *)F.rho, (const S *)F.cs, (const S *)F.vx, (const S *)F.vy,
                                         (const S *)F.vz, F.vxmed[j + k * m.sy] - bg_at(F.vbg, j + k * m.sy), nu,
                                         alpha, D.cfl, i, j, k, bad));
    i += blockDim.x;
    while (i >= m.nx) { i -= m.nx; r++; }
  }
  if (bad) atomicOr(dtmin + 1, 1ull);
  if ((int)threadIdx.x < nr) {
    const int j = j0 + threadIdx.x;
    const double shear = cfl_shear(g, F.vxmed, D.cfl, D.mindx, j + k * m.sy, j);
    if (shear < mn) mn = shear;
  }
  cfl_commit(mn, dtmin);
}

// FP32 2D: 128 columns x CFL32_R rows a tile (fb_sources32.cuh)
static __global__ void __launch_bounds__(128, FB_CFL32_MINB) kb_cfl_cyl32(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  b_cfl_cyl32(dims_of(D), geo_of<float>(D.geom), (const float *)F.rho, (const float *)F.cs, (const float *)F.vx,
              (const float *)F.vy, F.vxmed, F.vbg, (float)scp->nu, (float)scp->alpha, D.cfl, D.mindx,
              (unsigned long long *)D.dtmin, bid);
}

template <typename T, typename S>
__global__ void __launch_bounds__(SRC2_TX *SRC2_TY, sizeof(S) == 4 ? FB_SRC_MINB : 1) kb_sources_cyl(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  b_sources_cyl<T, SRC2_TX, SRC2_TY, S>(dims_of(D), geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom), geo_of<double>(D.geomd), (const S *)F.rho,
                                     (const S *)F.cs, (const S *)F.vx, (const S *)F.vy, (S *)F.vxt, (S *)F.vyt, scp,
                                     F.dust, !F.dust, F.vbg, (S *)nullptr, bid);
}

// FP32 storage, 2D: FP32 arithmetic, column-marching warps (fb_sources32.cuh)
static __global__ void __launch_bounds__(S32_WARPS * 32, FB_S32_MINB) kb_sources_cyl32(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  b_sources_cyl32(dims_of(D), geo_of<float>(D.geom), geo_of<double>(D.geomd), (const float *)F.rho,
                  (const float *)F.cs, (const float *)F.vx, (const float *)F.vy, (float *)F.vxt, (float *)F.vyt, scp,
                  F.dust, !F.dust, F.vbg, (const float *)F.shear_bg, bid);
}

template <typename T, typename S>
__global__ void __launch_bounds__(SRC3_TX *SRC3_TY, sizeof(T) == 4 ? 1 : FB_SPH64_MINB) kb_sources_sph(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  b_sources_sph<T, SRC3_TX, SRC3_TY, S>(dims_of(D), geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom), geo_of<double>(D.geomd), (const S *)F.rho,
                                     (const S *)F.cs, (const S *)F.vx, (const S *)F.vy, (const S *)F.vz, (S *)F.vxt,
                                     (S *)F.vyt, (S *)F.vzt, scp, F.dust, !F.dust, F.vbg, bid);
}

template <typename T, typename S>
__global__ void kb_bnd(const fb_disk_dev *ds, const int4 *items, int f, int vtemp, int zside) {
  FB_TILE
  Dims m = dims_of(D);
  BndTab tb{D.bnd_tab, m.sy, m.sz};
  S *vx = (S *)(vtemp ? F.vxt : F.vx), *vy = (S *)(vtemp ? F.vyt : F.vy), *vz = (S *)(vtemp ? F.vzt : F.vz);
  if (zside) b_bnd_z<T, S>(m, geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom), tb, (S *)F.rho, vx, vy, vz, scp, !vtemp, F.vbg, bid);
  else b_bnd_y<T, S>(m, geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom), tb, (S *)F.rho, vx, vy, vz, scp, !vtemp, F.vbg, bid);
}

template <typename T, int N, typename S>
__global__ void __launch_bounds__(128) kb_collisions(const fb_disk_dev *ds, const int4 *items) {
  const int4 w = items[blockIdx.x];
  const fb_disk_dev &D = ds[w.x];
  if (D.scal_dev->skip) return;
  b_collisions<T, N, S>(D, dims_of(D), geo_of<double>(D.geomd), D.scal_dev, make_uint3(w.y, w.z, w.w));
}

// FP32 2D disks: the radial sweep of fb_sources32.cuh
template <int COL_NS>
static __global__ void __launch_bounds__(COL_BX, FB_COL32_MINB) kb_sweep_col32(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  b_sweep_col32<COL_NS>(dims_of(D), geo_of<float>(D.geom), (const float *)F.rho, (const float *)F.vxt,
                        (const float *)F.vyt, (const float *)F.dlb_y, FB_NGH - 1, D.ny + FB_NGH - 1, (float *)F.rho_a,
                        (float *)F.mpx, (float *)F.mmx, (float *)F.mpy, (float *)F.mmy, scp, bid);
}

template <typename T, int DIR, int COL_NS, typename S>
__global__ void __launch_bounds__(COL_BX, sizeof(T) == 4 ? FB_COL_MINB32 : FB_COL64_MINB) kb_sweep_col(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  Dims m = dims_of(D);
  const int ylo = FB_NGH - 1, yhi = m.ny + FB_NGH - 1;
  QSrc<T, S> src;
  src.vxt = (const S *)F.vxt; src.vyt = (const S *)F.vyt; src.vzt = (const S *)F.vzt; src.of = (T)0;
  src.dl = (const T *)(DIR == 1 ? F.dlb_z : F.dlb_y);
  if (!m.is3d || DIR == 1) {
    src.rho = (const S *)F.rho;
    for (int q = 0; q < 6; q++) src.q[q] = nullptr;
    src.from_v = 1;
  } else {
    src.rho = (const S *)F.rho_a;
    src.q[0] = (const S *)F.mpx; src.q[1] = (const S *)F.mmx; src.q[2] = (const S *)F.mpy;
    src.q[3] = (const S *)F.mmy; src.q[4] = (const S *)F.mpz; src.q[5] = (const S *)F.mmz;
    src.from_v = 0;
  }
  if (!m.is3d) {
    b_sweep_col<T, 0, COL_NS, S>(m, geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom), src, 4, ylo, yhi, 0, (S *)F.rho_a, (S *)F.mpx, (S *)F.mmx,
                              (S *)F.mpy, (S *)F.mmy, nullptr, nullptr, scp, bid);
  } else if (DIR == 1) {
    b_sweep_col<T, 1, COL_NS, S>(m, geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom), src, 6, FB_NGH - 1, m.nz + FB_NGH - 1, 0, (S *)F.rho_a,
                              (S *)F.mpx, (S *)F.mmx, (S *)F.mpy, (S *)F.mmy, (S *)F.mpz, (S *)F.mmz, scp, bid);
  } else {
    b_sweep_col<T, 0, COL_NS, S>(m, geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom), src, 6, ylo, yhi, FB_NGH - 1, (S *)F.rho_b, (S *)F.mpx_b,
                              (S *)F.mmx_b, (S *)F.mpy_b, (S *)F.mmy_b, (S *)F.mpz_b, (S *)F.mmz_b, scp, bid);
  }
}

template <typename T, int C, typename S>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? FB_SX_MINB32 : FB_SX64_MINB) kb_sweep_x(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  Dims m = dims_of(D);
  const bool b = m.is3d;
  const int nj = m.ny + 1, nrings = nj * (b ? m.nz + 1 : 1);
  b_sweep_x2<T, C, 256, S>(m, geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom), geo_of<double>(D.geomd), b ? 6 : 4, FB_NGH - 1, b ? FB_NGH - 1 : 0,
                        nj, nrings, (S *)(b ? F.rho_b : F.rho_a), (S *)(b ? F.mpx_b : F.mpx),
                        (S *)(b ? F.mmx_b : F.mmx), (S *)(b ? F.mpy_b : F.mpy), (S *)(b ? F.mmy_b : F.mmy),
                        (S *)(b ? F.mpz_b : F.mpz), (S *)(b ? F.mmz_b : F.mmz), (const S *)F.vxt, F.vxmed_t, F.nshift,
                        scp, (unsigned long long *)D.dtmin + 1, F.vbg, wait_limit(D), bid);
}

template <typename T, typename S>
__global__ void __launch_bounds__(NV_BX) kb_newvel(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  Dims m = dims_of(D);
  const bool b = m.is3d;
  const Geo<T> g = geo_of<T>(sizeof(T) == 8 ? D.geomd : D.geom);
  for (int r = 0; r < NV_R; r++) {   // NV_R rows per CTA
    const uint3 rb = make_uint3(bid.x, bid.y * NV_R + r, bid.z);
    if ((int)rb.y >= m.ny) break;
    b_newvel<T, S>(m, g, (const S *)(b ? F.rho_b : F.rho_a), (const S *)(b ? F.mpx_b : F.mpx),
                (const S *)(b ? F.mmx_b : F.mmx), (const S *)(b ? F.mpy_b : F.mpy), (const S *)(b ? F.mmy_b : F.mmy),
                (const S *)(b ? F.mpz_b : F.mpz), (const S *)(b ? F.mmz_b : F.mmz), (S *)F.rho, (S *)F.vx,
                (S *)F.vy, (S *)F.vz, (const S *)F.rho0, (const S *)F.vx0, (const S *)F.vy0, (const S *)F.vz0,
                D.ramps, D.stockholm, scp, rb);
  }
}

// FP32 2D: column-marching rows (fb_sources32.cuh); 128 columns x NV32_R rows a tile
static __global__ void __launch_bounds__(Q32_T) kb_cfl_cyl32q(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  b_cfl_cyl32q(dims_of(D), geo_of<float>(D.geom), (const float *)F.rho, (const float *)F.cs, (const float *)F.vx,
               (const float *)F.vy, F.vxmed, F.vbg, (float)scp->nu, (float)scp->alpha, D.cfl, D.mindx,
               (unsigned long long *)D.dtmin, (int)bid.x);
}
static __global__ void __launch_bounds__(Q32_T) kb_newvel_cyl32q(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  b_newvel_cyl32q(dims_of(D), geo_of<float>(D.geom), (const float *)F.rho_a, (const float *)F.mpx,
                  (const float *)F.mmx, (const float *)F.mpy, (const float *)F.mmy, (float *)F.rho, (float *)F.vx,
                  (float *)F.vy, (const float *)F.rho0, (const float *)F.vx0, (const float *)F.vy0, D.ramps,
                  D.stockholm, scp, (int)bid.x);
}
static __global__ void __launch_bounds__(128, FB_NV32_MINB) kb_newvel_cyl32(const fb_disk_dev *ds, const int4 *items, int f) {
  FB_TILE
  b_newvel_cyl32(dims_of(D), geo_of<float>(D.geom), (const float *)F.rho_a, (const float *)F.mpx,
                 (const float *)F.mmx, (const float *)F.mpy, (const float *)F.mmy, (float *)F.rho, (float *)F.vx,
                 (float *)F.vy, (const float *)F.rho0, (const float *)F.vx0, (const float *)F.vy0, D.ramps,
                 D.stockholm, scp, bid);
}

// The disk's acceleration at planet n of every disk whose planet n feels the
// disk (ComputeAccel for AdvanceSystemFromDisk, planets.c:86-114), from the
// density and planets at the start of the step: the ring sums (one lane per
// ring, the reference's order), then one thread per disk folds them.  The
// smoothing is the planet's (compute_potential's RocheSmoothing or the
// flared thickness), formed on the device.
__device__ __forceinline__ bool force_planet(const fb_disk_dev &D, const fb_psys &S, int n, double &x, double &y,
                                             double &z, double &rs) {
  if (!D.feeldisk || n >= S.np || !S.feeldisk[n]) return false;
  x = S.px[n]; y = S.py[n]; z = S.pz[n];
  const double r = sqrt(x * x + y * y + z * z), mp = S.pmass[n];
  if (S.roche_smoothing != 0) rs = r * pow(mp / 3. / FB_MSTAR, 1. / 3.) * S.roche_smoothing;
  else rs = S.aspectratio * pow(r / FB_R0, S.flaringindex) * r * S.thickness_smoothing;
  return true;
}
template <typename S>
static __global__ void __launch_bounds__(128) kb_disk_force_rings(const fb_disk_dev *ds, const fb_psys *ps,
                                                                  const int4 *items, int n) {
  const int4 w = items[blockIdx.x];
  const fb_disk_dev &D = ds[w.x];
  if (D.scal_dev->skip) return;
  double x, y, z, rs;
  if (!force_planet(D, ps[w.x], n, x, y, z, rs)) return;
  b_disk_force_rings<S>(D, x, y, z, rs, D.ring3, w.y * 128 + threadIdx.x);
}
static __global__ void kb_disk_force_fold(const fb_disk_dev *ds, const fb_psys *ps, const int *dl, int nd, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nd) return;
  const int i = dl ? dl[t] : t;
  const fb_disk_dev &D = ds[i];
  if (D.nx == 0 || D.scal_dev->skip) return;
  double x, y, z, rs;
  if (!force_planet(D, ps[i], n, x, y, z, rs)) return;
  b_disk_force_fold(D, x, y, z, D.ring3, D.facc + 3 * n);
}

// The scalar work of the step for every disk of the list dl (all n disks when
// dl is null), one thread per disk; then the
// CFL minimum is reset for the next step.  dtmin[1] carries the kernels'
// non-finite flag.  A disk with an end time uses it as its DT interval, so
// its last step is clipped to land on it; that step still runs in full, and
// the disk is frozen (FB_DONE) when the next step's scalar work finds it
// there.  Empty slots (zeroed descriptors) are passed over.
static __global__ void kb_scalars(const fb_disk_dev *ds, fb_psys *ps, const int *dl, int n, double DT) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = dl ? dl[t] : t;
  const fb_disk_dev &D = ds[i];
  if (D.nx == 0) return;
  unsigned long long *dm = (unsigned long long *)D.dtmin;
  fb_scalars sc = *D.scal_dev;
  if (!sc.skip) {
    fb_psys S = ps[i];
    const double cflmin = __longlong_as_double((long long)dm[0]);
    if (S.status == FB_DONE) {
      sc.skip = 1;
    } else if (dm[1] != 0ull) {
      S.status = FB_ERR_NONFINITE;
      sc.skip = 1;
    } else if (fb_psys_step(&S, cflmin, S.t_end > 0.0 ? S.t_end : DT, &sc, D.feeldisk ? D.facc : nullptr) < 0.0) {
      sc.skip = 1;
    } else if (S.t_end > 0.0 && S.dtemp >= S.t_end) {
      S.status = FB_DONE;
    }
    ps[i] = S;
    *D.scal_dev = sc;
  }
  dm[0] = 0x4415AF1D78B58C40ULL;  // 1e20, the MIN reduction start (define.h:165)
}

}  // namespace fb

using namespace fb;

#define FB_MAX_CHAINS 8
/* FP32 batches step as 4 concurrent chains (measured: 0.741 ms -> 0.684 ms for
   the 64-disk workload); FP64 batches, whose stage kernels fill the GPU on
   their own, as one */
#define FB_DEFAULT_CHAINS_F32 4
#define FB_DEFAULT_CHAINS_F64 1

// Slots: state[i] 0 empty, 1 reserved (created, not activated), 2 active.
// n is the capacity; the work lists cover the active slots only.
struct fb_batch {
  int n, precision, device, is3d, nfluids;
  std::vector<int> state;
  std::vector<double> t_end;
  int dirty;
  char *arena;   // one allocation lent to the members of fb_batch_create (or null)
  cudaStream_t stream;
  std::vector<fb_disk *> disks;
  fb_disk_dev *d_disks;
  fb_psys *d_psys;
  int4 *items[ST_N];
  int nitems[ST_N];
  /* concurrent step chains: the active disks split into nchains groups of
     about equal cells, each group stepped on its own stream with its own work
     lists (chain c: citems[c], its disks cdisks[c]), so that one group's
     latency-bound launches (the scalar step, reductions, boundaries, launch
     tails) overlap another's throughput-bound ones */
  void *lists;    /* one device allocation holding every work list below */
  void *h_act;    /* page-locked staging of the members' activation uploads */
  int force_np;   /* planet indices that feel the disk in some member (0: none) */
  int nchains;
  cudaStream_t cstream[FB_MAX_CHAINS];
  cudaEvent_t ev_fork, ev_join[FB_MAX_CHAINS];
  int4 *citems[FB_MAX_CHAINS][ST_N];
  int ncitems[FB_MAX_CHAINS][ST_N];
  int *cdisks[FB_MAX_CHAINS];
  int ncdisks[FB_MAX_CHAINS];
  std::vector<int> chain_of;
  size_t smem_x[NXC];  /* shared memory of each chunk-width class of the azimuthal sweep */
  cudaGraphExec_t exec;
  int graph_steps;
  double graph_dt;
};

static int tiles(fb_batch *B, int st, std::vector<int4> &v, int chain = -1) {
  for (int di = 0; di < B->n; di++) {
    if (B->state[di] != 2) continue;
    if (chain >= 0 && B->chain_of[di] != chain) continue;
    const fb_disk_dev &D = *fb_disk_internal_dev(B->disks[di]);
    const int nx = D.nx, ny = D.ny, nz = D.nz, sy = D.sy, sz = D.sz;
    // FP32 2D disks whose rings hold a multiple of 4 cells: CFL and
    // NewVelocity four cells a thread (fb_sources32.cuh)
    const bool quad = !D.is3d && B->precision == FB_FP32 && nx % 4 == 0;
    dim3 g(1, 1, 1);
    switch (st) {
      case ST_ROWSUM: g = dim3(B->precision == FB_FP64 ? (sy * sz + 31) / 32 : (sy * sz + 7) / 8); break;
      case ST_CFL:
        if (quad) g = dim3(0);
        else if (!D.is3d && B->precision == FB_FP32) g = dim3((nx + 127) / 128, (ny + CFL32_R - 1) / CFL32_R);
        else g = dim3((ny + CFL_R - 1) / CFL_R, D.is3d ? nz : 1);
        break;
      case ST_SOURCES:
        if (D.is3d) g = dim3((nx + SRC3_TX - 1) / SRC3_TX, (ny + SRC3_TY - 1) / SRC3_TY, nz);
        else if (B->precision == FB_FP32) g = dim3((nx + S32_COLS - 1) / S32_COLS, (ny + S32_NS - 1) / S32_NS);
        else g = dim3((nx + SRC2_TX - 1) / SRC2_TX, (ny + SRC2_TY - 1) / SRC2_TY);
        break;
      case ST_BND_Z: g = D.is3d ? dim3((nx + BND_BX - 1) / BND_BX, sy, 6) : dim3(0); break;
      case ST_BND_Y: g = dim3((nx + BND_BX - 1) / BND_BX, 6, sz); break;
      case ST_COLL: g = D.nfluids > 1 ? dim3((nx + 127) / 128, sy - 1, D.is3d ? sz - 1 : 1) : dim3(0); break;
      case ST_Z4: case ST_Z8: case ST_Z16: {
        const int ns = 4 << (st - ST_Z4);
        g = D.is3d && disk_ns(D) == ns ? dim3((nx + COL_BX - 1) / COL_BX, sy - 1, (nz + 1 + ns - 1) / ns) : dim3(0);
        break;
      }
      case ST_Y4: case ST_Y8: case ST_Y16: {
        const int ns = 4 << (st - ST_Y4);
        g = disk_ns(D) == ns ? dim3((nx + COL_BX - 1) / COL_BX, D.is3d ? nz + 1 : 1, (ny + 1 + ns - 1) / ns)
                             : dim3(0);
        break;
      }
      case ST_X1: case ST_X2: case ST_X4: case ST_X8: case ST_X16: {
        const int c = 1 << (st - ST_X1);
        if (disk_cx(D) != c) { g = dim3(0); break; }
        const int rpc = 256 / (nx / c), nr = (ny + 1) * (D.is3d ? nz + 1 : 1);
        g = dim3((nr + rpc - 1) / rpc);
        break;
      }
      case ST_FORCE: {
        const int nr = ny * (D.is3d ? nz : 1);
        g = D.feeldisk ? dim3((nr + 127) / 128) : dim3(0);
        break;
      }
      case ST_CFL4: case ST_NEWVEL4:
        g = quad ? dim3((nx / 4 * ny + Q32_T - 1) / Q32_T) : dim3(0);
        break;
      case ST_NEWVEL:
        if (quad) g = dim3(0);
        else if (!D.is3d && B->precision == FB_FP32) g = dim3((nx + 127) / 128, (ny + NV32_R - 1) / NV32_R);
        else g = dim3((nx + NV_BX - 1) / NV_BX, (ny + NV_R - 1) / NV_R, D.is3d ? nz : 1);
        break;
    }
    for (unsigned z = 0; z < g.z; z++)
      for (unsigned y = 0; y < g.y; y++)
        for (unsigned x = 0; x < g.x; x++) v.push_back(make_int4(di, (int)x, (int)y, (int)z));
  }
  return (int)v.size();
}

template <typename T, typename S>
static void configure_sweep_x(fb_batch *B) {
  static size_t done[NXC];
  for (int k = 0; k < NXC; k++) {
    if (done[k] >= B->smem_x[k]) continue;
    done[k] = B->smem_x[k];
    const int sm = (int)B->smem_x[k];
    switch (k) {
      case 4: cudaFuncSetAttribute(kb_sweep_x<T, 16, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); break;
      case 3: cudaFuncSetAttribute(kb_sweep_x<T, 8, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); break;
      case 2: cudaFuncSetAttribute(kb_sweep_x<T, 4, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); break;
      case 1: cudaFuncSetAttribute(kb_sweep_x<T, 2, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); break;
      default: cudaFuncSetAttribute(kb_sweep_x<T, 1, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); break;
    }
  }
}

// optional per-launch timing of an eager (uncaptured) step
struct Prof {
  cudaEvent_t ev[40];
  const char *name[40];
  int n;
};
extern Prof *g_prof;
static void pmark(cudaStream_t st, const char *name) {
  if (!g_prof || g_prof->n >= 40) return;
  cudaEventCreate(&g_prof->ev[g_prof->n]);
  cudaEventRecord(g_prof->ev[g_prof->n], st);
  g_prof->name[g_prof->n++] = name;
}

// T: compute type of the source stage; TC, TX, TN, TF: of the column sweeps,
// the azimuthal sweep, NewVelocity and the CFL's per-cell limits (its
// minimum is always FP64); S: storage type.
// chain < 0: every active disk on the batch's stream (one chain); else the
// disks of that chain on its stream.
template <typename T, typename S, typename TC = T, typename TX = T, typename TN = T, typename TF = T>
static int launch_step(fb_batch *B, double DT, int chain) {
  int4 *const *items = chain < 0 ? B->items : B->citems[chain];
  const int *nitems = chain < 0 ? B->nitems : B->ncitems[chain];
  if (nitems[ST_ROWSUM] == 0) return 0;  // no active disk
  configure_sweep_x<TX, S>(B);
  cudaStream_t st = chain < 0 ? B->stream : B->cstream[chain];
  pmark(st, "start");
  const fb_disk_dev *ds = B->d_disks;
  const int nf = B->nfluids;
  auto grid = [&](int s) { return dim3((unsigned)nitems[s]); };
  for (int f = 0; f < nf; f++) {
    if (B->precision == FB_FP64) kb_rowsum<T, true, S><<<grid(ST_ROWSUM), 256, 0, st>>>(ds, items[ST_ROWSUM], f, 0);
    else kb_rowsum<T, false, S><<<grid(ST_ROWSUM), 256, 0, st>>>(ds, items[ST_ROWSUM], f, 0);
  }
  pmark(st, "rowsum");
  for (int f = 0; f < nf; f++) {
    if (nitems[ST_CFL4]) kb_cfl_cyl32q<<<grid(ST_CFL4), Q32_T, 0, st>>>(ds, items[ST_CFL4], f);
    if (!nitems[ST_CFL]) continue;
    if (!B->is3d && sizeof(S) == 4) kb_cfl_cyl32<<<grid(ST_CFL), 128, 0, st>>>(ds, items[ST_CFL], f);
    else kb_cfl<TF, S><<<grid(ST_CFL), 256, 0, st>>>(ds, items[ST_CFL], f);
  }
  pmark(st, "cfl");
  {
    const int nd = chain < 0 ? B->n : B->ncdisks[chain];
    const int *dl = chain < 0 ? nullptr : B->cdisks[chain];
    if (nitems[ST_FORCE]) {   // planets that feel the disk, one planet index at a time
      for (int n = 0; n < B->force_np; n++) {
        kb_disk_force_rings<S><<<grid(ST_FORCE), 128, 0, st>>>(ds, B->d_psys, items[ST_FORCE], n);
        kb_disk_force_fold<<<(nd + 63) / 64, 64, 0, st>>>(ds, B->d_psys, dl, nd, n);
      }
      pmark(st, "disk_force");
    }
    kb_scalars<<<(nd + 63) / 64, 64, 0, st>>>(ds, B->d_psys, dl, nd, DT);
  }
  pmark(st, "scalars");
  for (int f = 0; f < nf; f++) {
    if (B->is3d) kb_sources_sph<T, S><<<grid(ST_SOURCES), dim3(SRC3_TX, SRC3_TY), 0, st>>>(ds, items[ST_SOURCES], f);
    else if (sizeof(S) == 4) kb_sources_cyl32<<<grid(ST_SOURCES), S32_WARPS * 32, 0, st>>>(ds, items[ST_SOURCES], f);
    else kb_sources_cyl<T, S><<<grid(ST_SOURCES), dim3(SRC2_TX, SRC2_TY), 0, st>>>(ds, items[ST_SOURCES], f);
    pmark(st, "sources");
    if (B->is3d) kb_bnd<T, S><<<grid(ST_BND_Z), BND_BX, 0, st>>>(ds, items[ST_BND_Z], f, 1, 1);
    kb_bnd<T, S><<<grid(ST_BND_Y), BND_BX, 0, st>>>(ds, items[ST_BND_Y], f, 1, 0);
    pmark(st, "bnd_vtemp");
  }
  if (nf > 1 && nitems[ST_COLL]) {  // implicit drag between the fluids
    const int4 *it = items[ST_COLL];
    switch (nf) {
      case 2: kb_collisions<T, 2, S><<<grid(ST_COLL), 128, 0, st>>>(ds, it); break;
      case 3: kb_collisions<T, 3, S><<<grid(ST_COLL), 128, 0, st>>>(ds, it); break;
      case 4: kb_collisions<T, 4, S><<<grid(ST_COLL), 128, 0, st>>>(ds, it); break;
      case 5: kb_collisions<T, 5, S><<<grid(ST_COLL), 128, 0, st>>>(ds, it); break;
      case 6: kb_collisions<T, 6, S><<<grid(ST_COLL), 128, 0, st>>>(ds, it); break;
      case 7: kb_collisions<T, 7, S><<<grid(ST_COLL), 128, 0, st>>>(ds, it); break;
      default: kb_collisions<T, 8, S><<<grid(ST_COLL), 128, 0, st>>>(ds, it); break;
    }
    pmark(st, "collisions");
  }
  for (int f = 0; f < nf; f++) {
    if (B->precision == FB_FP64) kb_rowsum<T, true, S><<<grid(ST_ROWSUM), 256, 0, st>>>(ds, items[ST_ROWSUM], f, 1);
    else kb_rowsum<T, false, S><<<grid(ST_ROWSUM), 256, 0, st>>>(ds, items[ST_ROWSUM], f, 1);
    pmark(st, "rowsum_vtemp");
    if (B->is3d) {
      if (nitems[ST_Z4]) kb_sweep_col<TC, 1, 4, S><<<grid(ST_Z4), COL_BX, 0, st>>>(ds, items[ST_Z4], f);
      if (nitems[ST_Z8]) kb_sweep_col<TC, 1, 8, S><<<grid(ST_Z8), COL_BX, 0, st>>>(ds, items[ST_Z8], f);
      if (nitems[ST_Z16]) kb_sweep_col<TC, 1, 16, S><<<grid(ST_Z16), COL_BX, 0, st>>>(ds, items[ST_Z16], f);
    }
    if (!B->is3d && sizeof(S) == 4 && sizeof(TC) == 4) {   // FP32 2D
      if (nitems[ST_Y4]) kb_sweep_col32<4><<<grid(ST_Y4), COL_BX, 0, st>>>(ds, items[ST_Y4], f);
      if (nitems[ST_Y8]) kb_sweep_col32<8><<<grid(ST_Y8), COL_BX, 0, st>>>(ds, items[ST_Y8], f);
      if (nitems[ST_Y16]) kb_sweep_col32<16><<<grid(ST_Y16), COL_BX, 0, st>>>(ds, items[ST_Y16], f);
    } else {
      if (nitems[ST_Y4]) kb_sweep_col<TC, 0, 4, S><<<grid(ST_Y4), COL_BX, 0, st>>>(ds, items[ST_Y4], f);
      if (nitems[ST_Y8]) kb_sweep_col<TC, 0, 8, S><<<grid(ST_Y8), COL_BX, 0, st>>>(ds, items[ST_Y8], f);
      if (nitems[ST_Y16]) kb_sweep_col<TC, 0, 16, S><<<grid(ST_Y16), COL_BX, 0, st>>>(ds, items[ST_Y16], f);
    }
    pmark(st, "sweep_cols");
    for (int k = 0; k < NXC; k++) {
      const int n = nitems[ST_X1 + k];
      if (!n) continue;
      const int4 *it = items[ST_X1 + k];
      const size_t sm = B->smem_x[k];
      switch (k) {
        case 4: kb_sweep_x<TX, 16, S><<<n, 256, sm, st>>>(ds, it, f); break;
        case 3: kb_sweep_x<TX, 8, S><<<n, 256, sm, st>>>(ds, it, f); break;
        case 2: kb_sweep_x<TX, 4, S><<<n, 256, sm, st>>>(ds, it, f); break;
        case 1: kb_sweep_x<TX, 2, S><<<n, 256, sm, st>>>(ds, it, f); break;
        default: kb_sweep_x<TX, 1, S><<<n, 256, sm, st>>>(ds, it, f); break;
      }
    }
    pmark(st, "sweep_x");
  }
  for (int f = 0; f < nf; f++) {
    if (nitems[ST_NEWVEL4]) kb_newvel_cyl32q<<<grid(ST_NEWVEL4), Q32_T, 0, st>>>(ds, items[ST_NEWVEL4], f);
    if (nitems[ST_NEWVEL]) {
      if (!B->is3d && sizeof(S) == 4) kb_newvel_cyl32<<<grid(ST_NEWVEL), 128, 0, st>>>(ds, items[ST_NEWVEL], f);
      else kb_newvel<TN, S><<<grid(ST_NEWVEL), NV_BX, 0, st>>>(ds, items[ST_NEWVEL], f);
    }
    pmark(st, "newvel");
    if (B->is3d) kb_bnd<T, S><<<grid(ST_BND_Z), BND_BX, 0, st>>>(ds, items[ST_BND_Z], f, 0, 1);
    kb_bnd<T, S><<<grid(ST_BND_Y), BND_BX, 0, st>>>(ds, items[ST_BND_Y], f, 0, 0);
    pmark(st, "bnd");
  }
  return (int)cudaGetLastError();
}

