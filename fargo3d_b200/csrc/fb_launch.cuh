// fb_launch.cuh -- host-side launchers of the stage kernels for one precision.
// Included once per precision by fb_kernels_f64.cu / fb_kernels_f32.cu with
// FB_REAL and FB_SUF defined.
#include "fb_kernels.cuh"

namespace fb {

template <typename T, typename S>
static inline QSrc<T, S> qsrc_from_v(const fb_fluid_dev &F, T of) {
  QSrc<T, S> s;
  s.rho = (const S *)F.rho; s.vxt = (const S *)F.vxt; s.vyt = (const S *)F.vyt; s.vzt = (const S *)F.vzt;
  for (int q = 0; q < 6; q++) s.q[q] = nullptr;
  s.from_v = 1;
  s.of = of;
  s.dl = nullptr;
  return s;
}

template <typename T, typename S>
static int launch_rowsum(const fb_disk_dev *d, int f, int which, cudaStream_t st) {
  const fb_fluid_dev &F = d->fl[f];
  Dims m = dims_of(*d);
  Geo<double> gd = geo_of<double>(d->geomd);
  const int nring = m.sy * m.sz;
  const S *v = (const S *)(which == 0 ? F.vx : F.vxt);
  double *out = which == 0 ? F.vxmed : F.vxmed_t;
  if (d->precision != FB_FP64) {  // order-free: one warp per ring
    k_rowsum_warp<S><<<(nring + 7) / 8, 256, 0, st>>>(m, gd, v, out, d->xlen, F.vbg);
    return (int)cudaGetLastError();
  }
  if (nring < 32 * 148) {  // few rings: 8 per CTA
    dim3 grid((nring + 7) / 8);
    if (d->precision == FB_FP64) k_rowsum<T, true, S, 8><<<grid, 256, 0, st>>>(m, gd, v, out, d->xlen);
    else k_rowsum<T, false, S, 8><<<grid, 256, 0, st>>>(m, gd, v, out, d->xlen);
  } else {
    dim3 grid((nring + 31) / 32);
    if (d->precision == FB_FP64) k_rowsum<T, true, S, 32><<<grid, 256, 0, st>>>(m, gd, v, out, d->xlen);
    else k_rowsum<T, false, S, 32><<<grid, 256, 0, st>>>(m, gd, v, out, d->xlen);
  }
  return (int)cudaGetLastError();
}

template <typename T, typename S>
static int launch_cfl(const fb_disk_dev *d, int f, cudaStream_t st) {
  const fb_fluid_dev &F = d->fl[f];
  Dims m = dims_of(*d);
  Geo<T> g = geo_of<T>(sizeof(T) == 8 ? d->geomd : d->geom);
  dim3 grid(m.ny, m.is3d ? m.nz : 1);
  k_cfl<T, S><<<grid, 256, 0, st>>>(m, g, (const S *)F.rho, (const S *)F.cs, (const S *)F.vx, (const S *)F.vy,
                                  (const S *)F.vz, F.vxmed, d->scal_dev, d->cfl, d->mindx,
                                  (unsigned long long *)d->dtmin, F.vbg);
  return (int)cudaGetLastError();
}

template <typename T, typename S>
static int launch_sources(const fb_disk_dev *d, int f, cudaStream_t st) {
  const fb_fluid_dev &F = d->fl[f];
  Dims m = dims_of(*d);
  Geo<T> g = geo_of<T>(sizeof(T) == 8 ? d->geomd : d->geom);
  Geo<double> gd = geo_of<double>(d->geomd);
  const int viscous = !F.dust;
  if (!m.is3d && sizeof(S) == 4) {   // FP32 storage: FP32 arithmetic, column-marching warps
    dim3 grid((m.nx + S32_COLS - 1) / S32_COLS, (m.ny + S32_NS - 1) / S32_NS);
    k_sources_cyl32<<<grid, S32_WARPS * 32, 0, st>>>(m, geo_of<float>(d->geom), gd, (const float *)F.rho,
        (const float *)F.cs, (const float *)F.vx, (const float *)F.vy, (float *)F.vxt, (float *)F.vyt, d->scal_dev,
        F.dust, viscous, F.vbg, (const float *)F.shear_bg);
  } else if (!m.is3d) {
    constexpr int TX = 32, TY = 8;
    // adiabatic: one more row (the outer edge face, read by SubStep3)
    dim3 grid((m.nx + TX - 1) / TX, (m.ny + m.adiab + TY - 1) / TY);
    k_sources_cyl<T, TX, TY, S><<<grid, dim3(TX, TY), 0, st>>>(m, g, gd, (const S *)F.rho, (const S *)F.cs,
        (const S *)F.vx, (const S *)F.vy, (S *)F.vxt, (S *)F.vyt, d->scal_dev, F.dust, viscous, F.vbg, (S *)F.et);
  } else {
    constexpr int TX = 32, TY = 4;
    dim3 grid((m.nx + TX - 1) / TX, (m.ny + TY - 1) / TY, m.nz);
    k_sources_sph<T, TX, TY, S><<<grid, dim3(TX, TY), 0, st>>>(m, g, gd, (const S *)F.rho, (const S *)F.cs,
        (const S *)F.vx, (const S *)F.vy, (const S *)F.vz, (S *)F.vxt, (S *)F.vyt, (S *)F.vzt, d->scal_dev,
        F.dust, viscous, F.vbg);
  }
  return (int)cudaGetLastError();
}

template <typename T, typename S>
static int launch_bnd(const fb_disk_dev *d, int f, int vtemp, cudaStream_t st) {
  const fb_fluid_dev &F = d->fl[f];
  Dims m = dims_of(*d);
  Geo<T> g = geo_of<T>(sizeof(T) == 8 ? d->geomd : d->geom);
  BndTab tb{d->bnd_tab, m.sy, m.sz};
  S *rho = (S *)F.rho;
  S *vx = (S *)(vtemp ? F.vxt : F.vx), *vy = (S *)(vtemp ? F.vyt : F.vy), *vz = (S *)(vtemp ? F.vzt : F.vz);
  const int bx = 128;
  if (m.is3d) {
    dim3 gz((m.nx + bx - 1) / bx, m.sy, 6);
    k_bnd_z<T, S><<<gz, bx, 0, st>>>(m, g, tb, rho, vx, vy, vz, d->scal_dev, !vtemp, F.vbg);
  }
  dim3 gy((m.nx + bx - 1) / bx, 6, m.sz);
  // adiabatic disks: the energy's ghosts too, after the sources and at the end
  k_bnd_y<T, S><<<gy, bx, 0, st>>>(m, g, tb, rho, vx, vy, vz, d->scal_dev, !vtemp, F.vbg,
                                  m.adiab ? (S *)F.cs : (S *)nullptr);
  return (int)cudaGetLastError();
}

template <typename T, typename S, int NS>
static int launch_sweep_cols_n(const fb_disk_dev *d, int f, cudaStream_t st) {
  const fb_fluid_dev &F = d->fl[f];
  Dims m = dims_of(*d);
  Geo<T> g = geo_of<T>(sizeof(T) == 8 ? d->geomd : d->geom);
  Geo<double> gd = geo_of<double>(d->geomd);
  const int bx = 128;
  const int ylo = FB_NGH - 1, yhi = m.ny + FB_NGH - 1;  // rows 2 .. Ny+2
  S *rho_out;
  S *q[6];
  int nq;
  (void)gd;
  if (!m.is3d && sizeof(S) == 4 && sizeof(T) == 4) {   // FP32 2D (fb_sources32.cuh)
    dim3 grid((m.nx + bx - 1) / bx, 1, (yhi - ylo + NS) / NS);
    k_sweep_col32<NS><<<grid, bx, 0, st>>>(m, geo_of<float>(d->geom), (const float *)F.rho, (const float *)F.vxt,
        (const float *)F.vyt, (const float *)F.dlb_y, ylo, yhi, (float *)F.rho_a, (float *)F.mpx, (float *)F.mmx,
        (float *)F.mpy, (float *)F.mmy, d->scal_dev);
    return (int)cudaGetLastError();
  }
  if (!m.is3d) {
    nq = 4;
    QSrc<T, S> src = qsrc_from_v<T, S>(F, (T)0);
    src.dl = (const T *)F.dlb_y;
    rho_out = (S *)F.rho_a;
    q[0] = (S *)F.mpx; q[1] = (S *)F.mmx; q[2] = (S *)F.mpy; q[3] = (S *)F.mmy; q[4] = q[5] = nullptr;
    dim3 grid((m.nx + bx - 1) / bx, 1, (yhi - ylo + NS) / NS);
    // adiabatic disks transport their energy into e_a as a fifth quantity
    k_sweep_col<T, 0, NS, S><<<grid, bx, 0, st>>>(m, g, src, nq, ylo, yhi, 0, rho_out, q[0], q[1], q[2], q[3], q[4],
                                               q[5], d->scal_dev, m.adiab ? (const S *)F.cs : (const S *)nullptr,
                                               m.adiab ? (S *)F.e_a : (S *)nullptr);
  } else {
    nq = 6;
    const int zlo = FB_NGH - 1, zhi = m.nz + FB_NGH - 1;
    // Z sweep from V_temp into set A, rows 0 .. sy-2
    QSrc<T, S> src = qsrc_from_v<T, S>(F, (T)0);
    src.dl = (const T *)F.dlb_z;
    dim3 gz((m.nx + bx - 1) / bx, m.sy - 1, (zhi - zlo + NS) / NS);
    k_sweep_col<T, 1, NS, S><<<gz, bx, 0, st>>>(m, g, src, nq, zlo, zhi, 0, (S *)F.rho_a, (S *)F.mpx, (S *)F.mmx,
                                             (S *)F.mpy, (S *)F.mmy, (S *)F.mpz, (S *)F.mmz, d->scal_dev,
                                             (const S *)nullptr, (S *)nullptr);
    // Y sweep from set A into set B, layers 2 .. Nz+2
    QSrc<T, S> sa;
    sa.rho = (const S *)F.rho_a; sa.vxt = (const S *)F.vxt; sa.vyt = (const S *)F.vyt; sa.vzt = (const S *)F.vzt;
    sa.q[0] = (const S *)F.mpx; sa.q[1] = (const S *)F.mmx; sa.q[2] = (const S *)F.mpy;
    sa.q[3] = (const S *)F.mmy; sa.q[4] = (const S *)F.mpz; sa.q[5] = (const S *)F.mmz;
    sa.from_v = 0; sa.of = (T)0; sa.dl = (const T *)F.dlb_y;
    dim3 gy((m.nx + bx - 1) / bx, zhi - zlo + 1, (yhi - ylo + NS) / NS);
    rho_out = (S *)F.rho_b;
    q[0] = (S *)F.mpx_b; q[1] = (S *)F.mmx_b; q[2] = (S *)F.mpy_b; q[3] = (S *)F.mmy_b; q[4] = (S *)F.mpz_b;
    q[5] = (S *)F.mmz_b;
    k_sweep_col<T, 0, NS, S><<<gy, bx, 0, st>>>(m, g, sa, nq, ylo, yhi, zlo, rho_out, q[0], q[1], q[2], q[3], q[4],
                                             q[5], d->scal_dev, (const S *)nullptr, (S *)nullptr);
  }
  return (int)cudaGetLastError();
}

// column segment length: the disk's tile choice (4, 8 or 16 cells)
template <typename T, typename S>
static int launch_sweep_cols(const fb_disk_dev *d, int f, cudaStream_t st) {
  switch (disk_ns(*d)) {
    case 4: return launch_sweep_cols_n<T, S, 4>(d, f, st);
    case 16: return launch_sweep_cols_n<T, S, 16>(d, f, st);
    default: return launch_sweep_cols_n<T, S, 8>(d, f, st);
  }
}

template <typename T, typename S>
static int launch_sweep_x(const fb_disk_dev *d, int f, cudaStream_t st) {
  const fb_fluid_dev &F = d->fl[f];
  Dims m = dims_of(*d);
  Geo<T> g = geo_of<T>(sizeof(T) == 8 ? d->geomd : d->geom);
  Geo<double> gd = geo_of<double>(d->geomd);
  const int ylo = FB_NGH - 1, yhi = m.ny + FB_NGH - 1;
  const bool b = m.is3d;
  // 2D adiabatic disks: the energy is the fifth transported quantity
  const int nq = b ? 6 : (m.adiab ? 5 : 4);
  S *rho_out = (S *)(b ? F.rho_b : F.rho_a);
  S *q[6] = {(S *)(b ? F.mpx_b : F.mpx), (S *)(b ? F.mmx_b : F.mmx), (S *)(b ? F.mpy_b : F.mpy),
             (S *)(b ? F.mmy_b : F.mmy), (S *)(b ? F.mpz_b : (m.adiab ? F.e_a : F.mpz)), (S *)(b ? F.mmz_b : F.mmz)};
  // azimuthal sweep: C cells per thread, whole rings per CTA of 256 threads
  const int C = disk_cx(*d);
  if (!valid_cx(m.nx, C)) return (int)cudaErrorInvalidValue;
  const int nj = yhi - ylo + 1, nrings = nj * (m.is3d ? m.nz + 1 : 1);
  const int rpc = 256 / (m.nx / C);
  const size_t smem = sweep_x2_smem(m.nx, C, 256, nq, sizeof(T));
  const int klo = m.is3d ? FB_NGH - 1 : 0;
  dim3 gx((nrings + rpc - 1) / rpc);
#define FB_SX(CC)                                                                                          \
  {                                                                                                        \
    static size_t conf = 0;                                                                                \
    if (smem > conf) {                                                                                     \
      cudaFuncSetAttribute(k_sweep_x2<T, CC, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
      conf = smem;                                                                                         \
    }                                                                                                      \
    k_sweep_x2<T, CC, S><<<gx, 256, smem, st>>>(m, g, gd, nq, ylo, klo, nj, nrings, rho_out, q[0], q[1], q[2], \
                                             q[3], q[4], q[5], (const S *)F.vxt, F.vxmed_t, F.nshift,      \
                                             d->scal_dev, (unsigned long long *)d->dtmin + 1, F.vbg, wait_limit(*d));                         \
  }
  switch (C) {
    case 16: FB_SX(16) break;
    case 8: FB_SX(8) break;
    case 4: FB_SX(4) break;
    case 2: FB_SX(2) break;
    default: FB_SX(1) break;
  }
#undef FB_SX
  return (int)cudaGetLastError();
}

template <typename T, typename S>
static int launch_newvel(const fb_disk_dev *d, int f, cudaStream_t st) {
  const fb_fluid_dev &F = d->fl[f];
  Dims m = dims_of(*d);
  Geo<T> g = geo_of<T>(sizeof(T) == 8 ? d->geomd : d->geom);
  const bool b = m.is3d;
  const S *rt = (const S *)(b ? F.rho_b : F.rho_a);
  const S *mpx = (const S *)(b ? F.mpx_b : F.mpx), *mmx = (const S *)(b ? F.mmx_b : F.mmx);
  const S *mpy = (const S *)(b ? F.mpy_b : F.mpy), *mmy = (const S *)(b ? F.mmy_b : F.mmy);
  const S *mpz = (const S *)(b ? F.mpz_b : F.mpz), *mmz = (const S *)(b ? F.mmz_b : F.mmz);
  const int bx = 128;
  if (!m.is3d && sizeof(S) == 4) {   // FP32 2D: column-marching rows
    dim3 g2((m.nx + bx - 1) / bx, (m.ny + NV32_R - 1) / NV32_R);
    k_newvel_cyl32<<<g2, bx, 0, st>>>(m, geo_of<float>(d->geom), (const float *)rt, (const float *)mpx,
        (const float *)mmx, (const float *)mpy, (const float *)mmy, (float *)F.rho, (float *)F.vx, (float *)F.vy,
        (const float *)F.rho0, (const float *)F.vx0, (const float *)F.vy0, d->ramps, d->stockholm, d->scal_dev);
    return (int)cudaGetLastError();
  }
  dim3 grid((m.nx + bx - 1) / bx, m.ny, m.is3d ? m.nz : 1);
  k_newvel<T, S><<<grid, bx, 0, st>>>(m, g, rt, mpx, mmx, mpy, mmy, mpz, mmz, (S *)F.rho, (S *)F.vx, (S *)F.vy,
                                   (S *)F.vz, (const S *)F.rho0, (const S *)F.vx0, (const S *)F.vy0,
                                   (const S *)F.vz0, d->ramps, d->stockholm, d->scal_dev,
                                   m.adiab ? (const S *)F.e_a : (const S *)nullptr, m.adiab ? (S *)F.cs : (S *)nullptr);
  return (int)cudaGetLastError();
}

// implicit drag of all fluids (fluid count 2..FB_MAXFLUIDS)
template <typename T, typename S>
static int launch_collisions(const fb_disk_dev *d, cudaStream_t st) {
  Dims m = dims_of(*d);
  Geo<double> gd = geo_of<double>(d->geomd);
  dim3 g((m.nx + 127) / 128, m.sy - 1, m.is3d ? m.sz - 1 : 1);
  switch (d->nfluids) {
    case 2: k_collisions<T, 2, S><<<g, 128, 0, st>>>(*d, m, gd, d->scal_dev); break;
    case 3: k_collisions<T, 3, S><<<g, 128, 0, st>>>(*d, m, gd, d->scal_dev); break;
    case 4: k_collisions<T, 4, S><<<g, 128, 0, st>>>(*d, m, gd, d->scal_dev); break;
    case 5: k_collisions<T, 5, S><<<g, 128, 0, st>>>(*d, m, gd, d->scal_dev); break;
    case 6: k_collisions<T, 6, S><<<g, 128, 0, st>>>(*d, m, gd, d->scal_dev); break;
    case 7: k_collisions<T, 7, S><<<g, 128, 0, st>>>(*d, m, gd, d->scal_dev); break;
    case 8: k_collisions<T, 8, S><<<g, 128, 0, st>>>(*d, m, gd, d->scal_dev); break;
    default: return (int)cudaErrorInvalidValue;
  }
  return (int)cudaGetLastError();
}

// DustDiffusion_Main for dust fluid f (FP64, 2D): the diffused density into
// rho_a (free until transport), copied back over the active rows, then the
// density's ghosts (FillGhosts(DENS))
template <typename T, typename S>
static int launch_dust_diffusion(const fb_disk_dev *d, int f, cudaStream_t st) {
  if (!d->dust_diffusion || f < 1 || sizeof(S) != 8 || d->is3d) return (int)cudaErrorInvalidValue;
  const fb_fluid_dev &F = d->fl[f], &G = d->fl[0];
  Dims m = dims_of(*d);
  const Geo<double> g = geo_of<double>(d->geomd);
  const dim3 grid((m.nx + 127) / 128, m.ny);
  k_dust_diffusion<double, double><<<grid, 128, 0, st>>>(m, g, (const double *)F.rho, (const double *)G.rho,
                                                          (const double *)G.cs, (double *)F.rho_a, d->scal_dev);
  k_copy_rows<double><<<grid, 128, 0, st>>>(m, (const double *)F.rho_a, (double *)F.rho);
  k_bnd_rho_y<double, double><<<dim3((m.nx + 127) / 128, 6), 128, 0, st>>>(m, g, d->bnd_tab, (double *)F.rho);
  return (int)cudaGetLastError();
}

// SubStep3 of an adiabatic disk (FP64 storage and arithmetic)
template <typename T, typename S>
static int launch_substep3(const fb_disk_dev *d, int f, cudaStream_t st) {
  if (!d->adiabatic || sizeof(S) != 8) return (int)cudaErrorInvalidValue;
  const fb_fluid_dev &F = d->fl[f];
  Dims m = dims_of(*d);
  k_substep3<double><<<dim3((m.nx + 127) / 128, m.ny), 128, 0, st>>>(
      m, geo_of<double>(d->geomd), (const double *)F.et, (const double *)F.vxt, (const double *)F.vyt,
      (double *)F.cs, d->scal_dev);
  return (int)cudaGetLastError();
}

// the disk's acceleration at one point (ComputeAccel), FP64 in every precision
template <typename S>
static int launch_disk_force(const fb_disk_dev *d, double x, double y, double z, double rs, double *ring3,
                             double *out3, cudaStream_t st) {
  const int nr = d->ny * (d->is3d ? d->nz : 1);
  k_disk_force_rings<S><<<(nr + 127) / 128, 128, 0, st>>>(*d, x, y, z, rs, ring3);
  k_disk_force_fold<<<1, 32, 0, st>>>(*d, x, y, z, ring3, out3);
  return (int)cudaGetLastError();
}

// compensated mass of one fluid into out (device double); part: 2 x active
// rings doubles of scratch
template <typename S>
static int launch_mass(const fb_disk_dev *d, int f, double *part, double *out, cudaStream_t st) {
  Dims m = dims_of(*d);
  const int nr = m.ny * (m.is3d ? m.nz : 1);
  k_mass_rings<S><<<(nr + 7) / 8, 256, 0, st>>>(m, geo_of<double>(d->geomd), (const S *)d->fl[f].rho, part);
  k_mass_fold<<<1, 256, 0, st>>>(part, nr, out);
  return (int)cudaGetLastError();
}

}  // namespace fb

#define FB_CAT2(a, b) a##_##b
#define FB_CAT(a, b) FB_CAT2(a, b)

extern "C" {
int FB_CAT(fb_launch_rowsum, FB_SUF)(const fb_disk_dev *d, int fluid, int which, void *s) {
  return fb::launch_rowsum<FB_REAL, FB_STORE>(d, fluid, which, (cudaStream_t)s);
}
int FB_CAT(fb_launch_cfl, FB_SUF)(const fb_disk_dev *d, int fluid, void *s) {
  return fb::launch_cfl<FB_REAL_TR, FB_STORE>(d, fluid, (cudaStream_t)s);
}
int FB_CAT(fb_launch_sources, FB_SUF)(const fb_disk_dev *d, int fluid, void *s) {
  return fb::launch_sources<FB_REAL, FB_STORE>(d, fluid, (cudaStream_t)s);
}
int FB_CAT(fb_launch_bnd, FB_SUF)(const fb_disk_dev *d, int fluid, int vtemp, void *s) {
  return fb::launch_bnd<FB_REAL, FB_STORE>(d, fluid, vtemp, (cudaStream_t)s);
}
int FB_CAT(fb_launch_sweep_cols, FB_SUF)(const fb_disk_dev *d, int fluid, void *s) {
  return fb::launch_sweep_cols<FB_REAL_TR, FB_STORE>(d, fluid, (cudaStream_t)s);
}
int FB_CAT(fb_launch_sweep_x, FB_SUF)(const fb_disk_dev *d, int fluid, void *s) {
  return fb::launch_sweep_x<FB_REAL_TR, FB_STORE>(d, fluid, (cudaStream_t)s);
}
int FB_CAT(fb_launch_newvel, FB_SUF)(const fb_disk_dev *d, int fluid, void *s) {
  return fb::launch_newvel<FB_REAL_TR, FB_STORE>(d, fluid, (cudaStream_t)s);
}
int FB_CAT(fb_launch_collisions, FB_SUF)(const fb_disk_dev *d, void *s) {
  return fb::launch_collisions<FB_REAL, FB_STORE>(d, (cudaStream_t)s);
}
int FB_CAT(fb_launch_dust_diffusion, FB_SUF)(const fb_disk_dev *d, int fluid, void *s) {
  return fb::launch_dust_diffusion<FB_REAL, FB_STORE>(d, fluid, (cudaStream_t)s);
}
int FB_CAT(fb_launch_substep3, FB_SUF)(const fb_disk_dev *d, int fluid, void *s) {
  return fb::launch_substep3<FB_REAL, FB_STORE>(d, fluid, (cudaStream_t)s);
}
int FB_CAT(fb_launch_mass, FB_SUF)(const fb_disk_dev *d, int fluid, double *part, double *out, void *s) {
  return fb::launch_mass<FB_STORE>(d, fluid, part, out, (cudaStream_t)s);
}
int FB_CAT(fb_launch_disk_force, FB_SUF)(const fb_disk_dev *d, double x, double y, double z, double rs,
                                          double *ring3, double *out3, void *s) {
  return fb::launch_disk_force<FB_STORE>(d, x, y, z, rs, ring3, out3, (cudaStream_t)s);
}
}
