/*
 * fb_dev.h -- plain-C description of one disk's device state, shared by the C
 * host driver (fb_host.c) and the CUDA launchers (fb_kernels_*.cu).
 */
#ifndef FB_DEV_H
#define FB_DEV_H

#include "fb_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Geometry tables on the device: one double set and, for FP32 disks, a float
 * mirror of the same layout (same order of fields as FbGeom<T>). */
typedef struct {
  const void *xmin, *ymin, *zmin, *xmed, *ymed, *zmed, *invdiffxmed;
  const void *sxi, *sxj, *syj, *szj, *sxk, *syk, *szk, *invvj;
  const void *sin_zmed, *cos_zmed, *sin_zmin, *cos_zmin;
  const void *cos_xmed, *sin_xmed;
  const void *visc_j, *viscm_j, *tau_j;
  /* frame-rotation radius tables (FP32 path): ymed^2, its row differences,
     sin^2(zmed) and its layer differences, differenced in double */
  const void *r2_j, *dr2_j, *s2_k, *ds2_k;
  /* per-row reciprocals and the star's potential (FP32-storage sources):
     1/Ymed, 1/Ymin, 1/(Ymed(j) - Ymed(j-1)), -G M / r at Ymed */
  const void *inv_ymed, *inv_ymin, *inv_dymed, *pot_star;
} fb_geom_dev;

typedef struct {
  void *rho, *cs, *vx, *vy, *vz;
  void *vxt, *vyt, *vzt;
  void *mpx, *mmx, *mpy, *mmy, *mpz, *mmz;   /* transport buffers (set A) */
  void *rho_a;                               /* transported density (set A) */
  void *mpx_b, *mmx_b, *mpy_b, *mmy_b, *mpz_b, *mmz_b, *rho_b;  /* set B (3D) */
  double *vxmed, *vxmed_t;
  int *nshift;
  void *rho0, *vx0, *vy0, *vz0;
  int dust;
  /* FP32 disks: the azimuthal velocities (vx, vxt, vx0) are stored relative
     to a per-ring background vbg ([sz][sy] doubles: the FP64 ring mean of the
     first vx the caller gave), so a stored float carries the deviation from
     the ring's rotation, not the rotation itself.  dlb_y / dlb_z hold the
     neighbour differences of vbg * R along y / z (R the cylindrical radius,
     differenced in double, stored in the disk's precision): the column sweeps
     add them to the frame's OMEGAFRAME * R^2 differences.  Null (FP64 disks)
     or zero (no vx given yet) means no background. */
  double *vbg;
  void *dlb_y, *dlb_z;
  /* the background's r-phi shear of face j (2D cylindrical sources):
     (vbg(j) - vbg(j-1)) / (Ymed(j) - Ymed(j-1)) - (vbg(j) + vbg(j-1)) / (2 Ymin(j)),
     formed in double, stored in the disk's precision */
  void *shear_bg;
  int has_bg;
  /* adiabatic disks: the energy after SubStep2_b (et, read by SubStep3) and
     the transported energy (e_a, copied to the Energy field after transport) */
  void *et, *e_a;
} fb_fluid_dev;

/* Per-step scalars (host-computed on the one-disk path, device-computed in
 * batches). */
typedef struct {
  double dt;
  double omegaframe, omegaframe0, domega;
  double nu, alpha, cfl;
  int nplanets;
  double px[FB_MAXPLANETS], py[FB_MAXPLANETS], pz[FB_MAXPLANETS];
  double pmass[FB_MAXPLANETS], psmooth2[FB_MAXPLANETS], pdist3[FB_MAXPLANETS];
  int indirect_term;
  int skip;               /* batched runs: this disk is frozen (error status) */
} fb_scalars;

typedef struct {
  int nx, ny, nz, sy, sz, pitch;
  long long stride;
  int is3d, spherical, alpha_visc;
  int precision;          /* FB_FP64 / FB_FP32 */
  double xlen;            /* XMAX - XMIN */
  double ymin_p, ymax_p, zmin_p, zmax_p;  /* YMIN, YMAX, ZMIN, ZMAX */
  double y_inf, y_sup, z_inf, z_sup;       /* Stockholm ramp limits */
  double cfl, mindx;
  int stockholm;
  double aspectratio, sigmaslope, flaringindex;
  int adiabatic;          /* ADIABATIC: fl[].cs holds the internal energy */
  int dust_diffusion;     /* DUSTDIFFUSION of the dust fluids */
  int bc_lo, bc_hi;       /* the inner / outer radial edge is the mesh's own (1) or a slab's (0) */
  double gamma;           /* GAMMA */
  fb_geom_dev geom;       /* precision of the disk */
  fb_geom_dev geomd;      /* always double */
  fb_fluid_dev fl[FB_MAXFLUIDS];
  int nfluids;
  double *dtmin;          /* device scalar: CFL minimum (bits as u64 min) */
  fb_scalars *scal_dev;   /* device copy of the per-step scalars */
  double *ringsum;        /* per-ring scratch of the mass reduction: 2 x rings + 2 doubles */
  int feeldisk;           /* some planet feels the disk (AdvanceSystemFromDisk) */
  double *ring3;          /* per-ring scratch of the disk's force on a planet: 3 x rings */
  double *facc;           /* the disk's acceleration at each planet: 3 x FB_MAXPLANETS */
  double *bnd_tab;        /* boundary factor tables (double) */
  int bnd_tab_n;
  double *ramps;          /* Stockholm ramps: [sy] radial, [sz] zmed, [sz] zmin */
  int tile_cx;            /* azimuthal sweep cells per thread (0: default) */
  int tile_ns;            /* column sweep segment length (0: default) */
  long long wait_limit;   /* polls of a bounded wait (0: default 2^22; < 0: none) */
  /* collision rates between the fluids, alpha[p + o * nfluids] (ColRate,
     colrate.c:10-23): alpha[0 + f n] = alpha[f + 0 n] = 1/St of dust fluid f */
  double alpha[FB_MAXFLUIDS * FB_MAXFLUIDS];
} fb_disk_dev;

/* Launchers (fb_kernels_f64.cu / fb_kernels_f32.cu). Return cudaError_t. */
#define FB_DECL_LAUNCHERS(SUF)                                                       \
  int fb_launch_rowsum_##SUF(const fb_disk_dev *d, int fluid, int which, void *stream); \
  int fb_launch_cfl_##SUF(const fb_disk_dev *d, int fluid, void *stream);           \
  int fb_launch_sources_##SUF(const fb_disk_dev *d, int fluid, void *stream);       \
  int fb_launch_bnd_##SUF(const fb_disk_dev *d, int fluid, int vtemp, void *stream); \
  int fb_launch_sweep_cols_##SUF(const fb_disk_dev *d, int fluid, void *stream);    \
  int fb_launch_sweep_x_##SUF(const fb_disk_dev *d, int fluid, void *stream);       \
  int fb_launch_newvel_##SUF(const fb_disk_dev *d, int fluid, void *stream);        \
  int fb_launch_collisions_##SUF(const fb_disk_dev *d, void *stream);                 \
  int fb_launch_substep3_##SUF(const fb_disk_dev *d, int fluid, void *stream);        \
  int fb_launch_dust_diffusion_##SUF(const fb_disk_dev *d, int fluid, void *stream);  \
  int fb_launch_mass_##SUF(const fb_disk_dev *d, int fluid, double *part, double *out, void *stream); \
  int fb_launch_disk_force_##SUF(const fb_disk_dev *d, double x, double y, double z, double rs, double *ring3, \
                                 double *out3, void *stream);

FB_DECL_LAUNCHERS(f64)
FB_DECL_LAUNCHERS(f32)

/* Internal accessors of a disk (fb_host.c) for the batched driver. */
struct fb_disk;
fb_disk_dev *fb_disk_internal_dev(struct fb_disk *d);
struct fb_psys_s *fb_disk_internal_psys(struct fb_disk *d);
int fb_disk_internal_initialize_async(struct fb_disk *d);
/* fluid f's state of n disks sharing one stream, one wait (fb_host.c) */
int fb_disks_set_state(struct fb_disk **ds, int n, int f, const double *const *rho, const double *const *vx,
                       const double *const *vy, const double *const *vz, const double *const *cs);
int fb_disks_get_state(struct fb_disk **ds, int n, int f, double *const *rho, double *const *vx, double *const *vy,
                       double *const *vz);
void *fb_disk_internal_scalars(struct fb_disk *d);
size_t fb_disk_internal_esz(struct fb_disk *d);
int fb_internal_fail(int code, const char *what, int cuda_err);
/* FP64 <-> FP32 copy of n values on the device (fb_kernels_f64.cu) */
int fb_launch_convert(void *dst, const void *src, size_t n, int to_f32, void *stream);
/* several FP64 <-> FP32 conversions of a staging chunk in one launch: segment
   k moves n values between staging offset off and the FP32 field f, less (to
   FP32) or plus (to FP64) the per-ring offset bg[i / nx] when bg is set */
#define FB_MAXSEG 48
typedef struct {
  float *f;
  const double *bg;
  long long off, n;
  int nx;
} fb_seg;
typedef struct {
  int n;
  fb_seg s[FB_MAXSEG];
} fb_segs;
int fb_launch_convert_segs(double *st, const fb_segs *segs, int to_f32, void *stream);
/* the same for values of whole rings of nx cells less (to FP32) or plus (to
 * FP64) the per-ring offset off[ring0 + i / nx] */
int fb_launch_convert_off(void *dst, const void *src, size_t n, int to_f32, const double *off, int nx,
                          long long ring0, void *stream);
/* out[r] = mean of the nx doubles of ring r, r < nrings (fixed summation order) */
int fb_launch_ring_mean(double *out, const double *src, int nx, int nrings, void *stream);
/* the background's neighbour differences dlb_y / dlb_z of fluid f (FP32 disks) */
int fb_launch_bg_diffs(const fb_disk_dev *d, int fluid, void *stream);

#ifdef __cplusplus
}
#endif
#endif
