// fb_common.cuh -- shared device-side types of the B200 hydro step.
//
// Layout (the reference's, define.h:455): a field of one disk is a dense array
// [sz][sy][pitch] with x (azimuth) fastest, sy = Ny + 6 rows (3 ghost rows on
// each radial side), sz = Nz + 6 colatitude layers in 3D and 1 in 2D.  The
// azimuth has no ghost cells: it is periodic inside the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "fb_abi.h"

#define FB_NG 3

// Geometry arrays of one disk on the device (double; float mirrors for the
// FP32 kernels).  Everything that the reference computes with libm from mesh
// coordinates is tabulated on the host with the same libm call, so device
// arithmetic sees the identical operands.
template <typename T>
struct FbGeom {
  const T *xmin, *ymin, *zmin, *xmed, *ymed, *zmed, *invdiffxmed;
  const T *sxi, *sxj, *syj, *szj, *sxk, *syk, *szk, *invvj;
  const T *sin_zmed, *cos_zmed, *sin_zmin, *cos_zmin;  // per layer k
  const T *cos_xmed, *sin_xmed;                        // per column i
  const T *visc_j, *viscm_j;  // sqrt(ymed^3/(G M)), sqrt(ymin^3/(G M)) (alpha-nu)
  const T *tau_j;             // TauDamp * sqrt(ymed^3/G/MSTAR) (stockholm.c:134)
};

struct FbDims {
  int nx, ny, nz;      // active zones (nz = 1 in 2D)
  int sy, sz;          // stored rows / layers
  int pitch;           // elements between rows (>= nx)
  long long stride;    // elements between layers (pitch * sy)
  int is3d, spherical, alpha_visc;
};

// Per-step scalars produced on the host (FP64 path) or by the scalar kernel.
struct FbStepScalars {
  double dt;
  double omegaframe, omegaframe0, domega;
  double nu, alpha, cfl;
  int nplanets;
  double px[FB_MAXPLANETS], py[FB_MAXPLANETS], pz[FB_MAXPLANETS];
  double pmass[FB_MAXPLANETS], psmooth2[FB_MAXPLANETS], pdist3[FB_MAXPLANETS];
  int indirect_term;
};

// Fields of one fluid of one disk.
template <typename T>
struct FbFluid {
  T *rho, *cs, *vx, *vy, *vz;        // persistent state
  T *vxt, *vyt, *vzt;                // V_temp
  T *mpx, *mmx, *mpy, *mmy, *mpz, *mmz;  // momenta during transport
  double *vxmed;                     // 2D [sz][sy] FP64 ring mean
  double *vxmed_t;                   // ring mean of V_temp
  int *nshift;                       // 2D [sz][sy]
  T *rho0, *vx0, *vy0, *vz0;         // Stockholm references (2D)
  int dust;
};

__host__ __device__ inline long long fb_l(const FbDims &d, int i, int j, int k) {
  return (long long)i + (long long)j * d.pitch + (long long)k * d.stride;
}
