// fb_noalloc.cu -- the CFL time step of a state held in caller-owned device
// memory, computed without allocating anything.
//
// Who needs this: code that owns every byte of device memory itself and does
// not let a library call cudaMalloc -- FARGO3D's own GPU build, whose Fields
// are allocated once by CreateField and whose _gpu functions run between
// them, a host application running from a fixed memory pool, or a caller that
// wants the CFL step while it must not touch the allocator (for instance in
// a latency-critical loop).  Such callers pass their field and mesh pointers
// and get the time step written to a device double they own.
//
// The scratch this computation needs (the ring means of v_phi and the running
// minimum) lives in one file-scope __device__ array of fixed size, so every
// GPU that loads this library holds it (FB_NOALLOC_MAX_RINGS + 64 doubles,
// 512.5 KiB) until the process exits.  Host code cannot use the array's name
// as a device address: its device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, the first time the entry
// point runs on it -- make that first call before any stream capture.  All
// calls share the array and it keeps the last call's contents; the kernels
// reset the running minimum and the failure word at the start of each call.
// Two calls whose work overlaps on the GPU (different streams, no ordering
// between them) race on the array and must not be issued.
//
// Fields may be pitched (FARGO3D's GPU build allocates them with
// cudaMallocPitch and indexes them by Pitch_gpu / Stride_gpu, allocate.c:
// 169-206): the arguments carry the element pitch and stride.
#include <cuda_runtime.h>

#include <mutex>

#include "fargo_b200.h"
#include "fb_kernels.cuh"

#define FB_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double fb_noalloc_scratch[FB_NOALLOC_MAX_RINGS + 64];

namespace {

std::mutex g_mu;
double *g_scratch[FB_NOALLOC_MAX_DEVICES];

// cfl.c:135-258 and cfl_b.c:14-39 with the mesh terms formed in the kernel
// from the edge arrays exactly as the host forms its tables
// (Ymed = 0.5*(Ymin[j+1]+Ymin[j]), Sxi = Xmin[i+1]-Xmin[i]).
__global__ void __launch_bounds__(256) k_cfl_static(fb_cfl_static_args a, const double *__restrict__ vxmed,
                                                    unsigned long long *__restrict__ dtmin, long long pitch,
                                                    long long stride) {
  const int j = 3 + blockIdx.x;
  const int is3d = a.nz > 1;
  const int k = is3d ? 3 + blockIdx.y : 0;
  const int sy = a.ny + 6;
  bool bad = false;
  const double ymed = 0.5 * (a.ymin[j + 1] + a.ymin[j]);
  const double ymedp = 0.5 * (a.ymin[j + 2] + a.ymin[j + 1]);
  const double zy = (a.ymin[j + 1] - a.ymin[j]);
  const double vm = vxmed[j + k * sy];
  const double szm = (is3d && a.spherical) ? a.sin_zmed[k] : 1.0;
  double zz = 1.0;
  if (is3d) zz = a.spherical ? ((a.zmin[k + 1] - a.zmin[k]) * ymed) : (a.zmin[k + 1] - a.zmin[k]);
  double mn = 1e20;
  for (int i = threadIdx.x; i < a.nx; i += blockDim.x) {
    const long long l = i + j * pitch + k * stride;
    const long long lxp = (i < a.nx - 1) ? l + 1 : l - (a.nx - 1);
    const double sxi = a.xmin[i + 1] - a.xmin[i];
    const double zx = a.spherical ? (sxi * ymed * szm) : (sxi * ymed);
    const double vxx = a.vx[l] - vm, vxxp = a.vx[lxp] - vm;
    const double c = a.cs[l];
    const double visc = a.alpha_visc ? a.alpha * c * c * sqrt(ymed * ymed * ymed / (1.0 * 1.0)) : a.nu;
    const double ss = sqrt(c * c);
    double c1c = 0, c4 = 0, c5c = 0, c7c = 0;
    if (is3d) c1c = ss / zz;
    const double c1 = fb::dmax3(ss / zx, ss / zy, c1c);
    const double c2 = (fb::dmax2(fabs(vxx), fabs(vxxp))) / zx;
    const double c3 = (fb::dmax2(fabs(a.vy[l]), fabs(a.vy[l + pitch]))) / zy;
    if (is3d) c4 = (fb::dmax2(fabs(a.vz[l]), fabs(a.vz[l + stride]))) / zz;
    const double c5a = fabs(a.vx[lxp] - a.vx[l]) / zx;
    const double c5b = fabs(a.vy[l + pitch] - a.vy[l]) / zy;
    if (is3d) c5c = fabs(a.vz[l + stride] - a.vz[l]) / zz;
    const double c5 = fb::dmax3(c5a, c5b, c5c) * 4.0 * FB_CVNR;
    if (is3d) c7c = 1.0 / zz;
    const double mx7 = fb::dmax3(1.0 / zx, 1.0 / zy, c7c);
    const double c7 = 4.0 * visc * (mx7 * mx7);
    const double dtc = a.cfl / sqrt(c1 * c1 + c2 * c2 + c3 * c3 + c4 * c4 + c5 * c5 + 0.0 * 0.0 + c7 * c7 +
                                    0.0 * 0.0 + 0.0 * 0.0 + 0.0 * 0.0);
    bad |= !(dtc == dtc) || !(a.rho[l] > 0.0);
    mn = fmin(mn, dtc);
  }
  // a non-finite limit or a non-positive density: the step comes out NaN
  if (bad) atomicOr(dtmin + 1, 1ull);
  if (threadIdx.x == 0) {
    const double shear = a.cfl * a.mindx / fabs(vm / ymed - vxmed[j + 1 + k * sy] / ymedp);
    if (shear < mn) mn = shear;
  }
  for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  __shared__ double wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = mn;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : 1e20;
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    // a zero limit folds too: the step is then 0, the reference's null step
    if (threadIdx.x == 0 && v >= 0.0) atomicMin(dtmin, (unsigned long long)__double_as_longlong(v + 0.0));
  }
}

// resets the running minimum to the MIN reduction's start value (1e20,
// define.h:165) and the failure word before the rings are summed
__global__ void k_reset_min(unsigned long long *dtmin) {
  dtmin[0] = 0x4415AF1D78B58C40ULL;
  dtmin[1] = 0ull;
}

// CflFluidsMin (cfl_fluids_min.c:9-13): StepTime = min(1e30, Min); NaN when
// some cell had a non-finite limit or a non-positive density
__global__ void k_finish_dt(const unsigned long long *dtmin, double *dt_out) {
  const double m = __longlong_as_double((long long)dtmin[0]);
  double step = 1e30;
  if (step > m) step = m;
  *dt_out = dtmin[1] ? __longlong_as_double(0x7ff8000000000000LL) : step;
}

}  // namespace

extern "C" int fb_cfl_dt_static(const fb_cfl_static_args *a, double *dt_out, void *stream) {
  int dev = 0;
  double *scr;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (!a || !dt_out || a->nx < 4 || a->ny < 4) return fb_internal_fail(FB_ERR_ARG, "fb_cfl_dt_static: invalid mesh", 0);
  if (!a->rho || !a->cs || !a->vx || !a->vy || !a->xmin || !a->ymin)
    return fb_internal_fail(FB_ERR_ARG, "fb_cfl_dt_static: null field or mesh pointer", 0);
  const int is3d = a->nz > 1;
  if (is3d && (!a->vz || !a->zmin || (a->spherical && !a->sin_zmed)))
    return fb_internal_fail(FB_ERR_ARG, "fb_cfl_dt_static: null 3D field or mesh pointer", 0);
  const int sy = a->ny + 6;
  const long long nring = (long long)sy * (is3d ? a->nz + 6 : 1);
  if (nring > FB_NOALLOC_MAX_RINGS)
    return fb_internal_fail(FB_ERR_TOO_LARGE, "fb_cfl_dt_static: more rings than FB_NOALLOC_MAX_RINGS", 0);
  const long long pitch = a->pitch > 0 ? a->pitch : a->nx;
  const long long stride = a->stride > 0 ? a->stride : pitch * sy;
  if (pitch < a->nx || (is3d && stride < pitch * sy))
    return fb_internal_fail(FB_ERR_ARG, "fb_cfl_dt_static: pitch below Nx or stride below pitch x (Ny+6)", 0);
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return fb_internal_fail(FB_ERR_CUDA, "fb_cfl_dt_static: cudaGetDevice", (int)e);
  if (dev < 0 || dev >= FB_NOALLOC_MAX_DEVICES) return fb_internal_fail(FB_ERR_CUDA, "fb_cfl_dt_static: device index", 0);
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[dev]) {
      void *p = nullptr;
      if ((e = cudaGetSymbolAddress(&p, fb_noalloc_scratch)) != cudaSuccess || !p)
        return fb_internal_fail(FB_ERR_CUDA, "fb_cfl_dt_static: cudaGetSymbolAddress", (int)e);
      g_scratch[dev] = (double *)p;
    }
    scr = g_scratch[dev];
  }
  double *vxmed = scr;                                                  // [nring]
  unsigned long long *dtmin = (unsigned long long *)(scr + FB_NOALLOC_MAX_RINGS);
  fb::Dims m;
  m.nx = a->nx; m.ny = a->ny; m.nz = is3d ? a->nz : 1; m.sy = a->ny + 6; m.sz = is3d ? a->nz + 6 : 1;
  m.pitch = (int)pitch; m.stride = stride; m.is3d = is3d; m.sph = a->spherical;
  m.alpha = a->alpha_visc;
  m.adiab = 0; m.gam = 0.0;   // isothermal fields
  m.bclo = m.bchi = 1;
  fb::Geo<double> gd{};
  gd.xmin = a->xmin;
  k_reset_min<<<1, 1, 0, st>>>(dtmin);
  fb::k_rowsum<double, true><<<(unsigned)((nring + 31) / 32), 256, 0, st>>>(m, gd, a->vx, vxmed, a->xlen);
  dim3 grid(a->ny, is3d ? a->nz : 1);
  k_cfl_static<<<grid, 256, 0, st>>>(*a, vxmed, dtmin, pitch, stride);
  k_finish_dt<<<1, 1, 0, st>>>(dtmin, dt_out);
  // peek, not get: an error pending from the caller's own work stays theirs
  if ((e = cudaPeekAtLastError()) != cudaSuccess) return fb_internal_fail(FB_ERR_CUDA, "fb_cfl_dt_static: launch", (int)e);
  return FB_OK;
}
