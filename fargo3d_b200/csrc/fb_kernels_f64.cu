// FP64 instantiation of the stage kernels.  Built with --fmad=false so that
// every product and sum rounds as the reference's CPU build does.
#define FB_REAL double
#define FB_REAL_TR double
#define FB_STORE double
#define FB_SUF f64
#include "fb_launch.cuh"

// State conversion for FP32 disks: the host's doubles cross the bus as they
// are and are rounded on the device (round to nearest even, subnormals kept:
// this file is built without flush-to-zero), the same value a host (float)
// cast gives; the way back is exact.
__global__ void k_to_f32(float *__restrict__ dst, const double *__restrict__ src, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = __double2float_rn(src[i]);
}
__global__ void k_to_f64(double *__restrict__ dst, const float *__restrict__ src, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

extern "C" int fb_launch_convert(void *dst, const void *src, size_t n, int to_f32, void *stream) {
  if (n == 0) return 0;
  size_t b = (n + 255) / 256;
  unsigned grid = (unsigned)(b < 148 * 8 ? b : 148 * 8);
  if (to_f32)
    k_to_f32<<<grid, 256, 0, (cudaStream_t)stream>>>((float *)dst, (const double *)src, n);
  else
    k_to_f64<<<grid, 256, 0, (cudaStream_t)stream>>>((double *)dst, (const float *)src, n);
  return (int)cudaGetLastError();
}

__global__ void k_convert_segs(double *__restrict__ st, const fb_segs S, int to_f32) {
  const fb_seg g = S.s[blockIdx.y];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.n; i += (long long)gridDim.x * blockDim.x) {
    if (to_f32)
      g.f[i] = __double2float_rn(g.bg ? st[g.off + i] - g.bg[i / g.nx] : st[g.off + i]);
    else
      st[g.off + i] = g.bg ? (double)g.f[i] + g.bg[i / g.nx] : (double)g.f[i];
  }
}
extern "C" int fb_launch_convert_segs(double *st, const fb_segs *segs, int to_f32, void *stream) {
  if (segs->n <= 0) return 0;
  long long mx = 0;
  for (int k = 0; k < segs->n; k++) mx = segs->s[k].n > mx ? segs->s[k].n : mx;
  const long long b = (mx + 255) / 256;
  const dim3 grid((unsigned)(b < 148 * 2 ? b : 148 * 2), (unsigned)segs->n);
  k_convert_segs<<<grid, 256, 0, (cudaStream_t)stream>>>(st, *segs, to_f32);
  return (int)cudaGetLastError();
}

// FP32 disks keep each fluid's azimuthal velocity relative to a per-ring
// background: the conversions subtract (to FP32) or add back (to FP64) the
// ring's value off[ring0 + i / nx] in double before rounding.
__global__ void k_to_f32_off(float *__restrict__ dst, const double *__restrict__ src, size_t n,
                             const double *__restrict__ off, int nx, long long ring0) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = __double2float_rn(src[i] - off[ring0 + (long long)(i / (size_t)nx)]);
}
__global__ void k_to_f64_off(double *__restrict__ dst, const float *__restrict__ src, size_t n,
                             const double *__restrict__ off, int nx, long long ring0) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i] + off[ring0 + (long long)(i / (size_t)nx)];
}

extern "C" int fb_launch_convert_off(void *dst, const void *src, size_t n, int to_f32, const double *off, int nx,
                                     long long ring0, void *stream) {
  if (n == 0) return 0;
  size_t b = (n + 255) / 256;
  unsigned grid = (unsigned)(b < 148 * 8 ? b : 148 * 8);
  if (to_f32)
    k_to_f32_off<<<grid, 256, 0, (cudaStream_t)stream>>>((float *)dst, (const double *)src, n, off, nx, ring0);
  else
    k_to_f64_off<<<grid, 256, 0, (cudaStream_t)stream>>>((double *)dst, (const float *)src, n, off, nx, ring0);
  return (int)cudaGetLastError();
}

// One warp per ring: lanes stride over the ring, then a fixed shuffle tree
// (the result depends on the ring's values only, never on the launch).
__global__ void __launch_bounds__(256) k_ring_mean(double *__restrict__ out, const double *__restrict__ src, int nx,
                                                   int nrings) {
  const int ring = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (ring >= nrings) return;
  const double *row = src + (size_t)ring * nx;
  double acc = 0.0;
  for (int i = lane; i < nx; i += 32) acc += row[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[ring] = acc / (double)nx;
}

extern "C" int fb_launch_ring_mean(double *out, const double *src, int nx, int nrings, void *stream) {
  if (nrings <= 0) return 0;
  k_ring_mean<<<(nrings + 7) / 8, 256, 0, (cudaStream_t)stream>>>(out, src, nx, nrings);
  return (int)cudaGetLastError();
}

// Neighbour differences of l(j, k) = vbg(j, k) R(j, k) along y and z (R the
// cylindrical radius: Ymed, or Ymed sin(Zmed) on spherical meshes), taken in
// double and stored in the disk's FP32 precision; 0 at the first row / layer.
// Also the background's r-phi shear of face j for the 2D sources:
// (vbg(j) - vbg(j-1)) / (Ymed(j) - Ymed(j-1)) - (vbg(j) + vbg(j-1)) / (2 Ymin(j)).
__global__ void k_bg_diffs(const double *__restrict__ vbg, const double *__restrict__ ymed,
                           const double *__restrict__ ymin, const double *__restrict__ szmed, int sy, int sz,
                           int sph, float *__restrict__ dly, float *__restrict__ dlz, float *__restrict__ shb) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= sy * sz) return;
  const int j = r % sy, k = r / sy;
  auto ell = [&](int jj, int kk) { return vbg[jj + kk * sy] * (ymed[jj] * (sph ? szmed[kk] : 1.0)); };
  const double l0 = ell(j, k);
  dly[r] = j > 0 ? (float)(l0 - ell(j - 1, k)) : 0.0f;
  dlz[r] = k > 0 ? (float)(l0 - ell(j, k - 1)) : 0.0f;
  shb[r] = j > 0 ? (float)((vbg[r] - vbg[r - 1]) / (ymed[j] - ymed[j - 1]) - 0.5 * (vbg[r] + vbg[r - 1]) / ymin[j])
                 : 0.0f;
}

extern "C" int fb_launch_bg_diffs(const fb_disk_dev *d, int fluid, void *stream) {
  const fb_fluid_dev &F = d->fl[fluid];
  if (!F.vbg || !F.dlb_y || !F.dlb_z || !F.shear_bg) return 0;
  const int n = d->sy * d->sz;
  k_bg_diffs<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
      F.vbg, (const double *)d->geomd.ymed, (const double *)d->geomd.ymin, (const double *)d->geomd.sin_zmed, d->sy,
      d->sz, d->spherical, (float *)F.dlb_y, (float *)F.dlb_z, (float *)F.shear_bg);
  return (int)cudaGetLastError();
}
