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
