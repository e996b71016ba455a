// FP32 instantiation of the stage kernels (transport and sources in FP32; the
// ring means, the shift and the potential stay FP64 inside the kernels).
#define FB_REAL double
#define FB_REAL_TR float
#define FB_STORE float
#define FB_SUF f32
#include "fb_launch.cuh"
