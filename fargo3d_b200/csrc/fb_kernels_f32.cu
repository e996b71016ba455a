// FP32 instantiation of the stage kernels (transport and sources in FP32; the
// ring means, the shift and the potential stay FP64 inside the kernels).
#define FB_REAL float
#define FB_SUF f32
#include "fb_launch.cuh"
