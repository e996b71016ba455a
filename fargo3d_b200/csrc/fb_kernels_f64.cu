// FP64 instantiation of the stage kernels.  Built with --fmad=false so that
// every product and sum rounds as the reference's CPU build does.
#define FB_REAL double
#define FB_REAL_TR double
#define FB_STORE double
#define FB_SUF f64
#include "fb_launch.cuh"
