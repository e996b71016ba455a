// FP32 batched stage kernels: FP32 storage; the CFL and source stages compute
// in FP64, the transport stages in the types below (approximate
// single-precision division and square root where they compute in FP32).
#include "fb_batch.cuh"
#ifndef FB_TC
#define FB_TC float
#endif
#ifndef FB_TX
#define FB_TX float
#endif
#ifndef FB_TN
#define FB_TN float
#endif
extern "C" int fb_batch_launch_step_f32(fb_batch *B, double DT) {
  return launch_step<double, float, FB_TC, FB_TX, FB_TN>(B, DT);
}
// element size of the azimuthal sweep's shared-memory rings
extern "C" size_t fb_batch_sweep_x_esz_f32(void) { return sizeof(FB_TX); }
