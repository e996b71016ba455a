// FP32 batched stage kernels: FP32 storage; the source stage computes in FP64
// (its viscous stresses in FP32), the transport stages and the CFL's per-cell
// limits in the types below (approximate single-precision division and square
// root where they compute in FP32); shift, ring means and the CFL minimum FP64.
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
#ifndef FB_TF
#define FB_TF float
#endif
extern "C" int fb_batch_launch_step_f32(fb_batch *B, double DT, int chain) {
  return launch_step<double, float, FB_TC, FB_TX, FB_TN, FB_TF>(B, DT, chain);
}
// element size of the azimuthal sweep's shared-memory rings
extern "C" size_t fb_batch_sweep_x_esz_f32(void) { return sizeof(FB_TX); }
