// FP32 batched stage kernels (approximate single-precision division and
// square root; the FP64 parts of the kernels are unaffected).
#include "fb_batch.cuh"
extern "C" int fb_batch_launch_step_f32(fb_batch *B, double DT) { return launch_step<double, float>(B, DT); }
