// FP64 batched stage kernels, built with --fmad=false like fb_kernels_f64.cu.
#include "fb_batch.cuh"
extern "C" int fb_batch_launch_step_f64(fb_batch *B, double DT, int chain) {
  return launch_step<double, double>(B, DT, chain);
}
