// fb_batch.cu -- many independent disks advanced together (host side).
//
// Every stage of a hydro step runs as ONE launch over the tiles of all disks:
// the host enumerates each stage's tiles (disk, bx, by, bz) once into a work
// list, and a batched wrapper maps blockIdx.x to a tile and runs the same
// kernel body as the one-disk path on that disk's descriptor.  The scalar
// work between the CFL reduction and the sources (time step, planets, frame;
// fb_psys.h) runs on the device, one thread per disk, so a step needs no host
// round trip and whole sequences of steps are captured into one CUDA graph.
// A disk whose state goes non-finite or whose time step collapses is frozen
// (its tiles return immediately) while the others continue.  The stage
// kernels are compiled per precision (fb_batch_f64.cu, fb_batch_f32.cu).
#include "fb_batch.cuh"

Prof *g_prof = nullptr;

extern "C" int fb_batch_launch_step_f64(fb_batch *B, double DT);
extern "C" int fb_batch_launch_step_f32(fb_batch *B, double DT);
extern "C" size_t fb_batch_sweep_x_esz_f32(void);

static int launch_step_any(fb_batch *B, double DT) {
  return B->precision == FB_FP64 ? fb_batch_launch_step_f64(B, DT) : fb_batch_launch_step_f32(B, DT);
}

extern "C" {

int fb_batch_destroy(fb_batch *B) {
  if (!B) return FB_OK;
  cudaSetDevice(B->device);
  if (B->stream) cudaStreamSynchronize(B->stream);
  if (B->exec) cudaGraphExecDestroy(B->exec);
  for (int s = 0; s < ST_N; s++)
    if (B->items[s]) cudaFree(B->items[s]);
  if (B->d_disks) cudaFree(B->d_disks);
  if (B->d_psys) cudaFree(B->d_psys);
  for (fb_disk *d : B->disks) fb_disk_destroy(d);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
  return FB_OK;
}

int fb_batch_create(const fb_params *ps, int n, int precision, int device, fb_batch **out) {
  *out = nullptr;
  if (!ps || n < 1) return FB_ERR_ARG;
  fb_batch *B = new fb_batch();
  B->n = n; B->precision = precision; B->device = device;
  B->is3d = ps[0].nz > 1;
  B->nfluids = ps[0].nfluids;
  for (int i = 0; i < n; i++) {
    if ((ps[i].nz > 1) != B->is3d || ps[i].nfluids != B->nfluids) { fb_batch_destroy(B); return FB_ERR_ARG; }
    fb_disk *d = nullptr;
    int rc = fb_disk_create(&ps[i], precision, device, &d);
    if (rc) { fb_batch_destroy(B); return rc; }
    B->disks.push_back(d);
  }
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess) {
    fb_batch_destroy(B);
    return FB_ERR_CUDA;
  }
  std::vector<fb_disk_dev> hd(n);
  std::vector<fb_psys> hp(n);
  int maxnx = 0;
  for (int i = 0; i < n; i++) {
    hd[i] = *fb_disk_internal_dev(B->disks[i]);
    hp[i] = *fb_disk_internal_psys(B->disks[i]);
    if (hd[i].nx > maxnx) maxnx = hd[i].nx;
  }
  if (cudaMalloc(&B->d_disks, sizeof(fb_disk_dev) * n) != cudaSuccess ||
      cudaMalloc(&B->d_psys, sizeof(fb_psys) * n) != cudaSuccess) {
    fb_batch_destroy(B);
    return FB_ERR_NOMEM;
  }
  cudaMemcpy(B->d_disks, hd.data(), sizeof(fb_disk_dev) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(B->d_psys, hp.data(), sizeof(fb_psys) * n, cudaMemcpyHostToDevice);
  // one chunk width for the whole batch: the first of 4, 8, 16, 2, 1 that
  // every ring fits
  {
    const int cs[5] = {4, 8, 16, 2, 1};
    B->cx = 0;
    for (int t = 0; t < 5 && !B->cx; t++) {
      bool ok = true;
      for (int i = 0; i < n; i++) ok = ok && hd[i].nx % cs[t] == 0 && hd[i].nx / cs[t] <= 256;
      if (ok) B->cx = cs[t];
    }
    if (!B->cx) { fb_batch_destroy(B); return FB_ERR_ARG; }
  }
  for (int s = 0; s < ST_N; s++) {
    std::vector<int4> v;
    B->nitems[s] = tiles(B, s, v);
    if (B->nitems[s] > 0) {
      if (cudaMalloc(&B->items[s], sizeof(int4) * v.size()) != cudaSuccess) { fb_batch_destroy(B); return FB_ERR_NOMEM; }
      cudaMemcpy(B->items[s], v.data(), sizeof(int4) * v.size(), cudaMemcpyHostToDevice);
    }
  }
  B->smem_x = 0;
  (void)maxnx;
  for (int i = 0; i < n; i++) {
    /* the sweep keeps its rings in its compute precision */
    size_t s = sweep_x2_smem(hd[i].nx, B->cx, 256, B->is3d ? 6 : 4, precision == FB_FP64 ? 8 : fb_batch_sweep_x_esz_f32());
    if (s > B->smem_x) B->smem_x = s;
  }
  *out = B;
  return FB_OK;
}

int fb_batch_disk(fb_batch *B, int i, fb_disk **d) {
  if (!B || i < 0 || i >= B->n) return FB_ERR_ARG;
  *d = B->disks[i];
  return FB_OK;
}

int fb_batch_initialize(fb_batch *B) {
  if (!B) return FB_ERR_ARG;
  for (fb_disk *d : B->disks) {
    int rc = fb_disk_initialize(d);
    if (rc) return rc;
  }
  // scalars uploaded by fb_disk_initialize; start the CFL minimum and flags
  cudaSetDevice(B->device);
  for (fb_disk *d : B->disks) {
    unsigned long long init[2] = {0x4415AF1D78B58C40ULL, 0ull};
    if (cudaMemcpy(fb_disk_internal_dev(d)->dtmin, init, sizeof init, cudaMemcpyHostToDevice) != cudaSuccess)
      return FB_ERR_CUDA;
  }
  return FB_OK;
}

// Advance every disk by nsteps hydro steps without host round trips.  The
// steps are issued through one captured CUDA graph of `chunk` steps.
int fb_batch_run(fb_batch *B, int nsteps, double DT) {
  if (!B || nsteps < 0) return FB_ERR_ARG;
  if (cudaSetDevice(B->device) != cudaSuccess) return FB_ERR_CUDA;
  const int chunk = 10;  // steps per captured graph; a remainder runs eagerly
  if (nsteps >= chunk && (!B->exec || B->graph_steps != chunk || B->graph_dt != DT)) {
    if (B->exec) { cudaGraphExecDestroy(B->exec); B->exec = nullptr; }
    cudaGraph_t g;
    if (cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FB_ERR_CUDA;
    for (int s = 0; s < chunk; s++) launch_step_any(B, DT);
    if (cudaStreamEndCapture(B->stream, &g) != cudaSuccess) return FB_ERR_CUDA;
    if (cudaGraphInstantiate(&B->exec, g, 0) != cudaSuccess) { cudaGraphDestroy(g); return FB_ERR_CUDA; }
    cudaGraphDestroy(g);
    B->graph_steps = chunk;
    B->graph_dt = DT;
  }
  int done = 0;
  while (done + chunk <= nsteps) {
    if (cudaGraphLaunch(B->exec, B->stream) != cudaSuccess) return FB_ERR_CUDA;
    done += chunk;
  }
  for (; done < nsteps; done++) {
    if (launch_step_any(B, DT)) return FB_ERR_CUDA;
  }
  return FB_OK;
}

int fb_batch_sync(fb_batch *B) {
  if (!B) return FB_ERR_ARG;
  cudaSetDevice(B->device);
  return cudaStreamSynchronize(B->stream) == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// Scalars of disk i ([0] PhysicalTime [1] OMEGAFRAME [2] last dt [3..6]
// planet 0 x, y, vx, vy [7] Domega) and its status (FB_OK or the error that
// froze it).
int fb_batch_get_scalars(fb_batch *B, int i, double *o, int *status) {
  if (!B || i < 0 || i >= B->n) return FB_ERR_ARG;
  fb_psys S;
  cudaSetDevice(B->device);
  if (cudaStreamSynchronize(B->stream) != cudaSuccess) return FB_ERR_CUDA;
  if (cudaMemcpy(&S, B->d_psys + i, sizeof S, cudaMemcpyDeviceToHost) != cudaSuccess) return FB_ERR_CUDA;
  if (o) {
    o[0] = S.phys_time; o[1] = S.omegaframe; o[2] = S.last_dt;
    o[3] = S.np ? S.px[0] : 0; o[4] = S.np ? S.py[0] : 0;
    o[5] = S.np ? S.pvx[0] : 0; o[6] = S.np ? S.pvy[0] : 0; o[7] = S.domega;
  }
  if (status) *status = S.status;
  return FB_OK;
}

void *fb_batch_stream(fb_batch *B) { return B ? (void *)B->stream : nullptr; }

// One eager step of every disk with CUDA events between the launch groups;
// ms[i] is the device time of group names[i].  Returns the group count.
int fb_batch_profile_step(fb_batch *B, double DT, float *ms, const char **names, int max) {
  if (!B) return FB_ERR_ARG;
  cudaSetDevice(B->device);
  Prof P;
  P.n = 0;
  g_prof = &P;
  int rc = launch_step_any(B, DT);
  g_prof = nullptr;
  if (rc) return FB_ERR_CUDA;
  cudaEventSynchronize(P.ev[P.n - 1]);
  int k = 0;
  for (int i = 1; i < P.n && k < max; i++, k++) {
    cudaEventElapsedTime(&ms[k], P.ev[i - 1], P.ev[i]);
    names[k] = P.name[i];
  }
  for (int i = 0; i < P.n; i++) cudaEventDestroy(P.ev[i]);
  return k;
}

}  // extern "C"
