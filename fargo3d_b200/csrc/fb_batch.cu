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
//
// Membership is by slots: a disk is added to a free slot, activated (state
// uploaded, initialised), and removed when its caller is done with it.  The
// device descriptor array and the per-disk planet systems are indexed by slot;
// the work lists (the azimuthal sweep has one per chunk width) and the graph
// depend on the active set and are rebuilt lazily at the next run.
#include "fb_batch.cuh"

#include <stdio.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <thread>

Prof *g_prof = nullptr;

extern "C" int fb_batch_launch_step_f64(fb_batch *B, double DT, int chain);
extern "C" int fb_batch_launch_step_f32(fb_batch *B, double DT, int chain);
extern "C" size_t fb_batch_sweep_x_esz_f32(void);
// fb_host.c: lend a region of one batch-wide allocation and the batch's
// stream to the next fb_disk_create on this thread
extern "C" void fb_disk_internal_provide(void *arena, size_t size, void *stream);
extern "C" size_t fb_disk_internal_arena_bytes(const fb_params *p, int precision);

static int launch_step_chain(fb_batch *B, double DT, int chain) {
  return B->precision == FB_FP64 ? fb_batch_launch_step_f64(B, DT, chain) : fb_batch_launch_step_f32(B, DT, chain);
}

// nsteps steps of every active disk.  With several chains the batch's stream
// forks into the chains' streams, each runs its disks' nsteps steps, and the
// batch's stream joins them: the chains share no data, so they need no
// ordering between one another inside the run (also when captured).
static int launch_steps(fb_batch *B, double DT, int nsteps) {
  int e = 0;
  if (B->nchains <= 1) {
    for (int s = 0; s < nsteps && !e; s++) e = launch_step_chain(B, DT, -1);
    return e;
  }
  if ((e = (int)cudaEventRecord(B->ev_fork, B->stream))) return e;
  for (int c = 0; c < B->nchains && !e; c++) {
    if (c > 0 && (e = (int)cudaStreamWaitEvent(B->cstream[c], B->ev_fork, 0))) break;
    for (int s = 0; s < nsteps && !e; s++) e = launch_step_chain(B, DT, c);
    if (!e && c > 0) {
      if ((e = (int)cudaEventRecord(B->ev_join[c], B->cstream[c]))) break;
      e = (int)cudaStreamWaitEvent(B->stream, B->ev_join[c], 0);
    }
  }
  return e;
}

static void free_lists(fb_batch *B) {
  if (B->lists) cudaFree(B->lists);
  B->lists = nullptr;
  for (int s = 0; s < ST_N; s++) {
    B->items[s] = nullptr;
    B->nitems[s] = 0;
  }
  for (int c = 0; c < FB_MAX_CHAINS; c++) {
    for (int s = 0; s < ST_N; s++) {
      B->citems[c][s] = nullptr;
      B->ncitems[c][s] = 0;
    }
    B->cdisks[c] = nullptr;
    B->ncdisks[c] = 0;
  }
}

// The work lists and chain disk lists of a rebuild, gathered on the host
// and uploaded as one allocation with one copy (a batch rebuilds them for
// every change of membership; dozens of small allocations and synchronous
// copies would cost milliseconds).
struct ListPack {
  std::vector<unsigned char> host;
  std::vector<std::pair<void **, size_t>> fix;   // pointer to set, offset in the pack
  void add(void **dst, const void *src, size_t bytes) {
    if (!bytes) { *dst = nullptr; return; }
    const size_t off = (host.size() + 15) & ~(size_t)15;
    host.resize(off + bytes);
    memcpy(host.data() + off, src, bytes);
    fix.push_back(std::make_pair(dst, off));
  }
  int upload(fb_batch *B) {
    if (host.empty()) return FB_OK;
    if (cudaMalloc(&B->lists, host.size()) != cudaSuccess) return FB_ERR_NOMEM;
    cudaError_t e = cudaMemcpy(B->lists, host.data(), host.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fb_internal_fail(FB_ERR_CUDA, "work list upload", (int)e);
    for (auto &f : fix) *f.first = (void *)((unsigned char *)B->lists + f.second);
    return FB_OK;
  }
};

// Work lists, chunk width and shared-memory size for the active set; drops
// the captured graph.
static int rebuild(fb_batch *B) {
  if (B->exec) { cudaGraphExecDestroy(B->exec); B->exec = nullptr; }
  B->graph_steps = 0;
  free_lists(B);
  std::vector<const fb_disk_dev *> act;
  for (int i = 0; i < B->n; i++)
    if (B->state[i] == 2) act.push_back(fb_disk_internal_dev(B->disks[i]));
  B->dirty = 0;
  if (act.empty()) return FB_OK;
  // per chunk-width class: the largest shared-memory need of its disks
  for (int k = 0; k < NXC; k++) B->smem_x[k] = 0;
  for (const fb_disk_dev *d : act) {
    const int c = disk_cx(*d);
    if (!valid_cx(d->nx, c)) return FB_ERR_ARG;
    int k = 0;
    while ((1 << k) < c) k++;
    // the sweep keeps its rings in its compute precision
    size_t s = sweep_x2_smem(d->nx, c, 256, B->is3d ? 6 : 4,
                             B->precision == FB_FP64 ? 8 : fb_batch_sweep_x_esz_f32());
    if (s > B->smem_x[k]) B->smem_x[k] = s;
  }
  ListPack pack;
  for (int s = 0; s < ST_N; s++) {
    std::vector<int4> v;
    B->nitems[s] = tiles(B, s, v);
    pack.add((void **)&B->items[s], v.data(), sizeof(int4) * v.size());
  }
  // the planet indices some member's disk force is needed for
  B->force_np = 0;
  for (int i = 0; i < B->n; i++) {
    if (B->state[i] != 2) continue;
    const fb_psys *S = fb_disk_internal_psys(B->disks[i]);
    for (int n = 0; n < S->np; n++)
      if (S->feeldisk[n] && n + 1 > B->force_np) B->force_np = n + 1;
  }
  // chains: the largest disks first, each to the chain with the fewest cells
  B->chain_of.assign(B->n, -1);
  if (B->nchains > 1) {
    std::vector<int> order;
    for (int i = 0; i < B->n; i++)
      if (B->state[i] == 2) order.push_back(i);
    auto cells = [&](int i) {
      const fb_disk_dev &D = *fb_disk_internal_dev(B->disks[i]);
      return (long long)D.nx * D.ny * (D.is3d ? D.nz : 1);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells(a) > cells(b); });
    long long load[FB_MAX_CHAINS] = {0};
    std::vector<int> members[FB_MAX_CHAINS];
    for (int i : order) {
      int c = 0;
      for (int k = 1; k < B->nchains; k++)
        if (load[k] < load[c]) c = k;
      B->chain_of[i] = c;
      load[c] += cells(i);
      members[c].push_back(i);
    }
    for (int c = 0; c < B->nchains; c++) {
      std::sort(members[c].begin(), members[c].end());
      B->ncdisks[c] = (int)members[c].size();
      pack.add((void **)&B->cdisks[c], members[c].data(), sizeof(int) * members[c].size());
      for (int s = 0; s < ST_N; s++) {
        std::vector<int4> v;
        B->ncitems[c][s] = tiles(B, s, v, c);
        pack.add((void **)&B->citems[c][s], v.data(), sizeof(int4) * v.size());
      }
    }
  }
  return pack.upload(B);
}

extern "C" {

int fb_batch_destroy(fb_batch *B) {
  if (!B) return FB_OK;
  cudaSetDevice(B->device);
  if (B->stream) cudaStreamSynchronize(B->stream);
  for (int c = 1; c < FB_MAX_CHAINS; c++)
    if (B->cstream[c]) cudaStreamSynchronize(B->cstream[c]);
  if (B->exec) cudaGraphExecDestroy(B->exec);
  free_lists(B);
  for (int c = 1; c < FB_MAX_CHAINS; c++) {
    if (B->cstream[c]) cudaStreamDestroy(B->cstream[c]);
    if (B->ev_join[c]) cudaEventDestroy(B->ev_join[c]);
  }
  if (B->ev_fork) cudaEventDestroy(B->ev_fork);
  if (B->h_act) cudaFreeHost(B->h_act);
  if (B->d_disks) cudaFree(B->d_disks);
  if (B->d_psys) cudaFree(B->d_psys);
  for (fb_disk *d : B->disks)
    if (d) fb_disk_destroy(d);
  if (B->arena) cudaFree(B->arena);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
  return FB_OK;
}

int fb_batch_create_slots(int capacity, int precision, int device, int is3d, int nfluids, fb_batch **out) {
  if (!out) return FB_ERR_ARG;
  *out = nullptr;
  if (capacity < 1 || nfluids < 1 || nfluids > FB_MAXFLUIDS || (precision != FB_FP64 && precision != FB_FP32))
    return FB_ERR_ARG;
  fb_batch *B = new fb_batch();
  B->n = capacity; B->precision = precision; B->device = device;
  B->is3d = is3d ? 1 : 0;
  B->nfluids = nfluids;
  B->state.assign(capacity, 0);
  B->t_end.assign(capacity, 0.0);
  B->disks.assign(capacity, nullptr);
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&B->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
    fb_batch_destroy(B);
    return FB_ERR_CUDA;
  }
  B->cstream[0] = B->stream;
  for (int c = 1; c < FB_MAX_CHAINS; c++)
    if (cudaStreamCreateWithFlags(&B->cstream[c], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&B->ev_join[c], cudaEventDisableTiming) != cudaSuccess) {
      fb_batch_destroy(B);
      return FB_ERR_CUDA;
    }
  B->nchains = precision == FB_FP32 ? FB_DEFAULT_CHAINS_F32 : FB_DEFAULT_CHAINS_F64;
  if (cudaMalloc(&B->d_disks, sizeof(fb_disk_dev) * capacity) != cudaSuccess ||
      cudaMalloc(&B->d_psys, sizeof(fb_psys) * capacity) != cudaSuccess) {
    fb_batch_destroy(B);
    return FB_ERR_NOMEM;
  }
  // zeroed descriptors mark empty slots for the scalar kernel
  cudaMemset(B->d_disks, 0, sizeof(fb_disk_dev) * capacity);
  cudaMemset(B->d_psys, 0, sizeof(fb_psys) * capacity);
  *out = B;
  return FB_OK;
}

int fb_batch_add(fb_batch *B, const fb_params *p, double t_end, int *slot) {
  if (!B || !p || !slot) return FB_ERR_ARG;
  if ((p->nz > 1) != (B->is3d != 0) || p->nfluids != B->nfluids) return FB_ERR_ARG;
  if (p->adiabatic || p->dust_diffusion)   // the batched stages have neither
    return fb_internal_fail(FB_ERR_ARG, "adiabatic disks and dust diffusion run on the one-disk path (fb_disk_step)", 0);
  int s = -1;
  for (int i = 0; i < B->n && s < 0; i++)
    if (B->state[i] == 0) s = i;
  if (s < 0) return FB_ERR_TOO_LARGE;
  fb_disk *d = nullptr;
  int rc = fb_disk_create(p, B->precision, B->device, &d);
  if (rc) return rc;
  B->disks[s] = d;
  B->state[s] = 1;
  B->t_end[s] = t_end > 0.0 ? t_end : 0.0;
  *slot = s;
  return FB_OK;
}

// Slot s's initialisation and descriptor uploads queued on the batch's stream
// (the member's own stream); the caller waits.
struct ActivationStage {   // page-locked source of one slot's activation uploads
  fb_disk_dev dd;
  fb_psys ps;
  unsigned long long init[2];
};
static int activate_async(fb_batch *B, int s) {
  fb_disk *d = B->disks[s];
  int rc = fb_disk_internal_initialize_async(d);
  if (rc) return rc;
  if (cudaSetDevice(B->device) != cudaSuccess) return FB_ERR_CUDA;
  if (!B->h_act && cudaMallocHost(&B->h_act, sizeof(ActivationStage) * B->n) != cudaSuccess) {
    B->h_act = nullptr;
    return FB_ERR_NOMEM;
  }
  // CFL minimum start and flag word; the scalars were uploaded by the
  // initialisation.  The uploads come from page-locked memory, so they are
  // queued without waiting; the batch's stream may still be running other
  // members: it orders them.
  ActivationStage *a = (ActivationStage *)B->h_act + s;
  a->init[0] = 0x4415AF1D78B58C40ULL;
  a->init[1] = 0ull;
  a->ps = *fb_disk_internal_psys(d);
  a->ps.t_end = B->t_end[s];
  a->dd = *fb_disk_internal_dev(d);
  if (cudaMemcpyAsync(a->dd.dtmin, a->init, sizeof a->init, cudaMemcpyHostToDevice, B->stream) != cudaSuccess ||
      cudaMemcpyAsync(B->d_psys + s, &a->ps, sizeof a->ps, cudaMemcpyHostToDevice, B->stream) != cudaSuccess ||
      cudaMemcpyAsync(B->d_disks + s, &a->dd, sizeof(fb_disk_dev), cudaMemcpyHostToDevice, B->stream) != cudaSuccess)
    return FB_ERR_CUDA;
  B->state[s] = 2;
  B->dirty = 1;
  return FB_OK;
}

int fb_batch_activate(fb_batch *B, int s) {
  if (!B || s < 0 || s >= B->n || B->state[s] != 1) return FB_ERR_ARG;
  int rc = activate_async(B, s);
  if (rc) return rc;
  return cudaStreamSynchronize(B->stream) == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

int fb_batch_remove(fb_batch *B, int s) {
  if (!B || s < 0 || s >= B->n || B->state[s] == 0) return FB_ERR_ARG;
  cudaSetDevice(B->device);
  if (cudaStreamSynchronize(B->stream) != cudaSuccess) return FB_ERR_CUDA;
  if (cudaMemset(B->d_disks + s, 0, sizeof(fb_disk_dev)) != cudaSuccess) return FB_ERR_CUDA;
  if (B->state[s] == 2) B->dirty = 1;
  fb_disk_destroy(B->disks[s]);
  B->disks[s] = nullptr;
  B->state[s] = 0;
  B->t_end[s] = 0.0;
  return FB_OK;
}

int fb_batch_capacity(fb_batch *B) { return B ? B->n : 0; }

int fb_batch_set_tiles(fb_batch *B, int s, int sweep_x_cells, int col_segment) {
  if (!B || s < 0 || s >= B->n || !B->disks[s]) return FB_ERR_ARG;
  int rc = fb_disk_set_tiles(B->disks[s], sweep_x_cells, col_segment);
  if (rc) return rc;
  if (B->state[s] == 2) B->dirty = 1;
  return FB_OK;
}

// All members at once (the original interface): slots 0..n-1 in order.
int fb_batch_create(const fb_params *ps, int n, int precision, int device, fb_batch **out) {
  if (!out) return FB_ERR_ARG;
  *out = nullptr;
  if (!ps || n < 1) return FB_ERR_ARG;
  fb_batch *B = nullptr;
  int rc = fb_batch_create_slots(n, precision, device, ps[0].nz > 1, ps[0].nfluids, &B);
  if (rc) return rc;
  // one zeroed allocation for every member's arena and the batch's stream
  // for all of them: creation costs one cudaMalloc + one memset in total
  std::vector<size_t> off(n + 1, 0);
  for (int i = 0; i < n; i++) off[i + 1] = off[i] + ((fb_disk_internal_arena_bytes(&ps[i], precision) + 255) & ~(size_t)255);
  if (off[n] > 0 && cudaMalloc((void **)&B->arena, off[n]) == cudaSuccess &&
      cudaMemsetAsync(B->arena, 0, off[n], B->stream) == cudaSuccess &&
      cudaStreamSynchronize(B->stream) == cudaSuccess) {
  } else {
    if (B->arena) cudaFree(B->arena);
    B->arena = nullptr;   // members allocate their own
    cudaGetLastError();
  }
  for (int i = 0; i < n; i++)   // what fb_batch_add refuses, before any member exists
    if ((ps[i].nz > 1) != (B->is3d != 0) || ps[i].nfluids != B->nfluids || ps[i].adiabatic || ps[i].dust_diffusion) {
      fb_batch_destroy(B);
      return fb_internal_fail(FB_ERR_ARG, ps[i].adiabatic || ps[i].dust_diffusion
                                              ? "adiabatic disks and dust diffusion run on the one-disk path (fb_disk_step)"
                                              : "batch members share dimensionality and fluid count", 0);
    }
  // Members are independent: their host-side set-up (mesh, libm tables, the
  // table image and its upload on the batch's stream) runs on up to 8 host
  // threads, each disk in its own region of the arena.
  std::vector<fb_disk *> made(n, nullptr);
  std::vector<int> rcs(n, 0);
  std::vector<std::string> errs(n);
  std::atomic<int> next(0);
  auto work = [&]() {
    for (int i; (i = next++) < n;) {
      if (B->arena) fb_disk_internal_provide(B->arena + off[i], off[i + 1] - off[i], B->stream);
      rcs[i] = fb_disk_create(&ps[i], precision, device, &made[i]);
      fb_disk_internal_provide(nullptr, 0, nullptr);
      if (rcs[i]) errs[i] = fb_last_error();
    }
  };
  const unsigned hw = std::thread::hardware_concurrency();
  const int nt = std::min(n, std::max(1, std::min(8, (int)(hw ? hw : 1))));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; t++) {
    try {
      pool.emplace_back(work);
    } catch (...) {   // no thread to be had: the calling thread does the rest
      break;
    }
  }
  work();
  for (auto &t : pool) t.join();
  cudaSetDevice(device);
  for (int i = 0; i < n; i++) {
    if (!rcs[i]) continue;
    for (int k = 0; k < n; k++)
      if (made[k]) fb_disk_destroy(made[k]);
    fb_batch_destroy(B);
    return fb_internal_fail(rcs[i], errs[i].c_str(), 0);
  }
  for (int i = 0; i < n; i++) {
    B->disks[i] = made[i];
    B->state[i] = 1;
    B->t_end[i] = 0.0;
  }
  // the members' table uploads, queued on the batch's stream, waited for once
  if (cudaStreamSynchronize(B->stream) != cudaSuccess) { fb_batch_destroy(B); return FB_ERR_CUDA; }
  *out = B;
  return FB_OK;
}

int fb_batch_disk(fb_batch *B, int i, fb_disk **d) {
  if (!B || !d || i < 0 || i >= B->n || !B->disks[i]) return FB_ERR_ARG;
  *d = B->disks[i];
  return FB_OK;
}

// Activate every reserved slot (the members' states set beforehand).
int fb_batch_initialize(fb_batch *B) {
  if (!B) return FB_ERR_ARG;
  for (int i = 0; i < B->n; i++) {   // every reserved member, one wait
    if (B->state[i] != 1) continue;
    int rc = activate_async(B, i);
    if (rc) return rc;
  }
  cudaSetDevice(B->device);
  return cudaStreamSynchronize(B->stream) == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// Advance every active disk by nsteps hydro steps without host round trips.
// The steps are issued through one captured CUDA graph of `chunk` steps.
int fb_batch_run(fb_batch *B, int nsteps, double DT) {
  if (!B || nsteps < 0) return FB_ERR_ARG;
  if (cudaSetDevice(B->device) != cudaSuccess) return FB_ERR_CUDA;
  if (B->dirty) {
    int rc = rebuild(B);
    if (rc) return rc;
  }
  if (B->nitems[ST_ROWSUM] == 0) return FB_OK;
  const int chunk = 10;  // steps per captured graph; a remainder runs eagerly
  if (nsteps >= chunk && (!B->exec || B->graph_steps != chunk || B->graph_dt != DT)) {
    // a run of two chunks or more takes its first chunk eagerly, so the
    // device works while the host captures and instantiates the graph of
    // the following ones (a one-chunk run, e.g. the server's, replays the
    // graph it captures)
    if (nsteps >= 2 * chunk) {
      const int e0 = launch_steps(B, DT, chunk);
      if (e0) return fb_internal_fail(FB_ERR_CUDA, "batched step launch", e0);
      nsteps -= chunk;
    }
    if (B->exec) { cudaGraphExecDestroy(B->exec); B->exec = nullptr; }
    cudaGraph_t g;
    if (cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FB_ERR_CUDA;
    const int le = launch_steps(B, DT, chunk);
    cudaError_t e = cudaStreamEndCapture(B->stream, &g);
    if (le && e == cudaSuccess) { cudaGraphDestroy(g); return fb_internal_fail(FB_ERR_CUDA, "step graph capture", le); }
    if (e != cudaSuccess) return fb_internal_fail(FB_ERR_CUDA, "step graph capture", (int)e);
    if (cudaGraphInstantiate(&B->exec, g, 0) != cudaSuccess) { cudaGraphDestroy(g); return FB_ERR_CUDA; }
    cudaGraphDestroy(g);
    B->graph_steps = chunk;
    B->graph_dt = DT;
  }
  int done = 0;
  while (done + chunk <= nsteps) {
    cudaError_t e = cudaGraphLaunch(B->exec, B->stream);
    if (e != cudaSuccess) return fb_internal_fail(FB_ERR_CUDA, "cudaGraphLaunch", (int)e);
    done += chunk;
  }
  if (done < nsteps) {
    int e = launch_steps(B, DT, nsteps - done);
    if (e) return fb_internal_fail(FB_ERR_CUDA, "batched step launch", e);
  }
  return FB_OK;
}

int fb_batch_set_chains(fb_batch *B, int chains) {
  if (!B || chains < 1 || chains > FB_MAX_CHAINS) return FB_ERR_ARG;
  if (cudaSetDevice(B->device) != cudaSuccess || cudaStreamSynchronize(B->stream) != cudaSuccess) return FB_ERR_CUDA;
  if (chains != B->nchains) {
    B->nchains = chains;
    B->dirty = 1;
  }
  return FB_OK;
}

int fb_batch_get_chains(fb_batch *B) { return B ? B->nchains : FB_ERR_ARG; }

// Fluid f's state of every member at once: arrays indexed by slot (a NULL
// array or entry skips that field or slot).  All transfers go through the
// batch's stream with one wait at the end.
static int gather(fb_batch *B, const void *const *a, std::vector<fb_disk *> &ds, std::vector<const void *> &out,
                  std::vector<int> &slots) {
  if (slots.empty())
    for (int i = 0; i < B->n; i++)
      if (B->disks[i]) slots.push_back(i);
  if (ds.empty())
    for (int i : slots) ds.push_back(B->disks[i]);
  out.clear();
  if (a)
    for (int i : slots) out.push_back(a[i]);
  return 0;
}

int fb_batch_set_states(fb_batch *B, int fluid, const double *const *rho, const double *const *vx,
                        const double *const *vy, const double *const *vz, const double *const *cs) {
  if (!B) return FB_ERR_ARG;
  std::vector<fb_disk *> ds;
  std::vector<int> slots;
  std::vector<const void *> p[5];
  const double *const *in[5] = {rho, vx, vy, vz, cs};
  for (int q = 0; q < 5; q++) gather(B, (const void *const *)in[q], ds, p[q], slots);
  if (ds.empty()) return FB_OK;
  auto arr = [&](int q) { return in[q] ? (const double *const *)p[q].data() : nullptr; };
  return fb_disks_set_state(ds.data(), (int)ds.size(), fluid, arr(0), arr(1), arr(2), arr(3), arr(4));
}

int fb_batch_get_states(fb_batch *B, int fluid, double *const *rho, double *const *vx, double *const *vy,
                        double *const *vz) {
  if (!B) return FB_ERR_ARG;
  std::vector<fb_disk *> ds;
  std::vector<int> slots;
  std::vector<const void *> p[4];
  double *const *in[4] = {rho, vx, vy, vz};
  for (int q = 0; q < 4; q++) gather(B, (const void *const *)in[q], ds, p[q], slots);
  if (ds.empty()) return FB_OK;
  auto arr = [&](int q) { return in[q] ? (double *const *)p[q].data() : nullptr; };
  return fb_disks_get_state(ds.data(), (int)ds.size(), fluid, arr(0), arr(1), arr(2), arr(3));
}

int fb_batch_sync(fb_batch *B) {
  if (!B) return FB_ERR_ARG;
  cudaSetDevice(B->device);
  return cudaStreamSynchronize(B->stream) == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// Scalars of disk i ([0] PhysicalTime [1] OMEGAFRAME [2] last dt [3..6]
// planet 0 x, y, vx, vy [7] Domega) and its status (FB_OK, FB_DONE or the
// error that froze it).
int fb_batch_get_scalars(fb_batch *B, int i, double *o, int *status) {
  if (!B || i < 0 || i >= B->n || B->state[i] != 2) return FB_ERR_ARG;
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

int fb_batch_poll(fb_batch *B, int *status, double *phys_time, long long *steps) {
  if (!B) return FB_ERR_ARG;
  cudaSetDevice(B->device);
  if (cudaStreamSynchronize(B->stream) != cudaSuccess) return FB_ERR_CUDA;
  std::vector<fb_psys> h(B->n);
  if (cudaMemcpy(h.data(), B->d_psys, sizeof(fb_psys) * B->n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return FB_ERR_CUDA;
  for (int i = 0; i < B->n; i++) {
    const bool act = B->state[i] == 2;
    if (status) status[i] = act ? h[i].status : (B->state[i] == 1 ? FB_SLOT_RESERVED : FB_SLOT_EMPTY);
    if (phys_time) phys_time[i] = act ? h[i].phys_time : 0.0;
    if (steps) steps[i] = act ? h[i].step_count : 0;
  }
  return FB_OK;
}

void *fb_batch_stream(fb_batch *B) { return B ? (void *)B->stream : nullptr; }

// One eager step of every disk with CUDA events between the launch groups;
// ms[i] is the device time of group names[i].  Returns the group count.
int fb_batch_profile_step(fb_batch *B, double DT, float *ms, const char **names, int max) {
  if (!B) return FB_ERR_ARG;
  cudaSetDevice(B->device);
  if (B->dirty) {
    int rc = rebuild(B);
    if (rc) return rc;
  }
  if (B->nitems[ST_ROWSUM] == 0) return 0;
  Prof P;
  P.n = 0;
  g_prof = &P;
  int rc = launch_step_chain(B, DT, -1);   // one chain: the launch groups in order
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
