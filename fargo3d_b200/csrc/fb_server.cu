// fb_server.cu -- continuous-batching server of disk-planet solves.
//
// Callers submit requests (parameters, initial state in host memory, end
// time) from any thread; one worker thread owns the GPU work.  Each turn of
// the worker:
//   1. admits queued requests in arrival order while a slot is free and the
//      request's device bytes (fb_params_bytes, an upper bound) fit in what is
//      left of the HBM budget: creates the disk in a free slot of one slotted
//      batch, uploads the state, initialises it;
//   2. runs `chunk` hydro steps of every admitted disk together (one batched
//      launch per stage, replayed from a CUDA graph; fb_batch.cu);
//   3. polls the members' statuses in one copy and retires every disk that
//      reached its end time (or failed): its final state goes to host memory,
//      its slot and bytes are freed.
// A request that arrives while others run joins them at the next turn, and
// leaves as soon as it is done: the batch's membership changes every turn.
// No counterpart in the reference, which runs one disk per process.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "fargo_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

long long shape_key(int nx, int ny, int nz) { return ((long long)nx << 40) | ((long long)ny << 20) | (nz > 1 ? nz : 1); }

struct Req {
  long long id;
  fb_params p;
  double t_end;
  std::vector<double> in[5];   // rho, vx, vy, vz, cs
  std::vector<double> out[4];  // rho, vx, vy, vz
  int state = FB_REQ_QUEUED;
  int status = FB_OK;
  int slot = -1;
  size_t bytes = 0;
  double t_submit = 0, t_admit = 0, t_done = 0, phys = 0;
  long long steps = 0, cells = 0;
  size_t ncell = 0;
};

}  // namespace

struct fb_server {
  int precision, device, is3d, max_disks, chunk;
  size_t budget;
  fb_batch *B = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req *> queue;
  std::map<long long, Req *> reqs;
  std::vector<Req *> slot_req;
  std::map<long long, std::pair<int, int>> tiles;  // shape key -> (sweep_x_cells, col_segment)
  size_t reserved = 0;
  int nrunning = 0, nfinished = 0;
  long long next_id = 1;
  bool stop = false;
  int fatal = FB_OK;
  double chunks = 0, cell_updates = 0;
  Clock::time_point t0;
  std::thread worker;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void finish(Req *r, int state, int status) {  // with mu held
    r->state = state;
    r->status = status;
    r->t_done = now();
    reserved -= r->bytes;
    nfinished++;
    for (auto &v : r->in) std::vector<double>().swap(v);
    cv_done.notify_all();
  }
  void run();
};

void fb_server::run() {
  cudaSetDevice(device);
  std::vector<int> st(max_disks);
  std::vector<double> ph(max_disks);
  std::vector<long long> ns(max_disks);
  for (;;) {
    std::vector<Req *> admit;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || !queue.empty() || nrunning > 0; });
      if (stop) return;
      while (!queue.empty() && nrunning + (int)admit.size() < max_disks) {
        Req *r = queue.front();
        if (reserved + r->bytes > budget) {
          if (nrunning == 0 && admit.empty()) {  // can never fit
            queue.pop_front();
            reserved += r->bytes;
            finish(r, FB_REQ_FAILED, FB_ERR_TOO_LARGE);
            continue;
          }
          break;  // arrival order: wait for room
        }
        queue.pop_front();
        reserved += r->bytes;
        admit.push_back(r);
      }
    }
    // allocations and uploads outside the lock: submitters never wait on them
    for (Req *r : admit) {
      int slot = -1, rc;
      fb_disk *d = nullptr;
      rc = fb_batch_add(B, &r->p, r->t_end, &slot);
      if (!rc) rc = fb_batch_disk(B, slot, &d);
      if (!rc)
        rc = fb_disk_set_state(d, 0, r->in[0].data(), r->in[1].data(), r->in[2].data(),
                               r->in[3].empty() ? nullptr : r->in[3].data(), r->in[4].data());
      if (!rc) {
        std::pair<int, int> t(0, 0);
        {
          std::lock_guard<std::mutex> lk(mu);
          auto it = tiles.find(shape_key(r->p.nx, r->p.ny, r->p.nz));
          if (it != tiles.end()) t = it->second;
        }
        if (t.first || t.second) rc = fb_batch_set_tiles(B, slot, t.first, t.second);
      }
      if (!rc) rc = fb_batch_activate(B, slot);
      std::lock_guard<std::mutex> lk(mu);
      if (rc) {
        if (slot >= 0) fb_batch_remove(B, slot);
        finish(r, FB_REQ_FAILED, rc);
        continue;
      }
      r->slot = slot;
      r->state = FB_REQ_RUNNING;
      r->t_admit = now();
      slot_req[slot] = r;
      nrunning++;
      for (auto &v : r->in) std::vector<double>().swap(v);
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      if (nrunning == 0) continue;
    }
    int rc = fb_batch_run(B, chunk, 1e30);
    if (!rc) rc = fb_batch_poll(B, st.data(), ph.data(), ns.data());
    if (rc) {  // the device is unusable: fail everything
      std::lock_guard<std::mutex> lk(mu);
      fatal = rc;
      for (int s = 0; s < max_disks; s++)
        if (slot_req[s]) { finish(slot_req[s], FB_REQ_FAILED, rc); slot_req[s] = nullptr; }
      nrunning = 0;
      while (!queue.empty()) {
        reserved += queue.front()->bytes;
        finish(queue.front(), FB_REQ_FAILED, rc);
        queue.pop_front();
      }
      stop = true;
      return;
    }
    chunks += 1;
    for (int s = 0; s < max_disks; s++) {
      Req *r = slot_req[s];
      if (!r || st[s] == FB_OK) continue;
      fb_disk *d = nullptr;
      int grc = fb_batch_disk(B, s, &d);
      if (!grc) {
        for (auto &v : r->out) v.assign(r->ncell, 0.0);
        grc = fb_disk_get_state(d, 0, r->out[0].data(), r->out[1].data(), r->out[2].data(),
                                is3d ? r->out[3].data() : nullptr);
      }
      r->steps = ns[s];
      r->phys = ph[s];
      fb_batch_remove(B, s);
      std::lock_guard<std::mutex> lk(mu);
      slot_req[s] = nullptr;
      nrunning--;
      cell_updates += (double)r->steps * (double)r->cells;
      if (st[s] == FB_DONE && !grc) finish(r, FB_REQ_DONE, FB_DONE);
      else finish(r, FB_REQ_FAILED, grc ? grc : st[s]);
    }
  }
}

extern "C" {

int fb_server_create(int precision, int device, int is3d, size_t hbm_budget, int max_disks, int chunk_steps,
                     fb_server **out) {
  if (!out) return FB_ERR_ARG;
  *out = nullptr;
  if (max_disks < 1 || chunk_steps < 1) return FB_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return FB_ERR_CUDA;
  if (hbm_budget == 0) {  // default: 90 % of the device memory free now
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return FB_ERR_CUDA;
    hbm_budget = fr / 10 * 9;
  }
  fb_server *S = new fb_server();
  S->precision = precision; S->device = device; S->is3d = is3d ? 1 : 0;
  S->max_disks = max_disks; S->chunk = chunk_steps; S->budget = hbm_budget;
  S->slot_req.assign(max_disks, nullptr);
  S->t0 = Clock::now();
  int rc = fb_batch_create_slots(max_disks, precision, device, S->is3d, 1, &S->B);
  if (rc) { delete S; return rc; }
  S->worker = std::thread([S] { S->run(); });
  *out = S;
  return FB_OK;
}

int fb_server_submit(fb_server *S, const fb_params *p, const double *rho, const double *vx, const double *vy,
                     const double *vz, const double *cs, double t_end, long long *id) {
  if (!S || !p || !rho || !vx || !vy || !cs || !id || !(t_end > 0.0)) return FB_ERR_ARG;
  if ((p->nz > 1) != (S->is3d != 0) || p->nfluids != 1 || (S->is3d && !vz)) return FB_ERR_ARG;
  Req *r = new Req();
  r->p = *p;
  r->t_end = t_end;
  const size_t sy = (size_t)p->ny + 6, sz = p->nz > 1 ? (size_t)p->nz + 6 : 1;
  r->ncell = (size_t)p->nx * sy * sz;
  r->cells = (long long)p->nx * p->ny * (p->nz > 1 ? p->nz : 1);
  int rc = fb_params_bytes(p, S->precision, &r->bytes);
  if (rc) { delete r; return rc; }
  const double *src[5] = {rho, vx, vy, S->is3d ? vz : nullptr, cs};
  for (int q = 0; q < 5; q++)
    if (src[q]) r->in[q].assign(src[q], src[q] + r->ncell);
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) { delete r; return S->fatal ? S->fatal : FB_ERR_ARG; }
  r->id = S->next_id++;
  r->t_submit = S->now();
  S->reqs[r->id] = r;
  S->queue.push_back(r);
  S->cv_work.notify_one();
  *id = r->id;
  return FB_OK;
}

int fb_server_status(fb_server *S, long long id, int *state) {
  if (!S || !state) return FB_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return FB_ERR_ARG;
  *state = it->second->state;
  return FB_OK;
}

int fb_server_wait(fb_server *S, long long id, double timeout_s, int *state) {
  if (!S) return FB_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return FB_ERR_ARG;
  Req *r = it->second;
  S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                      [&] { return r->state == FB_REQ_DONE || r->state == FB_REQ_FAILED; });
  if (state) *state = r->state;
  return FB_OK;
}

int fb_server_fetch(fb_server *S, long long id, double *rho, double *vx, double *vy, double *vz, double info[8]) {
  if (!S) return FB_ERR_ARG;
  Req *r;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return FB_ERR_ARG;
    r = it->second;
    if (r->state != FB_REQ_DONE && r->state != FB_REQ_FAILED) return FB_ERR_ARG;
    S->reqs.erase(it);
    S->nfinished--;
  }
  double *dst[4] = {rho, vx, vy, vz};
  for (int q = 0; q < 4; q++)
    if (dst[q] && r->out[q].size() == r->ncell) std::copy(r->out[q].begin(), r->out[q].end(), dst[q]);
  if (info) {
    info[0] = r->t_submit; info[1] = r->t_admit; info[2] = r->t_done; info[3] = (double)r->steps;
    info[4] = r->phys; info[5] = r->status; info[6] = (double)r->bytes; info[7] = (double)r->cells;
  }
  const int ok = r->state == FB_REQ_DONE;
  const int status = r->status;
  delete r;
  return ok ? FB_OK : (status < 0 ? status : FB_ERR_ARG);
}

int fb_server_stats(fb_server *S, double *o) {
  if (!S || !o) return FB_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  o[0] = (double)S->queue.size(); o[1] = S->nrunning; o[2] = S->nfinished;
  o[3] = (double)S->reserved; o[4] = (double)S->budget; o[5] = S->chunks; o[6] = S->cell_updates;
  o[7] = S->now();
  return FB_OK;
}

double fb_server_clock(fb_server *S) { return S ? S->now() : 0.0; }

int fb_server_set_tiles(fb_server *S, int nx, int ny, int nz, int sweep_x_cells, int col_segment) {
  if (!S || nx < 1 || ny < 1) return FB_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  S->tiles[shape_key(nx, ny, nz)] = std::make_pair(sweep_x_cells, col_segment);
  return FB_OK;
}

int fb_server_destroy(fb_server *S) {
  if (!S) return FB_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_work.notify_all();
  }
  if (S->worker.joinable()) S->worker.join();
  fb_batch_destroy(S->B);
  for (auto &kv : S->reqs) delete kv.second;
  delete S;
  return FB_OK;
}

}  // extern "C"
