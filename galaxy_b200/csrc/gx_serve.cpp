// gx_serve.cpp -- continuous-batching server of gravity scenarios.
//
// Requests (one particle system each, with its own G, softening, theta, dt and step
// count) are submitted from any host thread. A stepping thread owned by the server
// admits waiting requests in arrival order whenever the device budget allows --
// between two batched steps, so new requests join systems already in flight -- keeps
// every admitted system's state, sort buffers and tree resident on the device
// (a gx_batch), advances all live systems together by one KDK step per iteration
// (one launch per stage for the whole mix), and retires each system when it has taken
// its steps, copying its final state back for the client. Each batched step's device
// time is recorded; the server reports p50/p99 step latency, aggregate particle-
// steps/s and per-request queueing delay.
//
// Because a batch steps each system with exactly the single-system arithmetic, a
// request's result is bit-identical whether it ran alone or in any mix.
#include <algorithm>
#include <cstdio>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime_api.h>

#include "../../include/galaxy_b200.h"
#include "gx_snapshot.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  uint64_t rid = 0;
  size_t n = 0;
  std::vector<double> pos, vel, mass;
  double g = 1, eps = 0, theta = 0.5, dt = 0;
  uint64_t steps = 0, done = 0;
  uint64_t sys = 0;
  int status = GX_REQ_QUEUED;
  Clock::time_point t_submit, t_admit, t_done;
  double time_out = 0.0;
  // snapshot emission (gx_server_submit_snapshots): one file per `snap_every` steps and
  // after the last, staged on the device and written by the server's writer thread
  uint64_t snap_every = 0;
  std::string snap_prefix;
  gx::SnapHeader snap_hdr;
  void* d_stage = nullptr;  // device staging buffer
  void* h_stage = nullptr;  // pinned copy the writer reads
  cudaEvent_t snap_ev = nullptr;
  int snap_pending = 0;  // staged but not yet written (guarded by the server mutex)
  uint64_t snaps_written = 0;
  std::string snap_err;
  bool cancel = false;  // leave the batch at the next step boundary
};

struct SnapJob {
  Req* r;
  uint64_t step;
  double time;
  size_t n;
};

void free_snap(Req* r) {
  if (r->d_stage) cudaFree(r->d_stage);
  if (r->h_stage) cudaFreeHost(r->h_stage);
  if (r->snap_ev) cudaEventDestroy(r->snap_ev);
  r->d_stage = r->h_stage = nullptr;
  r->snap_ev = nullptr;
}

double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

double percentile(std::vector<float> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double idx = p / 100.0 * (v.size() - 1);
  const size_t lo = static_cast<size_t>(idx);
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (idx - lo) * (v[hi] - v[lo]);
}

}  // namespace

struct gx_server {
  gx_batch* batch = nullptr;
  std::mutex mu;
  std::condition_variable cv, cv_done;
  std::thread th;
  bool stop = false, started = false;
  std::deque<Req*> queue;
  std::vector<Req*> live;
  std::unordered_map<uint64_t, Req*> all;
  uint64_t next_rid = 1;
  std::string err;
  int loop_error = GX_OK;
  // statistics (guarded by mu)
  std::vector<float> step_ms;
  std::vector<float> queue_s;
  uint64_t particle_steps = 0, steps = 0, completed = 0, max_live = 0;
  double busy_s = 0.0;
  Clock::time_point t_start;
  // snapshot emission
  int device = 0;
  cudaStream_t copy_stream = nullptr;
  std::thread writer;
  std::deque<SnapJob> jobs;
  std::condition_variable cv_jobs;
  bool writer_stop = false, writer_started = false;
  // metrics stream (gx_server_set_metrics_log), written by the stepping thread
  FILE* metrics = nullptr;
};

namespace {

// Writes staged snapshots as their copies complete (FIFO), outside the server mutex.
void writer_loop(gx_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    SnapJob j{};
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_jobs.wait(lk, [&] { return s->writer_stop || !s->jobs.empty(); });
      if (s->jobs.empty()) return;
      j = s->jobs.front();
      s->jobs.pop_front();
    }
    const cudaError_t e = cudaEventSynchronize(j.r->snap_ev);
    gx::SnapHeader h = j.r->snap_hdr;
    h.time = j.time;
    h.step = j.step;
    char suffix[48];
    std::snprintf(suffix, sizeof suffix, ".%08llu.glxysnap", static_cast<unsigned long long>(j.step));
    std::string err = e == cudaSuccess ? "" : cudaGetErrorString(e);
    const bool ok = e == cudaSuccess && gx::write_glxysnap_staged(j.r->snap_prefix + suffix, h, j.n, j.r->h_stage, err);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      j.r->snap_pending -= 1;
      if (ok)
        j.r->snaps_written += 1;
      else
        j.r->snap_err = err;
    }
    s->cv_done.notify_all();
  }
}

// Stage request r's snapshot at its current step (called by the stepping thread with
// the server mutex held in lk).
void stage_snapshot(gx_server* s, Req* r, std::unique_lock<std::mutex>& lk) {
  if (!r->d_stage) {
    const size_t bytes = gx::snapshot_stage_bytes(r->n);
    if (cudaMalloc(&r->d_stage, bytes) != cudaSuccess || cudaHostAlloc(&r->h_stage, bytes, 0) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->snap_ev, cudaEventDisableTiming) != cudaSuccess) {
      free_snap(r);
      r->snap_err = "cannot allocate the snapshot buffers";
      r->snap_every = 0;
      return;
    }
  }
  // the previous snapshot of r must be written before its buffer is reused
  s->cv_done.wait(lk, [&] { return r->snap_pending == 0; });
  double t = 0.0;
  size_t n = 0;
  const int rc = gx::batch_stage_snapshot(s->batch, r->sys, r->d_stage, r->h_stage, s->copy_stream, r->snap_ev, &t, &n);
  if (rc != GX_OK) {
    r->snap_err = gx_batch_last_error(s->batch);
    return;
  }
  r->snap_pending += 1;
  s->jobs.push_back(SnapJob{r, r->done, t, n});
  s->cv_jobs.notify_one();
}

void run_loop(gx_server* s) {
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      // Admit waiting requests in arrival order while the budget allows.
      while (!s->queue.empty()) {
        Req* r = s->queue.front();
        uint64_t sid = 0;
        const int rc = gx_system_add(s->batch, r->n, r->pos.data(), r->vel.data(), r->mass.data(), r->g, r->eps,
                                     r->theta, r->dt, &sid);
        if (rc == GX_ERR_BUDGET) {
          if (s->live.empty()) {  // can never fit: reject rather than wait forever
            r->status = GX_REQ_REJECTED;
            s->queue.pop_front();
            s->cv_done.notify_all();
            continue;
          }
          break;
        }
        s->queue.pop_front();
        if (rc != GX_OK) {
          r->status = GX_REQ_REJECTED;
          s->err = gx_batch_last_error(s->batch);
          s->cv_done.notify_all();
          continue;
        }
        r->sys = sid;
        r->status = GX_REQ_RUNNING;
        r->t_admit = Clock::now();
        s->queue_s.push_back(static_cast<float>(seconds(r->t_submit, r->t_admit)));
        // Owned by the batch now: release the host copy of the initial state.
        std::vector<double>().swap(r->vel);
        s->live.push_back(r);
      }
      s->max_live = std::max<uint64_t>(s->max_live, s->live.size());
      if (s->live.empty()) {
        if (s->stop) return;
        s->cv.wait(lk, [&] { return s->stop || !s->queue.empty(); });
        continue;
      }
    }
    // One batched step of every live system (outside the lock: submissions proceed).
    const auto t0 = Clock::now();
    const int rc = gx_batch_step(s->batch, 1);
    const auto t1 = Clock::now();
    gx_batch_stats bs{};
    gx_batch_stats_get(s->batch, &bs);
    std::unique_lock<std::mutex> lk(s->mu);
    if (rc != GX_OK) {
      s->loop_error = rc;
      s->err = gx_batch_last_error(s->batch);
      for (Req* r : s->live) r->status = GX_REQ_REJECTED;
      s->live.clear();
      s->cv_done.notify_all();
      continue;
    }
    s->step_ms.push_back(bs.ms_last_step);
    s->busy_s += seconds(t0, t1);
    s->steps += 1;
    std::vector<Req*> keep;
    uint64_t step_particles = 0;
    const size_t stepped = s->live.size();  // systems this step advanced
    for (Req* r : s->live) {
      if (r->cancel) {  // cancelled while running: leave the batch, no result
        gx_system_remove(s->batch, r->sys);
        r->status = GX_REQ_CANCELLED;
        r->t_done = Clock::now();
        continue;
      }
      s->particle_steps += r->n;
      step_particles += r->n;
      ++r->done;
      if (r->snap_every && (r->done % r->snap_every == 0 || r->done == r->steps)) stage_snapshot(s, r, lk);
      if (r->done < r->steps) {
        keep.push_back(r);
        continue;
      }
      r->pos.resize(3 * r->n);
      r->vel.resize(3 * r->n);
      const int src = gx_system_snapshot(s->batch, r->sys, r->pos.data(), r->vel.data(), &r->time_out);
      gx_system_remove(s->batch, r->sys);
      r->status = src == GX_OK ? GX_REQ_DONE : GX_REQ_REJECTED;
      r->t_done = Clock::now();
      s->completed += 1;
    }
    s->live.swap(keep);
    if (s->metrics) {
      std::fprintf(s->metrics,
                   "{\"step\": %llu, \"ms\": %.6f, \"live\": %zu, \"particles\": %llu, \"queued\": %zu, "
                   "\"completed\": %llu, \"bytes_in_use\": %llu}\n",
                   static_cast<unsigned long long>(s->steps), static_cast<double>(bs.ms_last_step), stepped,
                   static_cast<unsigned long long>(step_particles), s->queue.size(),
                   static_cast<unsigned long long>(s->completed), static_cast<unsigned long long>(bs.bytes_in_use));
      std::fflush(s->metrics);
    }
    s->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

int gx_server_create(size_t budget_bytes, const gx_options* opt, gx_server** out) {
  if (!out) return GX_ERR_INVALID_ARG;
  *out = nullptr;
  gx_batch* b = nullptr;
  const int rc = gx_batch_create(budget_bytes, opt, &b);
  if (rc != GX_OK) return rc;
  gx_server* s = new gx_server();
  s->batch = b;
  s->t_start = Clock::now();
  cudaGetDevice(&s->device);
  if (cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    gx_batch_destroy(b);
    delete s;
    return GX_ERR_CUDA;
  }
  s->writer = std::thread(writer_loop, s);
  s->writer_started = true;
  s->th = std::thread(run_loop, s);
  s->started = true;
  *out = s;
  return GX_OK;
}

void gx_server_destroy(gx_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (Req* r : s->queue) r->status = GX_REQ_REJECTED;
    s->queue.clear();
    for (Req* r : s->live) r->status = GX_REQ_REJECTED;
    s->live.clear();
  }
  s->cv.notify_all();
  if (s->started) s->th.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->writer_stop = true;  // the writer drains the staged snapshots first
  }
  s->cv_jobs.notify_all();
  if (s->writer_started) s->writer.join();
  gx_batch_destroy(s->batch);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  if (s->metrics) std::fclose(s->metrics);
  for (auto& kv : s->all) {
    free_snap(kv.second);
    delete kv.second;
  }
  delete s;
}

const char* gx_server_last_error(const gx_server* s) { return s ? s->err.c_str() : ""; }

int gx_server_submit(gx_server* s, size_t n, const double* pos, const double* vel, const double* mass, double g,
                     double softening, double theta, double dt, uint64_t steps, uint64_t* rid_out) {
  return gx_server_submit_snapshots(s, n, pos, vel, mass, g, softening, theta, dt, steps, nullptr, rid_out);
}

int gx_server_submit_snapshots(gx_server* s, size_t n, const double* pos, const double* vel, const double* mass,
                               double g, double softening, double theta, double dt, uint64_t steps,
                               const gx_snap_opts* snap, uint64_t* rid_out) {
  if (!s || !rid_out || n == 0 || !pos || !vel || !mass || steps == 0) return GX_ERR_INVALID_ARG;
  Req* r = new Req();
  r->n = n;
  r->pos.assign(pos, pos + 3 * n);
  r->vel.assign(vel, vel + 3 * n);
  r->mass.assign(mass, mass + n);
  r->g = g;
  r->eps = softening;
  r->theta = theta;
  r->dt = dt;
  r->steps = steps;
  r->t_submit = Clock::now();
  if (snap && snap->struct_size && snap->every) {
    if (snap->struct_size < sizeof(gx_snap_opts) || !snap->path_prefix) {
      delete r;
      return GX_ERR_INVALID_ARG;
    }
    r->snap_every = snap->every;
    r->snap_prefix = snap->path_prefix;
    r->snap_hdr.softening = softening;
    r->snap_hdr.rng_seed = snap->rng_seed;
    r->snap_hdr.config_hash = snap->config_hash;
    if (snap->units) r->snap_hdr.units = snap->units;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;
      return GX_ERR_STATE;
    }
    r->rid = s->next_rid++;
    s->all[r->rid] = r;
    s->queue.push_back(r);
    *rid_out = r->rid;
  }
  s->cv.notify_all();
  return GX_OK;
}

int gx_server_cancel(gx_server* s, uint64_t rid) {
  if (!s) return GX_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(rid);
    if (it == s->all.end()) return GX_ERR_NOT_FOUND;
    Req* r = it->second;
    if (r->status == GX_REQ_QUEUED) {
      s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
      r->status = GX_REQ_CANCELLED;
      r->t_done = Clock::now();
    } else if (r->status == GX_REQ_RUNNING) {
      r->cancel = true;
    } else {
      return GX_ERR_STATE;
    }
  }
  s->cv_done.notify_all();
  return GX_OK;
}

int gx_server_set_metrics_log(gx_server* s, const char* path) {
  if (!s) return GX_ERR_INVALID_ARG;
  FILE* f = nullptr;
  if (path) {
    f = std::fopen(path, "a");
    if (!f) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->err = std::string("cannot open ") + path;
      return GX_ERR_INVALID_ARG;
    }
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->metrics) std::fclose(s->metrics);
  s->metrics = f;
  return GX_OK;
}

int gx_server_snapshots_written(gx_server* s, uint64_t rid, uint64_t* written_out) {
  if (!s || !written_out) return GX_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(rid);
  if (it == s->all.end()) return GX_ERR_NOT_FOUND;
  *written_out = it->second->snaps_written;
  if (!it->second->snap_err.empty()) {
    s->err = it->second->snap_err;
    return GX_ERR_STATE;
  }
  return GX_OK;
}

int gx_server_status(gx_server* s, uint64_t rid, int* status_out, uint64_t* steps_done) {
  if (!s || !status_out) return GX_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(rid);
  if (it == s->all.end()) return GX_ERR_NOT_FOUND;
  *status_out = it->second->status;
  if (steps_done) *steps_done = it->second->done;
  return GX_OK;
}

int gx_server_wait(gx_server* s, uint64_t rid, double timeout_s) {
  if (!s) return GX_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(rid);
  if (it == s->all.end()) return GX_ERR_NOT_FOUND;
  Req* r = it->second;
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    return (r->status == GX_REQ_DONE || r->status == GX_REQ_REJECTED || r->status == GX_REQ_CANCELLED) &&
           r->snap_pending == 0;
  });
  if (!ok) return GX_ERR_STATE;
  if (r->status == GX_REQ_CANCELLED) return GX_ERR_CANCELLED;
  return r->status == GX_REQ_DONE ? GX_OK : GX_ERR_BUDGET;
}

int gx_server_result(gx_server* s, uint64_t rid, double* pos_out, double* vel_out, double* time_out) {
  if (!s) return GX_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(rid);
  if (it == s->all.end()) return GX_ERR_NOT_FOUND;
  Req* r = it->second;
  if (r->status != GX_REQ_DONE) return GX_ERR_STATE;
  if (pos_out) memcpy(pos_out, r->pos.data(), 3 * r->n * sizeof(double));
  if (vel_out) memcpy(vel_out, r->vel.data(), 3 * r->n * sizeof(double));
  if (time_out) *time_out = r->time_out;
  return GX_OK;
}

int gx_server_release(gx_server* s, uint64_t rid) {
  if (!s) return GX_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(rid);
  if (it == s->all.end()) return GX_ERR_NOT_FOUND;
  const int st = it->second->status;
  if (st != GX_REQ_DONE && st != GX_REQ_REJECTED && st != GX_REQ_CANCELLED) return GX_ERR_STATE;
  if (it->second->snap_pending > 0) return GX_ERR_STATE;  // a snapshot is still being written
  free_snap(it->second);
  delete it->second;
  s->all.erase(it);
  return GX_OK;
}

int gx_server_stats_get(gx_server* s, gx_server_stats* out) {
  if (!s || !out) return GX_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof(*out));
  out->steps = s->steps;
  out->particle_steps = s->particle_steps;
  out->completed = s->completed;
  out->queued = s->queue.size();
  out->live = s->live.size();
  out->max_live = s->max_live;
  out->busy_s = s->busy_s;
  out->wall_s = seconds(s->t_start, Clock::now());
  out->step_ms_p50 = percentile(s->step_ms, 50.0);
  out->step_ms_p99 = percentile(s->step_ms, 99.0);
  out->step_ms_mean = 0.0;
  double device_s = 0.0;
  for (float v : s->step_ms) device_s += v / 1e3;
  out->step_ms_mean = s->step_ms.empty() ? 0.0 : device_s * 1e3 / s->step_ms.size();
  out->particle_steps_per_s_device = device_s > 0 ? s->particle_steps / device_s : 0.0;
  out->queue_s_p50 = percentile(s->queue_s, 50.0);
  out->queue_s_p99 = percentile(s->queue_s, 99.0);
  gx_batch_stats bs{};
  gx_batch_stats_get(s->batch, &bs);
  out->bytes_in_use = bs.bytes_in_use;
  return GX_OK;
}

}  // extern "C"
