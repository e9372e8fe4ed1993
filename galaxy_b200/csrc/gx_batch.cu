// gx_batch.cu -- many independent systems stepped together: every stage is one launch
// over all systems (tiles never straddle systems; each system has its own bounding
// cube, digit histograms, look-back chain, tree and walk items), the tree walk is a
// persistent kernel whose warps steal (system, 32-target) items largest system
// first, and a steady-state step is replayed as one CUDA graph.
//
// The per-system arithmetic is exactly the single-system path's (tie-breaks use
// positions local to the system), so a system's trajectory is bit-identical whether
// it is stepped alone or inside any mix.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/galaxy_b200.h"
#include "gx_kernels.h"
#include "gx_runtime.h"
#include "gx_snapshot.h"

using namespace gx;

namespace {

struct BatchSys {
  uint64_t id;
  uint32_t off, n;
  double g, eps, theta, dt, time;
  bool pending;
  uint64_t steps;
};

}  // namespace

struct gx_batch {
  gx_options opt{};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::string err;
  size_t budget = 0;
  Arena ar;
  std::vector<BatchSys> systems;
  uint64_t next_id = 1;
  uint32_t total = 0;
  bool tables_dirty = true;
  bool use_graph = true;
  cudaGraphExec_t graph = nullptr;
  float ms_last = 0.f;
  uint64_t steps_total = 0;
};

namespace {

int bfail(gx_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  return code;
}

#define GB_CK(bt, call)                                                                  \
  do {                                                                                   \
    cudaError_t _e = (call);                                                             \
    if (_e != cudaSuccess)                                                               \
      return bfail((bt), GX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

WalkCfg bcfg(const gx_batch* bt, bool inside) {
  WalkCfg c;
  c.precision = bt->opt.precision == GX_PREC_F64 ? 1 : 0;
  c.quad = (bt->opt.multipole == GX_MULTIPOLE_QUAD && c.precision == 0) ? 1 : 0;
  c.kahan = (bt->opt.flags & GX_FLAG_NO_KAHAN) ? 0 : 1;
  c.stats = (bt->opt.flags & GX_FLAG_STATS) ? 1 : 0;
  c.inside_test = inside ? 1 : 0;
  c.block = bt->opt.walk_block ? static_cast<int>(bt->opt.walk_block) : kWalkThreads;
  gx_tuning t;
  if (!bt->opt.walk_block && !bt->opt.walk_ctas_per_sm && tuned_lookup(bt->device, bt->opt, 1, bt->total, &t)) {
    c.block = static_cast<int>(t.walk_block);
    c.persistent_ctas = bt->sm_count * static_cast<int>(t.walk_ctas_per_sm);
    return c;
  }
  c.persistent_ctas = bt->sm_count * (bt->opt.walk_ctas_per_sm ? static_cast<int>(bt->opt.walk_ctas_per_sm)
                                                               : walk_resident_ctas(c));
  return c;
}

void drop_graph(gx_batch* bt) {
  if (bt->graph) {
    cudaGraphExecDestroy(bt->graph);
    bt->graph = nullptr;
  }
}

// Upload tables for the listed systems (indices into bt->systems); sets b counts.
int upload_tables(gx_batch* bt, const std::vector<size_t>& which, bool* inside) {
  std::vector<SysDesc> in, sys;
  std::vector<TileDesc> tiles;
  std::vector<WalkItem> items;
  *inside = false;
  for (size_t w : which) {
    const BatchSys& s = bt->systems[w];
    SysDesc d{};
    d.off = s.off;
    d.n = s.n;
    d.g = s.g;
    d.eps = s.eps;
    d.theta = s.theta;
    d.dt = s.dt;
    d.flags = s.pending ? kSysPendingKick : 0u;
    // the grouping the system would have alone, so its result equals the alone result
    d.group = system_walk_group(bt->device, bt->opt, s.n);
    in.push_back(d);
    *inside = *inside || s.theta >= 0.57;
  }
  make_tables(in, sys, tiles, items);
  // Largest systems' items first, so stealing warps finish together.
  std::stable_sort(items.begin(), items.end(),
                   [&](const WalkItem& a, const WalkItem& b) { return sys[a.sys].n > sys[b.sys].n; });
  StepBufs& b = bt->ar.b;
  b.n = bt->total;
  b.key64 = (bt->opt.flags & GX_FLAG_MORTON63) ? 1 : 0;
  // one digit width for the whole batch (the sort is exact: any width gives every system
  // its own permutation)
  b.radix_bits = (!b.key64 && bt->opt.radix_bits == kRadixBitsWide) ? kRadixBitsWide : kRadixBits;
  b.nsys = static_cast<uint32_t>(sys.size());
  b.ntiles = static_cast<uint32_t>(tiles.size());
  b.nitems = static_cast<uint32_t>(items.size());
  b.zero_bytes = reinterpret_cast<char*>(b.counters) - reinterpret_cast<char*>(b.zero_begin) + kCounterWords * sizeof(uint32_t);
  GB_CK(bt, cudaMemcpyAsync(bt->ar.sys_rw, sys.data(), sys.size() * sizeof(SysDesc), cudaMemcpyHostToDevice,
                            bt->stream));
  GB_CK(bt, cudaMemcpyAsync(bt->ar.tiles_rw, tiles.data(), tiles.size() * sizeof(TileDesc), cudaMemcpyHostToDevice,
                            bt->stream));
  GB_CK(bt, cudaMemcpyAsync(bt->ar.items_rw, items.data(), items.size() * sizeof(WalkItem), cudaMemcpyHostToDevice,
                            bt->stream));
  return cudaStreamSynchronize(bt->stream) == cudaSuccess ? GX_OK : bfail(bt, GX_ERR_CUDA, "table upload");
}

void enqueue_step(gx_batch* bt, int kick, bool inside) {
  NvtxRange r("gx.batch_step");
  const StepBufs& b = bt->ar.b;
  cudaStream_t st = bt->stream;
  cudaMemsetAsync(b.zero_begin, 0, b.zero_bytes, st);
  launch_kick_drift_bbox(b, kick, 0, st);
  launch_morton_hist(b, nullptr, st);
  launch_sort(b, st);
  const int quad = bt->opt.multipole == GX_MULTIPOLE_QUAD && bt->opt.precision != GX_PREC_F64;
  launch_build(b, quad, bt->opt.precision == GX_PREC_F64, st);
  launch_walk(b, bcfg(bt, inside), st);
}

int bfinish(gx_batch* bt) {
  GB_CK(bt, cudaStreamSynchronize(bt->stream));
  GB_CK(bt, cudaGetLastError());
  DevCtl ctl;
  GB_CK(bt, cudaMemcpy(&ctl, bt->ar.b.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost));
  if (ctl.err) {
    cudaMemset(bt->ar.b.slots, 0xFF, bt->ar.cap_n * sizeof(unsigned long long));
    cudaMemset(bt->ar.b.ctl, 0, sizeof(DevCtl));
    return bfail(bt, GX_ERR_DEVICE_CHECK, "device check tripped (error word " + std::to_string(ctl.err) + ")");
  }
  return GX_OK;
}

// Grow the arena to hold `n_total` particles in `nsys` systems, keeping the state of
// the systems already resident.
int grow(gx_batch* bt, size_t n_total, size_t nsys) {
  const size_t tiles = n_total / kTile + nsys + 1;
  const size_t items = n_total / 8 + nsys + 1;  // systems' walk items of 8 targets at the narrowest
  Arena& ar = bt->ar;
  const int quad = bt->opt.multipole == GX_MULTIPOLE_QUAD;
  const int f64 = bt->opt.precision == GX_PREC_F64;
  if (n_total <= ar.cap_n && tiles <= ar.cap_tiles && items <= ar.cap_items && nsys <= ar.cap_sys) return GX_OK;
  drop_graph(bt);
  double* tmp = nullptr;
  const size_t keep = bt->total;
  if (keep) {
    GB_CK(bt, cudaMalloc(&tmp, 10 * keep * sizeof(double)));
    GB_CK(bt, cudaMemcpyAsync(tmp, ar.b.pos, 3 * keep * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(tmp + 3 * keep, ar.b.vel, 3 * keep * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(tmp + 6 * keep, ar.b.acc, 3 * keep * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(tmp + 9 * keep, ar.mass_rw, keep * 8, cudaMemcpyDeviceToDevice, bt->stream));
  }
  cudaError_t e = ar.ensure(n_total, tiles, items, nsys, quad, f64, bt->stream);
  if (e != cudaSuccess) {
    if (tmp) cudaFree(tmp);
    return bfail(bt, GX_ERR_CUDA, std::string("arena: ") + cudaGetErrorString(e));
  }
  if (keep) {
    GB_CK(bt, cudaMemcpyAsync(ar.b.pos, tmp, 3 * keep * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(ar.b.vel, tmp + 3 * keep, 3 * keep * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(ar.b.acc, tmp + 6 * keep, 3 * keep * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(ar.mass_rw, tmp + 9 * keep, keep * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaStreamSynchronize(bt->stream));
    cudaFree(tmp);
  }
  bt->tables_dirty = true;
  return GX_OK;
}

size_t index_of(const gx_batch* bt, uint64_t id) {
  for (size_t i = 0; i < bt->systems.size(); ++i)
    if (bt->systems[i].id == id) return i;
  return SIZE_MAX;
}

}  // namespace

namespace gx {

namespace {

// One system's snapshot columns: pos, vel (+ the owed closing half kick v + a (0.5 dt),
// one rounding each, as gx_system_snapshot), mass as f32 (round to nearest).
__global__ void k_stage_snapshot(uint32_t off, uint32_t n, const double* __restrict__ pos,
                                 const double* __restrict__ vel, const double* __restrict__ acc,
                                 const double* __restrict__ mass, int pending, double dt, double* __restrict__ out) {
  const double h = dmul(0.5, dt);
  double* o_pos = out;
  double* o_vel = out + 3 * (size_t)n;
  float* o_mass = reinterpret_cast<float*>(out + 6 * (size_t)n);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const size_t g = (size_t)off + i;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o_pos[3 * (size_t)i + c] = pos[3 * g + c];
      double v = vel[3 * g + c];
      if (pending) v = dadd(v, dmul(acc[3 * g + c], h));
      o_vel[3 * (size_t)i + c] = v;
    }
    o_mass[i] = __double2float_rn(mass[g]);
  }
}

}  // namespace

int batch_stage_snapshot(gx_batch* bt, uint64_t id, void* d_stage, void* host_dst, cudaStream_t copy_stream,
                         cudaEvent_t copied, double* time_out, size_t* n_out) {
  if (!bt || !d_stage || !host_dst) return GX_ERR_INVALID_ARG;
  const size_t i = index_of(bt, id);
  if (i == SIZE_MAX) return bfail(bt, GX_ERR_NOT_FOUND, "unknown system id");
  cudaSetDevice(bt->device);
  const BatchSys& s = bt->systems[i];
  const StepBufs& b = bt->ar.b;
  const uint32_t grid = std::max(1u, std::min((s.n + 255u) / 256u, 148u * 8u));
  k_stage_snapshot<<<grid, 256, 0, bt->stream>>>(s.off, s.n, b.pos, b.vel, b.acc, b.mass, s.pending ? 1 : 0, s.dt,
                                                 static_cast<double*>(d_stage));
  GB_CK(bt, cudaGetLastError());
  cudaEvent_t staged = nullptr;
  GB_CK(bt, cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(staged, bt->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(copy_stream, staged, 0);
  cudaEventDestroy(staged);  // released once the recorded work completes
  GB_CK(bt, e);
  GB_CK(bt, cudaMemcpyAsync(host_dst, d_stage, snapshot_stage_bytes(s.n), cudaMemcpyDeviceToHost, copy_stream));
  GB_CK(bt, cudaEventRecord(copied, copy_stream));
  if (time_out) *time_out = s.time;
  if (n_out) *n_out = s.n;
  return GX_OK;
}

}  // namespace gx

extern "C" {

int gx_batch_create(size_t budget_bytes, const gx_options* opt, gx_batch** out) {
  if (!out) return GX_ERR_INVALID_ARG;
  *out = nullptr;
  gx_options o{};
  o.device = -1;
  if (opt && opt->struct_size) {
    if (opt->struct_size < sizeof(gx_options)) return GX_ERR_INVALID_ARG;
    o = *opt;
  }
  if (!options_valid(o)) {
    set_global_err("invalid gx_options");
    return GX_ERR_INVALID_ARG;
  }
  std::string err;
  if (!check_device(o.device, err)) {
    set_global_err(err);
    return GX_ERR_NO_DEVICE;
  }
  gx_batch* bt = new gx_batch();
  bt->opt = o;
  bt->budget = budget_bytes;
  int dev = o.device;
  if (dev < 0) cudaGetDevice(&dev);
  bt->device = dev;
  cudaSetDevice(dev);
  prepare_device(dev);
  cudaDeviceGetAttribute(&bt->sm_count, cudaDevAttrMultiProcessorCount, dev);
  if (cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&bt->e0) != cudaSuccess || cudaEventCreate(&bt->e1) != cudaSuccess) {
    set_global_err("stream/event creation failed");
    delete bt;
    return GX_ERR_CUDA;
  }
  *out = bt;
  return GX_OK;
}

void gx_batch_destroy(gx_batch* bt) {
  if (!bt) return;
  cudaSetDevice(bt->device);
  if (bt->stream) cudaStreamSynchronize(bt->stream);
  drop_graph(bt);
  bt->ar.release();
  if (bt->e0) cudaEventDestroy(bt->e0);
  if (bt->e1) cudaEventDestroy(bt->e1);
  if (bt->stream) cudaStreamDestroy(bt->stream);
  delete bt;
}

const char* gx_batch_last_error(const gx_batch* bt) { return bt ? bt->err.c_str() : global_err(); }

int gx_system_bytes(const gx_batch* bt, size_t n, size_t* bytes_out) {
  if (!bt || !bytes_out) return GX_ERR_INVALID_ARG;
  const int quad = bt->opt.multipole == GX_MULTIPOLE_QUAD;
  const int f64 = bt->opt.precision == GX_PREC_F64;
  *bytes_out = Arena::bytes_for(bt->total + n, bt->systems.size() + 1, quad, f64) -
               (bt->total ? Arena::bytes_for(bt->total, bt->systems.size(), quad, f64) : 0);
  return GX_OK;
}

int gx_system_add(gx_batch* bt, size_t n, const double* pos, const double* vel, const double* mass, double g,
                  double softening, double theta, double dt, uint64_t* id_out) {
  if (!bt || !id_out) return GX_ERR_INVALID_ARG;
  if (n == 0 || !pos || !vel || !mass) return bfail(bt, GX_ERR_INVALID_ARG, "empty system or null array");
  if (!(softening >= 0.0) || !(theta >= 0.0) || !(dt == dt)) return bfail(bt, GX_ERR_INVALID_ARG, "bad parameters");
  if (static_cast<size_t>(bt->total) + n > (1u << 30)) return bfail(bt, GX_ERR_CAPACITY, "batch above 2^30 particles");
  cudaSetDevice(bt->device);
  const int quad = bt->opt.multipole == GX_MULTIPOLE_QUAD;
  const int f64 = bt->opt.precision == GX_PREC_F64;
  const size_t need = Arena::bytes_for(bt->total + n, bt->systems.size() + 1, quad, f64);
  if (bt->budget && need > bt->budget) return bfail(bt, GX_ERR_BUDGET, "system does not fit the device budget");
  int rc = grow(bt, bt->total + n, bt->systems.size() + 1);
  if (rc) return rc;
  StepBufs& b = bt->ar.b;
  const size_t off = bt->total;
  GB_CK(bt, cudaMemcpyAsync(b.pos + 3 * off, pos, 3 * n * 8, cudaMemcpyHostToDevice, bt->stream));
  GB_CK(bt, cudaMemcpyAsync(b.vel + 3 * off, vel, 3 * n * 8, cudaMemcpyHostToDevice, bt->stream));
  GB_CK(bt, cudaMemcpyAsync(bt->ar.mass_rw + off, mass, n * 8, cudaMemcpyHostToDevice, bt->stream));
  GB_CK(bt, cudaMemsetAsync(b.acc + 3 * off, 0, 3 * n * 8, bt->stream));
  BatchSys s{};
  s.id = bt->next_id++;
  s.off = static_cast<uint32_t>(off);
  s.n = static_cast<uint32_t>(n);
  s.g = g;
  s.eps = softening;
  s.theta = theta;
  s.dt = dt;
  s.time = 0.0;
  s.pending = false;
  bt->systems.push_back(s);
  bt->total += static_cast<uint32_t>(n);
  // Prime a(x0) of the new system only.
  bool inside = false;
  rc = upload_tables(bt, {bt->systems.size() - 1}, &inside);
  if (rc) return rc;
  enqueue_step(bt, 0, inside);
  bt->tables_dirty = true;
  drop_graph(bt);
  rc = bfinish(bt);
  if (rc) {
    bt->systems.pop_back();
    bt->total -= static_cast<uint32_t>(n);
    return rc;
  }
  *id_out = s.id;
  return GX_OK;
}

int gx_system_remove(gx_batch* bt, uint64_t id) {
  if (!bt) return GX_ERR_INVALID_ARG;
  const size_t i = index_of(bt, id);
  if (i == SIZE_MAX) return bfail(bt, GX_ERR_NOT_FOUND, "unknown system id");
  cudaSetDevice(bt->device);
  const BatchSys s = bt->systems[i];
  const size_t tail = bt->total - (s.off + s.n);
  StepBufs& b = bt->ar.b;
  if (tail) {
    double* tmp = nullptr;
    GB_CK(bt, cudaMalloc(&tmp, 10 * tail * sizeof(double)));
    const size_t src = s.off + s.n, dst = s.off;
    GB_CK(bt, cudaMemcpyAsync(tmp, b.pos + 3 * src, 3 * tail * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(tmp + 3 * tail, b.vel + 3 * src, 3 * tail * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(tmp + 6 * tail, b.acc + 3 * src, 3 * tail * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(tmp + 9 * tail, bt->ar.mass_rw + src, tail * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(b.pos + 3 * dst, tmp, 3 * tail * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(b.vel + 3 * dst, tmp + 3 * tail, 3 * tail * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(b.acc + 3 * dst, tmp + 6 * tail, 3 * tail * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaMemcpyAsync(bt->ar.mass_rw + dst, tmp + 9 * tail, tail * 8, cudaMemcpyDeviceToDevice, bt->stream));
    GB_CK(bt, cudaStreamSynchronize(bt->stream));
    cudaFree(tmp);
  }
  for (size_t j = i + 1; j < bt->systems.size(); ++j) bt->systems[j].off -= s.n;
  bt->systems.erase(bt->systems.begin() + i);
  bt->total -= s.n;
  bt->tables_dirty = true;
  drop_graph(bt);
  return GX_OK;
}

int gx_batch_set_graph(gx_batch* bt, int enable) {
  if (!bt) return GX_ERR_INVALID_ARG;
  bt->use_graph = enable != 0;
  if (!bt->use_graph) drop_graph(bt);
  return GX_OK;
}

int gx_batch_autotune(gx_batch* bt, uint32_t repeats, gx_tuning* best, gx_tuning* tried, uint32_t* n_tried) {
  if (!bt || !best) return GX_ERR_INVALID_ARG;
  if (bt->systems.empty()) return bfail(bt, GX_ERR_STATE, "autotune of an empty batch");
  cudaSetDevice(bt->device);
  GB_CK(bt, cudaStreamSynchronize(bt->stream));
  std::vector<size_t> all(bt->systems.size());
  for (size_t i = 0; i < all.size(); ++i) all[i] = i;
  bool inside = false;
  int rc = upload_tables(bt, all, &inside);
  if (rc) return rc;
  bt->tables_dirty = false;
  const gx_options user = bt->opt;
  const uint32_t reps = repeats ? repeats : 3;
  // The batch always walks with a persistent kernel (items of uneven systems).
  std::vector<gx_tuning> cand = tune_candidates(bcfg(bt, inside), false, false);
  int best_i = -1;
  for (size_t i = 0; i < cand.size() && rc == GX_OK; ++i) {
    bt->opt.walk_block = cand[i].walk_block;
    bt->opt.walk_ctas_per_sm = cand[i].walk_ctas_per_sm;
    // Force evaluations only (no kick or drift): every system's state is unchanged.
    enqueue_step(bt, 0, inside);
    rc = bfinish(bt);
    std::vector<float> ms;
    for (uint32_t r = 0; r < reps && rc == GX_OK; ++r) {
      cudaEventRecord(bt->e0, bt->stream);
      enqueue_step(bt, 0, inside);
      cudaEventRecord(bt->e1, bt->stream);
      rc = bfinish(bt);
      float t = 0.f;
      if (rc == GX_OK) cudaEventElapsedTime(&t, bt->e0, bt->e1);
      ms.push_back(t);
    }
    if (rc) break;
    std::sort(ms.begin(), ms.end());
    cand[i].ms = ms[ms.size() / 2];
    if (best_i < 0 || cand[i].ms < cand[best_i].ms) best_i = static_cast<int>(i);
  }
  bt->opt = user;
  drop_graph(bt);  // captured with the previous launch configuration
  if (rc) return rc;
  *best = cand[best_i];
  tuned_store(bt->device, user, 1, bt->total, *best);
  if (tried) std::copy(cand.begin(), cand.end(), tried);
  if (n_tried) *n_tried = static_cast<uint32_t>(cand.size());
  return GX_OK;
}

int gx_batch_step(gx_batch* bt, uint64_t steps) {
  if (!bt) return GX_ERR_INVALID_ARG;
  if (bt->systems.empty() || steps == 0) return GX_OK;
  cudaSetDevice(bt->device);
  bool inside = false;
  std::vector<size_t> all(bt->systems.size());
  for (size_t i = 0; i < all.size(); ++i) all[i] = i;
  bool any_fresh = false;
  for (auto& s : bt->systems) any_fresh = any_fresh || !s.pending;
  for (auto& s : bt->systems) inside = inside || s.theta >= 0.57;
  cudaEventRecord(bt->e0, bt->stream);
  uint64_t k = 0;
  if (bt->tables_dirty || any_fresh) {
    int rc = upload_tables(bt, all, &inside);
    if (rc) return rc;
    bt->tables_dirty = false;
    if (any_fresh) {
      // One eager step owes no closing kick for fresh systems; afterwards every
      // system owes one, which the next table upload records.
      enqueue_step(bt, 1, inside);
      for (auto& s : bt->systems) {
        s.pending = true;
        s.time += s.dt;
        s.steps += 1;
      }
      k = 1;
      rc = upload_tables(bt, all, &inside);
      if (rc) return rc;
    }
  }
  const bool graph = bt->use_graph && !(bt->opt.flags & GX_FLAG_STATS);
  if (k < steps && graph && !bt->graph) {
    cudaGraph_t g = nullptr;
    GB_CK(bt, cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(bt, 1, inside);
    GB_CK(bt, cudaStreamEndCapture(bt->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&bt->graph, g, 0);
    cudaGraphDestroy(g);
    GB_CK(bt, e);
  }
  for (; k < steps; ++k) {
    if (graph)
      GB_CK(bt, cudaGraphLaunch(bt->graph, bt->stream));
    else
      enqueue_step(bt, 1, inside);
    for (auto& s : bt->systems) {
      s.time += s.dt;
      s.steps += 1;
    }
  }
  cudaEventRecord(bt->e1, bt->stream);
  int rc = bfinish(bt);
  if (rc) return rc;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, bt->e0, bt->e1);
  bt->ms_last = ms / static_cast<float>(steps);
  bt->steps_total += steps;
  return GX_OK;
}

int gx_system_snapshot(gx_batch* bt, uint64_t id, double* pos_out, double* vel_out, double* time_out) {
  if (!bt) return GX_ERR_INVALID_ARG;
  const size_t i = index_of(bt, id);
  if (i == SIZE_MAX) return bfail(bt, GX_ERR_NOT_FOUND, "unknown system id");
  cudaSetDevice(bt->device);
  const BatchSys& s = bt->systems[i];
  const StepBufs& b = bt->ar.b;
  std::vector<double> vel(3 * (size_t)s.n), acc(3 * (size_t)s.n);
  if (pos_out) GB_CK(bt, cudaMemcpyAsync(pos_out, b.pos + 3 * (size_t)s.off, 3 * (size_t)s.n * 8, cudaMemcpyDeviceToHost, bt->stream));
  GB_CK(bt, cudaMemcpyAsync(vel.data(), b.vel + 3 * (size_t)s.off, 3 * (size_t)s.n * 8, cudaMemcpyDeviceToHost, bt->stream));
  if (s.pending)
    GB_CK(bt, cudaMemcpyAsync(acc.data(), b.acc + 3 * (size_t)s.off, 3 * (size_t)s.n * 8, cudaMemcpyDeviceToHost, bt->stream));
  GB_CK(bt, cudaStreamSynchronize(bt->stream));
  if (s.pending) {
    // The owed closing half kick, applied to the copy (v + a*(0.5 dt), one rounding each).
    volatile double h = 0.5 * s.dt;
    for (size_t j = 0; j < vel.size(); ++j) {
      volatile double t = acc[j] * h;
      vel[j] = vel[j] + t;
    }
  }
  if (vel_out) memcpy(vel_out, vel.data(), vel.size() * sizeof(double));
  if (time_out) *time_out = s.time;
  return GX_OK;
}

int gx_system_len(const gx_batch* bt, uint64_t id, size_t* n_out) {
  if (!bt || !n_out) return GX_ERR_INVALID_ARG;
  const size_t i = index_of(bt, id);
  if (i == SIZE_MAX) return GX_ERR_NOT_FOUND;
  *n_out = bt->systems[i].n;
  return GX_OK;
}

int gx_batch_stats_get(const gx_batch* bt, gx_batch_stats* out) {
  if (!bt || !out) return GX_ERR_INVALID_ARG;
  out->systems = bt->systems.size();
  out->particles = bt->total;
  out->steps = bt->steps_total;
  out->bytes_in_use = bt->ar.bytes;
  out->budget_bytes = bt->budget;
  out->ms_last_step = bt->ms_last;
  return GX_OK;
}

}  // extern "C"
