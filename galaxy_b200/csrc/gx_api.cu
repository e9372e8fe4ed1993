// gx_api.cu -- the C ABI of one system: ForceSolver-style calls, resident leapfrog
// stepping, stage entry points and diagnostics (declared in include/galaxy_b200.h).
//
// Reference interfaces: core/src/traits.rs:24-157 (ForceSolver),
// gpu/src/gpu_lbvh_fused.rs:44-146 (the drop-in GPU backend),
// gpu/src/gpu_resident.rs:1685-1960 (upload / step / step_many / snapshot / time).
// The closing half kick of a step is deferred into the next step's kick + drift
// kernel (two separately rounded half kicks, as integrator.rs:61-73 applies them)
// or into a snapshot, so it costs no extra pass over the state.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <limits>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/galaxy_b200.h"
#include "gx_kernels.h"
#include "gx_runtime.h"
#include "gx_sph.h"

using namespace gx;

namespace gx {

thread_local std::string g_global_err;

void set_global_err(const std::string& s) { g_global_err = s; }
const char* global_err() { return g_global_err.c_str(); }

bool check_device(int device, std::string& err) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    err = std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count 0");
    return false;
  }
  int dev = device;
  if (dev < 0) {
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  }
  if (dev >= count) {
    err = "device ordinal out of range";
    return false;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
    err = "cudaGetDeviceProperties failed";
    return false;
  }
  if (p.major != 10) {
    err = std::string("libgalaxy_b200 is built for sm_100a (B200); device is ") + p.name + " sm_" +
          std::to_string(p.major) + std::to_string(p.minor);
    return false;
  }
  return true;
}

bool options_valid(const gx_options& o) {
  return o.precision <= GX_PREC_F64 && o.multipole <= GX_MULTIPOLE_QUAD &&
         !(o.walk_block && (o.walk_block % 32 || o.walk_block > static_cast<uint32_t>(kWalkThreads))) &&
         (o.walk_group == 0 || o.walk_group == 8 || o.walk_group == 16 || o.walk_group == 32) &&
         (o.radix_bits == 0 || o.radix_bits == kRadixBits || o.radix_bits == kRadixBitsWide);
}

// Once per device, with the device current: kernel attributes the launches rely on.
void prepare_device(int dev) {
  static std::mutex mu;
  static uint64_t done = 0;
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64 || (done >> dev) & 1u) return;
  walk_prepare();
  build_prepare();
  done |= 1ull << dev;
}

// ---- Arena: one system's device buffers -------------------------------------------
void Arena::release() {
  for (void* p : allocs)
    if (p) cudaFree(p);
  allocs.clear();
  bytes = 0;
  b = StepBufs();
  cap_n = 0;
  cap_tiles = 0;
  cap_items = 0;
  cap_sys = 0;
}

cudaError_t Arena::alloc(void** p, size_t nbytes) {
  nbytes = (nbytes + 255) & ~size_t(255);
  if (nbytes == 0) nbytes = 256;
  cudaError_t e = cudaMalloc(p, nbytes);
  if (e == cudaSuccess) {
    allocs.push_back(*p);
    bytes += nbytes;
  }
  return e;
}

size_t Arena::bytes_for(size_t n, size_t nsys, int quad, int f64rec) {
  const size_t tiles = n / kTile + nsys + 1;
  size_t s = 0;
  s += 3 * 3 * n * 8 + n * 8;                 // pos, vel, acc, mass
  s += 6 * n * 4;                             // codes, keys_alt (u64-capable), order, vals_alt
  s += n * 32 + n * 80;                       // leaf64, sibling-pair walk records
  s += n * 8 + 2 * n * 4 + n * sizeof(Agg64); // kids, parent, agg64
  s += 2 * n * 16;                            // nodeC, nodeD
  s += n * 8;                                 // slots
  if (quad) s += 2 * n * 16 + 6 * n * 8;
  if (f64rec) s += n * sizeof(Node64);
  s += tiles * sizeof(TileDesc) + (n / 8 + nsys + 1) * sizeof(WalkItem);
  s += nsys * (sizeof(SysDesc) + sizeof(Bounds) + 48 + kHistWords * 4);
  s += tiles * kStatusWordsPerTile * 4 + 64;
  s += (n / 256 + 1) * 8 * 8;  // diagnostic partials
  return s + 64 * 256;         // alignment slack
}

cudaError_t Arena::ensure(size_t n, size_t tiles, size_t items, size_t nsys, int quad, int f64rec, cudaStream_t st) {
  if (n <= cap_n && tiles <= cap_tiles && items <= cap_items && nsys <= cap_sys && quad <= cap_quad &&
      f64rec <= cap_f64)
    return cudaSuccess;
  // Grow (never shrink) only the dimensions that are short, each with headroom so a
  // slowly growing batch does not reallocate on every call.
  auto grown = [](size_t need, size_t cap, size_t floor_) {
    return need <= cap ? cap : std::max({need, cap + cap / 4, floor_});
  };
  size_t nn = grown(n, cap_n, 0);
  size_t nt = grown(tiles, cap_tiles, 0);
  size_t ni = grown(items, cap_items, 0);
  size_t ns = grown(nsys, cap_sys, 16);
  int q = std::max(quad, cap_quad), f = std::max(f64rec, cap_f64);
  cudaStreamSynchronize(st);
  release();
  cudaError_t e = cudaSuccess;
#define GX_A(ptr, count, T)                                              \
  do {                                                                   \
    void* _p = nullptr;                                                  \
    e = alloc(&_p, (size_t)(count) * sizeof(T));                         \
    if (e != cudaSuccess) return e;                                      \
    ptr = reinterpret_cast<decltype(ptr)>(_p);                           \
  } while (0)
  GX_A(b.pos, 3 * nn, double);
  GX_A(b.vel, 3 * nn, double);
  GX_A(b.acc, 3 * nn, double);
  double* mass = nullptr;
  GX_A(mass, nn, double);
  b.mass = mass;
  mass_rw = mass;
  GX_A(b.codes, 2 * nn, uint32_t);     // room for 63-bit keys
  GX_A(b.keys_alt, 2 * nn, uint32_t);
  GX_A(b.order, nn, uint32_t);
  GX_A(b.vals_alt, nn, uint32_t);
  GX_A(b.leaf64, nn, double4);
  GX_A(b.pairs, 5 * nn, float4);  // sibling-pair walk records, one per internal node
  GX_A(b.kids, nn, uint2);
  GX_A(b.parent, 2 * nn, uint32_t);
  GX_A(b.agg64, nn, Agg64);
  GX_A(b.nodeC, nn, float4);
  GX_A(b.nodeD, nn, float4);
  if (q) {
    GX_A(b.nodeQ, 2 * nn, float4);
    GX_A(b.q64, 6 * nn, double);
  }
  if (f) GX_A(b.node64, nn, Node64);
  GX_A(b.slots, nn, unsigned long long);
  TileDesc* tl = nullptr;
  GX_A(tl, nt, TileDesc);
  b.tiles = tl;
  tiles_rw = tl;
  WalkItem* it = nullptr;
  GX_A(it, ni, WalkItem);
  b.items = it;
  items_rw = it;
  SysDesc* sd = nullptr;
  GX_A(sd, ns, SysDesc);
  b.sys = sd;
  sys_rw = sd;
  GX_A(b.bounds, ns, Bounds);
  // One zeroed region per step: bbox words, histograms, look-back status, counters.
  const size_t z_bbox = 6 * ns * sizeof(unsigned long long);
  const size_t z_hist = ns * kHistWords * sizeof(uint32_t);
  const size_t z_stat = (size_t)nt * kStatusWordsPerTile * sizeof(uint32_t);
  const size_t z_ctr = kCounterWords * sizeof(uint32_t);
  char* z = nullptr;
  GX_A(z, z_bbox + z_hist + z_stat + z_ctr, char);
  b.bbox_enc = reinterpret_cast<unsigned long long*>(z);
  b.hist = reinterpret_cast<uint32_t*>(z + z_bbox);
  b.sort_status = reinterpret_cast<uint32_t*>(z + z_bbox + z_hist);
  b.counters = reinterpret_cast<uint32_t*>(z + z_bbox + z_hist + z_stat);
  b.zero_begin = z;
  b.zero_bytes = z_bbox + z_hist + z_stat + z_ctr;
  GX_A(b.ctl, 1, DevCtl);
  diag_cap = nn / 256 + 2;
  GX_A(diag_partial, 8 * diag_cap, double);
#undef GX_A
  e = cudaMemsetAsync(b.slots, 0xFF, nn * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(b.ctl, 0, sizeof(DevCtl), st);
  if (e != cudaSuccess) return e;
  cap_n = nn;
  cap_tiles = nt;
  cap_items = ni;
  cap_sys = ns;
  cap_quad = q;
  cap_f64 = f;
  return cudaStreamSynchronize(st);
}

// Host-side tile and walk-item tables of a list of systems packed back to back.
void make_tables(const std::vector<SysDesc>& in, std::vector<SysDesc>& sys, std::vector<TileDesc>& tiles,
                 std::vector<WalkItem>& items) {
  sys = in;
  tiles.clear();
  items.clear();
  for (uint32_t s = 0; s < sys.size(); ++s) {
    SysDesc& d = sys[s];
    d.first_tile = static_cast<uint32_t>(tiles.size());
    for (uint32_t b0 = 0; b0 < d.n; b0 += kTile) {
      TileDesc t;
      t.sys = s;
      t.begin = d.off + b0;
      t.end = d.off + std::min<uint32_t>(d.n, b0 + kTile);
      t.pad = 0;
      tiles.push_back(t);
    }
    d.ntiles = static_cast<uint32_t>(tiles.size()) - d.first_tile;
    if (d.group != 8 && d.group != 16) d.group = 32;
    for (uint32_t b0 = 0; b0 < d.n; b0 += d.group) items.push_back(WalkItem{d.off + b0, s});
  }
}

namespace {

struct TuneKey {
  int device, precision, multipole, key64, batched, bucket;
  bool operator<(const TuneKey& o) const {
    return std::tie(device, precision, multipole, key64, batched, bucket) <
           std::tie(o.device, o.precision, o.multipole, o.key64, o.batched, o.bucket);
  }
};

std::mutex g_tune_mu;
std::map<TuneKey, gx_tuning> g_tune;

TuneKey tune_key(int device, const gx_options& opt, int batched, size_t n) {
  int bucket = 0;
  while (bucket < 63 && (size_t{2} << bucket) <= n) ++bucket;  // floor(log2 n)
  return TuneKey{device, static_cast<int>(opt.precision), static_cast<int>(opt.multipole),
                 (opt.flags & GX_FLAG_MORTON63) ? 1 : 0, batched ? 1 : 0, bucket};
}

}  // namespace

bool tuned_lookup(int device, const gx_options& opt, int batched, size_t n, gx_tuning* out) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_key(device, opt, batched, n));
  if (it == g_tune.end()) return false;
  *out = it->second;
  return true;
}

void tuned_store(int device, const gx_options& opt, int batched, size_t n, const gx_tuning& t) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[tune_key(device, opt, batched, n)] = t;
}

// Targets a warp of the FP32 walk when nothing is tuned: narrow groups for small systems,
// whose walk is the latency of few warps (more warps, tighter group boxes), 32 targets
// for large ones.
uint32_t default_walk_group(size_t n) { return n < (size_t{1} << 16) ? 8u : n < (size_t{1} << 19) ? 16u : 32u; }

uint32_t system_radix_bits(int device, const gx_options& opt, size_t n) {
  if (opt.flags & GX_FLAG_MORTON63) return kRadixBits;
  if (opt.radix_bits) return opt.radix_bits;
  gx_tuning t;
  if (tuned_lookup(device, opt, 0, n, &t) && t.radix_bits) return t.radix_bits;
  return kRadixBits;
}

uint32_t system_walk_group(int device, const gx_options& opt, size_t n) {
  if (opt.precision == GX_PREC_F64) return 32u;  // the FP64 walk takes 32 targets a warp
  if (opt.walk_group) return opt.walk_group;
  gx_tuning t;
  if (tuned_lookup(device, opt, 0, n, &t) && t.walk_group) return t.walk_group;
  return default_walk_group(n);
}

std::vector<gx_tuning> tune_candidates(const WalkCfg& base, bool with_grid, bool with_groups) {
  std::vector<gx_tuning> out;
  const std::vector<uint32_t> groups = with_groups ? std::vector<uint32_t>{8u, 16u, 32u} : std::vector<uint32_t>{0u};
  for (uint32_t grp : groups) {
    for (int block : {64, kWalkThreads}) {
      WalkCfg c = base;
      c.block = block;
      const int full = walk_resident_ctas(c);
      if (with_grid) out.push_back(gx_tuning{static_cast<uint32_t>(block), 0u, grp, 0u, 0.f, 0.f});
      if (full / 2 >= 1)
        out.push_back(gx_tuning{static_cast<uint32_t>(block), static_cast<uint32_t>(full / 2), grp, 0u, 0.f, 0.f});
      out.push_back(gx_tuning{static_cast<uint32_t>(block), static_cast<uint32_t>(full), grp, 0u, 0.f, 0.f});
    }
  }
  if (out.size() > GX_TUNE_MAX_CANDIDATES) out.resize(GX_TUNE_MAX_CANDIDATES);
  return out;
}

}  // namespace gx

// ===================================================================================
struct gx_handle {
  double g = 1.0, eps = 0.0, theta = 0.5;
  gx_options opt{};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[8] = {};  // stage boundaries; [5] gx_step_many_timed, [6] end of SPH, [7] end of its density
  cudaEvent_t chunk_ev[8] = {};  // gx_kdk_step_host: acceleration chunks copied back
  DevCtl* ctl_host = nullptr;     // pinned copy of the device error word
  std::string err;
  Arena ar;
  // current layout
  size_t n_layout = 0;
  double dt_layout = 0.0;
  uint32_t group_layout = 0;  // targets a warp of the laid-out walk items
  // resident state
  size_t n = 0;
  double time = 0.0;
  bool resident = false;
  bool pending_kick = false;
  uint64_t launches = 0;
  gx_stats stats{};
  // every tree build bumps tree_gen; the stale-tree cache is valid while it holds
  uint64_t tree_gen = 0, cache_gen = ~0ull;
  size_t cache_n = 0;
  // active-subset walk (gx_accelerations_active): buffers grown on demand
  struct Active {
    uint32_t* active = nullptr;  // the caller's active indices
    uint32_t* inv = nullptr;     // original index -> sorted position
    uint32_t* flags = nullptr;   // per sorted position
    uint32_t* chunks = nullptr;  // compaction chunk offsets, then the count
    uint32_t* list = nullptr;    // active sorted positions, in sorted order
    WalkItem* items = nullptr;
    double* out = nullptr;       // gathered accelerations
    size_t cap_n = 0, cap_a = 0;
  } act;
  // gas mode (GpuResidentLeapfrog::new_with_sph): SPH on the gas rows after gravity
  SphState sph;
  bool resident_gas = false;     // the resident state has gas and runs SPH in each force
  size_t sph_host_hint_ngas = 0;  // gx_sph_accelerations: gas count of the last call
  size_t sph_rho_scratch_ngas = 0;  // gx_sph_accelerations_active: its rho scratch is set
  uint64_t sph_rho_gen = 0;         // ... in this allocation of the SPH buffers
  // graph of one resident step (pending closing kick + opening kick, drift, force)
  cudaGraphExec_t step_graph = nullptr;
  size_t graph_n = 0;
  double graph_dt = 0.0;
};

namespace {

int fail(gx_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define GX_CK(h, call)                                                                        \
  do {                                                                                        \
    cudaError_t _e = (call);                                                                  \
    if (_e != cudaSuccess)                                                                    \
      return fail((h), GX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));      \
  } while (0)

WalkCfg walk_cfg(const gx_handle* h) {
  WalkCfg c;
  c.precision = h->opt.precision == GX_PREC_F64 ? 1 : 0;
  c.quad = (h->opt.multipole == GX_MULTIPOLE_QUAD && c.precision == 0) ? 1 : 0;
  c.kahan = (h->opt.flags & GX_FLAG_NO_KAHAN) ? 0 : 1;
  c.stats = (h->opt.flags & GX_FLAG_STATS) ? 1 : 0;
  c.inside_test = h->theta >= 0.57 ? 1 : 0;
  c.block = h->opt.walk_block ? static_cast<int>(h->opt.walk_block) : kWalkThreads;
  c.persistent_ctas = h->opt.walk_ctas_per_sm ? static_cast<int>(h->opt.walk_ctas_per_sm) * h->sm_count : 0;
  gx_tuning t;
  if (!h->opt.walk_block && !h->opt.walk_ctas_per_sm && tuned_lookup(h->device, h->opt, 0, h->n_layout, &t)) {
    c.block = static_cast<int>(t.walk_block);
    c.persistent_ctas = static_cast<int>(t.walk_ctas_per_sm) * h->sm_count;
  }
  return c;
}

// Lay out one system of n particles (tables + SysDesc) with step dt.
int layout(gx_handle* h, size_t n, double dt) {
  if (n > (1u << 30)) return fail(h, GX_ERR_INVALID_ARG, "N above 2^30 is not supported (30-bit look-back counts)");
  if (n == h->n_layout && dt == h->dt_layout && h->ar.cap_n >= n &&
      system_walk_group(h->device, h->opt, n) == h->group_layout &&
      static_cast<int>(system_radix_bits(h->device, h->opt, n)) == h->ar.b.radix_bits)
    return GX_OK;
  std::vector<SysDesc> in(1), sys;
  in[0].off = 0;
  in[0].n = static_cast<uint32_t>(n);
  in[0].g = h->g;
  in[0].eps = h->eps;
  in[0].theta = h->theta;
  in[0].dt = dt;
  in[0].group = system_walk_group(h->device, h->opt, n);
  std::vector<TileDesc> tiles;
  std::vector<WalkItem> items;
  make_tables(in, sys, tiles, items);
  const int quad = h->opt.multipole == GX_MULTIPOLE_QUAD;
  const int f64 = h->opt.precision == GX_PREC_F64;
  // Items are sized for the narrowest grouping, so a new grouping never reallocates
  // (which would lose the resident state).
  GX_CK(h, h->ar.ensure(n, tiles.size(), std::max(items.size(), n / 8 + 2), 1, quad, f64, h->stream));
  StepBufs& b = h->ar.b;
  b.n = static_cast<uint32_t>(n);
  b.key64 = (h->opt.flags & GX_FLAG_MORTON63) ? 1 : 0;
  b.radix_bits = static_cast<int>(system_radix_bits(h->device, h->opt, n));
  b.nsys = 1;
  b.ntiles = static_cast<uint32_t>(tiles.size());
  b.nitems = static_cast<uint32_t>(items.size());
  // The per-step zero region: bbox words, histograms, look-back status, counters.
  b.zero_bytes = reinterpret_cast<char*>(b.counters) - reinterpret_cast<char*>(b.zero_begin) + kCounterWords * sizeof(uint32_t);
  GX_CK(h, cudaMemcpyAsync(h->ar.sys_rw, sys.data(), sizeof(SysDesc), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.tiles_rw, tiles.data(), tiles.size() * sizeof(TileDesc), cudaMemcpyHostToDevice,
                           h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.items_rw, items.data(), items.size() * sizeof(WalkItem), cudaMemcpyHostToDevice,
                           h->stream));
  GX_CK(h, cudaStreamSynchronize(h->stream));
  h->n_layout = n;
  h->dt_layout = dt;
  h->group_layout = sys[0].group;
  if (h->step_graph) {
    cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
  }
  return GX_OK;
}

// Enqueue bbox (+kick/drift) -> Morton -> sort -> build on b.
void enqueue_tree(gx_handle* h, const StepBufs& b, int kick, int pending, bool timed) {
  cudaStream_t st = h->stream;
  ++h->tree_gen;
  if (timed) cudaEventRecord(h->ev[0], st);
  {
    NvtxRange r("gx.kick_drift_bbox_morton");
    cudaMemsetAsync(b.zero_begin, 0, b.zero_bytes, st);
    launch_kick_drift_bbox(b, kick, pending, st);
    launch_morton_hist(b, nullptr, st);
  }
  if (timed) cudaEventRecord(h->ev[1], st);
  {
    NvtxRange r("gx.sort");
    launch_sort(b, st);
  }
  if (timed) cudaEventRecord(h->ev[2], st);
  {
    NvtxRange r("gx.build");
    launch_build(b, h->opt.multipole == GX_MULTIPOLE_QUAD && h->opt.precision != GX_PREC_F64,
                 h->opt.precision == GX_PREC_F64, st);
  }
  if (timed) cudaEventRecord(h->ev[3], st);
}

// Enqueue the tree and the walk of every target on b.
void enqueue_force(gx_handle* h, const StepBufs& b, int kick, int pending, bool timed) {
  NvtxRange r("gx.step");
  enqueue_tree(h, b, kick, pending, timed);
  NvtxRange w("gx.walk");
  launch_walk(b, walk_cfg(h), h->stream);
  if (timed) cudaEventRecord(h->ev[4], h->stream);
  if (h->resident && h->resident_gas) {
    NvtxRange g("gx.sph");
    sph_enqueue_force(h->sph, b.pos, b.vel, b.mass, b.acc, true, true, b.ctl, h->stream, timed ? h->ev[7] : nullptr);
    if (timed) cudaEventRecord(h->ev[6], h->stream);
  }
  h->launches += 1;
}

// Wait for the stream, then turn the device error word into a status.
int finish(gx_handle* h, bool timed) {
  GX_CK(h, cudaStreamSynchronize(h->stream));
  GX_CK(h, cudaGetLastError());
  if (!h->ar.b.ctl) return GX_OK;  // nothing allocated yet (empty system)
  DevCtl ctl;
  GX_CK(h, cudaMemcpy(&ctl, h->ar.b.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost));
  if (timed) {
    cudaEventElapsedTime(&h->stats.ms_bbox_morton, h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&h->stats.ms_sort, h->ev[1], h->ev[2]);
    cudaEventElapsedTime(&h->stats.ms_build, h->ev[2], h->ev[3]);
    cudaEventElapsedTime(&h->stats.ms_walk, h->ev[3], h->ev[4]);
    cudaEventElapsedTime(&h->stats.ms_total, h->ev[0], h->ev[4]);
    h->stats.ms_sph = h->stats.ms_sph_density = 0.0f;
    if (h->resident && h->resident_gas) {
      cudaEventElapsedTime(&h->stats.ms_sph, h->ev[4], h->ev[6]);
      cudaEventElapsedTime(&h->stats.ms_sph_density, h->ev[4], h->ev[7]);
    }
  }
  h->stats.leaf_interactions = ctl.stats[0];
  h->stats.far_interactions = ctl.stats[1];
  h->stats.nodes_opened = ctl.stats[2];
  h->stats.f64_rechecks = ctl.stats[3];
  h->stats.warp_node_visits = ctl.stats[4];
  if (ctl.err) {
    // Re-arm the climb slots and clear the word so the handle stays usable.
    cudaMemset(h->ar.b.slots, 0xFF, h->ar.cap_n * sizeof(unsigned long long));
    cudaMemset(h->ar.b.ctl, 0, sizeof(DevCtl));
    char buf[128];
    snprintf(buf, sizeof buf, "device check tripped (error word 0x%x)", ctl.err);
    return fail(h, GX_ERR_DEVICE_CHECK, buf);
  }
  if (h->opt.flags & GX_FLAG_STATS) cudaMemset(h->ar.b.ctl, 0, sizeof(DevCtl));
  return GX_OK;
}

bool stats_on(const gx_handle* h) { return (h->opt.flags & GX_FLAG_STAGE_TIMES) != 0; }

void free_active(gx_handle* h) {
  auto& a = h->act;
  for (void* p : {static_cast<void*>(a.active), static_cast<void*>(a.inv), static_cast<void*>(a.flags),
                  static_cast<void*>(a.chunks), static_cast<void*>(a.list), static_cast<void*>(a.items),
                  static_cast<void*>(a.out)})
    if (p) cudaFree(p);
  a = gx_handle::Active{};
}

// Grow (never shrink) the active-walk buffers to n particles and na active ones.
cudaError_t ensure_active(gx_handle* h, size_t n, size_t na) {
  auto& a = h->act;
  if (n <= a.cap_n && na <= a.cap_a) return cudaSuccess;
  const size_t cn = std::max(n, a.cap_n), ca = std::max(na, a.cap_a);
  cudaStreamSynchronize(h->stream);
  free_active(h);
  const size_t nchunks = active_chunk_count(static_cast<uint32_t>(cn)) + 1;
  const size_t litems = ca;  // one item per active target at the smallest group
  cudaError_t e = cudaMalloc(&a.active, ca * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&a.inv, cn * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&a.flags, cn * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&a.chunks, (nchunks + 1) * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&a.list, (ca + 32) * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&a.items, litems * sizeof(WalkItem));
  if (e == cudaSuccess) e = cudaMalloc(&a.out, 3 * ca * sizeof(double));
  if (e != cudaSuccess) {
    free_active(h);
    return e;
  }
  a.cap_n = cn;
  a.cap_a = ca;
  return cudaSuccess;
}

}  // namespace

// ===================================================================================
extern "C" {

int gx_create(double g, double softening, double theta, const gx_options* opt, gx_handle** out) {
  if (!out) return GX_ERR_INVALID_ARG;
  *out = nullptr;
  if (!(softening >= 0.0) || !(theta >= 0.0) || !(g == g)) {
    set_global_err("softening and theta must be >= 0");
    return GX_ERR_INVALID_ARG;
  }
  gx_options o{};
  o.device = -1;
  if (opt && opt->struct_size) {
    if (opt->struct_size < sizeof(gx_options)) {
      set_global_err("gx_options.struct_size too small");
      return GX_ERR_INVALID_ARG;
    }
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
  gx_handle* h = new gx_handle();
  h->g = g;
  h->eps = softening;
  h->theta = theta;
  h->opt = o;
  int dev = o.device;
  if (dev < 0) cudaGetDevice(&dev);
  h->device = dev;
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaSetDevice(dev);
  if (e == cudaSuccess) prepare_device(dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  for (int i = 0; i < 8 && e == cudaSuccess; ++i) e = cudaEventCreate(&h->ev[i]);
  for (int i = 0; i < 8 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&h->chunk_ev[i], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaHostAlloc(&h->ctl_host, sizeof(DevCtl), cudaHostAllocDefault);
  if (e != cudaSuccess) {
    set_global_err(std::string("stream/event creation failed: ") + cudaGetErrorString(e));
    delete h;
    return GX_ERR_CUDA;
  }
  *out = h;
  return GX_OK;
}

void gx_destroy(gx_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_active(h);
  if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
  sph_free(h->sph);
  h->ar.release();
  for (auto& e : h->chunk_ev)
    if (e) cudaEventDestroy(e);
  if (h->ctl_host) cudaFreeHost(h->ctl_host);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

const char* gx_last_error(const gx_handle* h) { return h ? h->err.c_str() : global_err(); }

int gx_selftest_bounded_wait(int device, uint32_t spins, uint32_t* err_word_out) {
  if (!err_word_out) return GX_ERR_INVALID_ARG;
  std::string err;
  if (!check_device(device, err)) {
    set_global_err(err);
    return GX_ERR_NO_DEVICE;
  }
  int dev = device;
  if (dev < 0) cudaGetDevice(&dev);
  cudaSetDevice(dev);
  DevCtl* ctl = nullptr;
  uint32_t* word = nullptr;
  cudaError_t e = cudaMalloc(&ctl, sizeof(DevCtl));
  if (e == cudaSuccess) e = cudaMalloc(&word, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(ctl, 0, sizeof(DevCtl));
  if (e == cudaSuccess) e = cudaMemset(word, 0, sizeof(uint32_t));
  if (e == cudaSuccess) {
    launch_selftest_wait(word, spins, ctl, nullptr);
    e = cudaDeviceSynchronize();
  }
  DevCtl host{};
  if (e == cudaSuccess) e = cudaMemcpy(&host, ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost);
  if (ctl) cudaFree(ctl);
  if (word) cudaFree(word);
  if (e != cudaSuccess) {
    set_global_err(std::string("self-test: ") + cudaGetErrorString(e));
    return GX_ERR_CUDA;
  }
  *err_word_out = host.err;
  if (host.err) {
    set_global_err("device check tripped (bounded wait ran out)");
    return GX_ERR_DEVICE_CHECK;
  }
  return GX_OK;
}

int gx_device_synchronize(int device) {
  int dev = device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return GX_ERR_NO_DEVICE;
  cudaError_t e = cudaSetDevice(dev);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_global_err(std::string("device synchronize: ") + cudaGetErrorString(e));
    return GX_ERR_CUDA;
  }
  return GX_OK;
}

int gx_device_info(int device, char* name_out, size_t name_len, int* sm_count, int* cc_major, int* cc_minor,
                   size_t* total_mem) {
  cudaDeviceProp p;
  cudaError_t e = cudaGetDeviceProperties(&p, device < 0 ? 0 : device);
  if (e != cudaSuccess) {
    set_global_err(cudaGetErrorString(e));
    return GX_ERR_NO_DEVICE;
  }
  if (name_out && name_len) {
    strncpy(name_out, p.name, name_len - 1);
    name_out[name_len - 1] = 0;
  }
  if (sm_count) *sm_count = p.multiProcessorCount;
  if (cc_major) *cc_major = p.major;
  if (cc_minor) *cc_minor = p.minor;
  if (total_mem) *total_mem = p.totalGlobalMem;
  return GX_OK;
}

int gx_accelerations(gx_handle* h, size_t n, const double* pos, const double* mass, double* acc_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (n == 0) return GX_OK;
  if (!pos || !mass || !acc_out) return fail(h, GX_ERR_INVALID_ARG, "null array");
  if (n == 1) {
    acc_out[0] = acc_out[1] = acc_out[2] = 0.0;
    return GX_OK;
  }
  cudaSetDevice(h->device);
  // A ForceSolver call does not disturb resident state: it uses the same arena, so
  // the resident system is dropped.
  h->resident = false;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  enqueue_force(h, b, 0, 0, stats_on(h));
  GX_CK(h, cudaMemcpyAsync(acc_out, b.acc, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  h->stats.n = n;
  return finish(h, stats_on(h));
}

int gx_accelerations_device(gx_handle* h, size_t n, const double* d_pos, const double* d_mass, double* d_acc) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (n == 0) return GX_OK;
  if (!d_pos || !d_mass || !d_acc) return fail(h, GX_ERR_INVALID_ARG, "null array");
  cudaSetDevice(h->device);
  if (n == 1) {
    GX_CK(h, cudaMemsetAsync(d_acc, 0, 3 * sizeof(double), h->stream));
    return GX_OK;
  }
  h->resident = false;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs b = h->ar.b;
  b.pos = const_cast<double*>(d_pos);
  b.mass = d_mass;
  b.acc = d_acc;
  enqueue_force(h, b, 0, 0, false);
  h->stats.n = n;
  return GX_OK;
}

namespace {

// The active targets' walk on the tree in the arena (fresh or cached): list, walk,
// gather, copy back, scatter into acc_out.
int walk_active(gx_handle* h, size_t n, size_t n_active, const uint32_t* active, double* acc_out, bool timed) {
  StepBufs& b = h->ar.b;
  auto& a = h->act;
  const uint32_t na = static_cast<uint32_t>(n_active);
  uint32_t* count = a.chunks + active_chunk_count(static_cast<uint32_t>(n)) + 1;
  // Targets per warp: a sparse subset spreads 32 consecutive active targets over a wide
  // region (a large union walk), so fewer lanes take part the sparser it is. Thresholds
  // from a sweep on the 2^20 collision (walk ms at 0.3% / 1% / 3% / 10% / 30% active:
  // 4 lanes 3.3 / 3.0 / 3.6 / 6.9 / 16.0, 8 lanes 4.2 / 3.2 / 3.2 / 5.1 / 9.8, 32 lanes
  // 8.0 / 5.4 / 3.8 / 3.8 / 5.3; the full walk takes 9.5).
  const double frac = static_cast<double>(n_active) / static_cast<double>(n);
  const uint32_t group = frac >= 0.08 ? 32u : frac >= 0.04 ? 16u : frac >= 0.015 ? 8u : 4u;
  launch_active_targets(b, a.active, na, group, a.inv, a.flags, a.chunks, a.list, count, a.items, h->stream);
  StepBufs bl = b;  // the same tree, walked for the listed targets only
  bl.targets = a.list;
  bl.ntargets = count;
  bl.group = group;
  bl.items = a.items;
  bl.nitems = (na + group - 1) / group;
  launch_walk(bl, walk_cfg(h), h->stream);
  if (timed) cudaEventRecord(h->ev[4], h->stream);
  h->launches += 1;
  launch_gather_acc(b.acc, a.active, na, a.out, h->stream);
  std::vector<double> got(3 * n_active);
  GX_CK(h, cudaMemcpyAsync(got.data(), a.out, 3 * n_active * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  h->stats.n = n;
  const int rc = finish(h, timed);
  if (rc) return rc;
  for (size_t i = 0; i < n_active; ++i)
    for (int c = 0; c < 3; ++c) acc_out[3 * (size_t)active[i] + c] = got[3 * i + c];
  return GX_OK;
}

int check_active(gx_handle* h, size_t n, const double* pos, const double* mass, size_t n_active,
                 const uint32_t* active, double* acc_out) {
  if (!pos || !mass || !active || !acc_out) return fail(h, GX_ERR_INVALID_ARG, "null array");
  if (n_active > (size_t{1} << 31)) return fail(h, GX_ERR_INVALID_ARG, "too many active indices");
  for (size_t i = 0; i < n_active; ++i)
    if (active[i] >= n) return fail(h, GX_ERR_INVALID_ARG, "active index out of range");
  return GX_OK;
}

}  // namespace

int gx_accelerations_active(gx_handle* h, size_t n, const double* pos, const double* mass, size_t n_active,
                            const uint32_t* active, double* acc_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (n == 0 || n_active == 0) return GX_OK;
  int rc = check_active(h, n, pos, mass, n_active, active, acc_out);
  if (rc) return rc;
  if (n == 1) {
    acc_out[0] = acc_out[1] = acc_out[2] = 0.0;  // a lone particle feels no force
    return GX_OK;
  }
  cudaSetDevice(h->device);
  h->resident = false;  // shares the arena with the resident state
  rc = layout(h, n, 0.0);
  if (rc) return rc;
  GX_CK(h, ensure_active(h, n, n_active));
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->act.active, active, n_active * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  const bool timed = stats_on(h);
  enqueue_tree(h, b, 0, 0, timed);
  return walk_active(h, n, n_active, active, acc_out, timed);
}

int gx_rebuild_gravity_cache(gx_handle* h, size_t n, const double* pos, const double* mass) {
  if (!h) return GX_ERR_INVALID_ARG;
  h->cache_gen = ~0ull;
  h->cache_n = n;
  if (n < 2) return GX_OK;  // nothing to cache: the walks of 0 or 1 particle are trivial
  if (!pos || !mass) return fail(h, GX_ERR_INVALID_ARG, "null array");
  cudaSetDevice(h->device);
  h->resident = false;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  enqueue_tree(h, b, 0, 0, false);
  rc = finish(h, false);
  if (rc) return rc;
  h->cache_gen = h->tree_gen;
  return GX_OK;
}

int gx_gravity_active_cached(gx_handle* h, size_t n, const double* pos, const double* mass, size_t n_active,
                             const uint32_t* active, double* acc_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (n != h->cache_n) return fail(h, GX_ERR_STATE, "no cached tree for this many particles");
  if (n == 0 || n_active == 0) return GX_OK;
  int rc = check_active(h, n, pos, mass, n_active, active, acc_out);
  if (rc) return rc;
  if (n == 1) {
    acc_out[0] = acc_out[1] = acc_out[2] = 0.0;
    return GX_OK;
  }
  if (h->cache_gen != h->tree_gen)
    return fail(h, GX_ERR_STATE, "the cached tree was replaced: call gx_rebuild_gravity_cache");
  cudaSetDevice(h->device);
  GX_CK(h, ensure_active(h, n, n_active));
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->act.active, active, n_active * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  // the walk's own per-step counters start at zero (the tree is not rebuilt)
  GX_CK(h, cudaMemsetAsync(b.counters, 0, kCounterWords * sizeof(uint32_t), h->stream));
  launch_refresh_leaves(b, h->stream);
  return walk_active(h, n, n_active, active, acc_out, false);
}

int gx_synchronize(gx_handle* h) {
  if (!h) return GX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  return finish(h, stats_on(h));  // stage times of the last step when they are on
}

int gx_potential_energy(gx_handle* h, size_t n, const double* pos, const double* mass, double* out) {
  if (!h || !out) return GX_ERR_INVALID_ARG;
  *out = 0.0;
  if (n < 2) return GX_OK;
  if (!pos || !mass) return fail(h, GX_ERR_INVALID_ARG, "null array");
  cudaSetDevice(h->device);
  h->resident = false;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const uint32_t np = potential_partials(static_cast<uint32_t>(n));
  launch_potential_f64(static_cast<uint32_t>(n), b.pos, b.mass, h->g, h->eps, h->ar.diag_partial, np, h->stream);
  std::vector<double> part(np);
  GX_CK(h, cudaMemcpyAsync(part.data(), h->ar.diag_partial, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  GX_CK(h, cudaStreamSynchronize(h->stream));
  double u = 0.0;
  for (double v : part) u += v;
  *out = u;
  return GX_OK;
}

int gx_direct_sum_f64(gx_handle* h, size_t n, const double* pos, const double* mass, size_t n_targets,
                      const uint32_t* targets, double* acc_out) {
  if (!h || !pos || !mass || !acc_out) return GX_ERR_INVALID_ARG;
  if (n == 0) return GX_OK;
  if (!targets) n_targets = n;
  for (size_t t = 0; targets && t < n_targets; ++t)
    if (targets[t] >= n) return fail(h, GX_ERR_INVALID_ARG, "target index out of range");
  cudaSetDevice(h->device);
  h->resident = false;
  int rc = layout(h, std::max(n, n_targets), 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  uint32_t* d_t = nullptr;
  if (targets) {
    d_t = b.keys_alt;
    GX_CK(h, cudaMemcpyAsync(d_t, targets, n_targets * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  }
  launch_direct_sum_f64(static_cast<uint32_t>(n), b.pos, b.mass, h->g, h->eps, static_cast<uint32_t>(n_targets), d_t,
                        b.acc, h->stream);
  GX_CK(h, cudaMemcpyAsync(acc_out, b.acc, 3 * n_targets * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  GX_CK(h, cudaStreamSynchronize(h->stream));
  return GX_OK;
}

// ---- resident ----------------------------------------------------------------------
namespace {
// GpuResidentLeapfrog::upload (gpu_resident.rs:1685-1800); `gas` (ascending global
// indices) and u (per particle, nullable) put the state in gas mode.
int upload_impl(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                const std::vector<uint32_t>* gas, const double* u) {
  cudaSetDevice(h->device);
  if (h->step_graph) {  // captured for the previous state (its gas map and SPH buffers)
    cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
  }
  h->resident_gas = false;
  h->n = n;
  h->time = 0.0;
  h->pending_kick = false;
  h->resident = true;
  if (n == 0) return GX_OK;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(b.vel, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  h->sph_host_hint_ngas = 0;
  if (gas && !gas->empty()) {
    // the gas map is rebuilt from the species at every upload (gpu_resident_sph.rs:170-194)
    h->sph.gas_idx_host = *gas;
    GX_CK(h, sph_reserve(h->sph, gas->size(), false, 0.0, h->stream));
    if (u) {
      std::vector<double> gu(gas->size());
      for (size_t k = 0; k < gas->size(); ++k) gu[k] = u[(*gas)[k]];
      GX_CK(h, cudaMemcpy(h->sph.gu, gu.data(), gu.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    h->resident_gas = true;
  }
  if (n == 1) {
    GX_CK(h, cudaMemsetAsync(b.acc, 0, 3 * sizeof(double), h->stream));
    if (h->resident_gas)
      sph_enqueue_force(h->sph, b.pos, b.vel, b.mass, b.acc, true, true, b.ctl, h->stream);
    return finish(h, false);
  }
  // Prime a(x0) (gpu_resident.rs:1793-1799).
  enqueue_force(h, b, 0, 0, stats_on(h));
  h->stats.n = n;
  return finish(h, stats_on(h));
}
}  // namespace

int gx_upload(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (n && (!pos || !vel || !mass)) return fail(h, GX_ERR_INVALID_ARG, "null array");
  return upload_impl(h, n, pos, vel, mass, nullptr, nullptr);
}

namespace {
int step_enqueue(gx_handle* h, double dt, uint64_t steps) {
  if (!h->resident) return fail(h, GX_ERR_STATE, "step before upload");
  if (h->n == 0 || steps == 0) {
    h->time += static_cast<double>(steps) * dt;
    return GX_OK;
  }
  int rc = layout(h, h->n, dt);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  if (h->n == 1) {
    // No force on a lone particle: kick is zero, drift x += v dt each step.
    for (uint64_t s = 0; s < steps; ++s) launch_kick_drift_bbox(b, 1, 0, h->stream);
    h->time += static_cast<double>(steps) * dt;
    return GX_OK;
  }
  uint64_t s = 0;
  const bool timed = stats_on(h);
  if (!h->pending_kick || timed) {
    // First step after upload/snapshot (no deferred closing kick) runs eagerly.
    enqueue_force(h, b, 1, h->pending_kick ? 1 : 0, timed);
    h->pending_kick = true;
    h->time += dt;
    s = 1;
  }
  if (s < steps) {
    if (timed) {
      for (; s < steps; ++s) {
        enqueue_force(h, b, 1, 1, true);
        h->time += dt;
      }
      return GX_OK;
    }
    if (!h->step_graph) {
      cudaGraph_t g = nullptr;
      GX_CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      enqueue_force(h, b, 1, 1, false);
      h->launches -= 1;
      GX_CK(h, cudaStreamEndCapture(h->stream, &g));
      cudaError_t e = cudaGraphInstantiate(&h->step_graph, g, 0);
      cudaGraphDestroy(g);
      GX_CK(h, e);
    }
    for (; s < steps; ++s) {
      GX_CK(h, cudaGraphLaunch(h->step_graph, h->stream));
      h->launches += 1;
      h->time += dt;
    }
  }
  return GX_OK;
}
}  // namespace

int gx_step_many_async(gx_handle* h, double dt, uint64_t steps) {
  if (!h) return GX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  return step_enqueue(h, dt, steps);
}

int gx_step_many(gx_handle* h, double dt, uint64_t steps) {
  if (!h) return GX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  int rc = step_enqueue(h, dt, steps);
  if (rc) return rc;
  return finish(h, stats_on(h));  // stage times of the last step when they are on
}

int gx_step(gx_handle* h, double dt) { return gx_step_many(h, dt, 1); }

int gx_step_many_timed(gx_handle* h, double dt, uint64_t steps, float* ms_out) {
  if (!h || !ms_out) return GX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  GX_CK(h, cudaEventRecord(h->ev[5], h->stream));
  int rc = step_enqueue(h, dt, steps);
  if (rc) return rc;
  GX_CK(h, cudaEventRecord(h->ev[4], h->stream));
  rc = finish(h, false);
  if (rc) return rc;
  GX_CK(h, cudaEventElapsedTime(ms_out, h->ev[5], h->ev[4]));
  return GX_OK;
}

int gx_kdk_step_host(gx_handle* h, size_t n, double* pos, double* vel, const double* mass, double* acc,
                     int* primed, double dt) {
  if (!h || !primed) return GX_ERR_INVALID_ARG;
  if (n == 0) return GX_OK;
  if (!pos || !vel || !mass || !acc) return fail(h, GX_ERR_INVALID_ARG, "null array");
  int rc;
  if (!*primed) {
    rc = gx_accelerations(h, n, pos, mass, acc);
    if (rc) return rc;
    *primed = 1;
  }
  const double half = 0.5 * dt;
  if (n == 1) {  // a lone particle: no force
    for (size_t i = 0; i < 3; ++i) {
      vel[i] = vel[i] + acc[i] * half;
      pos[i] = pos[i] + vel[i] * dt;
      acc[i] = 0.0;
      vel[i] = vel[i] + acc[i] * half;
    }
    return GX_OK;
  }
  // Opening half kick and drift (integrator.rs:59-67: v += a h, then x += v dt, each
  // rounded separately), on all host threads and in chunks, each chunk's positions
  // copied to the device while the next chunk is computed. Then the force as in
  // gx_accelerations, and the closing half kick of each chunk of accelerations as soon
  // as that chunk is back (after the error word, so nothing is kicked by a failed step).
  cudaSetDevice(h->device);
  h->resident = false;
  rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const size_t chunk = std::max<size_t>(size_t{1} << 16, (n + 7) / 8);
  for (size_t c0 = 0; c0 < n; c0 += chunk) {
    const long long i0 = static_cast<long long>(3 * c0);
    const long long i1 = static_cast<long long>(3 * std::min(n, c0 + chunk));
#pragma omp parallel for schedule(static)
    for (long long i = i0; i < i1; ++i) {
      vel[i] = vel[i] + acc[i] * half;
      pos[i] = pos[i] + vel[i] * dt;
    }
    GX_CK(h, cudaMemcpyAsync(b.pos + i0, pos + i0, (i1 - i0) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }
  enqueue_force(h, b, 0, 0, stats_on(h));
  GX_CK(h, cudaMemcpyAsync(h->ctl_host, b.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->stream));
  int nch = 0;
  for (size_t c0 = 0; c0 < n; c0 += chunk, ++nch) {
    const size_t i0 = 3 * c0, i1 = 3 * std::min(n, c0 + chunk);
    GX_CK(h, cudaMemcpyAsync(acc + i0, b.acc + i0, (i1 - i0) * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    GX_CK(h, cudaEventRecord(h->chunk_ev[nch], h->stream));
  }
  h->stats.n = n;
  for (int c = 0; c < nch; ++c) {
    GX_CK(h, cudaEventSynchronize(h->chunk_ev[c]));
    if (c == 0 && h->ctl_host->err) return finish(h, stats_on(h));  // the step failed: report, no kick
    const long long i0 = static_cast<long long>(3 * (size_t)c * chunk);
    const long long i1 = static_cast<long long>(3 * std::min(n, ((size_t)c + 1) * chunk));
#pragma omp parallel for schedule(static)
    for (long long i = i0; i < i1; ++i) vel[i] = vel[i] + acc[i] * half;
  }
  return finish(h, stats_on(h));
}

int gx_host_alloc(size_t bytes, void** out) {
  if (!out) return GX_ERR_INVALID_ARG;
  cudaError_t e = cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    set_global_err(std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
    *out = nullptr;
    return GX_ERR_CUDA;
  }
  return GX_OK;
}

void gx_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

namespace {
int apply_pending(gx_handle* h) {
  if (h->pending_kick && h->n > 1) {
    launch_kick_half(h->ar.b, h->stream);
    h->pending_kick = false;
  }
  return GX_OK;
}
}  // namespace

int gx_snapshot(gx_handle* h, double* pos_out, double* vel_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (!h->resident) return fail(h, GX_ERR_STATE, "snapshot before upload");
  if (h->n == 0) return GX_OK;
  cudaSetDevice(h->device);
  apply_pending(h);
  const size_t bytes = 3 * h->n * sizeof(double);
  if (pos_out) GX_CK(h, cudaMemcpyAsync(pos_out, h->ar.b.pos, bytes, cudaMemcpyDeviceToHost, h->stream));
  if (vel_out) GX_CK(h, cudaMemcpyAsync(vel_out, h->ar.b.vel, bytes, cudaMemcpyDeviceToHost, h->stream));
  return finish(h, false);
}

int gx_resident_accelerations(gx_handle* h, double* acc_out) {
  if (!h || !acc_out) return GX_ERR_INVALID_ARG;
  if (!h->resident) return fail(h, GX_ERR_STATE, "no resident state");
  if (h->n == 0) return GX_OK;
  cudaSetDevice(h->device);
  GX_CK(h, cudaMemcpyAsync(acc_out, h->ar.b.acc, 3 * h->n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return finish(h, false);
}

int gx_time(const gx_handle* h, double* t_out) {
  if (!h || !t_out) return GX_ERR_INVALID_ARG;
  *t_out = h->time;
  return GX_OK;
}

int gx_len(const gx_handle* h, size_t* n_out) {
  if (!h || !n_out) return GX_ERR_INVALID_ARG;
  *n_out = h->resident ? h->n : 0;
  return GX_OK;
}

int gx_launches(const gx_handle* h, uint64_t* out) {
  if (!h || !out) return GX_ERR_INVALID_ARG;
  *out = h->launches;
  return GX_OK;
}

int gx_diagnostics(gx_handle* h, int with_potential, double* out) {
  if (!h || !out) return GX_ERR_INVALID_ARG;
  if (!h->resident) return fail(h, GX_ERR_STATE, "no resident state");
  for (int i = 0; i < 8; ++i) out[i] = 0.0;
  if (h->n == 0) return GX_OK;
  cudaSetDevice(h->device);
  apply_pending(h);
  const uint32_t n = static_cast<uint32_t>(h->n);
  StepBufs& b = h->ar.b;
  const uint32_t nd = std::min<uint32_t>(potential_partials(n), 1024u);
  launch_diag_sums(n, b.pos, b.vel, b.mass, h->ar.diag_partial, nd, h->stream);
  std::vector<double> part(7 * nd);
  GX_CK(h, cudaMemcpyAsync(part.data(), h->ar.diag_partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream));
  GX_CK(h, cudaStreamSynchronize(h->stream));
  for (uint32_t i = 0; i < nd; ++i) {
    out[0] += part[7 * i];
    for (int c = 0; c < 3; ++c) {
      out[2 + c] += part[7 * i + 1 + c];
      out[5 + c] += part[7 * i + 4 + c];
    }
  }
  if (with_potential && n > 1) {
    const uint32_t np = potential_partials(n);
    launch_potential_f64(n, b.pos, b.mass, h->g, h->eps, h->ar.diag_partial, np, h->stream);
    std::vector<double> pp(np);
    GX_CK(h, cudaMemcpyAsync(pp.data(), h->ar.diag_partial, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    GX_CK(h, cudaStreamSynchronize(h->stream));
    for (double v : pp) out[1] += v;
  }
  return finish(h, false);
}

int gx_autotune(gx_handle* h, uint32_t repeats, gx_tuning* best, gx_tuning* tried, uint32_t* n_tried) {
  if (!h || !best) return GX_ERR_INVALID_ARG;
  if (!h->resident) return fail(h, GX_ERR_STATE, "autotune before upload");
  if (h->n < 2) return fail(h, GX_ERR_STATE, "autotune needs at least two particles");
  cudaSetDevice(h->device);
  int rc = finish(h, false);  // nothing of the caller's may still be in flight
  if (rc) return rc;
  const gx_options user = h->opt;
  const uint32_t reps = repeats ? repeats : 3;
  WalkCfg base = walk_cfg(h);
  // the FP64 walk has one grouping; a grouping fixed by the options is the only one tried
  std::vector<gx_tuning> cand = tune_candidates(base, true, h->opt.precision != GX_PREC_F64 && user.walk_group == 0);
  if (user.walk_group)
    for (gx_tuning& c : cand) c.walk_group = user.walk_group;
  StepBufs& b = h->ar.b;
  const double dt_keep = h->dt_layout;
  int best_i = -1;
  for (size_t i = 0; i < cand.size() && rc == GX_OK; ++i) {
    h->opt.walk_block = cand[i].walk_block;
    h->opt.walk_ctas_per_sm = cand[i].walk_ctas_per_sm;
    h->opt.walk_group = cand[i].walk_group;
    rc = layout(h, h->n, dt_keep);  // walk items of this grouping
    if (rc) break;
    // Force evaluations on the current positions recompute a(x) bit for bit, so the
    // resident state is untouched whatever the candidate.
    enqueue_force(h, b, 0, 0, false);
    rc = finish(h, false);
    std::vector<float> ms;
    for (uint32_t r = 0; r < reps && rc == GX_OK; ++r) {
      cudaEventRecord(h->ev[5], h->stream);
      enqueue_force(h, b, 0, 0, false);
      cudaEventRecord(h->ev[4], h->stream);
      rc = finish(h, false);
      float t = 0.f;
      if (rc == GX_OK) cudaEventElapsedTime(&t, h->ev[5], h->ev[4]);
      ms.push_back(t);
    }
    if (rc) break;
    std::sort(ms.begin(), ms.end());
    cand[i].ms = ms[ms.size() / 2];
    if (best_i < 0 || cand[i].ms < cand[best_i].ms) best_i = static_cast<int>(i);
  }
  h->opt = user;
  if (h->step_graph) {  // captured with the previous launch configuration
    cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
  }
  if (rc) {
    layout(h, h->n, dt_keep);
    return rc;
  }
  *best = cand[best_i];
  // The sort's digit width (30-bit keys): time the sort stage of force evaluations with
  // the chosen walk launch, 8-bit then 10-bit digits.
  best->radix_bits = kRadixBits;
  if (!(user.flags & GX_FLAG_MORTON63)) {
    float best_sort = 0.f;
    for (uint32_t bits : {static_cast<uint32_t>(kRadixBits), static_cast<uint32_t>(kRadixBitsWide)}) {
      h->opt.walk_block = best->walk_block;
      h->opt.walk_ctas_per_sm = best->walk_ctas_per_sm;
      h->opt.walk_group = best->walk_group;
      h->opt.radix_bits = bits;
      rc = layout(h, h->n, dt_keep);
      std::vector<float> ms;
      for (uint32_t r = 0; r <= reps && rc == GX_OK; ++r) {
        enqueue_force(h, b, 0, 0, true);
        rc = finish(h, false);
        float t = 0.f;
        if (rc == GX_OK) cudaEventElapsedTime(&t, h->ev[1], h->ev[2]);
        if (r > 0) ms.push_back(t);  // the first evaluation warms the new layout
      }
      if (rc) break;
      std::sort(ms.begin(), ms.end());
      const float med = ms[ms.size() / 2];
      if (bits == kRadixBits || med < best_sort) {
        best_sort = med;
        best->radix_bits = bits;
      }
    }
    best->sort_ms = best_sort;
    h->opt = user;
    if (h->step_graph) {
      cudaGraphExecDestroy(h->step_graph);
      h->step_graph = nullptr;
    }
    if (rc) {
      layout(h, h->n, dt_keep);
      return rc;
    }
  }
  // A grouping fixed by the options was not tuned: the table's entry leaves it open (0),
  // so handles of this N bucket with the grouping open keep their default one.
  gx_tuning rec = *best;
  if (user.walk_group) rec.walk_group = 0;
  tuned_store(h->device, user, 0, h->n, rec);
  rc = layout(h, h->n, dt_keep);  // the tuned grouping and digit width (unless the options fix them)
  if (rc) return rc;
  // The resident accelerations are those of the configuration the handle now uses (the
  // grouping sets the FP32 summation order), not of the last candidate timed.
  enqueue_force(h, b, 0, 0, false);
  rc = finish(h, false);
  if (rc) return rc;
  if (tried) std::copy(cand.begin(), cand.end(), tried);
  if (n_tried) *n_tried = static_cast<uint32_t>(cand.size());
  return GX_OK;
}

int gx_tuning_lookup(int device, size_t n, const gx_options* opt, int batched, gx_tuning* out) {
  if (!out) return GX_ERR_INVALID_ARG;
  gx_options o{};
  if (opt && opt->struct_size) o = *opt;
  int dev = device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return GX_ERR_NO_DEVICE;
  return tuned_lookup(dev, o, batched, n, out) ? GX_OK : GX_ERR_STATE;
}

int gx_get_stats(const gx_handle* h, gx_stats* out) {
  if (!h || !out) return GX_ERR_INVALID_ARG;
  *out = h->stats;
  return GX_OK;
}

// ---- stage entry points -------------------------------------------------------------
int gx_stage_morton(gx_handle* h, size_t n, const double* pos, uint32_t* lanes_out, uint32_t* codes_out,
                    double* bounds_out) {
  if (!h || !pos || !codes_out) return GX_ERR_INVALID_ARG;
  if (h->opt.flags & GX_FLAG_MORTON63) return fail(h, GX_ERR_INVALID_ARG, "stage entry points take 30-bit keys");
  if (n == 0) return fail(h, GX_ERR_INVALID_ARG, "reference_morton requires a non-empty system");
  cudaSetDevice(h->device);
  h->resident = false;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemsetAsync(b.zero_begin, 0, b.zero_bytes, h->stream));
  launch_kick_drift_bbox(b, 0, 0, h->stream);
  // Lanes (3n u32) are staged in the walk records, unused by this stage.
  uint32_t* d_lanes = lanes_out ? reinterpret_cast<uint32_t*>(b.pairs) : nullptr;
  launch_morton_hist(b, d_lanes, h->stream);
  GX_CK(h, cudaMemcpyAsync(codes_out, b.codes, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  if (lanes_out)
    GX_CK(h, cudaMemcpyAsync(lanes_out, d_lanes, 3 * n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  Bounds bd;
  GX_CK(h, cudaMemcpyAsync(&bd, b.bounds, sizeof(Bounds), cudaMemcpyDeviceToHost, h->stream));
  rc = finish(h, false);
  if (rc) return rc;
  if (bounds_out) {
    bounds_out[0] = bd.bmin[0];
    bounds_out[1] = bd.bmin[1];
    bounds_out[2] = bd.bmin[2];
    bounds_out[3] = bd.size;
    bounds_out[4] = bd.scale;
  }
  return GX_OK;
}

int gx_stage_sort(gx_handle* h, size_t n, const uint32_t* codes, uint32_t* order_out, uint32_t* sorted_codes_out) {
  if (!h || (n && (!codes || !order_out))) return GX_ERR_INVALID_ARG;
  if (h->opt.flags & GX_FLAG_MORTON63) return fail(h, GX_ERR_INVALID_ARG, "stage entry points take 30-bit keys");
  if (n == 0) return GX_OK;
  for (size_t i = 0; i < n; ++i)
    if (codes[i] >= (1u << 30)) return fail(h, GX_ERR_INVALID_ARG, "codes must be 30-bit");
  cudaSetDevice(h->device);
  h->resident = false;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.codes, codes, n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemsetAsync(b.zero_begin, 0, b.zero_bytes, h->stream));
  launch_code_hist(b, h->stream);
  launch_sort(b, h->stream);
  GX_CK(h, cudaMemcpyAsync(order_out, b.order, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  if (sorted_codes_out)
    GX_CK(h, cudaMemcpyAsync(sorted_codes_out, b.codes, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  return finish(h, false);
}

int gx_stage_build(gx_handle* h, size_t n, const uint32_t* sorted_codes, const double* sorted_pos,
                   const double* sorted_mass, uint32_t* left, uint32_t* right, uint32_t* parent, double* aabb_min,
                   double* aabb_max, double* com, double* mass, double* quad_out) {
  if (!h || !sorted_codes || !sorted_pos || !sorted_mass || !parent) return GX_ERR_INVALID_ARG;
  if (n == 0) return fail(h, GX_ERR_INVALID_ARG, "reference_karras requires a non-empty system");
  if (n > 1 && (!left || !right)) return GX_ERR_INVALID_ARG;
  if (h->opt.flags & GX_FLAG_MORTON63) return fail(h, GX_ERR_INVALID_ARG, "stage entry points take 30-bit keys");
  if (quad_out && h->opt.multipole != GX_MULTIPOLE_QUAD)
    return fail(h, GX_ERR_INVALID_ARG, "quadrupole output needs a GX_MULTIPOLE_QUAD handle");
  cudaSetDevice(h->device);
  h->resident = false;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  std::vector<uint32_t> iota(n);
  for (size_t i = 0; i < n; ++i) iota[i] = static_cast<uint32_t>(i);
  GX_CK(h, cudaMemcpyAsync(b.codes, sorted_codes, n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(b.order, iota.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(b.pos, sorted_pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, sorted_mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const int quad = h->opt.multipole == GX_MULTIPOLE_QUAD && h->opt.precision != GX_PREC_F64;
  GX_CK(h, cudaMemsetAsync(b.bounds, 0, sizeof(Bounds), h->stream));  // no Morton stage here
  launch_build(b, quad, h->opt.precision == GX_PREC_F64, h->stream);
  std::vector<uint2> kids(n > 1 ? n - 1 : 1);
  std::vector<Agg64> agg(n > 1 ? n - 1 : 1);
  std::vector<double4> leaf(n);
  std::vector<double> q64(quad ? 6 * n : 0);
  if (n > 1) {
    GX_CK(h, cudaMemcpyAsync(kids.data(), b.kids, (n - 1) * sizeof(uint2), cudaMemcpyDeviceToHost, h->stream));
    GX_CK(h, cudaMemcpyAsync(agg.data(), b.agg64, (n - 1) * sizeof(Agg64), cudaMemcpyDeviceToHost, h->stream));
    if (quad)
      GX_CK(h, cudaMemcpyAsync(q64.data(), b.q64, 6 * (n - 1) * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  GX_CK(h, cudaMemcpyAsync(parent, b.parent, (2 * n - 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  GX_CK(h, cudaMemcpyAsync(leaf.data(), b.leaf64, n * sizeof(double4), cudaMemcpyDeviceToHost, h->stream));
  rc = finish(h, false);
  if (rc) return rc;
  for (size_t i = 0; i + 1 < n; ++i) {
    left[i] = kids[i].x;
    right[i] = kids[i].y;
  }
  for (size_t u = 0; u < 2 * n - 1; ++u) {
    double mn[3], mx[3], cm[3], m;
    if (u < n) {
      const double4 l = leaf[u];
      mn[0] = mx[0] = cm[0] = l.x;
      mn[1] = mx[1] = cm[1] = l.y;
      mn[2] = mx[2] = cm[2] = l.z;
      m = l.w;
    } else {
      const Agg64& a = agg[u - n];
      for (int c = 0; c < 3; ++c) {
        mn[c] = a.mn[c];
        mx[c] = a.mx[c];
        cm[c] = a.com[c];
      }
      m = a.m;
    }
    for (int c = 0; c < 3; ++c) {
      if (aabb_min) aabb_min[3 * u + c] = mn[c];
      if (aabb_max) aabb_max[3 * u + c] = mx[c];
      if (com) com[3 * u + c] = cm[c];
    }
    if (mass) mass[u] = m;
    if (quad_out)
      for (int c = 0; c < 6; ++c) quad_out[6 * u + c] = u < n ? 0.0 : q64[6 * (u - n) + c];
  }
  return GX_OK;
}

// ---- SPH on the gas subset ------------------------------------------------------------
void gx_sph_default_params(gx_sph_params* out) {
  if (!out) return;
  out->n_ngb = 48.0;
  out->h_tol_rel = 1e-3;
  out->eos = GX_EOS_ISOTHERMAL;
  out->warm_start = 1;
  out->c_s = 1.0;
  out->gamma = 5.0 / 3.0;
  out->alpha = 1.0;
  out->beta = 2.0;
  out->visc_eps2 = 0.01;
}

namespace {

// Species column -> gas map (ascending global index); kind values other than 0 / 1 are
// rejected (core/src/state.rs:17-22 has two species).
int gas_map(gx_handle* h, size_t n, const uint8_t* kind, std::vector<uint32_t>& gas) {
  gas.clear();
  if (!kind) return GX_OK;
  for (size_t i = 0; i < n; ++i) {
    if (kind[i] > 1) return fail(h, GX_ERR_INVALID_ARG, "kind must be 0 (collisionless) or 1 (gas)");
    if (kind[i] == 1) gas.push_back(static_cast<uint32_t>(i));
  }
  return GX_OK;
}

int need_sph(gx_handle* h) {
  if (!h->sph.enabled) return fail(h, GX_ERR_STATE, "SPH call without gas mode (gx_sph_enable)");
  return GX_OK;
}

double dec_max_host(unsigned long long e) {
  const unsigned long long b = (e >> 63) ? (e & 0x7FFFFFFFFFFFFFFFull) : ~e;
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
}

// The arena and gas map of a host-state SPH call on n particles whose gas rows are
// `gas` (identity when gas is null): the resident state is dropped.
int host_sph_setup(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                   const std::vector<uint32_t>* gas, bool keep_hint, bool host_s_est) {
  h->resident = false;
  h->resident_gas = false;
  int rc = layout(h, n, 0.0);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  GX_CK(h, cudaMemcpyAsync(b.pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (vel) GX_CK(h, cudaMemcpyAsync(b.vel, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (mass) GX_CK(h, cudaMemcpyAsync(h->ar.mass_rw, mass, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (gas) {
    h->sph.gas_idx_host = *gas;
  } else {
    h->sph.gas_idx_host.resize(n);
    for (size_t i = 0; i < n; ++i) h->sph.gas_idx_host[i] = static_cast<uint32_t>(i);
  }
  const size_t ng = h->sph.gas_idx_host.size();
  const double s_est = host_s_est ? sph_host_s_est(ng, pos, h->sph.gas_idx_host.data()) : 0.0;
  GX_CK(h, sph_reserve(h->sph, ng, keep_hint, s_est, h->stream));
  return GX_OK;
}

// max_stable_dt, sf_fields and coupled_pairs are &self in the reference
// (solvers/src/sph/gravity_sph.rs:351-382): they leave the warm-start smoothing lengths
// and the individual-timestep path's scratch as they were. Each runs its own cold-start
// density solve over the device h; the keeper saves h (host copy) before it and puts it
// back after, with the hint and scratch flags, so the next force call warm-starts and the
// active path reads its stale neighbours as if no diagnostic had run.
struct SphScratchKeeper {
  gx_handle* h;
  size_t ng, hint, rho_ngas;
  uint64_t rho_gen, gen;
  std::vector<double> hs;
  SphScratchKeeper(gx_handle* h_, size_t ng_)
      : h(h_), ng(ng_), hint(h_->sph_host_hint_ngas), rho_ngas(h_->sph_rho_scratch_ngas), rho_gen(h_->sph_rho_gen),
        gen(h_->sph.alloc_gen) {}
  int save() {
    if (ng && hint == ng && h->sph.hs && h->sph.cap >= ng) {
      hs.resize(ng);
      GX_CK(h, cudaMemcpyAsync(hs.data(), h->sph.hs, ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      GX_CK(h, cudaStreamSynchronize(h->stream));
    }
    h->sph_host_hint_ngas = 0;  // until restored: a failed diagnostic leaves no stale hint
    return GX_OK;
  }
  int restore() {
    const bool same = h->sph.alloc_gen == gen && h->sph.n_gas == ng;
    if (same && !hs.empty()) {
      GX_CK(h, cudaMemcpyAsync(h->sph.hs, hs.data(), ng * sizeof(double), cudaMemcpyHostToDevice, h->stream));
      GX_CK(h, cudaStreamSynchronize(h->stream));
      h->sph_host_hint_ngas = hint;
    }
    h->sph_rho_scratch_ngas = same ? rho_ngas : 0;
    h->sph_rho_gen = rho_gen;
    return GX_OK;
  }
};

int put_gas(gx_handle* h, double* dst, const double* src, size_t count) {
  if (src) GX_CK(h, cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  return GX_OK;
}

}  // namespace

int gx_sph_enable(gx_handle* h, const gx_sph_params* params) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (!params) return GX_OK;
  const gx_sph_params& p = *params;
  if (!(p.n_ngb > 32.0 / 3.0))
    return fail(h, GX_ERR_INVALID_ARG, "n_ngb must exceed the self-term floor 32/3 (density.rs:172-176)");
  if (!(p.h_tol_rel > 0.0) || (p.eos != GX_EOS_ISOTHERMAL && p.eos != GX_EOS_ADIABATIC) || !(p.c_s >= 0.0) ||
      (p.eos == GX_EOS_ADIABATIC && !(p.gamma > 1.0)) || !(p.visc_eps2 >= 0.0))
    return fail(h, GX_ERR_INVALID_ARG, "invalid gx_sph_params");
  h->sph.p = p;
  h->sph.enabled = true;
  h->sph_host_hint_ngas = 0;
  return GX_OK;
}

int gx_upload_species(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                      const uint8_t* kind, const double* u) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (n && (!pos || !vel || !mass)) return fail(h, GX_ERR_INVALID_ARG, "null array");
  std::vector<uint32_t> gas;
  int rc = gas_map(h, n, kind, gas);
  if (rc) return rc;
  if (!h->sph.enabled || gas.empty()) return upload_impl(h, n, pos, vel, mass, nullptr, nullptr);
  if (h->sph.p.eos != GX_EOS_ISOTHERMAL)
    return fail(h, GX_ERR_INVALID_ARG, "the resident gas mode runs the isothermal EOS (u is not evolved)");
  return upload_impl(h, n, pos, vel, mass, &gas, u);
}

int gx_gas_count(const gx_handle* h, size_t* n_gas_out) {
  if (!h || !n_gas_out) return GX_ERR_INVALID_ARG;
  *n_gas_out = h->resident_gas ? h->sph.n_gas : 0;
  return GX_OK;
}

int gx_snapshot_gas_density(gx_handle* h, uint32_t* gas_idx_out, double* rho_out, double* h_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  if (!h->resident) return fail(h, GX_ERR_STATE, "no resident state");
  if (!h->resident_gas) return GX_OK;
  cudaSetDevice(h->device);
  const size_t ng = h->sph.n_gas;
  if (gas_idx_out) std::memcpy(gas_idx_out, h->sph.gas_idx_host.data(), ng * sizeof(uint32_t));
  if (rho_out) GX_CK(h, cudaMemcpyAsync(rho_out, h->sph.rho, ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (h_out) GX_CK(h, cudaMemcpyAsync(h_out, h->sph.hs, ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return finish(h, false);
}

int gx_snapshot_gas_accel(gx_handle* h, double* acc_out, double* dudt_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  if (!h->resident) return fail(h, GX_ERR_STATE, "no resident state");
  if (!h->resident_gas) return GX_OK;
  cudaSetDevice(h->device);
  const size_t ng = h->sph.n_gas;
  if (acc_out)
    GX_CK(h, cudaMemcpyAsync(acc_out, h->sph.gacc, 3 * ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (dudt_out)
    GX_CK(h, cudaMemcpyAsync(dudt_out, h->sph.dudt, ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return finish(h, false);
}

int gx_snapshot_accel(gx_handle* h, double* acc_out) { return gx_resident_accelerations(h, acc_out); }

namespace {
int resident_cfl(gx_handle* h, double c_cfl, double* dt_out, double* min_out) {
  if (int rc = need_sph(h)) return rc;
  if (!h->resident) return fail(h, GX_ERR_STATE, "no resident state");
  if (!h->resident_gas || h->sph.n_gas == 0) {
    if (min_out) *min_out = std::numeric_limits<double>::infinity();
    return GX_OK;
  }
  cudaSetDevice(h->device);
  apply_pending(h);  // the current velocities
  const StepBufs& b = h->ar.b;
  sph_enqueue_cfl(h->sph, b.pos, b.vel, c_cfl, false, b.ctl, h->stream);
  unsigned long long enc = 0;
  GX_CK(h, cudaMemcpyAsync(&enc, &h->sph.sc->min_dt_enc, sizeof enc, cudaMemcpyDeviceToHost, h->stream));
  if (dt_out)
    GX_CK(h, cudaMemcpyAsync(dt_out, h->sph.dtv, h->sph.n_gas * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  int rc = finish(h, false);
  if (rc) return rc;
  if (min_out) *min_out = -dec_max_host(enc);
  return GX_OK;
}
}  // namespace

int gx_min_stable_dt(gx_handle* h, double c_cfl, double* out) {
  if (!h || !out) return GX_ERR_INVALID_ARG;
  return resident_cfl(h, c_cfl, nullptr, out);
}

int gx_snapshot_gas_dt(gx_handle* h, double c_cfl, double* dt_out) {
  if (!h || !dt_out) return GX_ERR_INVALID_ARG;
  return resident_cfl(h, c_cfl, dt_out, nullptr);
}

int gx_sph_accelerations(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                         const uint8_t* kind, const double* u, double* acc_out) {
  return gx_sph_accel_and_dudt(h, n, pos, vel, mass, kind, u, acc_out, nullptr);
}

int gx_sph_accel_and_dudt(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                          const uint8_t* kind, const double* u, double* acc_out, double* dudt_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  if (n == 0) return GX_OK;
  if (!pos || !vel || !mass || !acc_out) return fail(h, GX_ERR_INVALID_ARG, "null array");
  std::vector<uint32_t> gas;
  int rc = gas_map(h, n, kind, gas);
  if (rc) return rc;
  cudaSetDevice(h->device);
  const bool keep = h->sph.p.warm_start && !gas.empty() && h->sph_host_hint_ngas == gas.size();
  h->sph_host_hint_ngas = 0;
  rc = host_sph_setup(h, n, pos, vel, mass, &gas, keep, true);
  if (rc) return rc;
  StepBufs& b = h->ar.b;
  if (n == 1)
    GX_CK(h, cudaMemsetAsync(b.acc, 0, 3 * sizeof(double), h->stream));
  else
    enqueue_force(h, b, 0, 0, stats_on(h));
  if (!gas.empty()) {
    if (u) {
      std::vector<double> gu(gas.size());
      for (size_t k = 0; k < gas.size(); ++k) gu[k] = u[gas[k]];
      GX_CK(h, cudaMemcpy(h->sph.gu, gu.data(), gu.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    sph_enqueue_force(h->sph, b.pos, b.vel, b.mass, b.acc, true, true, b.ctl, h->stream);
  }
  GX_CK(h, cudaMemcpyAsync(acc_out, b.acc, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  std::vector<double> gdudt;
  if (dudt_out && !gas.empty()) {
    gdudt.resize(gas.size());
    GX_CK(h, cudaMemcpyAsync(gdudt.data(), h->sph.dudt, gas.size() * sizeof(double), cudaMemcpyDeviceToHost,
                             h->stream));
  }
  h->stats.n = n;
  rc = finish(h, stats_on(h));
  if (rc != GX_OK) return rc;
  h->sph_host_hint_ngas = gas.size();
  if (dudt_out) {
    std::fill(dudt_out, dudt_out + n, 0.0);
    for (size_t k = 0; k < gas.size(); ++k) dudt_out[gas[k]] = gdudt[k];
  }
  return GX_OK;
}

int gx_sph_accelerations_active(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                                const uint8_t* kind, const double* u, size_t n_active, const uint32_t* active,
                                double* acc_out) {
  return gx_sph_accel_and_dudt_active(h, n, pos, vel, mass, kind, u, n_active, active, acc_out, nullptr);
}

int gx_sph_accel_and_dudt_active(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                                 const uint8_t* kind, const double* u, size_t n_active, const uint32_t* active,
                                 double* acc_out, double* dudt_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  if (n == 0) return GX_OK;
  if (!pos || !vel || !mass || !acc_out || (n_active && !active)) return fail(h, GX_ERR_INVALID_ARG, "null array");
  for (size_t i = 0; i < n_active; ++i)
    if (active[i] >= n) return fail(h, GX_ERR_INVALID_ARG, "active index out of range");
  std::vector<uint32_t> gas;
  int rc = gas_map(h, n, kind, gas);
  if (rc) return rc;
  cudaSetDevice(h->device);
  const size_t ng = gas.size();
  // gravity_sph.rs:88-150 (active_gas): a scratch that is unset for this gas count forces a
  // refresh of every gas particle, warm-started from h when h is set
  const bool h_set0 = ng && h->sph_host_hint_ngas == ng;
  const bool rho_set0 = ng && h->sph_rho_scratch_ngas == ng;
  const uint64_t gen0 = h->sph.alloc_gen;
  h->sph_host_hint_ngas = 0;
  h->sph_rho_scratch_ngas = 0;
  // density_adaptive_active always warm-starts from the persistent h (gravity_sph.rs:
  // 247-286), whatever warm_start says
  rc = host_sph_setup(h, n, pos, vel, mass, &gas, h_set0, true);
  if (rc) return rc;
  const bool same_alloc = h->sph.alloc_gen == gen0;  // a reallocation loses both scratches
  const bool h_set = h_set0 && same_alloc;
  const bool rho_set = rho_set0 && same_alloc && h->sph_rho_gen == gen0;
  StepBufs& b = h->ar.b;
  if (n == 1)
    GX_CK(h, cudaMemsetAsync(b.acc, 0, 3 * sizeof(double), h->stream));
  else
    enqueue_force(h, b, 0, 0, stats_on(h));
  std::vector<uint32_t> local;
  const bool all = !(h_set && rho_set);
  if (ng && !all) {
    std::vector<uint8_t> mark(ng, 0);
    std::vector<uint32_t> g2l(n, 0xFFFFFFFFu);
    for (size_t k = 0; k < ng; ++k) g2l[gas[k]] = static_cast<uint32_t>(k);
    for (size_t i = 0; i < n_active; ++i)
      if (g2l[active[i]] != 0xFFFFFFFFu) mark[g2l[active[i]]] = 1;
    for (size_t k = 0; k < ng; ++k)
      if (mark[k]) local.push_back(static_cast<uint32_t>(k));
  }
  if (ng) {
    if (u) {
      std::vector<double> gu(ng);
      for (size_t k = 0; k < ng; ++k) gu[k] = u[gas[k]];
      GX_CK(h, cudaMemcpy(h->sph.gu, gu.data(), ng * sizeof(double), cudaMemcpyHostToDevice));
    }
    // the density pass writes the refreshed rows over the active path's rho scratch
    if (rho_set)
      GX_CK(h, cudaMemcpyAsync(h->sph.rho, h->sph.rho_act, ng * sizeof(double), cudaMemcpyDeviceToDevice,
                               h->stream));
    if (!all && !local.empty())
      GX_CK(h, cudaMemcpyAsync(h->sph.targets, local.data(), local.size() * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, h->stream));
    if (all || !local.empty())
      sph_enqueue_force(h->sph, b.pos, b.vel, b.mass, b.acc, true, true, b.ctl, h->stream, nullptr,
                        all ? nullptr : h->sph.targets, static_cast<uint32_t>(local.size()), true);
    GX_CK(h, cudaMemcpyAsync(h->sph.rho_act, h->sph.rho, ng * sizeof(double), cudaMemcpyDeviceToDevice,
                             h->stream));
  }
  GX_CK(h, cudaMemcpyAsync(acc_out, b.acc, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  std::vector<double> gdudt;
  if (dudt_out && ng && (all || !local.empty())) {
    gdudt.resize(ng);  // per gas-local index; rows of the refreshed targets are current
    GX_CK(h, cudaMemcpyAsync(gdudt.data(), h->sph.dudt, ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  h->stats.n = n;
  rc = finish(h, stats_on(h));  // also keeps `local` alive until its copy has run
  if (rc != GX_OK) return rc;
  h->sph_host_hint_ngas = ng;
  h->sph_rho_scratch_ngas = ng;
  h->sph_rho_gen = h->sph.alloc_gen;
  if (dudt_out) {
    // gravity_sph.rs:288-319: zero on every row, the refreshed gas rows overwritten
    std::fill(dudt_out, dudt_out + n, 0.0);
    if (!gdudt.empty()) {
      if (all)
        for (size_t k = 0; k < ng; ++k) dudt_out[gas[k]] = gdudt[k];
      else
        for (uint32_t k : local) dudt_out[gas[k]] = gdudt[k];
    }
  }
  return GX_OK;
}

int gx_sph_sf_fields(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                     const uint8_t* kind, double* rho_out, double* div_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  if (n == 0) return GX_OK;
  if (!pos || !vel || !mass || !rho_out || !div_out) return fail(h, GX_ERR_INVALID_ARG, "null array");
  std::vector<uint32_t> gas;
  int rc = gas_map(h, n, kind, gas);
  if (rc) return rc;
  std::fill(rho_out, rho_out + n, 0.0);
  std::fill(div_out, div_out + n, 0.0);
  if (gas.empty()) return GX_OK;
  cudaSetDevice(h->device);
  SphScratchKeeper keep(h, gas.size());
  if ((rc = keep.save())) return rc;
  rc = host_sph_setup(h, n, pos, vel, mass, &gas, false, true);  // a cold-start solve
  if (rc) return rc;
  const StepBufs& b = h->ar.b;
  const size_t ng = gas.size();
  sph_enqueue_force(h->sph, b.pos, b.vel, b.mass, nullptr, true, false, b.ctl, h->stream);
  sph_enqueue_divergence(h->sph, h->sph.dudt, h->stream);  // dudt is free scratch here
  std::vector<double> rho(ng), dv(ng);
  GX_CK(h, cudaMemcpyAsync(rho.data(), h->sph.rho, ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  GX_CK(h, cudaMemcpyAsync(dv.data(), h->sph.dudt, ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  rc = finish(h, false);
  if (rc) return rc;
  if ((rc = keep.restore())) return rc;
  for (size_t k = 0; k < ng; ++k) {
    rho_out[gas[k]] = rho[k];
    div_out[gas[k]] = dv[k];
  }
  return GX_OK;
}

int gx_sph_max_stable_dt(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                         const uint8_t* kind, const double* u, double c_cfl, double* dt_out, double* min_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  const double inf = std::numeric_limits<double>::infinity();
  if (dt_out) std::fill(dt_out, dt_out + n, inf);
  if (min_out) *min_out = inf;
  if (n == 0) return GX_OK;
  if (!pos || !vel || !mass) return fail(h, GX_ERR_INVALID_ARG, "null array");
  std::vector<uint32_t> gas;
  int rc = gas_map(h, n, kind, gas);
  if (rc || gas.empty()) return rc;
  cudaSetDevice(h->device);
  SphScratchKeeper keep(h, gas.size());
  if ((rc = keep.save())) return rc;
  rc = host_sph_setup(h, n, pos, vel, mass, &gas, false, true);  // cfl.rs:66: a cold-start solve
  if (rc) return rc;
  const size_t ng = gas.size();
  if (u) {
    std::vector<double> gu(ng);
    for (size_t k = 0; k < ng; ++k) gu[k] = u[gas[k]];
    GX_CK(h, cudaMemcpy(h->sph.gu, gu.data(), ng * sizeof(double), cudaMemcpyHostToDevice));
  }
  const StepBufs& b = h->ar.b;
  sph_enqueue_force(h->sph, b.pos, b.vel, b.mass, nullptr, true, false, b.ctl, h->stream);
  sph_enqueue_cfl(h->sph, b.pos, b.vel, c_cfl, true, b.ctl, h->stream);
  unsigned long long enc = 0;
  std::vector<double> dt(ng);
  GX_CK(h, cudaMemcpyAsync(&enc, &h->sph.sc->min_dt_enc, sizeof enc, cudaMemcpyDeviceToHost, h->stream));
  GX_CK(h, cudaMemcpyAsync(dt.data(), h->sph.dtv, ng * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  rc = finish(h, false);
  if (rc) return rc;
  if ((rc = keep.restore())) return rc;
  if (dt_out)
    for (size_t k = 0; k < ng; ++k) dt_out[gas[k]] = dt[k];
  if (min_out) *min_out = -dec_max_host(enc);
  return GX_OK;
}

int gx_sph_coupled_pairs(gx_handle* h, size_t n, const double* pos, const double* mass, const uint8_t* kind,
                         uint64_t* pairs_out, size_t cap, size_t* count_out) {
  if (!h || !count_out) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  *count_out = 0;
  if (n == 0) return GX_OK;
  if (!pos || !mass || (cap && !pairs_out)) return fail(h, GX_ERR_INVALID_ARG, "null array");
  std::vector<uint32_t> gas;
  int rc = gas_map(h, n, kind, gas);
  if (rc || gas.empty()) return rc;
  cudaSetDevice(h->device);
  SphScratchKeeper keep(h, gas.size());
  if ((rc = keep.save())) return rc;
  rc = host_sph_setup(h, n, pos, nullptr, mass, &gas, false, true);
  if (rc) return rc;
  const StepBufs& b = h->ar.b;
  const size_t ng = gas.size();
  sph_enqueue_force(h->sph, b.pos, nullptr, b.mass, nullptr, true, false, b.ctl, h->stream);
  // pass 1: pairs per a; the host turns them into offsets; pass 2 writes the b's
  uint32_t* d_counts = nullptr;
  uint64_t* d_off = nullptr;
  uint32_t* d_list = nullptr;
  auto release = [&]() {
    if (d_counts) cudaFree(d_counts);
    if (d_off) cudaFree(d_off);
    if (d_list) cudaFree(d_list);
  };
  cudaError_t e = cudaMalloc(&d_counts, ng * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&d_off, ng * sizeof(uint64_t));
  if (e != cudaSuccess) {
    release();
    return fail(h, GX_ERR_CUDA, std::string("coupled pairs scratch: ") + cudaGetErrorString(e));
  }
  sph_enqueue_pairs(h->sph, d_counts, nullptr, nullptr, b.ctl, h->stream, true);
  std::vector<uint32_t> counts(ng);
  e = cudaMemcpyAsync(counts.data(), d_counts, ng * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  std::vector<uint64_t> off(ng + 1, 0);
  for (size_t k = 0; k < ng; ++k) off[k + 1] = off[k] + counts[k];
  const size_t total = off[ng];
  std::vector<uint32_t> list(total);
  if (e == cudaSuccess && total) {
    e = cudaMalloc(&d_list, total * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_off, off.data(), ng * sizeof(uint64_t), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) sph_enqueue_pairs(h->sph, nullptr, d_off, d_list, b.ctl, h->stream, false);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(list.data(), d_list, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream);
  }
  rc = e == cudaSuccess ? finish(h, false) : fail(h, GX_ERR_CUDA, std::string("coupled pairs: ") + cudaGetErrorString(e));
  release();
  if (rc) return rc;
  if ((rc = keep.restore())) return rc;
  // ascending (a, b): a runs in order, each run's b's sorted (cfl.rs:216-225)
  size_t w = 0;
  for (size_t a = 0; a < ng; ++a) {
    std::sort(list.begin() + off[a], list.begin() + off[a + 1]);
    for (uint64_t t = off[a]; t < off[a + 1]; ++t, ++w)
      if (w < cap) {
        pairs_out[2 * w] = gas[a];
        pairs_out[2 * w + 1] = gas[list[t]];
      }
  }
  *count_out = total;
  return GX_OK;
}

int gx_sph_density(gx_handle* h, size_t n, const double* pos, const double* mass, const double* h_init,
                   double* rho_out, double* h_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  if (n == 0) return GX_OK;
  if (!pos || !mass || !rho_out || !h_out) return fail(h, GX_ERR_INVALID_ARG, "null array");
  cudaSetDevice(h->device);
  h->sph_host_hint_ngas = 0;
  int rc = host_sph_setup(h, n, pos, nullptr, mass, nullptr, false, true);
  if (rc) return rc;
  const int warm = h->sph.p.warm_start;
  if (h_init) {
    rc = put_gas(h, h->sph.hs, h_init, n);
    if (rc) return rc;
    const uint32_t one = 1u;
    GX_CK(h, cudaMemcpyAsync(&h->sph.sc->hint_valid, &one, sizeof one, cudaMemcpyHostToDevice, h->stream));
    h->sph.p.warm_start = 1;
  }
  const StepBufs& b = h->ar.b;
  sph_enqueue_force(h->sph, b.pos, nullptr, b.mass, nullptr, true, false, b.ctl, h->stream);
  h->sph.p.warm_start = warm;
  GX_CK(h, cudaMemcpyAsync(rho_out, h->sph.rho, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  GX_CK(h, cudaMemcpyAsync(h_out, h->sph.hs, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return finish(h, false);
}

int gx_sph_hydro(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                 const double* rho, const double* hsml, const double* u, double* acc_out, double* dudt_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  if (n == 0) return GX_OK;
  if (!pos || !vel || !mass || !rho || !hsml || !acc_out) return fail(h, GX_ERR_INVALID_ARG, "null array");
  double h_max = 0.0;
  for (size_t i = 0; i < n; ++i) h_max = std::fmax(h_max, hsml[i]);
  if (!(h_max > 0.0) || !std::isfinite(h_max))
    return fail(h, GX_ERR_INVALID_ARG, "hydro needs positive finite smoothing lengths (forces.rs:282-285)");
  cudaSetDevice(h->device);
  h->sph_host_hint_ngas = 0;
  int rc = host_sph_setup(h, n, pos, vel, mass, nullptr, false, false);
  if (rc) return rc;
  if ((rc = put_gas(h, h->sph.rho, rho, n)) || (rc = put_gas(h, h->sph.hs, hsml, n)) || (rc = put_gas(h, h->sph.gu, u, n)))
    return rc;
  const StepBufs& b = h->ar.b;
  sph_enqueue_force(h->sph, b.pos, b.vel, b.mass, nullptr, false, true, b.ctl, h->stream);
  GX_CK(h, cudaMemcpyAsync(acc_out, h->sph.gacc, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (dudt_out) GX_CK(h, cudaMemcpyAsync(dudt_out, h->sph.dudt, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return finish(h, false);
}

int gx_sph_cfl(gx_handle* h, size_t n, const double* pos, const double* vel, const double* hsml, const double* u,
               double c_cfl, double* dt_out, double* min_out) {
  if (!h) return GX_ERR_INVALID_ARG;
  if (int rc = need_sph(h)) return rc;
  if (n == 0) {
    if (min_out) *min_out = std::numeric_limits<double>::infinity();
    return GX_OK;
  }
  if (!pos || !vel || !hsml || !dt_out) return fail(h, GX_ERR_INVALID_ARG, "null array");
  cudaSetDevice(h->device);
  h->sph_host_hint_ngas = 0;
  int rc = host_sph_setup(h, n, pos, vel, nullptr, nullptr, false, false);
  if (rc) return rc;
  if ((rc = put_gas(h, h->sph.hs, hsml, n)) || (rc = put_gas(h, h->sph.gu, u, n))) return rc;
  const StepBufs& b = h->ar.b;
  sph_enqueue_cfl(h->sph, b.pos, b.vel, c_cfl, true, b.ctl, h->stream);
  unsigned long long enc = 0;
  GX_CK(h, cudaMemcpyAsync(&enc, &h->sph.sc->min_dt_enc, sizeof enc, cudaMemcpyDeviceToHost, h->stream));
  GX_CK(h, cudaMemcpyAsync(dt_out, h->sph.dtv, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  rc = finish(h, false);
  if (rc) return rc;
  if (min_out) *min_out = -dec_max_host(enc);
  return GX_OK;
}

}  // extern "C"
