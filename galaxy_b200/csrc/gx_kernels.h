// gx_kernels.h -- device buffer bundle and kernel launchers of one step.
#pragma once

#include "gx_common.cuh"

namespace gx {

// Every device buffer a step touches (owned by gx_solver / gx_batch).
struct StepBufs {
  uint32_t n = 0;       // particles over all systems
  int key64 = 0;        // 63-bit Morton keys (codes/keys_alt hold u64) instead of 30-bit
  int radix_bits = 8;   // digit width of the 30-bit sort: 8 (4 passes) or 10 (3 passes)
  uint32_t nsys = 0;
  uint32_t ntiles = 0;
  uint32_t nitems = 0;  // walk items (32 targets each)
  const TileDesc* tiles = nullptr;
  const SysDesc* sys = nullptr;
  const WalkItem* items = nullptr;
  // particle state, original order
  double* pos = nullptr;
  double* vel = nullptr;
  double* acc = nullptr;
  const double* mass = nullptr;
  // per-step scratch (zeroed by one memset per step, see zero_begin/zero_bytes)
  unsigned long long* bbox_enc = nullptr;  // 6 per system
  uint32_t* hist = nullptr;                // nsys * kHistWords: [system][pass][digit]
  uint32_t* sort_status = nullptr;         // ntiles * kStatusWordsPerTile: [pass][tile][digit]
  uint32_t* counters = nullptr;            // 16 words: [0..7] sort tile counters, [8] walk item counter
  void* zero_begin = nullptr;
  size_t zero_bytes = 0;
  Bounds* bounds = nullptr;  // per system
  // sort
  uint32_t* codes = nullptr;     // keys (pass-0 input, final sorted keys); u64 when key64
  uint32_t* keys_alt = nullptr;  // sized for u64 keys
  uint32_t* order = nullptr;     // values (final permutation)
  uint32_t* vals_alt = nullptr;
  // leaves, sorted order
  double4* leaf64 = nullptr;
  // Sibling-pair walk records, 5 float4 per internal node i: its two children side by
  // side (L, R), so a float4 load yields float2 (L, R) operand pairs:
  //   pairs[5i+0] = (x_hi L, R, y_hi L, R)   pairs[5i+1] = (z_hi L, R, mass L, R)
  //   pairs[5i+2] = (x_lo L, R, y_lo L, R)   pairs[5i+3] = (z_lo L, R, take L, R)
  //   pairs[5i+4] = (open L, R, child L, child R)   (child codes: internal node index, or
  //                                                   kLeafCode | leaf index)
  // take / open: d^2 thresholds of the FP32 opening test (leaf: take -1, open -2).
  float4* pairs = nullptr;
  // internal nodes
  uint2* kids = nullptr;
  uint32_t* parent = nullptr;
  Agg64* agg64 = nullptr;
  float4* nodeC = nullptr;   // AABB centre (opening test for theta >= 1/sqrt 3)
  float4* nodeD = nullptr;   // AABB half extents (same)
  float4* nodeQ = nullptr;   // 2 per node (quadrupole mode)
  double* q64 = nullptr;     // 6 per node (quadrupole mode)
  Node64* node64 = nullptr;  // FP64 walk mode
  unsigned long long* slots = nullptr;  // climb exchange words, kEmptySlot between builds
  DevCtl* ctl = nullptr;
  // Target list of an active-subset walk (nullptr: every particle is a target). Item i
  // then covers targets[g i .. g i + g - 1] (sorted positions), g = group (a power of two
  // <= 32: sparse subsets use fewer lanes a warp so each warp's targets stay close);
  // *ntargets is their count.
  const uint32_t* targets = nullptr;
  const uint32_t* ntargets = nullptr;
  uint32_t group = 32;
};

struct WalkCfg {
  int precision = 0;  // 0 = FP32, 1 = FP64
  int quad = 0;
  int kahan = 1;
  int stats = 0;
  int inside_test = 0;  // some system has theta >= 1/sqrt(3)
  int block = kWalkThreads;
  int persistent_ctas = 0;  // 0 = one warp per item (no stealing)
};

// gx_step.cu
void launch_kick_drift_bbox(const StepBufs& b, int kick, int pending, cudaStream_t st);
void launch_kick_half(const StepBufs& b, cudaStream_t st);
void launch_morton_hist(const StepBufs& b, uint32_t* lanes_out, cudaStream_t st);
// gx_sort.cu: the four onesweep passes (codes, iota) -> (codes sorted, order)
void launch_sort(const StepBufs& b, cudaStream_t st);
// the four passes on explicit buffers: keys_in -> (keys_out, vals_out), values start as
// the identity; keys_tmp/vals_tmp hold passes 0 and 2
void launch_sort_passes(const uint32_t* keys_in, uint32_t* keys_out, uint32_t* vals_out, uint32_t* keys_tmp,
                        uint32_t* vals_tmp, const TileDesc* tiles, const SysDesc* sys, const uint32_t* hist,
                        uint32_t* status, uint32_t* counters, uint32_t ntiles, DevCtl* ctl, cudaStream_t st);
// per-system digit histograms of b.codes (when codes come from the host)
void launch_code_hist(const StepBufs& b, cudaStream_t st);
// gx_build.cu: gather leaves + bottom-up Karras build and aggregation
void launch_build(const StepBufs& b, int quad, int f64_records, cudaStream_t st);
// Per-device set-up of the build kernels (their dynamic shared-memory limit); call with the
// device current, before any stream capture.
void build_prepare();
// gx_walk.cu: tree walk, acc in original order
void launch_walk(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st);
// gx_diag.cu: one bounded wait on a word nothing sets (failure-detection self-test)
void launch_selftest_wait(const uint32_t* word, uint32_t spins, DevCtl* ctl, cudaStream_t st);
// gx_active.cu: the active-subset walk's target list. From the sorted order and the
// active particles (original indices) it builds, in sorted order, the list of active
// sorted positions (list, count in *count_out) and one walk item per `group` of them.
void launch_active_targets(const StepBufs& b, const uint32_t* active, uint32_t n_active, uint32_t group,
                           uint32_t* inv, uint32_t* flags, uint32_t* chunk_counts, uint32_t* list,
                           uint32_t* count_out, WalkItem* items, cudaStream_t st);
size_t active_chunk_count(uint32_t n);
// Stale-tree walk: leaf records and the leaves' halves of the pair records take the
// current pos / mass (single system); internal nodes keep the build's aggregates.
void launch_refresh_leaves(const StepBufs& b, cudaStream_t st);
// out[3i + c] = acc[3 active[i] + c]
void launch_gather_acc(const double* acc, const uint32_t* active, uint32_t n_active, double* out, cudaStream_t st);
// Blocks of cfg.block threads of the selected walk kernel resident on one SM.
int walk_resident_ctas(const WalkCfg& cfg);
// Shared memory of one FP32 walk block of `block` threads (quadrupole mode: more).
size_t walk_smem_bytes(int block, bool quad);
// Per-device set-up of the walk kernels (their dynamic shared-memory limit); call with the
// device current, before any stream capture.
void walk_prepare();
// gx_diag.cu
void launch_direct_sum_f64(uint32_t n, const double* pos, const double* mass, double g, double eps,
                           uint32_t n_targets, const uint32_t* targets, double* acc, cudaStream_t st);
void launch_potential_f64(uint32_t n, const double* pos, const double* mass, double g, double eps, double* partial,
                          uint32_t n_partial, cudaStream_t st);
void launch_diag_sums(uint32_t n, const double* pos, const double* vel, const double* mass, double* partial,
                      uint32_t n_partial, cudaStream_t st);
uint32_t potential_partials(uint32_t n);

}  // namespace gx
