// gx_active.cu -- the target list of an active-subset walk.
//
// Reference: core/src/traits.rs:52-54 (`accelerations_active`: the accelerations of the
// active particles, equal to what `accelerations` gives them) and :89-91
// (`gravity_active_cached`, which Lbvh leaves at that default). The tree is built from
// every particle as usual; only the walk is restricted. The active particles are
// listed by their sorted (Morton) position, in sorted order, so each walk item is 32
// spatially close targets like the full walk's: flags over the sorted positions, then
// an ordered compaction (per-chunk counts, one scan of the counts, per-chunk writes).
#include <algorithm>

#include "gx_kernels.h"

namespace gx {

namespace {

constexpr int kActThreads = 256;
constexpr uint32_t kActChunk = 4096;  // sorted positions per compaction block

// Every item starts empty (its first list entry past any count), so items beyond the
// number of distinct active particles walk nothing.
__global__ void __launch_bounds__(kActThreads) k_items_init(uint32_t nitems, WalkItem* __restrict__ items) {
  for (uint32_t j = blockIdx.x * kActThreads + threadIdx.x; j < nitems; j += gridDim.x * kActThreads)
    items[j] = WalkItem{0xFFFFFFE0u, 0u};
}

// inv[order[s]] = s (original index -> sorted position); the flags start cleared.
__global__ void __launch_bounds__(kActThreads) k_invert(uint32_t n, const uint32_t* __restrict__ order,
                                                        uint32_t* __restrict__ inv, uint32_t* __restrict__ flags) {
  for (uint32_t s = blockIdx.x * kActThreads + threadIdx.x; s < n; s += gridDim.x * kActThreads) {
    const uint32_t o = order[s];
    if (o < n) inv[o] = s;
    flags[s] = 0u;
  }
}

// flags[sorted position of an active particle] = 1 (indices were checked on the host).
__global__ void __launch_bounds__(kActThreads) k_mark(uint32_t n, const uint32_t* __restrict__ active,
                                                      uint32_t n_active, const uint32_t* __restrict__ inv,
                                                      uint32_t* __restrict__ flags) {
  for (uint32_t i = blockIdx.x * kActThreads + threadIdx.x; i < n_active; i += gridDim.x * kActThreads) {
    const uint32_t a = active[i];
    if (a < n) flags[inv[a]] = 1u;
  }
}

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t base = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kActThreads / 32; ++w) {
    base += (w < warp) ? s_warp[w] : 0u;
    all += s_warp[w];
  }
  __syncthreads();
  *total = all;
  return base + x - v;
}

// counts[c] = number of flags set in chunk c.
__global__ void __launch_bounds__(kActThreads) k_chunk_count(uint32_t n, const uint32_t* __restrict__ flags,
                                                             uint32_t* __restrict__ counts) {
  __shared__ uint32_t s_warp[kActThreads / 32];
  const uint32_t base = blockIdx.x * kActChunk;
  uint32_t c = 0;
  for (uint32_t s = base + threadIdx.x; s < min(n, base + kActChunk); s += kActThreads) c += flags[s];
  uint32_t total;
  block_excl_scan(c, s_warp, &total);
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// Exclusive scan of the chunk counts in place (one block); the sum goes to *count_out.
__global__ void __launch_bounds__(kActThreads) k_scan_counts(uint32_t nchunks, uint32_t* __restrict__ counts,
                                                             uint32_t* __restrict__ count_out) {
  __shared__ uint32_t s_warp[kActThreads / 32];
  uint32_t carry = 0;
  for (uint32_t b0 = 0; b0 < nchunks; b0 += kActThreads) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t v = i < nchunks ? counts[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_excl_scan(v, s_warp, &total);
    if (i < nchunks) counts[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *count_out = carry;
}

// Chunk c writes its flagged sorted positions, in order, from list[counts[c]]; the
// thread writing list entry j with j % group == 0 also writes walk item j / group.
__global__ void __launch_bounds__(kActThreads) k_chunk_write(uint32_t n, const uint32_t* __restrict__ flags,
                                                             const uint32_t* __restrict__ counts,
                                                             uint32_t* __restrict__ list, uint32_t group,
                                                             WalkItem* __restrict__ items) {
  __shared__ uint32_t s_warp[kActThreads / 32];
  constexpr uint32_t kPer = kActChunk / kActThreads;  // 16 consecutive positions a thread
  const uint32_t base = blockIdx.x * kActChunk + threadIdx.x * kPer;
  uint32_t f[kPer];
  uint32_t c = 0;
#pragma unroll
  for (uint32_t j = 0; j < kPer; ++j) {
    f[j] = (base + j < n) ? flags[base + j] : 0u;
    c += f[j];
  }
  uint32_t total;
  uint32_t at = counts[blockIdx.x] + block_excl_scan(c, s_warp, &total);
#pragma unroll
  for (uint32_t j = 0; j < kPer; ++j) {
    if (f[j]) {
      list[at] = base + j;
      if (at % group == 0u) items[at / group] = WalkItem{at, 0u};
      ++at;
    }
  }
}

__global__ void __launch_bounds__(kActThreads) k_gather_acc(const double* __restrict__ acc,
                                                            const uint32_t* __restrict__ active, uint32_t n_active,
                                                            double* __restrict__ out) {
  for (uint32_t i = blockIdx.x * kActThreads + threadIdx.x; i < n_active; i += gridDim.x * kActThreads) {
    const size_t a = active[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) out[3 * (size_t)i + c] = acc[3 * a + c];
  }
}

// Stale-tree walk: the leaves take the current positions (and masses, where the leaf
// had mass when the tree was built, so every skip decision stays the build's): the
// sorted leaf records and each leaf's half of its parent's pair record. Internal nodes
// keep the aggregates and thresholds of the build.
__global__ void __launch_bounds__(kActThreads) k_refresh_leaves(uint32_t n, const uint32_t* __restrict__ order,
                                                                const double* __restrict__ pos,
                                                                const double* __restrict__ mass,
                                                                const uint32_t* __restrict__ parent,
                                                                const uint2* __restrict__ kids, double4* leaf64,
                                                                float* __restrict__ pairs) {
  for (uint32_t k = blockIdx.x * kActThreads + threadIdx.x; k < n; k += gridDim.x * kActThreads) {
    const uint32_t o = order[k];
    if (o >= n) continue;
    const double frozen = leaf64[k].w;
    const double m = frozen > 0.0 ? mass[o] : frozen;
    const double4 x = make_double4(pos[3 * (size_t)o], pos[3 * (size_t)o + 1], pos[3 * (size_t)o + 2], m);
    leaf64[k] = x;
    const uint32_t p = parent[k];
    if (p < n || p >= 2 * n - 1) continue;  // the root leaf of a one-particle system
    const uint32_t gi = p - n;
    const int side = kids[gi].x == k ? 0 : 1;  // left fields are .x/.z, right .y/.w
    float hx, lx, hy, ly, hz, lz;
    split_ff(x.x, hx, lx);
    split_ff(x.y, hy, ly);
    split_ff(x.z, hz, lz);
    float* rec = pairs + 20 * (size_t)gi;  // 5 float4
    rec[0 + side] = hx;
    rec[2 + side] = hy;
    rec[4 + side] = hz;
    rec[6 + side] = __double2float_rn(m);
    rec[8 + side] = lx;
    rec[10 + side] = ly;
    rec[12 + side] = lz;
  }
}

uint32_t grid_for(uint32_t n) { return std::max(1u, std::min((n + kActThreads - 1) / kActThreads, 148u * 16u)); }

}  // namespace

size_t active_chunk_count(uint32_t n) { return (n + kActChunk - 1) / kActChunk; }

void launch_active_targets(const StepBufs& b, const uint32_t* active, uint32_t n_active, uint32_t group,
                           uint32_t* inv, uint32_t* flags, uint32_t* chunk_counts, uint32_t* list,
                           uint32_t* count_out, WalkItem* items, cudaStream_t st) {
  const uint32_t n = b.n;
  const uint32_t nchunks = static_cast<uint32_t>(active_chunk_count(n));
  const uint32_t nitems = (n_active + group - 1) / group;
  k_items_init<<<grid_for(nitems), kActThreads, 0, st>>>(nitems, items);
  k_invert<<<grid_for(n), kActThreads, 0, st>>>(n, b.order, inv, flags);
  k_mark<<<grid_for(n_active), kActThreads, 0, st>>>(n, active, n_active, inv, flags);
  k_chunk_count<<<nchunks, kActThreads, 0, st>>>(n, flags, chunk_counts);
  k_scan_counts<<<1, kActThreads, 0, st>>>(nchunks, chunk_counts, count_out);
  k_chunk_write<<<nchunks, kActThreads, 0, st>>>(n, flags, chunk_counts, list, group, items);
}

void launch_refresh_leaves(const StepBufs& b, cudaStream_t st) {
  k_refresh_leaves<<<grid_for(b.n), kActThreads, 0, st>>>(b.n, b.order, b.pos, b.mass, b.parent, b.kids, b.leaf64,
                                                          reinterpret_cast<float*>(b.pairs));
}

void launch_gather_acc(const double* acc, const uint32_t* active, uint32_t n_active, double* out, cudaStream_t st) {
  if (n_active) k_gather_acc<<<grid_for(n_active), kActThreads, 0, st>>>(acc, active, n_active, out);
}

}  // namespace gx
