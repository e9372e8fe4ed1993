// gx_sort.cu -- stable LSD radix sort of (Morton code, original index) pairs,
// one "onesweep" kernel per digit pass (8-bit digits, or 10-bit ones for 30-bit keys:
// 3 passes instead of 4), segmented by system.
//
// Reference: solvers/src/lbvh.rs:143-147 (`reference_sort`: the permutation that
// sorts by (code, original index)). A stable LSD sort fed with the identity
// permutation reproduces it bit for bit; every step below keeps stability:
//   * keys are ranked inside a tile in input order (warp-striped ownership, ranks
//     from __match_any_sync peer masks and running per-warp digit counters);
//   * tiles of a system are chained in index order through decoupled look-back;
//   * the scatter is staged through shared memory so each digit's run of a tile
//     is written as one contiguous, coalesced segment.
// The digit histograms of all passes come from the Morton kernel (one read of the
// keys), so each pass reads and writes every (key, index) pair once.
// Tiles never straddle systems and each system has its own histograms and
// look-back chain, so a batch of systems is sorted per system in one launch.
#include <mutex>

#include "gx_kernels.h"

namespace gx {

namespace {

constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;
constexpr int kWarps = kTileThreads / 32;

// Exclusive scan of one value per thread over a 256-thread CTA.
__device__ __forceinline__ uint32_t block_exclusive_scan_256(uint32_t v, uint32_t* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t base = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) base += (w < warp) ? s_warp[w] : 0u;
  __syncthreads();
  return base + x - v;
}

__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) { *reinterpret_cast<volatile uint32_t*>(p) = v; }

}  // namespace

// One onesweep pass over the tiles of every system, for 30-bit (u32) or 63-bit (u64)
// keys and 2^BITS-bin digits (thread t owns digits t RPT .. t RPT + RPT - 1). Shared
// memory (dynamic): the tile's keys and indices staged in sorted order.
template <typename K, int BITS>
__global__ void __launch_bounds__(kTileThreads) k_onesweep(int pass, const K* __restrict__ keys_in,
                                                           const uint32_t* __restrict__ vals_in,
                                                           K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                           const TileDesc* __restrict__ tiles,
                                                           const SysDesc* __restrict__ sys,
                                                           const uint32_t* __restrict__ hist,
                                                           uint32_t* __restrict__ status, uint32_t* counters,
                                                           uint32_t ntiles, DevCtl* ctl) {
  constexpr int BINS = 1 << BITS;
  constexpr int RPT = BINS / kTileThreads;
  static_assert(RPT >= 1 && RPT * kTileThreads == BINS, "digits per thread");
  extern __shared__ __align__(16) unsigned char s_dyn[];
  K* s_keys = reinterpret_cast<K*>(s_dyn);
  uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_dyn + kTile * sizeof(K));
  __shared__ uint32_t s_whist[kWarps][BINS];
  __shared__ uint32_t s_blk_start[BINS];
  __shared__ uint32_t s_glob[BINS];
  __shared__ uint32_t s_scan[kWarps];
  __shared__ uint32_t s_tile;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int shift = pass * BITS;
  if (threadIdx.x == 0) s_tile = atomicAdd(&counters[pass], 1u);
  for (int i = threadIdx.x; i < kWarps * BINS; i += kTileThreads) (&s_whist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  if (tile >= ntiles) {  // counters not re-armed: refuse rather than read past the table
    if (threadIdx.x == 0) raise_err(ctl, kErrBadIndex);
    return;
  }
  const TileDesc t = tiles[tile];
  const SysDesc sd = sys[t.sys];

  // Load: warp w owns the contiguous 512-key slice [w*512, w*512+512) of the tile,
  // item j of lane l at w*512 + 32 j + l (coalesced, and in index order per warp).
  K key[kItemsPerThread];
  uint32_t val[kItemsPerThread], rank[kItemsPerThread];
#pragma unroll
  for (int j = 0; j < kItemsPerThread; ++j) {
    const uint32_t idx = t.begin + warp * (32 * kItemsPerThread) + 32 * j + lane;
    if (idx < t.end) {
      key[j] = keys_in[idx];
      val[j] = vals_in ? vals_in[idx] : idx;
    } else {
      key[j] = ~K(0);  // pad: largest digit, ranked after every real key
      val[j] = 0;
    }
  }

  // Rank within the warp: peers holding the same digit, in lane order, after the
  // warp's earlier items of that digit.
  const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kItemsPerThread; ++j) {
    const uint32_t d = static_cast<uint32_t>(key[j] >> shift) & (BINS - 1);
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t before = s_whist[warp][d];
    rank[j] = before + __popc(peers & lt_mask);
    __syncwarp();
    if (lane == 31 - __clz(peers)) s_whist[warp][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // Thread t owns digits d = t RPT + r: per-warp exclusive offsets, tile totals, their
  // block-local starts.
  uint32_t total[RPT], local_excl[RPT];
  uint32_t local = 0;
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const uint32_t d = threadIdx.x * RPT + r;
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = s_whist[w][d];
      s_whist[w][d] = tot;
      tot += c;
    }
    total[r] = tot;
    local_excl[r] = local;
    local += tot;
  }
  const uint32_t blk_base = block_exclusive_scan_256(local, s_scan);
#pragma unroll
  for (int r = 0; r < RPT; ++r) s_blk_start[threadIdx.x * RPT + r] = blk_base + local_excl[r];

  // Decoupled look-back along this system's tiles (bounded waits).
  uint32_t* st = status + (size_t)pass * ntiles * BINS;
  const uint32_t tl = tile - sd.first_tile;
  uint32_t excl[RPT];
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const uint32_t d = threadIdx.x * RPT + r;
    excl[r] = 0;
    if (tl == 0) {
      st_volatile(&st[(size_t)tile * BINS + d], kFlagPrefix | (total[r] & kValMask));
    } else {
      st_volatile(&st[(size_t)tile * BINS + d], kFlagAgg | (total[r] & kValMask));
    }
  }
  if (tl != 0) {
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const uint32_t d = threadIdx.x * RPT + r;
      uint32_t p = tile - 1;
      for (;;) {
        uint32_t w = wait_flagged(&st[(size_t)p * BINS + d], kSpinLimit, ctl);
        if (w == 0u) w = kFlagPrefix;  // timed out (error raised): end the look-back
        excl[r] += w & kValMask;
        if ((w & ~kValMask) == kFlagPrefix || p == sd.first_tile) break;
        --p;
      }
      st_volatile(&st[(size_t)tile * BINS + d], kFlagPrefix | ((excl[r] + total[r]) & kValMask));
    }
  }
  // Global start of digit d for this tile: system offset + digits below d in the
  // whole system + the same digit in the system's earlier tiles.
  const uint32_t* hs = hist + (size_t)t.sys * kHistWords + (size_t)pass * BINS;
  uint32_t hv[RPT], hloc = 0;
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    hv[r] = hloc;
    hloc += hs[threadIdx.x * RPT + r];
  }
  const uint32_t pass_base = block_exclusive_scan_256(hloc, s_scan);
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const uint32_t d = threadIdx.x * RPT + r;
    s_glob[d] = sd.off + pass_base + hv[r] + excl[r] - s_blk_start[d];
  }
  __syncthreads();

  // Stage in shared memory at the block-local sorted position.
#pragma unroll
  for (int j = 0; j < kItemsPerThread; ++j) {
    const uint32_t dj = static_cast<uint32_t>(key[j] >> shift) & (BINS - 1);
    const uint32_t r = s_blk_start[dj] + s_whist[warp][dj] + rank[j];
    s_keys[r] = key[j];
    s_vals[r] = val[j];
  }
  __syncthreads();

  // Coalesced scatter: consecutive i of one digit land on consecutive addresses.
  // Pads sort behind every real key, so only the first `count` entries are real.
  const uint32_t count = t.end - t.begin;
  for (uint32_t i = threadIdx.x; i < count; i += kTileThreads) {
    const K k = s_keys[i];
    const uint32_t dst = s_glob[static_cast<uint32_t>(k >> shift) & (BINS - 1)] + i;
    keys_out[dst] = k;
    vals_out[dst] = s_vals[i];
  }
}

namespace {

template <typename K>
constexpr size_t onesweep_smem() {
  return kTile * (sizeof(K) + sizeof(uint32_t));
}

// keys_in -> (keys_out, vals_out) over `passes` passes of BITS-bit digits; keys_in may
// be keys_out (it is read by the first pass only), the values start as the identity.
// No pass writes the buffer it reads: with an even pass count the keys alternate
// keys_tmp, keys_out, ...; with an odd count they go keys_tmp, keys_tmp2, keys_tmp,
// ..., keys_out. The values alternate so that the last pass writes vals_out.
template <typename K, int BITS>
void run_passes(int passes, const K* keys_in, K* keys_out, uint32_t* vals_out, K* keys_tmp, K* keys_tmp2,
                uint32_t* vals_tmp, const TileDesc* tiles, const SysDesc* sys, const uint32_t* hist,
                uint32_t* status, uint32_t* counters, uint32_t ntiles, DevCtl* ctl, cudaStream_t st) {
  // The dynamic shared-memory opt-in is a per-device function attribute, set once per
  // device (handles on several host threads may reach here together).
  static std::mutex mu;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64) {
    std::lock_guard<std::mutex> lk(mu);
    if (!attr_set[dev]) {
      cudaFuncSetAttribute(k_onesweep<K, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(onesweep_smem<K>()));
      attr_set[dev] = true;
    }
  }
  const K* kin = keys_in;
  const uint32_t* vin = nullptr;
  for (int p = 0; p < passes; ++p) {
    K* kout;
    if (p == passes - 1)
      kout = keys_out;
    else if (passes % 2 == 0)
      kout = (p % 2 == 0) ? keys_tmp : keys_out;
    else
      kout = (p % 2 == 0) ? keys_tmp : keys_tmp2;
    uint32_t* vout = ((passes - 1 - p) % 2 == 0) ? vals_out : vals_tmp;
    k_onesweep<K, BITS><<<ntiles, kTileThreads, onesweep_smem<K>(), st>>>(p, kin, vin, kout, vout, tiles, sys, hist,
                                                                           status, counters, ntiles, ctl);
    kin = kout;
    vin = vout;
  }
}

}  // namespace

// Digit histograms of all passes (8-bit digits) from keys already in b.codes (stage
// entry point).
__global__ void __launch_bounds__(kTileThreads) k_code_hist(const TileDesc* __restrict__ tiles,
                                                            const uint32_t* __restrict__ codes,
                                                            uint32_t* __restrict__ hist) {
  __shared__ uint32_t sh[kRadixPasses * kRadixBins];
  const TileDesc t = tiles[blockIdx.x];
  for (int i = threadIdx.x; i < kRadixPasses * kRadixBins; i += kTileThreads) sh[i] = 0;
  __syncthreads();
  for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += kTileThreads) {
    const uint32_t c = codes[i];
#pragma unroll
    for (int p = 0; p < kRadixPasses; ++p) atomicAdd(&sh[p * kRadixBins + ((c >> (p * kRadixBits)) & (kRadixBins - 1))], 1u);
  }
  __syncthreads();
  uint32_t* hs = hist + (size_t)t.sys * kHistWords;
  for (int i = threadIdx.x; i < kRadixPasses * kRadixBins; i += kTileThreads)
    if (sh[i]) atomicAdd(&hs[i], sh[i]);
}

void launch_sort_passes(const uint32_t* keys_in, uint32_t* keys_out, uint32_t* vals_out, uint32_t* keys_tmp,
                        uint32_t* vals_tmp, const TileDesc* tiles, const SysDesc* sys, const uint32_t* hist,
                        uint32_t* status, uint32_t* counters, uint32_t ntiles, DevCtl* ctl, cudaStream_t st) {
  run_passes<uint32_t, kRadixBits>(kRadixPasses, keys_in, keys_out, vals_out, keys_tmp, nullptr, vals_tmp, tiles, sys,
                                   hist, status, counters, ntiles, ctl, st);
}

void launch_code_hist(const StepBufs& b, cudaStream_t st) {
  k_code_hist<<<b.ntiles, kTileThreads, 0, st>>>(b.tiles, b.codes, b.hist);
}

void launch_sort(const StepBufs& b, cudaStream_t st) {
  // (codes, identity) -> (codes sorted, order) through (keys_alt, vals_alt); the 3-pass
  // sort also uses the upper half of keys_alt (sized for 64-bit keys).
  if (b.key64)
    run_passes<uint64_t, kRadixBits>(kRadixPasses63, reinterpret_cast<const uint64_t*>(b.codes),
                                     reinterpret_cast<uint64_t*>(b.codes), b.order,
                                     reinterpret_cast<uint64_t*>(b.keys_alt), nullptr, b.vals_alt, b.tiles, b.sys,
                                     b.hist, b.sort_status, b.counters, b.ntiles, b.ctl, st);
  else if (b.radix_bits == kRadixBitsWide)
    run_passes<uint32_t, kRadixBitsWide>(kRadixPassesWide, b.codes, b.codes, b.order, b.keys_alt, b.keys_alt + b.n,
                                         b.vals_alt, b.tiles, b.sys, b.hist, b.sort_status, b.counters, b.ntiles,
                                         b.ctl, st);
  else
    run_passes<uint32_t, kRadixBits>(kRadixPasses, b.codes, b.codes, b.order, b.keys_alt, nullptr, b.vals_alt,
                                     b.tiles, b.sys, b.hist, b.sort_status, b.counters, b.ntiles, b.ctl, st);
}

}  // namespace gx
