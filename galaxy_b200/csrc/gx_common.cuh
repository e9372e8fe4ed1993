// gx_common.cuh -- shared device helpers and data layout of the LBVH gravity step.
//
// Layout in HBM for one system of N particles (or a batch of systems packed back
// to back; see gx_batch.cu):
//   particle state, original order, DVec3 layout (3 x f64 per particle):
//     pos[3N], vel[3N], acc[3N]; mass[N] (f64)
//   Morton codes code[N] (u32), the sort's ping-pong (key, index) buffers.
//   sorted leaves (leaf k = k-th particle in (code, index) order):
//     leaf64[k] = double4(x, y, z, m)          FP64 payload for folds and rechecks
//     order[k]  original index
//   sibling-pair walk records, 5 float4 per internal node i: both children side by
//   side (L, R) -- hi/lo float-float centre of mass, mass, the FP32 d^2 thresholds to
//   take / to open, and the children's unified indices (see StepBufs::pairs)
//   internal node i (Karras numbering, unified index N + i):
//     kids[i]   = uint2(left, right) unified children
//     parent[u] unified parent of every node (root: 0xFFFFFFFF)
//     agg64[i]  = {aabb_min[3], aabb_max[3], com[3], mass} FP64 (bit-exact fold)
//     nodeC[i], nodeD[i] = AABB centre, half extents (FP32; theta >= 1/sqrt 3)
//     nodeQ[i]  = 2 x float4 traceless quadrupole (xx, xy, xz, yy), (yz, zz, 0, 0)
//     node64[i] = {center[3], half[3], com[3], mass, delta, s}  FP64 walk record
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gx {

constexpr uint32_t kNoParent = 0xFFFFFFFFu;
constexpr uint64_t kEmptySlot = 0xFFFFFFFFFFFFFFFFull;
// Leaf flag of a child code in the FP32 walk records (N < 2^30, so it never collides).
constexpr uint32_t kLeafCode = 0x80000000u;

// Bounded waits: every spin in these kernels gives up after this many polls,
// raises the device error word and carries on, so no kernel can hang the GPU.
constexpr uint32_t kSpinLimit = 1u << 24;

// Relative guard band of the FP32 opening test: within it the decision is re-made in
// FP64 with the reference's expression (FP32 d^2 carries <= ~1e-6 relative error).
constexpr double kOpenBand = 4e-6;

// Device error word bits (read back by the host after each call).
constexpr uint32_t kErrLookbackTimeout = 1u << 0;
constexpr uint32_t kErrStackOverflow = 1u << 1;
constexpr uint32_t kErrBadIndex = 1u << 2;
constexpr uint32_t kErrClimb = 1u << 3;
constexpr uint32_t kErrSphIterations = 1u << 4;  // an SPH root-find ran past its iteration bound

struct Agg64 {
  double mn[3];
  double mx[3];
  double com[3];
  double m;
};

struct Node64 {
  double c[3];
  double h[3];
  double com[3];
  double m;
  double delta;
  double s;
};

// Morton bounding cube of one system (solvers/src/lbvh.rs:105-120 convention).
struct Bounds {
  double bmin[3];
  double size;
  double scale;
  double scale63;  // 2^21 / size, for 63-bit keys
  double lo[3];
  double hi[3];
  float tiny2;    // absolute guard for FP32 distance comparisons (coincident geometry)
  uint32_t pad;
};

// Work is cut into tiles of kTile particles that never straddle two systems; the
// bbox, Morton, sort and build kernels each run one CTA per tile.
constexpr int kTile = 4096;
constexpr int kTileThreads = 256;
// Threads per block of the tree walks (and the largest walk block accepted).
constexpr int kWalkThreads = 128;
constexpr int kItemsPerThread = kTile / kTileThreads;  // 16
constexpr int kRadixBits = 8;
constexpr int kRadixBins = 1 << kRadixBits;
constexpr int kRadixPasses = 4;     // 30-bit codes: 8 + 8 + 8 + 6 bits
constexpr int kRadixPasses63 = 8;   // 63-bit codes: 7 x 8 + 7 bits
constexpr int kMaxRadixPasses = 8;  // tile counters are sized for this
// The digit width of the 30-bit sort is 8 bits (4 passes) or 10 bits (3 passes): a
// tuning choice, never a change of result. 63-bit keys use 8-bit digits.
constexpr int kRadixBitsWide = 10;
constexpr int kRadixPassesWide = 3;
// Words of digit histograms per system and of look-back status per tile: the larger of
// 8 passes x 256 bins and 3 passes x 1024 bins.
constexpr int kHistWords = 3072;
constexpr int kStatusWordsPerTile = 3072;
static_assert(kMaxRadixPasses * kRadixBins <= kHistWords && kRadixPassesWide * (1 << kRadixBitsWide) <= kHistWords,
              "histogram stride");
// Slot of the per-step counters that the persistent walk steals items from; slots
// [0, kMaxRadixPasses) are the sort passes' tile counters.
constexpr int kWalkItemCounter = kMaxRadixPasses;
constexpr int kCounterWords = 16;  // per-step counter block (zeroed with the step's scratch)
static_assert(kWalkItemCounter < kCounterWords, "the walk's counter is in the block");
// Tree depth bound: the augmented key is (code, 32-bit position), so a root-to-leaf path
// has at most 30 + 32 (30-bit codes) or 63 + 32 (63-bit codes) internal levels.
constexpr int kMaxDepth = 100;

struct TileDesc {
  uint32_t sys, begin, end, pad;
};

// One independent particle system (a batch holds many, packed back to back).
struct SysDesc {
  uint32_t off, n;              // particle range [off, off + n)
  uint32_t first_tile, ntiles;  // its tiles
  double g, eps, theta, dt;
  uint32_t flags;               // kSysPendingKick: the closing half kick is still owed
  uint32_t group;               // targets a warp of the FP32 walk (8, 16 or 32; walk items hold this many)
};
constexpr uint32_t kSysPendingKick = 1u;

// Consecutive sorted targets of one system (its group: 8, 16 or 32 of them), walked
// by one warp.
struct WalkItem {
  uint32_t begin, sys;
};

// Order-preserving map of an f64 onto u64 so that unsigned atomicMax is a float max;
// 0 lies below every real number, so a zeroed word is the identity.
__device__ __forceinline__ unsigned long long enc_max(double x) {
  unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dec_max(unsigned long long e) {
  unsigned long long b = (e >> 63) ? (e & 0x7FFFFFFFFFFFFFFFull) : ~e;
  return __longlong_as_double(static_cast<long long>(b));
}

// Per-call device scalars.
struct DevCtl {
  uint32_t err;
  uint32_t bbox_done;
  uint32_t pad[2];
  unsigned long long stats[8];  // leaf, far, open, recheck, warp visits
};

// ---- exact f64 arithmetic (no contraction into FMA, as Rust's f64 ops) ---------
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }
// glam dot: (x*x + y*y) + z*z
__device__ __forceinline__ double dlen2(double x, double y, double z) {
  return dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z));
}

// ---- Morton (solvers/src/lbvh.rs:37-64) ----------------------------------------
__host__ __device__ __forceinline__ uint32_t expand10(uint32_t v) {
  uint32_t x = v & 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}
__host__ __device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return expand10(x) | (expand10(y) << 1) | (expand10(z) << 2);
}
// 63-bit keys (21 bits per axis): the finer grid the reference defers for dense cores
// and large coordinates (solvers/src/lbvh.rs:29-32). Spreads bit i of v to bit 3i.
__host__ __device__ __forceinline__ uint64_t expand21(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}
__host__ __device__ __forceinline__ uint64_t morton3_63(uint32_t x, uint32_t y, uint32_t z) {
  return expand21(x) | (expand21(y) << 1) | (expand21(z) << 2);
}
__device__ __forceinline__ uint32_t quantize_lane21(double v) {
  double f = floor(v);
  if (!(f >= 0.0)) return 0u;
  if (f >= 2097151.0) return 2097151u;
  return static_cast<uint32_t>(f);
}

// Rust `(v.floor().max(0.0) as u32).min(1023)`.
__device__ __forceinline__ uint32_t quantize_lane(double v) {
  double f = floor(v);
  if (!(f >= 0.0)) return 0u;  // negative or NaN
  if (f >= 1023.0) return 1023u;
  return static_cast<uint32_t>(f);
}

// ---- augmented-key common prefix over sorted codes (solvers/src/lbvh.rs:153-165)
// Positions are local to the system (the reference indexes each system from 0).
__device__ __forceinline__ int prefix_len(uint32_t ca, uint32_t cb, uint32_t a_local, uint32_t b_local) {
  if (ca == cb) return 32 + __clz(a_local ^ b_local);
  return __clz(ca ^ cb);
}
// The same over 64-bit codes: (code, position) is a 96-bit augmented key.
__device__ __forceinline__ int prefix_len(uint64_t ca, uint64_t cb, uint32_t a_local, uint32_t b_local) {
  if (ca == cb) return 64 + __clz(a_local ^ b_local);
  return __clzll(static_cast<long long>(ca ^ cb));
}

// ---- float-float split of an f64 coordinate ------------------------------------
__device__ __forceinline__ void split_ff(double x, float& hi, float& lo) {
  hi = __double2float_rn(x);
  lo = __double2float_rn(x - static_cast<double>(hi));
}

__device__ __forceinline__ void raise_err(DevCtl* ctl, uint32_t bit) { atomicOr(&ctl->err, bit); }

// Bounded wait for a status word whose top two bits become non-zero (set by another
// CTA): at most `limit` re-reads, backing off between them. Returns the word, or 0
// after raising kErrLookbackTimeout when the limit runs out -- no wait is unbounded.
__device__ __forceinline__ uint32_t wait_flagged(const uint32_t* p, uint32_t limit, DevCtl* ctl) {
  uint32_t w = *reinterpret_cast<const volatile uint32_t*>(p);
  for (uint32_t spins = 0; (w >> 30) == 0u; ++spins) {
    if (spins >= limit) {
      raise_err(ctl, kErrLookbackTimeout);
      return 0u;
    }
    __nanosleep(64);
    w = *reinterpret_cast<const volatile uint32_t*>(p);
  }
  return w;
}

}  // namespace gx
