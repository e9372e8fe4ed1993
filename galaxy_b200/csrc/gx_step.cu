// gx_step.cu -- the streaming stages of a step: leapfrog kick + drift fused with the
// per-system bounding-box reduction, and the Morton-code kernel fused with the
// radix sort's up-front digit histogram.
//
// Reference: core/src/integrator.rs:59-73 (half kicks and drift),
// solvers/src/lbvh.rs:105-129 (bbox, padded cube, lane quantisation, interleave).
// All f64 arithmetic uses round-to-nearest intrinsics, so no product is fused into
// an FMA and every value rounds as the reference's Rust f64 code.
#include "gx_kernels.h"

namespace gx {

namespace {

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// CTA-wide max of 6 values (x, y, z maxima and the maxima of -x, -y, -z), then one
// atomicMax per value into the system's encoded bounds.
__device__ __forceinline__ void block_bbox_commit(double v[6], unsigned long long* enc) {
  __shared__ double red[kTileThreads / 32][6];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 6; ++c) v[c] = warp_max(v[c]);
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c) red[warp][c] = v[c];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double m = red[0][threadIdx.x];
    for (int w = 1; w < kTileThreads / 32; ++w) m = fmax(m, red[w][threadIdx.x]);
    if (m == m) atomicMax(&enc[threadIdx.x], enc_max(m));  // skip empty (-inf identity) lanes
  }
}

}  // namespace

// One CTA per tile. kick: apply the (deferred closing +) opening half kick and the
// drift before reducing the bounding box of the new positions.
//   pending:  v += a*h   (closing half kick of the previous step, kept separate)
//   always:   v += a*h ; x += v*dt        with h = 0.5*dt     (integrator.rs:59-67)
__global__ void __launch_bounds__(kTileThreads) k_kick_drift_bbox(const TileDesc* __restrict__ tiles,
                                                                  const SysDesc* __restrict__ sys,
                                                                  double* __restrict__ pos, double* __restrict__ vel,
                                                                  const double* __restrict__ acc, int kick,
                                                                  int pending, unsigned long long* __restrict__ enc) {
  const TileDesc t = tiles[blockIdx.x];
  const SysDesc s = sys[t.sys];
  const double dt = s.dt;
  const double h = dmul(0.5, dt);
  const bool pend = pending || (s.flags & kSysPendingKick);
  double v6[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) v6[c] = -INFINITY;
  for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += kTileThreads) {
    double p[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) p[c] = pos[3 * (size_t)i + c];
    if (kick) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double a = acc[3 * (size_t)i + c];
        double v = vel[3 * (size_t)i + c];
        if (pend) v = dadd(v, dmul(a, h));
        v = dadd(v, dmul(a, h));
        p[c] = dadd(p[c], dmul(v, dt));
        vel[3 * (size_t)i + c] = v;
        pos[3 * (size_t)i + c] = p[c];
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v6[c] = fmax(v6[c], p[c]);
      v6[3 + c] = fmax(v6[3 + c], -p[c]);
    }
  }
  block_bbox_commit(v6, enc + 6 * (size_t)t.sys);
}

// Closing half kick only (applied before a snapshot when one is pending).
__global__ void __launch_bounds__(kTileThreads) k_kick_half(const TileDesc* __restrict__ tiles,
                                                            const SysDesc* __restrict__ sys, double* __restrict__ vel,
                                                            const double* __restrict__ acc) {
  const TileDesc t = tiles[blockIdx.x];
  const double h = dmul(0.5, sys[t.sys].dt);
  for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += kTileThreads) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
      vel[3 * (size_t)i + c] = dadd(vel[3 * (size_t)i + c], dmul(acc[3 * (size_t)i + c], h));
  }
}

// Cube of solvers/src/lbvh.rs:116-120 from the reduced lo/hi.
__device__ __forceinline__ void make_bounds(const unsigned long long* e, Bounds& b) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    b.hi[c] = dec_max(e[c]);
    b.lo[c] = -dec_max(e[3 + c]);
  }
  double ext = fmax(dsub(b.hi[0], b.lo[0]), fmax(dsub(b.hi[1], b.lo[1]), dsub(b.hi[2], b.lo[2])));
  double half = dmul(fmax(dmul(0.5, ext), 1e-12), 1.0 + 1e-9);
  double amax = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double center = dmul(dadd(b.lo[c], b.hi[c]), 0.5);
    b.bmin[c] = dsub(center, half);
    amax = fmax(amax, fmax(fabs(b.lo[c]), fabs(b.hi[c])));
  }
  b.size = dmul(2.0, half);
  b.scale = ddiv(1024.0, b.size);
  b.scale63 = ddiv(2097152.0, b.size);
  // The float-float split keeps ~2^-48 of a coordinate; below that, distance
  // comparisons are re-done in FP64.
  double t = amax * 0x1p-40;
  b.tiny2 = static_cast<float>(t * t);
}

// One CTA per tile: Morton code of every particle of the tile (original order) and
// the tile's contribution to the per-system digit histograms of all radix passes
// (4 for 30-bit keys, 8 for 63-bit). The tile's system cube is rebuilt from the
// reduced lo/hi by every CTA (a few flops), and the system's first tile publishes it.
template <bool K64, int BITS>
__global__ void __launch_bounds__(kTileThreads) k_morton_hist(const TileDesc* __restrict__ tiles,
                                                              const double* __restrict__ pos,
                                                              const unsigned long long* __restrict__ enc,
                                                              const SysDesc* __restrict__ sys,
                                                              Bounds* __restrict__ bounds, uint32_t* __restrict__ codes,
                                                              uint32_t* __restrict__ lanes_out,
                                                              uint32_t* __restrict__ hist) {
  constexpr int BINS = 1 << BITS;
  constexpr int P = K64 ? (63 + BITS - 1) / BITS : (30 + BITS - 1) / BITS;
  __shared__ uint32_t sh[P][BINS];
  __shared__ Bounds sb;
  const TileDesc t = tiles[blockIdx.x];
  for (int i = threadIdx.x; i < P * BINS; i += kTileThreads) (&sh[0][0])[i] = 0;
  if (threadIdx.x == 0) {
    make_bounds(enc + 6 * (size_t)t.sys, sb);
    if (sys[t.sys].first_tile == blockIdx.x) bounds[t.sys] = sb;
  }
  __syncthreads();
  const double bx = sb.bmin[0], by = sb.bmin[1], bz = sb.bmin[2];
  const double scale = K64 ? sb.scale63 : sb.scale;
  for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += kTileThreads) {
    const double vx = dmul(dsub(pos[3 * (size_t)i + 0], bx), scale);
    const double vy = dmul(dsub(pos[3 * (size_t)i + 1], by), scale);
    const double vz = dmul(dsub(pos[3 * (size_t)i + 2], bz), scale);
    if (K64) {
      const uint64_t code = morton3_63(quantize_lane21(vx), quantize_lane21(vy), quantize_lane21(vz));
      reinterpret_cast<uint64_t*>(codes)[i] = code;
#pragma unroll
      for (int p = 0; p < P; ++p) atomicAdd(&sh[p][(code >> (p * BITS)) & (BINS - 1)], 1u);
    } else {
      const uint32_t lx = quantize_lane(vx), ly = quantize_lane(vy), lz = quantize_lane(vz);
      const uint32_t code = morton3(lx, ly, lz);
      codes[i] = code;
      if (lanes_out) {
        lanes_out[3 * (size_t)i + 0] = lx;
        lanes_out[3 * (size_t)i + 1] = ly;
        lanes_out[3 * (size_t)i + 2] = lz;
      }
#pragma unroll
      for (int p = 0; p < P; ++p) atomicAdd(&sh[p][(code >> (p * BITS)) & (BINS - 1)], 1u);
    }
  }
  __syncthreads();
  uint32_t* hs = hist + (size_t)t.sys * kHistWords;
  for (int i = threadIdx.x; i < P * BINS; i += kTileThreads) {
    const uint32_t c = (&sh[0][0])[i];
    if (c) atomicAdd(&hs[i], c);
  }
}

// ---- host launchers ---------------------------------------------------------------
void launch_kick_drift_bbox(const StepBufs& b, int kick, int pending, cudaStream_t st) {
  k_kick_drift_bbox<<<b.ntiles, kTileThreads, 0, st>>>(b.tiles, b.sys, b.pos, b.vel, b.acc, kick, pending, b.bbox_enc);
}

void launch_kick_half(const StepBufs& b, cudaStream_t st) {
  k_kick_half<<<b.ntiles, kTileThreads, 0, st>>>(b.tiles, b.sys, b.vel, b.acc);
}

void launch_morton_hist(const StepBufs& b, uint32_t* lanes_out, cudaStream_t st) {
  if (b.key64)
    k_morton_hist<true, kRadixBits><<<b.ntiles, kTileThreads, 0, st>>>(b.tiles, b.pos, b.bbox_enc, b.sys, b.bounds,
                                                                        b.codes, nullptr, b.hist);
  else if (b.radix_bits == kRadixBitsWide)
    k_morton_hist<false, kRadixBitsWide><<<b.ntiles, kTileThreads, 0, st>>>(b.tiles, b.pos, b.bbox_enc, b.sys,
                                                                             b.bounds, b.codes, lanes_out, b.hist);
  else
    k_morton_hist<false, kRadixBits><<<b.ntiles, kTileThreads, 0, st>>>(b.tiles, b.pos, b.bbox_enc, b.sys, b.bounds,
                                                                         b.codes, lanes_out, b.hist);
}

}  // namespace gx
