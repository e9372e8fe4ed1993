// gx_walk.cu -- warp-cooperative Barnes-Hut tree walk.
//
// Reference: solvers/src/lbvh.rs:469-524 (LbvhFlat::accel: skip the subtree of a
// massless node; a leaf adds the Plummer-softened pair term unless it is the target
// itself; an internal node is accepted as a monopole iff the target is not inside
// its AABB and theta*(d - delta) >= s, s = 2*max(half extents); otherwise it is
// opened) and :673-675 (result times G).
//
// One warp walks the tree for 32 Morton-consecutive targets of one system. The warp
// visits the union of the 32 per-target walks in depth-first, left-before-right
// order (an explicit stack of (node, lane mask) pairs kept in registers, entry j in
// lane j % 32); every node record is loaded once per warp (a broadcast load) and
// each lane applies its OWN opening decision, so the sequence of terms a lane adds
// is exactly the reference's skip-pointer walk for that target. A tree over 30-bit
// codes with a 32-bit position tie-break is at most 63 levels deep, so 64 stack
// entries always suffice (overflow raises the device error word).
//
// FP32 mode: node centres of mass and leaf positions are float-float (hi + lo), so
// dx = (c_hi - x_hi) + (c_lo - x_lo) keeps ~48 bits of the f64 coordinates; the
// opening test compares d^2 with rcrit^2 = (s/theta + delta)^2 and re-decides in
// FP64 with the reference's exact expression whenever the FP32 value lies within a
// relative 4e-6 band of the threshold (or touches the AABB within 2^-20), so every
// opening decision equals the reference's. Terms are accumulated in FP32 with Kahan
// compensation.
// FP64 mode: the reference's arithmetic, operation for operation, so accelerations
// are bit-identical to the reference's CPU walk on the same tree.
#include "gx_kernels.h"

namespace gx {

namespace {

constexpr float kBand = 4e-6f;

struct Acc32 {
  float s[3], c[3];
};

template <bool KAHAN>
__device__ __forceinline__ void acc_add(Acc32& a, float tx, float ty, float tz) {
  const float t[3] = {tx, ty, tz};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (KAHAN) {
      const float y = __fsub_rn(t[i], a.c[i]);
      const float u = __fadd_rn(a.s[i], y);
      a.c[i] = __fsub_rn(__fsub_rn(u, a.s[i]), y);
      a.s[i] = u;
    } else {
      a.s[i] += t[i];
    }
  }
}

// The reference's opening test (solvers/src/lbvh.rs:505-514) in f64 on the node's
// f64 aggregate, geometry derived as in reference_flatten (lbvh.rs:602-613).
__device__ __noinline__ bool exact_accept(const Agg64* __restrict__ agg, uint32_t gi, const double x[3],
                                          double theta) {
  const Agg64& a = agg[gi];
  double ctr[3], hf[3], dv[3], dx[3];
  bool inside = true;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ctr[c] = dmul(dadd(a.mn[c], a.mx[c]), 0.5);
    hf[c] = dmul(dsub(a.mx[c], a.mn[c]), 0.5);
    dv[c] = dsub(a.com[c], ctr[c]);
    inside = inside && (fabs(dsub(x[c], ctr[c])) <= hf[c]);
    dx[c] = dsub(a.com[c], x[c]);
  }
  const double delta = dsqrt(dlen2(dv[0], dv[1], dv[2]));
  const double d2 = dlen2(dx[0], dx[1], dx[2]);
  const double s = dmul(2.0, fmax(hf[0], fmax(hf[1], hf[2])));
  const double d = dsqrt(d2);
  return !inside && dmul(theta, dsub(d, delta)) >= s;
}

struct WarpStack {
  uint32_t u0, m0, u1, m1;
  int sp;
};

__device__ __forceinline__ bool stack_push(WarpStack& s, uint32_t u, uint32_t m, int lane) {
  if (s.sp < 32) {
    if (lane == s.sp) {
      s.u0 = u;
      s.m0 = m;
    }
  } else if (s.sp < 64) {
    if (lane == s.sp - 32) {
      s.u1 = u;
      s.m1 = m;
    }
  } else {
    return false;
  }
  ++s.sp;
  return true;
}

__device__ __forceinline__ void stack_pop(WarpStack& s, uint32_t& u, uint32_t& m) {
  --s.sp;
  const int src = s.sp & 31;
  const bool lo = s.sp < 32;
  u = __shfl_sync(0xffffffffu, lo ? s.u0 : s.u1, src);
  m = __shfl_sync(0xffffffffu, lo ? s.m0 : s.m1, src);
}

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace

template <int F64, bool QUAD, bool KAHAN, bool STATS, bool INSIDE>
__global__ void __launch_bounds__(256) k_walk(StepBufs b, int persistent) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps_total = (gridDim.x * blockDim.x) >> 5;
  uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n_total = b.n;
  while (item < b.nitems) {
    const WalkItem it = b.items[item];
    const SysDesc sd = b.sys[it.sys];
    const uint32_t end = sd.off + sd.n;
    const uint32_t k = it.begin + lane;
    const bool valid = k < end;
    const double g = sd.g;
    if (sd.n == 1) {
      // A lone particle feels no force (its only leaf is itself).
      if (valid) {
        const uint32_t o = b.order[k];
#pragma unroll
        for (int c = 0; c < 3; ++c) b.acc[3 * (size_t)o + c] = 0.0;
      }
    } else {
      const double eps2 = dmul(sd.eps, sd.eps);
      const float eps2f = __double2float_rn(eps2);
      const double theta = sd.theta;
      const float tiny2 = b.bounds[it.sys].tiny2;
      double x64[3] = {0, 0, 0};
      float xh[3] = {0, 0, 0}, xl[3] = {0, 0, 0};
      if (valid) {
        const double4 p = b.leaf64[k];
        x64[0] = p.x;
        x64[1] = p.y;
        x64[2] = p.z;
        if (!F64) {
          const float4 ha = b.leafA[k], hb = b.leafB[k];
          xh[0] = ha.x;
          xh[1] = ha.y;
          xh[2] = ha.z;
          xl[0] = hb.x;
          xl[1] = hb.y;
          xl[2] = hb.z;
        }
      }
      Acc32 a32 = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
      double a64[3] = {0.0, 0.0, 0.0};
      unsigned long long n_leaf = 0, n_far = 0, n_open = 0, n_re = 0, n_vis = 0;

      WarpStack stk{0, 0, 0, 0, 0};
      uint32_t u = n_total + sd.off;  // root: internal node 0 of this system
      uint32_t mask = __ballot_sync(0xffffffffu, valid);
      // Each node is reached at most once per warp (only through its parent), so a
      // walk longer than the system's node count means a corrupt tree: stop, flag.
      const uint32_t max_iters = 2u * sd.n + 64u;
      const uint32_t int_lo = n_total + sd.off, int_hi = n_total + sd.off + sd.n - 1;
      uint32_t iters = 0;
      for (;;) {
        if (++iters > max_iters) {
          if (lane == 0) raise_err(b.ctl, kErrBadIndex);
          break;
        }
        if (STATS) ++n_vis;
        const bool active = (mask >> lane) & 1u;
        if (u < n_total) {
          // ---- leaf u (sorted index) ----
          if (F64) {
            const double4 p = b.leaf64[u];
            if (active && u != k && p.w > 0.0) {
              const double dx = dsub(p.x, x64[0]), dy = dsub(p.y, x64[1]), dz = dsub(p.z, x64[2]);
              const double r2 = dadd(dlen2(dx, dy, dz), eps2);
              const double f = ddiv(p.w, dmul(r2, dsqrt(r2)));
              a64[0] = dadd(a64[0], dmul(dx, f));
              a64[1] = dadd(a64[1], dmul(dy, f));
              a64[2] = dadd(a64[2], dmul(dz, f));
              if (STATS) ++n_leaf;
            }
          } else {
            const float4 la = __ldg(&b.leafA[u]);
            const float4 lb = __ldg(&b.leafB[u]);
            if (active && u != k && la.w > 0.f) {
              const float dx = (la.x - xh[0]) + (lb.x - xl[0]);
              const float dy = (la.y - xh[1]) + (lb.y - xl[1]);
              const float dz = (la.z - xh[2]) + (lb.z - xl[2]);
              const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2f)));
              const float inv = rsqrtf(r2);
              const float f = la.w * inv * inv * inv;
              acc_add<KAHAN>(a32, dx * f, dy * f, dz * f);
              if (STATS) ++n_leaf;
            }
          }
        } else {
          // ---- internal node gi ----
          const uint32_t gi = u - n_total;
          bool open = false;
          if (F64) {
            const Node64 nd = b.node64[gi];
            if (active && nd.m > 0.0) {
              bool inside = true;
#pragma unroll
              for (int c = 0; c < 3; ++c) inside = inside && (fabs(dsub(x64[c], nd.c[c])) <= nd.h[c]);
              const double dx = dsub(nd.com[0], x64[0]), dy = dsub(nd.com[1], x64[1]), dz = dsub(nd.com[2], x64[2]);
              const double d2 = dlen2(dx, dy, dz);
              const double d = dsqrt(d2);
              if (!inside && dmul(theta, dsub(d, nd.delta)) >= nd.s) {
                const double r2 = dadd(d2, eps2);
                const double f = ddiv(nd.m, dmul(r2, dsqrt(r2)));
                a64[0] = dadd(a64[0], dmul(dx, f));
                a64[1] = dadd(a64[1], dmul(dy, f));
                a64[2] = dadd(a64[2], dmul(dz, f));
                if (STATS) ++n_far;
              } else {
                open = true;
              }
            }
          } else {
            const float4 na = __ldg(&b.nodeA[gi]);
            const float4 nb = __ldg(&b.nodeB[gi]);
            if (active && na.w > 0.f) {
              const float dx = (na.x - xh[0]) + (nb.x - xl[0]);
              const float dy = (na.y - xh[1]) + (nb.y - xl[1]);
              const float dz = (na.z - xh[2]) + (nb.z - xl[2]);
              const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
              const float rc2 = nb.w;
              int dec;  // 1 accept, 0 open, 2 undecided in FP32
              if (d2 > fmaf(rc2, kBand, rc2) + tiny2)
                dec = 1;
              else if (d2 < fmaf(rc2, -kBand, rc2) - tiny2)
                dec = 0;
              else
                dec = 2;
              if (INSIDE && dec == 1) {
                const float4 nc = __ldg(&b.nodeC[gi]);
                const float4 nd4 = __ldg(&b.nodeD[gi]);
                const float q0 = fabsf(xh[0] - nc.x) - nd4.x;
                const float q1 = fabsf(xh[1] - nc.y) - nd4.y;
                const float q2 = fabsf(xh[2] - nc.z) - nd4.z;
                const float t0 = 0x1p-20f * (fabsf(nc.x) + nd4.x) + 1e-30f;
                const float t1 = 0x1p-20f * (fabsf(nc.y) + nd4.y) + 1e-30f;
                const float t2 = 0x1p-20f * (fabsf(nc.z) + nd4.z) + 1e-30f;
                if (fabsf(q0) <= t0 || fabsf(q1) <= t1 || fabsf(q2) <= t2)
                  dec = 2;
                else if (q0 < 0.f && q1 < 0.f && q2 < 0.f)
                  dec = 0;  // clearly inside: open
              }
              if (dec == 2) {
                dec = exact_accept(b.agg64, gi, x64, theta) ? 1 : 0;
                if (STATS) ++n_re;
              }
              if (dec == 1) {
                const float r2 = d2 + eps2f;
                const float inv = rsqrtf(r2);
                const float inv2 = inv * inv;
                const float inv3 = inv * inv2;
                const float f = na.w * inv3;
                float tx = dx * f, ty = dy * f, tz = dz * f;
                if (QUAD) {
                  const float4 qa = __ldg(&b.nodeQ[2 * (size_t)gi]);
                  const float4 qb = __ldg(&b.nodeQ[2 * (size_t)gi + 1]);
                  // r = x - com = -d; a += Q r / r^5 - 2.5 (r.Q r) r / r^7
                  const float rx = -dx, ry = -dy, rz = -dz;
                  const float qx = qa.x * rx + qa.y * ry + qa.z * rz;
                  const float qy = qa.y * rx + qa.w * ry + qb.x * rz;
                  const float qz = qa.z * rx + qb.x * ry + qb.y * rz;
                  const float rqr = rx * qx + ry * qy + rz * qz;
                  const float inv5 = inv3 * inv2;
                  const float c7 = 2.5f * rqr * inv5 * inv2;
                  tx += qx * inv5 - rx * c7;
                  ty += qy * inv5 - ry * c7;
                  tz += qz * inv5 - rz * c7;
                }
                acc_add<KAHAN>(a32, tx, ty, tz);
                if (STATS) ++n_far;
              } else {
                open = true;
              }
            }
          }
          const uint32_t open_mask = __ballot_sync(0xffffffffu, open);
          if (open_mask) {
            if (STATS && open) ++n_open;
            const uint2 kd = __ldg(&b.kids[gi]);
            const bool kx_ok = (kd.x >= sd.off && kd.x < end) || (kd.x >= int_lo && kd.x < int_hi);
            const bool ky_ok = (kd.y >= sd.off && kd.y < end) || (kd.y >= int_lo && kd.y < int_hi);
            if (!kx_ok || !ky_ok) {
              if (lane == 0) raise_err(b.ctl, kErrBadIndex);
              break;
            }
            if (!stack_push(stk, kd.y, open_mask, lane)) {
              if (lane == 0) raise_err(b.ctl, kErrStackOverflow);
              break;
            }
            u = kd.x;
            mask = open_mask;
            continue;
          }
        }
        if (stk.sp == 0) break;
        stack_pop(stk, u, mask);
      }
      if (valid) {
        const uint32_t o = b.order[k];
        if (F64) {
#pragma unroll
          for (int c = 0; c < 3; ++c) b.acc[3 * (size_t)o + c] = dmul(a64[c], g);
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float v = KAHAN ? __fsub_rn(a32.s[c], a32.c[c]) : a32.s[c];
            b.acc[3 * (size_t)o + c] = dmul(static_cast<double>(v), g);
          }
        }
      }
      if (STATS) {
        n_leaf = warp_sum64(n_leaf);
        n_far = warp_sum64(n_far);
        n_open = warp_sum64(n_open);
        n_re = warp_sum64(n_re);
        if (lane == 0) {
          atomicAdd(&b.ctl->stats[0], n_leaf);
          atomicAdd(&b.ctl->stats[1], n_far);
          atomicAdd(&b.ctl->stats[2], n_open);
          atomicAdd(&b.ctl->stats[3], n_re);
          atomicAdd(&b.ctl->stats[4], n_vis);
        }
      }
    }
    // next item
    if (persistent) {
      uint32_t nxt = 0;
      if (lane == 0) nxt = atomicAdd(&b.counters[4], 1u) + warps_total;
      item = __shfl_sync(0xffffffffu, nxt, 0);
    } else {
      item = b.nitems;
    }
  }
}

namespace {

template <int F64, bool QUAD, bool KAHAN, bool STATS, bool INSIDE>
void launch_walk_t(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  const int block = cfg.block > 0 ? cfg.block : 256;
  const int wpb = block / 32;
  if (cfg.persistent_ctas > 0) {
    k_walk<F64, QUAD, KAHAN, STATS, INSIDE><<<cfg.persistent_ctas, block, 0, st>>>(b, 1);
  } else {
    const uint32_t grid = (b.nitems + wpb - 1) / wpb;
    if (grid) k_walk<F64, QUAD, KAHAN, STATS, INSIDE><<<grid, block, 0, st>>>(b, 0);
  }
}

template <int F64, bool QUAD, bool KAHAN>
void dispatch_si(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  if (cfg.stats) {
    if (cfg.inside_test)
      launch_walk_t<F64, QUAD, KAHAN, true, true>(b, cfg, st);
    else
      launch_walk_t<F64, QUAD, KAHAN, true, false>(b, cfg, st);
  } else {
    if (cfg.inside_test)
      launch_walk_t<F64, QUAD, KAHAN, false, true>(b, cfg, st);
    else
      launch_walk_t<F64, QUAD, KAHAN, false, false>(b, cfg, st);
  }
}

}  // namespace

void launch_walk(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  if (cfg.precision == 1) {
    // The FP64 walk has no quadrupole or compensation variants: it is the
    // reference's arithmetic.
    dispatch_si<1, false, false>(b, cfg, st);
  } else if (cfg.quad) {
    if (cfg.kahan)
      dispatch_si<0, true, true>(b, cfg, st);
    else
      dispatch_si<0, true, false>(b, cfg, st);
  } else {
    if (cfg.kahan)
      dispatch_si<0, false, true>(b, cfg, st);
    else
      dispatch_si<0, false, false>(b, cfg, st);
  }
}

}  // namespace gx
