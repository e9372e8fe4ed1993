// gx_walk.cu -- warp-cooperative Barnes-Hut tree walk.
//
// Reference: solvers/src/lbvh.rs:469-524 (LbvhFlat::accel: skip the subtree of a
// massless node; a leaf adds the Plummer-softened pair term unless it is the target
// itself; an internal node is accepted as a monopole iff the target is not inside
// its AABB and theta*(d - delta) >= s, s = 2*max(half extents); otherwise it is
// opened) and :673-675 (result times G).
//
// One warp walks the tree for 32 Morton-consecutive targets of one system. The warp
// visits the union of the 32 per-target walks (an explicit stack of (node, lane mask)
// pairs kept in registers, entry j in lane j % 32); every node record is loaded once
// per warp (a broadcast load) and each lane applies its OWN opening decision, so
// every lane takes exactly the reference's set of terms for its target. A tree over
// 30-bit (63-bit) codes with a 32-bit position tie-break is at most 63 (96) levels
// deep, so 96 stack entries always suffice (overflow raises the device error word).
//
// FP32 mode: node centres of mass and leaf positions are float-float (hi + lo), so
// dx = (c_hi - x_hi) + (c_lo - x_lo) keeps ~48 bits of the f64 coordinates; the
// opening test compares d^2 with rcrit^2 = (s/theta + delta)^2 and re-decides in
// FP64 with the reference's exact expression whenever the FP32 value lies within a
// relative 4e-6 band of the threshold (or touches the AABB within 2^-20), so every
// opening decision equals the reference's. Terms are accumulated in FP32 with Kahan
// compensation.
// FP64 mode: the reference's arithmetic, operation for operation and in its
// depth-first order, so accelerations are bit-identical to the reference's CPU walk.
#include "gx_kernels.h"

namespace gx {

namespace {


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

// The reference's decision for internal node gi (solvers/src/lbvh.rs:485-514) in f64
// on the node's f64 aggregate, geometry derived as in reference_flatten
// (lbvh.rs:602-613): 1 = take the monopole, 0 = open, -1 = skip (massless subtree).
__device__ __noinline__ int exact_decision(const Agg64* __restrict__ agg, uint32_t gi, const double x[3],
                                           double theta) {
  const Agg64& a = agg[gi];
  if (!(a.m > 0.0)) return -1;
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
  return (!inside && dmul(theta, dsub(d, delta)) >= s) ? 1 : 0;
}

// Stack of (node, lane mask) entries shared by the warp: entry j lives in lane j % 32
// of slot j / 32. 96 entries cover the deepest tree (kMaxDepth levels of at most one
// pending sibling each, bounded by 30 + 32 or 63 + 32 prefix bits).
constexpr int kStackCap = 96;

struct WarpStack {
  uint32_t u0, m0, u1, m1, u2, m2;
  int sp;
};

__device__ __forceinline__ bool stack_push(WarpStack& s, uint32_t u, uint32_t m, int lane) {
  if (s.sp >= kStackCap) return false;
  const bool w0 = lane == s.sp, w1 = lane == s.sp - 32, w2 = lane == s.sp - 64;
  s.u0 = w0 ? u : s.u0;
  s.m0 = w0 ? m : s.m0;
  s.u1 = w1 ? u : s.u1;
  s.m1 = w1 ? m : s.m1;
  s.u2 = w2 ? u : s.u2;
  s.m2 = w2 ? m : s.m2;
  ++s.sp;
  return true;
}

__device__ __forceinline__ void stack_pop(WarpStack& s, uint32_t& u, uint32_t& m) {
  --s.sp;
  const int src = s.sp & 31;
  const int slot = s.sp >> 5;
  u = __shfl_sync(0xffffffffu, slot == 0 ? s.u0 : (slot == 1 ? s.u1 : s.u2), src);
  m = __shfl_sync(0xffffffffu, slot == 0 ? s.m0 : (slot == 1 ? s.m1 : s.m2), src);
}

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace

// Exact FP64 walk: one node per warp iteration in strict depth-first, left-before-right
// order, so each lane adds its terms in the reference's order with the reference's
// arithmetic.
template <bool STATS, bool LIST>
__global__ void __launch_bounds__(kWalkThreads) k_walk_f64(StepBufs b, int persistent) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps_total = (gridDim.x * blockDim.x) >> 5;
  uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n_total = b.n;
  while (item < b.nitems) {
    const WalkItem it = b.items[item];
    const SysDesc sd = b.sys[it.sys];
    const uint32_t end = sd.off + sd.n;
    // a target list (active-subset walk) names the item's targets; else they are the
    // 32 sorted positions from it.begin
    const uint32_t li = it.begin + lane;
    const bool valid = LIST ? (lane < static_cast<int>(b.group) && li < *b.ntargets) : li < end;
    const uint32_t k = LIST ? (valid ? b.targets[li] : 0u) : li;
    if (sd.n == 1) {
      if (valid) {
        const uint32_t o = b.order[k];
#pragma unroll
        for (int c = 0; c < 3; ++c) b.acc[3 * (size_t)o + c] = 0.0;
      }
    } else {
      const double eps2 = dmul(sd.eps, sd.eps);
      const double theta = sd.theta;
      double x64[3] = {0, 0, 0};
      if (valid) {
        const double4 p = b.leaf64[k];
        x64[0] = p.x;
        x64[1] = p.y;
        x64[2] = p.z;
      }
      double a64[3] = {0.0, 0.0, 0.0};
      unsigned long long n_leaf = 0, n_far = 0, n_open = 0, n_vis = 0;
      WarpStack stk{0, 0, 0, 0, 0, 0, 0};
      uint32_t u = n_total + sd.off;
      uint32_t mask = __ballot_sync(0xffffffffu, valid);
      const uint32_t max_iters = 2u * sd.n + 64u;
      const uint32_t int_lo = n_total + sd.off, int_n = sd.n - 1;
      uint32_t iters = 0;
      for (;;) {
        if (++iters > max_iters) {
          if (lane == 0) raise_err(b.ctl, kErrBadIndex);
          break;
        }
        if (STATS) ++n_vis;
        const bool active = (mask >> lane) & 1u;
        if (u < n_total) {
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
          const uint32_t gi = u - n_total;
          bool open = false;
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
          const uint32_t open_mask = __ballot_sync(0xffffffffu, open);
          if (open_mask) {
            if (STATS && open) ++n_open;
            const uint2 kd = __ldg(&b.kids[gi]);
            const bool kx_ok = (kd.x - sd.off) < sd.n || (kd.x - int_lo) < int_n;
            const bool ky_ok = (kd.y - sd.off) < sd.n || (kd.y - int_lo) < int_n;
            if (!kx_ok || !ky_ok || !stack_push(stk, kd.y, open_mask, lane)) {
              if (lane == 0) raise_err(b.ctl, kx_ok && ky_ok ? kErrStackOverflow : kErrBadIndex);
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
#pragma unroll
        for (int c = 0; c < 3; ++c) b.acc[3 * (size_t)o + c] = dmul(a64[c], sd.g);
      }
      if (STATS) {
        n_leaf = warp_sum64(n_leaf);
        n_far = warp_sum64(n_far);
        n_open = warp_sum64(n_open);
        if (lane == 0) {
          atomicAdd(&b.ctl->stats[0], n_leaf);
          atomicAdd(&b.ctl->stats[1], n_far);
          atomicAdd(&b.ctl->stats[2], n_open);
          atomicAdd(&b.ctl->stats[4], n_vis);
        }
      }
    }
    if (persistent) {
      uint32_t nxt = 0;
      if (lane == 0) nxt = atomicAdd(&b.counters[kWalkItemCounter], 1u) + warps_total;
      item = __shfl_sync(0xffffffffu, nxt, 0);
    } else {
      item = b.nitems;
    }
  }
}

namespace {

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// FP32 term of one taken internal child's quadrupole (r = x - com = -d):
// a += Q r / r^5 - 2.5 (r.Q r) r / r^7, with r^2 softened like the monopole.
__device__ __forceinline__ void quad_term(const float4& qa, const float4& qb, float dx, float dy, float dz, float inv,
                                          float t[3]) {
  const float inv2 = inv * inv;
  const float inv5 = inv2 * inv2 * inv;
  const float rx = -dx, ry = -dy, rz = -dz;
  const float qx = qa.x * rx + qa.y * ry + qa.z * rz;
  const float qy = qa.y * rx + qa.w * ry + qb.x * rz;
  const float qz = qa.z * rx + qb.x * ry + qb.y * rz;
  const float rqr = rx * qx + ry * qy + rz * qz;
  const float c7 = 2.5f * rqr * inv5 * inv2;
  t[0] += qx * inv5 - rx * c7;
  t[1] += qy * inv5 - ry * c7;
  t[2] += qz * inv5 - rz * c7;
}

// Opening test for theta >= 1/sqrt(3): the target inside the child's AABB must open it.
// Returns the adjusted (take, open, amb) of a child whose distance test said "take".
__device__ __forceinline__ void inside_test(const StepBufs& b, const float xh[3], uint32_t gi, bool& take, bool& open,
                                            bool& amb) {
  const float4 nc = __ldg(&b.nodeC[gi]);
  const float4 nd4 = __ldg(&b.nodeD[gi]);
  const float q0 = fabsf(xh[0] - nc.x) - nd4.x;
  const float q1 = fabsf(xh[1] - nc.y) - nd4.y;
  const float q2 = fabsf(xh[2] - nc.z) - nd4.z;
  const float t0 = 0x1p-20f * (fabsf(nc.x) + nd4.x) + 1e-30f;
  const float t1 = 0x1p-20f * (fabsf(nc.y) + nd4.y) + 1e-30f;
  const float t2 = 0x1p-20f * (fabsf(nc.z) + nd4.z) + 1e-30f;
  const bool near_face = fabsf(q0) <= t0 || fabsf(q1) <= t1 || fabsf(q2) <= t2;
  const bool inside = q0 < 0.f && q1 < 0.f && q2 < 0.f;
  const bool t = take;
  take = t && !near_face && !inside;
  open = open || (t && !near_face && inside);
  amb = amb || (t && near_face);
}

// FP64 decision of an undecided child with record code c (a leaf is undecided only
// when massless: skip).
__device__ __forceinline__ void resolve(const StepBufs& b, uint32_t k, double theta, uint32_t c, bool& take,
                                        bool& open) {
  int dec = -1;
  if (!(c & kLeafCode)) {
    const double4 p = b.leaf64[k];
    const double x[3] = {p.x, p.y, p.z};
    dec = exact_decision(b.agg64, c, x, theta);
  }
  take = dec == 1;
  open = dec == 0;
}

}  // namespace

#ifndef GX_WALK_MINB
#define GX_WALK_MINB 7  // resident kWalkThreads-thread blocks per SM (72 registers a thread)
#endif

// FP32 walk over sibling-pair records. Each iteration decides both children of one
// opened internal node for every lane that opened it: the pair's record is five
// float4 loads, laid out so that every component pair is a float2 (left, right), and
// the distance, threshold and force arithmetic of the two children runs as sm_100
// packed FP32 instructions (__fadd2_rn / __fmul2_rn / __ffma2_rn). Terms of four
// iterations are summed and added to the lane's Kahan-compensated accumulator. The
// record carries the children's indices, so the next pair is known from the record
// just loaded (one dependent load per iteration); the warp's stack of pending pairs
// lives in shared memory. Indices are clamped into the record array, so even a
// corrupt tree cannot read out of bounds; a clamp or an exhausted iteration budget
// raises the device error word. Each lane takes exactly the reference's set of
// terms; only the order of summation differs from the FP64 walk.
template <bool QUAD, bool KAHAN, bool STATS, bool INSIDE, bool LIST>
__global__ void __launch_bounds__(kWalkThreads, GX_WALK_MINB) k_walk_f32(StepBufs b, int persistent) {
  __shared__ uint2 s_stack[kWalkThreads / 32][kStackCap];  // (internal node, lane mask)
  const int lane = threadIdx.x & 31;
  uint2* stack = s_stack[threadIdx.x >> 5];
  const uint32_t warps_total = (gridDim.x * blockDim.x) >> 5;
  uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n_total = b.n;
  const float4* __restrict__ pairs = b.pairs;
  while (item < b.nitems) {
    const WalkItem it = b.items[item];
    const SysDesc sd = b.sys[it.sys];
    const uint32_t end = sd.off + sd.n;
    // a target list (active-subset walk) names the item's targets; else they are the
    // 32 sorted positions from it.begin
    const uint32_t li = it.begin + lane;
    const bool valid = LIST ? (lane < static_cast<int>(b.group) && li < *b.ntargets) : li < end;
    const uint32_t k = LIST ? (valid ? b.targets[li] : 0u) : li;
    // Kahan state: (x, y) packed, z scalar.
    float2 sxy = f2(0.f, 0.f), cxy = f2(0.f, 0.f);
    float sz = 0.f, cz = 0.f;
    unsigned long long n_leaf = 0, n_far = 0, n_open = 0, n_re = 0, n_vis = 0;
    bool bad = false;
    // The root's box is the system's box, so every target is inside it and every lane
    // opens it -- unless the whole system is massless, when nothing is added.
    const uint32_t root = sd.off;  // internal node 0 of the system
    if (sd.n > 1 && __ldg(&b.agg64[root].m) > 0.0) {
      const float eps2f = __double2float_rn(dmul(sd.eps, sd.eps));
      const float2 eps2 = f2(eps2f, eps2f);
      float xh[3] = {0.f, 0.f, 0.f}, xl[3] = {0.f, 0.f, 0.f};
      if (valid) {
        const double4 p = b.leaf64[k];
        split_ff(p.x, xh[0], xl[0]);
        split_ff(p.y, xh[1], xl[1]);
        split_ff(p.z, xh[2], xl[2]);
      }
      // negated target coordinates, duplicated for both children
      const float2 nxh = f2(-xh[0], -xh[0]), nyh = f2(-xh[1], -xh[1]), nzh = f2(-xh[2], -xh[2]);
      const float2 nxl = f2(-xl[0], -xl[0]), nyl = f2(-xl[1], -xl[1]), nzl = f2(-xl[2], -xl[2]);
      const uint32_t gmax = n_total - 1;
      int sp = 0;
      uint32_t g = root;
      uint32_t mask = __ballot_sync(0xffffffffu, valid);
      const uint32_t max_iters = sd.n + 64u;
      uint32_t iters = 0;
      float2 tx = f2(0.f, 0.f), ty = f2(0.f, 0.f), tz = f2(0.f, 0.f);  // per-child term sums
      // One pair: decide both children for every active lane, add the taken terms,
      // move to the next pair. Returns false when the walk is over (or went wrong).
      auto pair_step = [&]() -> bool {
        bad |= g > gmax;
        g = min(g, gmax);
        if (STATS) ++n_vis;
        const float4* pr = pairs + 5 * (size_t)g;
        const float4 r0 = __ldg(pr), r1 = __ldg(pr + 1), r2 = __ldg(pr + 2), r3 = __ldg(pr + 3), r4 = __ldg(pr + 4);
        // child codes: internal node index, or kLeafCode | leaf index
        const uint32_t cL = __float_as_uint(r4.z), cR = __float_as_uint(r4.w);
        const bool act = (mask >> lane) & 1u;
        // d = (c_hi - x_hi) + (c_lo - x_lo) for both children at once
        const float2 dx = __fadd2_rn(__fadd2_rn(f2(r0.x, r0.y), nxh), __fadd2_rn(f2(r2.x, r2.y), nxl));
        const float2 dy = __fadd2_rn(__fadd2_rn(f2(r0.z, r0.w), nyh), __fadd2_rn(f2(r2.z, r2.w), nyl));
        const float2 dz = __fadd2_rn(__fadd2_rn(f2(r1.x, r1.y), nzh), __fadd2_rn(f2(r3.x, r3.y), nzl));
        const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        bool tL = act && d2.x > r3.z, tR = act && d2.y > r3.w;
        bool oL = act && d2.x < r4.x, oR = act && d2.y < r4.y;
        bool aL = act && !tL && !oL, aR = act && !tR && !oR;
        if (INSIDE) {
          if (tL && !(cL & kLeafCode)) inside_test(b, xh, cL, tL, oL, aL);
          if (tR && !(cR & kLeafCode)) inside_test(b, xh, cR, tR, oR, aR);
        }
        if (__any_sync(0xffffffffu, aL || aR)) {
          if (STATS) n_re += (aL ? 1 : 0) + (aR ? 1 : 0);
          if (aL) resolve(b, k, sd.theta, cL, tL, oL);
          if (aR) resolve(b, k, sd.theta, cR, tR, oR);
        }
        // Plummer-softened monopole terms; r^2 > 0 keeps the target's own leaf (d = 0)
        // an exact zero term.
        const float2 r2s = __fadd2_rn(d2, eps2);
        const float invL = rsqrtf(fmaxf(r2s.x, 1e-30f)), invR = rsqrtf(fmaxf(r2s.y, 1e-30f));
        const float2 inv = f2(invL, invR);
        const float2 inv3 = __fmul2_rn(inv, __fmul2_rn(inv, inv));
        float2 f = __fmul2_rn(f2(r1.z, r1.w), inv3);
        f.x = tL ? f.x : 0.f;
        f.y = tR ? f.y : 0.f;
        tx = __ffma2_rn(dx, f, tx);
        ty = __ffma2_rn(dy, f, ty);
        tz = __ffma2_rn(dz, f, tz);
        if (QUAD) {
          float tq[3] = {0.f, 0.f, 0.f};
          if (tL && !(cL & kLeafCode))
            quad_term(__ldg(&b.nodeQ[2 * (size_t)cL]), __ldg(&b.nodeQ[2 * (size_t)cL + 1]), dx.x, dy.x, dz.x, invL, tq);
          if (tR && !(cR & kLeafCode))
            quad_term(__ldg(&b.nodeQ[2 * (size_t)cR]), __ldg(&b.nodeQ[2 * (size_t)cR + 1]), dx.y, dy.y, dz.y, invR, tq);
          tx.x += tq[0];
          ty.x += tq[1];
          tz.x += tq[2];
        }
        if (STATS) {
          const uint32_t self = kLeafCode | k;
          n_leaf += (tL && (cL & kLeafCode) && cL != self ? 1 : 0) + (tR && (cR & kLeafCode) && cR != self ? 1 : 0);
          n_far += (tL && !(cL & kLeafCode) ? 1 : 0) + (tR && !(cR & kLeafCode) ? 1 : 0);
          n_open += (oL ? 1 : 0) + (oR ? 1 : 0);
        }
        const uint32_t m0 = __ballot_sync(0xffffffffu, oL);
        const uint32_t m1 = __ballot_sync(0xffffffffu, oR);
        if (m0) {
          if (m1) {
            // push the right child; continue with the left one
            if (sp >= kStackCap) {
              bad = true;
              return false;
            }
            if (lane == 0) stack[sp] = make_uint2(cR, m1);
            ++sp;
          }
          g = cL;
          mask = m0;
        } else if (m1) {
          g = cR;
          mask = m1;
        } else {
          if (sp == 0) return false;
          __syncwarp();
          const uint2 e = stack[--sp];
          g = e.x;
          mask = e.y;
        }
        return true;
      };
      // fold the children's sums of the last four pairs and add them with compensation
      auto fold = [&]() {
        const float2 txy = f2(tx.x + tx.y, ty.x + ty.y);
        const float tzz = tz.x + tz.y;
        if (KAHAN) {
          const float2 y = __fadd2_rn(txy, f2(-cxy.x, -cxy.y));
          const float2 u = __fadd2_rn(sxy, y);
          cxy = __fadd2_rn(__fadd2_rn(u, f2(-sxy.x, -sxy.y)), f2(-y.x, -y.y));
          sxy = u;
          const float yz = tzz - cz;
          const float uz = sz + yz;
          cz = (uz - sz) - yz;
          sz = uz;
        } else {
          sxy = __fadd2_rn(sxy, txy);
          sz += tzz;
        }
        tx = ty = tz = f2(0.f, 0.f);
      };
      for (;;) {
        // the iteration budget is checked once per four pairs
        iters += 4;
        if (iters > max_iters) {
          bad = true;
          break;
        }
        if (!pair_step() || !pair_step() || !pair_step() || !pair_step()) break;
        fold();
      }
      // fold what is left
      const float2 txy = f2(tx.x + tx.y, ty.x + ty.y);
      const float tzz = tz.x + tz.y;
      if (KAHAN) {
        const float2 y = __fadd2_rn(txy, f2(-cxy.x, -cxy.y));
        const float2 u = __fadd2_rn(sxy, y);
        cxy = __fadd2_rn(__fadd2_rn(u, f2(-sxy.x, -sxy.y)), f2(-y.x, -y.y));
        sxy = u;
        const float yz = tzz - cz;
        const float uz = sz + yz;
        cz = (uz - sz) - yz;
        sz = uz;
      } else {
        sxy = __fadd2_rn(sxy, txy);
        sz += tzz;
      }
      __syncwarp();  // the next item's pushes must not race this item's last pop
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) raise_err(b.ctl, kErrBadIndex);
    if (valid) {
      const uint32_t o = b.order[k];
      const float ax = KAHAN ? __fsub_rn(sxy.x, cxy.x) : sxy.x;
      const float ay = KAHAN ? __fsub_rn(sxy.y, cxy.y) : sxy.y;
      const float az = KAHAN ? __fsub_rn(sz, cz) : sz;
      b.acc[3 * (size_t)o + 0] = dmul(static_cast<double>(ax), sd.g);
      b.acc[3 * (size_t)o + 1] = dmul(static_cast<double>(ay), sd.g);
      b.acc[3 * (size_t)o + 2] = dmul(static_cast<double>(az), sd.g);
    }
    if (STATS) {
      n_leaf = warp_sum64(n_leaf);
      n_far = warp_sum64(n_far);
      n_open = warp_sum64(n_open);
      n_re = warp_sum64(n_re);
      const uint32_t n_valid = __popc(__ballot_sync(0xffffffffu, valid));  // the root, opened by all
      if (lane == 0) {
        atomicAdd(&b.ctl->stats[0], n_leaf);
        atomicAdd(&b.ctl->stats[1], n_far);
        atomicAdd(&b.ctl->stats[2], n_open + (sd.n > 1 ? n_valid : 0u));
        atomicAdd(&b.ctl->stats[3], n_re);
        atomicAdd(&b.ctl->stats[4], n_vis);
      }
    }
    if (persistent) {
      uint32_t nxt = 0;
      if (lane == 0) nxt = atomicAdd(&b.counters[kWalkItemCounter], 1u) + warps_total;
      item = __shfl_sync(0xffffffffu, nxt, 0);
    } else {
      item = b.nitems;
    }
  }
}

namespace {

template <class K>
void launch_k(K kern, const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  const int block = cfg.block > 0 ? cfg.block : 256;
  const int wpb = block / 32;
  if (cfg.persistent_ctas > 0) {
    kern<<<cfg.persistent_ctas, block, 0, st>>>(b, 1);
  } else {
    const uint32_t grid = (b.nitems + wpb - 1) / wpb;
    if (grid) kern<<<grid, block, 0, st>>>(b, 0);
  }
}

template <bool QUAD, bool KAHAN, bool LIST>
void dispatch_f32(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  if (cfg.stats) {
    if (cfg.inside_test)
      launch_k(k_walk_f32<QUAD, KAHAN, true, true, LIST>, b, cfg, st);
    else
      launch_k(k_walk_f32<QUAD, KAHAN, true, false, LIST>, b, cfg, st);
  } else {
    if (cfg.inside_test)
      launch_k(k_walk_f32<QUAD, KAHAN, false, true, LIST>, b, cfg, st);
    else
      launch_k(k_walk_f32<QUAD, KAHAN, false, false, LIST>, b, cfg, st);
  }
}

template <bool LIST>
void dispatch(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  if (cfg.precision == 1) {
    // The FP64 walk has no quadrupole or compensation variants: it is the
    // reference's arithmetic.
    if (cfg.stats)
      launch_k(k_walk_f64<true, LIST>, b, cfg, st);
    else
      launch_k(k_walk_f64<false, LIST>, b, cfg, st);
  } else if (cfg.quad) {
    if (cfg.kahan)
      dispatch_f32<true, true, LIST>(b, cfg, st);
    else
      dispatch_f32<true, false, LIST>(b, cfg, st);
  } else {
    if (cfg.kahan)
      dispatch_f32<false, true, LIST>(b, cfg, st);
    else
      dispatch_f32<false, false, LIST>(b, cfg, st);
  }
}

}  // namespace

namespace {

template <class K>
int resident(K kern, int block) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, block, 0) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

}  // namespace

int walk_resident_ctas(const WalkCfg& cfg) {
  const int block = cfg.block > 0 ? cfg.block : kWalkThreads;
  if (cfg.precision == 1) return resident(k_walk_f64<false, false>, block);
  if (cfg.quad) return resident(k_walk_f32<true, true, false, false, false>, block);
  return resident(k_walk_f32<false, true, false, false, false>, block);
}

void launch_walk(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  // A target list (active-subset walk) has its own instantiations, so the full walk's
  // code is not burdened with it.
  if (b.targets)
    dispatch<true>(b, cfg, st);
  else
    dispatch<false>(b, cfg, st);
}

}  // namespace gx
