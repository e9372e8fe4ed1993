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
template <bool STATS>
__global__ void __launch_bounds__(256) k_walk_f64(StepBufs b, int persistent) {
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
      if (lane == 0) nxt = atomicAdd(&b.counters[4], 1u) + warps_total;
      item = __shfl_sync(0xffffffffu, nxt, 0);
    } else {
      item = b.nitems;
    }
  }
}

namespace {

// Per-lane state of the FP32 walk.
struct Lane32 {
  float xh[3], xl[3];
  uint32_t k;
  float eps2f;
  double theta;
};

// FP32 opening decision state of one child for one lane.
struct Child32 {
  float dx, dy, dz, d2;
  bool take, open, amb;
};

// Distance and threshold tests of node u (A = rec[4u], B = rec[4u+1], open_thr =
// rec[4u+2].z, -2 for leaves) for a lane; no branches. take: a term; open: descend;
// amb: the FP32 value is inside the guard band and must be re-decided in FP64.
template <bool INSIDE>
__device__ __forceinline__ Child32 classify(const StepBufs& b, const Lane32& L, bool act, uint32_t u,
                                            const float4& A, const float4& B, float open_thr, uint32_t n_total) {
  Child32 c;
  c.dx = (A.x - L.xh[0]) + (B.x - L.xl[0]);
  c.dy = (A.y - L.xh[1]) + (B.y - L.xl[1]);
  c.dz = (A.z - L.xh[2]) + (B.z - L.xl[2]);
  c.d2 = fmaf(c.dx, c.dx, fmaf(c.dy, c.dy, c.dz * c.dz));
  // The target itself and massless subtrees are skipped (lbvh.rs:485-496).
  const bool ok = act && (u != L.k) && (A.w > 0.f);
  c.take = ok && (c.d2 > B.w);  // B.w: take threshold (-1 for leaves)
  c.open = ok && (c.d2 < open_thr);
  c.amb = ok && !c.take && !c.open;
  if (INSIDE && u >= n_total) {
    const float4 nc = __ldg(&b.rec[4 * (size_t)u + 3]);
    const float4 nd4 = __ldg(&b.nodeD[u - n_total]);
    const float q0 = fabsf(L.xh[0] - nc.x) - nd4.x;
    const float q1 = fabsf(L.xh[1] - nc.y) - nd4.y;
    const float q2 = fabsf(L.xh[2] - nc.z) - nd4.z;
    const float t0 = 0x1p-20f * (fabsf(nc.x) + nd4.x) + 1e-30f;
    const float t1 = 0x1p-20f * (fabsf(nc.y) + nd4.y) + 1e-30f;
    const float t2 = 0x1p-20f * (fabsf(nc.z) + nd4.z) + 1e-30f;
    const bool near_face = fabsf(q0) <= t0 || fabsf(q1) <= t1 || fabsf(q2) <= t2;
    const bool inside = q0 < 0.f && q1 < 0.f && q2 < 0.f;
    const bool t = c.take;
    c.take = t && !near_face && !inside;
    c.open = c.open || (t && !near_face && inside);
    c.amb = c.amb || (t && near_face);
  }
  return c;
}

// The term of a taken node (Plummer-softened monopole, plus the quadrupole of an
// internal node in QUAD mode), scaled by `take` (0 or 1) and added to t[].
template <bool QUAD>
__device__ __forceinline__ void add_term(const StepBufs& b, const Lane32& L, const Child32& c, bool take, float m,
                                         uint32_t u, uint32_t n_total, float t[3]) {
  const float r2 = c.d2 + L.eps2f;
  const float inv = rsqrtf(r2);
  const float inv2 = inv * inv;
  const float inv3 = inv * inv2;
  const float f = take ? m * inv3 : 0.f;
  t[0] = fmaf(c.dx, f, t[0]);
  t[1] = fmaf(c.dy, f, t[1]);
  t[2] = fmaf(c.dz, f, t[2]);
  if (QUAD && u >= n_total) {
    const uint32_t gi = u - n_total;
    const float4 qa = __ldg(&b.nodeQ[2 * (size_t)gi]);
    const float4 qb = __ldg(&b.nodeQ[2 * (size_t)gi + 1]);
    // r = x - com = -d;  a += Q r / r^5 - 2.5 (r.Q r) r / r^7
    const float rx = -c.dx, ry = -c.dy, rz = -c.dz;
    const float qx = qa.x * rx + qa.y * ry + qa.z * rz;
    const float qy = qa.y * rx + qa.w * ry + qb.x * rz;
    const float qz = qa.z * rx + qb.x * ry + qb.y * rz;
    const float rqr = rx * qx + ry * qy + rz * qz;
    const float inv5 = take ? inv3 * inv2 : 0.f;
    const float c7 = 2.5f * rqr * inv5 * inv2;
    t[0] += qx * inv5 - rx * c7;
    t[1] += qy * inv5 - ry * c7;
    t[2] += qz * inv5 - rz * c7;
  }
}

__device__ __forceinline__ void resolve_amb(const StepBufs& b, const Lane32& L, Child32& c, uint32_t u,
                                            uint32_t n_total) {
  if (c.amb) {
    const double4 p = b.leaf64[L.k];
    const double x[3] = {p.x, p.y, p.z};
    const bool acc = exact_accept(b.agg64, u - n_total, x, L.theta);
    c.take = acc;
    c.open = !acc;
  }
}

}  // namespace

// FP32 walk: each iteration decides the two children of one opened node for every
// lane that opened it; their terms are summed and added to the lane's Kahan-
// compensated accumulator. A node's record carries its children and both FP32
// thresholds, so the next pair to decide is known from the records just loaded (one
// dependent load per iteration), and the stack holds ready-to-load child pairs. The
// decisions are predicated (no per-lane branches); the rare FP64 re-check runs only
// when some lane of the warp needs it. Indices are clamped into the record array, so
// even a corrupt tree cannot read out of bounds; a clamp or an exhausted iteration
// budget raises the device error word. Each lane takes exactly the reference's set of
// terms; only the order of summation differs from the FP64 walk.
#ifndef GX_WALK_MINB
#define GX_WALK_MINB 3  // resident 256-thread blocks per SM the register budget is sized for
#endif

template <bool QUAD, bool KAHAN, bool STATS, bool INSIDE>
__global__ void __launch_bounds__(256, GX_WALK_MINB) k_walk_f32(StepBufs b, int persistent) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps_total = (gridDim.x * blockDim.x) >> 5;
  uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n_total = b.n;
  const uint32_t umax = 2 * n_total - 2;  // largest unified node index
  const float4* __restrict__ rec = b.rec;
  while (item < b.nitems) {
    const WalkItem it = b.items[item];
    const SysDesc sd = b.sys[it.sys];
    const uint32_t end = sd.off + sd.n;
    Lane32 L;
    L.k = it.begin + lane;
    const bool valid = L.k < end;
    Acc32 acc = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    unsigned long long n_leaf = 0, n_far = 0, n_open = 0, n_re = 0, n_vis = 0;
    const uint32_t root = n_total + sd.off;
    bool bad = false;
    // The root's box is the system's box, so every target is inside it and every lane
    // opens it -- unless the whole system is massless, when nothing is added.
    if (sd.n > 1 && __ldg(&rec[4 * (size_t)root]).w > 0.f) {
      L.eps2f = __double2float_rn(dmul(sd.eps, sd.eps));
      L.theta = sd.theta;
      if (valid) {
        const float4 ha = rec[4 * (size_t)L.k], hb = rec[4 * (size_t)L.k + 1];
        L.xh[0] = ha.x;
        L.xh[1] = ha.y;
        L.xh[2] = ha.z;
        L.xl[0] = hb.x;
        L.xl[1] = hb.y;
        L.xl[2] = hb.z;
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) L.xh[c] = L.xl[c] = 0.f;
      }
      // pair stack of kStackCap entries: entry j in lane j % 32 of slot j / 32
      uint32_t sx0 = 0, sy0 = 0, sm0 = 0, sx1 = 0, sy1 = 0, sm1 = 0, sx2 = 0, sy2 = 0, sm2 = 0;
      int sp = 0;
      const float4 r2 = __ldg(&rec[4 * (size_t)root + 2]);
      uint32_t cx = __float_as_uint(r2.x), cy = __float_as_uint(r2.y);
      uint32_t mask = __ballot_sync(0xffffffffu, valid);
      const uint32_t max_iters = sd.n + 64u;
      uint32_t iters = 0;
      for (;;) {
        bad |= (cx > umax) | (cy > umax);
        if (++iters > max_iters) {
          bad = true;
          break;
        }
        cx = min(cx, umax);
        cy = min(cy, umax);
        if (STATS) ++n_vis;
        const float4* p0 = rec + 4 * (size_t)cx;
        const float4* p1 = rec + 4 * (size_t)cy;
        const float4 a0 = __ldg(p0), b0 = __ldg(p0 + 1);
        const float4 a1 = __ldg(p1), b1 = __ldg(p1 + 1);
        const float4 k0 = cx >= n_total ? __ldg(p0 + 2) : make_float4(0.f, 0.f, -2.f, 0.f);
        const float4 k1 = cy >= n_total ? __ldg(p1 + 2) : make_float4(0.f, 0.f, -2.f, 0.f);
        const bool act = (mask >> lane) & 1u;
        Child32 c0 = classify<INSIDE>(b, L, act, cx, a0, b0, k0.z, n_total);
        Child32 c1 = classify<INSIDE>(b, L, act, cy, a1, b1, k1.z, n_total);
        if (__any_sync(0xffffffffu, c0.amb || c1.amb)) {
          if (STATS) n_re += (c0.amb ? 1 : 0) + (c1.amb ? 1 : 0);
          resolve_amb(b, L, c0, cx, n_total);
          resolve_amb(b, L, c1, cy, n_total);
        }
        float t[3] = {0.f, 0.f, 0.f};
        add_term<QUAD>(b, L, c0, c0.take, a0.w, cx, n_total, t);
        add_term<QUAD>(b, L, c1, c1.take, a1.w, cy, n_total, t);
        acc_add<KAHAN>(acc, t[0], t[1], t[2]);
        if (STATS) {
          n_leaf += (c0.take && cx < n_total ? 1 : 0) + (c1.take && cy < n_total ? 1 : 0);
          n_far += (c0.take && cx >= n_total ? 1 : 0) + (c1.take && cy >= n_total ? 1 : 0);
          n_open += (c0.open ? 1 : 0) + (c1.open ? 1 : 0);
        }
        const uint32_t m0 = __ballot_sync(0xffffffffu, c0.open);
        const uint32_t m1 = __ballot_sync(0xffffffffu, c1.open);
        const uint32_t n0x = __float_as_uint(k0.x), n0y = __float_as_uint(k0.y);
        const uint32_t n1x = __float_as_uint(k1.x), n1y = __float_as_uint(k1.y);
        if (m0 && m1) {
          // push the right child's pair; continue with the left child's
          if (sp >= kStackCap) {
            bad = true;
            break;
          }
          const bool w0 = lane == sp, w1 = lane == sp - 32, w2 = lane == sp - 64;
          sx0 = w0 ? n1x : sx0;
          sy0 = w0 ? n1y : sy0;
          sm0 = w0 ? m1 : sm0;
          sx1 = w1 ? n1x : sx1;
          sy1 = w1 ? n1y : sy1;
          sm1 = w1 ? m1 : sm1;
          sx2 = w2 ? n1x : sx2;
          sy2 = w2 ? n1y : sy2;
          sm2 = w2 ? m1 : sm2;
          ++sp;
        }
        if (m0) {
          cx = n0x;
          cy = n0y;
          mask = m0;
        } else if (m1) {
          cx = n1x;
          cy = n1y;
          mask = m1;
        } else {
          if (sp == 0) break;
          --sp;
          const int src = sp & 31;
          const int slot = sp >> 5;
          cx = __shfl_sync(0xffffffffu, slot == 0 ? sx0 : (slot == 1 ? sx1 : sx2), src);
          cy = __shfl_sync(0xffffffffu, slot == 0 ? sy0 : (slot == 1 ? sy1 : sy2), src);
          mask = __shfl_sync(0xffffffffu, slot == 0 ? sm0 : (slot == 1 ? sm1 : sm2), src);
        }
      }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) raise_err(b.ctl, kErrBadIndex);
    if (valid) {
      const uint32_t o = b.order[L.k];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float v = KAHAN ? __fsub_rn(acc.s[c], acc.c[c]) : acc.s[c];
        b.acc[3 * (size_t)o + c] = dmul(static_cast<double>(v), sd.g);
      }
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
      if (lane == 0) nxt = atomicAdd(&b.counters[4], 1u) + warps_total;
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

template <bool QUAD, bool KAHAN>
void dispatch_f32(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  if (cfg.stats) {
    if (cfg.inside_test)
      launch_k(k_walk_f32<QUAD, KAHAN, true, true>, b, cfg, st);
    else
      launch_k(k_walk_f32<QUAD, KAHAN, true, false>, b, cfg, st);
  } else {
    if (cfg.inside_test)
      launch_k(k_walk_f32<QUAD, KAHAN, false, true>, b, cfg, st);
    else
      launch_k(k_walk_f32<QUAD, KAHAN, false, false>, b, cfg, st);
  }
}

}  // namespace

void launch_walk(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  if (cfg.precision == 1) {
    // The FP64 walk has no quadrupole or compensation variants: it is the
    // reference's arithmetic.
    if (cfg.stats)
      launch_k(k_walk_f64<true>, b, cfg, st);
    else
      launch_k(k_walk_f64<false>, b, cfg, st);
  } else if (cfg.quad) {
    if (cfg.kahan)
      dispatch_f32<true, true>(b, cfg, st);
    else
      dispatch_f32<true, false>(b, cfg, st);
  } else {
    if (cfg.kahan)
      dispatch_f32<false, true>(b, cfg, st);
    else
      dispatch_f32<false, false>(b, cfg, st);
  }
}

}  // namespace gx
