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

// True when internal node gi's AABB (FP32 centre / half extents, rounded from FP64) and
// the targets' padded box (negated faces nlo, nhi) are apart along some axis by more than
// the rounding of the FP32 box, so that no target is inside the node.
__device__ __forceinline__ bool boxes_apart(const StepBufs& b, uint32_t gi, const float2 nlo[3], const float2 nhi[3]) {
  const float4 nc = __ldg(&b.nodeC[gi]);
  const float4 nd = __ldg(&b.nodeD[gi]);
  const float c[3] = {nc.x, nc.y, nc.z}, h[3] = {nd.x, nd.y, nd.z};
  bool apart = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float m = 0x1p-20f * (fabsf(c[a]) + h[a]) + 1e-30f;
    const float lo = -nlo[a].x, hi = -nhi[a].x;
    apart = apart || lo > c[a] + h[a] + m || hi < c[a] - h[a] - m;
  }
  return apart;
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
#define GX_WALK_MINB 4  // resident kWalkThreads-thread blocks per SM (shared memory bounds it at 4)
#endif

namespace {

// Margins of the warp-wide (group) opening test. A child is taken for every target of
// the warp when the squared distance from its centre of mass to the targets' bounding
// box, times (1 - 2^-20), exceeds the child's take threshold, and opened for every
// target when the squared distance to the box's farthest corner, times (1 + 2^-20),
// is below its open threshold. The box is padded by 2^-21 of its coordinates, which
// covers the float-float split of every target, and the margins cover the FP32
// rounding of the box distances (a few ulps), so a group decision is the decision
// the reference's exact test makes for each target: the thresholds already hold the
// 4e-6 band around rcrit^2.
constexpr float kGroupLo = 1.0f - 0x1p-20f;
// Per-warp stack and list sizes of the FP32 walk (see WarpLists).
constexpr int kWalkStack = 512;  // stack entries
constexpr int kWalkDeep = 224;   // above this many stacked entries a round takes one entry
constexpr int kWalkList = 96;    // entries per list: at most 31 left after an evaluation + 64 a round
constexpr int kWalkFlush = 32;   // a list is evaluated once it holds this many entries
constexpr float kGroupHi = 1.0f + 0x1p-20f;

// Order-preserving map of a float onto a signed int (for warp min / max reductions).
__device__ __forceinline__ int ford(float f) {
  const int i = __float_as_int(f);
  return i ^ ((i >> 31) & 0x7fffffff);
}
__device__ __forceinline__ float fdeord(int i) { return __int_as_float(i ^ ((i >> 31) & 0x7fffffff)); }

// Two list entries share each float4: entry e is half (e & 1) of float4 e >> 1, so a
// broadcast load of one float4 yields (entry 2p, entry 2p + 1) operand pairs for the
// packed FP32 instructions.
__device__ __forceinline__ void put2(float4* a, int e, float v0, float v1) {
  float* p = reinterpret_cast<float*>(a + (e >> 1)) + (e & 1);
  p[0] = v0;
  p[2] = v1;
}

}  // namespace

// Per-warp shared memory of the FP32 walk.
//   stk: (internal node, target mask) -- the node was opened for the targets in the mask
//        and its two children are still to be decided for them;
//   dense list: children every target of their mask takes (leaves, or nodes the group
//        test accepted for the whole warp): evaluated with no per-target decision, in
//        FP32 coordinates relative to the centre of the warp's target box;
//   undecided list: children some targets take and others open (or that need the FP64
//        re-decision), evaluated with each target's own decision on float-float
//        coordinates; afterwards each entry holds the mask of the targets that opened it.
// Two entries share each float4: entry e is half (e & 1) of float4 e >> 1.
struct WarpLists {
  uint2 stk[kWalkStack];
  float4 da[kWalkList / 2], db[kWalkList / 2];  // (x, y) (z, m) relative to the box centre
  uint2 dm[kWalkList / 2];                      // target masks
  uint32_t dcode[kWalkList];                    // child codes (quadrupole terms, statistics)
  float4 ua[kWalkList / 2], ub[kWalkList / 2], uc[kWalkList / 2], ud[kWalkList / 2], ue[kWalkList / 2],
      uf[kWalkList / 2];  // (xh,yh) (zh,m) (xl,yl) (zl,take) (open,code) (mask,opened)
  // The targets' padded box as negated faces (lo, hi) and its negated centre o, each
  // duplicated for packed pairs: warp-uniform, read by the rounds only (kept here rather
  // than in 18 registers of every lane).
  float2 nlo[3], nhi[3], no[3];
  float2 pad;
};
static_assert(sizeof(WarpLists) % 16 == 0, "warp lists keep 16-byte alignment");

// Bound of the stack: a normal round starts at most kWalkDeep entries high and pushes at
// most one entry per popped one (2 children each, <= 32 popped), an undecided evaluation
// pushes at most one entry per list entry (< kWalkList), the first deep round at most
// 2 + 33, and then the depth-first growth adds at most one entry per tree level.
static_assert(kWalkDeep + 32 + (kWalkList - 1) + 35 + kMaxDepth <= kWalkStack, "walk stack bound");

// Quadrupole mode: each listed internal node's traceless moments, fetched once by the lane
// that lists it and stored with the two entries of a pair side by side, as the packed
// evaluation reads them: a = (xx, xx', xy, xy'), b = (xz, xz', yy, yy'), c = (yz, yz', zz, zz').
// Slots of leaf entries are never written: the evaluation gives them a zero inverse
// distance, and the arrays are cleared at the kernel's start so that every slot holds
// finite values.
struct WarpQuads {
  float4 dqa[kWalkList / 2], dqb[kWalkList / 2], dqc[kWalkList / 2];
  float4 uqa[kWalkList / 2], uqb[kWalkList / 2], uqc[kWalkList / 2];
};

size_t walk_smem_bytes(int block, bool quad) {
  return static_cast<size_t>(block / 32) * (sizeof(WarpLists) + (quad ? sizeof(WarpQuads) : 0));
}

namespace {

// Plummer-softened monopole terms of two entries for one target: t += d m / (d^2 + eps^2)^1.5
// where the target takes the entry (t0, t1). r^2 is clamped at 1e-24 so that a zero
// distance (the target's own leaf) gives an exact zero term even without softening.
__device__ __forceinline__ void mono2(float2 dx, float2 dy, float2 dz, float2 m, float2 eps2, bool t0, bool t1,
                                      float2& tx, float2& ty, float2& tz, float& i0, float& i1) {
  const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
  const float2 r2s = __fadd2_rn(d2, eps2);
  i0 = rsqrtf(fmaxf(r2s.x, 1e-24f));
  i1 = rsqrtf(fmaxf(r2s.y, 1e-24f));
  const float2 inv = f2(i0, i1);
  const float2 inv3 = __fmul2_rn(inv, __fmul2_rn(inv, inv));
  float2 f = __fmul2_rn(m, inv3);
  f.x = t0 ? f.x : 0.f;
  f.y = t1 ? f.y : 0.f;
  tx = __ffma2_rn(dx, f, tx);
  ty = __ffma2_rn(dy, f, ty);
  tz = __ffma2_rn(dz, f, tz);
}

// Stores entry e's moments (xx, xy, xz, yy), (yz, zz) into the pair layout of WarpQuads.
__device__ __forceinline__ void put_quad(float4* qa, float4* qb, float4* qc, int e, const float4& a, const float4& c) {
  const int p = e >> 1, h = e & 1;
  float* A = reinterpret_cast<float*>(qa + p) + h;
  float* B = reinterpret_cast<float*>(qb + p) + h;
  float* C = reinterpret_cast<float*>(qc + p) + h;
  A[0] = a.x;
  A[2] = a.y;
  B[0] = a.z;
  B[2] = a.w;
  C[0] = c.x;
  C[2] = c.y;
}

// Quadrupole terms of the two entries of a pair for one target, packed FP32, added to the
// monopole accumulator: with r = x - com = -d, a += Q r / r^5 - 2.5 (r.Q r) r / r^7
// = -(Q d) / r^5 + 2.5 (d.Q d) d / r^7, r^2 softened like the monopole. inv is the
// inverse distance of an entry the target takes as an internal node, else 0.
__device__ __forceinline__ void quad2(float2 dx, float2 dy, float2 dz, float2 inv, const float4& qa, const float4& qb,
                                      const float4& qc, float2& tx, float2& ty, float2& tz) {
  const float2 xx = f2(qa.x, qa.y), xy = f2(qa.z, qa.w), xz = f2(qb.x, qb.y);
  const float2 yy = f2(qb.z, qb.w), yz = f2(qc.x, qc.y), zz = f2(qc.z, qc.w);
  const float2 qx = __ffma2_rn(xx, dx, __ffma2_rn(xy, dy, __fmul2_rn(xz, dz)));
  const float2 qy = __ffma2_rn(xy, dx, __ffma2_rn(yy, dy, __fmul2_rn(yz, dz)));
  const float2 qz = __ffma2_rn(xz, dx, __ffma2_rn(yz, dy, __fmul2_rn(zz, dz)));
  const float2 dqd = __ffma2_rn(dx, qx, __ffma2_rn(dy, qy, __fmul2_rn(dz, qz)));
  const float2 inv2 = __fmul2_rn(inv, inv);
  const float2 ninv5 = __fmul2_rn(__fmul2_rn(inv2, inv2), f2(-inv.x, -inv.y));      // -1 / r^5
  const float2 c7 = __fmul2_rn(__fmul2_rn(f2(-2.5f, -2.5f), dqd), __fmul2_rn(ninv5, inv2));  // 2.5 dQd / r^7
  tx = __ffma2_rn(dx, c7, __ffma2_rn(qx, ninv5, tx));
  ty = __ffma2_rn(dy, c7, __ffma2_rn(qy, ninv5, ty));
  tz = __ffma2_rn(dz, c7, __ffma2_rn(qz, ninv5, tz));
}

}  // namespace

// FP32 walk: one warp per G Morton-consecutive targets (G = 8, 16 or 32: the system's
// grouping, or the target list's), R = 32 / G lanes a target; the warp visits the union
// of their walks (each node is decided once for every target that reached it) but not
// one node at a time. A round pops up to 32 opened nodes from the warp's stack, one per
// lane, loads each one's sibling-pair record (both children: float-float centre of mass,
// mass, FP32 take / open thresholds, child codes) and decides each child for the whole
// warp against the padded bounding box of the warp's targets:
//   - taken by every target (or a leaf): appended to the dense list;
//   - opened by every target: pushed back on the stack with the same target mask;
//   - otherwise: appended to the undecided list.
// A list holding 32 entries is evaluated by all lanes together (the R lanes of a target
// take turns over its entries), four entries a lane-iteration with packed FP32: the dense
// list with no decisions, the undecided list with each target's exact test (FP64
// re-decision in the band, the inside test for theta >= 1/sqrt 3); the targets that open
// an undecided entry are recorded in it, and one pass afterwards pushes the opened
// entries. Rounds, lists and entries are independent of one another, so the walk has no
// dependent chain of one record per step. While the stack holds more than kWalkDeep
// entries, a round takes only the top entry (and evaluates its undecided children at
// once): the stack then grows like a depth-first walk, by at most one entry per tree
// level, which bounds it within kWalkStack. Every target takes exactly the reference's
// set of terms; only the order of summation differs from the FP64 walk. Terms are summed
// four at a time into a Kahan-compensated accumulator. Node indices are clamped into the
// record array and the number of records a warp visits is bounded by the system's node
// count, so even a corrupt tree cannot read out of bounds or loop; a clamp, an exhausted
// budget or a full stack raises the device error word.
template <bool QUAD, bool KAHAN, bool STATS, bool INSIDE, bool LIST>
__global__ void __launch_bounds__(kWalkThreads, GX_WALK_MINB) k_walk_f32(StepBufs b, int persistent) {
  extern __shared__ __align__(16) unsigned char s_walk_raw[];
  WarpLists& L = reinterpret_cast<WarpLists*>(s_walk_raw)[threadIdx.x >> 5];
  WarpQuads& Q = reinterpret_cast<WarpQuads*>(s_walk_raw + (blockDim.x >> 5) * sizeof(WarpLists))[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t warps_total = (gridDim.x * blockDim.x) >> 5;
  uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n_total = b.n;
  const float4* __restrict__ pairs = b.pairs;
  if (QUAD) {
    float4* z = reinterpret_cast<float4*>(&Q);
    for (int i = lane; i < static_cast<int>(sizeof(WarpQuads) / sizeof(float4)); i += 32) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncwarp();
  }
  while (item < b.nitems) {
    const WalkItem it = b.items[item];
    const SysDesc sd = b.sys[it.sys];
    const uint32_t end = sd.off + sd.n;
    // G targets a warp, R = 32 / G lanes a target: lane = sub * G + target, so the lanes of
    // one sub-lane index hold contiguous ballot bits. Masks have one bit per target.
    const uint32_t G = LIST ? b.group : sd.group;
    const int lg = __ffs(G) - 1;
    const uint32_t gmask = G == 32 ? 0xffffffffu : (1u << G) - 1u;
    const int tg = lane & (G - 1), sl = lane >> lg, R = 32 >> lg;
    // a target list (active-subset walk) names the item's G targets; else they are the
    // G sorted positions from it.begin
    const uint32_t li = it.begin + tg;
    const bool valid = LIST ? li < *b.ntargets : li < end;
    const uint32_t k = LIST ? (valid ? b.targets[li] : 0u) : li;
    const uint32_t vmask = __ballot_sync(0xffffffffu, valid) & gmask;
    // Kahan state: (x, y) packed, z scalar.
    float2 sxy = f2(0.f, 0.f), cxy = f2(0.f, 0.f);
    float sz = 0.f, cz = 0.f;
    unsigned long long n_leaf = 0, n_far = 0, n_open = 0, n_re = 0, n_vis = 0;
    bool bad = false;
    // The root's box is the system's box, so every target is inside it and every target
    // opens it -- unless the whole system is massless, when nothing is added.
    const uint32_t root = sd.off;  // internal node 0 of the system
    if (sd.n > 1 && vmask && __ldg(&b.agg64[root].m) > 0.0) {
      const float eps2f = __double2float_rn(dmul(sd.eps, sd.eps));
      const float2 eps2 = f2(eps2f, eps2f);
      // The inside rule (a target inside a node's box opens it) can only bind for
      // theta >= 1/sqrt(3); it follows the system's own theta (as the single-system
      // handle's choice of kernel does), so a system's terms and their order do not
      // depend on the other systems of a batch.
      const bool inside_rule = INSIDE && sd.theta >= 0.57;
      float xh[3] = {0.f, 0.f, 0.f}, xl[3] = {0.f, 0.f, 0.f};
      if (valid) {
        const double4 p = b.leaf64[k];
        split_ff(p.x, xh[0], xl[0]);
        split_ff(p.y, xh[1], xl[1]);
        split_ff(p.z, xh[2], xl[2]);
      }
      // negated target coordinates, duplicated for both entries of a packed pair
      const float2 nxh = f2(-xh[0], -xh[0]), nyh = f2(-xh[1], -xh[1]), nzh = f2(-xh[2], -xh[2]);
      const float2 nxl = f2(-xl[0], -xl[0]), nyl = f2(-xl[1], -xl[1]), nzl = f2(-xl[2], -xl[2]);
      // The targets' padded bounding box as negated faces (lo, hi), duplicated, and its
      // centre o (an FP32 value): dense entries and targets are stored relative to o. A
      // target that is not finite turns the box into all of space: no group decisions.
      const bool fin = isfinite(xh[0]) && isfinite(xh[1]) && isfinite(xh[2]);
      const bool all_fin = __all_sync(0xffffffffu, !valid || fin);
      float xr[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float l = fdeord(__reduce_min_sync(0xffffffffu, valid ? ford(xh[c]) : 0x7fffffff));
        float h = fdeord(__reduce_max_sync(0xffffffffu, valid ? ford(xh[c]) : static_cast<int>(0x80000000u)));
        const float o = all_fin ? 0.5f * l + 0.5f * h : 0.f;
        const float pad = (fabsf(l) + fabsf(h)) * 0x1p-21f + 1e-30f;
        l = all_fin ? l - pad : -INFINITY;
        h = all_fin ? h + pad : INFINITY;
        if (lane == 0) {
          L.nlo[c] = f2(-l, -l);
          L.nhi[c] = f2(-h, -h);
          L.no[c] = f2(-o, -o);
        }
        xr[c] = (xh[c] - o) + xl[c];  // the target relative to o
      }
      const float2 nxr = f2(-xr[0], -xr[0]), nyr = f2(-xr[1], -xr[1]), nzr = f2(-xr[2], -xr[2]);
      const uint32_t gmax = n_total - 1;
      const uint32_t max_pairs = sd.n + 64u;
      uint32_t pairs_done = 0;
      int sp = 1, dl = 0, ul = 0;
      if (lane == 0) L.stk[0] = make_uint2(root, vmask);
      __syncwarp();
      float2 tx = f2(0.f, 0.f), ty = f2(0.f, 0.f), tz = f2(0.f, 0.f);  // per-entry term sums
      // add the term sums of the last entries to the lane's compensated accumulator
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
      auto put_dense = [&](int e, float x_, float y_, float z_, float m_, uint32_t mask, uint32_t code) {
        put2(L.da, e, x_, y_);
        put2(L.db, e, z_, m_);
        reinterpret_cast<uint32_t*>(L.dm + (e >> 1))[e & 1] = mask;
        L.dcode[e] = code;
      };
      auto put_und = [&](int e, float xh_, float yh_, float zh_, float m_, float xl_, float yl_, float zl_,
                         float take, float open, uint32_t code, uint32_t mask) {
        put2(L.ua, e, xh_, yh_);
        put2(L.ub, e, zh_, m_);
        put2(L.uc, e, xl_, yl_);
        put2(L.ud, e, zl_, take);
        put2(L.ue, e, open, __uint_as_float(code));
        put2(L.uf, e, __uint_as_float(mask), 0.f);
      };
      // One round: the top kk stack entries, one per lane, each child decided for the
      // whole warp and appended to a list or pushed back.
      auto round = [&](int kk) {
        const bool act = lane < kk;
        uint32_t g = 0, M = 0;
        if (act) {
          const uint2 e = L.stk[sp - kk + lane];
          g = e.x;
          M = e.y;
        }
        sp -= kk;
        __syncwarp();  // popped before the pushes below overwrite the slots
        bad |= act && g > gmax;
        g = min(g, gmax);
        float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0, r2 = r0, r3 = r0, r4 = r0;
        if (act) {
          const float4* pr = pairs + 5 * (size_t)g;
          r0 = __ldg(pr);
          r1 = __ldg(pr + 1);
          r2 = __ldg(pr + 2);
          r3 = __ldg(pr + 3);
          r4 = __ldg(pr + 4);
        }
        const uint32_t cL = __float_as_uint(r4.z), cR = __float_as_uint(r4.w);
        const float2 nlo[3] = {L.nlo[0], L.nlo[1], L.nlo[2]}, nhi[3] = {L.nhi[0], L.nhi[1], L.nhi[2]};
        const float2 chx = f2(r0.x, r0.y), chy = f2(r0.z, r0.w), chz = f2(r1.x, r1.y);
        const float2 clx = f2(r2.x, r2.y), cly = f2(r2.z, r2.w), clz = f2(r3.x, r3.y);
        // c - lo and c - hi per axis, both children at once
        const float2 lx = __fadd2_rn(__fadd2_rn(chx, nlo[0]), clx), hx = __fadd2_rn(__fadd2_rn(chx, nhi[0]), clx);
        const float2 ly = __fadd2_rn(__fadd2_rn(chy, nlo[1]), cly), hy = __fadd2_rn(__fadd2_rn(chy, nhi[1]), cly);
        const float2 lz = __fadd2_rn(__fadd2_rn(chz, nlo[2]), clz), hz = __fadd2_rn(__fadd2_rn(chz, nhi[2]), clz);
        // distance to the box (0 inside) and to its farthest corner, per axis
        const float2 nx = f2(fmaxf(fmaxf(-lx.x, hx.x), 0.f), fmaxf(fmaxf(-lx.y, hx.y), 0.f));
        const float2 ny = f2(fmaxf(fmaxf(-ly.x, hy.x), 0.f), fmaxf(fmaxf(-ly.y, hy.y), 0.f));
        const float2 nz = f2(fmaxf(fmaxf(-lz.x, hz.x), 0.f), fmaxf(fmaxf(-lz.y, hz.y), 0.f));
        const float2 fx = f2(fmaxf(lx.x, -hx.x), fmaxf(lx.y, -hx.y));
        const float2 fy = f2(fmaxf(ly.x, -hy.x), fmaxf(ly.y, -hy.y));
        const float2 fz = f2(fmaxf(lz.x, -hz.x), fmaxf(lz.y, -hz.y));
        const float2 dmin2 = __ffma2_rn(nx, nx, __ffma2_rn(ny, ny, __fmul2_rn(nz, nz)));
        const float2 dmax2 = __ffma2_rn(fx, fx, __ffma2_rn(fy, fy, __fmul2_rn(fz, fz)));
        bool accL = act && dmin2.x * kGroupLo > r3.z, accR = act && dmin2.y * kGroupLo > r3.w;
        if (inside_rule) {
          // A target inside a node's box opens it: a node is taken for the whole warp only
          // when its box and the targets' box are apart along some axis.
          if (accL && !(cL & kLeafCode)) accL = boxes_apart(b, cL, nlo, nhi);
          if (accR && !(cR & kLeafCode)) accR = boxes_apart(b, cR, nlo, nhi);
        }
        const bool opnL = act && !accL && dmax2.x * kGroupHi < r4.x;
        const bool opnR = act && !accR && dmax2.y * kGroupHi < r4.y;
        const bool undL = act && !accL && !opnL, undR = act && !accR && !opnR;
        const uint32_t bAL = __ballot_sync(0xffffffffu, accL), bAR = __ballot_sync(0xffffffffu, accR);
        const uint32_t bUL = __ballot_sync(0xffffffffu, undL), bUR = __ballot_sync(0xffffffffu, undR);
        const uint32_t bOL = __ballot_sync(0xffffffffu, opnL), bOR = __ballot_sync(0xffffffffu, opnR);
        const int eAL = dl + __popc(bAL & lt), eAR = dl + __popc(bAL) + __popc(bAR & lt);
        const int eUL = ul + __popc(bUL & lt), eUR = ul + __popc(bUL) + __popc(bUR & lt);
        if (QUAD) {
          // the moments of the listed internal children, loaded side by side
          const bool qL = (accL || undL) && !(cL & kLeafCode), qR = (accR || undR) && !(cR & kLeafCode);
          float4 qaL = make_float4(0.f, 0.f, 0.f, 0.f), qbL = qaL, qaR = qaL, qbR = qaL;
          if (qL) {
            qaL = __ldg(&b.nodeQ[2 * (size_t)cL]);
            qbL = __ldg(&b.nodeQ[2 * (size_t)cL + 1]);
          }
          if (qR) {
            qaR = __ldg(&b.nodeQ[2 * (size_t)cR]);
            qbR = __ldg(&b.nodeQ[2 * (size_t)cR + 1]);
          }
          if (qL && accL) put_quad(Q.dqa, Q.dqb, Q.dqc, eAL, qaL, qbL);
          if (qL && undL) put_quad(Q.uqa, Q.uqb, Q.uqc, eUL, qaL, qbL);
          if (qR && accR) put_quad(Q.dqa, Q.dqb, Q.dqc, eAR, qaR, qbR);
          if (qR && undR) put_quad(Q.uqa, Q.uqb, Q.uqc, eUR, qaR, qbR);
        }
        if (accL || accR) {
          // dense entries relative to the box centre: (c_hi - o) + c_lo
          const float2 rx = __fadd2_rn(__fadd2_rn(chx, L.no[0]), clx);
          const float2 ry = __fadd2_rn(__fadd2_rn(chy, L.no[1]), cly);
          const float2 rz = __fadd2_rn(__fadd2_rn(chz, L.no[2]), clz);
          if (accL) put_dense(eAL, rx.x, ry.x, rz.x, r1.z, M, cL);
          if (accR) put_dense(eAR, rx.y, ry.y, rz.y, r1.w, M, cR);
        }
        dl += __popc(bAL) + __popc(bAR);
        if (undL) put_und(eUL, chx.x, chy.x, chz.x, r1.z, clx.x, cly.x, clz.x, r3.z, r4.x, cL, M);
        if (undR) put_und(eUR, chx.y, chy.y, chz.y, r1.w, clx.y, cly.y, clz.y, r3.w, r4.y, cR, M);
        ul += __popc(bUL) + __popc(bUR);
        const int npush = __popc(bOL) + __popc(bOR);
        if (sp + npush > kWalkStack) {
          bad = true;
        } else {
          if (opnL) L.stk[sp + __popc(bOL & lt)] = make_uint2(cL, M);
          if (opnR) L.stk[sp + __popc(bOL) + __popc(bOR & lt)] = make_uint2(cR, M);
          sp += npush;
        }
        if (STATS) {
          n_vis += kk;
          n_open += (opnL ? __popc(M) : 0) + (opnR ? __popc(M) : 0);
        }
        __syncwarp();
      };
      // The dense terms of pair p (entries 2p, 2p + 1) for this lane's target; on = 0 for
      // a lane past the list's end (it reads the last pair with no target bit).
      auto dense_pair = [&](int p, uint32_t on) {
        const float4 A = L.da[p], B = L.db[p];
        const uint2 Mk = L.dm[p];
        const float2 dx = __fadd2_rn(f2(A.x, A.y), nxr);
        const float2 dy = __fadd2_rn(f2(A.z, A.w), nyr);
        const float2 dz = __fadd2_rn(f2(B.x, B.y), nzr);
        const bool t0 = (Mk.x >> tg) & on, t1 = (Mk.y >> tg) & on;
        float i0, i1;
        mono2(dx, dy, dz, f2(B.z, B.w), eps2, t0, t1, tx, ty, tz, i0, i1);
        if (QUAD || STATS) {
          const uint32_t c0 = L.dcode[2 * p], c1 = L.dcode[2 * p + 1];
          if (QUAD) {
            const float2 iq = f2(t0 && !(c0 & kLeafCode) ? i0 : 0.f, t1 && !(c1 & kLeafCode) ? i1 : 0.f);
            quad2(dx, dy, dz, iq, Q.dqa[p], Q.dqb[p], Q.dqc[p], tx, ty, tz);
          }
          if (STATS) {
            const uint32_t self = kLeafCode | k;
            n_leaf += (t0 && (c0 & kLeafCode) && c0 != self ? 1 : 0) + (t1 && (c1 & kLeafCode) && c1 != self ? 1 : 0);
            n_far += (t0 && !(c0 & kLeafCode) ? 1 : 0) + (t1 && !(c1 & kLeafCode) ? 1 : 0);
          }
        }
      };
      // Evaluate the dense list: every target adds the terms of the entries in its mask.
      // The R lanes of a target take pairs (2u, 2u + 1) of quads u = q R + sl.
      auto flush_dense = [&]() {
        if (dl & 1) {
          if (lane == 0) put_dense(dl, 0.f, 0.f, 0.f, 0.f, 0u, kLeafCode);
          __syncwarp();
        }
        const int np = (dl + 1) >> 1;
        for (int q = 0; 2 * q * R < np; ++q) {
          const int pa = 2 * (q * R + sl), pb = pa + 1;
          dense_pair(min(pa, np - 1), pa < np ? 1u : 0u);
          dense_pair(min(pb, np - 1), pb < np ? 1u : 0u);
          fold();
        }
        dl = 0;
        __syncwarp();  // read before the next round overwrites the list
      };
      // The undecided pair p for this lane's target; records the targets that open each
      // entry in the entry (lane sub * G of each sub-lane writes its pair's).
      auto und_pair = [&](int p, uint32_t on) {
        const float4 A = L.ua[p], B = L.ub[p], C = L.uc[p], D = L.ud[p], E = L.ue[p], F = L.uf[p];
        const float2 dx = __fadd2_rn(__fadd2_rn(f2(A.x, A.y), nxh), __fadd2_rn(f2(C.x, C.y), nxl));
        const float2 dy = __fadd2_rn(__fadd2_rn(f2(A.z, A.w), nyh), __fadd2_rn(f2(C.z, C.w), nyl));
        const float2 dz = __fadd2_rn(__fadd2_rn(f2(B.x, B.y), nzh), __fadd2_rn(f2(D.x, D.y), nzl));
        const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        const uint32_t cL = __float_as_uint(E.z), cR = __float_as_uint(E.w);
        const bool a0 = (__float_as_uint(F.x) >> tg) & on, a1 = (__float_as_uint(F.y) >> tg) & on;
        bool tL = a0 && d2.x > D.z, tR = a1 && d2.y > D.w;
        bool oL = a0 && d2.x < E.x, oR = a1 && d2.y < E.y;
        bool aL = a0 && !tL && !oL, aR = a1 && !tR && !oR;
        if (inside_rule) {
          if (tL && !(cL & kLeafCode)) inside_test(b, xh, cL, tL, oL, aL);
          if (tR && !(cR & kLeafCode)) inside_test(b, xh, cR, tR, oR, aR);
        }
        if (__any_sync(0xffffffffu, aL || aR)) {
          if (STATS) n_re += (aL ? 1 : 0) + (aR ? 1 : 0);
          if (aL) resolve(b, k, sd.theta, cL, tL, oL);
          if (aR) resolve(b, k, sd.theta, cR, tR, oR);
        }
        float i0, i1;
        mono2(dx, dy, dz, f2(B.z, B.w), eps2, tL, tR, tx, ty, tz, i0, i1);
        if (QUAD) {
          const float2 iq = f2(tL && !(cL & kLeafCode) ? i0 : 0.f, tR && !(cR & kLeafCode) ? i1 : 0.f);
          quad2(dx, dy, dz, iq, Q.uqa[p], Q.uqb[p], Q.uqc[p], tx, ty, tz);
        }
        if (STATS) {
          const uint32_t self = kLeafCode | k;
          n_leaf += (tL && (cL & kLeafCode) && cL != self ? 1 : 0) + (tR && (cR & kLeafCode) && cR != self ? 1 : 0);
          n_far += (tL && !(cL & kLeafCode) ? 1 : 0) + (tR && !(cR & kLeafCode) ? 1 : 0);
          n_open += (oL ? 1 : 0) + (oR ? 1 : 0);
        }
        const uint32_t m0 = (__ballot_sync(0xffffffffu, oL) >> (sl * G)) & gmask;
        const uint32_t m1 = (__ballot_sync(0xffffffffu, oR) >> (sl * G)) & gmask;
        if (tg == 0 && on) reinterpret_cast<uint2*>(L.uf + p)[1] = make_uint2(m0, m1);
      };
      // Evaluate the undecided list, then push every entry some target opened.
      auto flush_und = [&]() {
        if (ul & 1) {
          if (lane == 0) put_und(ul, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, kLeafCode, 0u);
          __syncwarp();
        }
        const int np = (ul + 1) >> 1;
        for (int q = 0; 2 * q * R < np; ++q) {
          const int pa = 2 * (q * R + sl), pb = pa + 1;
          und_pair(min(pa, np - 1), pa < np ? 1u : 0u);
          und_pair(min(pb, np - 1), pb < np ? 1u : 0u);
          fold();
        }
        __syncwarp();  // the opened masks are written
        for (int e0 = 0; e0 < ul; e0 += 32) {
          const int e = e0 + lane;
          uint32_t om = 0, code = 0;
          if (e < ul) {
            om = reinterpret_cast<const uint32_t*>(L.uf + (e >> 1))[2 + (e & 1)];
            code = reinterpret_cast<const uint32_t*>(L.ue + (e >> 1))[2 + (e & 1)];
          }
          const uint32_t bp = __ballot_sync(0xffffffffu, om != 0u);
          if (sp + __popc(bp) > kWalkStack) {
            bad = true;
          } else {
            if (om) L.stk[sp + __popc(bp & lt)] = make_uint2(code, om);
            sp += __popc(bp);
          }
        }
        ul = 0;
        __syncwarp();  // pushes visible to the next round; list read before it is refilled
      };
      for (;;) {
        if (__any_sync(0xffffffffu, bad)) break;
        if (sp == 0) {
          if (ul == 0) break;
          flush_und();
          continue;
        }
        const bool deep = sp > kWalkDeep;
        const int kk = deep ? 1 : min(32, sp);
        pairs_done += kk;
        if (pairs_done > max_pairs) {
          bad = true;
          break;
        }
        round(kk);
        if (dl >= kWalkFlush) flush_dense();
        if (ul >= kWalkFlush || (deep && ul > 0)) flush_und();
      }
      if (dl > 0 && !__any_sync(0xffffffffu, bad)) flush_dense();
      fold();
      __syncwarp();  // the next item's stack writes must not race this item's last reads
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) raise_err(b.ctl, kErrBadIndex);
    float ax = KAHAN ? __fsub_rn(sxy.x, cxy.x) : sxy.x;
    float ay = KAHAN ? __fsub_rn(sxy.y, cxy.y) : sxy.y;
    float az = KAHAN ? __fsub_rn(sz, cz) : sz;
    // the R lanes of a target hold partial sums over disjoint entries
    for (int o = G; o < 32; o <<= 1) {
      ax += __shfl_xor_sync(0xffffffffu, ax, o);
      ay += __shfl_xor_sync(0xffffffffu, ay, o);
      az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    if (valid && sl == 0) {
      const uint32_t o = b.order[k];
      b.acc[3 * (size_t)o + 0] = dmul(static_cast<double>(ax), sd.g);
      b.acc[3 * (size_t)o + 1] = dmul(static_cast<double>(ay), sd.g);
      b.acc[3 * (size_t)o + 2] = dmul(static_cast<double>(az), sd.g);
    }
    if (STATS) {
      n_leaf = warp_sum64(n_leaf);
      n_far = warp_sum64(n_far);
      n_open = warp_sum64(n_open);
      n_re = warp_sum64(n_re);
      const uint32_t n_valid = __popc(vmask);  // the root, opened by all
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
void launch_k(K kern, const StepBufs& b, const WalkCfg& cfg, size_t smem, cudaStream_t st) {
  const int block = cfg.block > 0 ? cfg.block : kWalkThreads;
  const int wpb = block / 32;
  if (cfg.persistent_ctas > 0) {
    kern<<<cfg.persistent_ctas, block, smem, st>>>(b, 1);
  } else {
    const uint32_t grid = (b.nitems + wpb - 1) / wpb;
    if (grid) kern<<<grid, block, smem, st>>>(b, 0);
  }
}

template <bool QUAD, bool KAHAN, bool LIST>
void dispatch_f32(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  const size_t smem = walk_smem_bytes(cfg.block > 0 ? cfg.block : kWalkThreads, QUAD);
  if (cfg.stats) {
    if (cfg.inside_test)
      launch_k(k_walk_f32<QUAD, KAHAN, true, true, LIST>, b, cfg, smem, st);
    else
      launch_k(k_walk_f32<QUAD, KAHAN, true, false, LIST>, b, cfg, smem, st);
  } else {
    if (cfg.inside_test)
      launch_k(k_walk_f32<QUAD, KAHAN, false, true, LIST>, b, cfg, smem, st);
    else
      launch_k(k_walk_f32<QUAD, KAHAN, false, false, LIST>, b, cfg, smem, st);
  }
}

template <bool LIST>
void dispatch(const StepBufs& b, const WalkCfg& cfg, cudaStream_t st) {
  if (cfg.precision == 1) {
    // The FP64 walk has no quadrupole or compensation variants: it is the
    // reference's arithmetic.
    if (cfg.stats)
      launch_k(k_walk_f64<true, LIST>, b, cfg, 0, st);
    else
      launch_k(k_walk_f64<false, LIST>, b, cfg, 0, st);
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

template <class K>
int resident(K kern, int block, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, block, smem) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

// Quadrupole blocks take more than the default 48 KB of dynamic shared memory. (No
// carveout preference is set: the driver sizes the L1 / shared split per launch, which
// leaves the L1 of the kernels that follow the walk in a step as large as they need.)
template <class K>
void smem_attrs(K kern, bool quad) {
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(walk_smem_bytes(kWalkThreads, quad)));
}

template <bool QUAD, bool KAHAN, bool LIST>
void smem_f32() {
  smem_attrs(k_walk_f32<QUAD, KAHAN, false, false, LIST>, QUAD);
  smem_attrs(k_walk_f32<QUAD, KAHAN, false, true, LIST>, QUAD);
  smem_attrs(k_walk_f32<QUAD, KAHAN, true, false, LIST>, QUAD);
  smem_attrs(k_walk_f32<QUAD, KAHAN, true, true, LIST>, QUAD);
}

}  // namespace

void walk_prepare() {
  smem_f32<false, false, false>();
  smem_f32<false, true, false>();
  smem_f32<true, false, false>();
  smem_f32<true, true, false>();
  smem_f32<false, false, true>();
  smem_f32<false, true, true>();
  smem_f32<true, false, true>();
  smem_f32<true, true, true>();
}

int walk_resident_ctas(const WalkCfg& cfg) {
  const int block = cfg.block > 0 ? cfg.block : kWalkThreads;
  if (cfg.precision == 1) return resident(k_walk_f64<false, false>, block, 0);
  if (cfg.quad) return resident(k_walk_f32<true, true, false, false, false>, block, walk_smem_bytes(block, true));
  return resident(k_walk_f32<false, true, false, false, false>, block, walk_smem_bytes(block, false));
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
