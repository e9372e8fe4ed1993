// gx_build.cu -- leaf gather + bottom-up Karras radix-tree build + FP64 aggregation
// in one kernel, one thread per leaf, no waiting.
//
// Reference: solvers/src/lbvh.rs:153-306 (delta, karras_node, reference_karras),
// :329-379 and :623-636 (reference_aggregate, fold_agg), :560-614 (the node
// geometry of reference_flatten: center, half extents, delta = |com - center|).
//
// The tree is the binary radix tree over the augmented keys (code, local sorted
// position); it is unique, so any correct construction yields reference_karras's
// topology. This kernel builds it bottom-up: a node covering sorted leaves [l, r]
// is the left child of its parent iff delta(r, r+1) > delta(l-1, l) (its parent
// splits at r), else the right child (parent splits at l-1). The two children of a
// split meet through one 64-bit atomic exchange on that split's slot: the first to
// arrive leaves (unified index, far end of its range) and exits, the second reads
// its sibling's aggregate and folds the parent -- so no thread ever waits.
// Karras numbering follows from the same rule: a left child covering [l, r] is
// internal node r, a right child is internal node l, the root is internal node 0.
// The fold is fold_agg's exact f64 sequence in fixed (left, right) order, so
// every aggregate is bit-identical to reference_aggregate's.
#include "gx_kernels.h"

namespace gx {

namespace {

struct AggR {
  double mn[3], mx[3], com[3], m;
};

__device__ __forceinline__ void fold(const AggR& la, const AggR& ra, AggR& o) {
  o.m = dadd(la.m, ra.m);
  if (o.m > 0.0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) o.com[c] = ddiv(dadd(dmul(la.com[c], la.m), dmul(ra.com[c], ra.m)), o.m);
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) o.com[c] = dmul(dadd(dadd(dadd(la.mn[c], la.mx[c]), ra.mn[c]), ra.mx[c]), 0.25);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    o.mn[c] = fmin(la.mn[c], ra.mn[c]);
    o.mx[c] = fmax(la.mx[c], ra.mx[c]);
  }
}

// Parallel-axis shift of a traceless quadrupole of mass m by d (child com - parent com).
__device__ __forceinline__ void quad_shift_add(const double q[6], double m, const double d[3], double out[6]) {
  const double d2 = dlen2(d[0], d[1], d[2]);
  out[0] = dadd(out[0], dadd(q[0], dmul(m, dsub(dmul(dmul(3.0, d[0]), d[0]), d2))));
  out[1] = dadd(out[1], dadd(q[1], dmul(m, dmul(dmul(3.0, d[0]), d[1]))));
  out[2] = dadd(out[2], dadd(q[2], dmul(m, dmul(dmul(3.0, d[0]), d[2]))));
  out[3] = dadd(out[3], dadd(q[3], dmul(m, dsub(dmul(dmul(3.0, d[1]), d[1]), d2))));
  out[4] = dadd(out[4], dadd(q[4], dmul(m, dmul(dmul(3.0, d[1]), d[2]))));
  out[5] = dadd(out[5], dadd(q[5], dmul(m, dsub(dmul(dmul(3.0, d[2]), d[2]), d2))));
}

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

// One child's half of its parent's sibling-pair walk record (FP32).
struct ChildRec {
  float hx, hy, hz, lx, ly, lz, m, take, open;
};

// A child as the FP32 walk record names it: an internal node by its index, a leaf by
// kLeafCode | leaf index (so the walk's next pair needs no offset arithmetic).
__device__ __forceinline__ uint32_t child_code(uint32_t u, uint32_t n_total) {
  return u >= n_total ? u - n_total : (kLeafCode | u);
}

// Geometry of an aggregate as reference_flatten derives it (solvers/src/lbvh.rs:602-613).
__device__ __forceinline__ void node_geometry(const AggR& a, double ctr[3], double hf[3], double& delta, double& s) {
  double dv[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ctr[c] = dmul(dadd(a.mn[c], a.mx[c]), 0.5);
    hf[c] = dmul(dsub(a.mx[c], a.mn[c]), 0.5);
    dv[c] = dsub(a.com[c], ctr[c]);
  }
  delta = dsqrt(dlen2(dv[0], dv[1], dv[2]));
  s = dmul(2.0, fmax(hf[0], fmax(hf[1], hf[2])));
}

// FP32 record of a child: float-float centre of mass, mass, and the d^2 thresholds.
// A leaf is always a term (take -1, open -2). An internal node is taken above
// rcrit^2 (1 + band) + tiny2 and opened below rcrit^2 (1 - band) - tiny2, rcrit =
// s/theta + delta; in between the walk re-decides in FP64. NaN thresholds (theta = 0,
// a zero-size or a massless node; a massless leaf) send every visit to the FP64 path,
// which applies the reference's rules exactly.
__device__ __forceinline__ ChildRec child_record(const AggR& a, bool leaf, double theta, double tiny2) {
  ChildRec r;
  split_ff(a.com[0], r.hx, r.lx);
  split_ff(a.com[1], r.hy, r.ly);
  split_ff(a.com[2], r.hz, r.lz);
  r.m = __double2float_rn(a.m);
  const float nan = __int_as_float(0x7fffffff);
  if (leaf) {
    r.take = a.m > 0.0 ? -1.f : nan;
    r.open = -2.f;
  } else {
    double ctr[3], hf[3], delta, s;
    node_geometry(a, ctr, hf, delta, s);
    r.take = r.open = nan;
    if (theta > 0.0 && s > 0.0 && a.m > 0.0) {
      const double rc = s / theta + delta;
      const double rc2 = rc * rc;
      r.take = __double2float_ru(rc2 * (1.0 + kOpenBand) + tiny2);
      r.open = __double2float_rd(rc2 * (1.0 - kOpenBand) - tiny2);
    }
  }
  return r;
}

}  // namespace

// Exchange with release (this thread's writes are visible before the new value) and
// acquire (the previous owner's writes are visible after it) at device scope.
__device__ __forceinline__ unsigned long long exch_acq_rel(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.exch.b64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}

template <bool QUAD, typename K>
__global__ void __launch_bounds__(kTileThreads) k_build(const TileDesc* __restrict__ tiles,
                                                        const SysDesc* __restrict__ sys, uint32_t n_total,
                                                        const K* __restrict__ codes,
                                                        const uint32_t* __restrict__ order,
                                                        const double* __restrict__ pos,
                                                        const double* __restrict__ mass, StepBufs b, int f64rec) {
  // One leaf per thread: block j covers leaves [256 (j % 16), 256 (j % 16) + 256) of
  // tile j / 16, so every leaf climbs concurrently (the loop below runs at most once).
  const TileDesc t = tiles[blockIdx.x / kItemsPerThread];
  const SysDesc sd = sys[t.sys];
  const uint32_t off = sd.off, ns = sd.n;
  const double theta = sd.theta;
  const double tiny2 = b.bounds[t.sys].tiny2;
  const uint32_t first = t.begin + (blockIdx.x % kItemsPerThread) * kTileThreads;
  for (uint32_t k = first + threadIdx.x; k < t.end && k < first + kTileThreads; k += kTileThreads) {
    // ---- leaf: gather the particle into sorted order ----
    const uint32_t o = order[k];
    if (o >= n_total) {
      raise_err(b.ctl, kErrBadIndex);
      continue;
    }
    AggR cur;
#pragma unroll
    for (int c = 0; c < 3; ++c) cur.com[c] = pos[3 * (size_t)o + c];
    cur.m = mass[o];
    b.leaf64[k] = make_double4(cur.com[0], cur.com[1], cur.com[2], cur.m);
    if (ns == 1) {
      b.parent[k] = kNoParent;
      continue;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) cur.mn[c] = cur.mx[c] = cur.com[c];
    double q[6] = {0, 0, 0, 0, 0, 0};
    uint32_t l = k - off, r = k - off;  // local leaf range of the current node
    uint32_t cur_u = k;                 // unified index of the current node
    uint32_t lc = 0, rc = 0;            // children of the current node (if internal)
    ChildRec pl, pr;                    // their halves of the node's walk record
    bool internal = false;
    for (int level = 0; level < kMaxDepth; ++level) {
      const bool root = (l == 0 && r == ns - 1);
      bool is_left = true;
      if (!root) {
        if (l == 0) {
          is_left = true;
        } else if (r == ns - 1) {
          is_left = false;
        } else {
          const int dr = prefix_len(codes[off + r], codes[off + r + 1], r, r + 1);
          const int dl = prefix_len(codes[off + l - 1], codes[off + l], l - 1, l);
          is_left = dr > dl;
        }
      }
      if (internal) {
        // Karras index of this node, now that its side is known.
        const uint32_t gi = off + (root ? 0u : (is_left ? r : l));
        const uint32_t u = n_total + gi;
        cur_u = u;
        b.kids[gi] = make_uint2(lc, rc);
        b.parent[lc] = u;
        b.parent[rc] = u;
        Agg64 a;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          a.mn[c] = cur.mn[c];
          a.mx[c] = cur.mx[c];
          a.com[c] = cur.com[c];
        }
        a.m = cur.m;
        b.agg64[gi] = a;
        double ctr[3], hf[3], delta, s;
        node_geometry(cur, ctr, hf, delta, s);
        float4* pp = b.pairs + 5 * (size_t)gi;
        pp[0] = make_float4(pl.hx, pr.hx, pl.hy, pr.hy);
        pp[1] = make_float4(pl.hz, pr.hz, pl.m, pr.m);
        pp[2] = make_float4(pl.lx, pr.lx, pl.ly, pr.ly);
        pp[3] = make_float4(pl.lz, pr.lz, pl.take, pr.take);
        pp[4] = make_float4(pl.open, pr.open, __uint_as_float(child_code(lc, n_total)),
                            __uint_as_float(child_code(rc, n_total)));
        if (theta >= 0.57) {
          // box centre and half extents: read only by the walk's inside test, which binds
          // only for theta >= 1/sqrt(3) (the walk applies it from 0.57 on)
          b.nodeC[gi] = make_float4(__double2float_rn(ctr[0]), __double2float_rn(ctr[1]), __double2float_rn(ctr[2]), 0.f);
          b.nodeD[gi] = make_float4(__double2float_rn(hf[0]), __double2float_rn(hf[1]), __double2float_rn(hf[2]), 0.f);
        }
        if (f64rec) {
          Node64 nd;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            nd.c[c] = ctr[c];
            nd.h[c] = hf[c];
            nd.com[c] = cur.com[c];
          }
          nd.m = cur.m;
          nd.delta = delta;
          nd.s = s;
          b.node64[gi] = nd;
        }
        if (QUAD) {
#pragma unroll
          for (int c = 0; c < 6; ++c) b.q64[6 * (size_t)gi + c] = q[c];
          b.nodeQ[2 * (size_t)gi] = make_float4(q[0], q[1], q[2], q[3]);
          b.nodeQ[2 * (size_t)gi + 1] = make_float4(q[4], q[5], 0.f, 0.f);
        }
        if (root) {
          b.parent[u] = kNoParent;
          break;
        }
      }
      // Meet the sibling at the parent's split.
      const uint32_t gamma = is_left ? r : l - 1;
      unsigned long long* slot = &b.slots[off + gamma];
      const unsigned long long mine = (static_cast<unsigned long long>(cur_u) << 32) | (is_left ? l : r);
      const unsigned long long old = exch_acq_rel(slot, mine);
      if (old == kEmptySlot) break;  // first to arrive: the sibling folds the parent
      const uint32_t sib_u = static_cast<uint32_t>(old >> 32);
      const uint32_t sib_far = static_cast<uint32_t>(old);
      if (!((sib_u >= off && sib_u < off + ns) || (sib_u >= n_total + off && sib_u < n_total + off + ns - 1)) ||
          sib_far >= ns) {
        raise_err(b.ctl, kErrClimb);
        break;
      }
      AggR sib;
      double sq[6] = {0, 0, 0, 0, 0, 0};
      if (sib_u < n_total) {
        const double* lp = reinterpret_cast<const double*>(&b.leaf64[sib_u]);
#pragma unroll
        for (int c = 0; c < 3; ++c) sib.com[c] = sib.mn[c] = sib.mx[c] = ldcg(lp + c);
        sib.m = ldcg(lp + 3);
      } else {
        const double* ap = reinterpret_cast<const double*>(&b.agg64[sib_u - n_total]);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          sib.mn[c] = ldcg(ap + c);
          sib.mx[c] = ldcg(ap + 3 + c);
          sib.com[c] = ldcg(ap + 6 + c);
        }
        sib.m = ldcg(ap + 9);
        if (QUAD) {
#pragma unroll
          for (int c = 0; c < 6; ++c) sq[c] = ldcg(b.q64 + 6 * (size_t)(sib_u - n_total) + c);
        }
      }
      AggR par;
      if (is_left) {
        fold(cur, sib, par);
        lc = cur_u;
        rc = sib_u;
        r = sib_far;
      } else {
        fold(sib, cur, par);
        lc = sib_u;
        rc = cur_u;
        l = sib_far;
      }
      {
        const AggR& CL = is_left ? cur : sib;
        const AggR& CR = is_left ? sib : cur;
        pl = child_record(CL, lc < n_total, theta, tiny2);
        pr = child_record(CR, rc < n_total, theta, tiny2);
      }
      if (QUAD) {
        // Q_parent = shift(Q_left) + shift(Q_right), left first (oracle order).
        const AggR& L = is_left ? cur : sib;
        const AggR& R = is_left ? sib : cur;
        const double* qL = is_left ? q : sq;
        const double* qR = is_left ? sq : q;
        double np[6] = {0, 0, 0, 0, 0, 0};
        double dl[3], dr[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          dl[c] = dsub(L.com[c], par.com[c]);
          dr[c] = dsub(R.com[c], par.com[c]);
        }
        double sl[6] = {0, 0, 0, 0, 0, 0}, sr[6] = {0, 0, 0, 0, 0, 0};
        quad_shift_add(qL, L.m, dl, sl);
        quad_shift_add(qR, R.m, dr, sr);
#pragma unroll
        for (int c = 0; c < 6; ++c) np[c] = dadd(sl[c], sr[c]);
#pragma unroll
        for (int c = 0; c < 6; ++c) q[c] = np[c];
      }
      cur = par;
      internal = true;
      if (level == kMaxDepth - 1) raise_err(b.ctl, kErrClimb);
    }
  }
}

void launch_build(const StepBufs& b, int quad, int f64_records, cudaStream_t st) {
  // Every split's rendezvous slot starts empty (one memset instead of a re-arming
  // atomic per fold, which the next level's release would have to wait for).
  cudaMemsetAsync(b.slots, 0xFF, static_cast<size_t>(b.n) * sizeof(unsigned long long), st);
  const uint64_t* c64 = reinterpret_cast<const uint64_t*>(b.codes);
  if (b.key64) {
    if (quad)
      k_build<true, uint64_t><<<b.ntiles * kItemsPerThread, kTileThreads, 0, st>>>(b.tiles, b.sys, b.n, c64, b.order, b.pos, b.mass, b,
                                                                  f64_records);
    else
      k_build<false, uint64_t><<<b.ntiles * kItemsPerThread, kTileThreads, 0, st>>>(b.tiles, b.sys, b.n, c64, b.order, b.pos, b.mass,
                                                                   b, f64_records);
  } else {
    if (quad)
      k_build<true, uint32_t><<<b.ntiles * kItemsPerThread, kTileThreads, 0, st>>>(b.tiles, b.sys, b.n, b.codes, b.order, b.pos, b.mass,
                                                                  b, f64_records);
    else
      k_build<false, uint32_t><<<b.ntiles * kItemsPerThread, kTileThreads, 0, st>>>(b.tiles, b.sys, b.n, b.codes, b.order, b.pos,
                                                                   b.mass, b, f64_records);
  }
}

}  // namespace gx
