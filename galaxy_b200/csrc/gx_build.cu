// gx_build.cu -- leaf gather + bottom-up Karras radix-tree build + FP64 aggregation
// in two passes, one thread per leaf; no thread spins on another's progress (pass 1's
// rounds meet at block barriers).
//
// Reference: solvers/src/lbvh.rs:153-306 (delta, karras_node, reference_karras),
// :329-379 and :623-636 (reference_aggregate, fold_agg), :560-614 (the node
// geometry of reference_flatten: center, half extents, delta = |com - center|).
//
// The tree is the binary radix tree over the augmented keys (code, local sorted
// position); it is unique, so any correct construction yields reference_karras's
// topology. It is built bottom-up: a node covering sorted leaves [l, r] is the left
// child of its parent iff delta(r, r+1) > delta(l-1, l) (its parent splits at r), else
// the right child (parent splits at l-1). The two children of a split meet through one
// atomic exchange on that split's word: the first to arrive leaves (its index, the far
// end of its range) and exits, the second reads its sibling's aggregate and folds the
// parent -- so no thread ever waits. Karras numbering follows from the same rule: a
// left child covering [l, r] is internal node r, a right child is internal node l, the
// root is internal node 0. The fold is fold_agg's exact f64 sequence in fixed (left,
// right) order, so every aggregate is bit-identical to reference_aggregate's.
//
// Pass 1 (k_build_local) does every split whose parent lies inside one block's
// kBuildLeaves (256) leaves with shared-memory exchange words and aggregates; pass 2 (k_build_top)
// continues the few climbs that leave a block through device-scope exchange words. A
// one-pass climb through global memory spends a device-scope round trip on every level
// and keeps a block resident until its highest climber reaches the top; here almost all
// levels stay on chip and pass 1's blocks retire as soon as their own subtrees are done.
#include "gx_kernels.h"

namespace gx {

namespace {

struct AggR {
  double mn[3], mx[3], com[3], m;
};

// fold_agg. Both forms of the centre of mass are computed and one is kept, so that the
// three axes and the caller's other work form one scheduling region (a branch would
// serialise them); the division by a zero mass gives an unused infinity or NaN.
__device__ __forceinline__ void fold(const AggR& la, const AggR& ra, AggR& o) {
  o.m = dadd(la.m, ra.m);
  const bool massive = o.m > 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double w = ddiv(dadd(dmul(la.com[c], la.m), dmul(ra.com[c], ra.m)), o.m);
    const double q = dmul(dadd(dadd(dadd(la.mn[c], la.mx[c]), ra.mn[c]), ra.mx[c]), 0.25);
    o.com[c] = massive ? w : q;
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
// s/theta + delta; in between the walk re-decides in FP64 with the reference's exact
// test. The thresholds only have to bracket that test, so rcrit is formed without FP64
// division or square root (long dependent sequences on the build's critical path):
// s/theta as s * (1/theta) and delta = |com - centre|^2 * rsqrt(|com - centre|^2),
// relative errors of a few 1e-16 that the 4e-6 band absorbs. Every case is computed
// and selected without branches, so the records of both children and the parent's
// fold interleave. NaN thresholds (theta = 0, a zero-size or a massless node; a
// massless leaf) send every visit to the FP64 path, which applies the reference's
// rules exactly.
__device__ __forceinline__ ChildRec child_record(const AggR& a, bool leaf, double theta, double inv_theta,
                                                 double tiny2) {
  ChildRec r;
  split_ff(a.com[0], r.hx, r.lx);
  split_ff(a.com[1], r.hy, r.ly);
  split_ff(a.com[2], r.hz, r.lz);
  r.m = __double2float_rn(a.m);
  const float nan = __int_as_float(0x7fffffff);
  double hf[3], dv[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    hf[c] = dmul(dsub(a.mx[c], a.mn[c]), 0.5);
    dv[c] = dsub(a.com[c], dmul(dadd(a.mn[c], a.mx[c]), 0.5));
  }
  const double dv2 = dlen2(dv[0], dv[1], dv[2]);
  const double delta = dv2 > 0.0 ? dv2 * rsqrt(dv2) : 0.0;
  const double s = dmul(2.0, fmax(hf[0], fmax(hf[1], hf[2])));
  const double rc = s * inv_theta + delta;
  const double rc2 = rc * rc;
  const float take = __double2float_ru(rc2 * (1.0 + kOpenBand) + tiny2);
  const float open = __double2float_rd(rc2 * (1.0 - kOpenBand) - tiny2);
  const bool ok = theta > 0.0 && s > 0.0 && a.m > 0.0;
  r.take = leaf ? (a.m > 0.0 ? -1.f : nan) : (ok ? take : nan);
  r.open = leaf ? -2.f : (ok ? open : nan);
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

namespace {

// What a climbing thread holds: the node it has just completed.
struct Climb {
  AggR cur;         // its aggregate
  double q[6];      // its traceless quadrupole (quadrupole mode)
  uint32_t l, r;    // its local leaf range
  uint32_t u;       // its unified index (leaf: sorted position; internal: n_total + Karras index)
  uint32_t lc, rc;  // its children (internal nodes)
  ChildRec pl, pr;  // the children's halves of its walk record
};

// The records of the internal node just completed, now that its Karras index gi (and so
// its unified index c.u) is known. write_agg: what a sibling's fold reads (the FP64
// aggregate and quadrupole); write_rest: what only later stages read (children, parent
// links of the children, the sibling-pair walk record, the optional box / FP64 /
// quadrupole walk data).
template <bool QUAD>
__device__ __forceinline__ void write_agg(const StepBufs& b, uint32_t gi, const Climb& c) {
  Agg64 a;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    a.mn[k] = c.cur.mn[k];
    a.mx[k] = c.cur.mx[k];
    a.com[k] = c.cur.com[k];
  }
  a.m = c.cur.m;
  b.agg64[gi] = a;
  if (QUAD) {
#pragma unroll
    for (int k = 0; k < 6; ++k) b.q64[6 * (size_t)gi + k] = c.q[k];
  }
}

template <bool QUAD>
__device__ __forceinline__ void write_rest(const StepBufs& b, uint32_t gi, const Climb& c, uint32_t n_total,
                                           double theta, int f64rec) {
  b.kids[gi] = make_uint2(c.lc, c.rc);
  b.parent[c.lc] = c.u;
  b.parent[c.rc] = c.u;
  float4* pp = b.pairs + 5 * (size_t)gi;
  pp[0] = make_float4(c.pl.hx, c.pr.hx, c.pl.hy, c.pr.hy);
  pp[1] = make_float4(c.pl.hz, c.pr.hz, c.pl.m, c.pr.m);
  pp[2] = make_float4(c.pl.lx, c.pr.lx, c.pl.ly, c.pr.ly);
  pp[3] = make_float4(c.pl.lz, c.pr.lz, c.pl.take, c.pr.take);
  pp[4] = make_float4(c.pl.open, c.pr.open, __uint_as_float(child_code(c.lc, n_total)),
                      __uint_as_float(child_code(c.rc, n_total)));
  if (theta >= 0.57 || f64rec) {
    double ctr[3], hf[3], delta, sz;
    node_geometry(c.cur, ctr, hf, delta, sz);
    if (theta >= 0.57) {
      // box centre and half extents: read only by the walk's inside test, which binds
      // only for theta >= 1/sqrt(3) (the walk applies it from 0.57 on)
      b.nodeC[gi] = make_float4(__double2float_rn(ctr[0]), __double2float_rn(ctr[1]), __double2float_rn(ctr[2]), 0.f);
      b.nodeD[gi] = make_float4(__double2float_rn(hf[0]), __double2float_rn(hf[1]), __double2float_rn(hf[2]), 0.f);
    }
    if (f64rec) {
      Node64 nd;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        nd.c[k] = ctr[k];
        nd.h[k] = hf[k];
        nd.com[k] = c.cur.com[k];
      }
      nd.m = c.cur.m;
      nd.delta = delta;
      nd.s = sz;
      b.node64[gi] = nd;
    }
  }
  if (QUAD) {
    b.nodeQ[2 * (size_t)gi] = make_float4(c.q[0], c.q[1], c.q[2], c.q[3]);
    b.nodeQ[2 * (size_t)gi + 1] = make_float4(c.q[4], c.q[5], 0.f, 0.f);
  }
}

// Fold the held node with its sibling into their parent (fold_agg's order: left, then
// right); the parent becomes the held node. LEFT: the held node is the left child. The
// side is a template argument so that every operand is named directly (a run-time
// choice between the two aggregates would take their addresses and move them to the
// local-memory stack).
template <bool QUAD, bool LEFT>
__device__ __forceinline__ void combine_side(Climb& c, const AggR& sib, const double sq[6], uint32_t sib_u,
                                             uint32_t sib_far, uint32_t n_total, double theta, double inv_theta,
                                             double tiny2) {
  const AggR& CL = LEFT ? c.cur : sib;
  const AggR& CR = LEFT ? sib : c.cur;
  AggR par;
  fold(CL, CR, par);
  if (LEFT) {
    c.lc = c.u;
    c.rc = sib_u;
    c.r = sib_far;
  } else {
    c.lc = sib_u;
    c.rc = c.u;
    c.l = sib_far;
  }
  c.pl = child_record(CL, c.lc < n_total, theta, inv_theta, tiny2);
  c.pr = child_record(CR, c.rc < n_total, theta, inv_theta, tiny2);
  if (QUAD) {
    // Q_parent = shift(Q_left) + shift(Q_right), left first (oracle order).
    const double* qL = LEFT ? c.q : sq;
    const double* qR = LEFT ? sq : c.q;
    double dl[3], dr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      dl[k] = dsub(CL.com[k], par.com[k]);
      dr[k] = dsub(CR.com[k], par.com[k]);
    }
    double sl[6] = {0, 0, 0, 0, 0, 0}, sr[6] = {0, 0, 0, 0, 0, 0};
    quad_shift_add(qL, CL.m, dl, sl);
    quad_shift_add(qR, CR.m, dr, sr);
#pragma unroll
    for (int k = 0; k < 6; ++k) c.q[k] = dadd(sl[k], sr[k]);
  }
  c.cur = par;
}

template <bool QUAD>
__device__ __forceinline__ void combine(Climb& c, const AggR& sib, const double sq[6], bool is_left, uint32_t sib_u,
                                        uint32_t sib_far, uint32_t n_total, double theta, double inv_theta,
                                        double tiny2) {
  if (is_left)
    combine_side<QUAD, true>(c, sib, sq, sib_u, sib_far, n_total, theta, inv_theta, tiny2);
  else
    combine_side<QUAD, false>(c, sib, sq, sib_u, sib_far, n_total, theta, inv_theta, tiny2);
}

constexpr int kDeltaMax = 0x7fffffff;  // "no pair": past the end of a block's leaves

}  // namespace

#ifndef GX_BUILD_LEAVES
#define GX_BUILD_LEAVES 256
#endif
// Leaves (and threads) of one pass-1 block: a power of two from 64 to 256.
constexpr int kBuildLeaves = GX_BUILD_LEAVES;
constexpr int kBuildBlocksPerTile = kTile / kBuildLeaves;
static_assert(kBuildLeaves >= 64 && kBuildLeaves <= 256 && (kBuildLeaves & (kBuildLeaves - 1)) == 0, "block size");

constexpr uint32_t kUnset = 0xFFFFFFFEu;  // staged parent / child slot not written by pass 1

// Shared memory of one pass-1 block (dynamic: above the 48 KB static limit). Every record
// of the block's internal nodes (Karras indices [first, first + m)) and the parent links
// of its nodes are staged here and written out coalesced when the block is done.
template <bool QUAD>
struct BuildSmem {
  double4 leaf[kBuildLeaves];        // the block's leaves (com, mass)
  AggR inr[kBuildLeaves];            // internal node gi at gi - first
  float4 pairs[5 * kBuildLeaves];    // its sibling-pair walk record
  double q[QUAD ? 6 * kBuildLeaves : 1];
  unsigned long long slot[kBuildLeaves];  // exchange word of split j at j - clo
  uint2 work[kBuildLeaves];          // folds of the round (block-local indices)
  uint2 kids[kBuildLeaves];          // its children; .x = kUnset: not a node of this block
  uint32_t par_leaf[kBuildLeaves];   // parent of leaf first + i (kUnset: pass 2 writes it)
  uint32_t par_int[kBuildLeaves];    // parent of internal node first + i
  int d[kBuildLeaves + 2];           // delta(clo - 1 + i, clo + i), i <= m; kDeltaMax past m
  int pre[kBuildLeaves + 1];         // pre[i] = min(d[0 .. i - 1])
  int suf[kBuildLeaves + 2];         // suf[i] = min(d[i .. kBuildLeaves + 1])
  int wpre[kBuildLeaves / 32], wsuf[kBuildLeaves / 32];
  uint32_t ntops;
};

// Pass 1, one block per run of up to kBuildLeaves sorted leaves of one system (the block's
// leaves [clo, chi), system-local). Each thread gathers its particle into sorted order;
// then the block climbs in rounds, as long as a node's parent lies inside the block's
// leaves: both children of such a parent are built by this block, so they meet through
// a shared-memory exchange word and the fold reads both aggregates from shared memory.
// Whether a parent is inside follows from the adjacent-pair prefix lengths
// delta(j, j + 1) of the block, loaded once: the parent of a left child [l, r] (split at
// r) ends at the first j > r with delta(j, j + 1) < delta(r, r + 1), the parent of a
// right child [l, r] (split at l - 1) starts after the last j < l - 1 with
// delta(j, j + 1) < delta(l - 1, l); a system edge counts as delta -1. Suffix and prefix
// minima of the deltas answer either question in one lookup. A node whose parent
// reaches past the block is a block top: it is listed for pass 2 in the block's own
// slice of the (then idle) sort buffers -- record j at keys_alt[first + j] (as uint2:
// unified index | left-child bit 31, far end of its range), the count at
// vals_alt[first] -- so no block contends for a global counter.
// A round: (A) every node completed in the last round (leaves in round 0) stages its
// records and meets its sibling; (B) the second arrivals, compacted into the first
// threads of the block, fold their parents. Half of the climbers leave at every level,
// so compacting them keeps the FP64 folds in full warps; staging the records keeps the
// rounds free of scattered global stores. No thread waits on another except at the
// block's barriers.
template <bool QUAD, typename K>
__global__ void __launch_bounds__(kBuildLeaves, (QUAD ? 2 : 3) * (256 / kBuildLeaves)) k_build_local(const TileDesc* __restrict__ tiles,
                                                              const SysDesc* __restrict__ sys, uint32_t n_total,
                                                              const K* __restrict__ codes,
                                                              const uint32_t* __restrict__ order,
                                                              const double* __restrict__ pos,
                                                              const double* __restrict__ mass, StepBufs b, int f64rec) {
  extern __shared__ __align__(16) unsigned char s_build_raw[];
  BuildSmem<QUAD>& S = *reinterpret_cast<BuildSmem<QUAD>*>(s_build_raw);
  // block j covers leaves [L (j % B), L (j % B) + L) of tile j / B (L = kBuildLeaves, B = kTile / L)
  const TileDesc t = tiles[blockIdx.x / kBuildBlocksPerTile];
  const uint32_t first = t.begin + (blockIdx.x % kBuildBlocksPerTile) * kBuildLeaves;
  if (first >= t.end) return;  // the whole block
  const SysDesc sd = sys[t.sys];
  const uint32_t off = sd.off, ns = sd.n;
  const double theta = sd.theta;
  const double inv_theta = 1.0 / theta;
  const double tiny2 = b.bounds[t.sys].tiny2;
  const uint32_t m = min(t.end - first, static_cast<uint32_t>(kBuildLeaves));
  const uint32_t clo = first - off, chi = clo + m;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint2* __restrict__ tops = reinterpret_cast<uint2*>(b.keys_alt) + first;
  if (tid == 0) S.ntops = 0;
  // the leaf's particle index first: its load overlaps the code loads below
  const uint32_t k = first + tid;
  const uint32_t o = tid < static_cast<int>(m) ? order[k] : 0u;

  for (int i = tid; i < kBuildLeaves + 2; i += kBuildLeaves) {
    int d = kDeltaMax;
    if (i <= static_cast<int>(m)) {
      const long long j = static_cast<long long>(clo) - 1 + i;
      d = (j < 0 || j + 1 >= ns) ? -1
                                 : prefix_len(codes[off + j], codes[off + j + 1], static_cast<uint32_t>(j),
                                              static_cast<uint32_t>(j) + 1);
    }
    S.d[i] = d;
  }
  S.slot[tid] = kEmptySlot;
  S.kids[tid] = make_uint2(kUnset, kUnset);
  S.par_leaf[tid] = kUnset;
  S.par_int[tid] = kUnset;
  // the particle's coordinates, in flight during the scans below
  const bool gathered = tid < static_cast<int>(m) && o < n_total;
  double px = 0.0, py = 0.0, pz = 0.0, pm = 0.0;
  if (gathered) {
    px = pos[3 * (size_t)o];
    py = pos[3 * (size_t)o + 1];
    pz = pos[3 * (size_t)o + 2];
    pm = mass[o];
  }
  __syncthreads();
  {
    // prefix and suffix minima of d[0 .. 255] (warp scans, then across the warps);
    // the two entries past them only enter the suffix minima
    const int v = S.d[tid];
    int p = v, q = v;
#pragma unroll
    for (int of = 1; of < 32; of <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, p, of);
      const int z = __shfl_down_sync(0xffffffffu, q, of);
      if (lane >= of) p = min(p, y);
      if (lane + of < 32) q = min(q, z);
    }
    if (lane == 31) S.wpre[warp] = p;
    if (lane == 0) S.wsuf[warp] = q;
    __syncthreads();
    int before = kDeltaMax, after = min(S.d[kBuildLeaves], S.d[kBuildLeaves + 1]);
    for (int w = 0; w < kBuildLeaves / 32; ++w) {
      if (w < warp) before = min(before, S.wpre[w]);
      if (w > warp) after = min(after, S.wsuf[w]);
    }
    S.pre[tid + 1] = min(before, p);
    S.suf[tid] = min(after, q);
    if (tid == 0) {
      S.pre[0] = kDeltaMax;
      S.suf[kBuildLeaves] = min(S.d[kBuildLeaves], S.d[kBuildLeaves + 1]);
      S.suf[kBuildLeaves + 1] = S.d[kBuildLeaves + 1];
    }
  }
  // leaf: the particle in sorted order; it is the thread's first held node
  bool held = false;
  Climb c;
  if (tid < static_cast<int>(m)) {
    if (!gathered) {
      raise_err(b.ctl, kErrBadIndex);
    } else {
      c.cur.com[0] = c.cur.mn[0] = c.cur.mx[0] = px;
      c.cur.com[1] = c.cur.mn[1] = c.cur.mx[1] = py;
      c.cur.com[2] = c.cur.mn[2] = c.cur.mx[2] = pz;
      c.cur.m = pm;
      const double4 lf = make_double4(px, py, pz, pm);
      b.leaf64[k] = lf;
      S.leaf[tid] = lf;
      if (ns == 1) {
        S.par_leaf[tid] = kNoParent;
      } else {
        held = true;
#pragma unroll
        for (int a = 0; a < 6; ++a) c.q[a] = 0.0;
        c.l = c.r = k - off;
        c.u = k;
        c.lc = c.rc = 0;
      }
    }
  }
  __syncthreads();  // minima and leaves are in place
  bool internal = false;
  for (int round = 0;; ++round) {
    // (A) the held node: its records, then its sibling
    bool fold = false;
    uint2 item = make_uint2(0u, 0u);
    if (held && round > kBuildLeaves) {
      raise_err(b.ctl, kErrClimb);  // more levels than leaves: not a radix tree
      held = false;
    }
    if (held) {
      held = false;
      // Inside the block both ends' deltas are d entries (delta(l - 1, l) = d[l - clo],
      // delta(r, r + 1) = d[r - clo + 1]); -1 marks a system edge.
      const int d_lo = S.d[c.l - clo], d_hi = S.d[c.r - clo + 1];
      const bool root = d_lo < 0 && d_hi < 0;
      const bool is_left = root || d_hi > d_lo;
      bool go = true;
      if (internal) {
        const uint32_t gi = off + (root ? 0u : (is_left ? c.r : c.l));
        const uint32_t li = gi - first;  // inside the block: first <= gi < first + m
        c.u = n_total + gi;
        S.kids[li] = make_uint2(c.lc, c.rc);
        if (c.lc < n_total)
          S.par_leaf[c.lc - first] = c.u;
        else
          S.par_int[c.lc - n_total - first] = c.u;
        if (c.rc < n_total)
          S.par_leaf[c.rc - first] = c.u;
        else
          S.par_int[c.rc - n_total - first] = c.u;
        S.inr[li] = c.cur;
        if (QUAD) {
#pragma unroll
          for (int a = 0; a < 6; ++a) S.q[6 * li + a] = c.q[a];
        }
        float4* pp = S.pairs + 5 * li;
        pp[0] = make_float4(c.pl.hx, c.pr.hx, c.pl.hy, c.pr.hy);
        pp[1] = make_float4(c.pl.hz, c.pr.hz, c.pl.m, c.pr.m);
        pp[2] = make_float4(c.pl.lx, c.pr.lx, c.pl.ly, c.pr.ly);
        pp[3] = make_float4(c.pl.lz, c.pr.lz, c.pl.take, c.pr.take);
        pp[4] = make_float4(c.pl.open, c.pr.open, __uint_as_float(child_code(c.lc, n_total)),
                            __uint_as_float(child_code(c.rc, n_total)));
        if (root) {
          S.par_int[li] = kNoParent;
          go = false;
        }
      }
      if (go) {
        const bool parent_inside = is_left ? S.suf[c.r - clo + 2] < d_hi : S.pre[c.l - clo] < d_lo;
        if (!parent_inside) {
          // a block top (at most one per leaf of the block): pass 2 continues its climb
          const uint32_t j = atomicAdd(&S.ntops, 1u);
          if (j < m)
            tops[j] = make_uint2(c.u | (is_left ? 0x80000000u : 0u), is_left ? c.l : c.r);
          else
            raise_err(b.ctl, kErrClimb);
        } else {
          // Meet the sibling at the parent's split (inside the block: clo <= gamma < chi - 1);
          // the first to arrive is done, the second folds the parent in (B).
          const uint32_t gamma = is_left ? c.r : c.l - 1;
          const unsigned long long mine = (static_cast<unsigned long long>(c.u) << 32) | (is_left ? c.l : c.r);
          const unsigned long long old = atomicExch(&S.slot[gamma - clo], mine);
          if (old != kEmptySlot) {
            // the fold as block-local indices: x = (node, leaf?, l, r, left?), y = (sibling,
            // leaf?, its far end)
            const uint32_t sib_u = static_cast<uint32_t>(old >> 32), sib_far = static_cast<uint32_t>(old);
            const bool sib_leaf = sib_u < n_total;
            const uint32_t si = sib_leaf ? sib_u - first : sib_u - n_total - first;  // wraps when outside
            if (si >= m || sib_far < clo || sib_far >= chi) {
              raise_err(b.ctl, kErrClimb);
            } else {
              fold = true;
              const uint32_t xi = internal ? c.u - n_total - first : c.u - first;
              item.x = xi | (internal ? 0u : 256u) | ((c.l - clo) << 9) | ((c.r - clo) << 17) | (is_left ? 1u << 25 : 0u);
              item.y = si | (sib_leaf ? 256u : 0u) | ((sib_far - clo) << 9);
            }
          }
        }
      }
    }
    // compact the folds into the first threads of the block
    const uint32_t fb = __ballot_sync(0xffffffffu, fold);
    if (lane == 0) S.wpre[warp] = __popc(fb);
    __syncthreads();  // exchanges, staged records and the warp counts are in place
    const int cnt = lane < kBuildLeaves / 32 ? S.wpre[lane] : 0;
    const int total = __reduce_add_sync(0xffffffffu, cnt);
    const int base = __reduce_add_sync(0xffffffffu, lane < warp ? cnt : 0);
    if (fold) S.work[base + __popc(fb & ((1u << lane) - 1u))] = item;
    __syncthreads();  // the round's folds are listed (and every thread has read the counts)
    if (total == 0) break;
    // (B) fold item tid: the node that arrived second and its sibling, both from shared memory
    if (tid < total) {
      const uint2 w = S.work[tid];
      const uint32_t xi = w.x & 255u, si = w.y & 255u;
      const bool x_leaf = (w.x & 256u) != 0, sib_leaf = (w.y & 256u) != 0;
      const bool is_left = ((w.x >> 25) & 1u) != 0;
      c.l = clo + ((w.x >> 9) & 255u);
      c.r = clo + ((w.x >> 17) & 255u);
      c.u = x_leaf ? first + xi : n_total + first + xi;
      const uint32_t sib_u = sib_leaf ? first + si : n_total + first + si;
      const uint32_t sib_far = clo + ((w.y >> 9) & 255u);
      AggR sib;
      double sq[6] = {0, 0, 0, 0, 0, 0};
      if (x_leaf) {
        const double4 lf = S.leaf[xi];
        c.cur.com[0] = c.cur.mn[0] = c.cur.mx[0] = lf.x;
        c.cur.com[1] = c.cur.mn[1] = c.cur.mx[1] = lf.y;
        c.cur.com[2] = c.cur.mn[2] = c.cur.mx[2] = lf.z;
        c.cur.m = lf.w;
#pragma unroll
        for (int a = 0; a < 6; ++a) c.q[a] = 0.0;
      } else {
        c.cur = S.inr[xi];
        if (QUAD) {
#pragma unroll
          for (int a = 0; a < 6; ++a) c.q[a] = S.q[6 * xi + a];
        }
      }
      if (sib_leaf) {
        const double4 lf = S.leaf[si];
        sib.com[0] = sib.mn[0] = sib.mx[0] = lf.x;
        sib.com[1] = sib.mn[1] = sib.mx[1] = lf.y;
        sib.com[2] = sib.mn[2] = sib.mx[2] = lf.z;
        sib.m = lf.w;
      } else {
        sib = S.inr[si];
        if (QUAD) {
#pragma unroll
          for (int a = 0; a < 6; ++a) sq[a] = S.q[6 * si + a];
        }
      }
      combine<QUAD>(c, sib, sq, is_left, sib_u, sib_far, n_total, theta, inv_theta, tiny2);
      held = true;
    }
    internal = true;
  }
  // Write-out (the last round's barrier made every staged record visible): consecutive
  // threads write consecutive words; slots of nodes that pass 2 builds are skipped.
  if (tid == 0) b.vals_alt[first] = min(S.ntops, m);
  for (int i = tid; i < static_cast<int>(m); i += kBuildLeaves) {
    if (S.par_leaf[i] != kUnset) b.parent[first + i] = S.par_leaf[i];
    if (S.par_int[i] != kUnset) b.parent[n_total + first + i] = S.par_int[i];
    if (S.kids[i].x == kUnset) continue;
    const uint32_t gi = first + i;
    b.kids[gi] = S.kids[i];
    if (theta >= 0.57 || f64rec) {
      double ctr[3], hf[3], delta, sz;
      node_geometry(S.inr[i], ctr, hf, delta, sz);
      if (theta >= 0.57) {
        // box centre and half extents: read only by the walk's inside test, which binds
        // only for theta >= 1/sqrt(3) (the walk applies it from 0.57 on)
        b.nodeC[gi] = make_float4(__double2float_rn(ctr[0]), __double2float_rn(ctr[1]), __double2float_rn(ctr[2]), 0.f);
        b.nodeD[gi] = make_float4(__double2float_rn(hf[0]), __double2float_rn(hf[1]), __double2float_rn(hf[2]), 0.f);
      }
      if (f64rec) {
        Node64 nd;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          nd.c[a] = ctr[a];
          nd.h[a] = hf[a];
          nd.com[a] = S.inr[i].com[a];
        }
        nd.m = S.inr[i].m;
        nd.delta = delta;
        nd.s = sz;
        b.node64[gi] = nd;
      }
    }
  }
  {
    // the aggregates (10 doubles a node) and walk records (5 float4 a node), flat
    const double* src = reinterpret_cast<const double*>(S.inr);
    double* dst = reinterpret_cast<double*>(b.agg64 + first);
    for (int j = tid; j < 10 * static_cast<int>(m); j += kBuildLeaves)
      if (S.kids[j / 10].x != kUnset) dst[j] = src[j];
    float4* pdst = b.pairs + 5 * (size_t)first;
    for (int j = tid; j < 5 * static_cast<int>(m); j += kBuildLeaves)
      if (S.kids[j / 5].x != kUnset) pdst[j] = S.pairs[j];
    if (QUAD) {
      double* qdst = b.q64 + 6 * (size_t)first;
      for (int j = tid; j < 6 * static_cast<int>(m); j += kBuildLeaves)
        if (S.kids[j / 6].x != kUnset) qdst[j] = S.q[j];
      for (int j = tid; j < 2 * static_cast<int>(m); j += kBuildLeaves) {
        const int i = j >> 1;
        if (S.kids[i].x == kUnset) continue;
        const double* qq = S.q + 6 * i;
        b.nodeQ[2 * (size_t)first + j] =
            (j & 1) ? make_float4(qq[4], qq[5], 0.f, 0.f) : make_float4(qq[0], qq[1], qq[2], qq[3]);
      }
    }
  }
}

// Pass 2: the climbs of the block tops, one warp per block of pass 1 (its lanes take the
// block's tops), through device-scope exchange words in global memory: the two children
// of a split meet
// through one 64-bit atomic exchange on that split's slot; the first to arrive leaves
// (unified index, far end of its range) and exits, the second reads its sibling's
// aggregate from global memory and folds the parent -- so no thread ever waits. Every
// node above the block tops spans two blocks, so only these few climbs (a few per block)
// take device-scope round trips, and none of them holds a block of pass 1 resident.
template <bool QUAD, typename K>
__global__ void __launch_bounds__(kTileThreads) k_build_top(const TileDesc* __restrict__ tiles,
                                                            const SysDesc* __restrict__ sys, uint32_t n_total,
                                                            const K* __restrict__ codes, StepBufs b, int f64rec) {
  const uint32_t blk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // pass-1 block of this warp
  if (blk >= b.ntiles * kBuildBlocksPerTile) return;
  const TileDesc t = tiles[blk / kBuildBlocksPerTile];
  const uint32_t first = t.begin + (blk % kBuildBlocksPerTile) * kBuildLeaves;
  if (first >= t.end) return;
  const uint32_t count = min(b.vals_alt[first], static_cast<uint32_t>(kBuildLeaves));
  const uint2* __restrict__ tops = reinterpret_cast<const uint2*>(b.keys_alt) + first;
  const uint32_t si = t.sys;
  for (uint32_t i = threadIdx.x & 31; i < count; i += 32) {
    const uint2 rec = tops[i];
    const SysDesc sd = sys[si];
    const uint32_t off = sd.off, ns = sd.n;
    const double theta = sd.theta;
    const double inv_theta = 1.0 / theta;
    const double tiny2 = b.bounds[si].tiny2;
    Climb c;
    c.u = rec.x & 0x7fffffffu;
    bool is_left = (rec.x >> 31) != 0;
    const uint32_t far = rec.y;
    const bool leaf = c.u < n_total;
    const uint32_t loc = leaf ? c.u - off : c.u - n_total - off;  // wraps when outside
    if (loc >= ns || far >= ns || ns < 2) {
      raise_err(b.ctl, kErrClimb);
      continue;
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) c.q[a] = 0.0;
    if (leaf) {
      const double4 lf = b.leaf64[c.u];
      c.cur.com[0] = c.cur.mn[0] = c.cur.mx[0] = lf.x;
      c.cur.com[1] = c.cur.mn[1] = c.cur.mx[1] = lf.y;
      c.cur.com[2] = c.cur.mn[2] = c.cur.mx[2] = lf.z;
      c.cur.m = lf.w;
      c.l = c.r = loc;
    } else {
      const Agg64 a = b.agg64[c.u - n_total];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        c.cur.mn[k] = a.mn[k];
        c.cur.mx[k] = a.mx[k];
        c.cur.com[k] = a.com[k];
      }
      c.cur.m = a.m;
      if (QUAD) {
#pragma unroll
        for (int k = 0; k < 6; ++k) c.q[k] = b.q64[6 * (size_t)(c.u - n_total) + k];
      }
      // a left child is Karras node r, a right child Karras node l
      c.l = is_left ? far : loc;
      c.r = is_left ? loc : far;
    }
    if (c.l > c.r || (is_left ? c.r >= ns - 1 : c.l == 0)) {  // a top always has a parent split
      raise_err(b.ctl, kErrClimb);
      continue;
    }
    c.lc = c.rc = 0;
    uint32_t gi = 0;
    for (int level = 0; level < kMaxDepth; ++level) {
      // Meet the sibling at the parent's split. The release covers the aggregate of the
      // node (what the sibling reads); its other records are written after it.
      const uint32_t gamma = is_left ? c.r : c.l - 1;
      const unsigned long long mine = (static_cast<unsigned long long>(c.u) << 32) | (is_left ? c.l : c.r);
      const unsigned long long old = exch_acq_rel(&b.slots[off + gamma], mine);
      if (level > 0) write_rest<QUAD>(b, gi, c, n_total, theta, f64rec);
      if (old == kEmptySlot) break;  // first to arrive: the sibling folds the parent
      const uint32_t sib_u = static_cast<uint32_t>(old >> 32);
      const uint32_t sib_far = static_cast<uint32_t>(old);
      if (!((sib_u >= off && sib_u < off + ns) || (sib_u >= n_total + off && sib_u < n_total + off + ns - 1)) ||
          sib_far >= ns) {
        raise_err(b.ctl, kErrClimb);
        break;
      }
      // The parent's range and the four codes that decide its side, loaded together with
      // the sibling's aggregate (indices clamped into the system; unused at its edges).
      const uint32_t nl = is_left ? c.l : sib_far, nr = is_left ? sib_far : c.r;
      const bool proot = nl == 0 && nr == ns - 1;
      const K cl0 = codes[off + (nl > 0 ? nl - 1 : 0)], cl1 = codes[off + nl];
      const K cr0 = codes[off + nr], cr1 = codes[off + (nr + 1 < ns ? nr + 1 : nr)];
      AggR sib;
      double sq[6] = {0, 0, 0, 0, 0, 0};
      if (sib_u < n_total) {
        const double* lp = reinterpret_cast<const double*>(&b.leaf64[sib_u]);
#pragma unroll
        for (int k = 0; k < 3; ++k) sib.com[k] = sib.mn[k] = sib.mx[k] = ldcg(lp + k);
        sib.m = ldcg(lp + 3);
      } else {
        const double* ap = reinterpret_cast<const double*>(&b.agg64[sib_u - n_total]);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          sib.mn[k] = ldcg(ap + k);
          sib.mx[k] = ldcg(ap + 3 + k);
          sib.com[k] = ldcg(ap + 6 + k);
        }
        sib.m = ldcg(ap + 9);
        if (QUAD) {
#pragma unroll
          for (int k = 0; k < 6; ++k) sq[k] = ldcg(b.q64 + 6 * (size_t)(sib_u - n_total) + k);
        }
      }
      combine<QUAD>(c, sib, sq, is_left, sib_u, sib_far, n_total, theta, inv_theta, tiny2);
      // the parent's side (Karras: it is a left child iff delta(r, r + 1) > delta(l - 1, l), a
      // left child at the system's start, a right child at its end) and Karras index; its
      // aggregate for its sibling
      const int dr = prefix_len(cr0, cr1, nr, nr + 1), dl = prefix_len(cl0, cl1, nl - 1, nl);
      is_left = proot || nl == 0 || (nr != ns - 1 && dr > dl);
      gi = off + (proot ? 0u : (is_left ? c.r : c.l));
      c.u = n_total + gi;
      write_agg<QUAD>(b, gi, c);
      if (proot) {
        write_rest<QUAD>(b, gi, c, n_total, theta, f64rec);
        b.parent[c.u] = kNoParent;
        break;
      }
      if (level == kMaxDepth - 1) raise_err(b.ctl, kErrClimb);
    }
  }
}

namespace {

template <bool QUAD, typename K>
void launch_build_t(const StepBufs& b, const K* codes, int f64_records, cudaStream_t st) {
  const uint32_t blocks1 = b.ntiles * kBuildBlocksPerTile;
  k_build_local<QUAD, K><<<blocks1, kBuildLeaves, sizeof(BuildSmem<QUAD>), st>>>(b.tiles, b.sys, b.n, codes, b.order,
                                                                                 b.pos, b.mass, b, f64_records);
  // one warp per block of pass 1 (its tops: a few each)
  const uint32_t blocks2 = (blocks1 * 32 + kTileThreads - 1) / kTileThreads;
  k_build_top<QUAD, K><<<blocks2, kTileThreads, 0, st>>>(b.tiles, b.sys, b.n, codes, b, f64_records);
}

}  // namespace

void build_prepare() {
  // the shared memory of every resident block: the largest carveout
  auto set = [](auto kern, size_t bytes) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  };
  set(k_build_local<false, uint32_t>, sizeof(BuildSmem<false>));
  set(k_build_local<true, uint32_t>, sizeof(BuildSmem<true>));
  set(k_build_local<false, uint64_t>, sizeof(BuildSmem<false>));
  set(k_build_local<true, uint64_t>, sizeof(BuildSmem<true>));
}

void launch_build(const StepBufs& b, int quad, int f64_records, cudaStream_t st) {
  // Every split's global rendezvous slot starts empty (one memset instead of a re-arming
  // atomic per fold, which the next level's release would have to wait for).
  cudaMemsetAsync(b.slots, 0xFF, static_cast<size_t>(b.n) * sizeof(unsigned long long), st);
  const uint64_t* c64 = reinterpret_cast<const uint64_t*>(b.codes);
  if (b.key64) {
    if (quad)
      launch_build_t<true>(b, c64, f64_records, st);
    else
      launch_build_t<false>(b, c64, f64_records, st);
  } else {
    if (quad)
      launch_build_t<true>(b, static_cast<const uint32_t*>(b.codes), f64_records, st);
    else
      launch_build_t<false>(b, static_cast<const uint32_t*>(b.codes), f64_records, st);
  }
}

}  // namespace gx
