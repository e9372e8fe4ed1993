// lbvh_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A CPU f64 restatement of the galaxy reference's LBVH Barnes-Hut gravity path,
// written from the reference's Rust sources (paths relative to the reference
// project root):
//   solvers/src/lbvh.rs        Morton, sort, Karras, aggregate, flatten, walk
//   solvers/src/direct_sum.rs  O(N^2) softened direct sum (Newton-3 pairing)
//   solvers/src/potential.rs   O(N^2) softened potential
//   core/src/integrator.rs     LeapfrogKdk::step
//   core/src/diagnostics.rs    kinetic energy, momentum, angular momentum
// and the deterministic fixture generators of the reference tests
// (solvers/tests/lbvh.rs, gpu/tests/lbvh_sort.rs, gpu/tests/lbvh_tree.rs).
//
// Only the test-suite, the smoke check and bench.py's CPU-baseline leg may load
// this library; the product (libgalaxy_b200.so) never links or calls it.
//
// Arithmetic convention: glam's DVec3 operations are per-component IEEE f64 with
// no fused multiply-add (Rust never contracts), `length()` is
// sqrt((x*x + y*y) + z*z), `DVec3 / f64` divides each component. The file is
// compiled with -ffp-contract=off so every expression below rounds exactly as the
// Rust source does.
//
// Pinning: the Morton bit-spreading is pinned by the reference's known-answer
// tests (solvers/src/lbvh.rs:691-726, restated in tests/golden/). The rest is
// pinned by the reference's invariant tests (theta->0 equals direct summation to
// 1e-9, finite-theta error bounds, momentum flux, Karras structure, coincident
// determinism, empty/single), restated in tests/test_oracle.py. The reference is
// Rust and no Rust toolchain exists on this machine, so bitwise identity with the
// Rust binary itself is unpinned beyond those tests.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 {
  double x, y, z;
};
inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return V3{a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return V3{a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double length_squared(V3 a) { return dot(a, a); }
inline double length(V3 a) { return std::sqrt(dot(a, a)); }
// f64::min / f64::max: NaN-ignoring, like C fmin/fmax.
inline V3 vmin(V3 a, V3 b) { return V3{std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return V3{std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
inline double max_element(V3 a) { return std::fmax(a.x, std::fmax(a.y, a.z)); }
inline V3 load3(const double* p, size_t i) { return V3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline void store3(double* p, size_t i, V3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}

constexpr uint32_t MORTON_BITS = 10;     // solvers/src/lbvh.rs:32
constexpr uint32_t NO_PARENT = 0xFFFFFFFFu;  // solvers/src/lbvh.rs:244

// solvers/src/lbvh.rs:37-44
uint32_t expand10(uint32_t v) {
  uint32_t x = v & 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

// solvers/src/lbvh.rs:48-50
uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return expand10(x) | (expand10(y) << 1) | (expand10(z) << 2);
}

// Rust `(v.floor().max(0.0) as u32).min(cells - 1)`: f64::max maps NaN to 0.0 and
// the float->u32 cast saturates.  solvers/src/lbvh.rs:56-64
uint32_t quantize_lane(double v) {
  double f = std::fmax(std::floor(v), 0.0);
  uint32_t q = f >= 4294967295.0 ? 0xFFFFFFFFu : static_cast<uint32_t>(f);
  const uint32_t cells = 1u << MORTON_BITS;
  return std::min(q, cells - 1);
}

struct Bounds {
  V3 bmin;
  double size, scale;
};

// solvers/src/lbvh.rs:105-129 (bbox + pad + quantize convention)
Bounds morton_bounds(const double* pos, size_t n) {
  V3 lo = load3(pos, 0), hi = lo;
  for (size_t i = 0; i < n; ++i) {
    V3 p = load3(pos, i);
    lo = vmin(lo, p);
    hi = vmax(hi, p);
  }
  V3 center = (lo + hi) * 0.5;
  double half = std::fmax(0.5 * max_element(hi - lo), 1e-12) * (1.0 + 1e-9);
  Bounds b;
  b.bmin = center - V3{half, half, half};
  b.size = 2.0 * half;
  b.scale = static_cast<double>(1u << MORTON_BITS) / b.size;
  return b;
}

// solvers/src/lbvh.rs:153-165 -- augmented-key common prefix, -1 out of range.
inline int64_t delta(const uint32_t* codes, int64_t n, int64_t a, int64_t b) {
  if (b < 0 || b >= n) return -1;
  uint32_t ca = codes[a], cb = codes[b];
  if (ca == cb) {
    uint32_t x = static_cast<uint32_t>(a) ^ static_cast<uint32_t>(b);
    return 32 + (x == 0 ? 32 : __builtin_clz(x));
  }
  return __builtin_clz(ca ^ cb);
}

// The same prefix over 63-bit codes (extension with no reference counterpart: the
// 21-bit-per-axis keys the reference defers, solvers/src/lbvh.rs:29-32).
inline int64_t delta(const uint64_t* codes, int64_t n, int64_t a, int64_t b) {
  if (b < 0 || b >= n) return -1;
  uint64_t ca = codes[a], cb = codes[b];
  if (ca == cb) {
    uint32_t x = static_cast<uint32_t>(a) ^ static_cast<uint32_t>(b);
    return 64 + (x == 0 ? 32 : __builtin_clz(x));
  }
  return __builtin_clzll(ca ^ cb);
}

struct ChildRef {
  bool leaf;
  int64_t idx;
};

// solvers/src/lbvh.rs:195-240 -- Karras 2012 determineRange + findSplit with
// signed indices.
template <typename K>
void karras_node(const K* codes, int64_t n, int64_t i, ChildRef* left, ChildRef* right) {
  auto d0 = [&](int64_t a, int64_t b) { return delta(codes, n, a, b); };
  int64_t dir = d0(i, i + 1) > d0(i, i - 1) ? 1 : -1;
  int64_t delta_min = d0(i, i - dir);
  int64_t l_max = 2;
  while (d0(i, i + l_max * dir) > delta_min) l_max *= 2;
  int64_t l = 0;
  for (int64_t t = l_max / 2; t > 0; t /= 2)
    if (d0(i, i + (l + t) * dir) > delta_min) l += t;
  int64_t j = i + l * dir;
  int64_t delta_node = d0(i, j);
  int64_t s = 0;
  int64_t t = l;
  for (;;) {
    t = (t + 1) / 2;
    if (d0(i, i + (s + t) * dir) > delta_node) s += t;
    if (t <= 1) break;
  }
  int64_t gamma = i + s * dir + std::min<int64_t>(dir, 0);
  int64_t lo = std::min(i, j), hi = std::max(i, j);
  left->leaf = (lo == gamma);
  left->idx = gamma;
  right->leaf = (hi == gamma + 1);
  right->idx = gamma + 1;
}

struct Agg {
  double mass;
  V3 com, mn, mx;
};

// solvers/src/lbvh.rs:623-636 -- fixed (left, right) fold.
Agg fold_agg(const Agg& la, const Agg& ra) {
  Agg a;
  a.mass = la.mass + ra.mass;
  if (a.mass > 0.0)
    a.com = (la.com * la.mass + ra.com * ra.mass) / a.mass;
  else
    a.com = (la.mn + la.mx + ra.mn + ra.mx) * 0.25;
  a.mn = vmin(la.mn, ra.mn);
  a.mx = vmax(la.mx, ra.mx);
  return a;
}

struct Tree {
  size_t n;
  std::vector<uint32_t> left, right, parent;
};

// solvers/src/lbvh.rs:276-306
template <typename K>
Tree reference_karras(const K* sorted_codes, size_t n) {
  Tree t;
  t.n = n;
  t.left.assign(n - 1, 0);
  t.right.assign(n - 1, 0);
  t.parent.assign(2 * n - 1, NO_PARENT);
  auto unify = [&](ChildRef c) -> uint32_t {
    return c.leaf ? static_cast<uint32_t>(c.idx) : static_cast<uint32_t>(n + c.idx);
  };
  for (size_t i = 0; i + 1 < n; ++i) {
    ChildRef l, r;
    karras_node(sorted_codes, static_cast<int64_t>(n), static_cast<int64_t>(i), &l, &r);
    uint32_t lu = unify(l), ru = unify(r), me = static_cast<uint32_t>(n + i);
    t.left[i] = lu;
    t.right[i] = ru;
    t.parent[lu] = me;
    t.parent[ru] = me;
  }
  return t;
}

struct AggOut {
  std::vector<V3> mn, mx, com;
  std::vector<double> mass;
};

// solvers/src/lbvh.rs:352-379 (recursion depth <= tree depth <= 63 for 30-bit
// codes with a 32-bit position tie-break, so plain recursion is safe).
Agg agg_node(uint32_t u, const Tree& t, const std::vector<V3>& sp, const double* sm, AggOut& out) {
  Agg a;
  if (u < t.n) {
    a.mass = sm[u];
    a.com = a.mn = a.mx = sp[u];
  } else {
    size_t i = u - t.n;
    Agg la = agg_node(t.left[i], t, sp, sm, out);
    Agg ra = agg_node(t.right[i], t, sp, sm, out);
    a = fold_agg(la, ra);
  }
  out.mn[u] = a.mn;
  out.mx[u] = a.mx;
  out.com[u] = a.com;
  out.mass[u] = a.mass;
  return a;
}

// solvers/src/lbvh.rs:329-348
AggOut reference_aggregate(const Tree& t, const std::vector<V3>& sp, const double* sm) {
  size_t total = 2 * t.n - 1;
  AggOut o;
  o.mn.assign(total, V3{0, 0, 0});
  o.mx.assign(total, V3{0, 0, 0});
  o.com.assign(total, V3{0, 0, 0});
  o.mass.assign(total, 0.0);
  uint32_t root = t.n == 1 ? 0u : static_cast<uint32_t>(t.n);
  agg_node(root, t, sp, sm, o);
  return o;
}

// solvers/src/lbvh.rs:394-414
struct Node {
  V3 center, half, com;
  double mass, delta;
  uint32_t next, body_start, body_count;
};

struct Flat {
  std::vector<Node> nodes;
  std::vector<uint32_t> leaf_bodies;
};

// solvers/src/lbvh.rs:560-614
void flatten_unified(uint32_t u, const Tree& t, const AggOut& a, const uint32_t* order, Flat& f) {
  size_t me = f.nodes.size();
  if (u < t.n) {
    Node nd{};
    nd.center = a.com[u];
    nd.half = V3{0, 0, 0};
    nd.com = a.com[u];
    nd.mass = a.mass[u];
    nd.delta = 0.0;
    nd.next = static_cast<uint32_t>(me + 1);
    nd.body_start = static_cast<uint32_t>(f.leaf_bodies.size());
    nd.body_count = 1;
    f.leaf_bodies.push_back(order[u]);
    f.nodes.push_back(nd);
    return;
  }
  f.nodes.push_back(Node{});
  size_t i = u - t.n;
  flatten_unified(t.left[i], t, a, order, f);
  flatten_unified(t.right[i], t, a, order, f);
  V3 mn = a.mn[u], mx = a.mx[u];
  V3 center = (mn + mx) * 0.5;
  Node nd{};
  nd.center = center;
  nd.half = (mx - mn) * 0.5;
  nd.com = a.com[u];
  nd.mass = a.mass[u];
  nd.delta = length(a.com[u] - center);
  nd.next = static_cast<uint32_t>(f.nodes.size());
  nd.body_start = 0;
  nd.body_count = 0;
  f.nodes[me] = nd;
}

// solvers/src/lbvh.rs:545-554
Flat reference_flatten(const Tree& t, const AggOut& a, const uint32_t* order) {
  Flat f;
  f.nodes.reserve(2 * t.n - 1);
  f.leaf_bodies.reserve(t.n);
  uint32_t root = t.n == 1 ? 0u : static_cast<uint32_t>(t.n);
  flatten_unified(root, t, a, order, f);
  return f;
}

// solvers/src/lbvh.rs:143-147 -- stable by (code, original index).
template <typename K>
std::vector<uint32_t> reference_sort(const K* codes, size_t n) {
  std::vector<uint32_t> order(n);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return codes[a] < codes[b]; });
  return order;
}

// 63-bit Morton code of a position (21-bit lanes; same cube as the 30-bit codes).
uint64_t expand21(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}
uint32_t quantize_lane21(double v) {
  double f = std::fmax(std::floor(v), 0.0);
  uint32_t q = f >= 4294967295.0 ? 0xFFFFFFFFu : static_cast<uint32_t>(f);
  return std::min(q, (1u << 21) - 1);
}

template <typename K>
std::vector<K> morton_codes(const double* pos, size_t n);

template <>
std::vector<uint32_t> morton_codes<uint32_t>(const double* pos, size_t n) {
  Bounds b = morton_bounds(pos, n);
  std::vector<uint32_t> codes(n);
  for (size_t i = 0; i < n; ++i) {
    V3 p = load3(pos, i);
    codes[i] = morton3(quantize_lane((p.x - b.bmin.x) * b.scale), quantize_lane((p.y - b.bmin.y) * b.scale),
                       quantize_lane((p.z - b.bmin.z) * b.scale));
  }
  return codes;
}

template <>
std::vector<uint64_t> morton_codes<uint64_t>(const double* pos, size_t n) {
  Bounds b = morton_bounds(pos, n);
  const double scale = 2097152.0 / b.size;
  std::vector<uint64_t> codes(n);
  for (size_t i = 0; i < n; ++i) {
    V3 p = load3(pos, i);
    codes[i] = expand21(quantize_lane21((p.x - b.bmin.x) * scale)) |
               (expand21(quantize_lane21((p.y - b.bmin.y) * scale)) << 1) |
               (expand21(quantize_lane21((p.z - b.bmin.z) * scale)) << 2);
  }
  return codes;
}

// solvers/src/lbvh.rs:440-463 (K = uint32_t is the reference; uint64_t the 63-bit extension)
template <typename K = uint32_t>
Flat lbvh_build(const double* pos, const double* mass, size_t n) {
  std::vector<K> codes = morton_codes<K>(pos, n);
  std::vector<uint32_t> order = reference_sort(codes.data(), n);
  std::vector<K> sc(n);
  std::vector<V3> sp(n);
  std::vector<double> sm(n);
  for (size_t k = 0; k < n; ++k) {
    sc[k] = codes[order[k]];
    sp[k] = load3(pos, order[k]);
    sm[k] = mass[order[k]];
  }
  Tree t = reference_karras(sc.data(), n);
  AggOut a = reference_aggregate(t, sp, sm.data());
  return reference_flatten(t, a, order.data());
}

struct WalkStats {
  uint64_t leaf, far, open;
};

// solvers/src/lbvh.rs:469-524 -- stackless skip-pointer walk, Barnes (1994)
// opening test, Plummer softening, self excluded by original index.
V3 lbvh_accel(const Flat& f, size_t target, const double* pos, const double* mass, double theta, double eps2,
              WalkStats* st) {
  V3 xp = load3(pos, target);
  V3 a{0, 0, 0};
  uint32_t node = 0;
  const uint32_t n_nodes = static_cast<uint32_t>(f.nodes.size());
  while (node < n_nodes) {
    const Node& nd = f.nodes[node];
    if (nd.mass <= 0.0) {
      node = nd.next;
      continue;
    }
    if (nd.body_count > 0) {
      uint32_t end = nd.body_start + nd.body_count;
      for (uint32_t k = nd.body_start; k < end; ++k) {
        uint32_t b = f.leaf_bodies[k];
        if (b == target) continue;
        V3 dx = load3(pos, b) - xp;
        double r2 = length_squared(dx) + eps2;
        a = a + dx * (mass[b] / (r2 * std::sqrt(r2)));
        if (st) st->leaf++;
      }
      node = nd.next;
    } else {
      V3 he = nd.half;
      bool inside = std::fabs(xp.x - nd.center.x) <= he.x && std::fabs(xp.y - nd.center.y) <= he.y &&
                    std::fabs(xp.z - nd.center.z) <= he.z;
      V3 dx = nd.com - xp;
      double d2 = length_squared(dx);
      double s = 2.0 * max_element(he);
      double d = std::sqrt(d2);
      if (!inside && theta * (d - nd.delta) >= s) {
        double r2 = d2 + eps2;
        a = a + dx * (nd.mass / (r2 * std::sqrt(r2)));
        node = nd.next;
        if (st) st->far++;
      } else {
        node += 1;
        if (st) st->open++;
      }
    }
  }
  return a;
}

// ---------------------------------------------------------------------------
// Quadrupole extension (no counterpart in the reference, which is monopole
// only): same build and walk, plus the traceless quadrupole of every internal
// node about its centre of mass, Q = sum m (3 r r^T - |r|^2 I), combined
// bottom-up with the parallel-axis shift. The far-field term added on accept is
//   a += G [ Q r / r^5 - (5/2) (r^T Q r) r / r^7 ]   with r = x_target - com,
// which is minus the gradient of the potential -G (r^T Q r)/(2 r^5). Softening enters
// through r^2 -> r^2 + eps^2. Used only to grade the GPU quadrupole mode.
struct Quad {
  double xx, xy, xz, yy, yz, zz;
};

Quad quad_shift(const Quad& q, double m, V3 d) {
  // Q about a new origin where d = com_child - com_parent.
  double d2 = length_squared(d);
  Quad r;
  r.xx = q.xx + m * (3.0 * d.x * d.x - d2);
  r.yy = q.yy + m * (3.0 * d.y * d.y - d2);
  r.zz = q.zz + m * (3.0 * d.z * d.z - d2);
  r.xy = q.xy + m * (3.0 * d.x * d.y);
  r.xz = q.xz + m * (3.0 * d.x * d.z);
  r.yz = q.yz + m * (3.0 * d.y * d.z);
  return r;
}

Quad quad_node(uint32_t u, const Tree& t, const AggOut& a, std::vector<Quad>& out) {
  Quad q{0, 0, 0, 0, 0, 0};
  if (u >= t.n) {
    size_t i = u - t.n;
    uint32_t l = t.left[i], r = t.right[i];
    Quad ql = quad_node(l, t, a, out);
    Quad qr = quad_node(r, t, a, out);
    Quad sl = quad_shift(ql, a.mass[l], a.com[l] - a.com[u]);
    Quad sr = quad_shift(qr, a.mass[r], a.com[r] - a.com[u]);
    q = Quad{sl.xx + sr.xx, sl.xy + sr.xy, sl.xz + sr.xz, sl.yy + sr.yy, sl.yz + sr.yz, sl.zz + sr.zz};
  }
  out[u] = q;
  return q;
}

// Shared Plummer-sphere helpers (ic/src/plummer.rs:142-175 restated for the
// N=16,384 seed-0 parity case lives in the product IC module; the oracle only
// needs the LCG fixtures below).

// solvers/tests/lbvh.rs:27-44 / gpu/tests/lbvh_sort.rs:25-37 LCG draw in [0,1).
struct Lcg {
  uint64_t state;
  explicit Lcg(uint64_t seed) : state(seed | 1ull) {}
  double next() {
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    return static_cast<double>(state >> 11) / static_cast<double>(1ull << 53);
  }
  uint32_t next_code() {
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    return static_cast<uint32_t>(state >> 33) & ((1u << 30) - 1);
  }
};

}  // namespace

extern "C" {

// ---- Morton ---------------------------------------------------------------
uint32_t or_expand10(uint32_t v) { return expand10(v); }
uint32_t or_morton3(uint32_t x, uint32_t y, uint32_t z) { return morton3(x, y, z); }

// reference_morton: bounds_out = {bmin.x, bmin.y, bmin.z, size, scale}.
int or_reference_morton(size_t n, const double* pos, uint32_t* lanes_out, uint32_t* codes_out, double* bounds_out) {
  if (n == 0) return 1;
  Bounds b = morton_bounds(pos, n);
  for (size_t i = 0; i < n; ++i) {
    V3 p = load3(pos, i);
    uint32_t lx = quantize_lane((p.x - b.bmin.x) * b.scale);
    uint32_t ly = quantize_lane((p.y - b.bmin.y) * b.scale);
    uint32_t lz = quantize_lane((p.z - b.bmin.z) * b.scale);
    if (lanes_out) {
      lanes_out[3 * i] = lx;
      lanes_out[3 * i + 1] = ly;
      lanes_out[3 * i + 2] = lz;
    }
    codes_out[i] = morton3(lx, ly, lz);
  }
  if (bounds_out) {
    bounds_out[0] = b.bmin.x;
    bounds_out[1] = b.bmin.y;
    bounds_out[2] = b.bmin.z;
    bounds_out[3] = b.size;
    bounds_out[4] = b.scale;
  }
  return 0;
}

// ---- sort -------------------------------------------------------------------
void or_reference_sort(size_t n, const uint32_t* codes, uint32_t* order_out) {
  std::vector<uint32_t> o = reference_sort(codes, n);
  if (n) std::memcpy(order_out, o.data(), n * sizeof(uint32_t));
}

// ---- Karras -----------------------------------------------------------------
int or_reference_karras(size_t n, const uint32_t* sorted_codes, uint32_t* left, uint32_t* right, uint32_t* parent) {
  if (n == 0) return 1;
  Tree t = reference_karras(sorted_codes, n);
  if (n > 1) {
    std::memcpy(left, t.left.data(), (n - 1) * sizeof(uint32_t));
    std::memcpy(right, t.right.data(), (n - 1) * sizeof(uint32_t));
  }
  std::memcpy(parent, t.parent.data(), (2 * n - 1) * sizeof(uint32_t));
  return 0;
}

// ---- aggregate ------------------------------------------------------------
// Outputs per unified node (2n-1 entries): aabb_min[3], aabb_max[3], com[3], mass.
int or_reference_aggregate(size_t n, const uint32_t* left, const uint32_t* right, const double* sorted_pos,
                           const double* sorted_mass, double* aabb_min, double* aabb_max, double* com,
                           double* mass) {
  if (n == 0) return 1;
  Tree t;
  t.n = n;
  t.left.assign(left, left + (n - 1));
  t.right.assign(right, right + (n - 1));
  std::vector<V3> sp(n);
  for (size_t k = 0; k < n; ++k) sp[k] = load3(sorted_pos, k);
  AggOut a = reference_aggregate(t, sp, sorted_mass);
  for (size_t u = 0; u < 2 * n - 1; ++u) {
    store3(aabb_min, u, a.mn[u]);
    store3(aabb_max, u, a.mx[u]);
    store3(com, u, a.com[u]);
    mass[u] = a.mass[u];
  }
  return 0;
}

// ---- quadrupole (extension; see comment above) -----------------------------
// quad_out: 6 per unified node (xx, xy, xz, yy, yz, zz) about the node's com.
int or_quadrupole(size_t n, const uint32_t* left, const uint32_t* right, const double* com, const double* mass,
                  double* quad_out) {
  if (n == 0) return 1;
  Tree t;
  t.n = n;
  t.left.assign(left, left + (n - 1));
  t.right.assign(right, right + (n - 1));
  AggOut a;
  size_t total = 2 * n - 1;
  a.com.resize(total);
  a.mass.assign(mass, mass + total);
  for (size_t u = 0; u < total; ++u) a.com[u] = load3(com, u);
  std::vector<Quad> q(total);
  quad_node(n == 1 ? 0u : static_cast<uint32_t>(n), t, a, q);
  for (size_t u = 0; u < total; ++u) {
    quad_out[6 * u + 0] = q[u].xx;
    quad_out[6 * u + 1] = q[u].xy;
    quad_out[6 * u + 2] = q[u].xz;
    quad_out[6 * u + 3] = q[u].yy;
    quad_out[6 * u + 4] = q[u].yz;
    quad_out[6 * u + 5] = q[u].zz;
  }
  return 0;
}

// ---- flatten --------------------------------------------------------------
// node_f64: 11 doubles per node: center[3], half[3], com[3], mass, delta.
// node_u32: 3 per node: next, body_start, body_count.
int or_lbvh_flat(size_t n, const double* pos, const double* mass, double* node_f64, uint32_t* node_u32,
                 uint32_t* leaf_bodies) {
  if (n == 0) return 1;
  Flat f = lbvh_build(pos, mass, n);
  for (size_t k = 0; k < f.nodes.size(); ++k) {
    const Node& nd = f.nodes[k];
    double* o = node_f64 + 11 * k;
    o[0] = nd.center.x;
    o[1] = nd.center.y;
    o[2] = nd.center.z;
    o[3] = nd.half.x;
    o[4] = nd.half.y;
    o[5] = nd.half.z;
    o[6] = nd.com.x;
    o[7] = nd.com.y;
    o[8] = nd.com.z;
    o[9] = nd.mass;
    o[10] = nd.delta;
    node_u32[3 * k] = nd.next;
    node_u32[3 * k + 1] = nd.body_start;
    node_u32[3 * k + 2] = nd.body_count;
  }
  std::memcpy(leaf_bodies, f.leaf_bodies.data(), n * sizeof(uint32_t));
  return 0;
}

// ---- Lbvh::accelerations (solvers/src/lbvh.rs:662-676) --------------------
// threads <= 1 runs the reference's serial per-target loop; threads > 1 splits
// targets over OpenMP threads (each target is an independent accumulation, so
// the result is identical). stats (optional): {leaf, far, open} totals.
int or_lbvh_accelerations(size_t n, const double* pos, const double* mass, double g, double softening, double theta,
                          double* acc_out, int threads, uint64_t* stats) {
  if (n == 0) return 0;
  Flat f = lbvh_build(pos, mass, n);
  const double eps2 = softening * softening;
  uint64_t tl = 0, tf = 0, to = 0;
  if (threads <= 1) {
    WalkStats st{0, 0, 0};
    for (size_t i = 0; i < n; ++i) store3(acc_out, i, lbvh_accel(f, i, pos, mass, theta, eps2, stats ? &st : nullptr) * g);
    tl = st.leaf;
    tf = st.far;
    to = st.open;
  } else {
#pragma omp parallel for num_threads(threads) schedule(dynamic, 256) reduction(+ : tl, tf, to)
    for (long long i = 0; i < static_cast<long long>(n); ++i) {
      WalkStats st{0, 0, 0};
      store3(acc_out, i, lbvh_accel(f, i, pos, mass, theta, eps2, stats ? &st : nullptr) * g);
      tl += st.leaf;
      tf += st.far;
      to += st.open;
    }
  }
  if (stats) {
    stats[0] = tl;
    stats[1] = tf;
    stats[2] = to;
  }
  return 0;
}

// The same solver over 63-bit Morton keys (extension: no reference counterpart).
int or_lbvh_accelerations_k63(size_t n, const double* pos, const double* mass, double g, double softening,
                              double theta, double* acc_out, int threads, uint64_t* stats) {
  if (n == 0) return 0;
  Flat f = lbvh_build<uint64_t>(pos, mass, n);
  const double eps2 = softening * softening;
  uint64_t tl = 0, tf = 0, to = 0;
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 256) reduction(+ : tl, tf, to)
  for (long long i = 0; i < static_cast<long long>(n); ++i) {
    WalkStats st{0, 0, 0};
    store3(acc_out, i, lbvh_accel(f, i, pos, mass, theta, eps2, stats ? &st : nullptr) * g);
    tl += st.leaf;
    tf += st.far;
    to += st.open;
  }
  if (stats) {
    stats[0] = tl;
    stats[1] = tf;
    stats[2] = to;
  }
  return 0;
}

// Monopole walk restricted to a list of targets (bounded CPU samples for the
// baseline timing): builds the full tree, walks only `targets`.
int or_lbvh_accelerations_subset(size_t n, const double* pos, const double* mass, double g, double softening,
                                 double theta, size_t n_targets, const uint32_t* targets, double* acc_out,
                                 int threads) {
  if (n == 0) return 0;
  Flat f = lbvh_build(pos, mass, n);
  const double eps2 = softening * softening;
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64)
  for (long long k = 0; k < static_cast<long long>(n_targets); ++k)
    store3(acc_out, k, lbvh_accel(f, targets[k], pos, mass, theta, eps2, nullptr) * g);
  return 0;
}

// Stale-tree active walk, as TreeGravity::gravity_active_cached
// (solvers/src/barnes_hut.rs:683-710) does over its cached FlatTree, here over the
// LBVH: the tree (topology, cell aggregates, leaf skip flags) is built from
// (pos_build, mass_build); each target is walked at its current position and leaf
// sources are read from (pos_now, mass_now) -- lbvh_accel reads targets and bodies
// from the arrays it is given, so passing the current ones is exactly that.
int or_lbvh_accelerations_stale(size_t n, const double* pos_build, const double* mass_build, const double* pos_now,
                                const double* mass_now, double g, double softening, double theta, size_t n_targets,
                                const uint32_t* targets, double* acc_out, int threads) {
  if (n == 0) return 0;
  Flat f = lbvh_build(pos_build, mass_build, n);
  const double eps2 = softening * softening;
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64)
  for (long long k = 0; k < static_cast<long long>(n_targets); ++k)
    store3(acc_out, k, lbvh_accel(f, targets[k], pos_now, mass_now, theta, eps2, nullptr) * g);
  return 0;
}

// Quadrupole walk (extension): identical decisions to the monopole walk; on
// accept the softened quadrupole correction is added to the monopole term.
int or_lbvh_accelerations_quad(size_t n, const double* pos, const double* mass, double g, double softening,
                               double theta, double* acc_out, int threads) {
  if (n == 0) return 0;
  Bounds b = morton_bounds(pos, n);
  std::vector<uint32_t> codes(n);
  for (size_t i = 0; i < n; ++i) {
    V3 p = load3(pos, i);
    codes[i] = morton3(quantize_lane((p.x - b.bmin.x) * b.scale), quantize_lane((p.y - b.bmin.y) * b.scale),
                       quantize_lane((p.z - b.bmin.z) * b.scale));
  }
  std::vector<uint32_t> order = reference_sort(codes.data(), n);
  std::vector<uint32_t> sc(n);
  std::vector<V3> sp(n);
  std::vector<double> sm(n);
  for (size_t k = 0; k < n; ++k) {
    sc[k] = codes[order[k]];
    sp[k] = load3(pos, order[k]);
    sm[k] = mass[order[k]];
  }
  Tree t = reference_karras(sc.data(), n);
  AggOut a = reference_aggregate(t, sp, sm.data());
  Flat f = reference_flatten(t, a, order.data());
  std::vector<Quad> qu(2 * n - 1);
  quad_node(n == 1 ? 0u : static_cast<uint32_t>(n), t, a, qu);
  // Map flat pre-order slots back to unified indices (same recursion order).
  std::vector<uint32_t> slot_to_u;
  slot_to_u.reserve(2 * n - 1);
  std::vector<uint32_t> stk;
  stk.push_back(n == 1 ? 0u : static_cast<uint32_t>(n));
  while (!stk.empty()) {
    uint32_t u = stk.back();
    stk.pop_back();
    slot_to_u.push_back(u);
    if (u >= n) {
      stk.push_back(t.right[u - n]);
      stk.push_back(t.left[u - n]);
    }
  }
  const double eps2 = softening * softening;
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 256)
  for (long long i = 0; i < static_cast<long long>(n); ++i) {
    V3 xp = load3(pos, i);
    V3 acc{0, 0, 0};
    uint32_t node = 0;
    const uint32_t nn = static_cast<uint32_t>(f.nodes.size());
    while (node < nn) {
      const Node& nd = f.nodes[node];
      if (nd.mass <= 0.0) {
        node = nd.next;
        continue;
      }
      if (nd.body_count > 0) {
        uint32_t bb = f.leaf_bodies[nd.body_start];
        if (bb != static_cast<uint32_t>(i)) {
          V3 dx = load3(pos, bb) - xp;
          double r2 = length_squared(dx) + eps2;
          acc = acc + dx * (mass[bb] / (r2 * std::sqrt(r2)));
        }
        node = nd.next;
      } else {
        V3 he = nd.half;
        bool inside = std::fabs(xp.x - nd.center.x) <= he.x && std::fabs(xp.y - nd.center.y) <= he.y &&
                      std::fabs(xp.z - nd.center.z) <= he.z;
        V3 dx = nd.com - xp;
        double d2 = length_squared(dx);
        double s = 2.0 * max_element(he);
        double d = std::sqrt(d2);
        if (!inside && theta * (d - nd.delta) >= s) {
          double r2 = d2 + eps2;
          double inv = 1.0 / std::sqrt(r2);
          double inv2 = inv * inv;
          double inv3 = inv * inv2;
          acc = acc + dx * (nd.mass * inv3);
          const Quad& q = qu[slot_to_u[node]];
          // r = x_target - com = -dx
          V3 r{-dx.x, -dx.y, -dx.z};
          V3 qr{q.xx * r.x + q.xy * r.y + q.xz * r.z, q.xy * r.x + q.yy * r.y + q.yz * r.z,
                q.xz * r.x + q.yz * r.y + q.zz * r.z};
          double rqr = dot(r, qr);
          double inv5 = inv3 * inv2;
          double inv7 = inv5 * inv2;
          acc = acc + qr * inv5 - r * (2.5 * rqr * inv7);
          node = nd.next;
        } else {
          node += 1;
        }
      }
    }
    store3(acc_out, i, acc * g);
  }
  return 0;
}

// ---- DirectSum::accelerations (solvers/src/direct_sum.rs:25-45) ------------
void or_direct_sum(size_t n, const double* pos, const double* mass, double g, double softening, double* acc_out) {
  for (size_t i = 0; i < 3 * n; ++i) acc_out[i] = 0.0;
  const double eps2 = softening * softening;
  for (size_t i = 0; i < n; ++i) {
    V3 xi = load3(pos, i);
    double mi = mass[i];
    V3 ai = load3(acc_out, i);
    for (size_t j = i + 1; j < n; ++j) {
      V3 dx = load3(pos, j) - xi;
      double r2 = length_squared(dx) + eps2;
      double inv_r3 = 1.0 / (r2 * std::sqrt(r2));
      V3 w = dx * (g * inv_r3);
      ai = ai + w * mass[j];
      store3(acc_out, j, load3(acc_out, j) - w * mi);
    }
    store3(acc_out, i, ai);
  }
}

// FP64 direct sum on a subset of targets (per-target, unpaired): the force
// oracle for large systems. Not a reference function: an exact O(N * T) sum.
void or_direct_sum_targets(size_t n, const double* pos, const double* mass, double g, double softening,
                           size_t n_targets, const uint32_t* targets, double* acc_out, int threads) {
  const double eps2 = softening * softening;
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 16)
  for (long long k = 0; k < static_cast<long long>(n_targets); ++k) {
    size_t i = targets[k];
    V3 xi = load3(pos, i);
    V3 a{0, 0, 0};
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      V3 dx = load3(pos, j) - xi;
      double r2 = length_squared(dx) + eps2;
      a = a + dx * (mass[j] / (r2 * std::sqrt(r2)));
    }
    store3(acc_out, k, a * g);
  }
}

// ---- potential (solvers/src/potential.rs:17-58) ----------------------------
static double row_potential(size_t i, size_t n, const double* pos, const double* mass, double g, double eps2) {
  double u = 0.0;
  V3 pi = load3(pos, i);
  for (size_t j = i + 1; j < n; ++j) {
    V3 dx = load3(pos, j) - pi;
    double r = std::sqrt(length_squared(dx) + eps2);
    u -= g * mass[i] * mass[j] / r;
  }
  return u;
}

double or_potential_serial(size_t n, const double* pos, const double* mass, double g, double softening) {
  const double eps2 = softening * softening;
  double u = 0.0;
  for (size_t i = 0; i < n; ++i) u += row_potential(i, n, pos, mass, g, eps2);
  return u;
}

double or_potential_parallel(size_t n, const double* pos, const double* mass, double g, double softening,
                             int threads) {
  const double eps2 = softening * softening;
  double u = 0.0;
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64) reduction(+ : u)
  for (long long i = 0; i < static_cast<long long>(n); ++i) u += row_potential(i, n, pos, mass, g, eps2);
  return u;
}

// ---- diagnostics (core/src/diagnostics.rs:8-68) ---------------------------
// out: {kinetic, px, py, pz, lx, ly, lz}
void or_diagnostics(size_t n, const double* pos, const double* vel, const double* mass, double* out) {
  double k = 0.0;
  V3 p{0, 0, 0}, l{0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    V3 v = load3(vel, i), r = load3(pos, i);
    double m = mass[i];
    k += 0.5 * m * length_squared(v);
    p = p + v * m;
    V3 c{r.y * v.z - r.z * v.y, r.z * v.x - r.x * v.z, r.x * v.y - r.y * v.x};
    l = l + c * m;
  }
  out[0] = k;
  out[1] = p.x;
  out[2] = p.y;
  out[3] = p.z;
  out[4] = l.x;
  out[5] = l.y;
  out[6] = l.z;
}

// ---- LeapfrogKdk::step with the Lbvh solver (core/src/integrator.rs:38-78) --
// acc_io carries the cached acceleration between calls; primed_io is the
// integrator's `primed` flag. Runs `steps` KDK steps in place.
int or_kdk_lbvh(size_t n, double* pos, double* vel, const double* mass, double* acc_io, int* primed_io, double g,
                double softening, double theta, double dt, uint64_t steps, int threads) {
  if (n == 0) return 0;
  for (uint64_t s = 0; s < steps; ++s) {
    if (!*primed_io) {
      or_lbvh_accelerations(n, pos, mass, g, softening, theta, acc_io, threads, nullptr);
      *primed_io = 1;
    }
    const double half = 0.5 * dt;
    for (size_t i = 0; i < n; ++i) store3(vel, i, load3(vel, i) + load3(acc_io, i) * half);
    for (size_t i = 0; i < n; ++i) store3(pos, i, load3(pos, i) + load3(vel, i) * dt);
    or_lbvh_accelerations(n, pos, mass, g, softening, theta, acc_io, threads, nullptr);
    for (size_t i = 0; i < n; ++i) store3(vel, i, load3(vel, i) + load3(acc_io, i) * half);
  }
  return 0;
}

// ---- fixtures of the reference tests ---------------------------------------
// solvers/tests/lbvh.rs:27-44 `cluster`: pos in a 3-wide cube, vel 0, mass in [0.1,1).
void or_fixture_cluster(uint64_t seed, size_t n, double* pos, double* vel, double* mass) {
  Lcg r(seed);
  for (size_t i = 0; i < n; ++i) {
    double a = r.next() - 0.5;
    double b = r.next() - 0.5;
    double c = r.next() - 0.5;
    pos[3 * i] = a * 3.0;
    pos[3 * i + 1] = b * 3.0;
    pos[3 * i + 2] = c * 3.0;
    vel[3 * i] = vel[3 * i + 1] = vel[3 * i + 2] = 0.0;
    mass[i] = 0.1 + 0.9 * r.next();
  }
}

// gpu/tests/lbvh_sort.rs:25-37 `cloud`: center + (u - 0.5) * 2r per axis.
void or_fixture_cloud(uint64_t seed, size_t n, double r, double cx, double cy, double cz, double* pos) {
  Lcg g(seed);
  for (size_t i = 0; i < n; ++i) {
    double a = g.next() - 0.5;
    double b = g.next() - 0.5;
    double c = g.next() - 0.5;
    pos[3 * i] = cx + a * (2.0 * r);
    pos[3 * i + 1] = cy + b * (2.0 * r);
    pos[3 * i + 2] = cz + c * (2.0 * r);
  }
}

// gpu/tests/lbvh_tree.rs:47-58 `masses`: 0.5 + u.
void or_fixture_masses(uint64_t seed, size_t n, double* mass) {
  Lcg g(seed);
  for (size_t i = 0; i < n; ++i) mass[i] = 0.5 + g.next();
}

// gpu/tests/lbvh_sort.rs:41-51 `random_codes`: 30-bit codes from the LCG high bits.
void or_fixture_random_codes(uint64_t seed, size_t n, uint32_t* codes) {
  Lcg g(seed);
  for (size_t i = 0; i < n; ++i) codes[i] = g.next_code();
}

int or_openmp_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
