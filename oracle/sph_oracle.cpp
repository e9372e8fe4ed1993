// sph_oracle.cpp -- TEST INFRASTRUCTURE ONLY: a CPU f64 restatement of the galaxy
// reference's isothermal/adiabatic SPH toolkit and its gravity + SPH composite, the
// checker of the library's SPH kernels.
//
// Followed line by line (file:line in the reference project):
//   solvers/src/sph/kernel.rs:23-53      cubic spline W and its gradient
//   solvers/src/sph/grid.rs:24-90        the uniform hash grid (cells keyed by floor(x/cell))
//   solvers/src/sph/reference.rs:10-35   brute-force neighbours / density
//   solvers/src/sph/density.rs:53-327    fixed-h and adaptive-h density (DensitySetup, solve_one)
//   solvers/src/sph/forces.rs:223-379    HydroCtx::force_one (acceleration and du/dt)
//   solvers/src/sph/cfl.rs:49-185        max_stable_dt / max_stable_dt_per_particle
//   solvers/src/sph/gravity_sph.rs:172-207  GravitySph::accelerations (gravity on all,
//                                        hydro on the gas subset, h warm start)
//   core/src/integrator.rs:38-78         KDK stepping of that composite
//
// Arithmetic convention: glam's DVec3 operations are per-component IEEE f64 with no
// fused multiply-add; `length()` is sqrt((x*x + y*y) + z*z). The file is compiled with
// -ffp-contract=off, and every expression below keeps the reference's operand order.
// Parity pins: the reference's frozen output bits of hydro_accelerations
// (solvers/tests/sph_forces.rs:393-462) and of max_stable_dt
// (solvers/tests/sph_cfl.rs:189-212), checked by the oracle's tests.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <unordered_map>
#include <vector>

extern "C" int or_lbvh_accelerations(size_t n, const double* pos, const double* mass, double g, double softening,
                                     double theta, double* acc_out, int threads, void* stats);

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kSupport = 2.0;

struct D3 {
  double x, y, z;
};
inline D3 ld(const double* a, size_t i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double length(D3 a) { return std::sqrt(dot(a, a)); }
// f64::min / f64::max: the non-NaN operand when one is NaN.
inline double fmin_(double a, double b) { return std::fmin(a, b); }
inline double fmax_(double a, double b) { return std::fmax(a, b); }

// kernel.rs:27-38
double w(double r, double h) {
  const double q = r / h;
  const double norm = 1.0 / (kPi * h * h * h);
  if (q < 1.0) return norm * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
  if (q < 2.0) {
    const double t = 2.0 - q;
    return norm * 0.25 * t * t * t;
  }
  return 0.0;
}

// kernel.rs:40-53
D3 grad_w(D3 r_ij, double h) {
  const double r = length(r_ij);
  const double q = r / h;
  if (r == 0.0 || q >= 2.0) return {0.0, 0.0, 0.0};
  const double norm = 1.0 / (kPi * h * h * h);
  double dp;
  if (q < 1.0) {
    dp = -3.0 * q + 2.25 * q * q;
  } else {
    const double t = 2.0 - q;
    dp = -0.75 * t * t;
  }
  return mul(r_ij, norm * dp / (h * r));
}

// Rust's saturating `f64 as i64` (NaN -> 0).
int64_t sat_i64(double v) {
  if (std::isnan(v)) return 0;
  if (v >= 9223372036854775807.0) return std::numeric_limits<int64_t>::max();
  if (v <= -9223372036854775808.0) return std::numeric_limits<int64_t>::min();
  return static_cast<int64_t>(v);
}

struct CellKey {
  int64_t x, y, z;
  bool operator==(const CellKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct CellHash {
  size_t operator()(const CellKey& k) const {
    uint64_t h = static_cast<uint64_t>(k.x) * 0x9E3779B97F4A7C15ull;
    h ^= static_cast<uint64_t>(k.y) * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
    h ^= static_cast<uint64_t>(k.z) * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
    return static_cast<size_t>(h);
  }
};

// grid.rs:85-90
CellKey cell_of(D3 p, double cell) {
  return {sat_i64(std::floor(p.x / cell)), sat_i64(std::floor(p.y / cell)), sat_i64(std::floor(p.z / cell))};
}

// grid.rs:24-82: sparse cells of edge `cell`, each holding its particles ascending.
struct HashGrid {
  double cell = 1.0;
  std::unordered_map<CellKey, std::vector<uint32_t>, CellHash> cells;

  HashGrid(const double* pos, size_t n, double c) : cell(c) {
    for (size_t i = 0; i < n; ++i) cells[cell_of(ld(pos, i), cell)].push_back(static_cast<uint32_t>(i));
  }
  size_t bin_len(D3 p) const {
    auto it = cells.find(cell_of(p, cell));
    return it == cells.end() ? 0 : it->second.size();
  }
  // Indices j (ascending) with |pos[j] - center|^2 <= r^2.
  void within(const double* pos, D3 center, double r, std::vector<uint32_t>& out) const {
    out.clear();
    if (cells.empty() || r < 0.0) return;
    const double r2 = r * r;
    const CellKey lo = cell_of(sub(center, {r, r, r}), cell);
    const CellKey hi = cell_of(add(center, {r, r, r}), cell);
    for (int64_t cx = lo.x; cx <= hi.x; ++cx)
      for (int64_t cy = lo.y; cy <= hi.y; ++cy)
        for (int64_t cz = lo.z; cz <= hi.z; ++cz) {
          auto it = cells.find({cx, cy, cz});
          if (it == cells.end()) continue;
          for (uint32_t j : it->second) {
            const D3 d = sub(ld(pos, j), center);
            if (dot(d, d) <= r2) out.push_back(j);
          }
        }
    std::sort(out.begin(), out.end());
  }
};

// density.rs:156-289
struct DensitySetup {
  const double* pos;
  const double* mass;
  size_t n;
  double n_ngb, h_tol_rel;
  std::vector<double> seeds;
  double h_cap = 0.0;
  HashGrid* grid = nullptr;

  DensitySetup(const double* p, const double* m, size_t nn, double ngb, double tol)
      : pos(p), mass(m), n(nn), n_ngb(ngb), h_tol_rel(tol) {
    D3 lo_c = ld(pos, 0), hi_c = ld(pos, 0);
    for (size_t i = 0; i < n; ++i) {
      const D3 q = ld(pos, i);
      lo_c = {fmin_(lo_c.x, q.x), fmin_(lo_c.y, q.y), fmin_(lo_c.z, q.z)};
      hi_c = {fmax_(hi_c.x, q.x), fmax_(hi_c.y, q.y), fmax_(hi_c.z, q.z)};
    }
    const D3 extent = sub(hi_c, lo_c);
    const double diag = length(extent);
    const double vol = extent.x * extent.y * extent.z;
    const double s_est = vol > 0.0 ? std::cbrt(vol / static_cast<double>(n))
                                   : (diag > 0.0 ? diag / std::cbrt(static_cast<double>(n)) : 1.0);
    const double seed_scale = std::cbrt(3.0 * n_ngb / (32.0 * kPi));
    const double h_seed = s_est * seed_scale;
    h_cap = fmax_(64.0 * h_seed, 4.0 * diag);
    const double occ_bin = 4.0 * s_est;
    HashGrid occupancy(pos, n, occ_bin);
    seeds.resize(n);
    for (size_t i = 0; i < n; ++i) {
      const double c = static_cast<double>(std::max<size_t>(occupancy.bin_len(ld(pos, i)), 1));
      seeds[i] = fmin_((occ_bin / std::cbrt(c)) * seed_scale, h_cap);
    }
    std::vector<double> sorted = seeds;
    std::sort(sorted.begin(), sorted.end());
    const double cell = fmax_(fmin_(kSupport * sorted[n / 2], kSupport * h_seed), 1e-12);
    grid = new HashGrid(pos, n, cell);
  }
  ~DensitySetup() { delete grid; }

  double count(size_t i, double h, const std::vector<uint32_t>& cand) const {
    double sum = 0.0;
    const D3 xi = ld(pos, i);
    for (uint32_t j : cand) sum += w(length(sub(xi, ld(pos, j))), h);
    const double s = kSupport * h;
    return (4.0 * kPi / 3.0) * (s * s * s) * sum;
  }

  void solve_one(size_t i, const double* hint, double* rho_out, double* h_out) const {
    double seed = seeds[i];
    if (hint && std::isfinite(*hint) && *hint > 0.0) seed = *hint;
    double lo = fmin_(seed / 2.0, h_cap);
    double hi = fmin_(seed * 2.0, h_cap);
    std::vector<uint32_t> cand;
    const D3 xi = ld(pos, i);
    grid->within(pos, xi, kSupport * hi, cand);
    while (count(i, hi, cand) < n_ngb && hi < h_cap) {
      hi = fmin_(hi * 2.0, h_cap);
      grid->within(pos, xi, kSupport * hi, cand);
    }
    int shrinks = 0;
    while (count(i, lo, cand) > n_ngb && shrinks < 60) {
      lo /= 2.0;
      shrinks += 1;
    }
    double h;
    if (count(i, hi, cand) < n_ngb) {
      h = hi;
    } else if (count(i, lo, cand) > n_ngb) {
      h = lo;
    } else {
      while (hi - lo > h_tol_rel * hi) {
        const double mid = 0.5 * (lo + hi);
        if (count(i, mid, cand) < n_ngb)
          lo = mid;
        else
          hi = mid;
      }
      h = 0.5 * (lo + hi);
    }
    double rho = 0.0;
    for (uint32_t j : cand) rho += mass[j] * w(length(sub(xi, ld(pos, j))), h);
    *rho_out = rho;
    *h_out = h;
  }
};

// forces.rs: the EOS closure and one target's gather.
struct Hydro {
  const double *pos, *vel, *mass, *rho, *h, *u;
  size_t n;
  int adiabatic;
  double c_s, gamma, alpha, beta, visc_eps2;
  double cs2 = 0.0, h_max = 0.0;
  std::vector<double> cs;
  HashGrid* grid = nullptr;

  double term(size_t k) const { return adiabatic ? (gamma - 1.0) * u[k] / rho[k] : cs2 / rho[k]; }
  double c_bar(size_t i, size_t j) const { return adiabatic ? 0.5 * (cs[i] + cs[j]) : c_s; }

  void setup() {
    h_max = 0.0;
    for (size_t k = 0; k < n; ++k) h_max = fmax_(h_max, h[k]);
    grid = new HashGrid(pos, n, kSupport * h_max);
    if (adiabatic) {
      cs.resize(n);
      for (size_t k = 0; k < n; ++k) cs[k] = std::sqrt(gamma * (gamma - 1.0) * u[k]);
    } else {
      cs2 = c_s * c_s;
    }
  }
  ~Hydro() { delete grid; }

  void force_one(size_t i, D3* a_out, double* dudt_out) const {
    const D3 xi = ld(pos, i);
    const double term_i = term(i);
    std::vector<uint32_t> ngb;
    grid->within(pos, xi, kSupport * h_max, ngb);
    D3 a{0.0, 0.0, 0.0};
    double dudt_i = 0.0;
    for (uint32_t j : ngb) {
      if (j == i) continue;
      const D3 r_ij = sub(xi, ld(pos, j));
      const double r = length(r_ij);
      const D3 grad_avg = mul(add(grad_w(r_ij, h[i]), grad_w(r_ij, h[j])), 0.5);
      const double term_j = term(j);
      const D3 v_ij = sub(ld(vel, i), ld(vel, j));
      const double vr = dot(v_ij, r_ij);
      double visc = 0.0;
      if (vr < 0.0) {
        const double h_bar = 0.5 * (h[i] + h[j]);
        const double rho_bar = 0.5 * (rho[i] + rho[j]);
        const double mu = h_bar * vr / (r * r + visc_eps2 * h_bar * h_bar);
        const double cb = c_bar(i, j);
        visc = (-alpha * cb * mu + beta * mu * mu) / rho_bar;
      }
      const double coeff = term_i + term_j + visc;
      a = add(a, mul(grad_avg, -mass[j] * coeff));
      dudt_i += mass[j] * (term_i + 0.5 * visc) * dot(v_ij, grad_avg);
    }
    *a_out = a;
    *dudt_out = dudt_i;
  }
};

// cfl.rs:67-121 / 158-184: dt_i = c_cfl h_i / v_sig,i over a gas subset with given h.
void cfl_per_particle(size_t n, const double* gpos, const double* gvel, const double* h, const double* u,
                      int adiabatic, double c_s, double gamma, double c_cfl, double* dt_out, int threads) {
  double h_max = 0.0;
  for (size_t k = 0; k < n; ++k) h_max = fmax_(h_max, h[k]);
  HashGrid grid(gpos, n, kSupport * h_max);
  std::vector<double> cs;
  if (adiabatic) {
    cs.resize(n);
    for (size_t k = 0; k < n; ++k) cs[k] = std::sqrt(gamma * (gamma - 1.0) * u[k]);
  }
  const double two_cs = 2.0 * c_s;
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64)
  for (size_t i = 0; i < n; ++i) {
    std::vector<uint32_t> ngb;
    grid.within(gpos, ld(gpos, i), kSupport * h_max, ngb);
    double v_sig = adiabatic ? 2.0 * cs[i] : two_cs;
    for (uint32_t j : ngb) {
      if (j == i) continue;
      const D3 r_ij = sub(ld(gpos, i), ld(gpos, j));
      const double r = length(r_ij);
      if (r == 0.0 || r >= kSupport * fmax_(h[i], h[j])) continue;
      const double wv = dot(sub(ld(gvel, i), ld(gvel, j)), r_ij) / r;
      if (adiabatic) {
        const double approach = wv < 0.0 ? -3.0 * wv : 0.0;
        v_sig = fmax_(v_sig, cs[i] + cs[j] + approach);
      } else if (wv < 0.0) {
        v_sig = fmax_(v_sig, two_cs - 3.0 * wv);
      }
    }
    dt_out[i] = c_cfl * h[i] / v_sig;
  }
}

void gather_gas(size_t n, const uint8_t* kind, std::vector<size_t>& gas) {
  gas.clear();
  for (size_t i = 0; i < n; ++i)
    if (kind[i] == 1) gas.push_back(i);
}

void subset3(const double* a, const std::vector<size_t>& idx, std::vector<double>& out) {
  out.resize(3 * idx.size());
  for (size_t k = 0; k < idx.size(); ++k)
    for (int c = 0; c < 3; ++c) out[3 * k + c] = a[3 * idx[k] + c];
}
void subset1(const double* a, const std::vector<size_t>& idx, std::vector<double>& out) {
  out.resize(idx.size());
  for (size_t k = 0; k < idx.size(); ++k) out[k] = a ? a[idx[k]] : 0.0;
}

}  // namespace

extern "C" {

double or_sph_w(double r, double h) { return w(r, h); }

void or_sph_grad_w(double rx, double ry, double rz, double h, double* out3) {
  const D3 g = grad_w({rx, ry, rz}, h);
  out3[0] = g.x;
  out3[1] = g.y;
  out3[2] = g.z;
}

// grid.rs:57-82 (via HashGrid of edge `cell`) or reference.rs:10-18 (cell <= 0): the
// ascending neighbours of `center` within r; returns their count, writes up to cap.
size_t or_sph_neighbours(size_t n, const double* pos, double cell, const double* center, double r, uint32_t* out,
                         size_t cap) {
  std::vector<uint32_t> v;
  const D3 c{center[0], center[1], center[2]};
  if (cell > 0.0) {
    HashGrid g(pos, n, cell);
    g.within(pos, c, r, v);
  } else {
    const double r2 = r * r;
    for (size_t j = 0; j < n; ++j) {
      const D3 d = sub(ld(pos, j), c);
      if (dot(d, d) <= r2) v.push_back(static_cast<uint32_t>(j));
    }
  }
  for (size_t k = 0; k < v.size() && k < cap; ++k) out[k] = v[k];
  return v.size();
}

// reference.rs:25-35: brute-force density with given h (ascending j, all terms).
void or_sph_reference_density(size_t n, const double* pos, const double* mass, const double* h, double* rho_out) {
  for (size_t i = 0; i < n; ++i) {
    double rho = 0.0;
    for (size_t j = 0; j < n; ++j) rho += mass[j] * w(length(sub(ld(pos, i), ld(pos, j))), h[i]);
    rho_out[i] = rho;
  }
}

// density.rs:60-80: grid-accelerated density with caller-supplied h.
void or_sph_density_fixed(size_t n, const double* pos, const double* mass, const double* h, double* rho_out) {
  if (n == 0) return;
  double h_max = 0.0;
  for (size_t i = 0; i < n; ++i) h_max = fmax_(h_max, h[i]);
  HashGrid grid(pos, n, kSupport * h_max);
  std::vector<uint32_t> ngb;
  for (size_t i = 0; i < n; ++i) {
    grid.within(pos, ld(pos, i), kSupport * h[i], ngb);
    double rho = 0.0;
    for (uint32_t j : ngb) rho += mass[j] * w(length(sub(ld(pos, i), ld(pos, j))), h[i]);
    rho_out[i] = rho;
  }
}

// density.rs:86-96 / 303-327: adaptive-h density; h_init (nullable) seeds the brackets.
void or_sph_density_adaptive(size_t n, const double* pos, const double* mass, double n_ngb, double h_tol_rel,
                             const double* h_init, double* rho_out, double* h_out, int threads) {
  if (n == 0) return;
  DensitySetup s(pos, mass, n, n_ngb, h_tol_rel);
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64)
  for (size_t i = 0; i < n; ++i) s.solve_one(i, h_init ? h_init + i : nullptr, rho_out + i, h_out + i);
}

// The occupancy seeds and cap of DensitySetup::new (density.rs:166-220), for tests of
// the seed stage: seeds_out[n], scalars_out = {s_est, h_seed, h_cap, occ_bin}.
void or_sph_density_seeds(size_t n, const double* pos, double n_ngb, double* seeds_out, double* scalars_out) {
  if (n == 0) return;
  DensitySetup s(pos, nullptr, n, n_ngb, 1e-3);
  for (size_t i = 0; i < n; ++i) seeds_out[i] = s.seeds[i];
  scalars_out[0] = s.h_cap;
}

// forces.rs:339-379 (hydro_accel_and_dudt): eos 0 isothermal (eos_param = c_s), 1
// adiabatic (eos_param = gamma, reads u).
void or_sph_hydro(size_t n, const double* pos, const double* vel, const double* mass, const double* rho,
                  const double* h, const double* u, int eos, double eos_param, double alpha, double beta,
                  double visc_eps2, double* acc_out, double* dudt_out, int threads) {
  if (n == 0) return;
  Hydro H;
  H.pos = pos;
  H.vel = vel;
  H.mass = mass;
  H.rho = rho;
  H.h = h;
  H.u = u;
  H.n = n;
  H.adiabatic = eos;
  H.c_s = eos == 0 ? eos_param : 0.0;
  H.gamma = eos == 1 ? eos_param : 0.0;
  H.alpha = alpha;
  H.beta = beta;
  H.visc_eps2 = visc_eps2;
  H.setup();
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64)
  for (size_t i = 0; i < n; ++i) {
    D3 a;
    double d;
    H.force_one(i, &a, &d);
    acc_out[3 * i] = a.x;
    acc_out[3 * i + 1] = a.y;
    acc_out[3 * i + 2] = a.z;
    if (dudt_out) dudt_out[i] = d;
  }
}

// cfl.rs per-particle bound over a gas subset with caller-supplied h.
void or_sph_cfl_given_h(size_t n_gas, const double* gpos, const double* gvel, const double* h, const double* u,
                        int eos, double eos_param, double c_cfl, double* dt_out, int threads) {
  if (n_gas == 0) return;
  cfl_per_particle(n_gas, gpos, gvel, h, u, eos, eos == 0 ? eos_param : 0.0, eos == 1 ? eos_param : 0.0, c_cfl,
                   dt_out, threads);
}

// cfl.rs:49-125 max_stable_dt (and :134-185 per particle, state-indexed, +inf for
// non-gas rows, when dt_state_out is non-null): cold-start density over the gas.
double or_sph_max_stable_dt(size_t n, const double* pos, const double* vel, const double* mass,
                            const uint8_t* kind, const double* u, int eos, double eos_param, double n_ngb,
                            double h_tol_rel, double c_cfl, double* dt_state_out, int threads) {
  const double inf = std::numeric_limits<double>::infinity();
  if (dt_state_out)
    for (size_t i = 0; i < n; ++i) dt_state_out[i] = inf;
  std::vector<size_t> gas;
  gather_gas(n, kind, gas);
  if (gas.empty()) return inf;
  std::vector<double> gpos, gvel, gmass, gu;
  subset3(pos, gas, gpos);
  subset3(vel, gas, gvel);
  subset1(mass, gas, gmass);
  subset1(u, gas, gu);
  const size_t ng = gas.size();
  std::vector<double> rho(ng), h(ng), dt(ng);
  or_sph_density_adaptive(ng, gpos.data(), gmass.data(), n_ngb, h_tol_rel, nullptr, rho.data(), h.data(), threads);
  cfl_per_particle(ng, gpos.data(), gvel.data(), h.data(), gu.data(), eos, eos == 0 ? eos_param : 0.0,
                   eos == 1 ? eos_param : 0.0, c_cfl, dt.data(), threads);
  double min_dt = inf;
  for (size_t k = 0; k < ng; ++k) {
    min_dt = fmin_(min_dt, dt[k]);
    if (dt_state_out) dt_state_out[gas[k]] = dt[k];
  }
  return min_dt;
}

// gravity_sph.rs:172-207 GravitySph::accelerations. h_hint (n_gas entries, or null)
// is the warm start, overwritten with this call's h when h_hint_valid says it held one
// (*h_hint_valid set to 1 after the call). g <= 0 runs hydro only (gravity off).
int or_gravity_sph_accelerations(size_t n, const double* pos, const double* vel, const double* mass,
                                 const uint8_t* kind, const double* u, double g, double softening, double theta,
                                 int eos, double eos_param, double alpha, double beta, double visc_eps2,
                                 double n_ngb, double h_tol_rel, double* h_hint, int* h_hint_valid,
                                 double* rho_out, double* acc_out, int threads) {
  if (n == 0) return 0;
  if (g > 0.0)
    or_lbvh_accelerations(n, pos, mass, g, softening, theta, acc_out, threads, nullptr);
  else
    for (size_t i = 0; i < 3 * n; ++i) acc_out[i] = 0.0;
  std::vector<size_t> gas;
  gather_gas(n, kind, gas);
  if (gas.empty()) {
    if (h_hint_valid) *h_hint_valid = 0;
    return 0;
  }
  std::vector<double> gpos, gvel, gmass, gu;
  subset3(pos, gas, gpos);
  subset3(vel, gas, gvel);
  subset1(mass, gas, gmass);
  subset1(u, gas, gu);
  const size_t ng = gas.size();
  std::vector<double> rho(ng), h(ng), a(3 * ng);
  const bool warm = h_hint && h_hint_valid && *h_hint_valid;
  or_sph_density_adaptive(ng, gpos.data(), gmass.data(), n_ngb, h_tol_rel, warm ? h_hint : nullptr, rho.data(),
                          h.data(), threads);
  or_sph_hydro(ng, gpos.data(), gvel.data(), gmass.data(), rho.data(), h.data(), gu.data(), eos, eos_param, alpha,
               beta, visc_eps2, a.data(), nullptr, threads);
  for (size_t k = 0; k < ng; ++k)
    for (int c = 0; c < 3; ++c) acc_out[3 * gas[k] + c] = acc_out[3 * gas[k] + c] + a[3 * k + c];
  if (h_hint) {
    for (size_t k = 0; k < ng; ++k) h_hint[k] = h[k];
    if (h_hint_valid) *h_hint_valid = 1;
  }
  if (rho_out)
    for (size_t k = 0; k < ng; ++k) rho_out[k] = rho[k];
  return 0;
}

// divergence.rs:34-72 velocity_divergence over a gas subset with given rho / h.
void or_sph_velocity_divergence(size_t n, const double* pos, const double* vel, const double* mass, const double* rho,
                                const double* h, double* div_out, int threads) {
  if (n == 0) return;
  double h_max = 0.0;
  for (size_t i = 0; i < n; ++i) h_max = fmax_(h_max, h[i]);
  HashGrid grid(pos, n, kSupport * h_max);
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64)
  for (size_t i = 0; i < n; ++i) {
    std::vector<uint32_t> ngb;
    grid.within(pos, ld(pos, i), kSupport * h[i], ngb);
    double sum = 0.0;
    for (uint32_t j : ngb) {
      if (j == i) continue;
      const D3 gw = grad_w(sub(ld(pos, i), ld(pos, j)), h[i]);
      sum += mass[j] * dot(sub(ld(vel, j), ld(vel, i)), gw);
    }
    div_out[i] = sum / rho[i];
  }
}

// gravity_sph.rs:353-382 GravitySph::sf_fields: cold-start density over the gas and the
// divergence gather, scattered to the state's rows (collisionless rows 0, 0).
void or_sph_sf_fields(size_t n, const double* pos, const double* vel, const double* mass, const uint8_t* kind,
                      double n_ngb, double h_tol_rel, double* rho_out, double* div_out, int threads) {
  for (size_t i = 0; i < n; ++i) rho_out[i] = div_out[i] = 0.0;
  std::vector<size_t> gas;
  gather_gas(n, kind, gas);
  if (gas.empty()) return;
  std::vector<double> gpos, gvel, gmass;
  subset3(pos, gas, gpos);
  subset3(vel, gas, gvel);
  subset1(mass, gas, gmass);
  const size_t ng = gas.size();
  std::vector<double> rho(ng), h(ng), dv(ng);
  or_sph_density_adaptive(ng, gpos.data(), gmass.data(), n_ngb, h_tol_rel, nullptr, rho.data(), h.data(), threads);
  or_sph_velocity_divergence(ng, gpos.data(), gvel.data(), gmass.data(), rho.data(), h.data(), dv.data(), threads);
  for (size_t k = 0; k < ng; ++k) {
    rho_out[gas[k]] = rho[k];
    div_out[gas[k]] = dv[k];
  }
}

// cfl.rs:195-228 coupled_pairs: gas pairs (gas[a], gas[b]), a < b, with 0 < r <
// 2 max(h_a, h_b) after a cold density solve, in ascending (a, b). Writes up to cap pairs
// (2 per pair) and returns the count.
size_t or_sph_coupled_pairs(size_t n, const double* pos, const double* mass, const uint8_t* kind, double n_ngb,
                            double h_tol_rel, uint64_t* pairs_out, size_t cap, int threads) {
  std::vector<size_t> gas;
  gather_gas(n, kind, gas);
  if (gas.empty()) return 0;
  std::vector<double> gpos, gmass;
  subset3(pos, gas, gpos);
  subset1(mass, gas, gmass);
  const size_t ng = gas.size();
  std::vector<double> rho(ng), h(ng);
  or_sph_density_adaptive(ng, gpos.data(), gmass.data(), n_ngb, h_tol_rel, nullptr, rho.data(), h.data(), threads);
  double h_max = 0.0;
  for (size_t k = 0; k < ng; ++k) h_max = fmax_(h_max, h[k]);
  HashGrid grid(gpos.data(), ng, kSupport * h_max);
  size_t count = 0;
  std::vector<uint32_t> ngb;
  for (size_t a = 0; a < ng; ++a) {
    grid.within(gpos.data(), ld(gpos.data(), a), kSupport * h_max, ngb);
    for (uint32_t b : ngb) {
      if (b <= a) continue;
      const double r = length(sub(ld(gpos.data(), a), ld(gpos.data(), b)));
      if (r > 0.0 && r < kSupport * fmax_(h[a], h[b])) {
        if (count < cap) {
          pairs_out[2 * count] = gas[a];
          pairs_out[2 * count + 1] = gas[b];
        }
        ++count;
      }
    }
  }
  return count;
}

// gravity_sph.rs:247-286 GravitySph::accelerations_active (fresh gravity on all n), with
// :101-150 active_gas: h_scratch (shared with or_gravity_sph_accelerations' h_hint) and
// rho_scratch hold the persistent gas-subset scratch; a scratch that is not set forces a
// refresh of every gas particle (warm-started from h when h is set). Density
// (density.rs:118-140, density_adaptive_active) and hydro (forces.rs:188-217,
// hydro_accel_and_dudt_active) run for the active gas targets only, reading the inactive
// neighbours' rho / h from the scratch.
int or_gravity_sph_accelerations_active(size_t n, const double* pos, const double* vel, const double* mass,
                                        const uint8_t* kind, const double* u, double g, double softening,
                                        double theta, int eos, double eos_param, double alpha, double beta,
                                        double visc_eps2, double n_ngb, double h_tol_rel, double* h_scratch,
                                        int* h_valid, double* rho_scratch, int* rho_valid, size_t n_active,
                                        const uint32_t* active, double* acc_out, double* dudt_out, int threads) {
  if (n == 0) return 0;
  // accel_and_dudt_active (gravity_sph.rs:288-319): du/dt zero on every row, the active
  // gas rows overwritten below
  if (dudt_out)
    for (size_t i = 0; i < n; ++i) dudt_out[i] = 0.0;
  if (g > 0.0)
    or_lbvh_accelerations(n, pos, mass, g, softening, theta, acc_out, threads, nullptr);
  else
    for (size_t i = 0; i < 3 * n; ++i) acc_out[i] = 0.0;
  std::vector<size_t> gas;
  gather_gas(n, kind, gas);
  if (gas.empty()) {
    *h_valid = 0;
    *rho_valid = 0;
    return 0;
  }
  const size_t ng = gas.size();
  std::vector<double> gpos, gvel, gmass, gu;
  subset3(pos, gas, gpos);
  subset3(vel, gas, gvel);
  subset1(mass, gas, gmass);
  subset1(u, gas, gu);
  const bool h_init = !*h_valid, rho_init = !*rho_valid;
  if (h_init)
    for (size_t k = 0; k < ng; ++k) h_scratch[k] = 0.0;
  if (rho_init)
    for (size_t k = 0; k < ng; ++k) rho_scratch[k] = 0.0;
  std::vector<size_t> local;
  if (h_init || rho_init) {
    for (size_t k = 0; k < ng; ++k) local.push_back(k);
  } else {
    std::vector<size_t> g2l(n, SIZE_MAX);
    for (size_t k = 0; k < ng; ++k) g2l[gas[k]] = k;
    for (size_t a = 0; a < n_active; ++a)
      if (g2l[active[a]] != SIZE_MAX) local.push_back(g2l[active[a]]);
  }
  DensitySetup setup(gpos.data(), gmass.data(), ng, n_ngb, h_tol_rel);
  std::vector<double> nr(local.size()), nh(local.size());
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64)
  for (size_t t = 0; t < local.size(); ++t) setup.solve_one(local[t], h_scratch + local[t], &nr[t], &nh[t]);
  for (size_t t = 0; t < local.size(); ++t) {
    rho_scratch[local[t]] = nr[t];
    h_scratch[local[t]] = nh[t];
  }
  Hydro H;
  H.pos = gpos.data();
  H.vel = gvel.data();
  H.mass = gmass.data();
  H.rho = rho_scratch;
  H.h = h_scratch;
  H.u = gu.data();
  H.n = ng;
  H.adiabatic = eos;
  H.c_s = eos == 0 ? eos_param : 0.0;
  H.gamma = eos == 1 ? eos_param : 0.0;
  H.alpha = alpha;
  H.beta = beta;
  H.visc_eps2 = visc_eps2;
  H.setup();
  std::vector<D3> ca(local.size());
  std::vector<double> cd(local.size());
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(dynamic, 64)
  for (size_t t = 0; t < local.size(); ++t) H.force_one(local[t], &ca[t], &cd[t]);
  for (size_t t = 0; t < local.size(); ++t) {
    const size_t i = gas[local[t]];
    acc_out[3 * i] = acc_out[3 * i] + ca[t].x;
    acc_out[3 * i + 1] = acc_out[3 * i + 1] + ca[t].y;
    acc_out[3 * i + 2] = acc_out[3 * i + 2] + ca[t].z;
    if (dudt_out) dudt_out[i] = cd[t];
  }
  *h_valid = 1;
  *rho_valid = 1;
  return 0;
}

// integrator.rs:38-78 driving GravitySph: `steps` KDK steps in place; acc_io and
// primed_io carry the integrator's cached force, h_hint / h_hint_valid the composite's
// warm start (n_gas entries); rho_out (nullable) the last evaluation's gas densities.
int or_kdk_gravity_sph(size_t n, double* pos, double* vel, const double* mass, const uint8_t* kind, const double* u,
                       double g, double softening, double theta, int eos, double eos_param, double alpha,
                       double beta, double visc_eps2, double n_ngb, double h_tol_rel, double* h_hint,
                       int* h_hint_valid, double* rho_out, double* acc_io, int* primed_io, double dt, uint64_t steps,
                       int threads) {
  if (n == 0) return 0;
  for (uint64_t s = 0; s < steps; ++s) {
    if (!*primed_io) {
      or_gravity_sph_accelerations(n, pos, vel, mass, kind, u, g, softening, theta, eos, eos_param, alpha, beta,
                                   visc_eps2, n_ngb, h_tol_rel, h_hint, h_hint_valid, nullptr, acc_io, threads);
      *primed_io = 1;
    }
    const double half = 0.5 * dt;
    for (size_t i = 0; i < 3 * n; ++i) vel[i] = vel[i] + acc_io[i] * half;
    for (size_t i = 0; i < 3 * n; ++i) pos[i] = pos[i] + vel[i] * dt;
    or_gravity_sph_accelerations(n, pos, vel, mass, kind, u, g, softening, theta, eos, eos_param, alpha, beta,
                                 visc_eps2, n_ngb, h_tol_rel, h_hint, h_hint_valid, rho_out, acc_io, threads);
    for (size_t i = 0; i < 3 * n; ++i) vel[i] = vel[i] + acc_io[i] * half;
  }
  return 0;
}

// gpu/tests/gpu_resident_sph.rs:38-96 `gas_star_mix`: a dense gas blob at every
// (1 + n_star/n_gas)-th index inside a wider star field (kind 1 = gas, 0 = stars).
void or_fixture_gas_star_mix(uint64_t seed, size_t n_gas, size_t n_star, double* pos, double* vel, double* mass,
                             uint8_t* kind) {
  uint64_t s = seed | 1;
  auto next = [&s]() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return static_cast<double>(s >> 11) / static_cast<double>(1ull << 53);
  };
  std::vector<double> gp(3 * n_gas), gv(3 * n_gas), gm(n_gas), sp(3 * n_star), sv(3 * n_star), sm(n_star);
  for (size_t k = 0; k < n_gas; ++k) {
    for (int c = 0; c < 3; ++c) gp[3 * k + c] = (next() - 0.5) * 2.0;
    for (int c = 0; c < 3; ++c) gv[3 * k + c] = (next() - 0.5) * 0.1;
    gm[k] = 0.5 + 0.5 * next();
  }
  for (size_t k = 0; k < n_star; ++k) {
    for (int c = 0; c < 3; ++c) sp[3 * k + c] = (next() - 0.5) * 6.0;
    for (int c = 0; c < 3; ++c) sv[3 * k + c] = (next() - 0.5) * 0.1;
    sm[k] = 0.1 + 0.9 * next();
  }
  size_t gi = 0, si = 0, o = 0;
  const size_t take = std::max<size_t>(n_star / std::max<size_t>(n_gas, 1), 1);
  while (gi < n_gas || si < n_star) {
    if (gi < n_gas) {
      for (int c = 0; c < 3; ++c) {
        pos[3 * o + c] = gp[3 * gi + c];
        vel[3 * o + c] = gv[3 * gi + c];
      }
      mass[o] = gm[gi];
      kind[o] = 1;
      ++gi;
      ++o;
    }
    for (size_t t = 0; t < take; ++t) {
      if (si < n_star) {
        for (int c = 0; c < 3; ++c) {
          pos[3 * o + c] = sp[3 * si + c];
          vel[3 * o + c] = sv[3 * si + c];
        }
        mass[o] = sm[si];
        kind[o] = 0;
        ++si;
        ++o;
      }
    }
  }
}

// The reference SPH tests' `random_points` (solvers/tests/sph_forces.rs:18-29,
// sph_cfl.rs:10-21): offset = 0.5 gives (u - 0.5) * scale, offset = 0 gives u * scale.
void or_fixture_sph_points(uint64_t seed, size_t n, double scale, double offset, double* pos) {
  uint64_t s = seed | 1;
  auto next = [&s]() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return static_cast<double>(s >> 11) / static_cast<double>(1ull << 53);
  };
  for (size_t i = 0; i < n; ++i) {
    const double a = next() - offset;
    const double b = next() - offset;
    const double c = next() - offset;
    pos[3 * i] = a * scale;
    pos[3 * i + 1] = b * scale;
    pos[3 * i + 2] = c * scale;
  }
}

}  // extern "C"
