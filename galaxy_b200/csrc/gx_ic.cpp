// gx_ic.cpp -- seeded initial conditions used as the workloads of the gravity step.
//
// gx_ic_plummer restates Plummer::sample of the reference (ic/src/plummer.rs:94-175:
// SplitMix64 stream, Aarseth-Henon-Wielen radius inversion, rejection-sampled
// speed, isotropic directions, recentring), so the N=16,384 seed-0 sphere is the
// reference's own realisation (the same libm calls: pow, sqrt, cos, sin).
//
// The galaxy generators are this project's own synthetic stand-ins for the
// reference's collision scenarios (ic/src/disk_collision.rs, ic/src/encounter.rs):
// per galaxy an NFW halo (60% of particles), an exponential disk (35%, scale
// length Rd = 1, sech^2 scale height z0 = 0.1, circular velocity plus 10% Gaussian
// dispersion) and a Hernquist bulge (5%, a = 0.2); halo and bulge velocities are
// isotropic Gaussians with the Jeans dispersion of each component in the total
// (spherically averaged) potential. The pair is placed on a Kepler orbit of
// eccentricity 1 with the given pericentre (orbit in the x-y plane, pericentre on
// +x), each disk tilted about the x axis by its inclination.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/galaxy_b200.h"

namespace {

struct SplitMix64 {
  uint64_t state;
  explicit SplitMix64(uint64_t seed) : state(seed) {}
  uint64_t next_u64() {
    state += 0x9E3779B97F4A7C15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double next_f64() { return static_cast<double>(next_u64() >> 11) / static_cast<double>(1ull << 53); }
  double gauss() {
    double u1 = next_f64(), u2 = next_f64();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

const double kTau = 6.283185307179586;

void random_direction(SplitMix64& r, double out[3]) {
  double ct = 2.0 * r.next_f64() - 1.0;
  double st = std::sqrt(std::fmax(1.0 - ct * ct, 0.0));
  double phi = kTau * r.next_f64();
  out[0] = st * std::cos(phi);
  out[1] = st * std::sin(phi);
  out[2] = ct;
}

void recenter(double* pos, double* vel, const double* mass, size_t a, size_t b) {
  double mt = 0, cp[3] = {0, 0, 0}, cv[3] = {0, 0, 0};
  for (size_t i = a; i < b; ++i) {
    mt += mass[i];
    for (int c = 0; c < 3; ++c) {
      cp[c] += mass[i] * pos[3 * i + c];
      cv[c] += mass[i] * vel[3 * i + c];
    }
  }
  for (int c = 0; c < 3; ++c) {
    cp[c] /= mt;
    cv[c] /= mt;
  }
  for (size_t i = a; i < b; ++i)
    for (int c = 0; c < 3; ++c) {
      pos[3 * i + c] -= cp[c];
      vel[3 * i + c] -= cv[c];
    }
}

// ---- one composite galaxy of total mass mg, particles [a, b) -------------------------
struct Galaxy {
  double mg;
  double m_halo, m_disk, m_bulge;
  double rs = 3.0, rt = 30.0;       // NFW scale and truncation radius
  double rd = 1.0, z0 = 0.1, rdmax = 10.0;
  double ab = 0.2, rbmax = 6.0;     // bulge scale and truncation
  double nfw_norm;
  explicit Galaxy(double m) : mg(m), m_halo(0.8 * m), m_disk(0.15 * m), m_bulge(0.05 * m) {
    nfw_norm = nfw_mu(rt / rs);
  }
  static double nfw_mu(double x) { return std::log1p(x) - x / (1.0 + x); }
  double halo_menc(double r) const { return r >= rt ? m_halo : m_halo * nfw_mu(r / rs) / nfw_norm; }
  double bulge_menc(double r) const {
    double f = (r / (r + ab)) * (r / (r + ab));
    double fmax = (rbmax / (rbmax + ab)) * (rbmax / (rbmax + ab));
    return m_bulge * std::min(f / fmax, 1.0);
  }
  double disk_menc(double r) const {  // cylindrical mass inside R = r (spherical approximation)
    double x = std::min(r, rdmax) / rd;
    double xm = rdmax / rd;
    return m_disk * (1.0 - (1.0 + x) * std::exp(-x)) / (1.0 - (1.0 + xm) * std::exp(-xm));
  }
  double menc(double r) const { return halo_menc(r) + bulge_menc(r) + disk_menc(r); }
  double vcirc(double r) const {
    double rr = std::sqrt(r * r + 0.01 * 0.01);
    return std::sqrt(menc(r) / rr);
  }
};

// Isotropic Jeans dispersion sigma(r) of a component with enclosed-mass profile
// m_c(r) in the galaxy potential, tabulated on a log grid.
struct JeansTable {
  std::vector<double> r, s;
  template <class F>
  void build(const Galaxy& g, F mc, double rmin, double rmax) {
    const int n = 400;
    r.resize(n);
    s.resize(n);
    std::vector<double> rho(n);
    for (int i = 0; i < n; ++i) r[i] = rmin * std::pow(rmax / rmin, i / double(n - 1));
    for (int i = 0; i < n; ++i) {
      double r0 = r[i] * 0.999, r1 = r[i] * 1.001;
      rho[i] = std::max((mc(r1) - mc(r0)) / (4.0 / 3.0 * M_PI * (r1 * r1 * r1 - r0 * r0 * r0)), 1e-300);
    }
    double acc = 0.0;
    s[n - 1] = 0.0;
    for (int i = n - 2; i >= 0; --i) {
      double f0 = rho[i] * g.menc(r[i]) / (r[i] * r[i]);
      double f1 = rho[i + 1] * g.menc(r[i + 1]) / (r[i + 1] * r[i + 1]);
      acc += 0.5 * (f0 + f1) * (r[i + 1] - r[i]);
      s[i] = std::sqrt(acc / rho[i]);
    }
  }
  double at(double x) const {
    if (x <= r.front()) return s.front();
    if (x >= r.back()) return s.back();
    size_t k = std::upper_bound(r.begin(), r.end(), x) - r.begin();
    double t = (x - r[k - 1]) / (r[k] - r[k - 1]);
    return s[k - 1] + t * (s[k] - s[k - 1]);
  }
};

// Inverse of a monotone CDF on [lo, hi], tabulated once and interpolated linearly.
struct InverseCdf {
  std::vector<double> u, x;
  template <class F>
  InverseCdf(F cdf, double lo, double hi, int n = 8192) {
    x.resize(n);
    u.resize(n);
    for (int i = 0; i < n; ++i) {
      const double t = static_cast<double>(i) / (n - 1);
      x[i] = lo + (hi - lo) * t * t;  // denser near the centre, where the mass is
      u[i] = cdf(x[i]);
    }
  }
  double operator()(double v) const {
    if (v <= u.front()) return x.front();
    if (v >= u.back()) return x.back();
    const size_t k = std::upper_bound(u.begin(), u.end(), v) - u.begin();
    const double t = (v - u[k - 1]) / std::max(u[k] - u[k - 1], 1e-300);
    return x[k - 1] + t * (x[k] - x[k - 1]);
  }
};

void sample_galaxy(const Galaxy& g, SplitMix64& rng, double* pos, double* vel, double* mass, size_t a, size_t b,
                   bool with_bulge) {
  const size_t n = b - a;
  size_t nh = static_cast<size_t>(0.60 * n);
  size_t nb = with_bulge ? static_cast<size_t>(0.05 * n) : 0;
  size_t nd = n - nh - nb;
  const double mh = g.m_halo / nh;
  const double md = (with_bulge ? g.m_disk : g.m_disk + g.m_bulge) / nd;
  const double mb = nb ? g.m_bulge / nb : 0.0;
  JeansTable jh, jb;
  jh.build(g, [&](double r) { return g.halo_menc(r); }, 1e-3, g.rt);
  if (nb) jb.build(g, [&](double r) { return g.bulge_menc(r); }, 1e-4, g.rbmax);
  size_t i = a;
  // halo
  const InverseCdf halo_r([&](double x) { return Galaxy::nfw_mu(x) / g.nfw_norm; }, 0.0, g.rt / g.rs);
  for (size_t k = 0; k < nh; ++k, ++i) {
    double r = halo_r(rng.next_f64()) * g.rs, d[3];
    random_direction(rng, d);
    double sig = jh.at(r);
    for (int c = 0; c < 3; ++c) {
      pos[3 * i + c] = r * d[c];
      vel[3 * i + c] = sig * rng.gauss();
    }
    mass[i] = mh;
  }
  // disk
  const double xm = g.rdmax / g.rd;
  const double cdf_max = 1.0 - (1.0 + xm) * std::exp(-xm);
  const InverseCdf disk_r([&](double x) { return (1.0 - (1.0 + x) * std::exp(-x)) / cdf_max; }, 0.0, xm);
  for (size_t k = 0; k < nd; ++k, ++i) {
    double R = disk_r(rng.next_f64()) * g.rd;
    double phi = kTau * rng.next_f64();
    double w = 2.0 * rng.next_f64() - 1.0;
    w = std::max(-0.999999, std::min(0.999999, w));
    double z = g.z0 * std::atanh(w);
    double vc = g.vcirc(std::sqrt(R * R + z * z));
    double sg = 0.1 * vc;
    double vr = sg * rng.gauss(), vp = vc + sg * rng.gauss(), vz = sg * rng.gauss();
    double cp = std::cos(phi), sp = std::sin(phi);
    pos[3 * i] = R * cp;
    pos[3 * i + 1] = R * sp;
    pos[3 * i + 2] = z;
    vel[3 * i] = vr * cp - vp * sp;
    vel[3 * i + 1] = vr * sp + vp * cp;
    vel[3 * i + 2] = vz;
    mass[i] = md;
  }
  // bulge
  const double fmax = (g.rbmax / (g.rbmax + g.ab)) * (g.rbmax / (g.rbmax + g.ab));
  for (size_t k = 0; k < nb; ++k, ++i) {
    double X = fmax * rng.next_f64();
    double sx = std::sqrt(X);
    double r = g.ab * sx / (1.0 - sx), d[3];
    random_direction(rng, d);
    double sig = jb.at(r);
    for (int c = 0; c < 3; ++c) {
      pos[3 * i + c] = r * d[c];
      vel[3 * i + c] = sig * rng.gauss();
    }
    mass[i] = mb;
  }
  recenter(pos, vel, mass, a, b);
}

void rotate_x(double* v, size_t a, size_t b, double incl) {
  const double c = std::cos(incl), s = std::sin(incl);
  for (size_t i = a; i < b; ++i) {
    double y = v[3 * i + 1], z = v[3 * i + 2];
    v[3 * i + 1] = c * y - s * z;
    v[3 * i + 2] = s * y + c * z;
  }
}

}  // namespace

extern "C" {

int gx_ic_plummer(size_t n, uint64_t seed, double g, double total_mass, double scale_radius, double* pos,
                  double* vel, double* mass) {
  if (n == 0) return GX_OK;
  if (!pos || !vel || !mass || !(g > 0) || !(total_mass > 0) || !(scale_radius > 0)) return GX_ERR_INVALID_ARG;
  SplitMix64 rng(seed);
  const double a = scale_radius;
  const double m_each = total_mass / static_cast<double>(n);
  const double v_esc_coeff = std::sqrt(2.0 * g * total_mass);
  for (size_t i = 0; i < n; ++i) {
    double x = rng.next_f64();
    double r = a / std::sqrt(std::pow(x, -2.0 / 3.0) - 1.0);
    double d[3];
    random_direction(rng, d);
    for (int c = 0; c < 3; ++c) pos[3 * i + c] = d[c] * r;
    double q;
    for (;;) {
      q = rng.next_f64();
      double height = 0.1 * rng.next_f64();
      if (height < q * q * std::pow(1.0 - q * q, 3.5)) break;
    }
    double v_esc = v_esc_coeff * std::pow(r * r + a * a, -0.25);
    random_direction(rng, d);
    for (int c = 0; c < 3; ++c) vel[3 * i + c] = d[c] * (q * v_esc);
  }
  const double inv_n = 1.0 / static_cast<double>(n);
  double mp[3] = {0, 0, 0}, mv[3] = {0, 0, 0};
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      mp[c] = mp[c] + pos[3 * i + c];
      mv[c] = mv[c] + vel[3 * i + c];
    }
  for (int c = 0; c < 3; ++c) {
    mp[c] = mp[c] * inv_n;
    mv[c] = mv[c] * inv_n;
  }
  for (size_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) {
      pos[3 * i + c] = pos[3 * i + c] - mp[c];
      vel[3 * i + c] = vel[3 * i + c] - mv[c];
    }
    mass[i] = m_each;
  }
  return GX_OK;
}

int gx_ic_disk_galaxy(size_t n, uint64_t seed, double* pos, double* vel, double* mass) {
  if (n == 0) return GX_OK;
  if (n < 20 || !pos || !vel || !mass) return GX_ERR_INVALID_ARG;
  SplitMix64 rng(seed);
  Galaxy g(1.0);
  sample_galaxy(g, rng, pos, vel, mass, 0, n, true);
  return GX_OK;
}

int gx_ic_collision(size_t n_total, uint64_t seed, double mass_ratio, double pericentre, double incl1_deg,
                    double incl2_deg, double* pos, double* vel, double* mass) {
  if (n_total < 40 || !pos || !vel || !mass || !(mass_ratio > 0) || !(pericentre > 0)) return GX_ERR_INVALID_ARG;
  SplitMix64 rng(seed);
  const double m1 = 1.0, m2 = mass_ratio;
  size_t n1 = static_cast<size_t>(std::llround(static_cast<double>(n_total) * m1 / (m1 + m2)));
  n1 = std::max<size_t>(20, std::min(n1, n_total - 20));
  Galaxy g1(m1), g2(m2);
  sample_galaxy(g1, rng, pos, vel, mass, 0, n1, true);
  sample_galaxy(g2, rng, pos, vel, mass, n1, n_total, true);
  const double d2r = M_PI / 180.0;
  rotate_x(pos, 0, n1, incl1_deg * d2r);
  rotate_x(vel, 0, n1, incl1_deg * d2r);
  rotate_x(pos, n1, n_total, incl2_deg * d2r);
  rotate_x(vel, n1, n_total, incl2_deg * d2r);
  // Parabolic Kepler orbit (e = 1), incoming branch, pericentre on +x, x-y plane.
  const double mu = m1 + m2, e = 1.0, rp = pericentre;
  const double r0 = std::max(5.0 * rp, 30.0);
  const double p = rp * (1.0 + e);
  const double h = std::sqrt(mu * p);
  const double cnu = std::max(-1.0, std::min(1.0, (p / r0 - 1.0) / e));
  const double nu = -std::acos(cnu);
  const double sn = std::sin(nu), cn = std::cos(nu);
  const double vr = mu / h * e * sn, vt = mu / h * (1.0 + e * cn);
  const double rrel[3] = {r0 * cn, r0 * sn, 0.0};
  const double vrel[3] = {vr * cn - vt * sn, vr * sn + vt * cn, 0.0};
  const double f1 = -m2 / mu, f2 = m1 / mu;
  for (size_t i = 0; i < n_total; ++i) {
    const double f = i < n1 ? f1 : f2;
    for (int c = 0; c < 3; ++c) {
      pos[3 * i + c] += rrel[c] * f;
      vel[3 * i + c] += vrel[c] * f;
    }
  }
  return GX_OK;
}

}  // extern "C"
