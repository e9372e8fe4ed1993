// gx_sph.cu -- SPH on the gas subset: adaptive-h density, hydro force, CFL bound,
// velocity divergence and coupled pairs.
//
// Reference (file:line in the galaxy project):
//   solvers/src/sph/kernel.rs:23-53      cubic spline W(r, h) and grad W
//   solvers/src/sph/grid.rs:24-90        uniform grid, cell = floor(x / edge) per axis
//   solvers/src/sph/density.rs:156-289   DensitySetup (bbox, occupancy seeds, h cap) and
//                                        solve_one (bracket, expand, shrink, bisection)
//   solvers/src/sph/forces.rs:223-379    HydroCtx::force_one: symmetric P/rho^2 + Monaghan
//                                        viscosity, grad-averaged kernel, du/dt partner
//   solvers/src/sph/cfl.rs:49-228        v_sig,i and dt_i = c_cfl h_i / v_sig,i; coupled pairs
//   solvers/src/sph/divergence.rs:34-72  div v for the star-formation fields
//   solvers/src/sph/gravity_sph.rs       hydro added to the gas rows after gravity; the
//                                        active-subset pass over a persistent scratch
//   gpu/src/gpu_resident.rs:1537-1565    the resident order: gravity walk, then density,
//                                        hydro and the scatter-add into the gas rows
//
// Design. Every stage is FP64 and keeps the reference's per-pair operation order (this
// file is compiled without FMA contraction). The gas is binned into uniform grids whose
// cells are hashed into T = 2^k buckets; a stable radix sort by bucket (the library's
// onesweep sort) makes every bucket a contiguous run of cell-sorted copies of the gas
// (positions + mass, cell coordinates), so a query reads whole runs. A bucket may also
// hold another cell's particles: a bucket of one cell is matched against the queried cell
// once, a mixed bucket particle by particle, so each particle is seen once. Cell
// coordinates are clamped to the int32 range (monotone, so a clamped query box still
// covers its ball). One warp serves one target: its lanes walk the query box's buckets
// 32 at a time as one flattened list. The density warp keeps its candidates (radius,
// sorted slot) in shared memory and evaluates every bisection step from there (streaming
// the box again only when more than kCandCap candidates fall inside). It gathers a ball
// of 2.5 x the bracket seed instead of the reference's 2 x hi = 4 x seed: a comparison
// whose count needs a wider ball is settled by the lower bound of the gathered part when
// that clears n_ngb, else the gather widens first, so every comparison is the reference's.
// The hydro warp lists the neighbours that pass a support test, then runs the pair
// arithmetic 32 pairs at a time. Sums are lane-strided and reduced by a fixed shuffle
// tree, so results are deterministic; against the reference's ascending serial sums they
// differ by rounding only. The CFL bound is a max over pairs and a min over targets, and
// the coupled pairs a set, so both are exact given the same h.
#include <cmath>
#include <cstring>
#include <mutex>

#include "gx_sph.h"

namespace gx {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kFourThirdsPi = 4.0 * kPi / 3.0;  // (4 pi / 3), rounded as the reference's
constexpr int kSphThreads = 128;                  // one target per warp
constexpr int kSphWarps = kSphThreads / 32;
constexpr int kDensThreads = 256;                 // density: one target per warp, 8 a block
constexpr int kDensWarps = kDensThreads / 32;
constexpr int kCandCap = 512;                     // density candidates cached per warp
constexpr double kLowerBoundMargin = 1.0 + 1e-10; // a partial count this far above n_ngb decides
constexpr int kPairCap = 128;                     // hydro: neighbour slots listed per warp
constexpr uint32_t kBoxAxisMax = 1u << 10;        // a query box wider than this scans all
constexpr uint32_t kBoxCellsMax = 1u << 15;       //   gas instead of its cells
constexpr int kLoopCap = 512;                     // bound on every root-find loop
constexpr int kFlat = 256;
constexpr unsigned kFull = 0xffffffffu;

struct GridDev {
  const double* cell;
  uint32_t tmask, n;
  const uint32_t* start;
  const uint32_t* end;
  const uint32_t* mixed;  // bit per bucket: it holds more than one cell
  const double4* sp;
  const int4* sc;
};

GridDev view(const SphState& s, int g) {
  GridDev d;
  const SphScalars* sc = s.sc;
  d.cell = g == 0 ? &sc->occ_cell : (g == 1 ? &sc->dens_cell : &sc->hydro_cell);
  d.tmask = (1u << s.tbits) - 1u;
  d.n = static_cast<uint32_t>(s.n_gas);
  d.start = s.grid[g].start;
  d.end = s.grid[g].end;
  d.mixed = s.grid[g].mixed;
  d.sp = s.grid[g].sp;
  d.sc = s.grid[g].sc;
  return d;
}

// kernel.rs:27-38, W(r, h), with its normalisation 1 / (pi h^3) computed once per h by
// the caller (the same bits: it depends on h only).
__device__ __forceinline__ double sph_w_n(double r, double h, double norm) {
  const double q = r / h;
  if (q < 1.0) return norm * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
  if (q < 2.0) {
    const double t = 2.0 - q;
    return norm * 0.25 * t * t * t;
  }
  return 0.0;
}

__device__ __forceinline__ double sph_norm(double h) { return 1.0 / (kPi * h * h * h); }

// kernel.rs:40-53 with r = |r_ij| and the normalisation already computed; false when
// the gradient is zero.
__device__ __forceinline__ bool sph_grad(double rx, double ry, double rz, double r, double h, double norm, double& gx,
                                        double& gy, double& gz) {
  const double q = r / h;
  if (r == 0.0 || q >= 2.0) {
    gx = gy = gz = 0.0;
    return false;
  }
  double dp;
  if (q < 1.0) {
    dp = -3.0 * q + 2.25 * q * q;
  } else {
    const double t = 2.0 - q;
    dp = -0.75 * t * t;
  }
  const double s = norm * dp / (h * r);
  gx = rx * s;
  gy = ry * s;
  gz = rz * s;
  return true;
}

// floor(v / cell) clamped to int32 (NaN -> 0, as Rust's saturating cast).
__device__ __forceinline__ int cell_coord(double v, double cell) {
  const double f = floor(v / cell);
  if (!(f == f)) return 0;
  if (f >= 2147483647.0) return 2147483647;
  if (f <= -2147483648.0) return -2147483647 - 1;
  return static_cast<int>(f);
}

__device__ __forceinline__ uint32_t cell_hash(int x, int y, int z) {
  uint32_t h = static_cast<uint32_t>(x) * 0x9E3779B1u;
  h ^= static_cast<uint32_t>(y) * 0x85EBCA77u + 0x7F4A7C15u + (h << 6) + (h >> 2);
  h ^= static_cast<uint32_t>(z) * 0xC2B2AE3Du + 0x165667B1u + (h << 6) + (h >> 2);
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  return __shfl_sync(kFull, v, 0);
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(kFull, v, o));
  return __shfl_sync(kFull, v, 0);
}

// Every gas particle whose cell lies in the query box of centre c and half-width R,
// each exactly once: f(ok, slot) is called by all 32 lanes together (ok false for
// padding lanes and for bucket entries of another cell; a bucket that holds one cell is
// checked once, by its first entry). A box wider than the limits visits every slot instead.
template <class F>
__device__ __forceinline__ void visit_box(const GridDev& g, double cx, double cy, double cz, double R, F&& f) {
  const int lane = threadIdx.x & 31;
  const double cell = *g.cell;
  const int lx = cell_coord(cx - R, cell), hx = cell_coord(cx + R, cell);
  const int ly = cell_coord(cy - R, cell), hy = cell_coord(cy + R, cell);
  const int lz = cell_coord(cz - R, cell), hz = cell_coord(cz + R, cell);
  const long long nx = static_cast<long long>(hx) - lx + 1, ny = static_cast<long long>(hy) - ly + 1,
                  nz = static_cast<long long>(hz) - lz + 1;
  if (nx > kBoxAxisMax || ny > kBoxAxisMax || nz > kBoxAxisMax || nx * ny * nz > kBoxCellsMax) {
    for (uint32_t s0 = 0; s0 < g.n; s0 += 32) f(s0 + lane < g.n, s0 + lane);
    return;
  }
  const uint32_t nc = static_cast<uint32_t>(nx * ny * nz);
  const uint32_t nxu = static_cast<uint32_t>(nx), nxy = static_cast<uint32_t>(nx * ny);
  for (uint32_t c0 = 0; c0 < nc; c0 += 32) {
    const uint32_t c = c0 + lane;
    uint32_t st = 0, cnt = 0, mix = 0;
    int ox = 0, oy = 0, oz = 0;
    if (c < nc) {
      ox = lx + static_cast<int>(c % nxu);
      oy = ly + static_cast<int>((c / nxu) % static_cast<uint32_t>(ny));
      oz = lz + static_cast<int>(c / nxy);
      const uint32_t b = cell_hash(ox, oy, oz) & g.tmask;
      st = g.start[b];
      cnt = g.end[b] - st;
      mix = (g.mixed[b >> 5] >> (b & 31)) & 1u;
      if (cnt && !mix) {  // a bucket of one cell: this cell's, or none of it
        const int4 q = g.sc[st];
        if (q.x != ox || q.y != oy || q.z != oz) cnt = 0;
      }
    }
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t excl = incl - cnt;
    for (uint32_t t0 = 0; t0 < total; t0 += 32) {
      const uint32_t t = t0 + lane;
      // owner lane: the first whose inclusive count exceeds t
      int L = 0;
#pragma unroll
      for (int b = 16; b >= 1; b >>= 1) {
        const uint32_t v = __shfl_sync(kFull, incl, L + b - 1);
        if (t >= v) L += b;
      }
      L = min(L, 31);
      const uint32_t exL = __shfl_sync(kFull, excl, L), stL = __shfl_sync(kFull, st, L);
      const uint32_t mixL = __shfl_sync(kFull, mix, L);
      const int ax = __shfl_sync(kFull, ox, L), ay = __shfl_sync(kFull, oy, L), az = __shfl_sync(kFull, oz, L);
      bool ok = false;
      uint32_t s = 0;
      if (t < total) {
        s = stL + (t - exL);
        ok = true;
        if (mixL) {
          const int4 q = g.sc[s];
          ok = q.x == ax && q.y == ay && q.z == az;
        }
      }
      f(ok, s);
    }
  }
}

// ---- gather, scalars, grids ------------------------------------------------------
__global__ void __launch_bounds__(kFlat) k_sph_gather(uint32_t n_gas, const uint32_t* __restrict__ gas_idx,
                                                      const double* __restrict__ pos, const double* __restrict__ vel,
                                                      const double* __restrict__ mass, const double* __restrict__ gu,
                                                      double4* __restrict__ gp, double4* __restrict__ gv,
                                                      SphScalars* sc, int with_bbox) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t k = blockIdx.x * kFlat + threadIdx.x; k < n_gas; k += gridDim.x * kFlat) {
    const size_t i = gas_idx[k];
    const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    gp[k] = make_double4(x, y, z, mass ? mass[i] : 0.0);
    gv[k] = vel ? make_double4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], gu ? gu[k] : 0.0)
                : make_double4(0.0, 0.0, 0.0, gu ? gu[k] : 0.0);
    lo[0] = fmin(lo[0], x), lo[1] = fmin(lo[1], y), lo[2] = fmin(lo[2], z);
    hi[0] = fmax(hi[0], x), hi[1] = fmax(hi[1], y), hi[2] = fmax(hi[2], z);
  }
  if (!with_bbox) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double a = lo[c], b = hi[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a = fmin(a, __shfl_down_sync(kFull, a, o));
      b = fmax(b, __shfl_down_sync(kFull, b, o));
    }
    if ((threadIdx.x & 31) == 0 && a <= b) {
      atomicMax(&sc->bbox_enc[c], enc_max(-a));
      atomicMax(&sc->bbox_enc[3 + c], enc_max(b));
    }
  }
}

// DensitySetup::new's scalars (density.rs:166-181); s_est from the host when given.
__global__ void k_sph_scalars(uint32_t n_gas, SphScalars* sc) {
  const double lx = -dec_max(sc->bbox_enc[0]), ly = -dec_max(sc->bbox_enc[1]), lz = -dec_max(sc->bbox_enc[2]);
  const double hx = dec_max(sc->bbox_enc[3]), hy = dec_max(sc->bbox_enc[4]), hz = dec_max(sc->bbox_enc[5]);
  const double ex = hx - lx, ey = hy - ly, ez = hz - lz;
  const double diag = sqrt(ex * ex + ey * ey + ez * ez);
  const double vol = ex * ey * ez;
  const double n = static_cast<double>(n_gas);
  double s_est;
  if (sc->s_est_host > 0.0)
    s_est = sc->s_est_host;
  else
    s_est = vol > 0.0 ? cbrt(vol / n) : (diag > 0.0 ? diag / cbrt(n) : 1.0);
  const double h_seed = s_est * sc->seed_scale;
  sc->s_est = s_est;
  sc->h_seed = h_seed;
  sc->h_cap = fmax(64.0 * h_seed, 4.0 * diag);
  sc->occ_cell = 4.0 * s_est;
}

__global__ void __launch_bounds__(kFlat) k_grid_keys(uint32_t n, const double4* __restrict__ gp,
                                                     const double* __restrict__ cellp, uint32_t tmask,
                                                     uint32_t* __restrict__ key, int4* __restrict__ cc) {
  const double cell = *cellp;
  for (uint32_t k = blockIdx.x * kFlat + threadIdx.x; k < n; k += gridDim.x * kFlat) {
    const double4 p = gp[k];
    const int x = cell_coord(p.x, cell), y = cell_coord(p.y, cell), z = cell_coord(p.z, cell);
    key[k] = cell_hash(x, y, z) & tmask;
    cc[k] = make_int4(x, y, z, static_cast<int>(k));
  }
}

__global__ void __launch_bounds__(kFlat) k_grid_fill(uint32_t n, const uint32_t* __restrict__ skey,
                                                     const uint32_t* __restrict__ order, const double4* __restrict__ gp,
                                                     const int4* __restrict__ cc, double4* __restrict__ sp,
                                                     int4* __restrict__ sc, uint32_t* __restrict__ start,
                                                     uint32_t* __restrict__ end, uint32_t* __restrict__ inv) {
  for (uint32_t s = blockIdx.x * kFlat + threadIdx.x; s < n; s += gridDim.x * kFlat) {
    const uint32_t k = order[s];
    if (k >= n) continue;
    sp[s] = gp[k];
    sc[s] = cc[k];
    inv[k] = s;
    const uint32_t b = skey[s];
    if (s == 0 || skey[s - 1] != b) start[b] = s;
    if (s == n - 1 || skey[s + 1] != b) end[b] = s + 1;
  }
}

// Buckets holding more than one cell (their occupancy is counted cell by cell).
__global__ void __launch_bounds__(kFlat) k_grid_mixed(uint32_t n, const uint32_t* __restrict__ skey,
                                                      const int4* __restrict__ sc, const uint32_t* __restrict__ start,
                                                      uint32_t* __restrict__ mixed) {
  for (uint32_t s = blockIdx.x * kFlat + threadIdx.x; s < n; s += gridDim.x * kFlat) {
    const uint32_t b = skey[s];
    const int4 a = sc[s], f = sc[start[b]];
    if (a.x != f.x || a.y != f.y || a.z != f.z) atomicOr(&mixed[b >> 5], 1u << (b & 31));
  }
}

// density.rs:200-211: seeds from the occupancy of each particle's own bin.
__global__ void __launch_bounds__(kFlat) k_sph_seeds(GridDev g, const uint32_t* __restrict__ skey,
                                                     const uint32_t* __restrict__ mixed,
                                                     const double* __restrict__ cbrt_tab, SphScalars* sc,
                                                     double* __restrict__ seeds) {
  const double occ = sc->occ_cell, scale = sc->seed_scale, h_cap = sc->h_cap;
  for (uint32_t s = blockIdx.x * kFlat + threadIdx.x; s < g.n; s += gridDim.x * kFlat) {
    const uint32_t b = skey[s];
    const uint32_t st = g.start[b], en = g.end[b];
    const int4 me = g.sc[s];
    uint32_t c = en - st;
    if (mixed[b >> 5] & (1u << (b & 31))) {
      c = 0;
      for (uint32_t t = st; t < en; ++t) {
        const int4 q = g.sc[t];
        c += (q.x == me.x && q.y == me.y && q.z == me.z) ? 1u : 0u;
      }
    }
    c = max(c, 1u);
    const double cb = c < static_cast<uint32_t>(kSphCbrtTable) ? cbrt_tab[c] : cbrt(static_cast<double>(c));
    const double seed = fmin(occ / cb * scale, h_cap);
    seeds[me.w] = seed;
    const uint32_t e = static_cast<uint32_t>(__double_as_longlong(seed) >> 52) & 2047u;
    atomicAdd(&sc->seed_hist[e], 1u);
  }
}

// The density query cell from the median seed (density.rs:213-217); the cell only sets
// how a query's work divides into buckets, never which particles it finds.
__global__ void k_sph_dens_cell(uint32_t n, SphScalars* sc) {
  uint32_t acc = 0, e = 0;
  const uint32_t half = n / 2 + 1;
  for (; e < 2048; ++e) {
    acc += sc->seed_hist[e];
    if (acc >= half) break;
  }
  const double med = 1.4142135623730951 * ldexp(1.0, static_cast<int>(min(e, 2046u)) - 1023);  // bin centre
  sc->dens_cell = fmax(fmin(2.0 * med, 2.0 * sc->h_seed), 1e-12);
}

__global__ void __launch_bounds__(kFlat) k_sph_hmax(uint32_t n, const double* __restrict__ hs, SphScalars* sc) {
  double m = 0.0;
  for (uint32_t k = blockIdx.x * kFlat + threadIdx.x; k < n; k += gridDim.x * kFlat) m = fmax(m, hs[k]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(kFull, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0)
    atomicMax(&sc->h_max_bits, static_cast<unsigned long long>(__double_as_longlong(m)));
}

// forces.rs:286-293: the gather radius is SUPPORT * h_max; the grid's edge is h_max.
__global__ void k_sph_hydro_cell(SphScalars* sc) {
  const double h_max = __longlong_as_double(static_cast<long long>(sc->h_max_bits));
  sc->h_max = h_max;
  sc->hydro_cell = fmax(h_max, 1e-300);  // queries of radius 2 h_max span 3 to 5 cells an axis
}

// ---- density (density.rs:232-289) -----------------------------------------------------
struct DensArgs {
  GridDev g;
  const SphScalars* sc;
  const double* seeds;
  double* rho;
  double* hs;  // in: warm-start hints (when enabled and valid); out: h
  double n_ngb, tol;
  int warm;
  DevCtl* ctl;
  const uint32_t* targets;  // gas-local targets (nullptr: every gas particle, in grid order)
  uint32_t n_targets;
  const uint32_t* inv;      // gas-local index -> slot of this grid
};

__global__ void __launch_bounds__(kDensThreads) k_sph_density(DensArgs a) {
  __shared__ double s_r[kDensWarps][kCandCap];
  __shared__ uint32_t s_s[kDensWarps][kCandCap];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t w = blockIdx.x * kDensWarps + warp;
  if (w >= (a.targets ? a.n_targets : a.g.n)) return;  // warp-uniform
  double* cr = s_r[warp];
  uint32_t* cs = s_s[warp];
  const uint32_t slot = a.targets ? a.inv[a.targets[w]] : w;
  const double4 xi = a.g.sp[slot];
  const uint32_t k = static_cast<uint32_t>(a.g.sc[slot].w);
  const double h_cap = a.sc->h_cap;
  double seed = a.seeds[k];
  if (a.warm && a.sc->hint_valid) {
    const double hv = a.hs[k];
    if (isfinite(hv) && hv > 0.0) seed = hv;
  }
  double lo = fmin(seed / 2.0, h_cap);
  double hi = fmin(seed * 2.0, h_cap);
  uint32_t ncand = 0;
  bool over = false;
  double Rc = 0.0;

  auto gather = [&](double R) {
    Rc = R;
    ncand = 0;
    const double R2 = R * R;
    visit_box(a.g, xi.x, xi.y, xi.z, R, [&](bool ok, uint32_t s) {
      double r2 = 0.0;
      bool in = false;
      if (ok) {
        const double4 p = a.g.sp[s];
        const double dx = xi.x - p.x, dy = xi.y - p.y, dz = xi.z - p.z;
        r2 = dx * dx + dy * dy + dz * dz;
        in = r2 <= R2;
      }
      const unsigned m = __ballot_sync(kFull, in);
      const uint32_t at = ncand + __popc(m & ((1u << lane) - 1u));
      if (in && at < static_cast<uint32_t>(kCandCap)) {
        cr[at] = r2;
        cs[at] = s;
      }
      ncand += __popc(m);
    });
    over = ncand > static_cast<uint32_t>(kCandCap);
    __syncwarp();
    if (!over) {  // the distances, one pass with every lane busy
      for (uint32_t j = lane; j < ncand; j += 32) cr[j] = sqrt(cr[j]);
      __syncwarp();
    }
  };
  // sum over the candidates of W(r, h), mass-weighted or not
  // Candidates at r >= 2h add exact zeros (r >= 2h gives r / h >= 2 after rounding) and
  // are skipped without the division.
  auto wsum = [&](double h, bool weighted) -> double {
    double acc = 0.0;
    const double two_h = 2.0 * h, norm = sph_norm(h);
    if (!over) {
      for (uint32_t j = lane; j < ncand; j += 32) {
        const double r = cr[j];
        if (r >= two_h) continue;
        const double t = sph_w_n(r, h, norm);
        acc += weighted ? a.g.sp[cs[j]].w * t : t;
      }
    } else {
      const double R2 = Rc * Rc;
      visit_box(a.g, xi.x, xi.y, xi.z, Rc, [&](bool ok, uint32_t s) {
        if (!ok) return;
        const double4 p = a.g.sp[s];
        const double dx = xi.x - p.x, dy = xi.y - p.y, dz = xi.z - p.z;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= R2) {
          const double r = sqrt(r2);
          if (r < two_h) {
            const double t = sph_w_n(r, h, norm);
            acc += weighted ? p.w * t : t;
          }
        }
      });
    }
    return warp_sum(acc);
  };
  auto count = [&](double h) -> double {
    const double s = 2.0 * h;
    return kFourThirdsPi * (s * s * s) * wsum(h, false);
  };
  // The candidates are every particle within Rc of the target. count(h) needs all within
  // 2h; when 2h > Rc the candidates' sum is a lower bound of it (every term is >= 0),
  // which settles "count >= n_ngb" whenever it clears n_ngb by more than any rounding
  // could move it. Otherwise the gather widens to 2h first: the comparisons are the
  // reference's, on a gather that is usually a quarter of its 2 * hi ball.
  auto less = [&](double h) -> bool {  // count(h) < n_ngb
    if (2.0 * h <= Rc) return count(h) < a.n_ngb;
    if (count(h) >= a.n_ngb * kLowerBoundMargin) return false;
    gather(2.0 * h);
    return count(h) < a.n_ngb;
  };
  auto greater = [&](double h) -> bool {  // count(h) > n_ngb
    if (2.0 * h <= Rc) return count(h) > a.n_ngb;
    if (count(h) >= a.n_ngb * kLowerBoundMargin) return true;
    gather(2.0 * h);
    return count(h) > a.n_ngb;
  };

  bool bad = false;
  gather(fmin(2.0 * hi, 2.5 * seed));
  int it = 0;
  while (less(hi) && hi < h_cap) {
    if (++it > kLoopCap) {
      bad = true;
      break;
    }
    hi = fmin(hi * 2.0, h_cap);
  }
  int shrinks = 0;
  while (greater(lo) && shrinks < 60) {
    lo /= 2.0;
    shrinks += 1;
  }
  double h;
  if (less(hi)) {
    h = hi;
  } else if (greater(lo)) {
    h = lo;
  } else {
    it = 0;
    while (hi - lo > a.tol * hi) {
      if (++it > kLoopCap) {
        bad = true;
        break;
      }
      const double mid = 0.5 * (lo + hi);
      if (less(mid))
        lo = mid;
      else
        hi = mid;
    }
    h = 0.5 * (lo + hi);
  }
  if (2.0 * h > Rc) gather(2.0 * h);
  const double rho = wsum(h, true);
  if (lane == 0) {
    a.rho[k] = rho;
    a.hs[k] = h;
    if (bad) raise_err(a.ctl, kErrSphIterations);
  }
}

// Hydro grid order copies of each particle's velocity and h, and its per-particle
// closure terms: rho, term = P / rho^2 (cs2 / rho, or (gamma - 1) u / rho), the kernel
// normalisation 1 / (pi h^3) and the sound speed (forces.rs:233-255, the same
// expressions as the pair loop would evaluate, so the same bits).
__global__ void __launch_bounds__(kFlat) k_sph_pack(uint32_t n, const int4* __restrict__ sc,
                                                    const double4* __restrict__ gv, const double* __restrict__ hs,
                                                    const double* __restrict__ rho, int adiabatic, double c_s,
                                                    double gamma, double4* __restrict__ sv,
                                                    double4* __restrict__ sa, SphScalars* scal) {
  const double cs2 = c_s * c_s;
  for (uint32_t s = blockIdx.x * kFlat + threadIdx.x; s < n; s += gridDim.x * kFlat) {
    const uint32_t k = static_cast<uint32_t>(sc[s].w);
    const double4 v = gv[k];
    const double h = hs[k], r = rho[k];
    sv[s] = make_double4(v.x, v.y, v.z, h);
    const double term = adiabatic ? (gamma - 1.0) * v.w / r : cs2 / r;
    const double cs = adiabatic ? sqrt(gamma * (gamma - 1.0) * v.w) : c_s;
    sa[s] = make_double4(r, term, sph_norm(h), cs);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) scal->hint_valid = 1u;
}

// The smoothing lengths on the device seed the next evaluation's brackets.
__global__ void k_sph_done(SphScalars* scal) { scal->hint_valid = 1u; }

// ---- hydro (forces.rs:339-379) ----------------------------------------------------------
struct HydroArgs {
  GridDev g;
  const SphScalars* sc;
  const double4* sv;
  const double4* sa;
  double* gacc;
  double* dudt;
  int adiabatic;
  double c_s, gamma, alpha, beta, visc_eps2;
  const uint32_t* targets;  // gas-local targets (nullptr: every gas particle, in grid order)
  uint32_t n_targets;
  const uint32_t* inv;      // gas-local index -> slot of this grid
};

// Six blocks an SM (80 registers, a few spilled): the kernel is latency-bound on its
// neighbour loads, and 24 resident warps beat 16 at 112 registers (measured).
__global__ void __launch_bounds__(kSphThreads, 6) k_sph_hydro(HydroArgs a) {
  __shared__ uint32_t s_pair[kSphWarps][kPairCap];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t wi = blockIdx.x * kSphWarps + warp;
  if (wi >= (a.targets ? a.n_targets : a.g.n)) return;  // warp-uniform
  uint32_t* pl = s_pair[warp];
  const uint32_t w = a.targets ? a.inv[a.targets[wi]] : wi;  // the target's slot
  const double4 xi = a.g.sp[w];
  const uint32_t k = static_cast<uint32_t>(a.g.sc[w].w);
  const double4 vi = a.sv[w];
  const double h_i = vi.w;
  const double4 ai = a.sa[w];  // rho, term, norm, c_s of the target
  const double term_i = ai.y;
  const double R = 2.0 * a.sc->h_max;
  const double R2 = R * R;
  double ax = 0.0, ay = 0.0, az = 0.0, du = 0.0;
  uint32_t np = 0;
  // The pairs of the list, 32 at a time (every lane busy).
  auto flush = [&]() {
    for (uint32_t j = lane; j < np; j += 32) {
      const uint32_t s = pl[j];
      const double4 p = a.g.sp[s];
      const double rx = xi.x - p.x, ry = xi.y - p.y, rz = xi.z - p.z;
      const double r = sqrt(rx * rx + ry * ry + rz * rz);
      const double4 vj = a.sv[s];
      // beyond both supports both gradients are zero and the pair adds exact zeros
      if (r >= 2.0 * fmax(h_i, vj.w)) continue;
      const double4 aj = a.sa[s];
      double gix, giy, giz, gjx, gjy, gjz;
      const bool nzi = sph_grad(rx, ry, rz, r, h_i, ai.z, gix, giy, giz);
      const bool nzj = sph_grad(rx, ry, rz, r, vj.w, aj.z, gjx, gjy, gjz);
      if (!nzi && !nzj) continue;
      const double gax = (gix + gjx) * 0.5, gay = (giy + gjy) * 0.5, gaz = (giz + gjz) * 0.5;
      const double term_j = aj.y;
      const double vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
      const double vr = vx * rx + vy * ry + vz * rz;
      double visc = 0.0;
      if (vr < 0.0) {
        const double h_bar = 0.5 * (h_i + vj.w);
        const double rho_bar = 0.5 * (ai.x + aj.x);
        const double mu = h_bar * vr / (r * r + a.visc_eps2 * h_bar * h_bar);
        const double c_bar = a.adiabatic ? 0.5 * (ai.w + aj.w) : a.c_s;
        visc = (-a.alpha * c_bar * mu + a.beta * mu * mu) / rho_bar;
      }
      const double coeff = term_i + term_j + visc;
      const double sc_ = -p.w * coeff;
      ax += gax * sc_;
      ay += gay * sc_;
      az += gaz * sc_;
      du += p.w * (term_i + 0.5 * visc) * (vx * gax + vy * gay + vz * gaz);
    }
    np = 0;
    __syncwarp();
  };
  // Scan the box: a neighbour whose squared distance is below (2 max(h_i, h_j))^2, with
  // a margin over its rounding, goes to the list (a superset of the coupled pairs; the
  // exact test r >= 2 max(h_i, h_j) is made again in the flush).
  visit_box(a.g, xi.x, xi.y, xi.z, R, [&](bool ok, uint32_t s) {
    bool take = false;
    if (ok && s != w) {  // slot w is the target itself
      const double4 p = a.g.sp[s];
      const double rx = xi.x - p.x, ry = xi.y - p.y, rz = xi.z - p.z;
      const double r2 = rx * rx + ry * ry + rz * rz;
      if (r2 <= R2) {
        const double lim = 2.0 * fmax(h_i, a.sv[s].w);
        take = r2 < lim * lim * (1.0 + 1e-12);
      }
    }
    const unsigned m = __ballot_sync(kFull, take);
    if (take) pl[np + __popc(m & ((1u << lane) - 1u))] = s;
    np += __popc(m);
    __syncwarp();
    if (np > static_cast<uint32_t>(kPairCap - 32)) flush();
  });
  flush();
  ax = warp_sum(ax);
  ay = warp_sum(ay);
  az = warp_sum(az);
  du = warp_sum(du);
  if (lane == 0) {
    a.gacc[3 * (size_t)k] = ax;
    a.gacc[3 * (size_t)k + 1] = ay;
    a.gacc[3 * (size_t)k + 2] = az;
    a.dudt[k] = du;
  }
}

// acc[gas row] += hydro (gravity_sph.rs:203-205), for every gas particle or the listed ones.
__global__ void __launch_bounds__(kFlat) k_sph_scatter(uint32_t n_gas, const uint32_t* __restrict__ gas_idx,
                                                       const uint32_t* __restrict__ targets,
                                                       const double* __restrict__ gacc, double* __restrict__ acc) {
  for (uint32_t t = blockIdx.x * kFlat + threadIdx.x; t < n_gas; t += gridDim.x * kFlat) {
    const uint32_t k = targets ? targets[t] : t;
    const size_t i = gas_idx[k];
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[3 * i + c] = acc[3 * i + c] + gacc[3 * (size_t)k + c];
  }
}

// ---- velocity divergence (divergence.rs:34-72) and coupled pairs (cfl.rs:195-228) ----------
// On the density grid of the same call: per target the gather of radius 2 h_i,
// div v_i = sum_{j != i} m_j (v_j - v_i) . grad_i W(r_ij, h_i) / rho_i.
__global__ void __launch_bounds__(kSphThreads) k_sph_divergence(GridDev g, const double4* __restrict__ gv,
                                                                const double* __restrict__ hs,
                                                                const double* __restrict__ rho,
                                                                double* __restrict__ div) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t w = blockIdx.x * kSphWarps + warp;
  if (w >= g.n) return;
  const double4 xi = g.sp[w];
  const uint32_t k = static_cast<uint32_t>(g.sc[w].w);
  const double4 vi = gv[k];
  const double h_i = hs[k], norm_i = sph_norm(h_i);
  const double R = 2.0 * h_i, R2 = R * R;
  double sum = 0.0;
  visit_box(g, xi.x, xi.y, xi.z, R, [&](bool ok, uint32_t s) {
    if (!ok || s == w) return;  // slot w is the target itself
    const double4 p = g.sp[s];
    const double rx = xi.x - p.x, ry = xi.y - p.y, rz = xi.z - p.z;
    const double r2 = rx * rx + ry * ry + rz * rz;
    if (!(r2 <= R2)) return;
    double gx, gy, gz;
    if (!sph_grad(rx, ry, rz, sqrt(r2), h_i, norm_i, gx, gy, gz)) return;
    const double4 vj = gv[static_cast<uint32_t>(g.sc[s].w)];
    sum += p.w * ((vj.x - vi.x) * gx + (vj.y - vi.y) * gy + (vj.z - vi.z) * gz);
  });
  sum = warp_sum(sum);
  if (lane == 0) div[k] = sum / rho[k];
}

// Coupled pairs (a, b), a < b gas-local, 0 < r < 2 max(h_a, h_b), on the hydro grid (radius
// 2 h_max as the reference's gather): counts[a] when list is null, else the b of each pair
// written from list[offsets[a]] on (in the grid's visit order; the host sorts each run).
__global__ void __launch_bounds__(kSphThreads) k_sph_pairs(GridDev g, const SphScalars* sc, const double* __restrict__ hs,
                                                           uint32_t* __restrict__ counts,
                                                           const uint64_t* __restrict__ offsets,
                                                           uint32_t* __restrict__ list) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t w = blockIdx.x * kSphWarps + warp;
  if (w >= g.n) return;
  const double4 xi = g.sp[w];
  const uint32_t a = static_cast<uint32_t>(g.sc[w].w);
  const double h_a = hs[a];
  const double R = 2.0 * sc->h_max, R2 = R * R;
  uint32_t cnt = 0;
  visit_box(g, xi.x, xi.y, xi.z, R, [&](bool ok, uint32_t s) {
    bool take = false;
    uint32_t b = 0;
    if (ok) {
      b = static_cast<uint32_t>(g.sc[s].w);
      if (b > a) {
        const double4 p = g.sp[s];
        const double rx = xi.x - p.x, ry = xi.y - p.y, rz = xi.z - p.z;
        const double r2 = rx * rx + ry * ry + rz * rz;
        if (r2 <= R2) {
          const double r = sqrt(r2);
          take = r > 0.0 && r < 2.0 * fmax(h_a, hs[b]);
        }
      }
    }
    const unsigned m = __ballot_sync(kFull, take);
    if (list && take) list[offsets[a] + cnt + __popc(m & ((1u << lane) - 1u))] = b;
    cnt += __popc(m);
  });
  if (!list && lane == 0) counts[a] = cnt;
}

// ---- CFL (cfl.rs:67-121) ----------------------------------------------------------------
struct CflArgs {
  GridDev g;
  SphScalars* sc;
  const double4* gv;  // current velocities (gas-local), .w = u
  const double* hs;
  double* dtv;
  int adiabatic;
  double c_s, gamma, c_cfl;
};

__global__ void __launch_bounds__(kSphThreads) k_sph_cfl(CflArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t w = blockIdx.x * kSphWarps + warp;
  if (w >= a.g.n) return;
  const double4 xi = a.g.sp[w];
  const uint32_t k = static_cast<uint32_t>(a.g.sc[w].w);
  const double4 vi = a.gv[k];
  const double h_i = a.hs[k];
  const double cs_i = a.adiabatic ? sqrt(a.gamma * (a.gamma - 1.0) * vi.w) : a.c_s;
  const double two_cs = 2.0 * a.c_s;
  const double R = 2.0 * a.sc->h_max;
  const double R2 = R * R;
  double v_sig = a.adiabatic ? 2.0 * cs_i : two_cs;
  visit_box(a.g, xi.x, xi.y, xi.z, R, [&](bool ok, uint32_t s) {
    if (!ok) return;
    const uint32_t j = static_cast<uint32_t>(a.g.sc[s].w);
    if (j == k) return;
    const double4 p = a.g.sp[s];
    const double rx = xi.x - p.x, ry = xi.y - p.y, rz = xi.z - p.z;
    const double r2 = rx * rx + ry * ry + rz * rz;
    if (!(r2 <= R2)) return;
    const double r = sqrt(r2);
    const double h_j = a.hs[j];
    if (r == 0.0 || r >= 2.0 * fmax(h_i, h_j)) return;
    const double4 vj = a.gv[j];
    const double wv = ((vi.x - vj.x) * rx + (vi.y - vj.y) * ry + (vi.z - vj.z) * rz) / r;
    if (a.adiabatic) {
      const double approach = wv < 0.0 ? -3.0 * wv : 0.0;
      v_sig = fmax(v_sig, cs_i + sqrt(a.gamma * (a.gamma - 1.0) * vj.w) + approach);
    } else if (wv < 0.0) {
      v_sig = fmax(v_sig, two_cs - 3.0 * wv);
    }
  });
  v_sig = warp_max(v_sig);
  if (lane == 0) {
    const double dt = a.c_cfl * h_i / v_sig;
    a.dtv[k] = dt;
    atomicMax(&a.sc->min_dt_enc, enc_max(-dt));
  }
}

uint32_t flat_grid(size_t n) {
  return static_cast<uint32_t>(std::max<size_t>(1, std::min<size_t>((n + kFlat - 1) / kFlat, 148 * 8)));
}
uint32_t warp_grid(size_t n) { return static_cast<uint32_t>((n + kSphWarps - 1) / kSphWarps); }

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Build grid g over the gathered gas: keys, stable sort by bucket, runs, mixed buckets.
void grid_build(SphState& s, int g, DevCtl* ctl, cudaStream_t st) {
  SphGrid& G = s.grid[g];
  const uint32_t n = static_cast<uint32_t>(s.n_gas);
  const size_t T = size_t{1} << s.tbits;
  const GridDev d = view(s, g);
  cudaMemsetAsync(G.start, 0, T * sizeof(uint32_t), st);
  cudaMemsetAsync(G.end, 0, T * sizeof(uint32_t), st);
  cudaMemsetAsync(s.hist, 0, kMaxRadixPasses * kRadixBins * sizeof(uint32_t), st);
  cudaMemsetAsync(s.status, 0, size_t(kRadixPasses) * s.ntiles * kRadixBins * sizeof(uint32_t), st);
  cudaMemsetAsync(s.counters, 0, kCounterWords * sizeof(uint32_t), st);
  k_grid_keys<<<flat_grid(n), kFlat, 0, st>>>(n, s.gp, d.cell, d.tmask, G.key, G.cc);
  StepBufs b;
  b.n = n;
  b.nsys = 1;
  b.ntiles = s.ntiles;
  b.tiles = s.tiles;
  b.sys = s.sys;
  b.codes = G.key;
  b.hist = s.hist;
  launch_code_hist(b, st);
  launch_sort_passes(G.key, G.skey, G.order, s.keys_tmp, s.vals_tmp, s.tiles, s.sys, s.hist, s.status, s.counters,
                     s.ntiles, ctl, st);
  k_grid_fill<<<flat_grid(n), kFlat, 0, st>>>(n, G.skey, G.order, s.gp, G.cc, G.sp, G.sc, G.start, G.end, G.inv);
  cudaMemsetAsync(G.mixed, 0, (T / 32 + 1) * sizeof(uint32_t), st);
  k_grid_mixed<<<flat_grid(n), kFlat, 0, st>>>(n, G.skey, G.sc, G.start, G.mixed);
}

std::mutex g_tab_mu;

}  // namespace

double sph_host_s_est(size_t n_gas, const double* pos, const uint32_t* gas_idx) {
  if (n_gas == 0) return 0.0;
  const size_t i0 = gas_idx ? gas_idx[0] : 0;
  double lo[3] = {pos[3 * i0], pos[3 * i0 + 1], pos[3 * i0 + 2]}, hi[3] = {lo[0], lo[1], lo[2]};
  for (size_t k = 0; k < n_gas; ++k) {
    const size_t i = gas_idx ? gas_idx[k] : k;
    for (int c = 0; c < 3; ++c) {
      lo[c] = std::fmin(lo[c], pos[3 * i + c]);
      hi[c] = std::fmax(hi[c], pos[3 * i + c]);
    }
  }
  const double ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  const double diag = std::sqrt(ex * ex + ey * ey + ez * ez);
  const double vol = ex * ey * ez;
  const double n = static_cast<double>(n_gas);
  return vol > 0.0 ? std::cbrt(vol / n) : (diag > 0.0 ? diag / std::cbrt(n) : 1.0);
}

cudaError_t sph_reserve(SphState& s, size_t n_gas, bool keep_hint, double s_est_host, cudaStream_t st) {
  s.n_gas = n_gas;
  if (n_gas == 0) return cudaSuccess;
  uint32_t tb = 1;
  while ((size_t{1} << tb) < 2 * n_gas && tb < 30) ++tb;
  const uint32_t ntiles = static_cast<uint32_t>((n_gas + kTile - 1) / kTile);
  const bool fits = s.block && n_gas <= s.cap && tb <= s.tbits;
  if (!fits) {
    if (s.block) cudaFree(s.block);
    s.block = nullptr;
    const size_t cap = n_gas + n_gas / 4;
    uint32_t cb = tb;
    while ((size_t{1} << cb) < 2 * cap && cb < 30) ++cb;
    const size_t T = size_t{1} << cb;
    const size_t ct = (cap + kTile - 1) / kTile;
    size_t off = 0;
    auto take = [&](size_t bytes) {
      const size_t o = off;
      off = align256(off + bytes);
      return o;
    };
    const size_t o_idx = take(cap * 4), o_gp = take(cap * 32), o_gv = take(cap * 32), o_gu = take(cap * 8),
                 o_rho = take(cap * 8), o_hs = take(cap * 8), o_seeds = take(cap * 8), o_gacc = take(cap * 24),
                 o_dudt = take(cap * 8), o_dtv = take(cap * 8), o_sv = take(cap * 32), o_sa = take(cap * 32),
                 o_sc = take(sizeof(SphScalars));
    size_t o_g[3][10];
    for (int g = 0; g < 3; ++g) {
      o_g[g][0] = take(cap * 4);
      o_g[g][1] = take(cap * 4);
      o_g[g][2] = take(cap * 4);
      o_g[g][3] = take(cap * 16);
      o_g[g][4] = take(cap * 32);
      o_g[g][5] = take(cap * 16);
      o_g[g][6] = take(T * 4);
      o_g[g][7] = take(T * 4);
      o_g[g][8] = take((T / 32 + 1) * 4);
      o_g[g][9] = take(cap * 4);
    }
    const size_t o_tg = take(cap * 4), o_rho_act = take(cap * 8);
    const size_t o_kt = take(cap * 4), o_vt = take(cap * 4), o_hist = take(kMaxRadixPasses * kRadixBins * 4),
                 o_status = take(size_t(kRadixPasses) * ct * kRadixBins * 4), o_cnt = take(kCounterWords * 4),
                 o_tiles = take(ct * sizeof(TileDesc)), o_sys = take(sizeof(SysDesc)),
                 o_tab = take(kSphCbrtTable * sizeof(double));
    void* blk = nullptr;
    cudaError_t e = cudaMalloc(&blk, off);
    if (e != cudaSuccess) return e;
    s.block = blk;
    ++s.alloc_gen;
    char* B = static_cast<char*>(blk);
    s.cap = cap;
    s.tbits = cb;
    s.gas_idx = reinterpret_cast<uint32_t*>(B + o_idx);
    s.gp = reinterpret_cast<double4*>(B + o_gp);
    s.gv = reinterpret_cast<double4*>(B + o_gv);
    s.gu = reinterpret_cast<double*>(B + o_gu);
    s.rho = reinterpret_cast<double*>(B + o_rho);
    s.hs = reinterpret_cast<double*>(B + o_hs);
    s.seeds = reinterpret_cast<double*>(B + o_seeds);
    s.gacc = reinterpret_cast<double*>(B + o_gacc);
    s.dudt = reinterpret_cast<double*>(B + o_dudt);
    s.dtv = reinterpret_cast<double*>(B + o_dtv);
    s.sv = reinterpret_cast<double4*>(B + o_sv);
    s.sa = reinterpret_cast<double4*>(B + o_sa);
    s.sc = reinterpret_cast<SphScalars*>(B + o_sc);
    for (int g = 0; g < 3; ++g) {
      SphGrid& G = s.grid[g];
      G.key = reinterpret_cast<uint32_t*>(B + o_g[g][0]);
      G.skey = reinterpret_cast<uint32_t*>(B + o_g[g][1]);
      G.order = reinterpret_cast<uint32_t*>(B + o_g[g][2]);
      G.cc = reinterpret_cast<int4*>(B + o_g[g][3]);
      G.sp = reinterpret_cast<double4*>(B + o_g[g][4]);
      G.sc = reinterpret_cast<int4*>(B + o_g[g][5]);
      G.start = reinterpret_cast<uint32_t*>(B + o_g[g][6]);
      G.end = reinterpret_cast<uint32_t*>(B + o_g[g][7]);
      G.mixed = reinterpret_cast<uint32_t*>(B + o_g[g][8]);
      G.inv = reinterpret_cast<uint32_t*>(B + o_g[g][9]);
    }
    s.targets = reinterpret_cast<uint32_t*>(B + o_tg);
    s.rho_act = reinterpret_cast<double*>(B + o_rho_act);
    s.keys_tmp = reinterpret_cast<uint32_t*>(B + o_kt);
    s.vals_tmp = reinterpret_cast<uint32_t*>(B + o_vt);
    s.hist = reinterpret_cast<uint32_t*>(B + o_hist);
    s.status = reinterpret_cast<uint32_t*>(B + o_status);
    s.counters = reinterpret_cast<uint32_t*>(B + o_cnt);
    s.tiles = reinterpret_cast<TileDesc*>(B + o_tiles);
    s.sys = reinterpret_cast<SysDesc*>(B + o_sys);
    s.cbrt_tab = reinterpret_cast<double*>(B + o_tab);
    // cbrt of the small integers from the host's libm, as the reference's seeds use it
    static std::vector<double> tab;
    {
      std::lock_guard<std::mutex> lk(g_tab_mu);
      if (tab.empty()) {
        tab.resize(kSphCbrtTable);
        tab[0] = 0.0;
        for (int c = 1; c < kSphCbrtTable; ++c) tab[c] = std::cbrt(static_cast<double>(c));
      }
    }
    e = cudaMemcpyAsync(s.cbrt_tab, tab.data(), kSphCbrtTable * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.sc, 0, sizeof(SphScalars), st);
    if (e != cudaSuccess) return e;
    keep_hint = false;
  }
  // tiles and the system descriptor of the n_gas-particle sort
  s.ntiles = ntiles;
  std::vector<TileDesc> tiles(ntiles);
  for (uint32_t t = 0; t < ntiles; ++t) {
    tiles[t].sys = 0;
    tiles[t].begin = t * kTile;
    tiles[t].end = static_cast<uint32_t>(std::min<size_t>(n_gas, size_t(t + 1) * kTile));
    tiles[t].pad = 0;
  }
  SysDesc sys{};
  sys.off = 0;
  sys.n = static_cast<uint32_t>(n_gas);
  sys.first_tile = 0;
  sys.ntiles = ntiles;
  cudaError_t e = cudaMemcpyAsync(s.tiles, tiles.data(), ntiles * sizeof(TileDesc), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s.sys, &sys, sizeof(SysDesc), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !s.gas_idx_host.empty())
    e = cudaMemcpyAsync(s.gas_idx, s.gas_idx_host.data(), n_gas * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.gu, 0, n_gas * sizeof(double), st);
  if (e != cudaSuccess) return e;
  // Host scalars: the seed scale, a constant of n_ngb computed by the host's libm; the
  // host's s_est when it has the positions (0: the device computes it); whether the
  // smoothing lengths on the device may seed the next brackets.
  struct {
    double seed_scale, s_est_host;
    uint32_t hint_valid;
  } hv{std::cbrt(3.0 * s.p.n_ngb / (32.0 * kPi)), s_est_host, 0u};
  e = cudaMemcpyAsync(&s.sc->seed_scale, &hv.seed_scale, sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&s.sc->s_est_host, &hv.s_est_host, sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !keep_hint)
    e = cudaMemcpyAsync(&s.sc->hint_valid, &hv.hint_valid, sizeof(uint32_t), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the host copies' sources go out of scope
  return e;
}

void sph_free(SphState& s) {
  if (s.block) cudaFree(s.block);
  s.block = nullptr;
  s.cap = 0;
  s.n_gas = 0;
}

void sph_enqueue_force(SphState& s, const double* pos, const double* vel, const double* mass, double* acc,
                       bool density, bool hydro, DevCtl* ctl, cudaStream_t st, cudaEvent_t after_density,
                       const uint32_t* targets, uint32_t n_targets, bool always_warm) {
  const uint32_t n = static_cast<uint32_t>(s.n_gas);
  if (n == 0) return;
  SphScalars* sc = s.sc;
  // reset the per-step reductions (bbox, h_max, seed histogram), keep the host values
  cudaMemsetAsync(sc->bbox_enc, 0, sizeof(sc->bbox_enc) + 2 * sizeof(unsigned long long), st);
  cudaMemsetAsync(sc->seed_hist, 0, sizeof(sc->seed_hist), st);
  k_sph_gather<<<flat_grid(n), kFlat, 0, st>>>(n, s.gas_idx, pos, vel, mass, s.gu, s.gp, s.gv, sc, 1);
  if (density) {
    k_sph_scalars<<<1, 1, 0, st>>>(n, sc);
    grid_build(s, 0, ctl, st);
    k_sph_seeds<<<flat_grid(n), kFlat, 0, st>>>(view(s, 0), s.grid[0].skey, s.grid[0].mixed, s.cbrt_tab, sc,
                                                s.seeds);
    k_sph_dens_cell<<<1, 1, 0, st>>>(n, sc);
    grid_build(s, 1, ctl, st);
    DensArgs da;
    da.g = view(s, 1);
    da.sc = sc;
    da.seeds = s.seeds;
    da.rho = s.rho;
    da.hs = s.hs;
    da.n_ngb = s.p.n_ngb;
    da.tol = s.p.h_tol_rel;
    da.warm = (s.p.warm_start || always_warm) ? 1 : 0;
    da.ctl = ctl;
    da.targets = targets;
    da.n_targets = n_targets;
    da.inv = s.grid[1].inv;
    const uint32_t nd = targets ? n_targets : n;
    if (nd) k_sph_density<<<(nd + kDensWarps - 1) / kDensWarps, kDensThreads, 0, st>>>(da);
  }
  if (after_density) cudaEventRecord(after_density, st);
  if (!hydro) {
    k_sph_done<<<1, 1, 0, st>>>(sc);
    return;
  }
  k_sph_hmax<<<flat_grid(n), kFlat, 0, st>>>(n, s.hs, sc);
  k_sph_hydro_cell<<<1, 1, 0, st>>>(sc);
  grid_build(s, 2, ctl, st);
  k_sph_pack<<<flat_grid(n), kFlat, 0, st>>>(n, s.grid[2].sc, s.gv, s.hs, s.rho, s.p.eos == GX_EOS_ADIABATIC,
                                             s.p.c_s, s.p.gamma, s.sv, s.sa, sc);
  HydroArgs ha;
  ha.g = view(s, 2);
  ha.sc = sc;
  ha.sv = s.sv;
  ha.sa = s.sa;
  ha.gacc = s.gacc;
  ha.dudt = s.dudt;
  ha.adiabatic = s.p.eos == GX_EOS_ADIABATIC;
  ha.c_s = s.p.c_s;
  ha.gamma = s.p.gamma;
  ha.alpha = s.p.alpha;
  ha.beta = s.p.beta;
  ha.visc_eps2 = s.p.visc_eps2;
  ha.targets = targets;
  ha.n_targets = n_targets;
  ha.inv = s.grid[2].inv;
  const uint32_t nh = targets ? n_targets : n;
  if (!nh) return;
  k_sph_hydro<<<warp_grid(nh), kSphThreads, 0, st>>>(ha);
  if (acc) k_sph_scatter<<<flat_grid(nh), kFlat, 0, st>>>(nh, s.gas_idx, targets, s.gacc, acc);
}

void sph_enqueue_divergence(SphState& s, double* div, cudaStream_t st) {
  const uint32_t n = static_cast<uint32_t>(s.n_gas);
  if (n) k_sph_divergence<<<warp_grid(n), kSphThreads, 0, st>>>(view(s, 1), s.gv, s.hs, s.rho, div);
}

void sph_enqueue_pairs(SphState& s, uint32_t* counts, const uint64_t* offsets, uint32_t* list, DevCtl* ctl,
                       cudaStream_t st, bool build_grid) {
  const uint32_t n = static_cast<uint32_t>(s.n_gas);
  if (!n) return;
  if (build_grid) {
    cudaMemsetAsync(&s.sc->h_max_bits, 0, sizeof(unsigned long long), st);
    k_sph_hmax<<<flat_grid(n), kFlat, 0, st>>>(n, s.hs, s.sc);
    k_sph_hydro_cell<<<1, 1, 0, st>>>(s.sc);
    grid_build(s, 2, ctl, st);
  }
  k_sph_pairs<<<warp_grid(n), kSphThreads, 0, st>>>(view(s, 2), s.sc, s.hs, counts, offsets, list);
}

void sph_enqueue_cfl(SphState& s, const double* pos, const double* vel, double c_cfl, bool rebuild, DevCtl* ctl,
                     cudaStream_t st) {
  const uint32_t n = static_cast<uint32_t>(s.n_gas);
  if (n == 0) return;
  SphScalars* sc = s.sc;
  cudaMemsetAsync(&sc->min_dt_enc, 0, sizeof(unsigned long long), st);
  if (rebuild) {
    cudaMemsetAsync(sc->bbox_enc, 0, sizeof(sc->bbox_enc) + sizeof(unsigned long long), st);
    k_sph_gather<<<flat_grid(n), kFlat, 0, st>>>(n, s.gas_idx, pos, vel, nullptr, s.gu, s.gp, s.gv, sc, 0);
    k_sph_hmax<<<flat_grid(n), kFlat, 0, st>>>(n, s.hs, sc);
    k_sph_hydro_cell<<<1, 1, 0, st>>>(sc);
    grid_build(s, 2, ctl, st);
  } else {
    // the current velocities (the grid's positions are those of the last evaluation)
    k_sph_gather<<<flat_grid(n), kFlat, 0, st>>>(n, s.gas_idx, pos, vel, nullptr, s.gu, s.gp, s.gv, sc, 0);
  }
  CflArgs ca;
  ca.g = view(s, 2);
  ca.sc = sc;
  ca.gv = s.gv;
  ca.hs = s.hs;
  ca.dtv = s.dtv;
  ca.adiabatic = s.p.eos == GX_EOS_ADIABATIC;
  ca.c_s = s.p.c_s;
  ca.gamma = s.p.gamma;
  ca.c_cfl = c_cfl;
  k_sph_cfl<<<warp_grid(n), kSphThreads, 0, st>>>(ca);
}

}  // namespace gx
