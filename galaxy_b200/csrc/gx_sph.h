// gx_sph.h -- resident SPH on the gas subset of one system (host-side declarations).
//
// Reference: solvers/src/sph/*.rs (the CPU toolkit and GravitySph composite) and the
// resident gas mode of gpu/src/gpu_resident.rs:1393-1565 (`new_with_sph`,
// `encode_sph_force`): gravity on every particle, then density, hydro force and a
// scatter-add of the hydro acceleration into the gas rows.
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/galaxy_b200.h"
#include "gx_kernels.h"

namespace gx {

// Per-step device scalars of the SPH stages.
struct SphScalars {
  unsigned long long bbox_enc[6];  // enc_max(-min x,y,z), enc_max(max x,y,z) of the gas
  unsigned long long h_max_bits;   // max h (positive doubles order like their bits)
  unsigned long long min_dt_enc;   // enc_max(-dt): the CFL minimum
  double s_est, h_seed, h_cap, occ_cell, dens_cell, hydro_cell, h_max;
  double seed_scale;               // cbrt(3 n_ngb / (32 pi)), from the host
  double s_est_host;               // > 0: the host computed s_est (used instead)
  uint32_t hint_valid;             // the previous h may seed this step's brackets
  uint32_t pad;
  uint32_t seed_hist[2048];        // exponent histogram of the seeds (density cell)
};

// One uniform grid over the gas: cells of edge *cell, hashed into T buckets; the gas
// sorted by bucket (stably), each bucket a run [start, end) of the sorted arrays.
struct SphGrid {
  uint32_t* key = nullptr;    // per gas particle: bucket
  uint32_t* skey = nullptr;   // sorted buckets
  uint32_t* order = nullptr;  // sorted slot -> gas-local index
  int4* cc = nullptr;         // per gas particle: cell coordinates, w = gas-local index
  double4* sp = nullptr;      // sorted: x, y, z, mass
  int4* sc = nullptr;         // sorted: cell coordinates, w = gas-local index
  uint32_t* start = nullptr;  // T
  uint32_t* end = nullptr;    // T
  uint32_t* mixed = nullptr;  // T / 32 bits: bucket holds more than one cell
  uint32_t* inv = nullptr;    // gas-local index -> sorted slot
};

struct SphState {
  gx_sph_params p{};
  bool enabled = false;
  size_t n_gas = 0, cap = 0;
  uint32_t tbits = 0;  // T = 2^tbits buckets
  std::vector<uint32_t> gas_idx_host;
  uint32_t* gas_idx = nullptr;
  double4* gp = nullptr;  // gas-local: x, y, z, mass
  double4* gv = nullptr;  // gas-local: vx, vy, vz, u
  double* gu = nullptr;   // gas-local internal energy (zero unless given)
  double* rho = nullptr;
  double* hs = nullptr;   // smoothing lengths (also the next step's warm start)
  double* seeds = nullptr;
  double* gacc = nullptr;  // hydro acceleration, 3 per gas particle
  double* dudt = nullptr;
  double* dtv = nullptr;   // CFL bound per gas particle
  uint32_t* targets = nullptr;  // gas-local targets of an active-subset pass
  double* rho_act = nullptr;    // the active path's persistent density scratch
  double4* sv = nullptr;   // hydro grid order: vx, vy, vz, h
  double4* sa = nullptr;   // hydro grid order: rho, P/rho^2 term, 1/(pi h^3), c_s
  SphScalars* sc = nullptr;
  SphGrid grid[3];  // occupancy, density query, hydro
  // sort scratch of the grids (one system of n_gas)
  uint32_t *keys_tmp = nullptr, *vals_tmp = nullptr, *hist = nullptr, *status = nullptr, *counters = nullptr;
  TileDesc* tiles = nullptr;
  SysDesc* sys = nullptr;
  uint32_t ntiles = 0;
  double* cbrt_tab = nullptr;  // cbrt(c) for integer c < kSphCbrtTable, from the host's libm
  void* block = nullptr;       // the single allocation behind every buffer above
  uint64_t alloc_gen = 0;      // bumped at every (re)allocation: device scratch is lost
};

constexpr int kSphCbrtTable = 65536;

// Allocate for n_gas gas particles (never shrinks) and upload the gas map
// (gas_idx_host) and the host scalars; the gas-local u starts at zero. keep_hint keeps
// the device's smoothing lengths as the next evaluation's warm start (same gas map);
// s_est_host > 0 replaces the device's spacing estimate.
cudaError_t sph_reserve(SphState& s, size_t n_gas, bool keep_hint, double s_est_host, cudaStream_t st);
void sph_free(SphState& s);
// Gas gather + bbox (pos, vel, mass of the system; vel nullable; u from gu), then the
// density (when `density`; otherwise rho / hs hold the caller's values), the hydro force
// (when `hydro`) and, when acc is non-null, its scatter-add into the gas rows of acc.
// targets (device, gas-local, n_targets of them; nullptr: every gas particle) restricts
// the density and hydro passes and the scatter to those particles; the grids, seeds and
// h_max cover all gas, the others' rho / h are read as they are (the active path).
// always_warm: the density brackets start from the kept h whenever it is valid, whatever
// warm_start says (the individual-timestep path: density_adaptive_active always
// warm-starts from its persistent h).
void sph_enqueue_force(SphState& s, const double* pos, const double* vel, const double* mass, double* acc,
                       bool density, bool hydro, DevCtl* ctl, cudaStream_t st, cudaEvent_t after_density = nullptr,
                       const uint32_t* targets = nullptr, uint32_t n_targets = 0, bool always_warm = false);
// The CFL bound per gas particle (dtv) and its minimum (sc->min_dt_enc) at the current
// velocities, on the hydro grid of the last force evaluation. With rebuild, the gas is
// gathered and the hydro grid rebuilt from hs first (the caller supplied h).
void sph_enqueue_cfl(SphState& s, const double* pos, const double* vel, double c_cfl, bool rebuild, DevCtl* ctl,
                     cudaStream_t st);
// div v of every gas particle (divergence.rs:34-72) into div (gas-local), on the density
// grid, h and rho of the density pass just enqueued and the velocities it gathered.
void sph_enqueue_divergence(SphState& s, double* div, cudaStream_t st);
// Coupled gas pairs (cfl.rs:195-228) on the hydro grid (built first when build_grid): with
// list null, counts[a] = pairs (a, b > a); else the b's from list[offsets[a]] on.
void sph_enqueue_pairs(SphState& s, uint32_t* counts, const uint64_t* offsets, uint32_t* list, DevCtl* ctl,
                       cudaStream_t st, bool build_grid);
// Host-side s_est of DensitySetup::new (density.rs:166-181) from host positions: the
// gas rows gas_idx[0 .. n_gas) of pos (gas_idx NULL: rows 0 .. n_gas).
double sph_host_s_est(size_t n_gas, const double* pos, const uint32_t* gas_idx);

}  // namespace gx
