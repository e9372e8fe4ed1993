// gx_runtime.h -- host-side device-memory arena shared by the single-system handle and
// the batch (one set of step buffers, grown lazily, never shrunk).
#pragma once

#include <string>
#include <vector>

#include "../../include/galaxy_b200.h"
#include "gx_kernels.h"

#include <nvtx3/nvToolsExt.h>

namespace gx {

// An NVTX range over a scope (host enqueue of a stage; free when no tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

struct Arena {
  StepBufs b;
  std::vector<void*> allocs;
  size_t bytes = 0;
  size_t cap_n = 0, cap_tiles = 0, cap_items = 0, cap_sys = 0;
  int cap_quad = 0, cap_f64 = 0;
  // writable aliases of the const pointers in b
  double* mass_rw = nullptr;
  TileDesc* tiles_rw = nullptr;
  WalkItem* items_rw = nullptr;
  SysDesc* sys_rw = nullptr;
  double* diag_partial = nullptr;
  size_t diag_cap = 0;

  cudaError_t alloc(void** p, size_t nbytes);
  cudaError_t ensure(size_t n, size_t tiles, size_t items, size_t nsys, int quad, int f64rec, cudaStream_t st);
  void release();
  // Device bytes an arena for n particles in nsys systems takes.
  static size_t bytes_for(size_t n, size_t nsys, int quad, int f64rec);
  ~Arena() { release(); }
};

void make_tables(const std::vector<SysDesc>& in, std::vector<SysDesc>& sys, std::vector<TileDesc>& tiles,
                 std::vector<WalkItem>& items);
bool check_device(int device, std::string& err);
// Once per device, with the device current: kernel attributes the launches rely on.
void prepare_device(int dev);
void set_global_err(const std::string& s);
const char* global_err();

// Process-wide table of tuned walk launches (see gx_autotune): keyed by device,
// precision, multipole, Morton key width, batch or single system and floor(log2 n).
bool tuned_lookup(int device, const gx_options& opt, int batched, size_t n, gx_tuning* out);
void tuned_store(int device, const gx_options& opt, int batched, size_t n, const gx_tuning& t);
// Walk launch candidates: blocks of 64 and 128 threads, each as a grid of one warp per
// item (ctas 0, when with_grid) and as a persistent kernel at half and full residency.
// Walk launch candidates: block sizes x schedulings (a grid when with_grid) x groupings
// (8, 16, 32 targets a warp when with_groups).
std::vector<gx_tuning> tune_candidates(const WalkCfg& base, bool with_grid, bool with_groups);
// Targets a warp of the FP32 walk of one system of n particles: the option, else the
// single-system tuning table's entry for n, else default_walk_group(n).
uint32_t system_walk_group(int device, const gx_options& opt, size_t n);
uint32_t default_walk_group(size_t n);
// Digit width of the sort of one system of n particles: the option, else the
// single-system tuning table's entry for n, else 8 (always 8 with 63-bit keys).
uint32_t system_radix_bits(int device, const gx_options& opt, size_t n);
bool options_valid(const gx_options& o);

}  // namespace gx
