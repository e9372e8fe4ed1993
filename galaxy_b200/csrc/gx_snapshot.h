// gx_snapshot.h -- GLXYSNAP v4 snapshot files and the staging of a batched system's
// snapshot on the device (host-only declarations: the server includes this header).
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/galaxy_b200.h"

namespace gx {

// Header fields of one snapshot (io/src/snapshot.rs:88-108; scale factor 1, n from the
// data, code version this library's).
struct SnapHeader {
  double time = 0.0;
  uint64_t step = 0;
  double softening = 0.0;
  uint64_t rng_seed = 0;
  uint64_t config_hash = 0;
  std::string units = "nbody-G1";
};

// Bytes of a staged snapshot of n particles: positions (3n f64), velocities (3n f64),
// masses (n f32) -- the state-dependent columns, in file order.
size_t snapshot_stage_bytes(size_t n);

// The calling thread's error text for entry points without a handle (gx_last_error(NULL)).
void set_global_err(const std::string& s);

// Write a GLXYSNAP v4 file from host arrays (mass f64, stored as f32 like the reference)
// or from a staged buffer (mass already f32). The columns the gravity path does not
// evolve take the reference State's defaults: id = index, progenitor 0, kind
// collisionless, u = 0, formation time -inf (State::PRIMORDIAL).
bool write_glxysnap(const std::string& path, const SnapHeader& h, size_t n, const double* pos, const double* vel,
                    const double* mass, std::string& err);
bool write_glxysnap_staged(const std::string& path, const SnapHeader& h, size_t n, const void* staged,
                           std::string& err);

// Stage system `id`'s snapshot: on the batch's stream a kernel writes its positions,
// its velocities with the owed closing half kick (as gx_system_snapshot) and its f32
// masses into d_stage; copy_stream then waits for that and copies d_stage to host_dst
// (pinned, snapshot_stage_bytes(n)), recording `copied` when done. The batch steps on
// meanwhile. time_out / n_out: the system's time and size at this point.
int batch_stage_snapshot(gx_batch* b, uint64_t id, void* d_stage, void* host_dst, cudaStream_t copy_stream,
                         cudaEvent_t copied, double* time_out, size_t* n_out);

}  // namespace gx
