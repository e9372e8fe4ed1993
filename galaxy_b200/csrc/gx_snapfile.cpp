// gx_snapfile.cpp -- GLXYSNAP v4 writer (io/src/snapshot.rs:130-199 `to_writer`).
//
// Layout, all little-endian: magic "GLXYSNAP", version u32 = 4; header time f64, step
// u64, scale_factor f64, softening f64, n u64, rng_seed u64, config_hash u64, units and
// code_version as (u32 length, UTF-8 bytes); then the columns SoA: pos (3 f64 per
// particle), vel (3 f64), mass (f32), id (u64), progenitor (u16), kind (u8), u (f64),
// formation_time (f64). The field order and types are the reference's, since readers
// of its files must read ours.
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>

#include "gx_snapshot.h"

namespace gx {

namespace {

constexpr char kMagic[8] = {'G', 'L', 'X', 'Y', 'S', 'N', 'A', 'P'};
constexpr uint32_t kVersion = 4;
constexpr size_t kMaxStr = size_t{1} << 16;  // the reference's header string limit
const char* const kCodeVersion = "galaxy_b200 0.1";

// The host is little-endian (x86-64 / aarch64), so values are written as their bytes.
class Out {
 public:
  explicit Out(FILE* f) : f_(f) {}
  bool ok() const { return ok_; }
  void bytes(const void* p, size_t n) {
    if (ok_ && n && std::fwrite(p, 1, n, f_) != n) ok_ = false;
  }
  template <typename T>
  void val(T v) {
    bytes(&v, sizeof v);
  }
  void str(const std::string& s) {
    val<uint32_t>(static_cast<uint32_t>(s.size()));
    bytes(s.data(), s.size());
  }
  // n copies of one value, through a bounded buffer
  template <typename T>
  void fill(T v, size_t n) {
    std::vector<T> buf(std::min<size_t>(n, 1 << 16), v);
    for (size_t done = 0; done < n;) {
      const size_t k = std::min(buf.size(), n - done);
      bytes(buf.data(), k * sizeof(T));
      done += k;
    }
  }

 private:
  FILE* f_;
  bool ok_ = true;
};

bool write_common(const std::string& path, const SnapHeader& h, size_t n, const double* pos, const double* vel,
                  const double* mass64, const float* mass32, std::string& err) {
  if (h.units.size() > kMaxStr) {
    err = "snapshot units string exceeds 65536 bytes";
    return false;
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path + " for writing";
    return false;
  }
  Out o(f);
  o.bytes(kMagic, sizeof kMagic);
  o.val<uint32_t>(kVersion);
  o.val<double>(h.time);
  o.val<uint64_t>(h.step);
  o.val<double>(1.0);  // scale factor: not a cosmological run
  o.val<double>(h.softening);
  o.val<uint64_t>(n);  // authoritative: the data's count
  o.val<uint64_t>(h.rng_seed);
  o.val<uint64_t>(h.config_hash);
  o.str(h.units);
  o.str(kCodeVersion);
  o.bytes(pos, 3 * n * sizeof(double));
  o.bytes(vel, 3 * n * sizeof(double));
  if (mass32) {
    o.bytes(mass32, n * sizeof(float));
  } else {
    std::vector<float> m(std::min<size_t>(n, 1 << 16));
    for (size_t done = 0; done < n;) {
      const size_t k = std::min(m.size(), n - done);
      for (size_t i = 0; i < k; ++i) m[i] = static_cast<float>(mass64[done + i]);  // round to nearest
      o.bytes(m.data(), k * sizeof(float));
      done += k;
    }
  }
  {
    std::vector<uint64_t> id(std::min<size_t>(n, 1 << 16));
    for (size_t done = 0; done < n;) {
      const size_t k = std::min(id.size(), n - done);
      for (size_t i = 0; i < k; ++i) id[i] = done + i;
      o.bytes(id.data(), k * sizeof(uint64_t));
      done += k;
    }
  }
  o.fill<uint16_t>(0, n);                                            // progenitor
  o.fill<uint8_t>(0, n);                                             // kind: collisionless
  o.fill<double>(0.0, n);                                            // u
  o.fill<double>(-std::numeric_limits<double>::infinity(), n);       // formation time: primordial
  const bool good = o.ok();
  if (std::fclose(f) != 0 || !good) {
    err = "write error on " + path;
    return false;
  }
  return true;
}

}  // namespace

size_t snapshot_stage_bytes(size_t n) { return n * (6 * sizeof(double) + sizeof(float)); }

bool write_glxysnap(const std::string& path, const SnapHeader& h, size_t n, const double* pos, const double* vel,
                    const double* mass, std::string& err) {
  return write_common(path, h, n, pos, vel, mass, nullptr, err);
}

bool write_glxysnap_staged(const std::string& path, const SnapHeader& h, size_t n, const void* staged,
                           std::string& err) {
  const double* p = static_cast<const double*>(staged);
  return write_common(path, h, n, p, p + 3 * n, nullptr, reinterpret_cast<const float*>(p + 6 * n), err);
}

}  // namespace gx

extern "C" int gx_glxysnap_write(const char* path, double time, uint64_t step, double softening, uint64_t rng_seed,
                                 uint64_t config_hash, const char* units, size_t n, const double* pos,
                                 const double* vel, const double* mass) {
  if (!path || (n && (!pos || !vel || !mass))) return GX_ERR_INVALID_ARG;
  gx::SnapHeader h;
  h.time = time;
  h.step = step;
  h.softening = softening;
  h.rng_seed = rng_seed;
  h.config_hash = config_hash;
  if (units) h.units = units;
  std::string err;
  if (gx::write_glxysnap(path, h, n, pos, vel, mass, err)) return GX_OK;
  gx::set_global_err(err);
  return GX_ERR_INVALID_ARG;
}
