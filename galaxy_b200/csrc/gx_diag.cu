// gx_diag.cu -- FP64 O(N^2) kernels for the force oracle and the energy diagnostics.
//
// Reference: solvers/src/direct_sum.rs:25-45 (Plummer-softened pairwise sum; here
// unpaired, one thread per target, so the summation order differs and results are
// compared with a tolerance), solvers/src/potential.rs:17-58 (softened potential,
// U = -sum_{i<j} G m_i m_j / sqrt(r^2 + eps^2), evaluated as half of the full
// double sum), core/src/diagnostics.rs:8-68 (kinetic energy, momentum, angular
// momentum). Per-block partials are summed on the host in block order, so every
// result is deterministic. Both O(N^2) sums use FMA and the FP64 reciprocal square
// root (about 15 FP64 operations a pair); they are checks, compared with tolerances.
#include "gx_kernels.h"

namespace gx {

namespace {
constexpr int kDiagThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kDiagThreads / 32; ++w) t += sh[w];
  return t;
}
}  // namespace

// acc[3t] for target t = targets ? targets[t] : t. Sources staged through shared
// memory in tiles of kDiagThreads.
__global__ void __launch_bounds__(kDiagThreads) k_direct_sum_f64(uint32_t n, const double* __restrict__ pos,
                                                                const double* __restrict__ mass, double g, double eps2,
                                                                uint32_t n_targets,
                                                                const uint32_t* __restrict__ targets,
                                                                double* __restrict__ acc) {
  __shared__ double4 src[kDiagThreads];
  const uint32_t t = blockIdx.x * kDiagThreads + threadIdx.x;
  const bool valid = t < n_targets;
  const uint32_t i = valid ? (targets ? targets[t] : t) : 0u;
  double xi[3] = {0, 0, 0};
  if (valid)
    for (int c = 0; c < 3; ++c) xi[c] = pos[3 * (size_t)i + c];
  double a[3] = {0, 0, 0};
  for (uint32_t base = 0; base < n; base += kDiagThreads) {
    const uint32_t j = base + threadIdx.x;
    __syncthreads();
    if (j < n)
      src[threadIdx.x] = make_double4(pos[3 * (size_t)j], pos[3 * (size_t)j + 1], pos[3 * (size_t)j + 2], mass[j]);
    else
      src[threadIdx.x] = make_double4(0, 0, 0, 0);
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kDiagThreads, n - base);
    for (uint32_t q = 0; q < cnt; ++q) {
      // the pair with itself adds nothing (massless, at unit distance)
      const bool self = base + q == i;
      const double4 s = src[q];
      const double dx = s.x - xi[0], dy = s.y - xi[1], dz = s.z - xi[2];
      const double r2 = self ? 1.0 : fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
      const double inv = rsqrt(r2);
      const double f = (self ? 0.0 : s.w) * (inv * inv * inv);
      a[0] = fma(dx, f, a[0]);
      a[1] = fma(dy, f, a[1]);
      a[2] = fma(dz, f, a[2]);
    }
  }
  if (valid)
    for (int c = 0; c < 3; ++c) acc[3 * (size_t)t + c] = a[c] * g;
}

// partial[b] = sum over this block's rows i of -G m_i / 2 * sum_{j != i} m_j / sqrt(r^2+eps^2).
__global__ void __launch_bounds__(kDiagThreads) k_potential_f64(uint32_t n, const double* __restrict__ pos,
                                                               const double* __restrict__ mass, double g, double eps2,
                                                               double* __restrict__ partial) {
  __shared__ double4 src[kDiagThreads];
  __shared__ double sh[kDiagThreads / 32];
  const uint32_t i = blockIdx.x * kDiagThreads + threadIdx.x;
  const bool valid = i < n;
  double xi[3] = {0, 0, 0}, mi = 0.0;
  if (valid) {
    for (int c = 0; c < 3; ++c) xi[c] = pos[3 * (size_t)i + c];
    mi = mass[i];
  }
  double u = 0.0;
  for (uint32_t base = 0; base < n; base += kDiagThreads) {
    const uint32_t j = base + threadIdx.x;
    __syncthreads();
    if (j < n)
      src[threadIdx.x] = make_double4(pos[3 * (size_t)j], pos[3 * (size_t)j + 1], pos[3 * (size_t)j + 2], mass[j]);
    else
      src[threadIdx.x] = make_double4(0, 0, 0, 0);
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kDiagThreads, n - base);
    for (uint32_t q = 0; q < cnt; ++q) {
      const bool self = base + q == i;
      const double4 s = src[q];
      const double dx = s.x - xi[0], dy = s.y - xi[1], dz = s.z - xi[2];
      const double r2 = self ? 1.0 : fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
      u = fma(self ? 0.0 : s.w, rsqrt(r2), u);  // sum_j m_j / sqrt(r^2 + eps^2)
    }
  }
  const double t = block_sum(valid ? -0.5 * g * mi * u : 0.0, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// partial[7 b + c]: kinetic, px, py, pz, lx, ly, lz sums over the block's particles.
__global__ void __launch_bounds__(kDiagThreads) k_diag_sums(uint32_t n, const double* __restrict__ pos,
                                                           const double* __restrict__ vel,
                                                           const double* __restrict__ mass,
                                                           double* __restrict__ partial) {
  __shared__ double sh[kDiagThreads / 32];
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (uint32_t i = blockIdx.x * kDiagThreads + threadIdx.x; i < n; i += gridDim.x * kDiagThreads) {
    const double m = mass[i];
    const double rx = pos[3 * (size_t)i], ry = pos[3 * (size_t)i + 1], rz = pos[3 * (size_t)i + 2];
    const double vx = vel[3 * (size_t)i], vy = vel[3 * (size_t)i + 1], vz = vel[3 * (size_t)i + 2];
    v[0] += dmul(dmul(0.5, m), dlen2(vx, vy, vz));
    v[1] += dmul(vx, m);
    v[2] += dmul(vy, m);
    v[3] += dmul(vz, m);
    v[4] += dmul(dsub(dmul(ry, vz), dmul(rz, vy)), m);
    v[5] += dmul(dsub(dmul(rz, vx), dmul(rx, vz)), m);
    v[6] += dmul(dsub(dmul(rx, vy), dmul(ry, vx)), m);
  }
  for (int c = 0; c < 7; ++c) {
    const double t = block_sum(v[c], sh);
    if (threadIdx.x == 0) partial[7 * blockIdx.x + c] = t;
  }
}

// Failure-detection self-test: lane 0 waits, through the sort look-back's bounded wait,
// for a word nothing sets; the wait runs out, raises the error word and returns.
__global__ void k_selftest_wait(const uint32_t* word, uint32_t spins, DevCtl* ctl) {
  if (threadIdx.x == 0) (void)wait_flagged(word, spins, ctl);
}

void launch_selftest_wait(const uint32_t* word, uint32_t spins, DevCtl* ctl, cudaStream_t st) {
  k_selftest_wait<<<1, 32, 0, st>>>(word, spins, ctl);
}

void launch_direct_sum_f64(uint32_t n, const double* pos, const double* mass, double g, double eps,
                           uint32_t n_targets, const uint32_t* targets, double* acc, cudaStream_t st) {
  const uint32_t grid = (n_targets + kDiagThreads - 1) / kDiagThreads;
  if (grid) k_direct_sum_f64<<<grid, kDiagThreads, 0, st>>>(n, pos, mass, g, eps * eps, n_targets, targets, acc);
}

uint32_t potential_partials(uint32_t n) { return (n + kDiagThreads - 1) / kDiagThreads; }

void launch_potential_f64(uint32_t n, const double* pos, const double* mass, double g, double eps, double* partial,
                          uint32_t n_partial, cudaStream_t st) {
  if (n_partial) k_potential_f64<<<n_partial, kDiagThreads, 0, st>>>(n, pos, mass, g, eps * eps, partial);
}

void launch_diag_sums(uint32_t n, const double* pos, const double* vel, const double* mass, double* partial,
                      uint32_t n_partial, cudaStream_t st) {
  if (n_partial) k_diag_sums<<<n_partial, kDiagThreads, 0, st>>>(n, pos, vel, mass, partial);
}

}  // namespace gx
