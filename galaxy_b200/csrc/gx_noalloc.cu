// gx_noalloc.cu -- gx_sort_noalloc: the (code, index) radix sort for callers that are
// not allowed to allocate device memory.
//
// Some callers cannot call cudaMalloc: a host application that owns all device memory
// through its own pool and forbids libraries from allocating, a real-time stepping
// loop that must not allocate after start-up, or a plugin host that hands a library
// device buffers but no allocation rights. This entry point takes the caller's device
// buffers for the input codes and the two outputs and keeps all of its own working
// memory -- the ping-pong key/index buffers of passes 0 and 2, the four passes'
// decoupled look-back status words, the digit histograms, the tile table and the
// device error word -- in one file-scope static __device__ array of
// kNoAllocScratchBytes (about 9 MiB, sized for GX_NOALLOC_MAX_KEYS = 2^20 keys). Every
// GPU that loads the library holds that array until the process exits.
//
// The array's name is only a host-side stand-in in host code, never a device address:
// the first call on each device, with that device current, looks the real address up
// with cudaGetSymbolAddress and caches it; that first call should therefore come
// before any stream capture. The cached address belongs to the device's primary
// context: after cudaDeviceReset (which also invalidates every other handle of this
// library on that device) the process must not call gx_sort_noalloc again. All calls share the one array, which keeps the last
// call's contents: each call clears what must start at zero (histograms, look-back
// status, tile counters, error word) on its stream before sorting. Calls that overlap
// on the GPU (two host threads, or two streams, sorting at once on one device) race
// on the array and must be serialised by the caller.
#include <mutex>
#include <string>

#include "../../include/galaxy_b200.h"
#include "gx_kernels.h"
#include "gx_runtime.h"

namespace gx {
namespace {

constexpr size_t kMaxKeys = GX_NOALLOC_MAX_KEYS;
constexpr size_t kMaxTiles = kMaxKeys / kTile + 1;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffKeys = 0;
constexpr size_t kOffVals = align256(kOffKeys + kMaxKeys * 4);
constexpr size_t kOffHist = align256(kOffVals + kMaxKeys * 4);
constexpr size_t kOffStatus = align256(kOffHist + kRadixPasses * kRadixBins * 4);
constexpr size_t kOffCounters = align256(kOffStatus + kRadixPasses * kMaxTiles * kRadixBins * 4);
constexpr size_t kOffTiles = align256(kOffCounters + 16 * 4);
constexpr size_t kOffSys = align256(kOffTiles + kMaxTiles * sizeof(TileDesc));
constexpr size_t kOffCtl = align256(kOffSys + sizeof(SysDesc));
constexpr size_t kNoAllocScratchBytes = align256(kOffCtl + sizeof(DevCtl));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
unsigned char* g_scratch_dev[256] = {};  // device address of g_noalloc_scratch, per device ordinal

// Clear the zero-start words and write the tile table of one system of n keys.
__global__ void k_noalloc_setup(unsigned char* scratch, uint32_t n, uint32_t ntiles) {
  uint32_t* hist = reinterpret_cast<uint32_t*>(scratch + kOffHist);
  uint32_t* status = reinterpret_cast<uint32_t*>(scratch + kOffStatus);
  uint32_t* counters = reinterpret_cast<uint32_t*>(scratch + kOffCounters);
  TileDesc* tiles = reinterpret_cast<TileDesc*>(scratch + kOffTiles);
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (uint32_t i = tid; i < kRadixPasses * kRadixBins; i += stride) hist[i] = 0;
  for (uint32_t i = tid; i < kRadixPasses * ntiles * kRadixBins; i += stride) status[i] = 0;
  for (uint32_t i = tid; i < 16; i += stride) counters[i] = 0;
  for (uint32_t t = tid; t < ntiles; t += stride) {
    TileDesc d;
    d.sys = 0;
    d.begin = t * kTile;
    d.end = min(n, (t + 1) * static_cast<uint32_t>(kTile));
    d.pad = 0;
    tiles[t] = d;
  }
  if (tid == 0) {
    SysDesc s{};
    s.off = 0;
    s.n = n;
    s.first_tile = 0;
    s.ntiles = ntiles;
    *reinterpret_cast<SysDesc*>(scratch + kOffSys) = s;
    DevCtl* ctl = reinterpret_cast<DevCtl*>(scratch + kOffCtl);
    ctl->err = 0;
  }
}

}  // namespace
}  // namespace gx

using namespace gx;

extern "C" int gx_sort_noalloc(const uint32_t* d_codes, uint32_t* d_sorted_codes, uint32_t* d_order, size_t n,
                               void* stream) {
  if (n == 0) return GX_OK;
  if (!d_codes || !d_sorted_codes || !d_order) {
    set_global_err("gx_sort_noalloc: null device pointer");
    return GX_ERR_INVALID_ARG;
  }
  if (n > kMaxKeys) {
    set_global_err("gx_sort_noalloc: n = " + std::to_string(n) + " exceeds GX_NOALLOC_MAX_KEYS = " +
                   std::to_string(kMaxKeys) + " (the size of its static scratch array)");
    return GX_ERR_CAPACITY;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 256) {
    set_global_err(std::string("gx_sort_noalloc: no current device: ") + cudaGetErrorString(e));
    return GX_ERR_NO_DEVICE;
  }
  unsigned char* scratch;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_dev[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        set_global_err(std::string("gx_sort_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        return GX_ERR_CUDA;
      }
      g_scratch_dev[dev] = static_cast<unsigned char*>(p);
    }
    scratch = g_scratch_dev[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t nn = static_cast<uint32_t>(n);
  const uint32_t ntiles = static_cast<uint32_t>((n + kTile - 1) / kTile);
  k_noalloc_setup<<<64, 256, 0, st>>>(scratch, nn, ntiles);
  StepBufs b;
  b.n = nn;
  b.nsys = 1;
  b.ntiles = ntiles;
  b.tiles = reinterpret_cast<const TileDesc*>(scratch + kOffTiles);
  b.sys = reinterpret_cast<const SysDesc*>(scratch + kOffSys);
  b.codes = const_cast<uint32_t*>(d_codes);  // read only by the histogram kernel
  b.hist = reinterpret_cast<uint32_t*>(scratch + kOffHist);
  launch_code_hist(b, st);
  DevCtl* ctl = reinterpret_cast<DevCtl*>(scratch + kOffCtl);
  launch_sort_passes(d_codes, d_sorted_codes, d_order, reinterpret_cast<uint32_t*>(scratch + kOffKeys),
                     reinterpret_cast<uint32_t*>(scratch + kOffVals), b.tiles, b.sys, b.hist,
                     reinterpret_cast<uint32_t*>(scratch + kOffStatus),
                     reinterpret_cast<uint32_t*>(scratch + kOffCounters), ntiles, ctl, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_global_err(std::string("gx_sort_noalloc: launch failed: ") + cudaGetErrorString(e));
    return GX_ERR_CUDA;
  }
  uint32_t err = 0;
  e = cudaMemcpyAsync(&err, &ctl->err, sizeof(err), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_global_err(std::string("gx_sort_noalloc: ") + cudaGetErrorString(e));
    return GX_ERR_CUDA;
  }
  if (err) {
    set_global_err("gx_sort_noalloc: device check tripped (error word " + std::to_string(err) + ")");
    return GX_ERR_DEVICE_CHECK;
  }
  return GX_OK;
}
