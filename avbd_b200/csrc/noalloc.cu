// avbd_exclusive_scan_noalloc: the device-wide exclusive scan of the
// collision pipeline, for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not an option -- a host
// application that owns the whole device-memory budget and hands this
// library only its input and output buffers (an engine plugin, an embedded
// simulator), or a real-time loop that must not take the device-wide
// synchronisation an allocation can cause.  The regular scan inside
// avbd_substep takes its block partials from the arena the caller allocates;
// this entry point keeps them in a fixed array of this library instead.
//
// The scratch is one file-scope device array (16 KiB).  Every GPU that loads
// the library holds it until the process exits, and every call on a device
// shares it: two calls whose work overlaps on the GPU (two streams, two host
// threads) race on it and give wrong results, so serialise them.  Nothing in
// it needs clearing between calls: each scan writes every partial it later
// reads.
//
// The array's device address is looked up once per device, with that device
// current, on the first call made there (so make that first call before any
// stream capture).  cudaDeviceReset unloads the library's module; its array
// may then sit elsewhere, so do not call this entry point after a
// cudaDeviceReset in the same process.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"

namespace avbd {
// The scan kernels of collide.cu (block partials passed by pointer).
__global__ void k_scan_reduce(const int* in, int n_host, const int* n_dev, int* part);
__global__ void k_scan_parts(int* part, int np);
__global__ void k_scan_down(const int* in, int* out, int n_host, const int* n_dev, const int* part, int np,
                            int* total_out);
void set_error_text(const char* what, cudaError_t e);
}  // namespace avbd

using namespace avbd;

namespace {

constexpr int kChunk = SCAN_CHUNK;  // ints per block of the scan kernels (common.cuh)
static_assert(kChunk == SCAN_T * SCAN_V, "the scan kernels cover SCAN_T x SCAN_V ints per block");
constexpr int kMaxParts = 4096;     // block partials the static scratch holds
constexpr int kMaxN = kMaxParts * kChunk - 1;  // 8,388,607 ints

// The scratch: block partial sums plus the total (kMaxParts + 1 ints).
static __device__ __align__(256) int g_scan_part[kMaxParts + 1];

std::mutex g_mu;
int* g_part_ptr[64];  // device address of g_scan_part, per device

// Device address of the scratch on the current device, looked up once per
// device with that device current.
cudaError_t scratch_on_current_device(int** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_part_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scan_part);
    if (e != cudaSuccess) return e;
    g_part_ptr[dev] = static_cast<int*>(p);
  }
  *out = g_part_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int avbd_exclusive_scan_noalloc(const int* in, int* out, int n, void* stream) {
  if (n < 0 || n > kMaxN) {
    set_error_text("avbd_exclusive_scan_noalloc: n must be in [0, 8388607]", cudaSuccess);
    return AVBD_E_INVALID;
  }
  if (!out || (n > 0 && !in)) {
    set_error_text("avbd_exclusive_scan_noalloc: null buffer", cudaSuccess);
    return AVBD_E_INVALID;
  }
  int* part = nullptr;
  cudaError_t e = scratch_on_current_device(&part);
  if (e != cudaSuccess) {
    set_error_text("avbd_exclusive_scan_noalloc: cudaGetSymbolAddress", e);
    return AVBD_E_CUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int np = (n + kChunk) / kChunk;  // blocks covering index n (the total)
  k_scan_reduce<<<np, SCAN_T, 0, st>>>(in, n, nullptr, part);
  k_scan_parts<<<1, SCAN_T, 0, st>>>(part, np);
  k_scan_down<<<np, SCAN_T, 0, st>>>(in, out, n, nullptr, part, np, nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error_text("avbd_exclusive_scan_noalloc: launch", e);
    return AVBD_E_CUDA;
  }
  return AVBD_OK;
}
