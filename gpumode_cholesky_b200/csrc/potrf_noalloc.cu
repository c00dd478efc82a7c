// b2p_potrf_batched_noalloc: the batched factorization for callers that
// cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they factor: code
// running inside an allocator-free region (a real-time or embedded host loop
// that must never block on the driver's allocator, a plugin whose host
// application owns every device allocation, or a pre-sized serving process
// that forbids allocation after start-up).  b2p_potrf_batched asks them for a
// workspace; this entry point does not.  The only scratch it needs (the
// per-matrix inverse of the current 64x64 diagonal block of the blocked path,
// n > 128) lives in the file-scope device array below, which every GPU that
// loads this library holds until the process exits.
//
// Limits and sharing:
//   * the scratch holds kNoAllocScratchBytes (16 MiB); a call whose path
//     needs more workspace than that is rejected with B2P_ERR_WORKSPACE
//     before anything is launched, and the message gives the largest batch
//     of that order and mode that fits.  Per matrix of order n > 128 the
//     need is 16 KiB in FP32 (the blocked path: 1024 matrices per call);
//     the tensor modes at n a multiple of 64 keep the panels' operand
//     copies, 8192 (n/64) (n/64 - 1) bytes (about 36 matrices of order 512,
//     8 of order 1024), plus 512 n bytes of panel buffers above order 1024
//     (no single matrix above order 2752 fits);
//   * every call on a device shares the one array and leaves its contents
//     behind; nothing in it has to start at zero (each block inverse is
//     written before it is read), so no clearing is needed;
//   * calls whose work overlaps on the GPU (other streams, other host
//     threads) race on the array: serialise them on one stream;
//   * the first call on each device looks up the array's device address with
//     cudaGetSymbolAddress (a host-side query, no allocation); make that first
//     call before any stream capture.  The first call that reaches the split
//     path (tensor modes above order 1024) or the FP32 path with its
//     look-ahead also creates that path's library-owned streams and events
//     once per device, so warm each path up once outside capture and outside
//     any region that must not touch the driver;
//   * the address is cached per device ordinal: after cudaDeviceReset (or
//     any other teardown of the device's primary context) it is stale, so
//     such a process must not call this entry point again.
#include <mutex>

#include "launch.h"

namespace b2p {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kNoAllocMaxDevices = 64;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};
std::mutex g_noalloc_mu;

// Device address of g_noalloc_scratch on the current device (looked up once).
int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
    return set_error(B2P_ERR_CUDA, "cannot query the current device");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return set_error(B2P_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return B2P_OK;
}
}  // namespace

}  // namespace b2p

using namespace b2p;

extern "C" {

size_t b2p_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

int b2p_potrf_batched_noalloc(const float* a, float* l, int64_t batch, int64_t n, int mode,
                              int32_t* info, void* stream) {
  const size_t need = b2p_potrf_workspace_size(batch, n, mode);
  if (need > kNoAllocScratchBytes) {
    // Largest batch of this order and mode whose workspace fits (the
    // workspace grows with the batch, so bisect on it).
    int64_t lo = 0, hi = batch;
    while (hi - lo > 1) {
      const int64_t mid = lo + (hi - lo) / 2;
      if (b2p_potrf_workspace_size(mid, n, mode) <= kNoAllocScratchBytes) lo = mid; else hi = mid;
    }
    return set_error(B2P_ERR_WORKSPACE,
                     "batch=%lld n=%lld mode 0x%x needs %zu bytes of scratch; the allocation-free entry point "
                     "holds %zu (at most %lld matrices of this order and mode per call)",
                     (long long)batch, (long long)n, mode, need, kNoAllocScratchBytes, (long long)lo);
  }
  void* scratch = nullptr;
  if (need > 0) {
    if (int st = noalloc_scratch(&scratch)) return st;
  }
  return b2p_potrf_batched(a, l, batch, n, mode, scratch, need, info, stream);
}

}  // extern "C"
