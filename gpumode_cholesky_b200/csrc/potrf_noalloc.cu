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
//   * the scratch holds kNoAllocScratchBytes (16 MiB); a call whose blocked
//     path needs more (batch * 16 KiB for n > 128) is rejected with
//     B2P_ERR_WORKSPACE before anything is launched;
//   * every call on a device shares the one array and leaves its contents
//     behind; nothing in it has to start at zero (each block inverse is
//     written before it is read), so no clearing is needed;
//   * calls whose work overlaps on the GPU (other streams, other host
//     threads) race on the array: serialise them on one stream;
//   * the first call on each device looks up the array's device address with
//     cudaGetSymbolAddress (a host-side query, no allocation); make that first
//     call before any stream capture.
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
  if (need > kNoAllocScratchBytes)
    return set_error(B2P_ERR_WORKSPACE,
                     "batch=%lld n=%lld needs %zu bytes of scratch; the allocation-free entry point "
                     "holds %zu (at most %zu matrices of order > 128 per call)",
                     (long long)batch, (long long)n, need, kNoAllocScratchBytes,
                     kNoAllocScratchBytes / (64 * 64 * sizeof(float)));
  void* scratch = nullptr;
  if (need > 0) {
    if (int st = noalloc_scratch(&scratch)) return st;
  }
  return b2p_potrf_batched(a, l, batch, n, mode, scratch, need, info, stream);
}

}  // extern "C"
