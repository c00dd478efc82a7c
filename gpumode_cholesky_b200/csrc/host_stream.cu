// Host-resident batches: b2p_potrf_batched_host streams a (batch, n, n) FP32
// batch from host memory through the device and back in chunks.  Three
// engines work at once: the copy-in stream loads chunk i+1, the caller's
// stream factors chunk i (b2p_potrf_batched), the copy-out stream stores
// chunk i-1.  PCIe is full duplex, so a call costs about one direction's
// transfer time plus one chunk, not the sum of both directions.
//
// Device workspace: two input and two output chunk buffers (one each when
// the batch fits one chunk), then the factorization's own workspace for the
// largest chunk.  Buffer b is reused by chunk i once chunk i-2 is done with
// it: the copy-in waits until chunk i-2 is factored, the factorization
// waits until chunk i-2 is stored.
#include <algorithm>
#include <mutex>

#include "launch.h"

namespace b2p {
namespace {

constexpr size_t kChunkTarget = 32ull << 20;  // default bytes per chunk
constexpr size_t kChunkMin = 4ull << 20;      // smallest default chunk
constexpr int kHostDevices = 64;

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

struct HostLayout {
  int64_t chunk = 0;    // matrices per chunk (the last may hold fewer)
  int64_t nchunks = 0;
  int nbuf = 0;         // chunk buffers per direction (1 or 2)
  size_t buf_bytes = 0; // one chunk buffer, 256-byte multiple
  size_t potrf_off = 0;
  size_t potrf_bytes = 0;
  size_t total = 0;
};

HostLayout host_layout(int64_t batch, int64_t n, int mode, int64_t chunk) {
  HostLayout h;
  const size_t mat = (size_t)n * (size_t)n * sizeof(float);
  if (chunk <= 0) {
    // About kChunkTarget per chunk and at least four chunks, so that the
    // last chunk's factorization and copy out (the part nothing overlaps)
    // stay short; never below kChunkMin, where copies get inefficient.
    const size_t total = (size_t)batch * mat;
    const size_t target = std::max(kChunkMin, std::min(kChunkTarget, total / 4));
    chunk = (int64_t)std::max<size_t>(1, target / mat);
  }
  h.chunk = std::min(chunk, batch);
  h.nchunks = (batch + h.chunk - 1) / h.chunk;
  h.nbuf = h.nchunks > 1 ? 2 : 1;
  h.buf_bytes = align256((size_t)h.chunk * mat);
  const int64_t last = batch - (h.nchunks - 1) * h.chunk;
  h.potrf_bytes = std::max(b2p_potrf_workspace_size(h.chunk, n, mode), b2p_potrf_workspace_size(last, n, mode));
  h.potrf_off = (size_t)2 * h.nbuf * h.buf_bytes;
  h.total = h.potrf_off + align256(h.potrf_bytes);
  return h;
}

// Per device: the copy streams and the events that order the chunks.
struct HostPipe {
  cudaStream_t in = nullptr;
  cudaStream_t out = nullptr;
  cudaEvent_t fork = nullptr;
  cudaEvent_t join = nullptr;
  cudaEvent_t loaded[2] = {nullptr, nullptr};
  cudaEvent_t factored[2] = {nullptr, nullptr};
  cudaEvent_t stored[2] = {nullptr, nullptr};
};
HostPipe g_pipe[kHostDevices];
std::mutex g_pipe_mu;  // held while a call enqueues (the events are shared)

// Caller holds g_pipe_mu.
int host_pipe(HostPipe** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kHostDevices)
    return set_error(B2P_ERR_CUDA, "no usable current device");
  HostPipe& p = g_pipe[dev];
  if (p.in == nullptr) {
    cudaError_t e = cudaStreamCreateWithFlags(&p.in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p.out, cudaStreamNonBlocking);
    cudaEvent_t* evs[] = {&p.fork, &p.join, &p.loaded[0], &p.loaded[1], &p.factored[0],
                          &p.factored[1], &p.stored[0], &p.stored[1]};
    for (cudaEvent_t* ev : evs)
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "host copy streams: %s", cudaGetErrorString(e));
  }
  *out = &p;
  return B2P_OK;
}

int check(cudaError_t e, const char* what) {
  return e == cudaSuccess ? B2P_OK : set_error(B2P_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace
}  // namespace b2p

using namespace b2p;

extern "C" {

size_t b2p_potrf_host_workspace_size(int64_t batch, int64_t n, int mode, int64_t chunk) {
  if (batch <= 0 || n <= 0 || n > (1 << 20) || chunk < 0) return 0;
  return host_layout(batch, n, mode, chunk).total;
}

int b2p_potrf_batched_host(const float* host_a, float* host_l, int64_t batch, int64_t n, int mode, int64_t chunk,
                           void* workspace, size_t workspace_bytes, int32_t* info, void* stream) {
  set_error(B2P_OK, "%s", "");
  if (batch < 0 || n < 0 || n > (1 << 20) || chunk < 0)
    return set_error(B2P_ERR_INVALID_ARG, "bad shape batch=%lld n=%lld chunk=%lld", (long long)batch, (long long)n,
                     (long long)chunk);
  if ((mode & ~(B2P_MODE_MASK | B2P_FLAG_FP64_DIAG | B2P_FLAG_GUARD)) != 0 || (mode & B2P_MODE_MASK) > B2P_MODE_FP8)
    return set_error(B2P_ERR_INVALID_ARG, "unknown mode 0x%x", mode);
  if (batch == 0 || n == 0) return B2P_OK;
  if (host_a == nullptr || host_l == nullptr) return set_error(B2P_ERR_INVALID_ARG, "null matrix pointer");
  const size_t mat_floats = (size_t)n * (size_t)n;
  const size_t bytes = (size_t)batch * mat_floats * sizeof(float);
  const char* pa = reinterpret_cast<const char*>(host_a);
  const char* pl = reinterpret_cast<const char*>(host_l);
  if (pa < pl + bytes && pl < pa + bytes) return set_error(B2P_ERR_INVALID_ARG, "input and output overlap");
  const HostLayout h = host_layout(batch, n, mode, chunk);
  if (workspace == nullptr || workspace_bytes < h.total)
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", h.total, workspace_bytes);
  if ((reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
    return set_error(B2P_ERR_INVALID_ARG, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  void* potrf_ws = h.potrf_bytes ? ws + h.potrf_off : nullptr;

  std::lock_guard<std::mutex> lock(g_pipe_mu);  // also guards the first call's stream set-up
  HostPipe* p = nullptr;
  if (int st = host_pipe(&p)) return st;
  // The copy streams start after the work already on the caller's stream
  // (it may still use the workspace or the host buffers).
  if (int st = check(cudaEventRecord(p->fork, s), "cudaEventRecord")) return st;
  if (int st = check(cudaStreamWaitEvent(p->in, p->fork, 0), "cudaStreamWaitEvent")) return st;
  if (int st = check(cudaStreamWaitEvent(p->out, p->fork, 0), "cudaStreamWaitEvent")) return st;
  int status = B2P_OK;
  for (int64_t i = 0; i < h.nchunks && status == B2P_OK; ++i) {
    const int b = (int)(i % h.nbuf);
    const int64_t first = i * h.chunk;
    const int64_t cnt = std::min(h.chunk, batch - first);
    const size_t cbytes = (size_t)cnt * mat_floats * sizeof(float);
    float* din = reinterpret_cast<float*>(ws + (size_t)b * h.buf_bytes);
    float* dout = reinterpret_cast<float*>(ws + (size_t)(h.nbuf + b) * h.buf_bytes);
    // Copy in: buffer b is free once chunk i - nbuf is factored.
    if (i >= h.nbuf) status = check(cudaStreamWaitEvent(p->in, p->factored[b], 0), "cudaStreamWaitEvent");
    if (status == B2P_OK)
      status = check(cudaMemcpyAsync(din, host_a + (size_t)first * mat_floats, cbytes, cudaMemcpyHostToDevice, p->in),
                     "cudaMemcpyAsync(host to device)");
    if (status == B2P_OK) status = check(cudaEventRecord(p->loaded[b], p->in), "cudaEventRecord");
    // Factor on the caller's stream: output buffer b is free once chunk
    // i - nbuf is stored.
    if (status == B2P_OK) status = check(cudaStreamWaitEvent(s, p->loaded[b], 0), "cudaStreamWaitEvent");
    if (status == B2P_OK && i >= h.nbuf) status = check(cudaStreamWaitEvent(s, p->stored[b], 0), "cudaStreamWaitEvent");
    if (status == B2P_OK)
      status = b2p_potrf_batched(din, dout, cnt, n, mode, potrf_ws, h.potrf_bytes, info ? info + first : nullptr, s);
    if (status == B2P_OK) status = check(cudaEventRecord(p->factored[b], s), "cudaEventRecord");
    // Copy out.
    if (status == B2P_OK) status = check(cudaStreamWaitEvent(p->out, p->factored[b], 0), "cudaStreamWaitEvent");
    if (status == B2P_OK)
      status = check(cudaMemcpyAsync(host_l + (size_t)first * mat_floats, dout, cbytes, cudaMemcpyDeviceToHost, p->out),
                     "cudaMemcpyAsync(device to host)");
    if (status == B2P_OK) status = check(cudaEventRecord(p->stored[b], p->out), "cudaEventRecord");
  }
  // Both copy streams rejoin the caller's stream, also after an error, so
  // that nothing the caller enqueues next races with a copy in flight.
  for (cudaStream_t side : {p->in, p->out}) {
    if (cudaEventRecord(p->join, side) == cudaSuccess) cudaStreamWaitEvent(s, p->join, 0);
  }
  return status;
}

}  // extern "C"
