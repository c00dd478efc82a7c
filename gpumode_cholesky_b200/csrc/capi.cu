// extern "C" entry points (include/b200_potrf.h) and the shape dispatcher.
//
// The dispatcher replaces the reference's exact-(batch, n) routing in
// custom_kernel (submission.py:4101-4268) by routing on n alone:
//   n <= 32    one warp per matrix            (potrf_warp32_kernel)
//   n <= 128   one CTA per matrix, in smem    (potrf_cta128_kernel)
//   n >  128   tensor modes, n % 64 == 0 (choose_path):
//                many CTAs per matrix when n > 1024 or the batch is too
//                small to fill the GPU one CTA per matrix (potrf_split);
//                else one CTA per matrix (potrf_fused / potrf_fused_ws);
//              FP32 or any other n: blocked right-looking (potrf_blocked)
// There is no CPU path and no vendor-library fallback.
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "launch.h"
#include "panel_copy.cuh"

namespace b2p {

namespace {
thread_local char g_msg[512] = "";
constexpr int kMaxDevices = 64;
int g_sms[kMaxDevices] = {0};
size_t g_smem_attr[kMaxDevices][kSlotCount] = {{0}};
std::mutex g_attr_mu;
}  // namespace

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return status;
}

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return B2P_OK;
}

static int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
  return dev;
}

int device_sms() {
  const int dev = current_device();
  if (g_sms[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    g_sms[dev] = v;
  }
  return g_sms[dev];
}

int ensure_smem_attr(const void* func, size_t bytes, int slot) {
  const int dev = current_device();
  std::lock_guard<std::mutex> lock(g_attr_mu);
  if (g_smem_attr[dev][slot] >= bytes) return B2P_OK;
  const cudaError_t e =
      cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess)
    return set_error(B2P_ERR_CUDA, "cudaFuncSetAttribute(%zu bytes): %s", bytes, cudaGetErrorString(e));
  g_smem_attr[dev][slot] = bytes;
  return B2P_OK;
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

bool path_supported(int path, int64_t batch, int64_t n, int mode) {
  switch (path) {
    case B2P_PATH_BLOCKED: return true;
    case B2P_PATH_FUSED: return fused_supported(n, mode);
    case B2P_PATH_FUSED_WS: return fused_ws_supported(batch, n, mode);
    case B2P_PATH_SPLIT: return split_supported(n, mode);
    default: return false;
  }
}

// The n > 128 algorithm for (batch, n, mode).  Tensor modes, measured on
// B200 (BF16x3): up to n = 1024 one CTA per matrix while the batch fills
// the GPU (640x512: 1225 us), else the warp-specialized kernel in clusters of
// up to 8 CTAs per matrix (60x1024: 646 us, 4x1024: 421 us); above 1024 the
// multi-CTA split path (8x2048: 1351 us).  FP32: blocked.
int choose_path(int64_t batch, int64_t n, int mode) {
  const int64_t sms = device_sms();
  if (fused_supported(n, mode)) return batch > sms ? B2P_PATH_FUSED : B2P_PATH_FUSED_WS;
  if (split_supported(n, mode)) return B2P_PATH_SPLIT;
  return B2P_PATH_BLOCKED;
}

size_t path_workspace_bytes(int path, int64_t batch, int64_t n, int mode) {
  switch (path) {
    case B2P_PATH_FUSED:
    case B2P_PATH_FUSED_WS: return fused_workspace_bytes(batch, n);
    case B2P_PATH_SPLIT: return split_workspace_bytes(batch, n);
    default: return blocked_workspace_bytes(batch, n, mode);
  }
}

int potrf_path(const float* a, float* l, int64_t batch, int n, int mode, int path, void* ws, size_t ws_bytes,
               int32_t* info, cudaStream_t s, GuardRec grd) {
  switch (path) {
    case B2P_PATH_FUSED: return potrf_fused(a, l, batch, n, mode, ws, ws_bytes, info, s, grd);
    case B2P_PATH_FUSED_WS: return potrf_fused_ws(a, l, batch, n, mode, ws, ws_bytes, info, s, grd);
    case B2P_PATH_SPLIT: return potrf_split(a, l, batch, n, mode, ws, ws_bytes, info, s, grd);
    default: return potrf_blocked(a, l, batch, n, mode, ws, ws_bytes, info, s);
  }
}

// Whether a call on `path` runs the pivot guard (and so its rescue).
static bool guarded(int path, int mode) {
  const int m = mode & B2P_MODE_MASK;
  return (mode & B2P_FLAG_GUARD) && (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3 || m == B2P_MODE_FP8) &&
         (path == B2P_PATH_FUSED || path == B2P_PATH_FUSED_WS || path == B2P_PATH_SPLIT);
}

static int check_mode(int mode) {
  const int m = mode & B2P_MODE_MASK;
  if (m > B2P_MODE_FP8 || (mode & ~(B2P_MODE_MASK | B2P_FLAG_FP64_DIAG | B2P_FLAG_GUARD)) != 0)
    return set_error(B2P_ERR_INVALID_ARG, "unknown mode 0x%x", mode);
  return B2P_OK;
}

}  // namespace b2p

using namespace b2p;

extern "C" {

int b2p_version(void) { return 100; }

const char* b2p_status_string(int status) {
  switch (status) {
    case B2P_OK: return "ok";
    case B2P_ERR_INVALID_ARG: return "invalid argument";
    case B2P_ERR_UNSUPPORTED: return "unsupported mode or size";
    case B2P_ERR_WORKSPACE: return "workspace missing or too small";
    case B2P_ERR_CUDA: return "CUDA error";
    case B2P_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
  }
}

const char* b2p_last_error(void) { return g_msg; }

size_t b2p_potrf_workspace_size(int64_t batch, int64_t n, int mode) {
  return b2p_potrf_path_workspace_size(batch, n, mode, B2P_PATH_AUTO);
}

size_t b2p_potrf_path_workspace_size(int64_t batch, int64_t n, int mode, int path) {
  if (batch <= 0 || n <= 128 || check_mode(mode) != B2P_OK) return 0;
  if (path == B2P_PATH_AUTO) path = choose_path(batch, n, mode);
  if (!path_supported(path, batch, n, mode)) return 0;
  return path_workspace_bytes(path, batch, n, mode) + (guarded(path, mode) ? guard_ws_bytes(batch, n) : 0);
}

int b2p_potrf_batched(const float* a, float* l, int64_t batch, int64_t n, int mode,
                      void* workspace, size_t workspace_bytes, int32_t* info, void* stream) {
  return b2p_potrf_batched_path(a, l, batch, n, mode, B2P_PATH_AUTO, workspace, workspace_bytes, info, stream);
}

int b2p_potrf_batched_path(const float* a, float* l, int64_t batch, int64_t n, int mode, int path,
                           void* workspace, size_t workspace_bytes, int32_t* info, void* stream) {
  return b2p_potrf_batched_ex(a, l, batch, n, mode, path, workspace, workspace_bytes, info, nullptr, stream);
}

int b2p_potrf_batched_ex(const float* a, float* l, int64_t batch, int64_t n, int mode, int path,
                         void* workspace, size_t workspace_bytes, int32_t* info, int32_t* fp32_from, void* stream) {
  g_msg[0] = '\0';
  if (int st = check_mode(mode)) return st;
  if (path < B2P_PATH_AUTO || path > B2P_PATH_SPLIT) return set_error(B2P_ERR_INVALID_ARG, "unknown path %d", path);
  if (batch < 0 || n < 0 || n > (1 << 20))
    return set_error(B2P_ERR_INVALID_ARG, "bad shape batch=%lld n=%lld", (long long)batch, (long long)n);
  if (batch == 0 || n == 0) return B2P_OK;
  if (a == nullptr || l == nullptr) return set_error(B2P_ERR_INVALID_ARG, "null matrix pointer");
  if (!aligned16(a) || !aligned16(l)) return set_error(B2P_ERR_INVALID_ARG, "buffers must be 16-byte aligned");
  const size_t bytes = (size_t)batch * (size_t)n * (size_t)n * sizeof(float);
  const char* pa = reinterpret_cast<const char*>(a);
  const char* pl = reinterpret_cast<const char*>(l);
  if (pa < pl + bytes && pl < pa + bytes) return set_error(B2P_ERR_INVALID_ARG, "input and output overlap");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool auto_path = path == B2P_PATH_AUTO;
  if (n > 128 && path == B2P_PATH_AUTO) path = choose_path(batch, n, mode);
  const bool guard = n > 128 && guarded(path, mode);
  // The guarded paths' state (first failing block column per matrix, -1
  // for none: the caller's fp32_from when given) and the rescue's barrier
  // words sit ahead of the path's own workspace.
  GuardRec grd;
  if (guard) {
    const size_t gb = guard_ws_bytes(batch, n);
    if (workspace == nullptr || workspace_bytes < gb)
      return set_error(B2P_ERR_WORKSPACE, "workspace of at least %zu bytes required, %zu given", gb, workspace_bytes);
    grd.state = fp32_from ? fp32_from : static_cast<int32_t*>(workspace);
    grd.piv = reinterpret_cast<float2*>(static_cast<uint8_t*>(workspace) + guard_piv_offset(batch));
    grd.bar = reinterpret_cast<int*>(static_cast<uint8_t*>(workspace) + gb - 256);
    workspace = static_cast<uint8_t*>(workspace) + gb;
    workspace_bytes -= gb;
  }
  if (fp32_from != nullptr && !guard) {
    // -1 everywhere (a guarded call's audit writes every matrix's entry).
    const cudaError_t e = cudaMemsetAsync(fp32_from, 0xff, (size_t)batch * sizeof(int32_t), s);
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "cudaMemsetAsync(fp32_from): %s", cudaGetErrorString(e));
  }
  if (n <= 32) return launch_warp32(a, l, dense_list(batch, (int)n), info, s);
  if (n <= 128) return launch_cta128(a, l, dense_list(batch, (int)n), info, s);
  if (!path_supported(path, batch, n, mode))
    return set_error(B2P_ERR_UNSUPPORTED, "path %d does not support n=%lld mode 0x%x", path, (long long)n, mode);
  int st = B2P_OK;
  bool done = false;
  if (auto_path && path == B2P_PATH_FUSED) {
    // One CTA per matrix runs in waves of `per` matrices; when the last wave
    // would be less than half full, those matrices run instead as clusters
    // of CTAs each (same workspace layout, so they take their own slice).
    const int64_t per = (int64_t)device_sms() * (n <= 512 ? 2 : 1);
    const int64_t tail = batch % per;
    if (batch > per && tail > 0 && tail * 2 <= per && fused_ws_supported(tail, n, mode)) {
      const int64_t head = batch - tail;
      st = potrf_fused(a, l, head, (int)n, mode, workspace, workspace_bytes, info, s, grd);
      if (st == B2P_OK) {
        const size_t moff = (size_t)head * (size_t)n * (size_t)n;
        const size_t woff = (size_t)head * 2 * panel_copy_region_bytes((int)n);
        st = potrf_fused_ws(a + moff, l + moff, tail, (int)n, mode, static_cast<uint8_t*>(workspace) + woff,
                            workspace_bytes - woff, info ? info + head : nullptr, s,
                            guard ? GuardRec{grd.piv + (size_t)head * (size_t)n, grd.state + head, grd.bar}
                                  : GuardRec());
      }
      done = true;
    }
  }
  if (!done) st = potrf_path(a, l, batch, (int)n, mode, path, workspace, workspace_bytes, info, s, grd);
  if (st != B2P_OK || !guard) return st;
  // Refactor in FP32 every matrix whose pivots failed the path's audit.
  return guard_rescue(a, l, batch, (int)n, mode, grd, info, s);
}

size_t b2p_potrf_backward_workspace_size(int64_t batch, int64_t n) {
  if (batch <= 0 || n <= 0) return 0;
  return backward_workspace_bytes(batch, n);
}

int b2p_potrf_backward(const float* l, const float* lbar, float* abar, int64_t batch, int64_t n, int mode,
                       void* workspace, size_t workspace_bytes, void* stream) {
  g_msg[0] = '\0';
  if (int st = check_mode(mode)) return st;
  if (batch < 0 || n < 0 || n > (1 << 16))
    return set_error(B2P_ERR_INVALID_ARG, "bad shape batch=%lld n=%lld", (long long)batch, (long long)n);
  if (batch == 0 || n == 0) return B2P_OK;
  if (l == nullptr || lbar == nullptr || abar == nullptr) return set_error(B2P_ERR_INVALID_ARG, "null pointer");
  const size_t bytes = (size_t)batch * (size_t)n * (size_t)n * sizeof(float);
  const char* pa = reinterpret_cast<const char*>(abar);
  const char* pl = reinterpret_cast<const char*>(l);
  const char* pg = reinterpret_cast<const char*>(lbar);
  if ((pa < pl + bytes && pl < pa + bytes) || (pa < pg + bytes && pg < pa + bytes))
    return set_error(B2P_ERR_INVALID_ARG, "abar overlaps l or lbar");
  return potrf_backward(l, lbar, abar, batch, (int)n, mode, workspace, workspace_bytes,
                        static_cast<cudaStream_t>(stream));
}

}  // extern "C"
