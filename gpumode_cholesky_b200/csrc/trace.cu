// Launch trace (b2p_trace_*): CUDA event pairs around every library launch.
#include <mutex>
#include <vector>

#include "launch.h"

namespace b2p {

namespace {
struct Entry {
  int id;
  double units;
  cudaEvent_t start, end;
};
std::mutex g_mu;
std::vector<Entry> g_entries;
int g_capacity = 0;
int g_used = 0;

const char* const kNames[kKCount] = {
    "potrf_warp32_kernel", "potrf_cta128_kernel", "copy_lower_kernel", "diag_kernel",
    "panel_kernel",        "trail_kernel",        "trail_tc_kernel",   "split_step_kernel",
    "split_update_kernel", "ragged_gather_kernel", "bwd_gemm_kernel",   "bwd_trsm_kernel",
    "bwd_sym_kernel",      "potrf_fused_kernel",  "potrf_fused_ws_kernel", "ragged_scatter_kernel", "split_wide_kernel",
    "trsv_kernel",         "gp_forward_kernel",   "gp_lbar_kernel",       "potrf_rescue_kernel"};

void free_all() {
  for (auto& e : g_entries) {
    cudaEventDestroy(e.start);
    cudaEventDestroy(e.end);
  }
  g_entries.clear();
  g_capacity = 0;
  g_used = 0;
}
}  // namespace

TraceScope::TraceScope(int kernel_id, cudaStream_t s, double units) : slot_(-1), s_(s) {
  if (g_capacity == 0) return;
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_used >= g_capacity) return;
  Entry e;
  e.id = kernel_id;
  e.units = units;
  if (cudaEventCreate(&e.start) != cudaSuccess) return;
  if (cudaEventCreate(&e.end) != cudaSuccess) {
    cudaEventDestroy(e.start);
    return;
  }
  cudaEventRecord(e.start, s);
  g_entries.push_back(e);
  slot_ = g_used++;
}

TraceScope::~TraceScope() {
  if (slot_ < 0) return;
  std::lock_guard<std::mutex> lock(g_mu);
  if (slot_ < (int)g_entries.size()) cudaEventRecord(g_entries[slot_].end, s_);
}

}  // namespace b2p

using namespace b2p;

extern "C" {

int b2p_trace_enable(int capacity) {
  std::lock_guard<std::mutex> lock(g_mu);
  free_all();
  if (capacity < 0) return set_error(B2P_ERR_INVALID_ARG, "negative trace capacity");
  g_capacity = capacity;
  g_entries.reserve(capacity);
  return B2P_OK;
}

int b2p_trace_read(int32_t* kernel_ids, float* ms, int max_entries) {
  std::lock_guard<std::mutex> lock(g_mu);
  int k = 0;
  for (auto& e : g_entries) {
    if (k >= max_entries) break;
    float t = -1.0f;
    if (cudaEventSynchronize(e.end) == cudaSuccess) cudaEventElapsedTime(&t, e.start, e.end);
    if (kernel_ids) kernel_ids[k] = e.id;
    if (ms) ms[k] = t;
    ++k;
  }
  return k;
}

int b2p_trace_read_starts(float* start_ms, int max_entries) {
  std::lock_guard<std::mutex> lock(g_mu);
  int k = 0;
  for (auto& e : g_entries) {
    if (k >= max_entries) break;
    float t = -1.0f;
    if (cudaEventSynchronize(e.start) == cudaSuccess) cudaEventElapsedTime(&t, g_entries[0].start, e.start);
    if (start_ms) start_ms[k] = t;
    ++k;
  }
  return k;
}

int b2p_trace_read_units(double* units, int max_entries) {
  std::lock_guard<std::mutex> lock(g_mu);
  int k = 0;
  for (auto& e : g_entries) {
    if (k >= max_entries) break;
    if (units) units[k] = e.units;
    ++k;
  }
  return k;
}

const char* b2p_kernel_name(int id) { return (id >= 0 && id < kKCount) ? kNames[id] : "unknown"; }

}  // extern "C"
