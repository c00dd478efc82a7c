// Ragged batches: many SPD matrices of different orders in one packed buffer.
//
// A plan (host side, built once per list of orders) sorts the matrices into
// buckets and precomputes every launch:
//   n <= 32     one persistent warp-per-matrix launch (potrf_warp32_kernel)
//   n <= 128    one persistent CTA-per-matrix launch  (potrf_cta128_kernel)
//   n >  128, tensor modes, n >= dense_min_n: padded dense groups.  Each
//               matrix is padded to p = n rounded up to the pad step (128 by
//               default; identity in the padding: the Schur complement of
//               the padded rows stays the identity, so L and info of the
//               first n rows are those of the unpadded matrix); matrices of
//               equal p form one dense batch that runs on the n > 128
//               dispatcher's path for (count, p) (potrf_fused /
//               potrf_fused_ws), above 1024 on potrf_fused_ws (or
//               potrf_split), the groups spread over several streams.  One
//               gather launch copies every such matrix into the padded
//               buffer and one scatter launch copies the factors (and info)
//               back.
//   n >  128 otherwise (FP32, or below dense_min_n): the blocked
//               right-looking schedule over all of them at once: matrices
//               sorted by n (descending), so the matrices still active at
//               block column k0 are a prefix of the list; each step launches
//               the diagonal kernel over that prefix and the panel / trailing
//               kernels over precomputed (matrix, tile) item lists.  In
//               tensor modes matrices with n >= kTrailTcMinN take the tcgen05
//               trailing update and smaller ones the FP32 SIMT one.
// The plan's tables (offsets, orders, bucket lists, item lists, gather list)
// are copied to device memory once; execution then reads only device memory
// and never synchronises, so the whole ragged factorization can be captured
// in one CUDA graph and replayed.
//
// The reference has no ragged path: its dispatcher routes exact (batch, n)
// shapes (submission.py:4111-4268) and falls back to per-shape cuSOLVER.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <numeric>
#include <vector>

#include "launch.h"

namespace b2p {

namespace {

// Defaults of the plan options, measured on B200 with the 3000-matrix
// log-uniform [16, 2048] draw (BF16x3): pad steps 128/128, warp-specialized
// groups above 1024, 4 streams: 16.7 ms; the same on one stream 23.2 ms;
// pad steps 64/64 on the split path, one stream: 30.4 ms.
constexpr int kPadStep = 128;       // padded orders are multiples of this
constexpr int kPadStepLarge = 128;  // ... above 1024
constexpr int kDefaultStreams = 4;
constexpr int kTrailTcMinN = 256;   // blocked schedule: tcgen05 trailing update from this order
constexpr int kDefaultDenseMinN = 129;
constexpr int kCopyRows = 32;       // rows per gather / scatter item
constexpr int kCopyThreads = 256;

// One matrix of the padded dense groups (device table, 32 bytes).
struct DenseEntry {
  int64_t src;  // element offset in the packed buffers
  int64_t dst;  // element offset in the padded buffers
  int32_t n;    // order
  int32_t p;    // padded order
  int32_t idx;  // matrix index (for info)
  int32_t pad;
};
static_assert(sizeof(DenseEntry) == 32, "DenseEntry layout");

// Padded copy of the lower block triangle (the 64-wide diagonal tiles whole):
// the dense kernels read block column k only from row 64k down.  Rows and
// columns >= n take the identity.  item = (entry, first row).
__global__ void __launch_bounds__(kCopyThreads) ragged_gather_kernel(const float* __restrict__ a,
                                                                      float* __restrict__ ap,
                                                                      const DenseEntry* __restrict__ ent,
                                                                      const int2* __restrict__ items, int64_t nitems) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 item = items[it];
    const DenseEntry e = ent[item.x];
    for (int rr = warp; rr < kCopyRows; rr += kCopyThreads / 32) {
      const int r = item.y + rr;
      if (r >= e.p) break;
      const int cw = min(e.p, (r / 64 + 1) * 64);
      float* dst = ap + e.dst + (int64_t)r * e.p;
      if (r < e.n) {
        const float* src = a + e.src + (int64_t)r * e.n;
        const int cn = min(cw, e.n);
#pragma unroll 4
        for (int c = lane; c < cn; c += 32) dst[c] = __ldg(src + c);
        for (int c = cn + lane; c < cw; c += 32) dst[c] = 0.0f;
      } else {
#pragma unroll 4
        for (int c = lane; c < cw; c += 32) dst[c] = (c == r) ? 1.0f : 0.0f;
      }
    }
  }
}

// Factors back into the packed layout (zeros above the diagonal), and info.
__global__ void __launch_bounds__(kCopyThreads) ragged_scatter_kernel(const float* __restrict__ lp, float* __restrict__ l,
                                                                       const DenseEntry* __restrict__ ent,
                                                                       const int2* __restrict__ items, int64_t nitems,
                                                                       const int32_t* __restrict__ ginfo,
                                                                       int32_t* __restrict__ info) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 item = items[it];
    const DenseEntry e = ent[item.x];
    if (item.y == 0 && threadIdx.x == 0 && info != nullptr) info[e.idx] = ginfo[item.x];
    for (int rr = warp; rr < kCopyRows; rr += kCopyThreads / 32) {
      const int r = item.y + rr;
      if (r >= e.n) break;
      const float* src = lp + e.dst + (int64_t)r * e.p;
      float* dst = l + e.src + (int64_t)r * e.n;
      const int cl = min(r + 1, e.n);
#pragma unroll 4
      for (int c = lane; c < cl; c += 32) dst[c] = src[c];
      for (int c = cl + lane; c < e.n; c += 32) dst[c] = 0.0f;
    }
  }
}

size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }
size_t align1k(size_t x) { return (x + 1023) & ~(size_t)1023; }

}  // namespace

struct DenseGroup {
  int p = 0;
  int path = 0;
  int stream = 0;       // 0: the caller's stream, else a library stream
  int64_t first = 0;    // first entry
  int64_t count = 0;
  int64_t elem = 0;     // element offset of the group in the padded buffers
  size_t ws_off = 0;    // dense-path workspace (offset from the dense area)
  size_t ws_bytes = 0;
};

constexpr int kRaggedMaxStreams = 8;

namespace {
// Per device: the library streams dense groups run on, with the events that
// fork them from and join them to the caller's stream.
struct GroupStreams {
  cudaStream_t st[kRaggedMaxStreams] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kRaggedMaxStreams] = {};
};
constexpr int kGroupStreamDevices = 64;
GroupStreams g_gs[kGroupStreamDevices];
std::mutex g_gs_mu;

int group_streams(GroupStreams** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kGroupStreamDevices)
    return set_error(B2P_ERR_CUDA, "no usable current device");
  std::lock_guard<std::mutex> lock(g_gs_mu);
  GroupStreams& gs = g_gs[dev];
  if (gs.fork == nullptr) {
    cudaError_t e = cudaEventCreateWithFlags(&gs.fork, cudaEventDisableTiming);
    for (int i = 1; i < kRaggedMaxStreams && e == cudaSuccess; ++i) {
      e = cudaStreamCreateWithFlags(&gs.st[i], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&gs.join[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "ragged streams: %s", cudaGetErrorString(e));
  }
  *out = &gs;
  return B2P_OK;
}
}  // namespace

struct RaggedPlanImpl {
  int mode = 0;
  int dense_min_n = 0;
  int64_t count = 0;
  int64_t n_small = 0, n_mid = 0, n_big = 0, n_dense = 0, n_items = 0;
  int max_n = 0;
  int nstreams = 1;
  std::vector<RaggedStep> steps;       // SIMT trail items
  std::vector<RaggedStep> steps_tc;    // tcgen05 trail items (tensor modes)
  std::vector<DenseGroup> groups;
  // device blob layout
  size_t off_offsets = 0, off_ns = 0, off_small = 0, off_mid = 0, off_order = 0, off_items = 0, off_dense = 0,
         off_ditems = 0, bytes = 0;
  // workspace layout (offsets from the 1024-aligned base)
  size_t ws_tws = 0, ws_ap = 0, ws_lp = 0, ws_ginfo = 0, ws_dense = 0, ws_dense_bytes = 0, ws_total = 0;
  std::vector<unsigned char> blob;
};

}  // namespace b2p

using namespace b2p;

struct b2p_ragged_plan {
  RaggedPlanImpl impl;
};

extern "C" {

int b2p_ragged_plan_create(const int64_t* offsets_host, const int32_t* n_host, int64_t count, int mode,
                           int tc_min_n, b2p_ragged_plan** plan_out) {
  b2p_ragged_options opt = {};
  opt.dense_min_n = tc_min_n;
  return b2p_ragged_plan_create_ex(offsets_host, n_host, count, mode, &opt, plan_out);
}

int b2p_ragged_plan_create_ex(const int64_t* offsets_host, const int32_t* n_host, int64_t count, int mode,
                              const b2p_ragged_options* options, b2p_ragged_plan** plan_out) {
  if (plan_out == nullptr) return set_error(B2P_ERR_INVALID_ARG, "null plan pointer");
  *plan_out = nullptr;
  b2p_ragged_options opt = {};
  if (options != nullptr) opt = *options;
  auto step_ok = [](int v) { return v == 0 || v == 64 || v == 128 || v == 256; };
  if (opt.dense_min_n < 0 || !step_ok(opt.pad_step) || !step_ok(opt.pad_step_large) ||
      (opt.large_path != B2P_PATH_AUTO && opt.large_path != B2P_PATH_SPLIT && opt.large_path != B2P_PATH_FUSED_WS) ||
      opt.streams < 0 || opt.streams > kRaggedMaxStreams)
    return set_error(B2P_ERR_INVALID_ARG,
                     "bad ragged options (pad steps 64/128/256; large path auto/split/fused_ws; streams 0..8)");
  const int step_small = opt.pad_step ? opt.pad_step : kPadStep;
  const int step_large = opt.pad_step_large ? opt.pad_step_large : kPadStepLarge;
  if (count < 0 || (count > 0 && (offsets_host == nullptr || n_host == nullptr)))
    return set_error(B2P_ERR_INVALID_ARG, "bad ragged list");
  const int m = mode & B2P_MODE_MASK;
  if (m > B2P_MODE_FP8 || (mode & ~(B2P_MODE_MASK | B2P_FLAG_FP64_DIAG | B2P_FLAG_GUARD)))
    return set_error(B2P_ERR_INVALID_ARG, "unknown mode 0x%x", mode);
  // The pivot guard is not applied to ragged batches: its FP32 rescue is a
  // cooperative launch over every SM, and the ragged groups run on several
  // streams at once.  The flag is accepted and ignored.
  mode &= ~B2P_FLAG_GUARD;
  if (m == B2P_MODE_FP8 || (mode & B2P_FLAG_FP64_DIAG))
    return set_error(B2P_ERR_UNSUPPORTED, "ragged batches support fp32, tf32 and bf16x3");
  const bool tensor = (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3);
  b2p_ragged_plan* plan = new (std::nothrow) b2p_ragged_plan;
  if (plan == nullptr) return set_error(B2P_ERR_INVALID_ARG, "out of host memory");
  RaggedPlanImpl& p = plan->impl;
  p.mode = mode;
  p.dense_min_n = opt.dense_min_n > 0 ? opt.dense_min_n : kDefaultDenseMinN;
  p.count = count;
  std::vector<int32_t> small, mid, big, dense;
  for (int64_t i = 0; i < count; ++i) {
    const int32_t n = n_host[i];
    if (n < 0 || n > (1 << 16) || offsets_host[i] < 0 || (offsets_host[i] & 3)) {
      delete plan;
      return set_error(B2P_ERR_INVALID_ARG, "matrix %lld: order %d / offset %lld (offsets must be multiples of 4)",
                       (long long)i, (int)n, (long long)offsets_host[i]);
    }
    if (n == 0) continue;
    if (n <= 32)
      small.push_back((int32_t)i);
    else if (n <= 128)
      mid.push_back((int32_t)i);
    else if (tensor && n >= p.dense_min_n)
      dense.push_back((int32_t)i);
    else
      big.push_back((int32_t)i);
  }
  std::stable_sort(big.begin(), big.end(), [&](int32_t x, int32_t y) { return n_host[x] > n_host[y]; });
  p.n_small = (int64_t)small.size();
  p.n_mid = (int64_t)mid.size();
  p.n_big = (int64_t)big.size();
  p.n_dense = (int64_t)dense.size();
  p.max_n = big.empty() ? 0 : n_host[big[0]];
  // Blocked schedule: item lists per block-column step.
  std::vector<int2> items;
  for (int k0 = 0; k0 < p.max_n; k0 += 64) {
    RaggedStep st{}, stc{};
    int64_t nd = 0;
    while (nd < (int64_t)big.size() && n_host[big[nd]] > k0) ++nd;
    st.ndiag = nd;
    stc.ndiag = 0;
    st.panel_beg = (int64_t)items.size();
    for (int64_t pos = 0; pos < nd; ++pos) {
      const int R = n_host[big[pos]] - k0 - 64;
      for (int ti = 0; R > 0 && ti < (R + 63) / 64; ++ti) items.push_back(make_int2((int)pos, ti));
    }
    st.npanel = (int64_t)items.size() - st.panel_beg;
    stc.panel_beg = st.panel_beg;
    stc.npanel = 0;
    st.trail_beg = (int64_t)items.size();
    for (int64_t pos = 0; pos < nd; ++pos) {
      const int n = n_host[big[pos]];
      const int R = n - k0 - 64;
      if (R <= 0 || (tensor && n >= kTrailTcMinN)) continue;
      const int T = (R + 63) / 64;
      for (int ti = 0; ti < T; ++ti)
        for (int tj = 0; tj <= ti; ++tj) items.push_back(make_int2((int)pos, ti | (tj << 16)));
    }
    st.ntrail = (int64_t)items.size() - st.trail_beg;
    stc.trail_beg = (int64_t)items.size();
    for (int64_t pos = 0; tensor && pos < nd; ++pos) {
      const int n = n_host[big[pos]];
      const int R = n - k0 - 64;
      if (R <= 0 || n < kTrailTcMinN) continue;
      const int T = (R + 127) / 128;
      for (int ti = 0; ti < T; ++ti)
        for (int tj = 0; tj <= ti; ++tj) items.push_back(make_int2((int)pos, ti | (tj << 16)));
    }
    stc.ntrail = (int64_t)items.size() - stc.trail_beg;
    p.steps.push_back(st);
    p.steps_tc.push_back(stc);
  }
  // Padded dense groups: by padded order, largest first.
  std::map<int, std::vector<int32_t>, std::greater<int>> by_p;
  for (int32_t i : dense) {
    const int n = n_host[i];
    const int step = n > 1024 ? step_large : step_small;
    by_p[(n + step - 1) / step * step].push_back(i);
  }
  std::vector<DenseEntry> dents;
  std::vector<int2> ditems;
  int64_t elem = 0;
  for (auto& kv : by_p) {
    DenseGroup g;
    g.p = kv.first;
    g.first = (int64_t)dents.size();
    g.count = (int64_t)kv.second.size();
    g.elem = elem;
    g.path = choose_path(g.count, g.p, mode);
    if (g.p > 1024 && opt.large_path != B2P_PATH_SPLIT && fused_ws_fits(g.count, g.p, mode))
      g.path = B2P_PATH_FUSED_WS;
    const bool ok = g.path == B2P_PATH_FUSED_WS ? fused_ws_fits(g.count, g.p, mode)
                                                 : path_supported(g.path, g.count, g.p, mode);
    if (!ok) {
      delete plan;
      return set_error(B2P_ERR_UNSUPPORTED, "no dense path for %lld matrices of padded order %d",
                       (long long)g.count, g.p);
    }
    for (int32_t i : kv.second) {
      DenseEntry e;
      e.src = offsets_host[i];
      e.dst = elem;
      e.n = n_host[i];
      e.p = g.p;
      e.idx = i;
      e.pad = 0;
      for (int r = 0; r < g.p; r += kCopyRows) ditems.push_back(make_int2((int)dents.size(), r));
      dents.push_back(e);
      elem += (int64_t)g.p * g.p;
    }
    g.ws_bytes = path_workspace_bytes(g.path, g.count, g.p, mode);
    p.groups.push_back(g);
  }
  // Streams: the largest groups first, each onto the least loaded stream
  // (work ~ count p^3); split-path groups stay on the caller's stream, since
  // their look-ahead shares one side stream per device.
  p.nstreams = std::max(1, std::min<int>(opt.streams ? opt.streams : kDefaultStreams, (int)p.groups.size()));
  {
    std::vector<double> load(p.nstreams, 0.0);
    std::vector<size_t> order(p.groups.size());
    std::iota(order.begin(), order.end(), 0);
    auto work = [&](const DenseGroup& g) { return (double)g.count * g.p * g.p * g.p; };
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t x, size_t y) { return work(p.groups[x]) > work(p.groups[y]); });
    for (size_t gi : order) {
      DenseGroup& g = p.groups[gi];
      int best = 0;
      if (g.path != B2P_PATH_SPLIT)
        for (int i = 1; i < p.nstreams; ++i)
          if (load[i] < load[best]) best = i;
      g.stream = best;
      load[best] += work(g);
    }
    std::vector<size_t> need(p.nstreams, 0), off(p.nstreams, 0);
    for (const DenseGroup& g : p.groups) need[g.stream] = std::max(need[g.stream], g.ws_bytes);
    for (int i = 0; i < p.nstreams; ++i) {
      off[i] = p.ws_dense_bytes;
      p.ws_dense_bytes = align1k(p.ws_dense_bytes + need[i]);
    }
    for (DenseGroup& g : p.groups) g.ws_off = off[g.stream];
  }
  p.n_items = (int64_t)ditems.size();
  // Workspace: blocked diagonal tiles, padded A and L, group info, dense path workspace.
  size_t w = 0;
  p.ws_tws = w;
  w = align1k(w + (size_t)p.n_big * 64 * 64 * sizeof(float));
  p.ws_ap = w;
  w = align1k(w + (size_t)elem * sizeof(float));
  p.ws_lp = w;
  w = align1k(w + (size_t)elem * sizeof(float));
  p.ws_ginfo = w;
  w = align1k(w + (size_t)p.n_dense * sizeof(int32_t));
  p.ws_dense = w;
  w = align1k(w + p.ws_dense_bytes);
  p.ws_total = (w == 0) ? 0 : w + 1024;  // slack for aligning the caller's pointer
  // Device blob.
  size_t o = 0;
  p.off_offsets = o;
  o = align16(o + sizeof(int64_t) * (size_t)count);
  p.off_ns = o;
  o = align16(o + sizeof(int32_t) * (size_t)count);
  p.off_small = o;
  o = align16(o + sizeof(int32_t) * small.size());
  p.off_mid = o;
  o = align16(o + sizeof(int32_t) * mid.size());
  p.off_order = o;
  o = align16(o + sizeof(int32_t) * big.size());
  p.off_items = o;
  o = align16(o + sizeof(int2) * items.size());
  p.off_dense = o;
  o = align16(o + sizeof(DenseEntry) * dents.size());
  p.off_ditems = o;
  o = align16(o + sizeof(int2) * ditems.size());
  p.bytes = std::max<size_t>(o, 16);
  p.blob.assign(p.bytes, 0);
  if (count) {
    std::memcpy(p.blob.data() + p.off_offsets, offsets_host, sizeof(int64_t) * (size_t)count);
    std::memcpy(p.blob.data() + p.off_ns, n_host, sizeof(int32_t) * (size_t)count);
  }
  if (!small.empty()) std::memcpy(p.blob.data() + p.off_small, small.data(), sizeof(int32_t) * small.size());
  if (!mid.empty()) std::memcpy(p.blob.data() + p.off_mid, mid.data(), sizeof(int32_t) * mid.size());
  if (!big.empty()) std::memcpy(p.blob.data() + p.off_order, big.data(), sizeof(int32_t) * big.size());
  if (!items.empty()) std::memcpy(p.blob.data() + p.off_items, items.data(), sizeof(int2) * items.size());
  if (!dents.empty()) std::memcpy(p.blob.data() + p.off_dense, dents.data(), sizeof(DenseEntry) * dents.size());
  if (!ditems.empty()) std::memcpy(p.blob.data() + p.off_ditems, ditems.data(), sizeof(int2) * ditems.size());
  *plan_out = plan;
  return B2P_OK;
}

void b2p_ragged_plan_destroy(b2p_ragged_plan* plan) { delete plan; }

size_t b2p_ragged_plan_table_bytes(const b2p_ragged_plan* plan) { return plan ? plan->impl.bytes : 0; }

size_t b2p_ragged_plan_workspace_bytes(const b2p_ragged_plan* plan) { return plan ? plan->impl.ws_total : 0; }

int b2p_ragged_plan_upload(const b2p_ragged_plan* plan, void* tables, void* stream) {
  if (plan == nullptr || tables == nullptr) return set_error(B2P_ERR_INVALID_ARG, "null plan or table buffer");
  if (reinterpret_cast<uintptr_t>(tables) & 15u) return set_error(B2P_ERR_INVALID_ARG, "tables must be 16-byte aligned");
  const cudaError_t e = cudaMemcpyAsync(tables, plan->impl.blob.data(), plan->impl.bytes, cudaMemcpyHostToDevice,
                                        static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "table upload: %s", cudaGetErrorString(e));
  // The host image must stay valid until the copy has read it.
  const cudaError_t e2 = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  if (e2 != cudaSuccess) return set_error(B2P_ERR_CUDA, "table upload: %s", cudaGetErrorString(e2));
  return B2P_OK;
}

int b2p_potrf_ragged(const b2p_ragged_plan* plan, const void* tables, const float* a, float* l, void* workspace,
                     size_t workspace_bytes, int32_t* info, void* stream) {
  if (plan == nullptr || tables == nullptr) return set_error(B2P_ERR_INVALID_ARG, "null plan or table buffer");
  const RaggedPlanImpl& p = plan->impl;
  if (p.count == 0) return B2P_OK;
  if (a == nullptr || l == nullptr || a == l) return set_error(B2P_ERR_INVALID_ARG, "bad matrix buffers");
  if ((reinterpret_cast<uintptr_t>(a) & 15u) || (reinterpret_cast<uintptr_t>(l) & 15u))
    return set_error(B2P_ERR_INVALID_ARG, "buffers must be 16-byte aligned");
  const size_t need = p.ws_total;
  if (need > 0 && (workspace == nullptr || workspace_bytes < need))
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", need, workspace_bytes);
  uint8_t* wsb = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(workspace) + 1023) & ~(uintptr_t)1023);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned char* t = static_cast<const unsigned char*>(tables);
  const int64_t* offsets = reinterpret_cast<const int64_t*>(t + p.off_offsets);
  const int32_t* ns = reinterpret_cast<const int32_t*>(t + p.off_ns);
  MatrixList ml;
  ml.offsets = offsets;
  ml.ns = ns;
  ml.n = 0;
  if (p.n_small) {
    ml.order = reinterpret_cast<const int32_t*>(t + p.off_small);
    ml.count = p.n_small;
    if (int st = launch_warp32(a, l, ml, info, s)) return st;
  }
  if (p.n_mid) {
    ml.order = reinterpret_cast<const int32_t*>(t + p.off_mid);
    ml.count = p.n_mid;
    if (int st = launch_cta128(a, l, ml, info, s)) return st;
  }
  if (p.n_dense) {
    const DenseEntry* ents = reinterpret_cast<const DenseEntry*>(t + p.off_dense);
    const int2* ditems = reinterpret_cast<const int2*>(t + p.off_ditems);
    float* ap = reinterpret_cast<float*>(wsb + p.ws_ap);
    float* lp = reinterpret_cast<float*>(wsb + p.ws_lp);
    int32_t* ginfo = reinterpret_cast<int32_t*>(wsb + p.ws_ginfo);
    const int grid = (int)std::min<int64_t>(p.n_items, (int64_t)device_sms() * (2048 / kCopyThreads));
    {
      TraceScope ts(kKRaggedGather, s);
      ragged_gather_kernel<<<grid, kCopyThreads, 0, s>>>(a, ap, ents, ditems, p.n_items);
      if (int st = check_launch("ragged_gather_kernel")) return st;
    }
    GroupStreams* gs = nullptr;
    auto check = [](cudaError_t e, const char* what) -> int {
      return e == cudaSuccess ? B2P_OK : set_error(B2P_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    };
    if (p.nstreams > 1) {
      if (int st = group_streams(&gs)) return st;
      if (int st = check(cudaEventRecord(gs->fork, s), "cudaEventRecord")) return st;
      for (int i = 1; i < p.nstreams; ++i)
        if (int st = check(cudaStreamWaitEvent(gs->st[i], gs->fork, 0), "cudaStreamWaitEvent")) return st;
    }
    for (const DenseGroup& g : p.groups) {
      cudaStream_t gst = g.stream == 0 ? s : gs->st[g.stream];
      if (int st = potrf_path(ap + g.elem, lp + g.elem, g.count, g.p, p.mode, g.path, wsb + p.ws_dense + g.ws_off,
                              g.ws_bytes, info ? ginfo + g.first : nullptr, gst))
        return st;
    }
    for (int i = 1; i < p.nstreams; ++i) {
      if (int st = check(cudaEventRecord(gs->join[i], gs->st[i]), "cudaEventRecord")) return st;
      if (int st = check(cudaStreamWaitEvent(s, gs->join[i], 0), "cudaStreamWaitEvent")) return st;
    }
    {
      TraceScope ts(kKRaggedScatter, s);
      ragged_scatter_kernel<<<grid, kCopyThreads, 0, s>>>(lp, l, ents, ditems, p.n_items, ginfo, info);
      if (int st = check_launch("ragged_scatter_kernel")) return st;
    }
  }
  if (p.n_big) {
    RaggedTables rt;
    rt.order = reinterpret_cast<const int32_t*>(t + p.off_order);
    rt.offsets = offsets;
    rt.ns = ns;
    rt.items = reinterpret_cast<const int2*>(t + p.off_items);
    float* tws = reinterpret_cast<float*>(wsb + p.ws_tws);
    for (size_t si = 0; si < p.steps.size(); ++si) {
      const int k0 = (int)si * 64;
      if (int st = ragged_blocked_step(a, l, rt, p.steps[si], k0, B2P_MODE_FP32, tws, info, s)) return st;
      const RaggedStep& tc = p.steps_tc[si];
      if (tc.ntrail > 0) {
        const float* src = (k0 == 0) ? a : l;
        Sched sr = ragged_sched(rt, rt.items + tc.trail_beg, tc.ntrail);
        if (int st = launch_syrk_tc(src, l, sr, true, 0, k0, p.mode, info, s)) return st;
      }
    }
  }
  return B2P_OK;
}

}  // extern "C"
