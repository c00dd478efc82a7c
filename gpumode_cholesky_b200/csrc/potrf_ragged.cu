// Ragged batches: many SPD matrices of different orders in one packed buffer.
//
// A plan (host side, built once per list of orders) sorts the matrices into
// three buckets and precomputes every launch:
//   n <= 32     one persistent warp-per-matrix launch (potrf_warp32_kernel)
//   n <= 128    one persistent CTA-per-matrix launch  (potrf_cta128_kernel)
//   n >  128    the blocked right-looking schedule over all of them at once:
//               big matrices sorted by n (descending), so the matrices still
//               active at block column k0 are a prefix of the list; each step
//               launches the diagonal kernel over that prefix and the panel /
//               trailing kernels over precomputed (matrix, tile) item lists.
//               In tensor modes matrices with n >= tc_min_n take the tcgen05
//               trailing update and the smaller ones the FP32 SIMT one (the
//               autotuner in gpumode_cholesky_b200/tuning.py picks tc_min_n).
// The plan's tables (offsets, orders, bucket lists, item lists) are copied
// to device memory once; execution then reads only device memory and never
// synchronises, so the whole ragged factorization can be captured in one
// CUDA graph and replayed.
//
// The reference has no ragged path: its dispatcher routes exact (batch, n)
// shapes (submission.py:4111-4268) and falls back to per-shape cuSOLVER.
#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "launch.h"

namespace b2p {

struct RaggedPlanImpl {
  int mode = 0;
  int tc_min_n = 0;
  int64_t count = 0;
  int64_t n_small = 0, n_mid = 0, n_big = 0;
  int max_n = 0;
  std::vector<RaggedStep> steps;       // SIMT trail items
  std::vector<RaggedStep> steps_tc;    // tcgen05 trail items (tensor modes)
  // device blob layout
  size_t off_offsets = 0, off_ns = 0, off_small = 0, off_mid = 0, off_order = 0, off_items = 0, bytes = 0;
  std::vector<unsigned char> blob;
};

static size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

}  // namespace b2p

using namespace b2p;

struct b2p_ragged_plan {
  RaggedPlanImpl impl;
};

extern "C" {

int b2p_ragged_plan_create(const int64_t* offsets_host, const int32_t* n_host, int64_t count, int mode,
                           int tc_min_n, b2p_ragged_plan** plan_out) {
  if (plan_out == nullptr) return set_error(B2P_ERR_INVALID_ARG, "null plan pointer");
  *plan_out = nullptr;
  if (count < 0 || (count > 0 && (offsets_host == nullptr || n_host == nullptr)))
    return set_error(B2P_ERR_INVALID_ARG, "bad ragged list");
  const int m = mode & B2P_MODE_MASK;
  if (m > B2P_MODE_FP8 || (mode & ~(B2P_MODE_MASK | B2P_FLAG_FP64_DIAG)))
    return set_error(B2P_ERR_INVALID_ARG, "unknown mode 0x%x", mode);
  if (m == B2P_MODE_FP8 || (mode & B2P_FLAG_FP64_DIAG))
    return set_error(B2P_ERR_UNSUPPORTED, "ragged batches support fp32, tf32 and bf16x3");
  const bool tensor = (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3);
  b2p_ragged_plan* plan = new (std::nothrow) b2p_ragged_plan;
  if (plan == nullptr) return set_error(B2P_ERR_INVALID_ARG, "out of host memory");
  RaggedPlanImpl& p = plan->impl;
  p.mode = mode;
  p.tc_min_n = tc_min_n > 0 ? tc_min_n : 256;
  p.count = count;
  std::vector<int32_t> small, mid, big;
  for (int64_t i = 0; i < count; ++i) {
    const int32_t n = n_host[i];
    if (n < 0 || n > (1 << 16) || offsets_host[i] < 0 || (offsets_host[i] & 3)) {
      delete plan;
      return set_error(B2P_ERR_INVALID_ARG, "matrix %lld: order %d / offset %lld (offsets must be multiples of 4)",
                       (long long)i, (int)n, (long long)offsets_host[i]);
    }
    if (n == 0) continue;
    (n <= 32 ? small : (n <= 128 ? mid : big)).push_back((int32_t)i);
  }
  std::stable_sort(big.begin(), big.end(), [&](int32_t x, int32_t y) { return n_host[x] > n_host[y]; });
  p.n_small = (int64_t)small.size();
  p.n_mid = (int64_t)mid.size();
  p.n_big = (int64_t)big.size();
  p.max_n = big.empty() ? 0 : n_host[big[0]];
  // Item lists per block-column step.
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
      if (R <= 0 || (tensor && n >= p.tc_min_n)) continue;
      const int T = (R + 63) / 64;
      for (int ti = 0; ti < T; ++ti)
        for (int tj = 0; tj <= ti; ++tj) items.push_back(make_int2((int)pos, ti | (tj << 16)));
    }
    st.ntrail = (int64_t)items.size() - st.trail_beg;
    stc.trail_beg = (int64_t)items.size();
    for (int64_t pos = 0; tensor && pos < nd; ++pos) {
      const int n = n_host[big[pos]];
      const int R = n - k0 - 64;
      if (R <= 0 || n < p.tc_min_n) continue;
      const int T = (R + 127) / 128;
      for (int ti = 0; ti < T; ++ti)
        for (int tj = 0; tj <= ti; ++tj) items.push_back(make_int2((int)pos, ti | (tj << 16)));
    }
    stc.ntrail = (int64_t)items.size() - stc.trail_beg;
    p.steps.push_back(st);
    p.steps_tc.push_back(stc);
  }
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
  *plan_out = plan;
  return B2P_OK;
}

void b2p_ragged_plan_destroy(b2p_ragged_plan* plan) { delete plan; }

size_t b2p_ragged_plan_table_bytes(const b2p_ragged_plan* plan) { return plan ? plan->impl.bytes : 0; }

size_t b2p_ragged_plan_workspace_bytes(const b2p_ragged_plan* plan) {
  if (plan == nullptr) return 0;
  return (size_t)plan->impl.n_big * 64 * 64 * sizeof(float);
}

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
  const size_t need = b2p_ragged_plan_workspace_bytes(plan);
  if (need > 0 && (workspace == nullptr || workspace_bytes < need))
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", need, workspace_bytes);
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
  if (p.n_big) {
    RaggedTables rt;
    rt.order = reinterpret_cast<const int32_t*>(t + p.off_order);
    rt.offsets = offsets;
    rt.ns = ns;
    rt.items = reinterpret_cast<const int2*>(t + p.off_items);
    float* tws = static_cast<float*>(workspace);
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
