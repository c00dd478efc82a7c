// Multi-CTA left-looking factorization on the tensor cores.
//
// For orders too large for one CTA per matrix (n > 1024), and for batches too
// small to fill the GPU that way, each block column k (k0 = 64k) of every
// matrix is produced by two launches that spread it over the whole GPU:
//
//   split_update_kernel     one thread-block cluster per (matrix, row tile t
//       of 128 rows starting at r0 = k0 + 128t), one CTA per K segment s (a
//       slice of a range of earlier block columns; split-K, so a late
//       column's long K runs on many SMs).  CTA s computes
//           U_s = L[r0:r0+128, cols of s] * L[k0:k0+64, cols of s]^T
//       on tcgen05 from the panel copies (panel_copy.cuh), streamed by one
//       thread with bulk copies through a two-stage ring, into a 128x64 FP32
//       TMEM accumulator; the epilogue parks U_s in its shared memory, and
//       after a cluster barrier the CTAs together form
//           P = base[r0:r0+128] - U_0 - U_1 - ...
//       (fixed order, read over distributed shared memory) into a per-matrix
//       FP32 panel buffer; base is A's block column or, for the second of a
//       column's two update launches, the panel buffer itself (see the
//       schedule above potrf_split).
//   split_step_kernel(k)    G CTAs per matrix.  Every CTA factors the
//       diagonal block P[k0:k0+64] in shared memory (diag64_factor) --
//       redundantly, which costs one diagonal engine per CTA but no extra
//       launch or grid-wide wait -- then solves its rows of the panel by
//       forward substitution, one row per thread (X L_kk^T = P, FP32), and
//       writes L and the panel copy of X.  CTA 0 of the matrix writes L_kk and
//       info; the zero strip right of the diagonal block is shared out.
//
// A is read once and L written once; the panel copies (4 bytes per element
// in either mode) are the only re-read data and mostly hit L2.  Results are
// deterministic (the split of each update is fixed by the shapes).  All waits are bounded; a timeout marks the matrix with
// info = -1.
//
// The reference runs its large orders left-looking through cuBLAS/cuSOLVER
// (submission.py:3319-3409 _left_looking_large, 3606-3676 FP16 shadow,
// 5152-5196 e62 diag-128 blocks with an inverse panel multiply).
#include <algorithm>
#include <mutex>

#include "diag64.cuh"
#include "launch.h"
#include "panel_copy.cuh"
#include "umma.cuh"

namespace b2p {

constexpr int kSplitSegCap = 8;  // most K segments per column (= cluster size)
constexpr uint32_t kSplitPolls = 1u << 24;

// ---- update kernel -----------------------------------------------------------
constexpr int kUThreads = 128;
constexpr uint32_t kUStageA = 32768;  // 128 rows x 2 regions
constexpr uint32_t kUStage = kUStageA + 16384;
constexpr uint32_t kUStaging = 2 * kUStage;
constexpr int kUParkLd = 68;  // parked accumulator: [128][kUParkLd] FP32 in the staging area
constexpr uint32_t kUSmemBytes = kUStaging + 128 + 1024;
constexpr uint32_t kUTmemCols = 64;
static_assert(128 * kUParkLd * 4 <= kUStaging, "parked accumulator must fit the staging area");

// Grid: one cluster of `segs` CTAs per (matrix, row tile); the cluster id
// enumerates (b, t) with t fastest.
// P = base - sum over the panels [c_begin, c_end) of block column k, where
// base element (r, c) of matrix b is base[b * base_mstride + r * base_ld + c]
// (A at column k0, or a panel buffer updated in place).
template <int MODE>
__global__ void __launch_bounds__(kUThreads, 2)
    split_update_kernel(const float* base, int64_t base_mstride, int base_ld, const uint8_t* __restrict__ ws,
                        float* pout, int n, int k, int c_begin, int c_end, int segs, int32_t* __restrict__ info) {
  extern __shared__ unsigned char uraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(uraw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kUStaging);  // [2]
  uint64_t* empty = full + 2;                                     // [2]
  uint64_t* done = full + 4;                                      // [1]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kUStaging + 48);
  int* flag = reinterpret_cast<int*>(sm + kUStaging + 56);
  float* park = reinterpret_cast<float*>(sm);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = n / 64, k0 = 64 * k;
  const int tiles = (n - k0 + 127) / 128;
  const size_t rbytes = panel_copy_region_bytes(n);
  const int s = (int)umma::cluster_rank();
  const int64_t bt = blockIdx.x / segs;
  const int t = (int)(bt % tiles);
  const int64_t b = bt / tiles;
  const int span = c_end - c_begin;
  const int c_lo = c_begin + s * span / segs, c_hi = c_begin + (s + 1) * span / segs;
  const int iters = c_hi - c_lo;
  const int r0 = k0 + 128 * t, vr = min(128, n - r0);
  const uint8_t* W0 = ws + (size_t)b * 2 * rbytes;
  const uint8_t* W1 = W0 + rbytes;

  if (tid == 0) *flag = 0;
  if (warp == 0) {
    umma::tmem_alloc(tslot, kUTmemCols);
    umma::tmem_relinquish();
  }
  if (tid == 32) {
    for (int i = 0; i < 5; ++i) umma::mbar_init(full + i, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;

  if (tid == 0) {
    bool ok = true;
    uint32_t ph_full[2] = {0u, 0u};
    uint32_t n_empty[2] = {0u, 0u};
    auto load = [&](int i, int st) {
      const int c = c_lo + i;
      const uint32_t abytes = (uint32_t)vr * 128u;
      const size_t aoff = panel_copy_row_byte(N, c, r0);
      const size_t boff = panel_copy_row_byte(N, c, k0);
      uint8_t* dst = sm + st * kUStage;
      umma::mbar_arrive_expect_tx(full + st, 2 * abytes + 2 * 8192u);
      umma::bulk_g2s(dst, W0 + aoff, abytes, full + st);
      umma::bulk_g2s(dst + 16384, W1 + aoff, abytes, full + st);
      umma::bulk_g2s(dst + kUStageA, W0 + boff, 8192u, full + st);
      umma::bulk_g2s(dst + kUStageA + 8192, W1 + boff, 8192u, full + st);
    };
    int loaded = 0, waited = 0;
    load(0, 0);
    ++loaded;
    if (iters > 1) {
      load(1, 1);
      ++loaded;
    }
    for (int i = 0; i < iters; ++i) {
      const int st = i & 1;
      if (!umma::mbar_wait_bounded(full + st, ph_full[st], kSplitPolls)) {
        ok = false;
        break;
      }
      ph_full[st] ^= 1u;
      ++waited;
      umma::fence_after_sync();
      const uint32_t sa = umma::smem_u32(sm + st * kUStage);
      panel_copy_mmas<MODE>(tmem, sa, sa + kUStageA, i > 0);
      umma::mma_commit(empty + st);
      ++n_empty[st];
      if (i + 2 < iters) {
        // Stage st is reused only once the MMAs reading it have completed.
        if (!umma::mbar_wait_bounded(empty + st, (n_empty[st] - 1u) & 1u, kSplitPolls)) {
          ok = false;
          break;
        }
        load(i + 2, st);
        ++loaded;
      }
    }
    if (!ok) {
      // Let copies still in flight land before the staging area is reused.
      for (int i = waited; i < loaded; ++i) {
        const int st = i & 1;
        if (umma::mbar_wait_bounded(full + st, ph_full[st], kSplitPolls)) ph_full[st] ^= 1u;
      }
      *flag = 1;
    }
    umma::mma_commit(done);
  }
  const bool got = umma::mbar_wait_bounded(done, 0u, kSplitPolls);
  umma::fence_after_sync();
  if (!got) *flag = 1;
  __syncthreads();
  const bool ok = *flag == 0;
  if (ok) {
    // Park U_s: thread -> accumulator row (TMEM lane) 32w + lane.
    const int rl = 32 * warp + lane;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float d[32];
      umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * h), d);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        *reinterpret_cast<float4*>(park + rl * kUParkLd + 32 * h + 4 * q) =
            make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
    }
  } else if (tid == 0 && info != nullptr) {
    info[b] = -1;
  }
  umma::fence_before_sync();
  umma::cluster_sync();
  // Every CTA of the cluster takes a share of the 128 x 16 float4 of P and
  // sums the parked accumulators of all segments in segment order.
  if (ok) {
    const float* B = base + (size_t)b * base_mstride;
    float* P = pout + (size_t)b * n * 64;
    for (int e = s * kUThreads + tid; e < vr * 16; e += segs * kUThreads) {
      const int row = e >> 4, c4 = (e & 15) * 4;
      float4 v = *reinterpret_cast<const float4*>(B + (size_t)(r0 + row) * base_ld + c4);
      for (int q = 0; q < segs; ++q) {
        const float4 u = umma::ld_cluster_f4(park + row * kUParkLd + c4, (uint32_t)q);
        v.x -= u.x;
        v.y -= u.y;
        v.z -= u.z;
        v.w -= u.w;
      }
      *reinterpret_cast<float4*>(P + (size_t)(r0 + row) * 64 + c4) = v;
    }
  }
  // No CTA leaves while another may still read its parked accumulator.
  umma::cluster_sync();
  if (!got) umma::mbar_wait_bounded(done, 0u, kSplitPolls);
  umma::fence_after_sync();
  if (warp == 0) umma::tmem_dealloc(tmem, kUTmemCols);
}

// ---- step kernel -------------------------------------------------------------
constexpr int kSThreads = 128;
constexpr uint32_t kSSmemBytes = (uint32_t)sizeof(Diag64Smem) + 128;

// Rows of the panel below the diagonal block are handled in chunks of
// kSThreads rows, chunk q = rows k0 + 64 + 128 q ..; CTA g of the matrix
// takes chunks g, g + G, ...  P comes from A (k == 0) or the panel buffer.
template <int MODE>
__global__ void __launch_bounds__(kSThreads, 4)
    split_step_kernel(const float* __restrict__ a, float* __restrict__ l, uint8_t* __restrict__ ws,
                      const float* __restrict__ pbuf, int64_t batch, int n, int k, int G,
                      int32_t* __restrict__ info) {
  extern __shared__ unsigned char sraw[];
  Diag64Smem& dg =
      *reinterpret_cast<Diag64Smem*>((reinterpret_cast<uintptr_t>(sraw) + 127) & ~(uintptr_t)127);
  const int tid = threadIdx.x;
  const int N = n / 64, k0 = 64 * k;
  const int chunks = (n - k0 - 64 + kSThreads - 1) / kSThreads;
  const size_t rbytes = panel_copy_region_bytes(n);
  const size_t n2 = (size_t)n * n;

  for (int64_t job = blockIdx.x; job < batch * G; job += gridDim.x) {
    const int64_t b = job / G;
    const int g = (int)(job - b * G);
    float* L = l + (size_t)b * n2;
    uint8_t* W0 = ws + (size_t)b * 2 * rbytes;
    uint8_t* W1 = W0 + rbytes;
    // Row r, column k0 + c of P is psrc[r * pld + c].
    const float* psrc = (k == 0) ? a + (size_t)b * n2 + k0 : pbuf + (size_t)b * n * 64;  // pbuf: this column's buffer
    const size_t pld = (k == 0) ? (size_t)n : 64;

    for (int e = tid; e < 64 * 16; e += kSThreads) {
      const int r = e >> 4, c = (e & 15) * 4;
      *reinterpret_cast<float4*>(dg.S + r * kD64Ld + c) =
          *reinterpret_cast<const float4*>(psrc + (size_t)(k0 + r) * pld + c);
    }
    __syncthreads();
    const int bad = diag64_factor(dg);
    if (g == 0) {
      for (int e = tid; e < 64 * 16; e += kSThreads) {
        const int r = e >> 4, c = (e & 15) * 4;
        const float* srow = dg.S + r * kD64Ld + c;
        *reinterpret_cast<float4*>(L + (size_t)(k0 + r) * n + k0 + c) =
            make_float4(c <= r ? srow[0] : 0.f, c + 1 <= r ? srow[1] : 0.f, c + 2 <= r ? srow[2] : 0.f,
                        c + 3 <= r ? srow[3] : 0.f);
      }
      if (tid == 0 && info != nullptr) {
        if (bad == kDiagTimeout)
          info[b] = -1;
        else if (k == 0)
          info[b] = bad >= 0 ? bad + 1 : 0;
        else if (bad >= 0 && info[b] == 0)
          info[b] = k0 + bad + 1;
      }
    }
    // Zero strip right of the diagonal block, shared by the matrix's CTAs.
    {
      const int s4 = (n - k0 - 64) >> 2;
      const int64_t total = (int64_t)64 * s4;
      for (int64_t e = (int64_t)g * kSThreads + tid; e < total; e += (int64_t)G * kSThreads) {
        const int r = (int)(e / s4), q = (int)(e - (int64_t)r * s4);
        reinterpret_cast<float4*>(L + (size_t)(k0 + r) * n + k0 + 64)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    // Panel rows: X L_kk^T = P, one row per thread.
    for (int q = g; q < chunks; q += G) {
      const int r = k0 + 64 + q * kSThreads + tid;
      if (r < n) {
        float x[64];
        const float4* src = reinterpret_cast<const float4*>(psrc + (size_t)r * pld);
#pragma unroll
        for (int c4 = 0; c4 < 16; ++c4) {
          const float4 v = src[c4];
          x[4 * c4 + 0] = v.x;
          x[4 * c4 + 1] = v.y;
          x[4 * c4 + 2] = v.z;
          x[4 * c4 + 3] = v.w;
        }
        panel_solve64(x, dg);
        float4* dst = reinterpret_cast<float4*>(L + (size_t)r * n + k0);
#pragma unroll
        for (int c4 = 0; c4 < 16; ++c4) dst[c4] = make_float4(x[4 * c4], x[4 * c4 + 1], x[4 * c4 + 2], x[4 * c4 + 3]);
        if (k + 1 < N) {
#pragma unroll
          for (int c8 = 0; c8 < 8; ++c8) {
            const float v[8] = {x[8 * c8],     x[8 * c8 + 1], x[8 * c8 + 2], x[8 * c8 + 3],
                                x[8 * c8 + 4], x[8 * c8 + 5], x[8 * c8 + 6], x[8 * c8 + 7]};
            panel_copy_store<MODE>(W0, W1, N, k, r, c8, v);
          }
        }
      }
    }
    // dg is rewritten by the next job.
    __syncthreads();
  }
}

// ---- host side -----------------------------------------------------------------

bool split_supported(int64_t n, int mode) {
  const int m = mode & B2P_MODE_MASK;
  return (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3) && !(mode & B2P_FLAG_FP64_DIAG) && n > 128 &&
         (n % 64) == 0 && n <= 65536;
}

// Panel copies, then two per-matrix FP32 panel buffers (n x 64 each; block
// columns alternate between them).
size_t split_workspace_bytes(int64_t batch, int64_t n) {
  return (size_t)batch * 2 * panel_copy_region_bytes((int)n) + 2 * (size_t)batch * n * 64 * sizeof(float) + 1024;
}

namespace {
// Per device: a second stream for the look-ahead part of the updates and
// the events that fork it from and join it to the caller's stream.
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[2] = {nullptr, nullptr};
};
constexpr int kSideDevices = 64;
SideStream g_side[kSideDevices];
std::mutex g_side_mu;

int side_stream(SideStream** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kSideDevices)
    return set_error(B2P_ERR_CUDA, "no usable current device");
  std::lock_guard<std::mutex> lock(g_side_mu);
  SideStream& ss = g_side[dev];
  if (ss.stream == nullptr) {
    cudaError_t e = cudaStreamCreateWithFlags(&ss.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss.join[0], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss.join[1], cudaEventDisableTiming);
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "side stream set-up: %s", cudaGetErrorString(e));
  }
  *out = &ss;
  return B2P_OK;
}
}  // namespace

// Schedule.  Block column j needs every earlier panel.  Panels 0..j-2 are
// final one step early, so their part of the update ("look-ahead", into the
// panel buffer of j) runs on the side stream while step j-1 runs; on the
// caller's stream only the newest panel j-1 ("tail") sits between step j-1
// and step j:
//   caller: tail(j) -> step(j) -> [fork] -> tail(j+1) -> step(j+1) -> ...
//   side:                          look-ahead(j+2) over panels 0..j
// tail(j) waits for look-ahead(j) (join event j % 2).  Column j uses panel
// buffer j % 2, which look-ahead(j+2) may only overwrite after step(j).
int potrf_split(const float* a, float* l, int64_t batch, int n, int mode, void* ws, size_t ws_bytes,
                int32_t* info, cudaStream_t s) {
  const size_t need = split_workspace_bytes(batch, n);
  if (ws == nullptr || ws_bytes < need)
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", need, ws_bytes);
  SideStream* side = nullptr;
  if (int st = side_stream(&side)) return st;
  uint8_t* copies = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(ws) + 1023) & ~(uintptr_t)1023);
  float* pb[2];
  pb[0] = reinterpret_cast<float*>(copies + (size_t)batch * 2 * panel_copy_region_bytes(n));
  pb[1] = pb[0] + (size_t)batch * n * 64;
  const int64_t sms = device_sms();
  const bool tf32 = (mode & B2P_MODE_MASK) == B2P_MODE_TF32;
  auto upd = tf32 ? split_update_kernel<B2P_MODE_TF32> : split_update_kernel<B2P_MODE_BF16X3>;
  auto stp = tf32 ? split_step_kernel<B2P_MODE_TF32> : split_step_kernel<B2P_MODE_BF16X3>;
  if (int st = ensure_smem_attr((const void*)upd, kUSmemBytes, tf32 ? kSlotSplitU0 : kSlotSplitU1)) return st;
  if (int st = ensure_smem_attr((const void*)stp, kSSmemBytes, tf32 ? kSlotSplitS0 : kSlotSplitS1)) return st;
  const int N = n / 64;
  const int64_t n2 = (int64_t)n * n;

  // Update of column k over panels [c0, c1) on stream `st`: P = base - sum,
  // split into about per_sm CTAs per SM.
  auto launch_update = [&](int k, int c0, int c1, const float* base, int64_t mstride, int ld, float* pout,
                           cudaStream_t st, int per_sm) -> int {
    const int tiles = (n - 64 * k + 127) / 128;
    const int64_t want = per_sm * sms / (batch * tiles);
    const int segs =
        (int)std::max<int64_t>(1, std::min<int64_t>({want, (int64_t)kSplitSegCap, (int64_t)(c1 - c0)}));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(batch * tiles * segs), 1, 1);
    cfg.blockDim = dim3(kUThreads, 1, 1);
    cfg.dynamicSmemBytes = kUSmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)segs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TraceScope ts(kKSplitUpdate, st);
    const cudaError_t e = cudaLaunchKernelEx(&cfg, upd, base, mstride, ld, (const uint8_t*)copies, pout, n, k,
                                             c0, c1, segs, info);
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "split_update_kernel: %s", cudaGetErrorString(e));
    return B2P_OK;
  };
  auto check = [](cudaError_t e, const char* what) -> int {
    return e == cudaSuccess ? B2P_OK : set_error(B2P_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  };

  for (int k = 0; k < N; ++k) {
    const int k0 = 64 * k;
    float* pk = pb[k & 1];
    if (k >= 1) {
      // Tail: panel k-1, onto the look-ahead result (k >= 2) or onto A.
      if (k >= 2) {
        if (int st = check(cudaStreamWaitEvent(s, side->join[k & 1], 0), "cudaStreamWaitEvent")) return st;
        if (int st = launch_update(k, k - 1, k, pk, (int64_t)n * 64, 64, pk, s, 2)) return st;
      } else {
        if (int st = launch_update(k, k - 1, k, a + k0, n2, n, pk, s, 2)) return st;
      }
    }
    // Step: CTAs per matrix for about four CTAs per SM in total.
    const int chunks = (n - k0 - 64 + kSThreads - 1) / kSThreads;
    const int G = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(chunks, 1), 4 * sms / batch));
    const int grid = (int)std::min<int64_t>(batch * G, 4 * sms);
    {
      TraceScope ts(kKSplitStep, s);
      stp<<<grid, kSThreads, kSSmemBytes, s>>>(a, l, copies, pk, batch, n, k, G, info);
      if (int st = check_launch("split_step_kernel")) return st;
    }
    // Look-ahead for column k + 2 over panels 0..k (all final now), at about
    // one CTA per SM so that the caller's stream keeps room for its tail and
    // step launches.
    if (k + 2 < N) {
      if (int st = check(cudaEventRecord(side->fork, s), "cudaEventRecord")) return st;
      if (int st = check(cudaStreamWaitEvent(side->stream, side->fork, 0), "cudaStreamWaitEvent")) return st;
      if (int st = launch_update(k + 2, 0, k + 1, a + 64 * (k + 2), n2, n, pb[k & 1], side->stream, 1)) return st;
      if (int st = check(cudaEventRecord(side->join[k & 1], side->stream), "cudaEventRecord")) return st;
    }
  }
  return B2P_OK;
}

}  // namespace b2p
