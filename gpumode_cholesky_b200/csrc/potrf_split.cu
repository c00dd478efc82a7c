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
//       FP32 panel buffer, over all but the newest earlier panel ("look-ahead",
//       see the schedule above potrf_split).
//   split_step_kernel(k)    G CTAs per matrix.  Every CTA applies the newest
//       panel k-1 to the diagonal rows and to its own 128-row chunk on
//       tcgen05 (bulk copies of the panel copy, one TMEM lane per row),
//       factors the diagonal block in shared memory (diag64_factor) --
//       redundantly, which costs one diagonal engine per CTA but no extra
//       launch or grid-wide wait -- then solves its rows by forward
//       substitution, one row per thread (X L_kk^T = P, FP32), and writes L
//       and the panel copy of X.  CTA 0 of the matrix writes L_kk and info;
//       the zero strip right of the diagonal block goes out as bulk stores.
//
//   split_wide_kernel       (n >= kWideMinN) the panels older than the
//       previous 512-column outer block, applied to a whole outer block at
//       once as 128 x 256 tensor-core tiles on a third stream, so that the
//       per-column look-ahead only applies the last 8-15 panels (see the
//       schedule above potrf_split).
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
#include "guard.cuh"
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
                        float* pout, int n, int k, int c_begin, int c_end, int segs, int32_t* __restrict__ info,
                        const float* __restrict__ sig) {
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
    // Park U_s: thread -> accumulator row (TMEM lane) 32w + lane.  FP8: the
    // accumulator holds 256 U / (s_row s_k) (panel_copy.cuh).
    const int rl = 32 * warp + lane;
    float sc = 1.0f;
    if (MODE == B2P_MODE_FP8) sc = sig[(size_t)b * N + min(r0 + rl, n - 1) / 64] * sig[(size_t)b * N + k] * kFp8Fold;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float d[32];
      umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * h), d);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        *reinterpret_cast<float4*>(park + rl * kUParkLd + 32 * h + 4 * q) =
            make_float4(d[4 * q] * sc, d[4 * q + 1] * sc, d[4 * q + 2] * sc, d[4 * q + 3] * sc);
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

// ---- wide update kernel ----------------------------------------------------------
// For large orders the panels older than the previous outer block (kWideCols
// block columns) are applied to a whole outer block at once:
//   Out[r, j] = base[r, j] - sum_{c in [c_begin, c_end)} L_c[r] L_c[j0 + j]^T,
//   rows r >= j0, columns j < nbw,
// as 128 x 256 tiles (MMA N = 256: each A tile of the panel copies feeds 256
// output columns instead of 64, which is what makes the update bandwidth
// affordable at n >= 8192).  item = (matrix, row tile, column tile).
//
// Warp roles: warp 8 (one thread) streams the panel copies through a
// two-stage ring of bulk copies and issues the MMAs; warps 0-7 own the
// accumulator.  The tensor core adds into its FP32 accumulator without
// round-to-nearest, and over K = n that bias grows with n; so the MMAs of
// every kXChunk panels go into one of two TMEM accumulators (ping-pong), and
// the consumer warps fold each finished one into FP32 registers (warp w:
// TMEM lanes 32 (w % 4) .., columns 128 (w / 4) ..) while the tensor core
// fills the other.
// With segs == 1 every CTA loops over items (a persistent grid, so the step
// kernels keep the other SMs); with segs > 1 each cluster of segs CTAs
// splits one item's K range and reduces over distributed shared memory in a
// fixed order.
constexpr int kXConsumers = 256;
constexpr int kXThreads = kXConsumers + 32;
constexpr int kXCols = 256;
constexpr int kXChunk = 4;                                    // panels per TMEM accumulation
constexpr uint32_t kXStageA = 32768;                          // 128 rows x 2 regions
constexpr uint32_t kXStage = kXStageA + 2u * kXCols * 128u;   // + 256 rows x 2 regions
constexpr uint32_t kXStaging = 2 * kXStage;
constexpr int kXParkLd = kXCols + 4;
constexpr uint32_t kXSmemBytes = kXStaging + 128 + 1024;
constexpr uint32_t kXTmemCols = 2 * kXCols;
static_assert(128 * kXParkLd * 4 <= kXStaging, "parked accumulator must fit the staging area");

template <int MODE>
__global__ void __launch_bounds__(kXThreads, 1)
    split_wide_kernel(const float* base, int64_t base_mstride, int base_ld, const uint8_t* __restrict__ ws,
                      float* out, int64_t out_mstride, int out_ld, int64_t batch, int n, int j0, int nbw,
                      int c_begin, int c_end, int segs, int32_t* __restrict__ info, const float* __restrict__ sig) {
  extern __shared__ unsigned char xraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(xraw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kXStaging);  // [2] stage loaded
  uint64_t* empty = full + 2;                                     // [2] stage read by its MMAs
  uint64_t* accf = full + 4;                                      // [2] accumulator complete
  uint64_t* accd = full + 6;                                      // [2] accumulator folded
  uint64_t* fin = full + 8;                                       // [1] every MMA done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kXStaging + 80);
  volatile int* flag = reinterpret_cast<volatile int*>(sm + kXStaging + 84);
  float* park = reinterpret_cast<float*>(sm);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = n / 64;
  const size_t rbytes = panel_copy_region_bytes(n);
  const int s = segs > 1 ? (int)umma::cluster_rank() : 0;
  const int64_t ncl = gridDim.x / segs;
  const int rt = (n - j0 + 127) / 128, ct = (nbw + kXCols - 1) / kXCols;
  const int64_t items = batch * rt * ct;
  const int span = c_end - c_begin;
  const int c_lo = c_begin + s * span / segs, c_hi = c_begin + (s + 1) * span / segs;
  const int iters = c_hi - c_lo;
  const int nch = (iters + kXChunk - 1) / kXChunk;

  if (tid == 0) *flag = 0;
  if (warp == 0) {
    umma::tmem_alloc(tslot, kXTmemCols);
    umma::tmem_relinquish();
  }
  if (tid == 32) {
    for (int i = 0; i < 4; ++i) umma::mbar_init(full + i, 1);   // full, empty
    for (int i = 4; i < 6; ++i) umma::mbar_init(full + i, 1);   // accf
    for (int i = 6; i < 8; ++i) umma::mbar_init(full + i, kXConsumers / 32);  // accd
    umma::mbar_init(fin, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;

  if (warp == kXConsumers / 32) {
    // ---------------- producer / MMA issuer ----------------
    if (lane == 0) {
      int64_t gi = 0, loaded = 0;  // panels consumed / loaded (all items)
      int64_t gc = 0;              // chunks started
      bool ok = true;
      for (int64_t item = blockIdx.x / segs; item < items && ok; item += ncl) {
        const int tj = (int)(item % ct);
        const int ti = (int)((item / ct) % rt);
        const int64_t b = item / ((int64_t)ct * rt);
        const int r0 = j0 + 128 * ti, vr = min(128, n - r0);
        const int cj = kXCols * tj, vc = min(kXCols, nbw - cj);
        const uint8_t* W0 = ws + (size_t)b * 2 * rbytes;
        const uint8_t* W1 = W0 + rbytes;
        // Panel i of this item into its ring stage (after the MMAs of the
        // panel two before it, which read that stage, have completed).
        auto load = [&](int i) -> bool {
          const int64_t g = loaded;
          const int st = (int)(g & 1);
          if (g >= 2 && !umma::mbar_wait_bounded(empty + st, (uint32_t)(((g - 2) >> 1) & 1), kSplitPolls))
            return false;
          const int c = c_lo + i;
          const uint32_t abytes = (uint32_t)vr * 128u, bbytes = (uint32_t)vc * 128u;
          const size_t aoff = panel_copy_row_byte(N, c, r0);
          const size_t boff = panel_copy_row_byte(N, c, j0 + cj);
          uint8_t* dst = sm + st * kXStage;
          umma::mbar_arrive_expect_tx(full + st, 2 * abytes + 2 * bbytes);
          umma::bulk_g2s(dst, W0 + aoff, abytes, full + st);
          umma::bulk_g2s(dst + 16384, W1 + aoff, abytes, full + st);
          umma::bulk_g2s(dst + kXStageA, W0 + boff, bbytes, full + st);
          umma::bulk_g2s(dst + kXStageA + kXCols * 128, W1 + boff, bbytes, full + st);
          ++loaded;
          return true;
        };
        if (!load(0)) {
          ok = false;
          break;
        }
        for (int ch = 0; ch < nch && ok; ++ch, ++gc) {
          const int p = (int)(gc & 1);
          // Accumulator p is free once the consumers folded chunk gc - 2.
          if (gc >= 2 && !umma::mbar_wait_bounded(accd + p, (uint32_t)(((gc - 2) >> 1) & 1), kSplitPolls)) {
            ok = false;
            break;
          }
          umma::fence_after_sync();
          const int i_end = min(iters, (ch + 1) * kXChunk);
          for (int i = ch * kXChunk; i < i_end; ++i, ++gi) {
            if (i + 1 < iters && !load(i + 1)) {
              ok = false;
              break;
            }
            const int st = (int)(gi & 1);
            if (!umma::mbar_wait_bounded(full + st, (uint32_t)((gi >> 1) & 1), kSplitPolls)) {
              ok = false;
              break;
            }
            umma::fence_after_sync();
            const uint32_t sa = umma::smem_u32(sm + st * kXStage);
            panel_copy_mmas<MODE, kXCols>(tmem + (uint32_t)(p * kXCols), sa, sa + kXStageA, i > ch * kXChunk);
            umma::mma_commit(empty + st);
          }
          if (ok) umma::mma_commit(accf + p);
        }
      }
      if (!ok) {
        // Copies still in flight land before anything leaves.
        for (int64_t g = gi; g < loaded; ++g) umma::mbar_wait_bounded(full + (g & 1), (uint32_t)((g >> 1) & 1), kSplitPolls);
        *flag = 1;
      }
      umma::mma_commit(fin);
    }
    __syncwarp();
  } else {
    // ---------------- consumers: fold the accumulators, write Out ----------------
    const int q = warp & 3, hh = warp >> 2;
    const int rl = 32 * q + lane;
    int64_t gc = 0;
    for (int64_t item = blockIdx.x / segs; item < items; item += ncl) {
      const int tj = (int)(item % ct);
      const int ti = (int)((item / ct) % rt);
      const int64_t b = item / ((int64_t)ct * rt);
      const int r0 = j0 + 128 * ti, vr = min(128, n - r0);
      const int cj = kXCols * tj, vc = min(kXCols, nbw - cj);
      float acc[128];
#pragma unroll
      for (int c = 0; c < 128; ++c) acc[c] = 0.0f;
      // FP8: the accumulators hold 256 U / (s_row s_col) per 64-column block.
      float sc[4] = {1.0f, 1.0f, 1.0f, 1.0f};
      if (MODE == B2P_MODE_FP8) {
        const float sr = sig[(size_t)b * N + min(r0 + rl, n - 1) / 64] * kFp8Fold;
#pragma unroll
        for (int j = 0; j < 4; ++j) sc[j] = sr * sig[(size_t)b * N + min(j0 + cj + 128 * hh + 32 * j, n - 1) / 64];
      }
      bool ok = true;
      for (int ch = 0; ch < nch; ++ch, ++gc) {
        const int p = (int)(gc & 1);
        const bool got = umma::mbar_wait_bounded(accf + p, (uint32_t)((gc >> 1) & 1), kSplitPolls) && *flag == 0;
        if (!__all_sync(0xffffffffu, got)) {
          ok = false;
          break;
        }
        umma::fence_after_sync();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          float d[32];
          umma::tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(p * kXCols + 128 * hh + 32 * j), d);
#pragma unroll
          for (int c = 0; c < 32; ++c) acc[32 * j + c] = fmaf(d[c], sc[j], acc[32 * j + c]);
        }
        umma::fence_before_sync();
        __syncwarp();
        if (lane == 0) umma::mbar_arrive(accd + p);
      }
      if (!ok) {
        *flag = 1;
        if (lane == 0 && info != nullptr) info[b] = -1;
        break;
      }
      const float* B = base + (size_t)b * base_mstride;
      float* O = out + (size_t)b * out_mstride;
      const int c0 = 128 * hh;
      if (segs == 1) {
        if (rl < vr && c0 < vc) {
          const float4* src = reinterpret_cast<const float4*>(B + (size_t)(r0 + rl) * base_ld + cj + c0);
          float4* dst = reinterpret_cast<float4*>(O + (size_t)(r0 + rl) * out_ld + cj + c0);
#pragma unroll
          for (int c4 = 0; c4 < 32; ++c4) {
            if (4 * c4 < vc - c0) {
              const float4 v = src[c4];
              dst[c4] = make_float4(v.x - acc[4 * c4], v.y - acc[4 * c4 + 1], v.z - acc[4 * c4 + 2],
                                    v.w - acc[4 * c4 + 3]);
            }
          }
        }
      } else {
        // One item per cluster: every copy into the staging area has landed
        // (all were read by MMAs), so it takes the parked accumulator.
#pragma unroll
        for (int c4 = 0; c4 < 32; ++c4)
          *reinterpret_cast<float4*>(park + rl * kXParkLd + c0 + 4 * c4) =
              make_float4(acc[4 * c4], acc[4 * c4 + 1], acc[4 * c4 + 2], acc[4 * c4 + 3]);
      }
    }
  }
  if (segs > 1) {
    // Sum the parked accumulators of the cluster in segment order.
    umma::cluster_sync();
    const int64_t item = blockIdx.x / segs;
    if (*flag == 0 && item < items) {
      const int tj = (int)(item % ct);
      const int ti = (int)((item / ct) % rt);
      const int64_t b = item / ((int64_t)ct * rt);
      const int r0 = j0 + 128 * ti, vr = min(128, n - r0);
      const int cj = kXCols * tj, vc = min(kXCols, nbw - cj);
      const float* B = base + (size_t)b * base_mstride;
      float* O = out + (size_t)b * out_mstride;
      const int c4n = vc / 4;
      for (int e = s * kXThreads + tid; e < vr * c4n; e += segs * kXThreads) {
        const int row = e / c4n, c4 = (e - row * c4n) * 4;
        float4 v = *reinterpret_cast<const float4*>(B + (size_t)(r0 + row) * base_ld + cj + c4);
        for (int qq = 0; qq < segs; ++qq) {
          const float4 u = umma::ld_cluster_f4(park + row * kXParkLd + c4, (uint32_t)qq);
          v.x -= u.x;
          v.y -= u.y;
          v.z -= u.z;
          v.w -= u.w;
        }
        *reinterpret_cast<float4*>(O + (size_t)(r0 + row) * out_ld + cj + c4) = v;
      }
    }
    // No CTA leaves while another may still read its park.
    umma::cluster_sync();
  }
  // Every MMA has completed before TMEM is released.
  umma::mbar_wait_bounded(fin, 0u, kSplitPolls);
  umma::fence_after_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kXTmemCols);
}

// ---- step kernel -------------------------------------------------------------
constexpr int kSThreads = 128;
constexpr int kSStripThread = 96;  // warp 3 lane 0
// Panel k-1 rows k0..k0+63: the B operand (region 0 at +0, region 1 at
// +8 KB), and also the diagonal product's A operand (A1 = 8 KB: its rows
// 64..127, whose accumulator lanes nobody reads, overlap what follows).
constexpr uint32_t kSB = 0;
constexpr uint32_t kSAo = 16384;       // the CTA's 128 rows of panel k-1: 2 x 16 KB
constexpr uint32_t kSZero = 49152;     // zeros for the strip's bulk stores
constexpr uint32_t kSZeroBytes = 4096;
constexpr uint32_t kSDiag = kSZero + kSZeroBytes;
constexpr uint32_t kSBar = kSDiag + (((uint32_t)sizeof(Diag64Smem) + 127u) & ~127u);
constexpr uint32_t kSSmemBytes = kSBar + 64 + 1024;
// Beside the outer-block update (n >= kWideMinN) two step CTAs share an SM
// (shared memory and 2 x 128 TMEM columns), so a column's chunks need half
// as many of the SMs it leaves free.  Below that the steps have the whole
// GPU, and a larger request keeps each step CTA alone on its SM (neither a
// second step CTA nor a look-ahead update CTA fits beside it): 1 x 8192 ran
// 3286 us that way and 3769 us with the SMs shared.
static_assert(2 * (kSSmemBytes + 1024) <= 228 * 1024, "two step CTAs per SM");
constexpr uint32_t kSSmemAlone = 140 * 1024;
constexpr uint32_t kSTmemCols = 128;   // [0, 64): diagonal rows; [64, 128): the CTA's rows

// Column k of every matrix, G CTAs per matrix.  P = base - X_{k-1} X_{k-1,kk}^T
// where base is A (k <= 1) or the panel buffer holding A minus the panels
// 0..k-2 (look-ahead), and the newest panel k-1 is applied here on tcgen05
// from its panel copy.  Then: factor the diagonal block (every CTA), solve
// the CTA's 128-row chunks by forward substitution (one row per thread,
// which is also one TMEM lane per thread), write L and the panel copy.
template <int MODE>
__global__ void __launch_bounds__(kSThreads, 2)
    split_step_kernel(const float* __restrict__ a, float* __restrict__ l, uint8_t* __restrict__ ws,
                      const float* __restrict__ pbuf, int64_t batch, int n, int k, int G,
                      int32_t* __restrict__ info, const float* __restrict__ sig, GuardRec grd) {
  __shared__ int s_gmin;
  // The last step resets the rescue's grid barrier (the rescue runs after it).
  if (grd.bar != nullptr && k == n / 64 - 1 && blockIdx.x == 0 && threadIdx.x == 0) grd.bar[0] = grd.bar[1] = 0;
  extern __shared__ unsigned char sraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(sraw) + 1023) & ~(uintptr_t)1023);
  Diag64Smem& dg = *reinterpret_cast<Diag64Smem*>(sm + kSDiag);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kSBar);
  uint64_t* done = full + 1;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSBar + 16);
  int* flag = reinterpret_cast<int*>(sm + kSBar + 24);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int N = n / 64, k0 = 64 * k;
  const int chunks = (n - k0 - 64 + kSThreads - 1) / kSThreads;
  const size_t rbytes = panel_copy_region_bytes(n);
  const size_t n2 = (size_t)n * n;
  const bool upd = k >= 1;

  for (uint32_t e = tid; e < kSZeroBytes / 16; e += kSThreads)
    reinterpret_cast<float4*>(sm + kSZero)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  umma::fence_proxy_async_smem();
  if (tid == 0) *flag = 0;
  if (upd && warp == 0) {
    umma::tmem_alloc(tslot, kSTmemCols);
    umma::tmem_relinquish();
  }
  if (tid == 32) {
    umma::mbar_init(full, 1);
    umma::mbar_init(done, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = upd ? *tslot : 0u;
  uint32_t ph_full = 0u, ph_done = 0u;
  bool ok = true;

  int64_t job = blockIdx.x;
  for (; job < batch * G && ok; job += gridDim.x) {
    const int64_t b = job / G;
    const int g = (int)(job - b * G);
    float* L = l + (size_t)b * n2;
    uint8_t* W0 = ws + (size_t)b * 2 * rbytes;
    uint8_t* W1 = W0 + rbytes;
    const float* base = (k >= 2) ? pbuf + (size_t)b * n * 64 : a + (size_t)b * n2 + k0;
    const size_t bld = (k >= 2) ? 64 : (size_t)n;

    // The newest panel's product for the diagonal rows and chunk q (or the
    // diagonal rows only when q is out of range); false on a timeout.
    auto newest_panel = [&](int q, bool first) -> bool {
      const bool own = q < chunks;
      const int r0 = k0 + 64 + q * kSThreads;
      const uint32_t vr = own ? (uint32_t)min(kSThreads, n - r0) : 0u;
      if (tid == 0) {
        const size_t boff = panel_copy_row_byte(N, k - 1, k0);
        umma::mbar_arrive_expect_tx(full, (first ? 2u * 8192u : 0u) + 2u * vr * 128u);
        if (first) {
          umma::bulk_g2s(sm + kSB, W0 + boff, 8192u, full);
          umma::bulk_g2s(sm + kSB + 8192, W1 + boff, 8192u, full);
        }
        if (own) {
          const size_t aoff = panel_copy_row_byte(N, k - 1, r0);
          umma::bulk_g2s(sm + kSAo, W0 + aoff, vr * 128u, full);
          umma::bulk_g2s(sm + kSAo + 16384, W1 + aoff, vr * 128u, full);
        }
        if (umma::mbar_wait_bounded(full, ph_full, kSplitPolls)) {
          umma::fence_after_sync();
          const uint32_t sb = umma::smem_u32(sm + kSB);
          if (first) panel_copy_mmas<MODE, 64, 8192u>(tmem, sb, sb, false);
          if (own) panel_copy_mmas<MODE>(tmem + 64, umma::smem_u32(sm + kSAo), sb, false);
        } else {
          *flag = 1;
        }
        umma::mma_commit(done);
      }
      ph_full ^= 1u;
      const bool got = umma::mbar_wait_bounded(done, ph_done, kSplitPolls);
      ph_done ^= 1u;
      umma::fence_after_sync();
      if (!got) *flag = 1;
      __syncthreads();
      return *flag == 0;
    };

    // 1. Diagonal block: P_kk = base - D (rows k0..k0+63), into dg.S.
    if (upd && !newest_panel(g, true)) {
      ok = false;
      if (tid == 0 && info != nullptr) info[b] = -1;
      break;
    }
    // 2. Zero strip right of the diagonal block: rows g, g + G, ... of it as
    //    bulk stores from the zero buffer, issued by warp 3 (idle in the
    //    P_kk formation and the diagonal factor) and left to run.
    if (tid == kSStripThread) {
      const uint32_t strip = 4u * (uint32_t)(n - k0 - 64);
      if (strip > 0) {
        for (int r = g; r < 64; r += G) {
          uint8_t* row = reinterpret_cast<uint8_t*>(L + (size_t)(k0 + r) * n + k0 + 64);
          for (uint32_t off = 0; off < strip; off += kSZeroBytes)
            umma::bulk_s2g(row + off, sm + kSZero, min(kSZeroBytes, strip - off));
        }
        umma::bulk_commit();
      }
    }
    if (warp < 2) {
      const float4* src = reinterpret_cast<const float4*>(base + (size_t)(k0 + tid) * bld);
      float4* dst = reinterpret_cast<float4*>(dg.S + tid * kD64Ld);
      // FP8: the accumulator holds 256 D / s_k^2 (panel_copy.cuh).
      const float sd = MODE == B2P_MODE_FP8 ? sig[(size_t)b * N + k] * sig[(size_t)b * N + k] * kFp8Fold : 1.0f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float d[32];
        if (upd) {
          umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * h), d);
        } else {
#pragma unroll
          for (int c = 0; c < 32; ++c) d[c] = 0.0f;
        }
#pragma unroll
        for (int c4 = 0; c4 < 8; ++c4) {
          const float4 v = src[8 * h + c4];
          dst[8 * h + c4] = make_float4(v.x - d[4 * c4] * sd, v.y - d[4 * c4 + 1] * sd, v.z - d[4 * c4 + 2] * sd,
                                        v.w - d[4 * c4 + 3] * sd);
        }
      }
    }
    umma::fence_before_sync();
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
      // The pivot record of a guarded call: (L_jj, A_jj); after the last
      // block column, the matrix's audit.
      if (grd.piv != nullptr && tid < 64)
        grd.piv[(size_t)b * n + k0 + tid] =
            make_float2(dg.S[tid * kD64Ld + tid], __ldg(a + (size_t)b * n2 + (size_t)(k0 + tid) * (n + 1)));
      if (grd.state != nullptr && k == N - 1) {
        const int f = guard_audit_matrix<kSThreads>(grd.piv + (size_t)b * n, n, MODE, &s_gmin, tid, CtaBarrier());
        if (tid == 0) grd.state[b] = f;
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
    // 3. Panel rows: X L_kk^T = P, one row (and one TMEM lane) per thread.
    for (int q = g; q < chunks; q += G) {
      if (upd && q != g && !newest_panel(q, false)) {
        ok = false;
        if (tid == 0 && info != nullptr) info[b] = -1;
        break;
      }
      const int r = k0 + 64 + q * kSThreads + tid;
      float d0[32], d1[32];
      if (upd) {
        umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + 64u, d0);
        umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + 96u, d1);
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) d0[c] = d1[c] = 0.0f;
      }
      if (r < n) {
        float x[64];
        const float4* src = reinterpret_cast<const float4*>(base + (size_t)r * bld);
        // FP8: the accumulator holds 256 D / (s_r s_k).
        const float sr =
            MODE == B2P_MODE_FP8 ? sig[(size_t)b * N + r / 64] * sig[(size_t)b * N + k] * kFp8Fold : 1.0f;
#pragma unroll
        for (int c4 = 0; c4 < 8; ++c4) {
          const float4 v = src[c4];
          x[4 * c4 + 0] = v.x - d0[4 * c4 + 0] * sr;
          x[4 * c4 + 1] = v.y - d0[4 * c4 + 1] * sr;
          x[4 * c4 + 2] = v.z - d0[4 * c4 + 2] * sr;
          x[4 * c4 + 3] = v.w - d0[4 * c4 + 3] * sr;
          const float4 w = src[8 + c4];
          x[32 + 4 * c4 + 0] = w.x - d1[4 * c4 + 0] * sr;
          x[32 + 4 * c4 + 1] = w.y - d1[4 * c4 + 1] * sr;
          x[32 + 4 * c4 + 2] = w.z - d1[4 * c4 + 2] * sr;
          x[32 + 4 * c4 + 3] = w.w - d1[4 * c4 + 3] * sr;
        }
        panel_solve64(x, dg);
        float4* dst = reinterpret_cast<float4*>(L + (size_t)r * n + k0);
#pragma unroll
        for (int c4 = 0; c4 < 16; ++c4) dst[c4] = make_float4(x[4 * c4], x[4 * c4 + 1], x[4 * c4 + 2], x[4 * c4 + 3]);
        if (k + 1 < N) {
          const float isig = MODE == B2P_MODE_FP8 ? 1.0f / sig[(size_t)b * N + r / 64] : 1.0f;
#pragma unroll
          for (int c8 = 0; c8 < 8; ++c8) {
            const float v[8] = {x[8 * c8],     x[8 * c8 + 1], x[8 * c8 + 2], x[8 * c8 + 3],
                                x[8 * c8 + 4], x[8 * c8 + 5], x[8 * c8 + 6], x[8 * c8 + 7]};
            panel_copy_store<MODE>(W0, W1, N, k, r, c8, v, isig);
          }
        }
      }
      // TMEM and the A staging are rewritten by the next chunk.
      umma::fence_before_sync();
      __syncthreads();
    }
    // dg is rewritten by the next job.
    __syncthreads();
  }
  // Matrices whose last step this CTA did not reach are not rescued.
  if (!ok && grd.state != nullptr && k == N - 1 && tid == 0)
    for (; job < batch * G; job += gridDim.x)
      if (job % G == 0) grd.state[job / G] = -1;
  if (!ok) umma::mbar_wait_bounded(done, ph_done, kSplitPolls);
  // The strip's bulk stores read the zero buffer until they complete.
  if (tid == kSStripThread) umma::bulk_wait_all();
  umma::fence_before_sync();
  __syncthreads();
  if (upd && warp == 0) umma::tmem_dealloc(tmem, kSTmemCols);
}

// ---- host side -----------------------------------------------------------------

bool split_supported(int64_t n, int mode) {
  const int m = mode & B2P_MODE_MASK;
  return (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3 || m == B2P_MODE_FP8) && !(mode & B2P_FLAG_FP64_DIAG) &&
         n > 128 && (n % 64) == 0 && n <= 65536;
}

// FP8 mode: the power-of-two scale of every 64-row block of every matrix,
// s = 2^ceil(log2(max_{rows i of the block} sqrt(A_ii) / 256)), so that
// |L[i][j]| <= sqrt(A_ii) <= 256 s (panel_copy.cuh).  One thread per block.
__global__ void fp8_scale_kernel(const float* __restrict__ a, float* __restrict__ sig, int64_t batch, int n) {
  const int N = n / 64;
  const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= batch * N) return;
  const int64_t b = id / N;
  const int blk = (int)(id - b * N);
  const float* d = a + (size_t)b * n * n + (size_t)(64 * blk) * (n + 1);
  float m = 0.0f;
  for (int i = 0; i < 64; ++i) m = fmaxf(m, __ldg(d + (size_t)i * (n + 1)));
  const float v = sqrtf(m) * (1.0f / 256.0f);
  sig[id] = (v > 0.0f && isfinite(v)) ? exp2f(ceilf(log2f(v))) : 1.0f;
}

// Orders from which the older panels are applied an outer block at a time
// (split_wide_kernel), and the outer block width in block columns.  At
// 1 x 8192 the wide stage does not pay yet (3681 us against 3628 us).
constexpr int kWideMinN = 12288;
constexpr int kWideCols = 8;  // 512 columns
static_assert(64 * kWideCols % kXCols == 0, "outer blocks are whole wide tiles");

// Panel copies, then two per-matrix FP32 panel buffers (n x 64 each; block
// columns alternate between them), then for large orders two per-matrix
// outer-block buffers (n x 512 each, alternating by outer block).
static size_t split_sig_offset(int64_t batch, int64_t n) {
  size_t bytes = (size_t)batch * 2 * panel_copy_region_bytes((int)n) + 2 * (size_t)batch * n * 64 * sizeof(float);
  if (n >= kWideMinN) bytes += 2 * (size_t)batch * n * 64 * kWideCols * sizeof(float);
  return bytes;
}
size_t split_workspace_bytes(int64_t batch, int64_t n) {
  // ... then the FP8 mode's block scales (batch x n/64 floats).
  return split_sig_offset(batch, n) + (((size_t)batch * (n / 64) * sizeof(float) + 255) & ~(size_t)255) + 1024;
}

namespace {
// Per device: a second stream for the look-ahead part of the updates and
// the events that fork it from and join it to the caller's stream.
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[2] = {nullptr, nullptr};
  // Large orders: the outer-block updates run on a third stream.
  cudaStream_t wide = nullptr;
  cudaEvent_t wide_done[2] = {nullptr, nullptr};
  cudaEvent_t wide_free[2] = {nullptr, nullptr};
  int step_priority = 0;  // the device's greatest (numerically lowest) priority
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
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ss.wide, cudaStreamNonBlocking);
    int least = 0, greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    ss.step_priority = greatest;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
      e = cudaEventCreateWithFlags(&ss.wide_done[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss.wide_free[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "side stream set-up: %s", cudaGetErrorString(e));
  }
  *out = &ss;
  return B2P_OK;
}
}  // namespace

// Schedule.  Block column j needs every earlier panel.  Panels 0..j-2 are
// final one step early, so their part of the update ("look-ahead", into the
// panel buffer of j) runs on the side stream beside step j-1; step j itself
// applies the newest panel j-1:
//   caller: step(j) -> [fork] -> step(j+1) -> ...
//   side:                look-ahead(j+2) over panels 0..j
// step(j) waits for look-ahead(j) (join event j % 2).  Column j uses panel
// buffer j % 2, which look-ahead(j+2) may only overwrite after step(j).
//
// Large orders (n >= kWideMinN) split the look-ahead further.  With outer
// blocks of W = kWideCols block columns, the panels older than the previous
// outer block are final a whole outer block before they are needed: right
// after the last step of outer block J-2, the wide stream computes
//   Bw_J = A[:, block J] - (panels 0 .. (J-1) W - 1) applied to block J
// (split_wide_kernel, buffer J % 2), and the look-ahead of a column j in
// block J >= 2 then starts from Bw_J and applies only the panels
// (J-1) W .. j-2 (fewer than 2 W).  The first look-ahead of block J waits
// for Bw_J (event wide_done[J % 2]); Bw_{J+2} waits until the last
// look-ahead of block J has read buffer J % 2 (event wide_free[J % 2]).  The
// wide kernel keeps to a bounded number of SMs so that the steps, which
// carry the critical path, always find free ones.
int potrf_split(const float* a, float* l, int64_t batch, int n, int mode, void* ws, size_t ws_bytes,
                int32_t* info, cudaStream_t s, GuardRec grd) {
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
  const int m = mode & B2P_MODE_MASK;
  const int mi = m == B2P_MODE_TF32 ? 0 : m == B2P_MODE_BF16X3 ? 1 : 2;
  auto upd = mi == 0 ? split_update_kernel<B2P_MODE_TF32>
             : mi == 1 ? split_update_kernel<B2P_MODE_BF16X3> : split_update_kernel<B2P_MODE_FP8>;
  auto stp = mi == 0 ? split_step_kernel<B2P_MODE_TF32>
             : mi == 1 ? split_step_kernel<B2P_MODE_BF16X3> : split_step_kernel<B2P_MODE_FP8>;
  auto wdk = mi == 0 ? split_wide_kernel<B2P_MODE_TF32>
             : mi == 1 ? split_wide_kernel<B2P_MODE_BF16X3> : split_wide_kernel<B2P_MODE_FP8>;
  const int uslot[3] = {kSlotSplitU0, kSlotSplitU1, kSlotSplitU2};
  const int sslot[3] = {kSlotSplitS0, kSlotSplitS1, kSlotSplitS2};
  const int wslot[3] = {kSlotSplitW0, kSlotSplitW1, kSlotSplitW2};
  if (int st = ensure_smem_attr((const void*)upd, kUSmemBytes, uslot[mi])) return st;
  if (int st = ensure_smem_attr((const void*)stp, kSSmemAlone, sslot[mi])) return st;
  float* sig = reinterpret_cast<float*>(copies + split_sig_offset(batch, n));
  if (m == B2P_MODE_FP8) {
    const int64_t blocks = batch * (n / 64);
    fp8_scale_kernel<<<(unsigned)((blocks + 127) / 128), 128, 0, s>>>(a, sig, batch, n);
    if (int st = check_launch("fp8_scale_kernel")) return st;
  }
  const int N = n / 64;
  const int64_t n2 = (int64_t)n * n;
  const bool wide = n >= kWideMinN;
  constexpr int W = kWideCols;
  const int nbw = 64 * W;
  float* bw[2] = {nullptr, nullptr};
  if (wide) {
    if (int st = ensure_smem_attr((const void*)wdk, kXSmemBytes, wslot[mi])) return st;
    bw[0] = pb[1] + (size_t)batch * n * 64;
    bw[1] = bw[0] + (size_t)batch * n * nbw;
  }
  // SMs the wide kernel may hold at once: 9/16 while the chain of steps
  // bounds the time, three quarters once the outer-block updates do.  Graph
  // replay, FP8, with two step CTAs per SM: 1 x 16384 9.78 ms at 74 of 148
  // SMs, 9.41 ms at 83, 9.80 ms at 92; 1 x 32768 47.1 ms at 98, 46.8 ms at
  // 111, 46.6 ms at 86.
  const int64_t wide_ctas = std::max<int64_t>(1, n >= 24576 ? sms * 3 / 4 : sms * 9 / 16);

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
    TraceScope ts(kKSplitUpdate, st, 2.0 * 64 * 64 * (double)(c1 - c0) * batch * (n - 64 * k));
    const cudaError_t e = cudaLaunchKernelEx(&cfg, upd, base, mstride, ld, (const uint8_t*)copies, pout, n, k,
                                             c0, c1, segs, info, (const float*)sig);
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "split_update_kernel: %s", cudaGetErrorString(e));
    return B2P_OK;
  };
  // Outer-block update of block J (J >= 2) on the wide stream.
  auto launch_wide = [&](int J) -> int {
    const int j0 = J * nbw;
    const int cols = std::min(nbw, n - j0);
    const int c1 = (J - 1) * W;
    const int64_t items = batch * ((n - j0 + 127) / 128) * ((cols + kXCols - 1) / kXCols);
    int segs = 1;
    int64_t grid = std::min<int64_t>(items, wide_ctas);
    if (items * 2 <= wide_ctas) {
      segs = (int)std::max<int64_t>(1, std::min<int64_t>({wide_ctas / items, (int64_t)kSplitSegCap, (int64_t)c1}));
      grid = items * segs;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(kXThreads, 1, 1);
    cfg.dynamicSmemBytes = kXSmemBytes;
    cfg.stream = side->wide;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)segs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TraceScope ts(kKSplitWide, side->wide, 2.0 * 64 * (double)c1 * cols * batch * (n - j0));
    const cudaError_t e = cudaLaunchKernelEx(&cfg, wdk, (const float*)(a + j0), n2, n, (const uint8_t*)copies,
                                             bw[J & 1], (int64_t)n * nbw, nbw, batch, n, j0, cols, 0, c1, segs, info,
                                             (const float*)sig);
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "split_wide_kernel: %s", cudaGetErrorString(e));
    return B2P_OK;
  };
  // Step CTAs of column k: two per SM on the SMs the wide kernel leaves
  // free, else one per SM.
  const int64_t step_sms = wide ? 2 * (sms - wide_ctas) : sms;
  const uint32_t step_smem = wide ? kSSmemBytes : kSSmemAlone;
  auto step_G = [&](int k) -> int {
    const int chunks = (n - 64 * k - 64 + kSThreads - 1) / kSThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(std::max(chunks, 1), step_sms / batch));
  };
  auto step_ctas = [&](int k) -> int64_t { return std::min<int64_t>(batch * step_G(k), step_sms); };
  auto check = [](cudaError_t e, const char* what) -> int {
    return e == cudaSuccess ? B2P_OK : set_error(B2P_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  };

  for (int k = 0; k < N; ++k) {
    float* pk = pb[k & 1];
    // Column k >= 2 reads the look-ahead result (panels 0..k-2) from pk.
    if (k >= 2) {
      if (int st = check(cudaStreamWaitEvent(s, side->join[k & 1], 0), "cudaStreamWaitEvent")) return st;
    }
    // Step (with the newest panel k-1): step_ctas(k) CTAs, one 128-row
    // chunk each where the SMs allow.
    const int G = step_G(k);
    const int grid = (int)step_ctas(k);
    {
      // The steps carry the critical path: their CTAs go first when the
      // look-ahead and outer-block kernels compete for SMs (also inside a
      // CUDA graph, where a kernel node keeps its launch priority).
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)grid, 1, 1);
      cfg.blockDim = dim3(kSThreads, 1, 1);
      cfg.dynamicSmemBytes = step_smem;
      cfg.stream = s;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributePriority;
      attr[0].val.priority = side->step_priority;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      // Diagonal factor, panel solve and the newest panel's product.
      const double rows = (double)(n - 64 * k - 64);
      TraceScope ts(kKSplitStep, s,
                    batch * (64.0 * 64 * 64 / 3 + rows * 64 * 64 + (k > 0 ? 2.0 * 64 * 64 * (rows + 64) : 0.0)));
      const cudaError_t e =
          cudaLaunchKernelEx(&cfg, stp, a, l, copies, (const float*)pk, batch, n, k, G, info, (const float*)sig, grd);
      if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "split_step_kernel: %s", cudaGetErrorString(e));
    }
    // Outer block J = (k + 1) / W + 1 needs the panels before block J - 1,
    // which are all final once step k, the last of block J - 2, is done.
    const int Jw = (k + 1) / W + 1;
    const bool start_wide = wide && (k + 1) % W == 0 && Jw >= 2 && Jw * W < N;
    if (k + 2 < N || start_wide) {
      if (int st = check(cudaEventRecord(side->fork, s), "cudaEventRecord")) return st;
    }
    if (start_wide) {
      if (int st = check(cudaStreamWaitEvent(side->wide, side->fork, 0), "cudaStreamWaitEvent")) return st;
      if (Jw >= 4) {
        if (int st = check(cudaStreamWaitEvent(side->wide, side->wide_free[Jw & 1], 0), "cudaStreamWaitEvent"))
          return st;
      }
      if (int st = launch_wide(Jw)) return st;
      if (int st = check(cudaEventRecord(side->wide_done[Jw & 1], side->wide), "cudaEventRecord")) return st;
    }
    // Look-ahead for column k + 2 over panels 0..k (all final now), beside
    // step k + 1.  About one CTA per SM: two of its CTAs fit on an SM, so the
    // scheduler leaves SMs free for the step.
    if (k + 2 < N) {
      if (int st = check(cudaStreamWaitEvent(side->stream, side->fork, 0), "cudaStreamWaitEvent")) return st;
      const int j = k + 2, J = j / W;
      if (wide && J >= 2) {
        if (j == J * W) {
          if (int st = check(cudaStreamWaitEvent(side->stream, side->wide_done[J & 1], 0), "cudaStreamWaitEvent"))
            return st;
        }
        if (int st = launch_update(j, (J - 1) * W, k + 1, bw[J & 1] + 64 * (j - J * W), (int64_t)n * nbw, nbw,
                                   pb[k & 1], side->stream, 1))
          return st;
        if (j == std::min(J * W + W, N) - 1) {
          if (int st = check(cudaEventRecord(side->wide_free[J & 1], side->stream), "cudaEventRecord")) return st;
        }
      } else {
        if (int st = launch_update(j, 0, k + 1, a + 64 * j, n2, n, pb[k & 1], side->stream, 1)) return st;
      }
      if (int st = check(cudaEventRecord(side->join[k & 1], side->stream), "cudaEventRecord")) return st;
    }
  }
  return B2P_OK;
}

}  // namespace b2p
