// Warp-specialized fused left-looking factorization on the tensor cores.
//
// Same dataflow as potrf_fused.cu (one CTA per matrix, A read once, L written
// once, update accumulated in TMEM from pre-swizzled panel copies), but the
// update of block column k+1 runs concurrently with the panel work of block
// column k:
//
//   warp 8 (producer, one thread)  streams the panel copies with
//        cp.async.bulk (two stages) and issues the tcgen05 MMAs of the next
//        block column tile by tile; per tile it commits `acc_ready`;
//   warps 0-7 (consumers)  per tile: wait `acc_ready`, read D from TMEM
//        (then arrive `acc_free`), P = A - D, factor + invert the diagonal
//        block (tile 0), X = P T^T in FP32, write L and the tensor-core copy
//        of X, then publish the tile's completion count.  While warps 0-3
//        factor the diagonal block, warps 4-7 form P of the CTA's later
//        tiles and park it in their TMEM slots (released, as before, when
//        each tile is processed).
//
// Small batches run as clusters of CL = 2, 4 or 8 CTAs per matrix: rank r
// takes the row tiles t = r (mod CL) of every block column (tile 0 holds the
// diagonal block), and every rank > 0 also accumulates its own copy of tile
// 0 to factor the diagonal block redundantly, so the CTAs share only panel
// copies in global memory.  A finished tile is announced to both CTAs'
// producers through per-tile completion counters (release stores at cluster
// scope, bounded acquire polls), which cannot alias the way an mbarrier
// phase can when its waiter falls behind a CTA it does not pace.
//
// Ordering rules (every mbarrier is waited at most one phase behind):
//   * MMA write #w into TMEM tile t waits for consumer read #(w-1) of t;
//   * the update of block column k, tile t, over column k-1 needs the panel
//     rows of column k-1 produced by consumer tiles {0, t, t+1} of step k-1;
//     older columns are ready, so their MMAs are issued first.
// All waits are bounded; a timeout sets a shared flag that both roles check,
// marks the matrix with info = -1 and drains outstanding copies and MMAs
// before TMEM is released.
//
// The reference's left-looking paths (submission.py:3319-3409, 3606-3676,
// 5152-5196) issue the same three phases as separate cuSOLVER / cuBLAS /
// CUDA calls with host round trips between them.
#include <algorithm>

#include "diag64.cuh"
#include "guard.cuh"
#include "launch.h"
#include "panel_copy.cuh"
#include "umma.cuh"
#include "xgemm.cuh"

namespace b2p {

constexpr int kWConsumers = 256;
constexpr int kWThreads = kWConsumers + 32;
constexpr int kWB = 64;
constexpr int kWM = 128;
constexpr int kWPtLd = 132;
constexpr uint32_t kWPolls = 1u << 24;
constexpr uint32_t kWTmemCols = 512;

constexpr uint32_t kWStageA = 32768;
constexpr uint32_t kWStage = kWStageA + 16384;
constexpr uint32_t kWDiagOff = 2 * kWStage;
constexpr uint32_t kWPtOff = kWDiagOff + (((uint32_t)sizeof(Diag64Smem) + 1023u) & ~1023u);
constexpr uint32_t kWZeroOff = kWPtOff + 64 * kWPtLd * 4;  // zeros, source of the strip's bulk stores
constexpr uint32_t kWZeroBytes = 4096;                    // strip rows are stored in chunks of this
constexpr uint32_t kWBarOff = kWZeroOff + kWZeroBytes;
constexpr uint32_t kWCntOff = kWBarOff + 256;  // per-tile completion counters
constexpr int kWMaxTiles = 64;                  // row tiles of a block column (n <= 8192)
constexpr int kWMaxSlots = 8;                   // TMEM accumulator slots (512 columns)
constexpr uint32_t kWSmemBytes = kWCntOff + 4 * kWMaxTiles + 1024;

using ConsumerBar = NamedBarrier1<kWConsumers>;
constexpr int kWStripThread = 128;  // consumer warp 4, free during the diagonal engine

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_u32(mbar)) : "memory");
}

// Bounded wait that also gives up when the other role has flagged a failure.
__device__ __forceinline__ bool ws_wait(uint64_t* mbar, uint32_t parity, volatile int* flag) {
  for (uint32_t i = 0; i < kWPolls; ++i) {
    if (umma::mbar_try_wait(mbar, parity)) return true;
    if ((i & 255u) == 255u && *flag) return false;
  }
  return false;
}

__device__ __forceinline__ int ld_acquire_cluster(const int* p) {
  int v;
  asm volatile("ld.acquire.cluster.shared::cta.b32 %0, [%1];" : "=r"(v) : "r"(umma::smem_u32(p)) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cluster(const int* local, uint32_t rank, int v) {
  asm volatile("st.release.cluster.shared::cluster.b32 [%0], %1;" ::"r"(umma::cluster_addr(local, rank)), "r"(v)
               : "memory");
}
// Bounded wait until the completion counter *p reaches `target`.
__device__ __forceinline__ bool ws_wait_count(const int* p, int target, volatile int* flag, bool block) {
  for (uint32_t i = 0; i < (block ? kWPolls : 1u); ++i) {
    if (ld_acquire_cluster(p) >= target) return true;
    if ((i & 255u) == 255u && *flag) return false;
  }
  return false;
}

// Row tiles of a block column (mt_n of them) that CTA `rank` of a CL-CTA
// cluster accumulates, as a list: rank 0 takes tiles 0, CL, 2 CL, ...; rank
// r > 0 takes its own copy of tile 0 (for the diagonal block) and tiles r,
// r + CL, ...  Entry j of the list uses TMEM slot j.
template <int CL>
__device__ __forceinline__ int ws_tile_count(int mt_n, int rank) {
  if (CL == 1) return mt_n;
  if (rank == 0) return (mt_n + CL - 1) / CL;
  return 1 + (mt_n > rank ? (mt_n - rank + CL - 1) / CL : 0);
}
template <int CL>
__device__ __forceinline__ int ws_tile_of(int j, int rank) {
  if (CL == 1) return j;
  if (rank == 0) return j * CL;
  return j == 0 ? 0 : rank + (j - 1) * CL;
}

struct WsBars {
  uint64_t* full;        // [2]
  uint64_t* empty;       // [2]
  uint64_t* acc_ready;   // [8]
  uint64_t* acc_free;    // [8]
  int* tile_done;        // [kWMaxTiles] completion counters (all matrices of this CTA)
  uint64_t* drain;       // [1]
  uint32_t* tslot;
  volatile int* flag;
  int* badp;
};

// ---------------------------------------------------------------------------
// Producer: one thread.
template <int MODE, int CL>
__device__ void ws_producer(const WsBars& br, uint8_t* sm, uint8_t* ws, int64_t batch, int n, uint32_t tmem,
                            int rank) {
  const int N = n / kWB;
  const size_t rbytes = panel_copy_region_bytes(n);
  uint32_t n_load[2] = {0u, 0u}, n_empty[2] = {0u, 0u};
  int writes[kWMaxSlots] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t biter = 0;
  bool ok = true;
  for (int64_t b = blockIdx.x / CL; b < batch && ok; b += gridDim.x / CL, ++biter) {
    const uint8_t* W0 = ws + (size_t)b * 2 * rbytes;
    const uint8_t* W1 = W0 + rbytes;
    for (int k = 1; k < N && ok; ++k) {
      const int k0 = k * kWB;
      const int mt_n = (n - k0 + kWM - 1) / kWM;
      const int prev_n = (n - k0 + kWB + kWM - 1) / kWM;
      const int iters = ws_tile_count<CL>(mt_n, rank) * k;
      // Dependencies of the chunk over column k-1 for tile mt.
      auto deps_ready = [&](int mt, bool block) -> bool {
        int ts[3];
        int nt = 0;
        if (mt == 0) ts[nt++] = 0;
        if (mt != 0) ts[nt++] = mt;
        if (mt + 1 < prev_n) ts[nt++] = mt + 1;
        for (int q = 0; q < nt; ++q) {
          const int t = ts[q];
          // Tile t completes once per block column it exists in (N - 2t per
          // matrix); column k-1 of this matrix is completion number target.
          const int target = (int)(biter * (int64_t)(N - 2 * t) + k);
          if (!ws_wait_count(br.tile_done + t, target, br.flag, block)) return false;
        }
        return true;
      };
      auto issue_load = [&](int i) -> bool {
        const int mt = ws_tile_of<CL>(i / k, rank), kc = i - (i / k) * k;
        const int s = i & 1;
        if (n_load[s] > 0) {
          // The stage held the previous chunk: wait until the MMAs that read it completed.
          if (!ws_wait(br.empty + s, (n_load[s] - 1u) & 1u, br.flag)) return false;
        }
        if (kc == k - 1 && !deps_ready(mt, true)) return false;
        const int r0 = k0 + mt * kWM;
        const uint32_t abytes = (uint32_t)min(kWM, n - r0) * 128u;
        const size_t aoff = panel_copy_row_byte(N, kc, r0);
        const size_t boff = panel_copy_row_byte(N, kc, k0);
        uint8_t* st = sm + s * kWStage;
        umma::mbar_arrive_expect_tx(br.full + s, 2 * abytes + 2 * 8192u);
        umma::bulk_g2s(st, W0 + aoff, abytes, br.full + s);
        umma::bulk_g2s(st + 16384, W1 + aoff, abytes, br.full + s);
        umma::bulk_g2s(st + kWStageA, W0 + boff, 8192u, br.full + s);
        umma::bulk_g2s(st + kWStageA + 8192, W1 + boff, 8192u, br.full + s);
        ++n_load[s];
        return true;
      };
      int next = 0;
      if (iters > 0) {
        if (!issue_load(0)) { ok = false; break; }
        next = 1;
      }
      for (int i = 0; i < iters && ok; ++i) {
        const int s = i & 1;
        const int slot = i / k, kc = i - (i / k) * k;
        // Prefetch the next chunk unless it would wait on consumers.
        bool prefetched = false;
        if (next == i + 1 && next < iters) {
          const int nmt = ws_tile_of<CL>(next / k, rank), nkc = next - (next / k) * k;
          if (nkc != k - 1 || deps_ready(nmt, false)) {
            if (!issue_load(next)) { ok = false; break; }
            ++next;
            prefetched = true;
          }
        }
        if (!ws_wait(br.full + s, (n_load[s] - 1u) & 1u, br.flag)) { ok = false; break; }
        if (kc == 0 && writes[slot] > 0) {
          // TMEM slot `slot` must have been read by the consumers.
          if (!ws_wait(br.acc_free + slot, (uint32_t)((writes[slot] - 1) & 1), br.flag)) { ok = false; break; }
        }
        umma::fence_after_sync();
        const uint32_t st = umma::smem_u32(sm + s * kWStage);
        panel_copy_mmas<MODE>(tmem + (uint32_t)(kWB * slot), st, st + kWStageA, kc > 0);
        umma::mma_commit(br.empty + s);
        ++n_empty[s];
        if (kc == k - 1) {
          umma::mma_commit(br.acc_ready + slot);
          ++writes[slot];
        }
        if (!prefetched && next == i + 1 && next < iters) {
          if (!issue_load(next)) { ok = false; break; }
          ++next;
        }
      }
    }
  }
  if (!ok) *br.flag = 1;
  // Drain: every copy lands and every MMA completes before TMEM is released.
  for (int s = 0; s < 2; ++s) {
    if (n_load[s] > 0) umma::mbar_wait_bounded(br.full + s, (n_load[s] - 1u) & 1u, kWPolls);
  }
  umma::mma_commit(br.drain);
  umma::mbar_wait_bounded(br.drain, 0u, kWPolls);
}

// ---------------------------------------------------------------------------
// Consumers: warps 0-7.
template <int MODE, int CL>
__device__ void ws_consumers(const WsBars& br, uint8_t* sm, const float* a, float* l, uint8_t* ws, int64_t batch,
                             int n, uint32_t tmem, int32_t* info, int rank, GuardRec grd) {
  __shared__ int s_gmin;
  const ConsumerBar cbar;
  Diag64Smem& dg = *reinterpret_cast<Diag64Smem*>(sm + kWDiagOff);
  float* PtT = reinterpret_cast<float*>(sm + kWPtOff);
  const float* zeros = reinterpret_cast<const float*>(sm + kWZeroOff);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = n / kWB;
  const size_t rbytes = panel_copy_region_bytes(n);
  uint32_t ready_par = 0u;  // bit t: parity of the next acc_ready phase of tile t
  int64_t biter = 0;
  for (int64_t b = blockIdx.x / CL; b < batch; b += gridDim.x / CL, ++biter) {
    const float* A = a + (size_t)b * n * n;
    float* L = l + (size_t)b * n * n;
    uint8_t* W0 = ws + (size_t)b * 2 * rbytes;
    uint8_t* W1 = W0 + rbytes;
    if (tid == 0) *br.badp = -1;
    bool failed = false;
    for (int k = 0; k < N && !failed; ++k) {
      const int k0 = k * kWB;
      const int mt_n = (n - k0 + kWM - 1) / kWM;
      const int nt = ws_tile_count<CL>(mt_n, rank);
      for (int j = 0; j < nt; ++j) {
        const int mt = ws_tile_of<CL>(j, rank);
        // A copy of tile 0 on rank > 0: only the diagonal block is used.
        const bool diag_only = CL > 1 && rank != 0 && mt == 0;
        const int r0 = k0 + mt * kWM;
        const int vr = diag_only ? 64 : min(kWM, n - r0);
        // (a) D from TMEM, P = A - D.  Tiles after the first were formed
        // during the diagonal phase (b) and hold P in their TMEM slot.
        const bool preformed = k > 0 && j > 0;
        {
          const int w4 = warp & 3, h = warp >> 2;
          const int rl = 32 * w4 + lane;
          float d[32];
          if (k > 0) {
            if (!preformed) {
              const bool got = ws_wait(br.acc_ready + j, (ready_par >> j) & 1u, br.flag);
              if (!got) *br.flag = 1;
            }
            ready_par ^= 1u << j;
          }
          cbar();
          if (*br.flag) {
            failed = true;
            break;
          }
          if (k > 0) {
            umma::fence_after_sync();
            umma::tmem_ld32(tmem + ((uint32_t)(32 * w4) << 16) + (uint32_t)(kWB * j + 32 * h), d);
            umma::fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(br.acc_free + j);
          } else {
#pragma unroll
            for (int q = 0; q < 32; ++q) d[q] = 0.0f;
          }
          float p[32];
          if (preformed) {
#pragma unroll
            for (int q = 0; q < 32; ++q) p[q] = d[q];
          } else if (rl < vr) {
            const float4* src = reinterpret_cast<const float4*>(A + (size_t)(r0 + rl) * n + k0 + 32 * h);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const float4 v = src[q];
              p[4 * q + 0] = v.x - d[4 * q + 0];
              p[4 * q + 1] = v.y - d[4 * q + 1];
              p[4 * q + 2] = v.z - d[4 * q + 2];
              p[4 * q + 3] = v.w - d[4 * q + 3];
            }
          } else {
#pragma unroll
            for (int q = 0; q < 32; ++q) p[q] = 0.0f;
          }
          if (!diag_only) {
#pragma unroll
            for (int q = 0; q < 32; ++q) PtT[(32 * h + q) * kWPtLd + rl] = p[q];
          }
          if (mt == 0 && rl < 64) {
#pragma unroll
            for (int q = 0; q < 32; ++q) dg.S[rl * kD64Ld + 32 * h + q] = p[q];
          }
        }
        cbar();
        // (b) diagonal block: L_kk and T^T (pipelined engine), zero strip.
        if (mt == 0) {
          // Warps 0-3 run the diagonal engine.  Warps 4-7 meanwhile form
          // P = A - D of this CTA's later tiles of the column (each warp its
          // TMEM lane quarter, both column halves) and store it in place of D;
          // their slots are released when those tiles are processed below.
          if (warp < 4) {
            diag64_factor_invert(dg, NamedBarrier2<kD64Threads>());
          } else {
            // Zero strip right of the diagonal block: one bulk store per row
            // from the zero buffer, issued by one thread and left to run.
            const uint32_t strip = 4u * (uint32_t)(n - k0 - kWB);
            if (tid == kWStripThread && rank == 0 && strip > 0) {
              for (int r = 0; r < 64; ++r) {
                uint8_t* row = reinterpret_cast<uint8_t*>(L + (size_t)(k0 + r) * n + k0 + kWB);
                for (uint32_t off = 0; off < strip; off += kWZeroBytes)
                  umma::bulk_s2g(row + off, zeros, min(kWZeroBytes, strip - off));
              }
              umma::bulk_commit();
            }
          }
          if (warp >= 4 && k > 0) {
            const int w4 = warp & 3;
            const int rl = 32 * w4 + lane;
            for (int j2 = 1; j2 < nt; ++j2) {
              const int mt2 = ws_tile_of<CL>(j2, rank);
              const int r2 = k0 + mt2 * kWM, v2 = min(kWM, n - r2);
              const bool got = ws_wait(br.acc_ready + j2, (ready_par >> j2) & 1u, br.flag);
              if (!__all_sync(0xffffffffu, got)) {
                *br.flag = 1;
                break;
              }
              umma::fence_after_sync();
#pragma unroll 1
              for (int h = 0; h < 2; ++h) {
                const uint32_t taddr = tmem + ((uint32_t)(32 * w4) << 16) + (uint32_t)(kWB * j2 + 32 * h);
                float d[32], p[32];
                umma::tmem_ld32(taddr, d);
                if (rl < v2) {
                  const float4* src = reinterpret_cast<const float4*>(A + (size_t)(r2 + rl) * n + k0 + 32 * h);
#pragma unroll
                  for (int q = 0; q < 8; ++q) {
                    const float4 v = src[q];
                    p[4 * q + 0] = v.x - d[4 * q + 0];
                    p[4 * q + 1] = v.y - d[4 * q + 1];
                    p[4 * q + 2] = v.z - d[4 * q + 2];
                    p[4 * q + 3] = v.w - d[4 * q + 3];
                  }
                } else {
#pragma unroll
                  for (int q = 0; q < 32; ++q) p[q] = 0.0f;
                }
                umma::tmem_st32(taddr, p);
              }
            }
            umma::tmem_wait_st();
          }
          umma::fence_before_sync();
          cbar();
          umma::fence_after_sync();
          const int bad = diag64_status(dg);
          if (bad == kDiagTimeout || *br.flag) {
            failed = true;
            if (tid == 0) *br.flag = 1;  // the producer gives up too
          }
          if (tid == 0 && bad >= 0 && *br.badp < 0) *br.badp = k0 + bad;
          // The pivot record of a guarded call: (L_jj, A_jj).
          if (grd.piv != nullptr && rank == 0 && tid < 64)
            grd.piv[(size_t)b * n + k0 + tid] =
                make_float2(dg.S[tid * kD64Ld + tid], __ldg(A + (size_t)(k0 + tid) * (n + 1)));
          for (int e = tid; e < (rank == 0 ? 64 * 16 : 0); e += kWConsumers) {
            const int r = e >> 4, c = (e & 15) * 4;
            const float* srow = dg.S + r * kD64Ld + c;
            const float4 v = make_float4(c <= r ? srow[0] : 0.f, c + 1 <= r ? srow[1] : 0.f,
                                         c + 2 <= r ? srow[2] : 0.f, c + 3 <= r ? srow[3] : 0.f);
            *reinterpret_cast<float4*>(L + (size_t)(k0 + r) * n + k0 + c) = v;
          }
          cbar();
        }
        if (diag_only) continue;
        // (c) X = P T^T (triangle skipped), then L and the tensor-core copy from X^T.
        xgemm_tri_inplace(PtT, kWPtLd, dg.T, kD64Ld, cbar);
        // Output: first the tensor-core copy, published to the producer's bulk
        // copies (the proxy fence then covers only these stores), then L.
        float v[4][8];
#pragma unroll
        for (int it = 0; it < 4; ++it) {
          const int item = tid + kWConsumers * it;
          const int rl = item & (kWM - 1), c = item >> 7;
#pragma unroll
          for (int j = 0; j < 8; ++j) v[it][j] = PtT[(8 * c + j) * kWPtLd + rl];
          if (k + 1 < N && rl < vr && !(mt == 0 && rl < 64)) panel_copy_store<MODE>(W0, W1, N, k, r0 + rl, c, v[it]);
        }
        umma::fence_proxy_async_all();
        cbar();
        if (tid == 0) {
          // Completion number of tile mt: once per block column it exists in.
          const int done = (int)(biter * (int64_t)(N - 2 * mt) + k + 1);
#pragma unroll
          for (int q = 0; q < CL; ++q) st_release_cluster(br.tile_done + mt, (uint32_t)q, done);
        }
#pragma unroll
        for (int it = 0; it < 4; ++it) {
          const int item = tid + kWConsumers * it;
          const int rl = item & (kWM - 1), c = item >> 7;
          if (rl >= vr || (mt == 0 && rl < 64)) continue;
          float4* dst = reinterpret_cast<float4*>(L + (size_t)(r0 + rl) * n + k0 + 8 * c);
          dst[0] = make_float4(v[it][0], v[it][1], v[it][2], v[it][3]);
          dst[1] = make_float4(v[it][4], v[it][5], v[it][6], v[it][7]);
        }
        cbar();
      }
    }
    if (tid == 0 && rank == 0 && info != nullptr) info[b] = failed ? -1 : (*br.badp < 0 ? 0 : *br.badp + 1);
    if (grd.state != nullptr && rank == 0) {
      const int f =
          failed ? -1 : guard_audit_matrix<kWConsumers>(grd.piv + (size_t)b * n, n, MODE, &s_gmin, tid, cbar);
      if (tid == 0) grd.state[b] = f;
    }
    if (failed) {
      // Matrices this cluster did not reach are not rescued.
      if (grd.state != nullptr && rank == 0 && tid == 0)
        for (int64_t b2 = b + gridDim.x / CL; b2 < batch; b2 += gridDim.x / CL) grd.state[b2] = -1;
      break;
    }
  }
  // The strip's bulk stores read the zero buffer until they complete.
  if (tid == kWStripThread) umma::bulk_wait_all();
}

template <int MODE, int CL>
__global__ void __launch_bounds__(kWThreads, 1)
    potrf_fused_ws_kernel(const float* __restrict__ a, float* __restrict__ l, int64_t batch, int n,
                          uint8_t* __restrict__ ws, int32_t* __restrict__ info, GuardRec grd) {
  // The rescue's grid barrier starts from zero (it runs after this kernel).
  if (grd.bar != nullptr && blockIdx.x == 0 && threadIdx.x == 0) grd.bar[0] = grd.bar[1] = 0;
  extern __shared__ unsigned char wraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(wraw) + 1023) & ~(uintptr_t)1023);
  WsBars br;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kWBarOff);
  br.full = bars;
  br.empty = bars + 2;
  br.acc_ready = bars + 4;
  br.acc_free = bars + 12;
  br.tile_done = reinterpret_cast<int*>(sm + kWCntOff);
  br.drain = bars + 28;
  br.tslot = reinterpret_cast<uint32_t*>(bars + 29);
  br.flag = reinterpret_cast<volatile int*>(bars + 30);
  br.badp = reinterpret_cast<int*>(bars + 30) + 1;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) *br.flag = 0;
  if (tid < kWMaxTiles) br.tile_done[tid] = 0;
  for (uint32_t e = tid; e < kWZeroBytes / 16; e += kWThreads)
    reinterpret_cast<float4*>(sm + kWZeroOff)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  // The zeros are read by the async proxy (bulk stores).
  umma::fence_proxy_async_smem();
  if (warp == 0) {
    umma::tmem_alloc(br.tslot, kWTmemCols);
    umma::tmem_relinquish();
  }
  if (tid == 32) {
    for (int i = 0; i < 4; ++i) umma::mbar_init(bars + i, 1);             // full, empty
    for (int i = 0; i < 8; ++i) umma::mbar_init(br.acc_ready + i, 1);     // tcgen05.commit
    for (int i = 0; i < 8; ++i) umma::mbar_init(br.acc_free + i, 8);      // one arrive per consumer warp
    umma::mbar_init(br.drain, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  // The peer's barriers are initialised before anyone arrives on them.
  if (CL > 1) umma::cluster_sync();
  umma::fence_after_sync();
  const uint32_t tmem = *br.tslot;
  const int rank = CL > 1 ? (int)umma::cluster_rank() : 0;
  if (warp == kWConsumers / 32) {
    if ((tid & 31) == 0) ws_producer<MODE, CL>(br, sm, ws, batch, n, tmem, rank);
  } else {
    ws_consumers<MODE, CL>(br, sm, a, l, ws, batch, n, tmem, info, rank, grd);
  }
  umma::fence_before_sync();
  __syncthreads();
  // No CTA leaves while its peer may still arrive on its barriers.
  if (CL > 1) umma::cluster_sync();
  if (warp == 0) umma::tmem_dealloc(tmem, kWTmemCols);
}

// CTAs per matrix for (batch, n): as many as the SMs allow (up to the
// portable cluster size of 8, no more than a block column has row tiles),
// and at least enough that every rank's tile list fits the TMEM slots.
// 0 if n needs more than 8.
static int ws_cluster_size(int64_t batch, int n) {
  const int mt_n = (n + kWM - 1) / kWM;
  int need = 1;
  while (need <= 8 && (mt_n + need - 1) / need + (need > 1 ? 1 : 0) > kWMaxSlots) need *= 2;
  if (need > 8 || mt_n > kWMaxTiles) return 0;
  const int64_t sms = device_sms();
  int cl = need;
  while (cl < 8 && batch * cl * 2 <= sms && cl * 2 <= mt_n) cl *= 2;
  return cl;
}

// Orders up to 1024.  Larger ones would fit (clusters big enough for TMEM),
// but with K up to n every CTA then streams its whole row range of panel
// copies per block column and is bound by its own bulk-copy bandwidth
// (8x2048: 1630 us against 1351 us on the split path; 1x4096: 7490 vs 2335).
bool fused_ws_fits(int64_t batch, int64_t n, int mode) {
  const int m = mode & B2P_MODE_MASK;
  return (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3) && !(mode & B2P_FLAG_FP64_DIAG) && n > 128 && n % 64 == 0 &&
         n <= 8192 && ws_cluster_size(batch, (int)n) > 0;
}

bool fused_ws_supported(int64_t batch, int64_t n, int mode) { return n <= 1024 && fused_ws_fits(batch, n, mode); }

int potrf_fused_ws(const float* a, float* l, int64_t batch, int n, int mode, void* ws, size_t ws_bytes,
                   int32_t* info, cudaStream_t s, GuardRec grd) {
  const size_t need = fused_workspace_bytes(batch, n);
  if (ws == nullptr || ws_bytes < need)
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", need, ws_bytes);
  uint8_t* wsa = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(ws) + 1023) & ~(uintptr_t)1023);
  const int64_t sms = device_sms();
  const int cl = ws_cluster_size(batch, n);
  if (cl == 0 || !fused_ws_fits(batch, n, mode))
    return set_error(B2P_ERR_UNSUPPORTED, "warp-specialized path: n=%d not supported", n);
  const int grid = cl * (int)std::max<int64_t>(1, std::min<int64_t>(batch, sms / cl));
  const bool tf32 = (mode & B2P_MODE_MASK) == B2P_MODE_TF32;
  using Kern = void (*)(const float*, float*, int64_t, int, uint8_t*, int32_t*, GuardRec);
  static const Kern kernels[2][4] = {
      {potrf_fused_ws_kernel<B2P_MODE_TF32, 1>, potrf_fused_ws_kernel<B2P_MODE_TF32, 2>,
       potrf_fused_ws_kernel<B2P_MODE_TF32, 4>, potrf_fused_ws_kernel<B2P_MODE_TF32, 8>},
      {potrf_fused_ws_kernel<B2P_MODE_BF16X3, 1>, potrf_fused_ws_kernel<B2P_MODE_BF16X3, 2>,
       potrf_fused_ws_kernel<B2P_MODE_BF16X3, 4>, potrf_fused_ws_kernel<B2P_MODE_BF16X3, 8>}};
  const int li = cl == 1 ? 0 : cl == 2 ? 1 : cl == 4 ? 2 : 3;
  const Kern kern = kernels[tf32 ? 0 : 1][li];
  if (int st = ensure_smem_attr((const void*)kern, kWSmemBytes, kSlotFusedWs0 + (tf32 ? 0 : 4) + li)) return st;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3(kWThreads, 1, 1);
  cfg.dynamicSmemBytes = kWSmemBytes;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  TraceScope ts(kKFusedWs, s, (double)batch * n * n * n / 3.0);
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, a, l, batch, n, wsa, info, grd);
  if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "potrf_fused_ws_kernel: %s", cudaGetErrorString(e));
  return B2P_OK;
}

}  // namespace b2p
