// Batched GEMM on the tcgen05 tensor cores with structure hints, used by the
// Cholesky adjoint (potrf_backward.cu).
//
//   C[b] = alpha * op1(X[b]) * op2(Y[b]) + beta * C[b]      (M x N, K inner)
//
// op1(X)[m][k] is X[m][k] (kTransNone) or X[k][m] (kTrans); op2(Y)[k][n] is
// Y[k][n] or Y[n][k].  Structure hints let a 128x128 output tile skip the
// parts of K where an operand is known to be zero (triangular operands), skip
// tiles strictly above the diagonal when only the lower triangle of C is
// wanted, and apply Phi (keep the lower triangle, halve the diagonal) in the
// epilogue.  One 128-thread CTA per output tile: per 64-wide K chunk every
// thread stages one operand row (128B-swizzled K-major, BF16 hi/lo split or
// TF32), thread 0 issues the MMAs into a 128x128 FP32 TMEM accumulator, and
// the epilogue reads TMEM with tcgen05.ld.  Waits are bounded.
#include <algorithm>

#include "launch.h"
#include "umma.cuh"

namespace b2p {

constexpr int kGT = 128;  // tile edge
constexpr int kGK = 64;   // K chunk
constexpr int kGThreads = 128;
constexpr uint32_t kGPolls = 1u << 24;
constexpr size_t kGOperand = 32768;
constexpr size_t kGSmem = 2 * kGOperand + 1024 + 64;


__device__ __forceinline__ float g_round_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Write 64 K values of operand row r into the swizzled tile.
template <int MODE>
__device__ __forceinline__ void g_store_row(uint8_t* op, int r, const float (&v)[64]) {
  if (MODE == B2P_MODE_TF32) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const float4 t = make_float4(g_round_tf32(v[4 * q]), g_round_tf32(v[4 * q + 1]), g_round_tf32(v[4 * q + 2]),
                                   g_round_tf32(v[4 * q + 3]));
      *reinterpret_cast<float4*>(op + (q >> 3) * 16384 + umma::sw128_offset(r, q & 7)) = t;
    }
  } else {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        __nv_bfloat16 h0, l0, h1, l1;
        umma::split_bf16(v[8 * c + 2 * p], h0, l0);
        umma::split_bf16(v[8 * c + 2 * p + 1], h1, l1);
        hi[p] = umma::pack_bf16(h0, h1);
        lo[p] = umma::pack_bf16(l0, l1);
      }
      const uint32_t off = umma::sw128_offset(r, c);
      *reinterpret_cast<uint4*>(op + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4*>(op + 16384 + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
  }
}

// Operand row `r` (0..127) of a tile: logical element (row0 + r, k0 + kk).
// `rowmajor`: element (i, kk) at mat[i*ld + kk] (K contiguous) else at
// mat[kk*ld + i] (rows contiguous across threads: coalesced).
template <int MODE>
__device__ __forceinline__ void g_stage(const float* mat, int ld, bool rowmajor, int rows, int kdim, int row0,
                                        int k0, uint8_t* op, int r) {
  float v[64];
  const int i = row0 + r;
  if (rowmajor) {
    const float* p = mat + (size_t)i * ld + k0;
    const bool full = (i < rows) && (k0 + kGK <= kdim) && ((ld & 3) == 0);
    if (full) {
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float4 t = reinterpret_cast<const float4*>(p)[q];
        v[4 * q] = t.x;
        v[4 * q + 1] = t.y;
        v[4 * q + 2] = t.z;
        v[4 * q + 3] = t.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < 64; ++q) v[q] = (i < rows && k0 + q < kdim) ? p[q] : 0.0f;
    }
  } else {
    const float* p = mat + (size_t)k0 * ld + i;
#pragma unroll
    for (int q = 0; q < 64; ++q) v[q] = (i < rows && k0 + q < kdim) ? p[(size_t)q * ld] : 0.0f;
  }
  g_store_row<MODE>(op, r, v);
}

template <int MODE>
__device__ __forceinline__ void g_mmas(uint32_t tmem, uint32_t a, uint32_t b, bool acc) {
  if (MODE == B2P_MODE_TF32) {
    constexpr uint32_t idesc = umma::idesc_f32acc(2, kGT, kGT);
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const uint32_t off = (uint32_t)((s >> 2) * 16384 + (s & 3) * 32);
      umma::mma_tf32(tmem, umma::desc_k_sw128(a + off), umma::desc_k_sw128(b + off), idesc, (acc || s) ? 1u : 0u);
    }
  } else {
    constexpr uint32_t idesc = umma::idesc_f32acc(1, kGT, kGT);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const uint32_t off = (uint32_t)(s * 32);
      const uint64_t ah = umma::desc_k_sw128(a + off), al = umma::desc_k_sw128(a + 16384 + off);
      const uint64_t bh = umma::desc_k_sw128(b + off), bl = umma::desc_k_sw128(b + 16384 + off);
      umma::mma_bf16(tmem, al, bh, idesc, (acc || s) ? 1u : 0u);
      umma::mma_bf16(tmem, ah, bl, idesc, 1u);
      umma::mma_bf16(tmem, ah, bh, idesc, 1u);
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(kGThreads, 1) gemm_tc_kernel(GemmArgs g, int tiles_n, int32_t* err) {
  extern __shared__ unsigned char graw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(graw) + 1023) & ~(uintptr_t)1023);
  uint8_t* opA = base;
  uint8_t* opB = base + kGOperand;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(base + 2 * kGOperand);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(base + 2 * kGOperand + 8);
  int* flag = reinterpret_cast<int*>(base + 2 * kGOperand + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // Tile coordinates (lower_out: triangular enumeration).
  int tm, tn;
  if (g.lower_out) {
    const int q = blockIdx.x;
    tm = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
    while ((tm + 1) * (tm + 2) / 2 <= q) ++tm;
    while (tm * (tm + 1) / 2 > q) --tm;
    tn = q - tm * (tm + 1) / 2;
  } else {
    tm = blockIdx.x / tiles_n;
    tn = blockIdx.x - tm * tiles_n;
  }
  const int m0 = tm * kGT, n0 = tn * kGT;
  // K range from the triangular hints.
  int klo = 0, khi = g.k;
  if (g.x_tri == 1) khi = min(khi, m0 + kGT);
  if (g.x_tri == 2) klo = max(klo, m0);
  if (g.y_tri == 1) klo = max(klo, n0);
  if (g.y_tri == 2) khi = min(khi, n0 + kGT);
  klo = (klo / kGK) * kGK;

  if (tid == 0) *flag = 0;
  if (warp == 0) {
    umma::tmem_alloc(tslot, kGT);
    umma::tmem_relinquish();
  }
  if (tid == 32) {
    umma::mbar_init(mbar, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  uint32_t parity = 0;
  bool ok = true;
  int64_t b = blockIdx.y;
  const int64_t nb2 = g.batch2 > 0 ? g.batch2 : 1;
  for (; b < g.batch * nb2 && ok; b += gridDim.y) {
    const int64_t b1 = b / nb2, b2 = b - (b / nb2) * nb2;
    const float* X = g.x + b1 * g.sx + b2 * g.sx2;
    const float* Y = g.y + b1 * g.sy + b2 * g.sy2;
    float* C = g.c + b1 * g.sc + b2 * g.sc2;
    const float* Cin = (g.c_in ? g.c_in : g.c) + b1 * g.sc + b2 * g.sc2;
    bool any = false;
    for (int k0 = klo; k0 < khi; k0 += kGK) {
      // A operand: rows m (op1(X)[m][k]); B operand: rows n (op2(Y)[k][n]).
      g_stage<MODE>(X, g.ldx, !g.trans_x, g.m, g.k, m0, k0, opA, tid);
      g_stage<MODE>(Y, g.ldy, g.trans_y, g.n, g.k, n0, k0, opB, tid);
      umma::fence_proxy_async_smem();
      umma::fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        umma::fence_after_sync();
        g_mmas<MODE>(tmem, umma::smem_u32(opA), umma::smem_u32(opB), any);
        umma::mma_commit(mbar);
      }
      const bool got = umma::mbar_wait_bounded(mbar, parity, kGPolls);
      parity ^= 1u;
      umma::fence_after_sync();
      if (!got) *flag = 1;
      __syncthreads();
      if (*flag) {
        ok = false;
        break;
      }
      any = true;
    }
    if (!ok) break;
    // Epilogue: row i = m0 + 32*warp + lane, 4 chunks of 32 columns.
    const int i = m0 + 32 * warp + lane;
#pragma unroll 1
    for (int ch = 0; ch < 4; ++ch) {
      float v[32];
      if (any) {
        umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * ch), v);
      } else {
#pragma unroll
        for (int e = 0; e < 32; ++e) v[e] = 0.0f;
      }
      if (i < g.m) {
        float* crow = C + (size_t)i * g.ldc;
        const float* cin = Cin + (size_t)i * g.ldc;
#pragma unroll
        for (int e = 0; e < 32; ++e) {
          const int j = n0 + 32 * ch + e;
          if (j < g.n && (!g.lower_out || j <= i)) {
            float r = g.alpha * v[e];
            if (g.phi) r = (j > i) ? 0.0f : (j == i ? 0.5f * r : r);
            if (g.beta != 0.0f) r += g.beta * cin[j];
            crow[j] = r;
          }
        }
      }
    }
    umma::fence_before_sync();
    __syncthreads();
  }
  if (!ok && tid == 0 && err != nullptr) atomicExch(err, B2P_ERR_TIMEOUT);
  if (!ok) umma::mbar_wait_bounded(mbar, parity ^ 1u, kGPolls);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kGT);
}

// ---- packed operands + bulk-copy pipeline ----------------------------------------
// Packed operand layout, per batch item: block (row tile t, K chunk c) of
// 32 KB at ((t * tiles_k) + c) * 32 KB -- exactly the shared-memory image
// g_stage writes (BF16 hi at +0 and lo at +16 KB, or the two TF32 K-halves),
// zero-filled beyond the matrix.
constexpr int kGStages = 3;
constexpr size_t kGStage = 2 * kGOperand;  // A + B
constexpr size_t kGBulkSmem = kGStages * kGStage + 1024 + 128;

size_t gemm_pack_bytes(int64_t batch, int rows, int kdim) {
  return (size_t)batch * (size_t)((rows + kGT - 1) / kGT) * (size_t)((kdim + kGK - 1) / kGK) * kGOperand;
}

// One 32 KB block (row tile, K chunk) per CTA; thread = (row r, 16-wide K
// part p), so that four threads share a row and the CTA keeps many loads in
// flight.  Reads are coalesced in either orientation (row-major: 64 bytes of
// one row per thread; transposed: consecutive rows across a warp).
constexpr int kPThreads = 512;

template <int MODE>
__global__ void __launch_bounds__(kPThreads) gemm_pack_kernel(const float* __restrict__ mat, int64_t s1, int64_t s2,
                                                              int64_t nb2, int ld, int rowmajor, int rows, int kdim,
                                                              int tiles_k, int64_t items, uint8_t* __restrict__ out) {
  const int tr = blockIdx.x / tiles_k, tk = blockIdx.x - (blockIdx.x / tiles_k) * tiles_k;
  const int r = threadIdx.x & 127, p = threadIdx.x >> 7;
  const int i = tr * kGT + r, k0 = tk * kGK + 16 * p;
  const size_t per = (size_t)((rows + kGT - 1) / kGT) * tiles_k * kGOperand;
  for (int64_t b = blockIdx.y; b < items; b += gridDim.y) {
    const int64_t b1 = b / nb2, b2 = b - (b / nb2) * nb2;
    const float* M = mat + b1 * s1 + b2 * s2;
    float v[16];
    if (rowmajor) {
      const float* src = M + (size_t)i * ld + k0;
      if (i < rows && k0 + 16 <= kdim && ((reinterpret_cast<uintptr_t>(src) & 15u) == 0)) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 t = __ldg(reinterpret_cast<const float4*>(src) + q);
          v[4 * q] = t.x;
          v[4 * q + 1] = t.y;
          v[4 * q + 2] = t.z;
          v[4 * q + 3] = t.w;
        }
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = (i < rows && k0 + q < kdim) ? __ldg(src + q) : 0.0f;
      }
    } else {
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = (i < rows && k0 + q < kdim) ? __ldg(M + (size_t)(k0 + q) * ld + i) : 0.0f;
    }
    uint8_t* op = out + b * per + (size_t)blockIdx.x * kGOperand;
    if (MODE == B2P_MODE_TF32) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int Q = 4 * p + q;  // float4 index within the 64-wide row
        const float4 t = make_float4(g_round_tf32(v[4 * q]), g_round_tf32(v[4 * q + 1]), g_round_tf32(v[4 * q + 2]),
                                     g_round_tf32(v[4 * q + 3]));
        *reinterpret_cast<float4*>(op + (Q >> 3) * 16384 + umma::sw128_offset(r, Q & 7)) = t;
      }
    } else {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          __nv_bfloat16 h0, l0, h1, l1;
          umma::split_bf16(v[8 * c + 2 * q], h0, l0);
          umma::split_bf16(v[8 * c + 2 * q + 1], h1, l1);
          hi[q] = umma::pack_bf16(h0, h1);
          lo[q] = umma::pack_bf16(l0, l1);
        }
        const uint32_t off = umma::sw128_offset(r, 2 * p + c);
        *reinterpret_cast<uint4*>(op + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(op + 16384 + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      }
    }
  }
}

// Persistent, warp-specialized product over packed operands.  Warp 4 (one
// thread) streams the packed 32 KB blocks through a 3-stage ring two chunks
// ahead of the MMAs (across tile boundaries) and issues the MMAs of each
// tile into one of two 128-column TMEM accumulators; warps 0-3 run the
// epilogue of the previous tile from the other accumulator meanwhile.
constexpr int kBEpi = 128;
constexpr int kBThreads = kBEpi + 32;

struct BulkTile {
  int64_t b;    // flattened batch item
  int m0, n0;   // output tile origin
  int kc0, nch; // K chunks [kc0, kc0 + nch)
};

__device__ __forceinline__ BulkTile bulk_decode(const GemmArgs& g, int tiles, int tiles_n, int64_t w) {
  BulkTile t;
  const int q = (int)(w % tiles);
  t.b = w / tiles;
  int tm, tn;
  if (g.lower_out) {
    tm = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
    while ((tm + 1) * (tm + 2) / 2 <= q) ++tm;
    while (tm * (tm + 1) / 2 > q) --tm;
    tn = q - tm * (tm + 1) / 2;
  } else {
    tm = q / tiles_n;
    tn = q - tm * tiles_n;
  }
  t.m0 = tm * kGT;
  t.n0 = tn * kGT;
  int klo = 0, khi = g.k;
  if (g.x_tri == 1) khi = min(khi, t.m0 + kGT);
  if (g.x_tri == 2) klo = max(klo, t.m0);
  if (g.y_tri == 1) klo = max(klo, t.n0);
  if (g.y_tri == 2) khi = min(khi, t.n0 + kGT);
  t.kc0 = klo / kGK;
  t.nch = khi > klo ? (khi + kGK - 1) / kGK - t.kc0 : 0;
  return t;
}

template <int MODE>
__global__ void __launch_bounds__(kBThreads, 1) gemm_bulk_kernel(GemmArgs g, int tiles_n, int tiles, int32_t* err) {
  extern __shared__ unsigned char graw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(graw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kGStages * kGStage);  // [kGStages]
  uint64_t* empty = full + kGStages;                                         // [kGStages]
  uint64_t* accf = empty + kGStages;                                         // [2] accumulator complete
  uint64_t* accd = accf + 2;                                                 // [2] accumulator read out
  uint64_t* fin = accd + 2;                                                  // [1] every MMA done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
  volatile int* flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int64_t nb2 = g.batch2 > 0 ? g.batch2 : 1;
  const int64_t W = (int64_t)tiles * g.batch * nb2;
  const int tiles_k = (g.k + kGK - 1) / kGK;
  const size_t per_x = (size_t)((g.m + kGT - 1) / kGT) * tiles_k * kGOperand;
  const size_t per_y = (size_t)((g.n + kGT - 1) / kGT) * tiles_k * kGOperand;

  if (tid == 0) *flag = 0;
  if (warp == 0) {
    umma::tmem_alloc(tslot, 2 * kGT);
    umma::tmem_relinquish();
  }
  if (tid == 32) {
    for (int i = 0; i < 2 * kGStages + 2; ++i) umma::mbar_init(full + i, 1);  // full, empty, accf
    for (int i = 0; i < 2; ++i) umma::mbar_init(accd + i, kBEpi / 32);
    umma::mbar_init(fin, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;

  if (warp == kBEpi / 32) {
    // ---------------- producer / MMA issuer ----------------
    if (lane == 0) {
      uint32_t gload = 0, guse = 0;
      bool ok = true;
      // Loader cursor: the next chunk to bring in (item lw, chunk lc).
      int64_t lw = blockIdx.x;
      int lc = 0;
      BulkTile lt = lw < W ? bulk_decode(g, tiles, tiles_n, lw) : BulkTile{};
      auto load_next = [&]() -> bool {
        while (lw < W && lc >= lt.nch) {
          lw += gridDim.x;
          lc = 0;
          if (lw < W) lt = bulk_decode(g, tiles, tiles_n, lw);
        }
        if (lw >= W) return true;  // nothing left to load
        const uint32_t st = gload % kGStages;
        if (gload >= (uint32_t)kGStages &&
            !umma::mbar_wait_bounded(empty + st, ((gload / kGStages) - 1u) & 1u, kGPolls))
          return false;
        const int tm = lt.m0 / kGT, tn = lt.n0 / kGT;
        const uint8_t* PX = g.pack_x + lt.b * per_x + ((size_t)tm * tiles_k + lt.kc0 + lc) * kGOperand;
        const uint8_t* PY = g.pack_y + lt.b * per_y + ((size_t)tn * tiles_k + lt.kc0 + lc) * kGOperand;
        uint8_t* dst = base + st * kGStage;
        umma::mbar_arrive_expect_tx(full + st, (uint32_t)(2 * kGOperand));
        umma::bulk_g2s(dst, PX, (uint32_t)kGOperand, full + st);
        umma::bulk_g2s(dst + kGOperand, PY, (uint32_t)kGOperand, full + st);
        ++gload;
        ++lc;
        return true;
      };
      for (int i = 0; i < kGStages - 1 && ok; ++i) ok = load_next();
      uint32_t li = 0;
      for (int64_t w = blockIdx.x; w < W && ok; w += gridDim.x, ++li) {
        const BulkTile t = bulk_decode(g, tiles, tiles_n, w);
        const uint32_t p = li & 1u;
        // Accumulator p is free once the epilogue has read tile li - 2.
        if (li >= 2 && !umma::mbar_wait_bounded(accd + p, ((li - 2) >> 1) & 1u, kGPolls)) {
          ok = false;
          break;
        }
        umma::fence_after_sync();
        for (int i = 0; i < t.nch && ok; ++i) {
          const uint32_t st = guse % kGStages;
          if (!umma::mbar_wait_bounded(full + st, (guse / kGStages) & 1u, kGPolls)) {
            ok = false;
            break;
          }
          ++guse;
          umma::fence_after_sync();
          const uint32_t sa = umma::smem_u32(base + st * kGStage);
          g_mmas<MODE>(tmem + p * kGT, sa, sa + (uint32_t)kGOperand, i > 0);
          umma::mma_commit(empty + st);
          // Refill the stage of chunk guse - 2 (its MMAs ran before this one's).
          ok = load_next();
        }
        if (ok) umma::mma_commit(accf + p);
      }
      if (!ok) {
        // Copies still in flight land before anything leaves.
        for (uint32_t c = guse; c < gload; ++c)
          umma::mbar_wait_bounded(full + (c % kGStages), (c / kGStages) & 1u, kGPolls);
        *flag = 1;
      }
      umma::mma_commit(fin);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue: row i = m0 + 32 warp + lane ----------------
    uint32_t li = 0;
    for (int64_t w = blockIdx.x; w < W; w += gridDim.x, ++li) {
      const BulkTile t = bulk_decode(g, tiles, tiles_n, w);
      const uint32_t p = li & 1u;
      const bool got = umma::mbar_wait_bounded(accf + p, (li >> 1) & 1u, kGPolls) && *flag == 0;
      if (!__all_sync(0xffffffffu, got)) {
        *flag = 1;
        if (lane == 0 && err != nullptr) atomicExch(err, B2P_ERR_TIMEOUT);
        break;
      }
      umma::fence_after_sync();
      const int64_t b1 = t.b / nb2, b2 = t.b - (t.b / nb2) * nb2;
      float* C = g.c + b1 * g.sc + b2 * g.sc2;
      const float* Cin = (g.c_in ? g.c_in : g.c) + b1 * g.sc + b2 * g.sc2;
      const int i = t.m0 + 32 * warp + lane;
#pragma unroll 1
      for (int ch = 0; ch < 4; ++ch) {
        float v[32];
        if (t.nch > 0) {
          umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + p * kGT + (uint32_t)(32 * ch), v);
        } else {
#pragma unroll
          for (int e = 0; e < 32; ++e) v[e] = 0.0f;
        }
        if (i < g.m) {
          float* crow = C + (size_t)i * g.ldc;
          const float* cin = Cin + (size_t)i * g.ldc;
#pragma unroll
          for (int e = 0; e < 32; ++e) {
            const int j = t.n0 + 32 * ch + e;
            if (j < g.n && (!g.lower_out || j <= i)) {
              float r = g.alpha * v[e];
              if (g.phi) r = (j > i) ? 0.0f : (j == i ? 0.5f * r : r);
              if (g.beta != 0.0f) r += g.beta * cin[j];
              crow[j] = r;
            }
          }
        }
      }
      umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(accd + p);
    }
  }
  // Every MMA has completed before TMEM is released.
  umma::mbar_wait_bounded(fin, 0u, kGPolls);
  umma::fence_after_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 2 * kGT);
}

template <int MODE>
static int launch_gemm_packed(const GemmArgs& g, int32_t* err, cudaStream_t s, int slot_bulk) {
  const int tm = (g.m + kGT - 1) / kGT, tn = (g.n + kGT - 1) / kGT, tk = (g.k + kGK - 1) / kGK;
  const int64_t nb2 = g.batch2 > 0 ? g.batch2 : 1;
  const int64_t items = g.batch * nb2;
  const unsigned by = (unsigned)std::min<int64_t>(items, 65535);
  {
    TraceScope ts(kKBwdGemm, s);
    gemm_pack_kernel<MODE><<<dim3(tm * tk, by), kPThreads, 0, s>>>(g.x, g.sx, g.sx2, nb2, g.ldx, !g.trans_x, g.m,
                                                                    g.k, tk, items, g.pack_x);
    gemm_pack_kernel<MODE><<<dim3(tn * tk, by), kPThreads, 0, s>>>(g.y, g.sy, g.sy2, nb2, g.ldy, g.trans_y, g.n,
                                                                    g.k, tk, items, g.pack_y);
    if (int st = check_launch("gemm_pack_kernel")) return st;
  }
  if (int st = ensure_smem_attr((const void*)gemm_bulk_kernel<MODE>, kGBulkSmem, slot_bulk)) return st;
  const int tiles = g.lower_out ? tm * (tm + 1) / 2 : tm * tn;
  const int64_t work = (int64_t)tiles * items;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(work, (int64_t)device_sms()));
  TraceScope ts(kKBwdGemm, s);
  gemm_bulk_kernel<MODE><<<grid, kBThreads, kGBulkSmem, s>>>(g, tn, tiles, err);
  return check_launch("gemm_bulk_kernel");
}

int launch_gemm_tc(const GemmArgs& g, int mode, int32_t* err, cudaStream_t s) {
  if (g.batch <= 0 || g.m <= 0 || g.n <= 0) return B2P_OK;
  if (g.pack_x != nullptr && g.pack_y != nullptr && g.k > 0) {
    if ((mode & B2P_MODE_MASK) == B2P_MODE_TF32) return launch_gemm_packed<B2P_MODE_TF32>(g, err, s, kSlotBwdBulk0);
    return launch_gemm_packed<B2P_MODE_BF16X3>(g, err, s, kSlotBwdBulk1);
  }
  const int tm = (g.m + kGT - 1) / kGT, tn = (g.n + kGT - 1) / kGT;
  const int tiles = g.lower_out ? tm * (tm + 1) / 2 : tm * tn;
  const dim3 grid(tiles, (unsigned)std::min<int64_t>(g.batch * (g.batch2 > 0 ? g.batch2 : 1), 65535));
  TraceScope ts(kKBwdGemm, s);
  if ((mode & B2P_MODE_MASK) == B2P_MODE_TF32) {
    if (int st = ensure_smem_attr((const void*)gemm_tc_kernel<B2P_MODE_TF32>, kGSmem, kSlotBwd0)) return st;
    gemm_tc_kernel<B2P_MODE_TF32><<<grid, kGThreads, kGSmem, s>>>(g, tn, err);
  } else {
    if (int st = ensure_smem_attr((const void*)gemm_tc_kernel<B2P_MODE_BF16X3>, kGSmem, kSlotBwd1)) return st;
    gemm_tc_kernel<B2P_MODE_BF16X3><<<grid, kGThreads, kGSmem, s>>>(g, tn, err);
  }
  return check_launch("gemm_tc_kernel");
}

}  // namespace b2p
