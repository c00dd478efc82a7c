// Tensor-core copy of solved panels, shared by the left-looking kernels
// (potrf_fused.cu, potrf_fused_ws.cu, potrf_split.cu).
//
// Every solved block column c (64 wide) of a matrix of order n = 64 N is
// stored a second time in a workspace, already in the operand format of
// tcgen05.mma: two regions per matrix (BF16 hi and lo of BF16x3, the two
// 32-column K-halves of TF32, or for FP8 the scaled BF16 hi and one 128-byte
// line of E4M3 [hi | lo]), each holding for column c the rows
// 64(c+1)..n-1 (the only rows later updates read) as 128-byte K-major lines
// in 8-row, 1024-byte 128B-swizzle atoms.  Rows of one column are contiguous,
// so a 128-row operand tile is one 16 KB bulk copy per region, and the row
// offset of column c is  64 (c (N-1) - c (c-1)/2)  rows from the region base.
#pragma once

#include <cuda_fp8.h>

#include "umma.cuh"

namespace b2p {

// Bytes of one region for a matrix of order n (n multiple of 64).
__host__ __device__ inline size_t panel_copy_region_bytes(int n) {
  const size_t N = (size_t)(n / 64);
  return 4096 * N * (N - 1);
}

// Byte offset of global row r (r >= 64 (c+1)) of column c within a region.
__device__ __forceinline__ size_t panel_copy_row_byte(int N, int c, int r) {
  return (size_t)(64 * (c * (N - 1) - c * (c - 1) / 2) + r - 64 * (c + 1)) * 128;
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// FP8 mode (per-tile-scaled E4M3 cross terms).  Each row r of the factor
// has a power-of-two scale s_r = sigma of its 64-row block, with
// |L[r][j]| <= sqrt(A_rr) <= 256 s_r.  With hi = bf16(x), lo = x - hi:
//   region 0:  h = hi * 16 / s_r            (BF16, exact: a power-of-two shift)
//   region 1:  bytes 0..63   q = e4m3(hi / s_r)
//              bytes 64..127 p = e4m3(lo * 256 / s_r)
// so that h_i h_j + q_i p_j + p_i q_j = 256 (x_i x_j) / (s_i s_j) up to the
// E4M3 rounding of the cross terms (relative 2^-4 of terms themselves 2^-8
// of the product: about 2^-12 in all).  The products accumulate in one FP32
// accumulator and the fold multiplies by s_i s_j / 256.
constexpr float kFp8Fold = 1.0f / 256.0f;

// Store columns 8 tx .. 8 tx + 7 (values v) of global row r of column c.
// isig = 1 / s_r (FP8 mode only).
template <int MODE>
__device__ __forceinline__ void panel_copy_store(uint8_t* w0, uint8_t* w1, int N, int c, int r, int tx,
                                                 const float (&v)[8], float isig = 1.0f) {
  const size_t row = panel_copy_row_byte(N, c, r);
  const int r8 = r & 7;
  if (MODE == B2P_MODE_FP8) {
    uint32_t h[4];
    uint32_t q[2], p[2];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * e]), h1 = __float2bfloat16_rn(v[2 * e + 1]);
      const float f0 = __bfloat162float(h0), f1 = __bfloat162float(h1);
      h[e] = umma::pack_bf16(__float2bfloat16_rn(f0 * 16.0f * isig), __float2bfloat16_rn(f1 * 16.0f * isig));
      const uint32_t qq = __nv_cvt_float2_to_fp8x2(make_float2(f0 * isig, f1 * isig), __NV_SATFINITE, __NV_E4M3);
      const uint32_t pp = __nv_cvt_float2_to_fp8x2(
          make_float2((v[2 * e] - f0) * 256.0f * isig, (v[2 * e + 1] - f1) * 256.0f * isig), __NV_SATFINITE,
          __NV_E4M3);
      if (e & 1) {
        q[e >> 1] |= qq << 16;
        p[e >> 1] |= pp << 16;
      } else {
        q[e >> 1] = qq;
        p[e >> 1] = pp;
      }
    }
    *reinterpret_cast<uint4*>(w0 + row + ((tx ^ r8) << 4)) = make_uint4(h[0], h[1], h[2], h[3]);
    // 8 E4M3 values = 8 bytes: half of 16-byte chunk tx / 2 (q) and of 4 + tx / 2 (p).
    const int half = (tx & 1) * 8;
    *reinterpret_cast<uint2*>(w1 + row + (((tx >> 1) ^ r8) << 4) + half) = make_uint2(q[0], q[1]);
    *reinterpret_cast<uint2*>(w1 + row + (((4 + (tx >> 1)) ^ r8) << 4) + half) = make_uint2(p[0], p[1]);
  } else if (MODE == B2P_MODE_TF32) {
    uint8_t* reg = (tx < 4) ? w0 : w1;
    const int c0 = 2 * (tx & 3);
    *reinterpret_cast<float4*>(reg + row + ((c0 ^ r8) << 4)) =
        make_float4(tf32_rna(v[0]), tf32_rna(v[1]), tf32_rna(v[2]), tf32_rna(v[3]));
    *reinterpret_cast<float4*>(reg + row + (((c0 + 1) ^ r8) << 4)) =
        make_float4(tf32_rna(v[4]), tf32_rna(v[5]), tf32_rna(v[6]), tf32_rna(v[7]));
  } else {
    uint32_t h[4], lo[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      __nv_bfloat16 h0, l0, h1, l1;
      umma::split_bf16(v[2 * p], h0, l0);
      umma::split_bf16(v[2 * p + 1], h1, l1);
      h[p] = umma::pack_bf16(h0, h1);
      lo[p] = umma::pack_bf16(l0, l1);
    }
    const size_t off = row + ((tx ^ r8) << 4);
    *reinterpret_cast<uint4*>(w0 + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(w1 + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
}

// D (128 x NB FP32 in TMEM) (+)= A B^T over one 64-wide column, from staged
// copies: A = 128 rows at sa (region 0 at +0, region 1 at +A1), B = NB rows
// at sb (region 0 at +0, region 1 at +128 NB).  One thread issues.  A1 below
// 16384 lets A overlap B's staging when only A's first A1 / 128 rows matter
// (their accumulator lanes); the rows beyond read whatever follows in
// shared memory.
template <int MODE, int NB = 64, uint32_t A1 = 16384u>
__device__ __forceinline__ void panel_copy_mmas(uint32_t d, uint32_t sa, uint32_t sb, bool acc) {
  static_assert(NB % 16 == 0 && NB >= 16 && NB <= 256, "MMA N for M = 128");
  static_assert(A1 % 1024 == 0, "SW128 operands start on 1024-byte boundaries");
  constexpr uint32_t kB1 = 128u * NB;
  if (MODE == B2P_MODE_FP8) {
    // h h^T on kind::f16 (K = 16 per instruction), then q p^T and p q^T on
    // kind::f8f6f4 (K = 32 per instruction): bytes 0..63 of a region-1
    // line hold q, bytes 64..127 p.
    constexpr uint32_t ib = umma::idesc_f32acc(1, 128, NB);
    constexpr uint32_t i8 = umma::idesc_f32acc(0, 128, NB);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const uint32_t o = (uint32_t)(s * 32);
      umma::mma_bf16(d, umma::desc_k_sw128(sa + o), umma::desc_k_sw128(sb + o), ib, (acc || s > 0) ? 1u : 0u);
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const uint32_t o = (uint32_t)(s * 32);
      umma::mma_f8(d, umma::desc_k_sw128(sa + A1 + o), umma::desc_k_sw128(sb + kB1 + 64 + o), i8, 1u);
      umma::mma_f8(d, umma::desc_k_sw128(sa + A1 + 64 + o), umma::desc_k_sw128(sb + kB1 + o), i8, 1u);
    }
  } else if (MODE == B2P_MODE_TF32) {
    constexpr uint32_t idesc = umma::idesc_f32acc(2, 128, NB);
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const uint32_t ka = (uint32_t)((s >> 2) * A1 + (s & 3) * 32);
      const uint32_t kb = (uint32_t)((s >> 2) * kB1 + (s & 3) * 32);
      umma::mma_tf32(d, umma::desc_k_sw128(sa + ka), umma::desc_k_sw128(sb + kb), idesc, (acc || s > 0) ? 1u : 0u);
    }
  } else {
    constexpr uint32_t idesc = umma::idesc_f32acc(1, 128, NB);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const uint32_t o = (uint32_t)(s * 32);
      const uint64_t ah = umma::desc_k_sw128(sa + o), al = umma::desc_k_sw128(sa + A1 + o);
      const uint64_t bh = umma::desc_k_sw128(sb + o), bl = umma::desc_k_sw128(sb + kB1 + o);
      umma::mma_bf16(d, al, bh, idesc, (acc || s > 0) ? 1u : 0u);
      umma::mma_bf16(d, ah, bl, idesc, 1u);
      umma::mma_bf16(d, ah, bh, idesc, 1u);
    }
  }
}

}  // namespace b2p
