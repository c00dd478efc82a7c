// Whole-matrix kernels for small orders.
//
//   potrf_warp32_kernel  n <= 32: one warp per matrix, one row per lane in
//                        registers.  HBM-bound: A's lower triangle is read
//                        once with coalesced 128-bit loads through a padded
//                        shared staging tile, L (zeros above the diagonal) is
//                        written once with 128-bit streaming stores.
//   potrf_cta128_kernel  32 < n <= 128: one 256-thread CTA per matrix, the
//                        matrix resident in shared memory (smem_potrf).
//
// These replace the reference's exact-shape kernels chol32_register_rank2
// (submission.py:100-171), cholesky64_rank2 (submission.py:204-290) and
// cholesky128_block16 (submission.py:316-411,555-608) for every order <= 128.
#include <algorithm>

#include "launch.h"
#include "matrix_list.cuh"
#include "tile_engine.cuh"

namespace b2p {

constexpr int kWarp32Warps = 4;
constexpr int kStageLd = 36;  // staging row stride: 16-byte rows, conflict-free float4

__device__ __forceinline__ float4 ld_stream(const float4* p) {
  float4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}

__device__ __forceinline__ void st_stream(float4* p, float4 v) {
  asm volatile("st.global.cs.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z),
               "f"(v.w)
               : "memory");
}

__global__ void __launch_bounds__(kWarp32Warps * 32, 7)
    potrf_warp32_kernel(const float* __restrict__ a, float* __restrict__ l, MatrixList ml,
                        int32_t* __restrict__ info) {
  __shared__ __align__(16) float stage[kWarp32Warps][32 * kStageLd];
  __shared__ __align__(16) float colbuf[kWarp32Warps][64];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  float* t = stage[warp];
  for (int64_t item = (int64_t)blockIdx.x * kWarp32Warps + warp; item < ml.count;
       item += (int64_t)gridDim.x * kWarp32Warps) {
    int64_t mat, off;
    int n;
    ml.get(item, mat, off, n);
    const float* src = a + off;
    float* dst = l + off;
    if (n == 32) {
      const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int idx = q * 32 + lane;  // float4 index: row idx>>3, cols 4*(idx&7)..
        const int r = idx >> 3, c = (idx & 7) * 4;
        if (c <= r) *reinterpret_cast<float4*>(t + r * kStageLd + c) = ld_stream(s4 + idx);
      }
    } else {
      for (int r = 0; r < n; ++r)
        if (lane <= r) t[r * kStageLd + lane] = src[(size_t)r * n + lane];
    }
    __syncwarp();
    float x[32];
#pragma unroll
    for (int c4 = 0; c4 < 8; ++c4) {
      const float4 v = *reinterpret_cast<const float4*>(t + lane * kStageLd + 4 * c4);
      x[4 * c4 + 0] = v.x;
      x[4 * c4 + 1] = v.y;
      x[4 * c4 + 2] = v.z;
      x[4 * c4 + 3] = v.w;
    }
    if (n < 32) {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (lane >= n || j >= n) x[j] = (lane == j) ? 1.0f : 0.0f;
    }
    float ip;
    const int bad = warp_factor32(x, lane, n, colbuf[warp], ip);
    __syncwarp();
#pragma unroll
    for (int c4 = 0; c4 < 8; ++c4) {
      float4 v;
      v.x = (4 * c4 + 0 <= lane) ? x[4 * c4 + 0] : 0.0f;
      v.y = (4 * c4 + 1 <= lane) ? x[4 * c4 + 1] : 0.0f;
      v.z = (4 * c4 + 2 <= lane) ? x[4 * c4 + 2] : 0.0f;
      v.w = (4 * c4 + 3 <= lane) ? x[4 * c4 + 3] : 0.0f;
      *reinterpret_cast<float4*>(t + lane * kStageLd + 4 * c4) = v;
    }
    __syncwarp();
    if (n == 32) {
      float4* d4 = reinterpret_cast<float4*>(dst);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int idx = q * 32 + lane;
        const int r = idx >> 3, c = (idx & 7) * 4;
        st_stream(d4 + idx, *reinterpret_cast<const float4*>(t + r * kStageLd + c));
      }
    } else {
      for (int r = 0; r < n; ++r)
        if (lane < n) dst[(size_t)r * n + lane] = t[r * kStageLd + lane];
    }
    if (info != nullptr && lane == 0) info[mat] = bad < 0 ? 0 : bad + 1;
    __syncwarp();
  }
}

constexpr int kCta128Threads = 256;
constexpr int kCta128Ld = 132;

size_t cta128_smem_bytes() {
  return sizeof(float) * (size_t)(128 * kCta128Ld + tile_scratch_floats(kCta128Ld));
}

__global__ void __launch_bounds__(kCta128Threads, 2)
    potrf_cta128_kernel(const float* __restrict__ a, float* __restrict__ l, MatrixList ml,
                        int32_t* __restrict__ info) {
  extern __shared__ __align__(16) float smem[];
  float* S = smem;
  const TileScratch sc = make_scratch(S + 128 * kCta128Ld, kCta128Ld);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  constexpr int kWarps = kCta128Threads / 32;
  for (int64_t item = blockIdx.x; item < ml.count; item += gridDim.x) {
    int64_t mat, off;
    int n;
    ml.get(item, mat, off, n);
    const float* src = a + off;
    float* dst = l + off;
    for (int r = warp; r < n; r += kWarps)
      for (int c = lane; c <= r; c += 32) S[r * kCta128Ld + c] = __ldg(src + (size_t)r * n + c);
    __syncthreads();
    const int bad = smem_potrf<kCta128Threads>(S, n, kCta128Ld, sc);
    for (int r = warp; r < n; r += kWarps)
      for (int c = lane; c < n; c += 32) dst[(size_t)r * n + c] = (c <= r) ? S[r * kCta128Ld + c] : 0.0f;
    if (info != nullptr && tid == 0) info[mat] = bad < 0 ? 0 : bad + 1;
    __syncthreads();
  }
}

int launch_warp32(const float* a, float* l, const MatrixList& ml, int32_t* info, cudaStream_t s) {
  if (ml.count == 0) return B2P_OK;
  const int64_t ctas = (ml.count + kWarp32Warps - 1) / kWarp32Warps;
  const int grid = (int)std::min<int64_t>(ctas, (int64_t)device_sms() * 8 * 16);
  {
    TraceScope ts(kKWarp32, s, ml.ns ? 0.0 : 8.0 * (double)ml.count * ml.n * ml.n);
    potrf_warp32_kernel<<<grid, kWarp32Warps * 32, 0, s>>>(a, l, ml, info);
  }
  return check_launch("potrf_warp32_kernel");
}

int launch_cta128(const float* a, float* l, const MatrixList& ml, int32_t* info, cudaStream_t s) {
  if (ml.count == 0) return B2P_OK;
  const size_t smem = cta128_smem_bytes();
  if (int st = ensure_smem_attr((const void*)potrf_cta128_kernel, smem, kSlotCta128)) return st;
  const int grid = (int)std::min<int64_t>(ml.count, (int64_t)device_sms() * 2 * 64);
  {
    TraceScope ts(kKCta128, s, ml.ns ? 0.0 : (double)ml.count * ml.n * ml.n * ml.n / 3.0);
    potrf_cta128_kernel<<<grid, kCta128Threads, smem, s>>>(a, l, ml, info);
  }
  return check_launch("potrf_cta128_kernel");
}

}  // namespace b2p
