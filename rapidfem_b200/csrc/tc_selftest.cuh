// tc_selftest.cuh -- a one-CTA tcgen05 GEMM through the same operand layout,
// descriptors, TMEM allocation and TMEM loads as the tensor-core RHS kernel:
// C[M x N] = A[M x K] * B[N x K]^T, with the 3xTF32 split products
// (hi*hi + hi*lo + lo*hi) or a single tf32 product, and the A operand in shared
// memory or in TMEM (written by tcgen05.st, one row per lane).  Test hook only.
// flags: bit 0 = 3xTF32, bit 1 = A from TMEM, bit 2 = M = 64 (else 128),
// bit 3 (with bit 2) = accumulator and TMEM A operand at lane offset 16.
// The output is the raw TMEM lanes: C[lane][n] for all 128 lanes.  At M = 128
// row r is lane r; at M = 64 row 16 q + r (r < 16) is lane 32 q + o + r, o the
// lane offset (0 or 16), and the TMEM A operand is written in that layout (the
// other 16 lanes of a quarter zero).
#pragma once
#include <cstdint>

#include "tc_util.cuh"

namespace dgtd {

constexpr int kSelftestMaxK = 64;
constexpr int kSelftestMaxN = 256;

__global__ void __launch_bounds__(128) k_tc_selftest(const float* __restrict__ A, const float* __restrict__ B,
                                                     float* __restrict__ C, int N, int K, int flags,
                                                     int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tc_sm[];
  const int M = (flags & 4) ? 64 : 128;
  float* a_hi = reinterpret_cast<float*>(tc_sm);
  float* a_lo = a_hi + M * K;
  float* b_hi = a_lo + M * K;
  float* b_lo = b_hi + N * K;
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto put = [&](float* base, int R, int r, int k, float v) {
    *reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(base) + tc::kmajor_off(r, k, R)) = v;
  };
  for (int idx = tid; idx < M * K; idx += blockDim.x) {
    const int r = idx / K, k = idx - r * K;
    const float v = A[idx];
    const float h = tc::to_tf32(v);
    put(a_hi, M, r, k, h);
    put(a_lo, M, r, k, tc::to_tf32(v - h));
  }
  for (int idx = tid; idx < N * K; idx += blockDim.x) {
    const int r = idx / K, k = idx - r * K;
    const float v = B[idx];
    const float h = tc::to_tf32(v);
    put(b_hi, N, r, k, h);
    put(b_lo, N, r, k, tc::to_tf32(v - h));
  }
  const bool split3 = (flags & 1) != 0, a_tmem = (flags & 2) != 0;
  const int n32 = (N + 31) & ~31, k32 = (K + 31) & ~31;
  const int a_hi_col = n32, a_lo_col = n32 + k32;
  uint32_t ncols = 32;
  while ((int)ncols < (a_tmem ? n32 + 2 * k32 : N)) ncols <<= 1;
  if (warp == 0) tc::tmem_alloc(&s_tmem, ncols);
  if (tid == 0) {
    tc::mbar_init(&s_bar, 1);
    tc::mbar_fence_init();
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (a_tmem) {
    // row tid of A -> TMEM lane tid (warp w owns lanes 32w..32w+31)
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const int row = M == 128 ? tid : warp * 16 + (lane & 15);
    const bool real = M == 128 || (lane >> 4) == ((flags >> 3) & 1);
    for (int k0 = 0; k0 < K; k0 += 8) {
      float h[8], l[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float v = real ? A[row * K + k0 + q] : 0.f;
        h[q] = tc::to_tf32(v);
        l[q] = tc::to_tf32(v - h[q]);
      }
      tc::tmem_st8(lane_addr + (uint32_t)(a_hi_col + k0), h);
      tc::tmem_st8(lane_addr + (uint32_t)(a_lo_col + k0), l);
    }
    tc::tmem_st_wait();
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
  }
  // lane offset of the accumulator (and of a TMEM A operand): 16 only at M = 64
  const uint32_t d_tm = tmem + ((M == 64 && (flags & 8)) ? (16u << 16) : 0u);
  if (tid == 0 && a_tmem) {
    const uint32_t id = tc::idesc_tf32(M, N);
    const uint32_t bh = tc::smem_u32(b_hi), bl = tc::smem_u32(b_lo);
    for (int ks = 0; ks < K / 8; ++ks) {
      const uint32_t ah = d_tm + (uint32_t)(a_hi_col + 8 * ks), al = d_tm + (uint32_t)(a_lo_col + 8 * ks);
      tc::mma_tf32_ta(d_tm, ah, tc::tf32_step_desc(bh, N, ks), id, ks > 0 ? 1u : 0u);
      if (split3) {
        tc::mma_tf32_ta(d_tm, ah, tc::tf32_step_desc(bl, N, ks), id, 1u);
        tc::mma_tf32_ta(d_tm, al, tc::tf32_step_desc(bh, N, ks), id, 1u);
      }
    }
    tc::mma_commit(&s_bar);
  } else if (tid == 0) {
    const uint32_t id = tc::idesc_tf32(M, N);
    const uint32_t ah = tc::smem_u32(a_hi), al = tc::smem_u32(a_lo);
    const uint32_t bh = tc::smem_u32(b_hi), bl = tc::smem_u32(b_lo);
    for (int ks = 0; ks < K / 8; ++ks) {
      tc::mma_tf32(d_tm, tc::tf32_step_desc(ah, M, ks), tc::tf32_step_desc(bh, N, ks), id, ks > 0 ? 1u : 0u);
      if (split3) {
        tc::mma_tf32(d_tm, tc::tf32_step_desc(ah, M, ks), tc::tf32_step_desc(bl, N, ks), id, 1u);
        tc::mma_tf32(d_tm, tc::tf32_step_desc(al, M, ks), tc::tf32_step_desc(bh, N, ks), id, 1u);
      }
    }
    tc::mma_commit(&s_bar);
  }
  __syncwarp();
  const bool ok = tc::mbar_wait(&s_bar, 0, 1u << 19);  // about 2 s (a failed poll suspends ~4 us)
  if (!ok && lane == 0) atomicExch(err, 1);
  tc::tc_fence_after();
  if (ok) {
    const int row = warp * 32 + lane;
    for (int c0 = 0; c0 < N; c0 += 8) {
      float v[8];
      tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      tc::tmem_ld_wait();
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (c0 + q < N) C[row * N + c0 + q] = v[q];
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

}  // namespace dgtd
