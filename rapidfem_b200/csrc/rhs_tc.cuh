// rhs_tc.cuh -- fused DG Maxwell right-hand side with the element contractions
// on the tcgen05 tensor cores (3xTF32: hi*hi + hi*lo + lo*hi, FP32 accumulate
// in TMEM).  Orders 1..4.
//
// One persistent CTA (24 compute warps + 1 control warp) per SM walks tiles of E = 20
// elements.  The MMA M dimension is the 128 rows (element, component): warp
// quarter w holds elements 5w..5w+4 in rows 32w + 6*(e%5) + c (rows 30, 31 of
// each quarter are padding), so the six components of an element sit in one
// warp's TMEM lanes and the curl can be combined with warp shuffles.
//
//   volume:  C_v[(e,c)][(k,i)] = sum_j F[(e,c)][j] * D_k[i][j]        (rhs.rs:39-85)
//   LIFT:    C_l[(e,c)][i]     = sum_s Flux[(e,c)][s] * LIFT[i][s]    (rhs.rs:1433-1439)
// The LIFT K axis is laid out face by face, each face padded to a multiple of
// 8, so the LIFT MMAs of faces 0-1 run while the fluxes of faces 2-3 are formed.
//
// Per tile:
//   0. the tile's state (E*6*Np f32, contiguous) and element records arrive by
//      bulk async copies issued one tile ahead (double buffered); the residual
//      register p of the tile is bulk-copied at the start of the tile;
//   1. the state is split into tf32 hi/lo K-major operands and the volume MMAs
//      are issued asynchronously;
//   2. fluxes of faces 0-1, then 2-3 (rhs.rs:1370-1441) fill the LIFT operand,
//      each half followed by its MMAs; the last ones are committed to an mbarrier;
//   3. each TMEM lane (one row) reads its reference derivatives and LIFT sum,
//      forms its two curl contributions, exchanges them by shuffle, applies the
//      material scaling (rhs.rs:1443-1454) and stages dy in shared memory;
//   4. the mode's epilogue runs in shared memory (dy, or the LSERK4 stage update
//      of explicit.rs:122-133 in place) and the results leave by bulk async
//      stores, so the writes overlap the next tile.
// The element count is padded on the device to a multiple of E with inert
// records (PEC faces, zero metric), so every tile is full.
#pragma once
#include <cstdint>

#include "dgtd_common.cuh"
#include "tc_util.cuh"

// Phase timers: compiled in only with -DDGTD_TC_PHASE_TIMERS (an instrumented
// build); otherwise the marks are empty.
#ifdef DGTD_TC_PHASE_TIMERS
#define DGTD_TC_MARK(i)                                     \
  do {                                                      \
    if (tid == 0) {                                         \
      const long long now__ = clock64();                    \
      clk_acc[i] += (unsigned long long)(now__ - clk_last); \
      clk_last = now__;                                     \
    }                                                       \
  } while (0)
#else
#define DGTD_TC_MARK(i) \
  do {                  \
  } while (0)
#endif

namespace dgtd {

constexpr int kTcTileE = 20;
constexpr int kTcThreads = 768;      // compute threads (24 warps)
constexpr int kTcThreadsAll = 800;   // + one control warp
constexpr int kTcGroups = kTcThreads / 128;  // epilogue node groups per TMEM lane quarter
constexpr uint32_t kTcWaitLimit = 1u << 24;

__host__ __device__ constexpr int tc_r8(int x) { return (x + 7) & ~7; }
__host__ __device__ constexpr int tc_r16(int x) { return (x + 15) & ~15; }
__host__ __device__ constexpr int tc_r128(int x) { return (x + 127) & ~127; }
__host__ __device__ constexpr int tc_pow2(int x) { return x <= 32 ? 32 : x <= 64 ? 64 : x <= 128 ? 128 : x <= 256 ? 256 : 512; }

template <int N>
struct TcCfg {
  static constexpr int NP = np_of(N), NFP = nfp_of(N), NF = 4 * NFP;
  static constexpr int E = kTcTileE;
  static constexpr int M = 128;
  static constexpr int KV = tc_r8(NP);        // volume K (nodes)
  static constexpr int NV = tc_r16(3 * NP);   // volume N ((k,i) pairs)
  static constexpr int KLF = tc_r8(NFP);      // LIFT K per face
  static constexpr int KL = 4 * KLF;          // LIFT K (face nodes, per-face padded)
  static constexpr int NL = tc_r16(NP);       // LIFT N (nodes)
  static constexpr int TMEM_COLS = tc_pow2(NV + NL);
  static constexpr int TILE_F = E * 6 * NP;   // floats of state per tile
  static constexpr int TILE_B = TILE_F * 4;
  static constexpr int META_B = E * kMetaWords * 4;
  // per-thread work items
  static constexpr int ITEMS_A = (M * (KV / 4) + kTcThreads - 1) / kTcThreads;   // volume operand chunks
  static constexpr int HALF_SLOTS = E * 2 * (KLF / 4) * 4;                       // flux slots per face pair
  static constexpr int ITEMS_F = (HALF_SLOTS + kTcThreads - 1) / kTcThreads;
  // byte sizes of the operands (hi or lo)
  static constexpr int BV_B = NV * KV * 4;
  static constexpr int BL_B = NL * KL * 4;
  static constexpr int AV_B = M * KV * 4;
  static constexpr int AL_B = M * KL * 4;
  // shared-memory map (bytes)
  static constexpr int O_BVH = 0;
  static constexpr int O_BVL = O_BVH + tc_r128(BV_B);
  static constexpr int O_BLH = O_BVL + tc_r128(BV_B);
  static constexpr int O_BLL = O_BLH + tc_r128(BL_B);
  static constexpr int O_AVH = O_BLL + tc_r128(BL_B);
  static constexpr int O_AVL = O_AVH + tc_r128(AV_B);
  static constexpr int O_ALH = O_AVL + tc_r128(AV_B);
  static constexpr int O_ALL = O_ALH + tc_r128(AL_B);
  static constexpr int O_Y0 = O_ALL + tc_r128(AL_B);
  static constexpr int O_Y1 = O_Y0 + tc_r128(TILE_B);
  static constexpr int O_M0 = O_Y1 + tc_r128(TILE_B);
  static constexpr int O_M1 = O_M0 + tc_r128(META_B);
  static constexpr int O_P = O_M1 + tc_r128(META_B);  // residual register tile (LSERK)
  static constexpr int O_TAB = O_P + tc_r128(TILE_B);
  static constexpr int TAB_B = 4 * NFP + kMaxGather * NFP;
  static constexpr int SMEM = O_TAB + tc_r128(TAB_B);
  static_assert(AL_B >= TILE_B, "dy / p staging reuses the LIFT A operand (hi half)");
  static_assert((TILE_B % 16) == 0 && (META_B % 16) == 0, "bulk copies need 16-byte sizes");
  static_assert(NV <= 256 && NL <= 256 && NV + NL <= 512, "MMA N / TMEM limits");
  static_assert(ITEMS_A <= 4 && ITEMS_F <= 2, "per-thread item tables");
  static_assert((kTcThreads % 128) == 0, "compute warps cover whole TMEM lane quarters");
};

// Constant operands prepared by the host: tf32 hi/lo of D (volume B) and LIFT,
// already in the chunk-major K-major byte layout (tc_util.cuh).
struct TcTables {
  const float* b_vol;    // [hi | lo], each NV*KV
  const float* b_lift;   // [hi | lo], each NL*KL (per-face padded K)
  const uint8_t* fnodes;
  const uint8_t* gtab;
  int n_gather;
};

// Row of (element le, component c) in the 128-row MMA tile.
__device__ __forceinline__ int tc_row(int le, int c) { return (le / 5) * 32 + (le % 5) * 6 + c; }

template <int N, int MODE>
__global__ void __launch_bounds__(kTcThreadsAll, 1)
rhs_tc_kernel(RhsParams P, TcTables T, int64_t n_tiles, int* err) {
  using C = TcCfg<N>;
  constexpr int NP = C::NP, NFP = C::NFP, E = C::E, M = C::M;
  constexpr int KV = C::KV, NV = C::NV, KLF = C::KLF, NL = C::NL;
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar_ld[2];
  __shared__ __align__(8) uint64_t s_bar_mma;
  __shared__ __align__(8) uint64_t s_bar_p;
  __shared__ int s_abort;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // warps 0..23 compute; warp 24 is the control warp, its lane 0 issues the
  // MMAs and the bulk copies
  const bool ctl = warp == kTcThreads / 32;
  const bool ctl0 = ctl && lane == 0;
  float* const sY0 = reinterpret_cast<float*>(tsm + C::O_Y0);
  float* const sM0 = reinterpret_cast<float*>(tsm + C::O_M0);
  constexpr int kYStride = (C::O_Y1 - C::O_Y0) / 4, kMStride = (C::O_M1 - C::O_M0) / 4;
  float* const sP = reinterpret_cast<float*>(tsm + C::O_P);
  const bool use_p = MODE == kModeLserk && P.read_p;
  unsigned char* const avh = tsm + C::O_AVH;
  unsigned char* const avl = tsm + C::O_AVL;
  unsigned char* const alh = tsm + C::O_ALH;
  unsigned char* const all = tsm + C::O_ALL;
  float* const sStage = reinterpret_cast<float*>(alh);  // p_out (or dy) staging after the MMAs
  uint8_t* const sFn = tsm + C::O_TAB;
  uint8_t* const sG = sFn + 4 * NFP;

  // ---- set-up: TMEM, barriers, constant operands, tables
  if (warp == 0) tc::tmem_alloc(&s_tmem, C::TMEM_COLS);
  if (tid == 0) {
    tc::mbar_init(&s_bar_ld[0], 1);
    tc::mbar_init(&s_bar_ld[1], 1);
    tc::mbar_init(&s_bar_mma, 1);
    tc::mbar_init(&s_bar_p, 1);
    tc::mbar_fence_init();
    s_abort = 0;
  }
  {
    const uint4* src = reinterpret_cast<const uint4*>(T.b_vol);
    for (int i = tid; i < C::BV_B / 16; i += kTcThreadsAll) {
      reinterpret_cast<uint4*>(tsm + C::O_BVH)[i] = src[i];
      reinterpret_cast<uint4*>(tsm + C::O_BVL)[i] = src[C::BV_B / 16 + i];
    }
    src = reinterpret_cast<const uint4*>(T.b_lift);
    for (int i = tid; i < C::BL_B / 16; i += kTcThreadsAll) {
      reinterpret_cast<uint4*>(tsm + C::O_BLH)[i] = src[i];
      reinterpret_cast<uint4*>(tsm + C::O_BLL)[i] = src[C::BL_B / 16 + i];
    }
    // LIFT operand padding (rows 30/31 of each quarter, face-padding columns)
    // must hold finite values: start from zero.  The staging that later
    // shares the hi half writes only finite numbers.
    for (int i = tid; i < C::AL_B / 16; i += kTcThreadsAll) {
      reinterpret_cast<uint4*>(alh)[i] = make_uint4(0, 0, 0, 0);
      reinterpret_cast<uint4*>(all)[i] = make_uint4(0, 0, 0, 0);
    }
    for (int i = tid; i < 4 * NFP; i += kTcThreadsAll) sFn[i] = T.fnodes[i];
    for (int i = tid; i < T.n_gather * NFP; i += kTcThreadsAll) sG[i] = T.gtab[i];
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t idv = tc::idesc_tf32(M, NV), idl = tc::idesc_tf32(M, NL);

  // ---- tile-invariant per-thread tables (compute threads)
  // volume operand chunks: source offset in the state tile (-1: padding row,
  // -2: no item), destination byte offset, K chunk
  int a_src[C::ITEMS_A], a_dst[C::ITEMS_A], a_kc[C::ITEMS_A];
#pragma unroll
  for (int u = 0; u < C::ITEMS_A; ++u) {
    const int idx = tid + u * kTcThreads;
    a_src[u] = -2;
    a_dst[u] = 0;
    a_kc[u] = 0;
    if (!ctl && idx < M * (KV / 4)) {
      const int r = idx & (M - 1), kc = idx >> 7;
      const int q = r >> 5, rr = r & 31;
      a_src[u] = rr < 30 ? ((q * 5 + rr / 6) * 6 + rr % 6) * NP + kc * 4 : -1;
      a_dst[u] = (int)tc::kmajor_off(r, kc * 4, M);
      a_kc[u] = kc;
    }
  }
  // flux slots of a face pair: (le, face within the pair, node m); le = -1 idle
  int f_le[C::ITEMS_F], f_fl[C::ITEMS_F], f_m[C::ITEMS_F];
#pragma unroll
  for (int u = 0; u < C::ITEMS_F; ++u) {
    const int q = tid + u * kTcThreads;
    f_le[u] = -1;
    f_fl[u] = 0;
    f_m[u] = 0;
    if (!ctl && q < C::HALF_SLOTS) {
      const int s4 = q & 3, le = (q >> 2) % E, rest = (q >> 2) / E;  // rest = fl * (KLF/4) + mg
      const int fl = rest / (KLF / 4), mg = rest % (KLF / 4);
      const int m = mg * 4 + s4;
      if (m < NFP) {
        f_le[u] = le;
        f_fl[u] = fl;
        f_m[u] = m;
      }
    }
  }
  // epilogue lane: row (le, c) of warp quarter qtr; rows 30, 31 are padding.
  // Node group grp covers nodes [grp*NPG, grp*NPG + NPG).
  constexpr int NPG = (NP + kTcGroups - 1) / kTcGroups;
  const int qtr = warp & 3, grp = (warp >> 2) % kTcGroups;
  const bool lane_real = lane < 30;
  const int e_le = qtr * 5 + (lane_real ? lane / 6 : 4);
  const int e_c = lane_real ? lane % 6 : 5;
  const int e_fld = e_c / 3, e_t = e_c % 3;
  const int e_srcA = lane_real ? (lane / 6) * 6 + 3 * (1 - e_fld) + (e_t + 2) % 3 : lane;
  const int e_srcB = lane_real ? (lane / 6) * 6 + 3 * (1 - e_fld) + (e_t + 1) % 3 : lane;
  const float e_sign = e_fld == 0 ? 1.f : -1.f;
  const int e_cA = (e_t + 2) % 3, e_cB = (e_t + 1) % 3;
  const int e_row_off = (e_le * 6 + e_c) * NP;
  const uint32_t e_taddr = tmem + ((uint32_t)(qtr * 32) << 16);

  uint32_t ld_phase = 0u, pending = 0u, mma_phase = 0u, p_phase = 0u;
  bool p_pending = false, mma_out = false;
#ifdef DGTD_TC_PHASE_TIMERS
  unsigned long long clk_acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  long long clk_last = clock64();
#endif

  int64_t tile = blockIdx.x;
  if (ctl0 && tile < n_tiles) {
    tc::mbar_expect_tx(&s_bar_ld[0], C::TILE_B + C::META_B);
    tc::bulk_g2s(sY0, P.y_in + tile * C::TILE_F, C::TILE_B, &s_bar_ld[0]);
    tc::bulk_g2s(sM0, P.meta + tile * E * kMetaWords, C::META_B, &s_bar_ld[0]);
  }
  if (tile < n_tiles) pending = 1u;

  for (int it = 0; tile < n_tiles; tile += gridDim.x, ++it) {
    const int buf = it & 1;
    const int64_t next = tile + gridDim.x;
    float* const sY = sY0 + buf * kYStride;
    const float* const sM = sM0 + buf * kMStride;
    const int64_t e0 = tile * E;
    p_pending = use_p;
    if (ctl) {
      if (ctl0) {
        if (use_p) {
          tc::fence_proxy_async_smem();
          tc::mbar_expect_tx(&s_bar_p, C::TILE_B);
          tc::bulk_g2s(sP, P.p + tile * C::TILE_F, C::TILE_B, &s_bar_p);
        }
        // the previous tile's bulk stores must have finished reading the
        // staging and state buffers before they are written again
        tc::bulk_wait_read0();
      }
      __syncwarp();
    } else {
      DGTD_TC_MARK(0);
      if (!tc::mbar_wait(&s_bar_ld[buf], (ld_phase >> buf) & 1u, kTcWaitLimit)) s_abort = 1;
      DGTD_TC_MARK(1);
      // ---- 1. volume operand: tf32 hi/lo of the state, rows (e,c), K = nodes
#pragma unroll
      for (int u = 0; u < C::ITEMS_A; ++u) {
        if (a_src[u] == -2) continue;
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        if (a_src[u] >= 0) {
#pragma unroll
          for (int w = 0; w < 4; ++w)
            if (a_kc[u] * 4 + w < NP) v[w] = sY[a_src[u] + w];
        }
        float4 h, l;
        h.x = tc::to_tf32(v[0]); l.x = tc::to_tf32(v[0] - h.x);
        h.y = tc::to_tf32(v[1]); l.y = tc::to_tf32(v[1] - h.y);
        h.z = tc::to_tf32(v[2]); l.z = tc::to_tf32(v[2] - h.z);
        h.w = tc::to_tf32(v[3]); l.w = tc::to_tf32(v[3] - h.w);
        *reinterpret_cast<float4*>(avh + a_dst[u]) = h;
        *reinterpret_cast<float4*>(avl + a_dst[u]) = l;
      }
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    DGTD_TC_MARK(2);
    if (s_abort) break;
    ld_phase ^= 1u << buf;
    pending &= ~(1u << buf);
    if (next < n_tiles) pending |= 1u << (buf ^ 1);  // issued by the control warp below

    // ---- 2. numerical flux into the LIFT operand, faces 0-1 then 2-3
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      if (ctl) {
        if (ctl0) {
          tc::tc_fence_after();
          if (half == 0) {
            const uint32_t ah = tc::smem_u32(avh), al = tc::smem_u32(avl);
            const uint32_t bh = tc::smem_u32(tsm + C::O_BVH), bl = tc::smem_u32(tsm + C::O_BVL);
#pragma unroll 1
            for (int ks = 0; ks < KV / 8; ++ks) {
              tc::mma_tf32(tmem, tc::tf32_step_desc(ah, M, ks), tc::tf32_step_desc(bh, NV, ks), idv,
                           ks > 0 ? 1u : 0u);
              tc::mma_tf32(tmem, tc::tf32_step_desc(ah, M, ks), tc::tf32_step_desc(bl, NV, ks), idv, 1u);
              tc::mma_tf32(tmem, tc::tf32_step_desc(al, M, ks), tc::tf32_step_desc(bh, NV, ks), idv, 1u);
            }
            // prefetch the next tile into the other buffer (its last reader,
            // the previous tile's state store, has finished)
            if (next < n_tiles) {
              uint64_t* bar = &s_bar_ld[buf ^ 1];
              tc::mbar_expect_tx(bar, C::TILE_B + C::META_B);
              tc::bulk_g2s(sY0 + (buf ^ 1) * kYStride, P.y_in + next * C::TILE_F, C::TILE_B, bar);
              tc::bulk_g2s(sM0 + (buf ^ 1) * kMStride, P.meta + next * E * kMetaWords, C::META_B, bar);
            }
          } else {
            const uint32_t ah = tc::smem_u32(alh), al = tc::smem_u32(all);
            const uint32_t bh = tc::smem_u32(tsm + C::O_BLH), bl = tc::smem_u32(tsm + C::O_BLL);
            const uint32_t tl = tmem + (uint32_t)NV;
            constexpr int KS_HALF = 2 * KLF / 8;
#pragma unroll 1
            for (int ks = 0; ks < KS_HALF; ++ks) {
              tc::mma_tf32(tl, tc::tf32_step_desc(ah, M, ks), tc::tf32_step_desc(bh, NL, ks), idl,
                           ks > 0 ? 1u : 0u);
              tc::mma_tf32(tl, tc::tf32_step_desc(ah, M, ks), tc::tf32_step_desc(bl, NL, ks), idl, 1u);
              tc::mma_tf32(tl, tc::tf32_step_desc(al, M, ks), tc::tf32_step_desc(bh, NL, ks), idl, 1u);
            }
          }
        }
        __syncwarp();
      } else {
        // out-of-tile neighbour traces first: independent L2 requests in flight together
        float nb[C::ITEMS_F][6];
#pragma unroll
        for (int u = 0; u < C::ITEMS_F; ++u) {
#pragma unroll
          for (int c = 0; c < 6; ++c) nb[u][c] = 0.f;
          if (f_le[u] < 0) continue;
          const int f = 2 * half + f_fl[u];
          const float* Me = sM + f_le[u] * kMetaWords;
          const uint32_t codes = __float_as_uint(Me[41 + (f >> 1)]);
          const uint32_t code = (f & 1) ? (codes >> 16) : (codes & 0xffffu);
          const int64_t lo = (int64_t)__float_as_int(Me[37 + f]) - e0;
          if (((code >> 8) & 3) == kInterior && !(lo >= 0 && lo < E)) {
            const float* Z = P.y_in + (e0 + lo) * 6 * NP + sG[(code & 0xff) * NFP + f_m[u]];
#pragma unroll
            for (int c = 0; c < 6; ++c) nb[u][c] = __ldg(Z + c * NP);
          }
        }
#pragma unroll
        for (int u = 0; u < C::ITEMS_F; ++u) {
          if (f_le[u] < 0) continue;
          const int le = f_le[u], f = 2 * half + f_fl[u], m = f_m[u];
          const float* Me = sM + le * kMetaWords;
          const float nx = Me[9 + 3 * f], ny = Me[10 + 3 * f], nz = Me[11 + 3 * f];
          const float coef = 0.5f * Me[21 + f];
          const uint32_t codes = __float_as_uint(Me[41 + (f >> 1)]);
          const uint32_t code = (f & 1) ? (codes >> 16) : (codes & 0xffffu);
          const int kind = (code >> 8) & 3;
          const float* Y = sY + le * 6 * NP + sFn[f * NFP + m];
          const float ex = Y[0 * NP], ey = Y[1 * NP], ez = Y[2 * NP];
          const float hx = Y[3 * NP], hy = Y[4 * NP], hz = Y[5 * NP];
          float jex, jey, jez, jhx, jhy, jhz;
          float a = P.alpha;
          if (kind == kPort) {
            // characteristic boundary against a zero incident field (rhs.rs:1380-1386)
            jex = ex; jey = ey; jez = ez; jhx = hx; jhy = hy; jhz = hz;
            a = 1.0f;
          } else if (kind == kPec) {
            // PEC ghost: [E] = 2 E_tan, [H] = 2 H_n (rhs.rs:1387-1402)
            const float edn = nx * ex + ny * ey + nz * ez;
            const float hdn = nx * hx + ny * hy + nz * hz;
            jex = 2.0f * (ex - edn * nx); jey = 2.0f * (ey - edn * ny); jez = 2.0f * (ez - edn * nz);
            jhx = 2.0f * (hdn * nx); jhy = 2.0f * (hdn * ny); jhz = 2.0f * (hdn * nz);
          } else {
            float px = nb[u][0], py = nb[u][1], pz = nb[u][2];
            float qx = nb[u][3], qy = nb[u][4], qz = nb[u][5];
            const int64_t lo = (int64_t)__float_as_int(Me[37 + f]) - e0;
            if (lo >= 0 && lo < E) {
              const float* Z = sY + lo * 6 * NP + sG[(code & 0xff) * NFP + m];
              px = Z[0 * NP]; py = Z[1 * NP]; pz = Z[2 * NP];
              qx = Z[3 * NP]; qy = Z[4 * NP]; qz = Z[5 * NP];
            }
            jex = ex - px; jey = ey - py; jez = ez - pz;
            jhx = hx - qx; jhy = hy - qy; jhz = hz - qz;
          }
          // fe = coef (-n x [H] + a n x (n x [E])), fh = coef (n x [E] + a n x (n x [H]))
          // (rhs.rs:1420-1432), with n x (n x v) = n (n.v) - v for the unit normal.
          const float ca = coef * a;
          const float de = ca * (nx * jex + ny * jey + nz * jez);
          const float dh = ca * (nx * jhx + ny * jhy + nz * jhz);
          float fl[6];
          fl[0] = fmaf(de, nx, fmaf(-ca, jex, -coef * (ny * jhz - nz * jhy)));
          fl[1] = fmaf(de, ny, fmaf(-ca, jey, -coef * (nz * jhx - nx * jhz)));
          fl[2] = fmaf(de, nz, fmaf(-ca, jez, -coef * (nx * jhy - ny * jhx)));
          fl[3] = fmaf(dh, nx, fmaf(-ca, jhx, coef * (ny * jez - nz * jey)));
          fl[4] = fmaf(dh, ny, fmaf(-ca, jhy, coef * (nz * jex - nx * jez)));
          fl[5] = fmaf(dh, nz, fmaf(-ca, jhz, coef * (nx * jey - ny * jex)));
          const int s = f * KLF + m;
          const uint32_t off = (uint32_t)((s >> 2) * (M / 8) * 128 + (s & 3) * 4 + tc_row(le, 0) * 16);
#pragma unroll
          for (int c = 0; c < 6; ++c) {
            const float h = tc::to_tf32(fl[c]);
            *reinterpret_cast<float*>(alh + off + c * 16) = h;
            *reinterpret_cast<float*>(all + off + c * 16) = tc::to_tf32(fl[c] - h);
          }
        }
      }
      tc::fence_proxy_async_smem();
      __syncthreads();
      DGTD_TC_MARK(3);
    }
    if (ctl0) {
      tc::tc_fence_after();
      const uint32_t ah = tc::smem_u32(alh), al = tc::smem_u32(all);
      const uint32_t bh = tc::smem_u32(tsm + C::O_BLH), bl = tc::smem_u32(tsm + C::O_BLL);
      const uint32_t tl = tmem + (uint32_t)NV;
      constexpr int KS_HALF = 2 * KLF / 8;
#pragma unroll 1
      for (int ks = KS_HALF; ks < 2 * KS_HALF; ++ks) {
        tc::mma_tf32(tl, tc::tf32_step_desc(ah, M, ks), tc::tf32_step_desc(bh, NL, ks), idl, 1u);
        tc::mma_tf32(tl, tc::tf32_step_desc(ah, M, ks), tc::tf32_step_desc(bl, NL, ks), idl, 1u);
        tc::mma_tf32(tl, tc::tf32_step_desc(al, M, ks), tc::tf32_step_desc(bh, NL, ks), idl, 1u);
      }
      tc::mma_commit(&s_bar_mma);
    }
    __syncwarp();
    mma_out = true;

    // ---- 3. epilogue from TMEM: curl by shuffles, LIFT, materials -> dy staging
    if (!ctl) {
      if (!tc::mbar_wait(&s_bar_mma, mma_phase, kTcWaitLimit)) s_abort = 1;
      tc::tc_fence_after();
      DGTD_TC_MARK(4);
      const float* Me = sM + e_le * kMetaWords;
      const float gA0 = Me[0 * 3 + e_cA], gA1 = Me[1 * 3 + e_cA], gA2 = Me[2 * 3 + e_cA];
      const float gB0 = Me[0 * 3 + e_cB], gB1 = Me[1 * 3 + e_cB], gB2 = Me[2 * 3 + e_cB];
      const float inv_w = Me[25 + 3 * e_fld + e_t];
      const float sig_w = Me[31 + 3 * e_fld + e_t];
      const float* yrow = sY + e_row_off;
      float* drow = sStage + e_row_off;
      constexpr int NCH = (NP + 7) / 8;
      for (int ch = grp; ch < NCH; ch += kTcGroups) {
        const int i0 = ch * 8;
        float r0[8], r1[8], r2[8], lf[8];
        tc::tmem_ld8(e_taddr + (uint32_t)i0, r0);
        tc::tmem_ld8(e_taddr + (uint32_t)(NP + i0), r1);
        tc::tmem_ld8(e_taddr + (uint32_t)(2 * NP + i0), r2);
        tc::tmem_ld8(e_taddr + (uint32_t)(NV + i0), lf);
        tc::tmem_ld_wait();
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          // my contributions: A to curl component (t+1)%3, B to (t+2)%3
          const float A = gA0 * r0[u] + gA1 * r1[u] + gA2 * r2[u];
          const float B = -(gB0 * r0[u] + gB1 * r1[u] + gB2 * r2[u]);
          const float pa = __shfl_sync(0xffffffffu, A, e_srcA);
          const float pb = __shfl_sync(0xffffffffu, B, e_srcB);
          const int i = i0 + u;
          if (lane_real && i < NP) drow[i] = inv_w * (e_sign * (pa + pb) + lf[u]) - sig_w * yrow[i];
        }
      }
      tc::tc_fence_before();
      if (p_pending && !tc::mbar_wait(&s_bar_p, p_phase, kTcWaitLimit)) s_abort = 1;
    }
    __syncthreads();
    DGTD_TC_MARK(5);
    if (s_abort) break;

    // ---- 4. epilogue in shared memory: the mode's update in place
    if (!ctl && MODE == kModeLserk) {
      float4* const d4 = reinterpret_cast<float4*>(sStage);
      float4* const y4 = reinterpret_cast<float4*>(sY);
      const float4* const p4 = reinterpret_cast<const float4*>(sP);
      const int64_t gb = tile * C::TILE_F;
      for (int idx = tid; idx < C::TILE_F / 4; idx += kTcThreads) {
        const float4 dy = d4[idx];
        const int64_t g = gb + 4 * (int64_t)idx;
        float k0 = dy.x, k1 = dy.y, k2 = dy.z, k3 = dy.w;
        if (P.src_vec != nullptr) {
          const float4 sv = __ldg(reinterpret_cast<const float4*>(P.src_vec + g));
          k0 = fmaf(P.src_g, sv.x, k0); k1 = fmaf(P.src_g, sv.y, k1);
          k2 = fmaf(P.src_g, sv.z, k2); k3 = fmaf(P.src_g, sv.w, k3);
        }
        const int64_t ds = P.src_idx - g;
        if (ds == 0) k0 += P.src_g;
        if (ds == 1) k1 += P.src_g;
        if (ds == 2) k2 += P.src_g;
        if (ds == 3) k3 += P.src_g;
        float4 pv = make_float4(P.dt * k0, P.dt * k1, P.dt * k2, P.dt * k3);
        if (P.read_p) {
          const float4 po = p4[idx];
          pv.x = fmaf(P.a, po.x, pv.x); pv.y = fmaf(P.a, po.y, pv.y);
          pv.z = fmaf(P.a, po.z, pv.z); pv.w = fmaf(P.a, po.w, pv.w);
        }
        d4[idx] = pv;  // p_out staged in place of dy
        const float4 yo = y4[idx];
        y4[idx] = make_float4(fmaf(P.b, pv.x, yo.x), fmaf(P.b, pv.y, yo.y), fmaf(P.b, pv.z, yo.z),
                              fmaf(P.b, pv.w, yo.w));
      }
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    mma_phase ^= 1u;
    mma_out = false;
    if (p_pending) p_phase ^= 1u;
    p_pending = false;
    if (ctl0) {
      const int64_t gb = tile * C::TILE_F;
      if (MODE == kModeApply) {
        tc::bulk_s2g(P.out + gb, sStage, C::TILE_B);
      } else {
        tc::bulk_s2g(P.out + gb, sY, C::TILE_B);
        if (P.write_p) tc::bulk_s2g(P.p + gb, sStage, C::TILE_B);
      }
      tc::bulk_commit();
    }
    DGTD_TC_MARK(6);
  }

  // ---- drain: stores complete; on an abort wait (bounded) for loads in flight
  if (ctl0) tc::bulk_wait0();
  if (s_abort) {
    if (tid == 0) atomicExch(err, 1);
    if (ctl0) {
      for (int b = 0; b < 2; ++b)
        if ((pending >> b) & 1u) (void)tc::mbar_wait(&s_bar_ld[b], (ld_phase >> b) & 1u, kTcWaitLimit);
      if (p_pending) (void)tc::mbar_wait(&s_bar_p, p_phase, kTcWaitLimit);
      if (mma_out) (void)tc::mbar_wait(&s_bar_mma, mma_phase, kTcWaitLimit);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
#ifdef DGTD_TC_PHASE_TIMERS
  if (tid == 0 && P.phase_clk != nullptr)
    for (int i = 0; i < 7; ++i) atomicAdd(P.phase_clk + i, clk_acc[i]);
#endif
  if (warp == 0) tc::tmem_dealloc(tmem, C::TMEM_COLS);
}

}  // namespace dgtd
