// rhs_tc.cuh -- fused DG Maxwell right-hand side with the element contractions
// on the tcgen05 tensor cores (3xTF32: hi*hi + hi*lo + lo*hi, FP32 accumulate
// in TMEM).  Orders 1..5.
//
// One persistent CTA per SM walks tiles of E elements.  The MMA M dimension is
// the rows (element, component), split into four lane quarters of QR = M/4
// rows; quarter q holds elements EQ q .. EQ q + EQ - 1 in rows
// QR q + 6 (e % EQ) + c, so the six components of an element sit in one warp's
// TMEM lanes and the curl can be combined with warp shuffles.
//   orders 1-4: M = 128, EQ = 5 (E = 20; rows 30, 31 of a quarter are padding),
//               two TMEM accumulator sets side by side in the columns;
//   order 5:    M = 64, EQ = 2 (E = 8; rows 12..15 of a quarter are padding).
//               A 64-row MMA keeps row 16 q + r of its accumulator (and of a
//               TMEM A operand, which must sit at the accumulator's lane offset)
//               in lane 32 q + o + r, o = 0 or 16, so a quarter's rows stay in
//               its own TMEM sub-partition and the two accumulator sets (each
//               with its own volume A operand) take the two lane halves of the
//               same columns; TMEM is read and written with the 16-lane shapes,
//               a warp's two thread halves on two column ranges.  Order 5 at 128
//               rows would need 608 TMEM columns for two accumulator sets and
//               about 370 KB of shared memory for its operands and state slots.
//
//   volume:  C_v[(e,c)][(k,i)] = sum_j F[(e,c)][j] * D_k[i][j]        (rhs.rs:39-85)
//   LIFT:    C_l[(e,c)][i]     = sum_s Flux[(e,c)][s] * LIFT[i][s]    (rhs.rs:1433-1439)
//
// The CTA is warp-specialised so that two tiles are in flight:
//   flux warps      build tile t's volume operand (tf32 hi/lo of the state,
//                   written to TMEM by tcgen05.st) and its numerical fluxes
//                   (rhs.rs:1370-1441) into the LIFT operand in shared memory;
//   epilogue warps  finish tile t-1 from its TMEM accumulators: reference
//                   derivatives -> curl by shuffles, LIFT sum, material scaling
//                   (rhs.rs:1443-1454) and the mode's update in place (dy, or the
//                   LSERK4 stage of explicit.rs:122-133 on y and p);
//   control lane    issues the bulk async loads (state + element records three
//                   tiles deep, residual register two deep), the MMAs of both
//                   contractions into one of two TMEM accumulator sets, and the
//                   bulk async stores.
// The LIFT operand is formed and multiplied in two halves (faces 0-1, 2-3),
// each released by its own MMA completion, so the LIFT MMAs of one half run
// while the flux warps form the other half (or the next tile's volume operand).
// All hand-offs are mbarriers; every wait is bounded and an expired wait stops
// the CTA cleanly with an error flag.  The element count is padded on the
// device to a multiple of E with inert records (PEC faces, zero metric), so
// every tile is full.
#pragma once
#include <cstdint>

#include "dgtd_common.cuh"
#include "tc_util.cuh"

// Phase timers: compiled in only with -DDGTD_TC_PHASE_TIMERS (an instrumented
// build); otherwise the marks are empty.  One thread per role records.
#ifdef DGTD_TC_PHASE_TIMERS
#define DGTD_TC_MARK(i)                                     \
  do {                                                      \
    if (timer_thread) {                                     \
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

constexpr int kTcTileE = 20;  // elements per tile at orders 1-4 (8 at order 5)
constexpr int kTcFluxWarps = 12;                          // warps 0..11
constexpr int kTcEpiWarps = 12;                           // warps 12..23
constexpr int kTcCtlWarp = kTcFluxWarps + kTcEpiWarps;    // warp 24, lane 0
constexpr int kTcThreadsAll = (kTcCtlWarp + 1) * 32;
constexpr int kTcFluxThreads = kTcFluxWarps * 32;
constexpr int kTcVolGroups = kTcFluxWarps / 4;            // column groups per lane quarter
constexpr int kTcEpiGroups = kTcEpiWarps / 4;
constexpr uint32_t kTcWaitLimit = 1u << 19;  // polls per bounded wait (about 2 s)
static_assert(kTcFluxWarps % 4 == 0 && kTcEpiWarps % 4 == 0, "roles cover whole TMEM lane quarters");

__host__ __device__ constexpr int tc_r8(int x) { return (x + 7) & ~7; }
__host__ __device__ constexpr int tc_r16(int x) { return (x + 15) & ~15; }
__host__ __device__ constexpr int tc_r128(int x) { return (x + 127) & ~127; }

// Tile shape of an order: MMA rows and elements per lane quarter (the file
// header says why order 5 differs).
__host__ __device__ constexpr int tc_m(int n) { return n == 5 ? 64 : 128; }
__host__ __device__ constexpr int tc_eq(int n) { return n == 5 ? 2 : 5; }
__host__ __device__ constexpr int tc_tile_e(int n) { return 4 * tc_eq(n); }
// MMA N of the volume and LIFT B operands (a 128-row MMA takes N in steps of 16,
// a 64-row one in steps of 8); the host lays out the constant operands with these.
__host__ __device__ constexpr int tc_nv(int n) { return tc_m(n) == 64 ? tc_r8(3 * np_of(n)) : tc_r16(3 * np_of(n)); }
__host__ __device__ constexpr int tc_nl(int n) { return tc_m(n) == 64 ? tc_r8(np_of(n)) : tc_r16(np_of(n)); }

template <int N>
struct TcCfg {
  static constexpr int NP = np_of(N), NFP = nfp_of(N), NF = 4 * NFP;
  static constexpr int M = tc_m(N);
  static constexpr int EQ = tc_eq(N);         // elements per lane quarter
  static constexpr int E = 4 * EQ;            // elements per tile
  static constexpr int QR = M / 4;            // MMA rows per lane quarter
  static constexpr int RL = 6 * EQ;           // real rows (lanes) per quarter
  // the two accumulator sets: side by side in the columns (M = 128), or in the
  // lane halves of the same columns (M = 64), each with its own A operand
  static constexpr bool LANE_SETS = M == 64;
  static constexpr int KV = tc_r8(NP);        // volume K (nodes)
  static constexpr int NV = tc_nv(N);         // volume N ((k,i) pairs)
  static constexpr int KLF = tc_r8(NFP);      // LIFT K per face
  static constexpr int KL = 4 * KLF;          // LIFT K (face nodes, per-face padded)
  static constexpr int NL = tc_nl(N);         // LIFT N (nodes)
  // The LIFT B operand stacks LIFT hi (rows 0..NL-1) over LIFT lo (rows NL..2NL-1),
  // so one MMA forms both products of an A half: N = 2 NL.
  static constexpr int NL2 = 2 * NL;
  // TMEM columns: the accumulator sets [vol | lift hi | lift lo], then the
  // volume A operand (hi, lo)
  static constexpr int ACC = NV + NL2;
  static constexpr int T_AHI = LANE_SETS ? ACC : 2 * ACC;
  static constexpr int T_ALO = T_AHI + KV;
  static constexpr int TMEM_COLS = 512;
  static constexpr int TILE_F = E * 6 * NP;   // floats of state per tile
  static constexpr int TILE_B = TILE_F * 4;
  static constexpr int META_B = E * kMetaWords * 4;
  // per-thread work
  static constexpr int SLOTS = E * KL;                                         // flux slots, all faces
  static constexpr int HSLOTS = SLOTS / 2;                                     // faces 0-1 | faces 2-3
  static constexpr int ITEMS_H = (HSLOTS + kTcFluxThreads - 1) / kTcFluxThreads;
  static constexpr int KS_H = KL / 16;                                         // LIFT k-steps per half
  static constexpr int VCH = KV / 8;                                           // volume-operand column chunks
  static constexpr int VCH_PER = (VCH + kTcVolGroups - 1) / kTcVolGroups;
  static constexpr int ECH = (NP + 3) / 4;                                     // epilogue node chunks of 4
  static constexpr int ECH_PER = (ECH + kTcEpiGroups - 1) / kTcEpiGroups;
  // M = 64: a 16-lane TMEM access serves two chunks of 4 columns (one per
  // thread half): the volume operand's K in VCH units of 8, the accumulator's
  // nodes in EPAIRS units of 8
  static constexpr int EPAIRS = (ECH + 1) / 2, EPAIR_PER = (EPAIRS + kTcEpiGroups - 1) / kTcEpiGroups;
  // byte sizes of the shared-memory operands (hi or lo)
  static constexpr int BV_B = NV * KV * 4;
  static constexpr int BL_B = NL2 * KL * 4;   // stacked hi/lo
  static constexpr int AL_B = M * KL * 4;
  static constexpr int YS_B = tc_r128(TILE_B);
  static constexpr int MS_B = tc_r128(META_B);
  // shared-memory map (bytes)
  static constexpr int O_BVH = 0;
  static constexpr int O_BVL = O_BVH + tc_r128(BV_B);
  static constexpr int O_BL = O_BVL + tc_r128(BV_B);
  static constexpr int O_ALH = O_BL + tc_r128(BL_B);
  static constexpr int O_ALL = O_ALH + tc_r128(AL_B);
  static constexpr int O_Y = O_ALL + tc_r128(AL_B);  // 3 state slots
  static constexpr int O_M = O_Y + 3 * YS_B;           // 3 element-record slots
  static constexpr int O_P = O_M + 3 * MS_B;           // 2 residual / output slots
  static constexpr int O_TAB = O_P + 2 * YS_B;
  static constexpr int TAB_B = 4 * NFP + kMaxGather * NFP;
  static constexpr int SMEM = O_TAB + tc_r128(TAB_B);
  static_assert(SMEM <= 232448 - 1024, "shared memory per CTA (dynamic + static)");
  static_assert(T_ALO + KV <= TMEM_COLS, "TMEM columns");
  static_assert((TILE_B % 16) == 0 && (META_B % 16) == 0, "bulk copies need 16-byte sizes");
  static_assert(NV <= 256 && NL2 <= 256 && (NV % (M == 128 ? 16 : 8)) == 0 && (NL2 % (M == 128 ? 16 : 8)) == 0,
                "MMA N limits");
  // at M = 64 quarter q's rows start at offset q (see tc_row)
  static_assert((M == 128 || M == 64) && RL <= QR && (!LANE_SETS || (3 + RL <= 16 && ECH % 2 == 0)), "tile shape");
  static_assert(NP <= NL && 3 * NP <= NV, "accumulator columns");
  // flux slot packing: element (5 bits), face (2), face node (MB), state offset
  static constexpr int MB = NFP <= 16 ? 4 : 5;
  static constexpr int OFF_SHIFT = 7 + MB;
  static_assert(E <= 32 && NFP <= (1 << MB) && TILE_F < (1 << (31 - OFF_SHIFT)), "flux slot packing");
  static_assert(ITEMS_H <= 2 && VCH_PER <= 4 && ECH_PER <= 8, "per-thread work tables");
  static_assert((KL % 16) == 0, "LIFT halves are whole k-steps");
};

// Constant operands prepared by the host: tf32 hi/lo of D (volume B) and LIFT,
// already in the chunk-major K-major byte layout (tc_util.cuh).
struct TcTables {
  const float* b_vol;    // [hi | lo], each NV*KV
  const float* b_lift;   // stacked [hi ; lo] rows, 2NL x KL (per-face padded K)
  const uint8_t* fnodes;
  const uint8_t* gtab;
  int n_gather;
};

// TMEM address offset of accumulator set s (and, at M = 64, of its A operand).
template <class C>
__device__ __forceinline__ uint32_t tc_set_off(int s) {
  return C::LANE_SETS ? ((uint32_t)(16 * s) << 16) : (uint32_t)(s * C::ACC);
}

// Row offset of lane quarter q's elements.  At M = 64 the flux warps store the
// LIFT operand of eight elements at once; starting quarter q's rows at q spreads
// their rows over more 16-byte bank groups (row mod 8) than a common start.
template <class C>
__device__ __forceinline__ int tc_qoff(int q) {
  return C::LANE_SETS ? q : 0;
}

// MMA row of (element le, component c) of a tile.
template <class C>
__device__ __forceinline__ int tc_row(int le, int c) {
  return (le / C::EQ) * C::QR + tc_qoff<C>(le / C::EQ) + (le % C::EQ) * 6 + c;
}

// Rotation of a row's node order at M = 64.  The element rows of a state tile
// are Np = 56 floats apart, so the twelve (element j, component c) rows a warp
// touches fall into four bank groups of three ((16 j + 24 c) mod 32); the
// three rows of a group start their four nodes at 0, 1 and 2.
__device__ __forceinline__ int tc_node_rot(int j, int c) { return j == 0 ? (c >= 4 ? 1 : 0) : (c >= 2 ? 2 : 1); }

// a[(v + k) & 3] for a compile-time v and a runtime k in 0..3, without
// indexing the register array at run time.
__device__ __forceinline__ float tc_pick4(const float (&a)[4], int v, int k) {
  const float x0 = a[v & 3], x1 = a[(v + 1) & 3], x2 = a[(v + 2) & 3], x3 = a[(v + 3) & 3];
  return k == 0 ? x0 : k == 1 ? x1 : k == 2 ? x2 : x3;
}

// Bounded waits.  A wait gives up after `limit` polls or once another role has
// raised the abort flag; the warp form is warp-uniform.  A poll that finds the
// phase incomplete suspends the thread until the phase completes or a hardware
// time limit passes, measured at 3.98 us on B200, so kTcWaitLimit = 2^19 polls
// bounds a wait at about 2.1 s of wall time.  (A wall-clock check inside the
// loop was tried: any extra state in these inlined loops slows the stage
// kernel by 7 %.)
#ifdef DGTD_TC_PHASE_TIMERS
__device__ unsigned long long g_tc_polls[3];
#endif
__device__ __forceinline__ bool tc_wait1(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                         uint32_t limit = kTcWaitLimit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (tc::mbar_try_wait(bar, parity)) {
#ifdef DGTD_TC_PHASE_TIMERS
      const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
      if (l == 0 && (w == 0 || w == kTcFluxWarps || w == kTcCtlWarp))
        atomicAdd(&g_tc_polls[w == 0 ? 0 : w == kTcFluxWarps ? 1 : 2], (unsigned long long)(i + 1));
#endif
      return true;
    }
    if ((i & 255u) == 255u && *abort_flag) return false;
  }
  return false;
}
__device__ __forceinline__ bool tc_waitw(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  const bool ok = tc_wait1(bar, parity, abort_flag);
  return __all_sync(0xffffffffu, ok);
}

// Test hook for the bounded wait: one thread waits, with the kernels' own
// helper, on an mbarrier that expects one arrival that never comes.  It gives
// up after `limit` polls, records the time it waited (global timer) and raises
// `err` as a stage kernel does; nothing faults and the context stays usable.
__global__ void k_tc_wait_probe(uint32_t limit, int* err, unsigned long long* waited_ns) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_abort;
  if (threadIdx.x != 0) return;
  tc::mbar_init(&bar, 1);
  tc::mbar_fence_init();
  s_abort = 0;
  unsigned long long t0, t1;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  const bool ok = tc_wait1(&bar, 0u, &s_abort, limit);
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
  *waited_ns = t1 - t0;
  if (!ok) atomicExch(err, 1);
}

template <int N, int MODE>
__global__ void __launch_bounds__(kTcThreadsAll, 1)
rhs_tc_kernel(RhsParams P, TcTables T, int64_t n_tiles, int* err) {
  using C = TcCfg<N>;
  constexpr int NP = C::NP, NFP = C::NFP, E = C::E, M = C::M;
  constexpr int KV = C::KV, NV = C::NV, KLF = C::KLF, NL = C::NL;
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t bar_ld[3];   // state + records of a slot landed
  __shared__ __align__(8) uint64_t bar_p[2];    // residual register of a slot landed
  __shared__ __align__(8) uint64_t bar_avol;    // flux warps: volume operand in TMEM
  __shared__ __align__(8) uint64_t bar_alift[2];  // flux warps: LIFT operand half (faces 0-1 | 2-3) written
  __shared__ __align__(8) uint64_t bar_l0done;    // the MMAs of LIFT half 0 done (half 0 free)
  __shared__ __align__(8) uint64_t bar_vdone;   // volume MMAs done (TMEM operand free)
  __shared__ __align__(8) uint64_t bar_mma[2];  // all MMAs of an accumulator set done
  __shared__ __align__(8) uint64_t bar_epi[2];  // epilogue of a tile done (results staged)
  __shared__ int s_abort;
  volatile int* const abort_flag = &s_abort;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool is_flux = warp < kTcFluxWarps;
  const bool is_epi = !is_flux && warp < kTcCtlWarp;
  const bool ctl0 = warp == kTcCtlWarp && lane == 0;
  unsigned char* const alh = tsm + C::O_ALH;
  unsigned char* const all = tsm + C::O_ALL;
  float* const sY0 = reinterpret_cast<float*>(tsm + C::O_Y);
  float* const sM0 = reinterpret_cast<float*>(tsm + C::O_M);
  float* const sP0 = reinterpret_cast<float*>(tsm + C::O_P);
  constexpr int kYStride = C::YS_B / 4, kMStride = C::MS_B / 4;
  uint8_t* const sFn = tsm + C::O_TAB;
  uint8_t* const sG = sFn + 4 * NFP;
  const bool use_p = MODE == kModeLserk && P.read_p;
  const int64_t tile0 = P.e_begin / E;  // the launch covers tiles [tile0, tile0 + n_tiles)
  const int64_t n_my =
      n_tiles > (int64_t)blockIdx.x ? (n_tiles - (int64_t)blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

  // a launch flagged off (adaptive stepping past its last attempt) does
  // nothing; the flag is read before any barrier or TMEM allocation
  if (P.skip != nullptr && *P.skip) return;

  // ---- set-up: TMEM, barriers, constant operands, tables
  if (warp == 0) tc::tmem_alloc(&s_tmem, C::TMEM_COLS);
  if (tid == 0) {
    for (int i = 0; i < 3; ++i) tc::mbar_init(&bar_ld[i], 1);
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&bar_p[i], 1);
      tc::mbar_init(&bar_mma[i], 1);
      tc::mbar_init(&bar_epi[i], kTcEpiWarps);
    }
    tc::mbar_init(&bar_avol, kTcFluxWarps);
    tc::mbar_init(&bar_alift[0], kTcFluxWarps);
    tc::mbar_init(&bar_alift[1], kTcFluxWarps);
    tc::mbar_init(&bar_l0done, 1);
    tc::mbar_init(&bar_vdone, 1);
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
    for (int i = tid; i < C::BL_B / 16; i += kTcThreadsAll) reinterpret_cast<uint4*>(tsm + C::O_BL)[i] = src[i];
    // LIFT operand padding (rows 30/31 of each quarter, face-padding columns)
    // must hold finite values and is never written again: start from zero.
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

#ifdef DGTD_TC_PHASE_TIMERS
  const bool timer_thread = lane == 0 && (warp == 0 || warp == kTcFluxWarps || warp == kTcCtlWarp);
  unsigned long long clk_acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  long long clk_last = clock64();
#endif

  if (is_flux) {
    // ================= flux warps: volume operand -> TMEM, fluxes -> LIFT operand
    const int q4 = warp & 3, vg = warp >> 2;
    // the TMEM row this lane writes: its own lane, or (16-lane stores at M = 64)
    // lane & 15 of the set's lane half, the thread half choosing the columns;
    // v_row = 6 (element in quarter) + component
    const int v_row = (C::LANE_SETS ? (lane & 15) : lane) - tc_qoff<C>(q4);
    const bool lane_real = v_row >= 0 && v_row < C::RL;
    const int v_src = lane_real ? ((q4 * C::EQ + v_row / 6) * 6 + v_row % 6) * NP : 0;
    const int v_rot = (C::LANE_SETS && lane_real) ? tc_node_rot(v_row / 6, v_row % 6) : 0;
    const uint32_t v_taddr = tmem + ((uint32_t)(q4 * 32) << 16);
    // flux slots q = (le, face, node-group, node-in-group) of each half (faces
    // 0-1, then 2-3).  What does not change from tile to tile is packed once:
    // f_item = le | f << 5 | m << 7 | (offset of the face node's state in the
    // tile) << (7 + MB), -1 idle; f_off = byte offset of the slot's entry
    // (component 0) in the LIFT operand.
    constexpr int kMMask = (1 << C::MB) - 1, kOffShift = C::OFF_SHIFT;
    int f_item[2][C::ITEMS_H];
    uint32_t f_off[2][C::ITEMS_H];
#pragma unroll
    for (int hh = 0; hh < 2; ++hh)
#pragma unroll
      for (int u = 0; u < C::ITEMS_H; ++u) {
        const int qh = tid + u * kTcFluxThreads;
        f_item[hh][u] = -1;
        f_off[hh][u] = 0u;
        if (qh < C::HSLOTS) {
          const int q = hh * C::HSLOTS + qh;
          const int s4 = q & 3, le = (q >> 2) % E, rest = (q >> 2) / E;  // rest = f * (KLF/4) + mg
          const int f = rest / (KLF / 4), m = (rest % (KLF / 4)) * 4 + s4;
          if (m < NFP) {
            f_item[hh][u] = le | (f << 5) | (m << 7) | ((le * 6 * NP + sFn[f * NFP + m]) << kOffShift);
            const int sl = f * KLF + m;
            f_off[hh][u] = (uint32_t)((sl >> 2) * (M / 8) * 128 + (sl & 3) * 4 + tc_row<C>(le, 0) * 16);
          }
        }
      }
    // Out-of-tile neighbour traces of this thread's slots in half hh (global
    // loads, zero where the neighbour is in the tile or absent).  They are
    // issued a phase ahead of their use: half 0's before the volume operand is
    // formed, half 1's right after it (before half 0's fluxes), so their
    // latency is hidden.
    // It also leaves, per slot, where the flux finds the neighbour trace:
    // zi >= 0 its offset in the tile's shared state, -1 the fetched registers,
    // -2 a PEC face, -3 a port face.
    const auto nb_fetch = [&](const float* sM, int64_t e0, int hh, float (&nb)[2][6], int (&zi)[2]) {
#pragma unroll
      for (int u = 0; u < 2; ++u) {
#pragma unroll
        for (int c = 0; c < 6; ++c) nb[u][c] = 0.f;
        zi[u] = -2;
        if (u >= C::ITEMS_H || f_item[hh][u] < 0) continue;
        const int x = f_item[hh][u];
        const int le = x & 31, f = (x >> 5) & 3, m = (x >> 7) & kMMask;
        const float* Me = sM + le * kMetaWords;
        const uint32_t codes = __float_as_uint(Me[41 + (f >> 1)]);
        const uint32_t code = (f & 1) ? (codes >> 16) : (codes & 0xffffu);
        const int nbr = __float_as_int(Me[37 + f]);
        const int kind = (code >> 8) & 3;
        const int gofs = sG[(code & 0xff) * NFP + m];
        const int lo = nbr - (int)e0;  // element ids fit in int
        if (kind == kInterior) {
          if ((uint32_t)lo < (uint32_t)E) {
            zi[u] = lo * 6 * NP + gofs;
          } else {
            zi[u] = -1;
            const float* Z = P.y_in + (int64_t)nbr * (6 * NP) + gofs;
#pragma unroll
            for (int c = 0; c < 6; ++c) nb[u][c] = __ldg(Z + c * NP);
          }
        } else {
          zi[u] = kind == kPort ? -3 : -2;
        }
      }
    };
    int ys = 0;
    uint32_t ld_par = 0u;  // bit s: parity of the next wait on bar_ld[s]
    for (int64_t it = 0; it < n_my; ++it) {
      const int64_t tile = tile0 + blockIdx.x + it * gridDim.x;
      const int64_t e0 = tile * E;
      const float* const sY = sY0 + ys * kYStride;
      const float* const sM = sM0 + ys * kMStride;
      bool ok = tc_waitw(&bar_ld[ys], (ld_par >> ys) & 1u, abort_flag);
      ld_par ^= 1u << ys;
      float nb_h[2][2][6];
      int zi_h[2][2];
      if (ok) nb_fetch(sM, e0, 0, nb_h[0], zi_h[0]);
      if (ok && it > 0) ok = tc_waitw(&bar_vdone, (uint32_t)((it - 1) & 1), abort_flag);
      if (!ok) {
        *abort_flag = 1;
        break;
      }
      tc::tc_fence_after();
      DGTD_TC_MARK(0);
      // ---- volume operand: row (e,c) of this lane, K = nodes, tf32 hi/lo -> TMEM
      if constexpr (C::LANE_SETS) {
        // 8-column unit w: this thread half's 4 columns 8 w + 4 (lane >> 4) ..,
        // in the lane half of the tile's accumulator set; the four nodes are
        // read from node v_rot on (no bank replays) and put back in order
        const uint32_t a_taddr = v_taddr + tc_set_off<C>((int)(it & 1));
#pragma unroll
        for (int cc = 0; cc < C::VCH_PER; ++cc) {
          const int w = vg + kTcVolGroups * cc;
          if (w < C::VCH) {
            const int n0 = 8 * w + 4 * (lane >> 4);
            float v4[4], h[4], l[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int k = n0 + ((q + v_rot) & 3);
              v4[q] = (lane_real && k < NP) ? sY[v_src + k] : 0.f;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float v = tc_pick4(v4, q, (4 - v_rot) & 3);  // node n0 + q
              h[q] = tc::tf32_round(v);
              l[q] = v - h[q];
            }
            tc::tmem_st16x2_4(a_taddr + (uint32_t)(C::T_AHI + w * 8), h);
            tc::tmem_st16x2_4(a_taddr + (uint32_t)(C::T_ALO + w * 8), l);
          }
        }
      } else {
#pragma unroll
        for (int cc = 0; cc < C::VCH_PER; ++cc) {
          const int ch = vg + kTcVolGroups * cc;
          if (ch < C::VCH) {
            float h[8], l[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const int k = ch * 8 + q;
              const float v = (lane_real && k < NP) ? sY[v_src + k] : 0.f;
              // hi/lo split as for the LIFT operand (flux section below)
              h[q] = tc::tf32_round(v);
              l[q] = v - h[q];
            }
            tc::tmem_st8(v_taddr + (uint32_t)(C::T_AHI + ch * 8), h);
            tc::tmem_st8(v_taddr + (uint32_t)(C::T_ALO + ch * 8), l);
          }
        }
      }
      tc::tmem_st_wait();
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&bar_avol);
      DGTD_TC_MARK(1);
      // ---- numerical flux (rhs.rs:1370-1441) by halves of the LIFT operand:
      // faces 0-1, then 2-3.  A half is free once the previous tile's MMAs of
      // that half are done; its own MMAs then run while the next half is formed.
      // half 1's traces: before the wait for half 0's operand to be free
      nb_fetch(sM, e0, 1, nb_h[1], zi_h[1]);
      // the numerical flux of slot u of half hh (false: an idle slot)
      const auto flux_of = [&](int hh, int u, float (&fl)[6]) -> bool {
        if (u >= C::ITEMS_H || f_item[hh][u] < 0) return false;
        const int x = f_item[hh][u];
        const int le = x & 31, f = (x >> 5) & 3;
        const float* Me = sM + le * kMetaWords;
        const float nx = Me[9 + 3 * f], ny = Me[10 + 3 * f], nz = Me[11 + 3 * f];
        const float coef = 0.5f * Me[21 + f];
        const int zi = zi_h[hh][u];
        const float* Y = sY + (x >> kOffShift);
        const float ex = Y[0 * NP], ey = Y[1 * NP], ez = Y[2 * NP];
        const float hx = Y[3 * NP], hy = Y[4 * NP], hz = Y[5 * NP];
        float jex, jey, jez, jhx, jhy, jhz;
        float a = P.alpha;
        if (zi == -3) {
          // characteristic boundary against a zero incident field (rhs.rs:1380-1386)
          jex = ex; jey = ey; jez = ez; jhx = hx; jhy = hy; jhz = hz;
          a = 1.0f;
        } else if (zi == -2) {
          // PEC ghost: [E] = 2 E_tan, [H] = 2 H_n (rhs.rs:1387-1402)
          const float edn = nx * ex + ny * ey + nz * ez;
          const float hdn = nx * hx + ny * hy + nz * hz;
          jex = 2.0f * (ex - edn * nx); jey = 2.0f * (ey - edn * ny); jez = 2.0f * (ez - edn * nz);
          jhx = 2.0f * (hdn * nx); jhy = 2.0f * (hdn * ny); jhz = 2.0f * (hdn * nz);
        } else {
          const float (&nb)[6] = nb_h[hh][u];
          float px = nb[0], py = nb[1], pz = nb[2];
          float qx = nb[3], qy = nb[4], qz = nb[5];
          if (zi >= 0) {
            const float* Z = sY + zi;
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
        fl[0] = fmaf(de, nx, fmaf(-ca, jex, -coef * (ny * jhz - nz * jhy)));
        fl[1] = fmaf(de, ny, fmaf(-ca, jey, -coef * (nz * jhx - nx * jhz)));
        fl[2] = fmaf(de, nz, fmaf(-ca, jez, -coef * (nx * jhy - ny * jhx)));
        fl[3] = fmaf(dh, nx, fmaf(-ca, jhx, coef * (ny * jez - nz * jey)));
        fl[4] = fmaf(dh, ny, fmaf(-ca, jhy, coef * (nz * jex - nx * jez)));
        fl[5] = fmaf(dh, nz, fmaf(-ca, jhz, coef * (nx * jey - ny * jex)));
        return true;
      };
      // ... into the LIFT operand: hi = tf32(fl), lo = fl - hi (exact,
      // |lo| <= 2^-11 |fl|).  lo is stored unrounded: the tf32 MMA reads only
      // its top 19 bits, an error below 2^-10 |lo| <= 2^-21 |fl|, under the
      // 3xTF32 products' own 2^-22-class terms in the sum of many products.
      const auto store_of = [&](int hh, int u, const float (&fl)[6]) {
        const uint32_t off = f_off[hh][u];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const float h = tc::tf32_round(fl[c]);
          *reinterpret_cast<float*>(alh + off + c * 16) = h;
          *reinterpret_cast<float*>(all + off + c * 16) = fl[c] - h;
        }
      };
      // At M = 64 (one slot per thread and half) both halves' fluxes are formed
      // before the waits for their operand halves to be free: two independent
      // chains per thread, and no flux arithmetic behind an MMA completion.
      float fe[2][6];
      bool fe_on[2] = {false, false};
      if constexpr (C::LANE_SETS) {
        fe_on[0] = flux_of(0, 0, fe[0]);
        fe_on[1] = flux_of(1, 0, fe[1]);
      }
      bool half_ok = true;
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        if (it > 0) {
          const bool free_ok = hh == 0 ? tc_waitw(&bar_l0done, (uint32_t)((it - 1) & 1), abort_flag)
                                       : tc_waitw(&bar_mma[(it - 1) & 1], (uint32_t)(((it - 1) >> 1) & 1), abort_flag);
          if (!free_ok) {
            half_ok = false;
            break;
          }
        }
        DGTD_TC_MARK(2);
        if constexpr (C::LANE_SETS) {
          if (fe_on[hh]) store_of(hh, 0, fe[hh]);
        } else {
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            float fl[6];
            if (flux_of(hh, u, fl)) store_of(hh, u, fl);
          }
        }
        tc::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&bar_alift[hh]);
      }
      if (!half_ok) {
        *abort_flag = 1;
        break;
      }
      DGTD_TC_MARK(3);
      ys = ys == 2 ? 0 : ys + 1;
    }
  } else if (is_epi) {
    // ================= epilogue warps: TMEM -> dy -> mode update, in place
    const int q4 = warp & 3, eg = (warp - kTcFluxWarps) >> 2;
    // the TMEM row of this lane: its own lane, or (16-lane loads at M = 64)
    // lane & 15, the thread half (hb = 0 | 16) reading the second chunk of a
    // pair; e_row = 6 (element in quarter) + component
    const int qo = tc_qoff<C>(q4), hb = C::LANE_SETS ? (lane & 16) : 0;
    const int e_row = (C::LANE_SETS ? (lane & 15) : lane) - qo;
    const bool lane_real = e_row >= 0 && e_row < C::RL;
    const int e_le = q4 * C::EQ + (lane_real ? e_row / 6 : C::EQ - 1);
    const int e_c = lane_real ? e_row % 6 : 5;
    const int e_fld = e_c / 3, e_t = e_c % 3;
    const int e_srcA = lane_real ? hb + qo + (e_row / 6) * 6 + 3 * (1 - e_fld) + (e_t + 2) % 3 : lane;
    const int e_srcB = lane_real ? hb + qo + (e_row / 6) * 6 + 3 * (1 - e_fld) + (e_t + 1) % 3 : lane;
    const int e_rot = (C::LANE_SETS && lane_real) ? tc_node_rot(e_row / 6, e_c) : 0;
    const float e_sign = e_fld == 0 ? 1.f : -1.f;
    const int e_cA = (e_t + 2) % 3, e_cB = (e_t + 1) % 3;
    const int e_row_off = (e_le * 6 + e_c) * NP;
    float kry_sig = 1.f, kry_g = 0.f;
    if (MODE == kModeKrylov) {
      kry_sig = (float)P.kry[0];
      kry_g = (float)P.kry[1];
    }
    float kcl_h = 0.f, kcl_gs = 0.f;
    if (MODE == kModeKcl) {
      kcl_h = *P.kcl_h;
      kcl_gs = P.kcl_g != nullptr ? P.kcl_g[*P.kcl_frame] : 0.f;
    }
    int ys = 0;
    uint32_t ld_par = 0u;
    for (int64_t it = 0; it < n_my; ++it) {
      const int64_t tile = tile0 + blockIdx.x + it * gridDim.x;
      const int ps = (int)(it & 1);
      const uint32_t ppar = (uint32_t)((it >> 1) & 1);
      bool ok = tc_waitw(&bar_mma[ps], ppar, abort_flag);
      if (ok) ok = tc_waitw(&bar_ld[ys], (ld_par >> ys) & 1u, abort_flag);
      ld_par ^= 1u << ys;
      if (ok && use_p) ok = tc_waitw(&bar_p[ps], ppar, abort_flag);
      if (!ok) {
        *abort_flag = 1;
        break;
      }
      tc::tc_fence_after();
      DGTD_TC_MARK(4);
      const float* Me = sM0 + ys * kMStride + e_le * kMetaWords;
      // curl partials (the B one negated) and material scaling with the curl sign folded in
      const float gA0 = Me[0 * 3 + e_cA], gA1 = Me[1 * 3 + e_cA], gA2 = Me[2 * 3 + e_cA];
      const float gB0 = -Me[0 * 3 + e_cB], gB1 = -Me[1 * 3 + e_cB], gB2 = -Me[2 * 3 + e_cB];
      const float inv_w = Me[25 + 3 * e_fld + e_t];
      const float w_curl = e_sign * inv_w;
      const float sig_w = Me[31 + 3 * e_fld + e_t];
      const float dt_e = P.dt * Me[43];  // the element's own step (batched instances)
      float* const yrow = sY0 + ys * kYStride + e_row_off;
      float* const prow = sP0 + ps * kYStride + e_row_off;  // p in, p out (LSERK) / dy out (Apply)
      const int64_t t0 = tile * C::TILE_F;
      // do the step's sources reach this tile? (uniform per tile)
      const bool src_here = (MODE == kModeLserk || MODE == kModeKrylov || MODE == kModeKcl) &&
                            (P.src_vec != nullptr || (P.src_idx >= t0 && P.src_idx < t0 + C::TILE_F));
      const int64_t g_row = t0 + e_row_off;  // SoA index of node 0 of this row
      const uint32_t acc = tmem + tc_set_off<C>(ps) + ((uint32_t)(q4 * 32) << 16);
      // node chunks of 4 (M = 128), or pairs of them, one per thread half (M = 64)
      constexpr int kIters = C::LANE_SETS ? C::EPAIR_PER : C::ECH_PER;
      constexpr int kUnits = C::LANE_SETS ? C::EPAIRS : C::ECH;
#pragma unroll
      for (int cc = 0; cc < kIters; ++cc) {
        const int ch = eg + kTcEpiGroups * cc;
        if (ch < kUnits) {
          const int c0 = C::LANE_SETS ? ch * 8 : ch * 4;  // first column of the access
          const int i0 = c0 + (hb >> 2);                  // this thread's first node
          float r0[4], r1[4], r2[4], lf[4], lg[4];
          if constexpr (C::LANE_SETS) {
            tc::tmem_ld16x2_4(acc + (uint32_t)c0, r0);
            tc::tmem_ld16x2_4(acc + (uint32_t)(NP + c0), r1);
            tc::tmem_ld16x2_4(acc + (uint32_t)(2 * NP + c0), r2);
            tc::tmem_ld16x2_4(acc + (uint32_t)(NV + c0), lf);
            tc::tmem_ld16x2_4(acc + (uint32_t)(NV + NL + c0), lg);
          } else {
            tc::tmem_ldw<4>(acc + (uint32_t)i0, r0);
            tc::tmem_ldw<4>(acc + (uint32_t)(NP + i0), r1);
            tc::tmem_ldw<4>(acc + (uint32_t)(2 * NP + i0), r2);
            tc::tmem_ldw<4>(acc + (uint32_t)(NV + i0), lf);
            tc::tmem_ldw<4>(acc + (uint32_t)(NV + NL + i0), lg);
          }
          tc::tmem_ld_wait();
          // the mode's update of node i of this row from its dy (yv: y at node i)
          const auto update = [&](int i, float dy, float yv) {
            if (MODE == kModeLserk) {
              // LSERK4 stage (explicit.rs:122-133): p = a p + dt (dy + src); y += b p
              float k = dy;
              if (src_here) {
                if (P.src_vec != nullptr) k = fmaf(P.src_g, __ldg(P.src_vec + g_row + i), k);
                if (P.src_idx == g_row + i) k += P.src_g;
              }
              float pv = dt_e * k;
              if (P.read_p) pv = fmaf(P.a, prow[i], pv);
              prow[i] = pv;
              yrow[i] = fmaf(P.b, pv, yv);
            } else if (MODE == kModeKcl) {
              // KCL stage (explicit_adaptive.rs:84-152) straight to global
              // memory, in the operation order of the separate stage kernel
              // (kcl.cuh k_kcl_stage); nothing is staged for the bulk store
              const int64_t g = g_row + i;
              float kk = dy;
              if (src_here) {
                if (P.src_vec != nullptr) kk += __ldg(P.src_vec + g) * kcl_gs;
                if (P.src_idx == g) kk += kcl_gs;
              }
              const float f = kcl_h * kk;
              const float yn = P.kcl_y[g] + P.kcl_b * f;
              P.kcl_y[g] = yn;
              P.kcl_e[g] = P.kcl_stage == 0 ? P.kcl_ew * f : P.kcl_e[g] + P.kcl_ew * f;
              if (P.kcl_next != nullptr) P.kcl_next[g] = yn + P.kcl_amb * f;
            } else if (MODE == kModeKrylov) {
              // Krylov matvec of a stored basis vector: its scale and the
              // augmented source coefficient from device memory
              float w = kry_sig * dy;
              if (src_here) {
                if (P.src_vec != nullptr) w = fmaf(kry_g, __ldg(P.src_vec + g_row + i), w);
                if (P.src_idx == g_row + i) w += kry_g;
              }
              prow[i] = w;
            } else {
              prow[i] = dy;
            }
          };
          if constexpr (C::LANE_SETS) {
            // curl and LIFT sums node by node (the shuffles pair one node), then
            // the row's four nodes from node e_rot on (no bank replays on the
            // state and residual tiles); same arithmetic as below
            float sc[4], sl[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const float A = fmaf(gA2, r2[u], fmaf(gA1, r1[u], gA0 * r0[u]));
              const float B = fmaf(gB2, r2[u], fmaf(gB1, r1[u], gB0 * r0[u]));
              sc[u] = __shfl_sync(0xffffffffu, A, e_srcA) + __shfl_sync(0xffffffffu, B, e_srcB);
              sl[u] = lf[u] + lg[u];
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              const int i = i0 + ((v + e_rot) & 3);
              if (lane_real && i < NP) {
                const float yv = yrow[i];
                update(i, fmaf(w_curl, tc_pick4(sc, v, e_rot), fmaf(inv_w, tc_pick4(sl, v, e_rot), -sig_w * yv)), yv);
              }
            }
          } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              // my contributions: A to curl component (t+1)%3, B to (t+2)%3
              const float A = fmaf(gA2, r2[u], fmaf(gA1, r1[u], gA0 * r0[u]));
              const float B = fmaf(gB2, r2[u], fmaf(gB1, r1[u], gB0 * r0[u]));
              const float pa = __shfl_sync(0xffffffffu, A, e_srcA);
              const float pb = __shfl_sync(0xffffffffu, B, e_srcB);
              const int i = i0 + u;
              if (lane_real && i < NP) {
                const float yv = yrow[i];
                update(i, fmaf(w_curl, pa + pb, fmaf(inv_w, lf[u] + lg[u], -sig_w * yv)), yv);
              }
            }
          }
        }
      }
      tc::tc_fence_before();
      tc::fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&bar_epi[ps]);
      DGTD_TC_MARK(5);
      ys = ys == 2 ? 0 : ys + 1;
    }
  } else if (ctl0) {
    // ================= control lane: loads, MMAs, stores
    uint32_t n_ld[3] = {0u, 0u, 0u}, n_p[2] = {0u, 0u}, n_mma[2] = {0u, 0u}, n_vd = 0u, n_l0 = 0u;
    const uint32_t idv = tc::idesc_tf32(M, NV), idl = tc::idesc_tf32(M, C::NL2);
    // Shared-memory descriptors of k-step 0, built once: k-step ks of an R-row
    // operand adds ks * 2R (16-byte units) to the start-address field, which
    // cannot carry (shared addresses are below 2^18).  With the k-steps fully
    // unrolled the issue of an MMA is an add and the instruction itself, so one
    // thread keeps the tensor pipe fed.
    const uint64_t dvh = tc::tf32_step_desc(tc::smem_u32(tsm + C::O_BVH), NV, 0);
    const uint64_t dvl = tc::tf32_step_desc(tc::smem_u32(tsm + C::O_BVL), NV, 0);
    const uint64_t dbl = tc::tf32_step_desc(tc::smem_u32(tsm + C::O_BL), C::NL2, 0);
    const uint64_t dah = tc::tf32_step_desc(tc::smem_u32(alh), M, 0);
    const uint64_t dal = tc::tf32_step_desc(tc::smem_u32(all), M, 0);
    auto load_y = [&](int64_t j) {  // tile j of this CTA -> slot j % 3
      const int s = (int)(j % 3);
      const int64_t tile = tile0 + blockIdx.x + j * gridDim.x;
      tc::mbar_expect_tx(&bar_ld[s], C::TILE_B + C::META_B);
      tc::bulk_g2s(sY0 + s * kYStride, P.y_in + tile * C::TILE_F, C::TILE_B, &bar_ld[s]);
      tc::bulk_g2s(sM0 + s * kMStride, P.meta + tile * E * kMetaWords, C::META_B, &bar_ld[s]);
      ++n_ld[s];
    };
    auto load_p = [&](int64_t j) {  // residual register of tile j -> slot j & 1
      const int s = (int)(j & 1);
      const int64_t tile = tile0 + blockIdx.x + j * gridDim.x;
      tc::mbar_expect_tx(&bar_p[s], C::TILE_B);
      tc::bulk_g2s(sP0 + s * kYStride, P.p + tile * C::TILE_F, C::TILE_B, &bar_p[s]);
      ++n_p[s];
    };
    auto store = [&](int64_t j) {
      const int64_t gb = (tile0 + (int64_t)blockIdx.x + j * gridDim.x) * C::TILE_F;
      const float* sy = sY0 + (int)(j % 3) * kYStride;
      const float* sp = sP0 + (int)(j & 1) * kYStride;
      if (MODE == kModeApply || MODE == kModeKrylov) {
        tc::bulk_s2g(P.out + gb, sp, C::TILE_B);
      } else if (MODE == kModeLserk) {
        tc::bulk_s2g(P.out + gb, sy, C::TILE_B);
        if (P.write_p) tc::bulk_s2g(P.p + gb, sp, C::TILE_B);
      }  // kModeKcl: the epilogue wrote global memory itself
      tc::bulk_commit();
    };
    if (n_my > 0) load_y(0);
    if (n_my > 1) load_y(1);
    if (n_my > 0 && use_p) load_p(0);
    bool ok = true;
    for (int64_t it = 0; it < n_my && ok; ++it) {
      const int as = (int)(it & 1);
      const uint32_t acc = tmem + tc_set_off<C>(as);
      // the volume A operand: one for both sets (M = 128) or the set's own (M = 64)
      const uint32_t a_base = tmem + (C::LANE_SETS ? tc_set_off<C>(as) : 0u);
      // volume MMAs: A = state hi/lo (TMEM), B = D hi/lo (shared)
      ok = tc_wait1(&bar_avol, (uint32_t)(it & 1), abort_flag);
      if (!ok) break;
      tc::tc_fence_after();
      DGTD_TC_MARK(6);
#pragma unroll
      for (int ks = 0; ks < KV / 8; ++ks) {
        const uint32_t a_h = a_base + (uint32_t)(C::T_AHI + 8 * ks), a_l = a_base + (uint32_t)(C::T_ALO + 8 * ks);
        const uint64_t bh = dvh + (uint64_t)(2 * NV * ks), bo = dvl + (uint64_t)(2 * NV * ks);
        tc::mma_tf32_ta(acc, a_h, bh, idv, ks > 0 ? 1u : 0u);
        tc::mma_tf32_ta(acc, a_h, bo, idv, 1u);
        tc::mma_tf32_ta(acc, a_l, bh, idv, 1u);
      }
      tc::mma_commit(&bar_vdone);
      ++n_vd;
      // Refills: the newest store group is tile it-2's (issued in the previous
      // iteration); once it has read its slots, they take tile it+1's state
      // (slot (it+1) % 3) and tile it's residual (slot it & 1).  Waiting after
      // the volume MMAs are issued keeps the wait off the tensor pipe's path.
      if (it > 0) {
        tc::bulk_wait_read0();
        DGTD_TC_MARK(7);
        if (it + 1 < n_my) load_y(it + 1);
        if (use_p) load_p(it);
      }
      // LIFT MMAs by halves: A = flux hi/lo (shared), B = stacked LIFT hi/lo
      // (shared): columns [NV, NV+NL) collect hi*hi + lo*hi, [NV+NL, NV+2NL)
      // hi*lo + lo*lo.  Half 0's commit frees it for the next tile's flux.
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        ok = tc_wait1(&bar_alift[hh], (uint32_t)(it & 1), abort_flag);
        if (!ok) break;
        tc::tc_fence_after();
        DGTD_TC_MARK(6);
#pragma unroll
        for (int j = 0; j < C::KS_H; ++j) {
          const int ks = hh * C::KS_H + j;
          const uint64_t bd = dbl + (uint64_t)(2 * C::NL2 * ks);
          tc::mma_tf32(acc + (uint32_t)NV, dah + (uint64_t)(2 * M * ks), bd, idl, ks > 0 ? 1u : 0u);
          tc::mma_tf32(acc + (uint32_t)NV, dal + (uint64_t)(2 * M * ks), bd, idl, 1u);
        }
        if (hh == 0) {
          tc::mma_commit(&bar_l0done);
          ++n_l0;
        } else {
          tc::mma_commit(&bar_mma[as]);
          ++n_mma[as];
        }
      }
      if (!ok) break;
      // results of the previous tile -> HBM
      if (it > 0) {
        ok = tc_wait1(&bar_epi[(it - 1) & 1], (uint32_t)(((it - 1) >> 1) & 1), abort_flag);
        if (!ok) break;
        DGTD_TC_MARK(6);
        store(it - 1);
      }
    }
    if (ok && n_my > 0) {
      ok = tc_wait1(&bar_epi[(n_my - 1) & 1], (uint32_t)(((n_my - 1) >> 1) & 1), abort_flag);
      if (ok) store(n_my - 1);
    }
    tc::bulk_wait0();
    if (!ok) {
      *abort_flag = 1;
      // let every async operation still in flight finish before the CTA exits
      for (int s = 0; s < 3; ++s)
        if (n_ld[s]) (void)tc::mbar_wait(&bar_ld[s], (n_ld[s] - 1) & 1u, kTcWaitLimit);
      for (int s = 0; s < 2; ++s) {
        if (n_p[s]) (void)tc::mbar_wait(&bar_p[s], (n_p[s] - 1) & 1u, kTcWaitLimit);
        if (n_mma[s]) (void)tc::mbar_wait(&bar_mma[s], (n_mma[s] - 1) & 1u, kTcWaitLimit);
      }
      if (n_vd) (void)tc::mbar_wait(&bar_vdone, (n_vd - 1) & 1u, kTcWaitLimit);
      if (n_l0) (void)tc::mbar_wait(&bar_l0done, (n_l0 - 1) & 1u, kTcWaitLimit);
    }
  }

  tc::tc_fence_before();
  __syncthreads();
  if (tid == 0 && s_abort) atomicExch(err, 1);
#ifdef DGTD_TC_PHASE_TIMERS
  if (timer_thread && P.phase_clk != nullptr)
    for (int i = 0; i < 8; ++i) atomicAdd(P.phase_clk + i, clk_acc[i]);
#endif
  if (warp == 0) tc::tmem_dealloc(tmem, C::TMEM_COLS);
}

}  // namespace dgtd
