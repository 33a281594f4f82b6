// rhs_fp32.cuh -- fused DG Maxwell right-hand side on the CUDA cores, in FP32
// (rhs_fp32_kernel, the FP32 engine and the Arnoldi matvec) or FP64
// (rhs_fp64_kernel, the FP64 path: f64 operators, element records and state).
//
// One persistent CTA per SM slot walks tiles of E elements.  Per tile:
//   1. the y tile (E*6*Np floats, contiguous in the SoA layout) and the element
//      records are copied to shared memory with 16-byte vector loads;
//   2. the numerical flux of all 4*Nfp face nodes of every element is formed
//      (rhs.rs:1370-1441): the neighbour trace comes from shared memory when
//      the neighbour is in the tile, else from L2/HBM;
//   3. each thread owns one (element, node): 18 reference derivatives
//      D_k * F_c (rhs.rs:39-85), combined with J^-1 into curl H / -curl E;
//   4. the LIFT sum over the 4*Nfp flux values (rhs.rs:1433-1439), the
//      material scaling (rhs.rs:1443-1454), and the mode's epilogue:
//      plain dy, the fused LSERK4 stage update (explicit.rs:122-133, so dy
//      never reaches HBM), or the Krylov matvec output (scaled dy plus the
//      augmented source column).
// D and LIFT live in shared memory for the whole kernel.
#pragma once
#include <cstdint>

#include "dgtd_common.cuh"

namespace dgtd {

template <int N, class R = float, int TD = 1>
struct Fp32Cfg {
  static constexpr int NP = np_of(N);
  static constexpr int NFP = nfp_of(N);
  static constexpr int NF = 4 * NFP;
  // Elements per tile: ~256 threads (TD = 1) or half as many (TD = 2, the
  // small-tile engine), E even so the tile start stays 16B aligned.
  static constexpr int E = (N == 1 ? 64 : N == 2 ? 24 : N == 3 ? 12 : N == 4 ? 8 : 4) / TD;
  static_assert(TD == 1 || TD == 2, "tile divisor");
  static constexpr int THREADS = ((E * NP + 31) / 32) * 32;
  static constexpr int TILE = E * 6 * NP;  // values of state per tile
  // shared memory layout (in R); every region starts on a 16-byte boundary
  // because the state tile and the element records are filled with 16-byte
  // vectors (4 floats or 2 doubles).
  static constexpr int PER16 = 16 / (int)sizeof(R);
  static constexpr int al4(int x) { return (x + PER16 - 1) / PER16 * PER16; }
  static constexpr int OFF_D = 0;
  static constexpr int OFF_L = al4(OFF_D + 3 * NP * NP);
  static constexpr int OFF_Y = al4(OFF_L + NF * NP);
  static constexpr int OFF_F = al4(OFF_Y + TILE);
  static constexpr int OFF_M = al4(OFF_F + E * 6 * NF);
  static constexpr int OFF_B = al4(OFF_M + E * kMetaWords);  // byte tables start (in R)
  static constexpr int BYTES_TAB = 4 * NFP + kMaxGather * NFP;
  static constexpr int SMEM = OFF_B * (int)sizeof(R) + ((BYTES_TAB + 15) / 16) * 16;
  static_assert(OFF_Y % PER16 == 0 && OFF_M % PER16 == 0, "vector regions must be 16-byte aligned");
  static_assert(((E * 6 * NP) % PER16) == 0, "consecutive tiles must start 16-byte aligned");
  static_assert((kMetaWords % PER16) == 0, "element records are whole 16-byte vectors");
};

template <class R> struct Vec16;
template <> struct Vec16<float> { using T = float4; };
template <> struct Vec16<double> { using T = double2; };

// Integer words of an element record: bit patterns in the f32 records, exact
// values in the f64 records.
__device__ __forceinline__ int rec_int(float v) { return __float_as_int(v); }
__device__ __forceinline__ int rec_int(double v) { return (int)v; }
__device__ __forceinline__ uint32_t rec_uint(float v) { return __float_as_uint(v); }
__device__ __forceinline__ uint32_t rec_uint(double v) { return (uint32_t)v; }

template <class R>
__device__ __forceinline__ void cross3f(R ax, R ay, R az, R bx, R by, R bz, R& ox, R& oy, R& oz) {
  ox = ay * bz - az * by;
  oy = az * bx - ax * bz;
  oz = ax * by - ay * bx;
}

template <int N, int MODE, class R, int TD = 1>
__device__ __forceinline__ void rhs_cc_body(const RhsParamsT<R>& P, const OpTablesT<R>& T) {
  using C = Fp32Cfg<N, R, TD>;
  using V = typename Vec16<R>::T;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, E = C::E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* smem = reinterpret_cast<R*>(smem_raw);
  R* sD = smem + C::OFF_D;
  R* sL = smem + C::OFF_L;
  R* sY = smem + C::OFF_Y;
  R* sF = smem + C::OFF_F;
  R* sM = smem + C::OFF_M;
  uint8_t* sFn = reinterpret_cast<uint8_t*>(smem + C::OFF_B);
  uint8_t* sG = sFn + 4 * NFP;
  const int tid = threadIdx.x;

  if (P.skip != nullptr && *P.skip) return;  // uniform: nothing to do for this launch

  for (int i = tid; i < 3 * NP * NP; i += blockDim.x) sD[i] = T.dT[i];
  for (int i = tid; i < NF * NP; i += blockDim.x) sL[i] = T.liftT[i];
  for (int i = tid; i < 4 * NFP; i += blockDim.x) sFn[i] = T.fnodes[i];
  for (int i = tid; i < T.n_gather * NFP; i += blockDim.x) sG[i] = T.gtab[i];

  R kry_sig = 1, kry_g = 0;
  if (MODE == kModeKrylov) {
    kry_sig = (R)P.kry[0];
    kry_g = (R)P.kry[1];
  }

  const int64_t n_tiles = (P.n_elem - P.e_begin + E - 1) / E;
  const int le_me = tid / NP;
  const int i_me = tid - le_me * NP;
  const bool owns = tid < E * NP;

  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t e0 = P.e_begin + tile * E;
    const int ne = (int)((P.n_elem - e0) < E ? (P.n_elem - e0) : E);
    __syncthreads();  // previous tile fully consumed (and tables loaded on the first pass)
    // ---- 1. state tile and element records -> shared memory
    const int nfloat = ne * 6 * NP;
    {
      const R* src = P.y_in + e0 * 6 * NP;
      if ((nfloat % C::PER16) == 0) {
        const V* s4 = reinterpret_cast<const V*>(src);
        V* d4 = reinterpret_cast<V*>(sY);
        for (int i = tid; i < nfloat / C::PER16; i += blockDim.x) d4[i] = __ldg(s4 + i);
      } else {
        for (int i = tid; i < nfloat; i += blockDim.x) sY[i] = __ldg(src + i);
      }
    }
    {
      const V* m4 = reinterpret_cast<const V*>(P.meta + e0 * kMetaWords);
      V* d4 = reinterpret_cast<V*>(sM);
      for (int i = tid; i < ne * kMetaWords / C::PER16; i += blockDim.x) d4[i] = __ldg(m4 + i);
    }
    __syncthreads();

    // ---- 2. numerical flux at the 4*Nfp face nodes of each element
    for (int q = tid; q < ne * NF; q += blockDim.x) {
      const int le = q / NF;
      const int s = q - le * NF;
      const int f = s / NFP;
      const int m = s - f * NFP;
      const R* M = sM + le * kMetaWords;
      const R nx = M[9 + 3 * f], ny = M[10 + 3 * f], nz = M[11 + 3 * f];
      const R coef = R(0.5) * M[21 + f];
      const int nbr = rec_int(M[37 + f]);
      const uint32_t codes = rec_uint(M[41 + (f >> 1)]);
      const uint32_t code = (f & 1) ? (codes >> 16) : (codes & 0xffffu);
      const int kind = (code >> 8) & 3;
      const int vi = sFn[f * NFP + m];
      const R* Y = sY + le * 6 * NP;
      const R ex = Y[0 * NP + vi], ey = Y[1 * NP + vi], ez = Y[2 * NP + vi];
      const R hx = Y[3 * NP + vi], hy = Y[4 * NP + vi], hz = Y[5 * NP + vi];
      R jex, jey, jez, jhx, jhy, jhz;
      R a = P.alpha;
      if (kind == kPort) {
        // characteristic boundary against a zero incident field (rhs.rs:1380-1386)
        jex = ex; jey = ey; jez = ez; jhx = hx; jhy = hy; jhz = hz;
        a = R(1);
      } else if (kind == kPec) {
        // PEC ghost: [E] = 2 E_tan, [H] = 2 H_n (rhs.rs:1387-1402)
        const R edn = nx * ex + ny * ey + nz * ez;
        const R hdn = nx * hx + ny * hy + nz * hz;
        jex = R(2) * (ex - edn * nx); jey = R(2) * (ey - edn * ny); jez = R(2) * (ez - edn * nz);
        jhx = R(2) * (hdn * nx); jhy = R(2) * (hdn * ny); jhz = R(2) * (hdn * nz);
      } else {
        const int vj = sG[(code & 0xff) * NFP + m];
        const int64_t lo = (int64_t)nbr - e0;
        R px, py, pz, qx, qy, qz;
        if (lo >= 0 && lo < ne) {
          const R* Z = sY + lo * 6 * NP;
          px = Z[0 * NP + vj]; py = Z[1 * NP + vj]; pz = Z[2 * NP + vj];
          qx = Z[3 * NP + vj]; qy = Z[4 * NP + vj]; qz = Z[5 * NP + vj];
        } else {
          const R* Z = P.y_in + (int64_t)nbr * 6 * NP;
          px = __ldg(Z + 0 * NP + vj); py = __ldg(Z + 1 * NP + vj); pz = __ldg(Z + 2 * NP + vj);
          qx = __ldg(Z + 3 * NP + vj); qy = __ldg(Z + 4 * NP + vj); qz = __ldg(Z + 5 * NP + vj);
        }
        jex = ex - px; jey = ey - py; jez = ez - pz;
        jhx = hx - qx; jhy = hy - qy; jhz = hz - qz;
      }
      // n x [H], n x [E], n x (n x [E]), n x (n x [H])   (rhs.rs:1420-1432)
      R nhx, nhy, nhz, nex, ney, nez, pex, pey, pez, phx, phy, phz;
      cross3f(nx, ny, nz, jhx, jhy, jhz, nhx, nhy, nhz);
      cross3f(nx, ny, nz, jex, jey, jez, nex, ney, nez);
      cross3f(nx, ny, nz, nex, ney, nez, pex, pey, pez);
      cross3f(nx, ny, nz, nhx, nhy, nhz, phx, phy, phz);
      R* F = sF + le * 6 * NF;
      F[0 * NF + s] = coef * (-nhx + a * pex);
      F[1 * NF + s] = coef * (-nhy + a * pey);
      F[2 * NF + s] = coef * (-nhz + a * pez);
      F[3 * NF + s] = coef * (nex + a * phx);
      F[4 * NF + s] = coef * (ney + a * phy);
      F[5 * NF + s] = coef * (nez + a * phz);
    }

    // ---- 3. volume term: reference derivatives of E and H at my node
    R dex = 0, dey = 0, dez = 0, dhx = 0, dhy = 0, dhz = 0;
    const bool active = owns && le_me < ne;
    if (active) {
      const R* Y = sY + le_me * 6 * NP;
      R r[3][6];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 6; ++c) r[k][c] = 0;
      if constexpr (N == 5 && sizeof(R) == 4) {
        // the element's state rows are 16-byte aligned (Np = 56): four nodes of
        // all six components per float4 (broadcast) load, same accumulation
        // order (order 5: 14 % faster; orders 3 and 4 measured no gain)
#pragma unroll 2
        for (int j0 = 0; j0 < NP; j0 += 4) {
          float4 yv[6];
#pragma unroll
          for (int c = 0; c < 6; ++c) yv[c] = *reinterpret_cast<const float4*>(Y + c * NP + j0);
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int j = j0 + jj;
            const float d0 = sD[(0 * NP + j) * NP + i_me];
            const float d1 = sD[(1 * NP + j) * NP + i_me];
            const float d2 = sD[(2 * NP + j) * NP + i_me];
#pragma unroll
            for (int c = 0; c < 6; ++c) {
              const float v = jj == 0 ? yv[c].x : jj == 1 ? yv[c].y : jj == 2 ? yv[c].z : yv[c].w;
              r[0][c] = fmaf(d0, v, r[0][c]);
              r[1][c] = fmaf(d1, v, r[1][c]);
              r[2][c] = fmaf(d2, v, r[2][c]);
            }
          }
        }
      } else {
#pragma unroll 5
        for (int j = 0; j < NP; ++j) {
          const R d0 = sD[(0 * NP + j) * NP + i_me];
          const R d1 = sD[(1 * NP + j) * NP + i_me];
          const R d2 = sD[(2 * NP + j) * NP + i_me];
#pragma unroll
          for (int c = 0; c < 6; ++c) {
            const R v = Y[c * NP + j];
            r[0][c] = fma(d0, v, r[0][c]);
            r[1][c] = fma(d1, v, r[1][c]);
            r[2][c] = fma(d2, v, r[2][c]);
          }
        }
      }
      // physical derivatives pd[p][c] = sum_k Jinv[k][p] r[k][c] (rhs.rs:62-75)
      const R* M = sM + le_me * kMetaWords;
      R pd[3][6];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const R j0 = M[0 * 3 + p], j1 = M[1 * 3 + p], j2 = M[2 * 3 + p];
#pragma unroll
        for (int c = 0; c < 6; ++c) pd[p][c] = j0 * r[0][c] + j1 * r[1][c] + j2 * r[2][c];
      }
      // dE = curl H, dH = -curl E (rhs.rs:78-84, :1365-1368)
      dex = pd[1][5] - pd[2][4];
      dey = pd[2][3] - pd[0][5];
      dez = pd[0][4] - pd[1][3];
      dhx = -(pd[1][2] - pd[2][1]);
      dhy = -(pd[2][0] - pd[0][2]);
      dhz = -(pd[0][1] - pd[1][0]);
    }
    __syncthreads();  // flux complete

    // ---- 4. LIFT, materials, epilogue
    if (active) {
      const R* F = sF + le_me * 6 * NF;
      // order 5: the element's flux rows (NF = 4 Nfp values each) are 16-byte
      // aligned, so four face nodes of all six components come per float4
      // (broadcast) load; same accumulation order
      static_assert(NF % 4 == 0, "flux rows are whole float4s");
      if constexpr (N == 5 && sizeof(R) == 4) {
#pragma unroll 2
      for (int s0 = 0; s0 < NF; s0 += 4) {
        float4 fv[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) fv[c] = *reinterpret_cast<const float4*>(F + c * NF + s0);
#pragma unroll
        for (int ss = 0; ss < 4; ++ss) {
          const float w = sL[(s0 + ss) * NP + i_me];
          const auto pick = [ss](const float4& q) { return ss == 0 ? q.x : ss == 1 ? q.y : ss == 2 ? q.z : q.w; };
          dex = fmaf(w, pick(fv[0]), dex);
          dey = fmaf(w, pick(fv[1]), dey);
          dez = fmaf(w, pick(fv[2]), dez);
          dhx = fmaf(w, pick(fv[3]), dhx);
          dhy = fmaf(w, pick(fv[4]), dhy);
          dhz = fmaf(w, pick(fv[5]), dhz);
        }
      }
      } else {
#pragma unroll 4
        for (int s = 0; s < NF; ++s) {
          const R w = sL[s * NP + i_me];
          dex = fma(w, F[0 * NF + s], dex);
          dey = fma(w, F[1 * NF + s], dey);
          dez = fma(w, F[2 * NF + s], dez);
          dhx = fma(w, F[3 * NF + s], dhx);
          dhy = fma(w, F[4 * NF + s], dhy);
          dhz = fma(w, F[5 * NF + s], dhz);
        }
      }
      const R* M = sM + le_me * kMetaWords;
      const R* Y = sY + le_me * 6 * NP;
      R dy[6];
      dy[0] = M[25] * dex - M[31] * Y[0 * NP + i_me];
      dy[1] = M[26] * dey - M[32] * Y[1 * NP + i_me];
      dy[2] = M[27] * dez - M[33] * Y[2 * NP + i_me];
      dy[3] = M[28] * dhx - M[34] * Y[3 * NP + i_me];
      dy[4] = M[29] * dhy - M[35] * Y[4 * NP + i_me];
      dy[5] = M[30] * dhz - M[36] * Y[5 * NP + i_me];
      const int64_t base = (e0 + le_me) * 6 * NP + i_me;
      if (MODE == kModeApply) {
#pragma unroll
        for (int c = 0; c < 6; ++c) P.out[base + c * NP] = dy[c];
      } else if (MODE == kModeLserk) {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const int64_t g = base + c * NP;
          R k = dy[c];
          if (P.src_vec != nullptr) k = fma(P.src_g, __ldg(P.src_vec + g), k);
          if (g == P.src_idx) k += P.src_g;
          R pv = (P.dt * M[43]) * k;
          if (P.read_p) pv = fma(P.a, P.p[g], pv);
          if (P.write_p) P.p[g] = pv;
          P.out[g] = fma(P.b, pv, Y[c * NP + i_me]);
        }
      } else if (MODE == kModeKcl) {
        // KCL stage (explicit_adaptive.rs:84-152), in the operation order of
        // the separate stage kernel (kcl.cuh k_kcl_stage)
        const R h = (R)*P.kcl_h;
        const R gs = P.kcl_g != nullptr ? (R)P.kcl_g[*P.kcl_frame] : R(0);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const int64_t g = base + c * NP;
          R kk = dy[c];
          if (P.src_vec != nullptr) kk += P.src_vec[g] * gs;
          if (g == P.src_idx) kk += gs;
          const R f = h * kk;
          const R yn = P.kcl_y[g] + P.kcl_b * f;
          P.kcl_y[g] = yn;
          P.kcl_e[g] = P.kcl_stage == 0 ? P.kcl_ew * f : P.kcl_e[g] + P.kcl_ew * f;
          if (P.kcl_next != nullptr) P.kcl_next[g] = yn + P.kcl_amb * f;
        }
      } else {
        // Krylov matvec of a stored basis vector: its scale and the source
        // coefficient of the augmented system come from device memory
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const int64_t g = base + c * NP;
          R w = kry_sig * dy[c];
          if (P.src_vec != nullptr) w = fma(kry_g, __ldg(P.src_vec + g), w);
          if (g == P.src_idx) w += kry_g;
          P.out[g] = w;
        }
      }
    }
  }
}

// FP32 engine (stage, RHS and the Krylov matvec of an f32 basis); TD = 2 is
// the same engine with half-size element tiles (DGTD_ENGINE_FP32_SMALL_TILES).
template <int N, int MODE, int TD = 1>
__global__ void __launch_bounds__(Fp32Cfg<N, float, TD>::THREADS) rhs_fp32_kernel(RhsParams P, OpTables T) {
  rhs_cc_body<N, MODE, float, TD>(P, T);
}

// FP64 path: the same algorithm with f64 operators, records and state (and
// the Krylov matvec of an f64 basis).
template <int N, int MODE>
__global__ void __launch_bounds__(Fp32Cfg<N, double>::THREADS)
rhs_fp64_kernel(RhsParamsT<double> P, OpTablesT<double> T) {
  rhs_cc_body<N, MODE, double>(P, T);
}

}  // namespace dgtd
