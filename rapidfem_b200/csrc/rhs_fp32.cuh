// rhs_fp32.cuh -- fused DG Maxwell right-hand side on the CUDA cores (FP32).
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
//      never reaches HBM), or the f64 Arnoldi matvec output.
// D and LIFT live in shared memory for the whole kernel.
#pragma once
#include <cstdint>

#include "dgtd_common.cuh"

namespace dgtd {

template <int N>
struct Fp32Cfg {
  static constexpr int NP = np_of(N);
  static constexpr int NFP = nfp_of(N);
  static constexpr int NF = 4 * NFP;
  // Elements per tile: ~256 threads, E even so the tile start stays 16B aligned.
  static constexpr int E = N == 1 ? 64 : N == 2 ? 24 : N == 3 ? 12 : N == 4 ? 8 : 4;
  static constexpr int THREADS = ((E * NP + 31) / 32) * 32;
  static constexpr int TILE = E * 6 * NP;  // floats of state per tile
  // shared memory layout (floats); every region starts on a 16-byte boundary
  // because the state tile and the element records are filled with float4.
  static constexpr int al4(int x) { return (x + 3) & ~3; }
  static constexpr int OFF_D = 0;
  static constexpr int OFF_L = al4(OFF_D + 3 * NP * NP);
  static constexpr int OFF_Y = al4(OFF_L + NF * NP);
  static constexpr int OFF_F = al4(OFF_Y + TILE);
  static constexpr int OFF_M = al4(OFF_F + E * 6 * NF);
  static constexpr int OFF_B = al4(OFF_M + E * kMetaWords);  // byte tables start (as floats)
  static constexpr int BYTES_TAB = 4 * NFP + kMaxGather * NFP;
  static constexpr int SMEM = OFF_B * 4 + ((BYTES_TAB + 15) / 16) * 16;
  static_assert(OFF_Y % 4 == 0 && OFF_M % 4 == 0, "float4 regions must be 16-byte aligned");
  static_assert((TILE % 4) == 0 || (E % 2) == 0, "tile start must stay 16-byte aligned");
  static_assert(((E * 6 * NP) % 4) == 0, "consecutive tiles must start 16-byte aligned");
};

__device__ __forceinline__ void cross3f(float ax, float ay, float az, float bx, float by, float bz,
                                        float& ox, float& oy, float& oz) {
  ox = ay * bz - az * by;
  oy = az * bx - ax * bz;
  oz = ax * by - ay * bx;
}

template <int N, int MODE>
__global__ void __launch_bounds__(Fp32Cfg<N>::THREADS)
rhs_fp32_kernel(RhsParams P, OpTables T) {
  using C = Fp32Cfg<N>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, E = C::E;
  extern __shared__ __align__(16) float smem[];
  float* sD = smem + C::OFF_D;
  float* sL = smem + C::OFF_L;
  float* sY = smem + C::OFF_Y;
  float* sF = smem + C::OFF_F;
  float* sM = smem + C::OFF_M;
  uint8_t* sFn = reinterpret_cast<uint8_t*>(smem + C::OFF_B);
  uint8_t* sG = sFn + 4 * NFP;
  const int tid = threadIdx.x;

  if (P.skip != nullptr && *P.skip) return;  // uniform: nothing to do for this launch

  for (int i = tid; i < 3 * NP * NP; i += blockDim.x) sD[i] = T.dT[i];
  for (int i = tid; i < NF * NP; i += blockDim.x) sL[i] = T.liftT[i];
  for (int i = tid; i < 4 * NFP; i += blockDim.x) sFn[i] = T.fnodes[i];
  for (int i = tid; i < T.n_gather * NFP; i += blockDim.x) sG[i] = T.gtab[i];

  double aug_s = 0.0;
  if (MODE == kModeArnoldi && P.aug_s != nullptr) aug_s = *P.aug_s;

  const int64_t n_tiles = (P.n_elem + E - 1) / E;
  const int le_me = tid / NP;
  const int i_me = tid - le_me * NP;
  const bool owns = tid < E * NP;

  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t e0 = tile * E;
    const int ne = (int)((P.n_elem - e0) < E ? (P.n_elem - e0) : E);
    __syncthreads();  // previous tile fully consumed (and tables loaded on the first pass)
    // ---- 1. state tile and element records -> shared memory
    const int nfloat = ne * 6 * NP;
    if (MODE == kModeArnoldi) {
      const double* src = P.y_in64 + e0 * 6 * NP;
      for (int i = tid; i < nfloat; i += blockDim.x) sY[i] = (float)src[i];
    } else {
      const float* src = P.y_in + e0 * 6 * NP;
      if ((nfloat & 3) == 0) {
        const float4* s4 = reinterpret_cast<const float4*>(src);
        float4* d4 = reinterpret_cast<float4*>(sY);
        for (int i = tid; i < nfloat / 4; i += blockDim.x) d4[i] = __ldg(s4 + i);
      } else {
        for (int i = tid; i < nfloat; i += blockDim.x) sY[i] = __ldg(src + i);
      }
    }
    {
      const float4* m4 = reinterpret_cast<const float4*>(P.meta + e0 * kMetaWords);
      float4* d4 = reinterpret_cast<float4*>(sM);
      for (int i = tid; i < ne * kMetaWords / 4; i += blockDim.x) d4[i] = __ldg(m4 + i);
    }
    __syncthreads();

    // ---- 2. numerical flux at the 4*Nfp face nodes of each element
    for (int q = tid; q < ne * NF; q += blockDim.x) {
      const int le = q / NF;
      const int s = q - le * NF;
      const int f = s / NFP;
      const int m = s - f * NFP;
      const float* M = sM + le * kMetaWords;
      const float nx = M[9 + 3 * f], ny = M[10 + 3 * f], nz = M[11 + 3 * f];
      const float coef = 0.5f * M[21 + f];
      const int nbr = __float_as_int(M[37 + f]);
      const uint32_t codes = __float_as_uint(M[41 + (f >> 1)]);
      const uint32_t code = (f & 1) ? (codes >> 16) : (codes & 0xffffu);
      const int kind = (code >> 8) & 3;
      const int vi = sFn[f * NFP + m];
      const float* Y = sY + le * 6 * NP;
      const float ex = Y[0 * NP + vi], ey = Y[1 * NP + vi], ez = Y[2 * NP + vi];
      const float hx = Y[3 * NP + vi], hy = Y[4 * NP + vi], hz = Y[5 * NP + vi];
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
        const int vj = sG[(code & 0xff) * NFP + m];
        const int64_t lo = (int64_t)nbr - e0;
        float px, py, pz, qx, qy, qz;
        if (lo >= 0 && lo < ne) {
          const float* Z = sY + lo * 6 * NP;
          px = Z[0 * NP + vj]; py = Z[1 * NP + vj]; pz = Z[2 * NP + vj];
          qx = Z[3 * NP + vj]; qy = Z[4 * NP + vj]; qz = Z[5 * NP + vj];
        } else if (MODE == kModeArnoldi) {
          const double* Z = P.y_in64 + (int64_t)nbr * 6 * NP;
          px = (float)Z[0 * NP + vj]; py = (float)Z[1 * NP + vj]; pz = (float)Z[2 * NP + vj];
          qx = (float)Z[3 * NP + vj]; qy = (float)Z[4 * NP + vj]; qz = (float)Z[5 * NP + vj];
        } else {
          const float* Z = P.y_in + (int64_t)nbr * 6 * NP;
          px = __ldg(Z + 0 * NP + vj); py = __ldg(Z + 1 * NP + vj); pz = __ldg(Z + 2 * NP + vj);
          qx = __ldg(Z + 3 * NP + vj); qy = __ldg(Z + 4 * NP + vj); qz = __ldg(Z + 5 * NP + vj);
        }
        jex = ex - px; jey = ey - py; jez = ez - pz;
        jhx = hx - qx; jhy = hy - qy; jhz = hz - qz;
      }
      // n x [H], n x [E], n x (n x [E]), n x (n x [H])   (rhs.rs:1420-1432)
      float nhx, nhy, nhz, nex, ney, nez, pex, pey, pez, phx, phy, phz;
      cross3f(nx, ny, nz, jhx, jhy, jhz, nhx, nhy, nhz);
      cross3f(nx, ny, nz, jex, jey, jez, nex, ney, nez);
      cross3f(nx, ny, nz, nex, ney, nez, pex, pey, pez);
      cross3f(nx, ny, nz, nhx, nhy, nhz, phx, phy, phz);
      float* F = sF + le * 6 * NF;
      F[0 * NF + s] = coef * (-nhx + a * pex);
      F[1 * NF + s] = coef * (-nhy + a * pey);
      F[2 * NF + s] = coef * (-nhz + a * pez);
      F[3 * NF + s] = coef * (nex + a * phx);
      F[4 * NF + s] = coef * (ney + a * phy);
      F[5 * NF + s] = coef * (nez + a * phz);
    }

    // ---- 3. volume term: reference derivatives of E and H at my node
    float dex = 0.f, dey = 0.f, dez = 0.f, dhx = 0.f, dhy = 0.f, dhz = 0.f;
    const bool active = owns && le_me < ne;
    if (active) {
      const float* Y = sY + le_me * 6 * NP;
      float r[3][6];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 6; ++c) r[k][c] = 0.f;
      if constexpr (N == 5) {
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
          const float d0 = sD[(0 * NP + j) * NP + i_me];
          const float d1 = sD[(1 * NP + j) * NP + i_me];
          const float d2 = sD[(2 * NP + j) * NP + i_me];
#pragma unroll
          for (int c = 0; c < 6; ++c) {
            const float v = Y[c * NP + j];
            r[0][c] = fmaf(d0, v, r[0][c]);
            r[1][c] = fmaf(d1, v, r[1][c]);
            r[2][c] = fmaf(d2, v, r[2][c]);
          }
        }
      }
      // physical derivatives pd[p][c] = sum_k Jinv[k][p] r[k][c] (rhs.rs:62-75)
      const float* M = sM + le_me * kMetaWords;
      float pd[3][6];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const float j0 = M[0 * 3 + p], j1 = M[1 * 3 + p], j2 = M[2 * 3 + p];
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
      const float* F = sF + le_me * 6 * NF;
      // order 5: the element's flux rows (NF = 4 Nfp values each) are 16-byte
      // aligned, so four face nodes of all six components come per float4
      // (broadcast) load; same accumulation order
      static_assert(NF % 4 == 0, "flux rows are whole float4s");
      if constexpr (N == 5) {
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
          const float w = sL[s * NP + i_me];
          dex = fmaf(w, F[0 * NF + s], dex);
          dey = fmaf(w, F[1 * NF + s], dey);
          dez = fmaf(w, F[2 * NF + s], dez);
          dhx = fmaf(w, F[3 * NF + s], dhx);
          dhy = fmaf(w, F[4 * NF + s], dhy);
          dhz = fmaf(w, F[5 * NF + s], dhz);
        }
      }
      const float* M = sM + le_me * kMetaWords;
      const float* Y = sY + le_me * 6 * NP;
      float dy[6];
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
          float k = dy[c];
          if (P.src_vec != nullptr) k = fmaf(P.src_g, __ldg(P.src_vec + g), k);
          if (g == P.src_idx) k += P.src_g;
          float pv = (P.dt * M[43]) * k;
          if (P.read_p) pv = fmaf(P.a, P.p[g], pv);
          if (P.write_p) P.p[g] = pv;
          P.out[g] = fmaf(P.b, pv, Y[c * NP + i_me]);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const int64_t g = base + c * NP;
          double w = (double)dy[c];
          if (P.src64 != nullptr) w += aug_s * P.src64[g];
          P.out64[g] = w;
        }
      }
    }
  }
}

}  // namespace dgtd
