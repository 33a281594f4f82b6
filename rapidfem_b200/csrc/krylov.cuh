// krylov.cuh -- device-resident Arnoldi / CGS2 for exp(tA)v and the ETD step.
//
// Follows propagator.rs:186-326 (expmv_into) and :338-373 (etd_step_into) and
// the reference GPU chunking of gpu/operator.rs:1175-1483, with every scalar of
// the iteration (Hessenberg H, projections, norms, the augmented components,
// the stop flag) kept in device memory: a chunk runs without a host round trip
// (the reference GPU path downloads the projections of every CGS pass and the
// norm partials of every step, gpu/operator.rs:1399-1443).
//
// Precision.  The basis is stored in the state type B: f32 for the FP32 and
// tensor-core engines, f64 for the FP64 path.  Every dot product and norm is
// accumulated in f64; H, the projections and the dense exponential are f64.
//
// Storage.  Basis vector i is sig[i] * (stored vector i): the Gram-Schmidt
// sweeps update the working vector in place in the slot of the next basis
// vector, and its normalisation 1/h_{j+1,j} is kept as the scale sig[j+1]
// instead of a rescaling sweep.
//
// Augmented system (the ETD step with a time-polynomial source).  With the
// source b*g(t0+tau), g(t0+tau) = sum_{m<P} a_m tau^m over the step, the
// exponential of
//     [[A, W], [0, J]],  W = b * (a_{P-1} (P-1)!, ..., a_1 1!, a_0 0!),
//     J the P x P upper shift,
// applied to [y; e_{P-1}] gives y(tau) = e^{tau A} y + sum_k tau^k
// phi_k(tau A) w_k in its first n components (Al-Mohy & Higham, SIAM J. Sci.
// Comput. 33 (2011), Theorem 2.1).  P = 1 with a_0 = 1 is the reference's
// held-source step exp(h[[A, b],[0, 0]])[y; 1] (propagator.rs:338-373); P = 0
// is expmv.  The augmented coordinates are scaled to the chunk's duration t
// (u_q -> u_q / t^(P-1-q), so J's entries become 1/t and W's columns
// a_{P-1-q} (P-1-q)! t^(P-1-q) b, the polynomial in scaled time) and by eta =
// 1/max(1, max|column coefficient|) (W -> eta W, e_{P-1} -> e_{P-1}/eta), so
// that the augmented part of the basis stays comparable to the state part.
// A basis vector's augmented part is the P-vector s[i]; the matvec of [v; u]
// is [A v + b*(c.u); J u] with c the scaled coefficients, so the RHS kernel
// adds (c.u) b with one device scalar (RhsParams::kry).
//
// One Arnoldi step j (cols = j+1 basis vectors), five launches:
//   RHS (mode Krylov)   w = sig_j A V_j + g_j b          (w in slot j+1)
//   k_kry_dots          block partials of V_i . w, i <= j, and of |w|^2
//   k_kry_update_dots   proj (every block reduces the partials itself), then
//                       w -= sum proj_i V_i, the second pass's partials and
//                       |w|^2 in the same sweep (one read of each V_i)
//   k_kry_update_norm   the second pass, only when the first removed more than
//                       half of |w|^2 (kReorth2): second-pass proj,
//                       w -= sum proj_i V_i, partials of |w|^2
//   k_kry_finish_norm   h_{j+1,j}, breakdown / last dimension / a-posteriori
//                       estimate h_{j+1,j}|exp(tH)_{d-1,0}| < tol (expm of H in
//                       one block), the next scale and augmented part
// Reductions are deterministic: fixed per-thread order, a fixed tree per
// block, a fixed-order sum over blocks.
#pragma once
#include <cstdint>

namespace dgtd {

constexpr int kKrylovMaxDim = 64;     // H capacity (64 x 64)
constexpr int kKryCols = 12;          // basis vectors of one chunk in the fused sweeps
constexpr int kKryMaxChunk = kKryCols;  // chunk dimension (the reference's KRYLOV_CHUNK is 12)
constexpr int kKryRow = 16;           // doubles per block row of sweep partials
constexpr int kKryNormCol = kKryRow - 1;  // the row's squared-norm column
// Second Gram-Schmidt pass only when the first one removed more than half of
// |w|^2, i.e. |w'| < |w| / sqrt(2) (Daniel, Gragg, Kaufman & Stewart, Math.
// Comp. 30 (1976): "twice is enough"); otherwise w' is orthogonal to the
// basis to working precision and the pass would not change it.
constexpr double kReorth2 = 0.5;
constexpr int kAugMax = 8;            // polynomial source terms
constexpr int kKrylovBlocks = 296;    // persistent reduction grid (2 per SM)
constexpr int kKrylovThreads = 256;

// Device-side scalar state of one Arnoldi chunk.
struct KrylovDev {
  double h[kKrylovMaxDim * kKrylovMaxDim];  // H, row-major, stride kKrylovMaxDim
  double sig[kKryCols];                     // basis vector i = sig[i] * stored vector i
  double s[kKryCols][kAugMax];              // augmented part of basis vector i
  double c[kAugMax];                        // scaled W / b (augmented source coefficients)
  double wa[3][kAugMax];                    // augmented part of w: after the matvec, pass 1, pass 2
  double coef[kKryCols];                    // result = sum coef[i] * stored vector i
  double mv[2];                             // next matvec: input scale, source coefficient
  double wn2;                               // |[w; wa]|^2 after the matvec (the pass-1 input)
  double hn2;                               // |[w'; wa]|^2 after pass 1, when pass 2 is skipped
  int reorth;                               // 1: pass 2 ran for the current step
  double beta, t, tol, est;
  int dim;                                  // dimension decided so far (the final one when done)
  int done;                                 // 1: stop growing the space
  int naug;                                 // P
  int max_dim;
  // accumulated over the chunks of one step (cleared by the host at its first chunk)
  int dim_total;                            // summed dimension
  int est_none;                             // a chunk formed no estimate
  double est_sum;                           // summed a-posteriori estimates
  int aborted;                              // a chunk missed its tolerance: later chunks are skipped
  int abort_chunks;                         // > 0: abort mode, the step's number of chunks
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Basis slot i: slot 0 is the chunk's input vector, slots 1.. are contiguous.
template <class B>
__host__ __device__ __forceinline__ const B* kry_col(const B* v0, const B* vb, int64_t len, int i) {
  return i == 0 ? v0 : vb + (int64_t)(i - 1) * len;
}

// Block sums of per-thread f64 values acc[0..cols) -> out[0..cols) (thread 0).
template <int NC>
__device__ __forceinline__ void block_sums(double (&acc)[NC], int cols, double* red /* [NC][8] shared */,
                                           double* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < NC; ++i)
    if (i < cols) {
      const double v = warp_sum(acc[i]);
      if (lane == 0) red[i * (kKrylovThreads / 32) + warp] = v;
    }
  __syncthreads();
  if (threadIdx.x < cols) {
    double s = 0.0;
    for (int q = 0; q < kKrylovThreads / 32; ++q) s += red[threadIdx.x * (kKrylovThreads / 32) + q];
    out[threadIdx.x] = s;
  }
}

// Sum over the blocks of a sweep's partial rows into out[kKryRow] (shared):
// the dot columns i < cols and the norm column, by all threads of a block of
// >= 256 threads: thread t adds the rows r, r + 16, ... (r = t / 16) of column
// t % 16, then the 16 values per column are added in a fixed order
// (deterministic, and the same in every block).
__device__ __forceinline__ void sum_partials(const double* partials, int nblocks, int cols, double* out) {
  constexpr int R = 256 / kKryRow;
  __shared__ double tmp[R * kKryRow];
  const int i = threadIdx.x % kKryRow, r = threadIdx.x / kKryRow;
  if (r < R) {
    double s = 0.0;
    if (i < cols || i == kKryNormCol)
      for (int b = r; b < nblocks; b += R) s += partials[(int64_t)b * kKryRow + i];
    tmp[threadIdx.x] = s;
  }
  __syncthreads();
  if ((int)threadIdx.x < kKryRow) {
    double t = 0.0;
    for (int q = 0; q < R; ++q) t += tmp[q * kKryRow + threadIdx.x];
    out[threadIdx.x] = t;
  }
  __syncthreads();
}

// The sweeps read whole 16-byte vectors (4 floats or 2 doubles): every vector
// is a state buffer of state length (whole tiles plus slack) whose entries
// past n are zero and stay zero, and every slot starts 16-byte aligned, so a
// sweep covers ceil(n / VW) vectors.  Each thread holds one vector of every
// column in registers before it accumulates, which keeps up to kKryCols
// 16-byte loads per thread in flight.
template <class B> struct KryVec;
template <> struct KryVec<float> {
  using T = float4;
  static constexpr int W = 4;
  __device__ static double at(const float4& v, int q) { return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w; }
  __device__ static void set(float4& v, int q, double x) {
    const float f = (float)x;
    if (q == 0) v.x = f; else if (q == 1) v.y = f; else if (q == 2) v.z = f; else v.w = f;
  }
};
template <> struct KryVec<double> {
  using T = double2;
  static constexpr int W = 2;
  __device__ static double at(const double2& v, int q) { return q == 0 ? v.x : v.y; }
  __device__ static void set(double2& v, int q, double x) {
    if (q == 0) v.x = x; else v.y = x;
  }
};

// partials[b*kKryRow + i] = sum over this block's k of V_i[k] * w[k], i < cols,
// and w . w in the norm column.
template <class B>
__global__ void __launch_bounds__(kKrylovThreads, 2)
k_kry_dots(const B* __restrict__ v0, const B* __restrict__ vb, int64_t len, int64_t n, int cols,
           const B* __restrict__ w, double* __restrict__ partials, const int* skip) {
  if (*skip) return;
  using KV = KryVec<B>;
  using T = typename KV::T;
  __shared__ double red[kKryCols * (kKrylovThreads / 32)];
  double acc[kKryCols];
#pragma unroll
  for (int i = 0; i < kKryCols; ++i) acc[i] = 0.0;
  double wn[1] = {0.0};
  const int64_t nv = (n + KV::W - 1) / KV::W;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += stride) {
    const T wk = reinterpret_cast<const T*>(w)[k];
    T vk[kKryCols];
#pragma unroll
    for (int i = 0; i < kKryCols; ++i)
      if (i < cols) vk[i] = reinterpret_cast<const T*>(kry_col(v0, vb, len, i))[k];
#pragma unroll
    for (int q = 0; q < KV::W; ++q) wn[0] = fma(KV::at(wk, q), KV::at(wk, q), wn[0]);
#pragma unroll
    for (int i = 0; i < kKryCols; ++i)
      if (i < cols)
#pragma unroll
        for (int q = 0; q < KV::W; ++q) acc[i] = fma(KV::at(vk[i], q), KV::at(wk, q), acc[i]);
  }
  double* row = partials + (int64_t)blockIdx.x * kKryRow;
  block_sums<kKryCols>(acc, cols, red, row);
  __syncthreads();
  block_sums<1>(wn, 1, red, row + kKryNormCol);
}

// The projections of a pass from the summed partials (every block computes them
// identically): proj_i = sig_i * sums[i] + s_i . wa_in.  Block 0 adds them to
// H[:, j] and writes wa_out = wa_in - sum_i proj_i s_i (pass 0 also records
// |[w; wa]|^2).  Returns, in shared u[], the update coefficients
// u_i = proj_i * sig_i of the stored vectors.
__device__ __forceinline__ void kry_proj(KrylovDev* st, const double* sums, int j, int pass, double* u) {
  __shared__ double proj[kKryCols];
  const int cols = j + 1;
  const int P = st->naug;
  if ((int)threadIdx.x < cols) {
    const int i = threadIdx.x;
    double s = sums[i] * st->sig[i];
    for (int q = 0; q < P; ++q) s += st->s[i][q] * st->wa[pass][q];
    proj[i] = s;
    u[i] = s * st->sig[i];
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int i = 0; i < cols; ++i) st->h[i * kKrylovMaxDim + j] += proj[i];
    for (int q = 0; q < P; ++q) {
      double d = st->wa[pass][q];
      for (int i = 0; i < cols; ++i) d -= proj[i] * st->s[i][q];
      st->wa[pass + 1][q] = d;
    }
    if (pass == 0) {
      double wa2 = 0.0;
      for (int q = 0; q < P; ++q) wa2 += st->wa[0][q] * st->wa[0][q];
      st->wn2 = sums[kKryNormCol] + wa2;
    }
  }
}

// First-pass update w -= sum u_i V_i and the second pass's dots in one sweep.
// NC (4, 8 or 12) bounds the columns held in registers: the launch picks the
// smallest NC >= j + 1.  Every instantiation fits 128 registers (two blocks
// per SM) with the f32 update of an f32 basis.
template <class B, int NC>
__global__ void __launch_bounds__(kKrylovThreads, 2)
k_kry_update_dots(KrylovDev* st, const B* __restrict__ v0, const B* __restrict__ vb, int64_t len, int64_t n,
                  int j, B* __restrict__ w, const double* __restrict__ partials_in, int nb_in,
                  double* __restrict__ partials_out, const int* skip) {
  static_assert(NC <= kKryCols, "columns");
  if (*skip) return;
  using KV = KryVec<B>;
  using T = typename KV::T;
  __shared__ double u[kKryCols];
  __shared__ double sums[kKryRow];
  __shared__ double red[kKryCols * (kKrylovThreads / 32)];
  const int cols = j + 1;
  sum_partials(partials_in, nb_in, cols, sums);
  kry_proj(st, sums, j, 0, u);
  __syncthreads();
  float uf[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) uf[i] = i < cols ? (float)u[i] : 0.f;
  double acc[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) acc[i] = 0.0;
  double wn[1] = {0.0};
  const int64_t nv = (n + KV::W - 1) / KV::W;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += stride) {
    T wk = reinterpret_cast<const T*>(w)[k];
    T vk[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i)
      if (i < cols) vk[i] = reinterpret_cast<const T*>(kry_col(v0, vb, len, i))[k];
    // per lane: the update, then the second pass's products with the stored
    // (rounded) value, so that only one lane's converted values are live.
    // An f32 basis takes the update in f32 (the stored vector is f32; the
    // dots that build H stay f64); an f64 basis keeps f64 throughout.
#pragma unroll
    for (int q = 0; q < KV::W; ++q) {
      if constexpr (sizeof(B) == 4) {
        float x = (float)KV::at(wk, q);
#pragma unroll
        for (int i = 0; i < NC; ++i)
          if (i < cols) x = fmaf(-uf[i], (float)KV::at(vk[i], q), x);
        KV::set(wk, q, x);
      } else {
        double x = KV::at(wk, q);
#pragma unroll
        for (int i = 0; i < NC; ++i)
          if (i < cols) x = fma(-u[i], KV::at(vk[i], q), x);
        KV::set(wk, q, x);
      }
      const double xs = KV::at(wk, q);
      wn[0] = fma(xs, xs, wn[0]);
#pragma unroll
      for (int i = 0; i < NC; ++i)
        if (i < cols) acc[i] = fma(KV::at(vk[i], q), xs, acc[i]);
    }
    reinterpret_cast<T*>(w)[k] = wk;
  }
  double* row = partials_out + (int64_t)blockIdx.x * kKryRow;
  block_sums<NC>(acc, cols, red, row);
  __syncthreads();
  block_sums<1>(wn, 1, red, row + kKryNormCol);
}

// The second pass, when it is needed: every block decides from the summed
// partials of pass 1 (|w'|^2 < kReorth2 |w|^2); without it block 0 records
// |[w'; wa]|^2 for the norm finisher and the sweep is skipped.  With it, the
// second-pass update and the partial sums of |w|^2 (the norm column).
template <class B, int NC>
__global__ void __launch_bounds__(kKrylovThreads, 2)
k_kry_update_norm(KrylovDev* st, const B* __restrict__ v0, const B* __restrict__ vb, int64_t len, int64_t n,
                  int j, B* __restrict__ w, const double* __restrict__ partials_in, int nb_in,
                  double* __restrict__ partials_out, const int* skip) {
  static_assert(NC <= kKryCols, "columns");
  if (*skip) return;
  using KV = KryVec<B>;
  using T = typename KV::T;
  __shared__ double u[kKryCols];
  __shared__ double sums[kKryRow];
  __shared__ double red[kKryCols * (kKrylovThreads / 32)];
  const int cols = j + 1;
  sum_partials(partials_in, nb_in, cols, sums);
  const int P = st->naug;
  double wa2 = 0.0;
  for (int q = 0; q < P; ++q) wa2 += st->wa[1][q] * st->wa[1][q];
  const double wn2_1 = sums[kKryNormCol] + wa2;
  if (!(wn2_1 < kReorth2 * st->wn2)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->reorth = 0;
      st->hn2 = wn2_1;
      for (int q = 0; q < kAugMax; ++q) st->wa[2][q] = st->wa[1][q];
    }
    return;  // uniform: every block takes the same decision
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->reorth = 1;
  kry_proj(st, sums, j, 1, u);
  __syncthreads();
  float uf[NC];
#pragma unroll
  for (int i = 0; i < NC; ++i) uf[i] = i < cols ? (float)u[i] : 0.f;
  double acc[1] = {0.0};
  const int64_t nv = (n + KV::W - 1) / KV::W;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += stride) {
    T wk = reinterpret_cast<const T*>(w)[k];
    T vk[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i)
      if (i < cols) vk[i] = reinterpret_cast<const T*>(kry_col(v0, vb, len, i))[k];
#pragma unroll
    for (int q = 0; q < KV::W; ++q) {
      if constexpr (sizeof(B) == 4) {  // f32 basis: the update in f32, as the first pass
        float x = (float)KV::at(wk, q);
#pragma unroll
        for (int i = 0; i < NC; ++i)
          if (i < cols) x = fmaf(-uf[i], (float)KV::at(vk[i], q), x);
        KV::set(wk, q, x);
      } else {
        double x = KV::at(wk, q);
#pragma unroll
        for (int i = 0; i < NC; ++i)
          if (i < cols) x = fma(-u[i], KV::at(vk[i], q), x);
        KV::set(wk, q, x);
      }
      const double xs = KV::at(wk, q);  // the stored (rounded) value
      acc[0] = fma(xs, xs, acc[0]);
    }
    reinterpret_cast<T*>(w)[k] = wk;
  }
  block_sums<1>(acc, 1, red, partials_out + (int64_t)blockIdx.x * kKryRow + kKryNormCol);
}

// Partial sums of x^2 (slot 0 of each block's row).
template <class B>
__global__ void __launch_bounds__(kKrylovThreads, 2)
k_kry_norm_partials(const B* __restrict__ x, int64_t n, double* __restrict__ partials) {
  __shared__ double red[kKrylovThreads / 32];
  double acc[1] = {0.0};
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double v = (double)x[k];
    acc[0] = fma(v, v, acc[0]);
  }
  block_sums<1>(acc, 1, red, partials + (int64_t)blockIdx.x * kKryRow + kKryNormCol);
}

// out[k] = sum_{i<dim} coef[i] * stored_i[k] (f64 accumulation), dim and coef
// from the device state; whole 16-byte vectors as the sweeps (the output's
// entries past n are written as the zero combination of zero entries).
template <class B>
__global__ void __launch_bounds__(kKrylovThreads, 2)
k_kry_lincomb(const B* __restrict__ v0, const B* __restrict__ vb, int64_t len, int64_t n, const KrylovDev* st,
              B* __restrict__ out) {
  using KV = KryVec<B>;
  using T = typename KV::T;
  __shared__ double c[kKryCols];
  const int dim = st->dim;
  if ((int)threadIdx.x < kKryCols) c[threadIdx.x] = (int)threadIdx.x < dim ? st->coef[threadIdx.x] : 0.0;
  __syncthreads();
  const int64_t nv = (n + KV::W - 1) / KV::W;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += (int64_t)gridDim.x * blockDim.x) {
    T vk[kKryCols];
#pragma unroll
    for (int i = 0; i < kKryCols; ++i)
      if (i < dim) vk[i] = reinterpret_cast<const T*>(kry_col(v0, vb, len, i))[k];
    T o;
#pragma unroll
    for (int q = 0; q < KV::W; ++q) {
      double x = 0.0;
#pragma unroll
      for (int i = 0; i < kKryCols; ++i)
        if (i < dim) x = fma(c[i], KV::at(vk[i], q), x);
      KV::set(o, q, x);
    }
    reinterpret_cast<T*>(out)[k] = o;
  }
}

// ---------------------------------------------------------------- dense expm
// exp(A) of a d x d matrix held in shared memory, Taylor-18 after scaling to
// ||.||_inf <= 1/2, then squaring (propagator.rs:69-114).  One block.
// Products use explicit round-to-nearest mul/add (no contraction), summing k
// in ascending order like the reference's matmul_into.
__device__ void block_matmul(const double* A, const double* B, double* C, int d) {
  for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) {
    const int i = idx / d, j = idx - i * d;
    double s = 0.0;
    for (int k = 0; k < d; ++k) {
      const double aik = A[i * d + k];
      if (aik == 0.0) continue;
      s = __dadd_rn(s, __dmul_rn(aik, B[k * d + j]));
    }
    C[idx] = s;
  }
}

// a: d*d input (shared), out: d*d result (shared), b, term, term2 scratch (shared).
// Each Taylor term and each squaring is one block-wide pass (the term's
// division by k and its addition to the sum ride along with the product,
// into the other buffer of a ping-pong pair), with the same operations in the
// same order per entry as a product followed by an update pass.
__device__ void block_expm(const double* a, int d, double* out, double* b, double* term, double* term2) {
  __shared__ int s_sq;
  __shared__ double s_row[kKrylovMaxDim];
  for (int i = threadIdx.x; i < d; i += blockDim.x) {
    double row = 0.0;
    for (int j = 0; j < d; ++j) row += fabs(a[i * d + j]);
    s_row[i] = row;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double nrm = 0.0;
    for (int i = 0; i < d; ++i) nrm = fmax(nrm, s_row[i]);
    // squarings: ceil(log2 |a|) + 1 for |a| > 1/2; a non-finite norm (a
    // Hessenberg matrix that overflowed) gets none, so the result is
    // non-finite and the caller rejects it, and a finite norm needs at most
    // 1025 (doubles stay below 2^1024)
    int sq = 0;
    if (nrm > 0.5 && nrm <= 1.7e308) sq = min(1025, (int)ceil(log2(nrm)) + 1);
    s_sq = sq;
  }
  __syncthreads();
  const int sq = s_sq;
  double scale = 1.0;
  for (int q = 0; q < sq; ++q) scale *= 2.0;
  for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) {
    b[idx] = a[idx] / scale;
    const int i = idx / d, j = idx - i * d;
    out[idx] = (i == j) ? 1.0 : 0.0;
    term[idx] = out[idx];
  }
  __syncthreads();
  double* cur = term;
  double* nxt = term2;
  for (int k = 1; k <= 18; ++k) {
    const double inv = 1.0 / (double)k;
    for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) {
      const int i = idx / d, j = idx - i * d;
      double s = 0.0;
      for (int q = 0; q < d; ++q) {
        const double aik = cur[i * d + q];
        if (aik == 0.0) continue;
        s = __dadd_rn(s, __dmul_rn(aik, b[q * d + j]));
      }
      const double t2 = s * inv;
      out[idx] += t2;
      nxt[idx] = t2;
    }
    __syncthreads();
    double* t = cur;
    cur = nxt;
    nxt = t;
  }
  // squarings, ping-ponging between out and term2
  double* src = out;
  double* dst = term2;
  for (int q = 0; q < sq; ++q) {
    block_matmul(src, src, dst, d);
    __syncthreads();
    double* t = src;
    src = dst;
    dst = t;
  }
  if (src != out) {
    for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) out[idx] = src[idx];
    __syncthreads();
  }
}

constexpr int kExpmThreads = 256;
constexpr size_t kExpmSmem = 5 * kKrylovMaxDim * kKrylovMaxDim * sizeof(double);

// ---------------------------------------------------------------- finishers
// All run as one block of kExpmThreads threads.

// Start of a chunk of duration t.  `a[P]` are the source polynomial's monomial
// coefficients about the step start, `delta` the chunk's offset in the step:
// the chunk's own coefficients are the Taylor shift
// a'_m = sum_{l>=m} a_l C(l,m) delta^(l-m).  beta = |[v; e_{P-1}/eta]|,
// sig[0] = 1/beta, s[0] = e_{P-1}/(eta beta).
__global__ void k_kry_start(KrylovDev* st, const double* partials, int nblocks, double t, double tol, int P,
                            const double* a, double delta, int max_dim, int* skip) {
  __shared__ double s_sums[kKryRow];
  if (st->aborted) {  // uniform: an earlier chunk of the step missed its tolerance
    if (threadIdx.x == 0) {
      st->dim = 0;
      st->est = 0.0;
      *skip = 1;
    }
    return;
  }
  sum_partials(partials, nblocks, 0, s_sums);
  if (threadIdx.x == 0) {
    double shifted[kAugMax], cu[kAugMax];
    double cmax = 0.0;
    for (int m = 0; m < P; ++m) {
      double acc = 0.0, binom = 1.0, dp = 1.0;  // C(l, m) delta^(l-m), l = m, m+1, ...
      for (int l = m; l < P; ++l) {
        acc += a[l] * binom * dp;
        binom = binom * (double)(l + 1) / (double)(l + 1 - m);
        dp *= delta;
      }
      shifted[m] = acc;
    }
    double fact = 1.0, tp = 1.0;
    for (int k = 0; k < P; ++k) {  // c_q = a'_{P-1-q} (P-1-q)! t^(P-1-q)
      if (k > 0) {
        fact *= (double)k;
        tp *= t;
      }
      cu[P - 1 - k] = shifted[k] * fact * tp;
    }
    for (int q = 0; q < P; ++q) cmax = fmax(cmax, fabs(cu[q]));
    const double eta = 1.0 / fmax(1.0, cmax);
    double s2 = s_sums[kKryNormCol];
    const double u_last = P > 0 ? 1.0 / eta : 0.0;
    s2 += u_last * u_last;
    const double beta = sqrt(s2);
    st->beta = beta;
    st->t = t;
    st->tol = tol;
    st->est = beta == 0.0 ? 0.0 : -1.0;  // -1: no estimate formed (tol = 0)
    st->naug = P;
    st->max_dim = max_dim;
    st->dim = beta == 0.0 ? 0 : max_dim;
    st->done = beta == 0.0 ? 1 : 0;
    for (int i = 0; i < kKryCols; ++i) {
      st->sig[i] = 0.0;
      st->coef[i] = 0.0;
      for (int q = 0; q < kAugMax; ++q) st->s[i][q] = 0.0;
    }
    for (int q = 0; q < kAugMax; ++q) {
      st->c[q] = q < P ? eta * cu[q] : 0.0;
      st->wa[0][q] = st->wa[1][q] = st->wa[2][q] = 0.0;
    }
    const double ib = beta > 0.0 ? 1.0 / beta : 0.0;
    st->sig[0] = ib;
    if (P > 0) st->s[0][P - 1] = u_last * ib;
    // the first matvec: scale of V_0, source coefficient c . s_0; and J s_0
    double g = 0.0;
    for (int q = 0; q < P; ++q) g += st->c[q] * st->s[0][q];
    st->mv[0] = ib;
    st->mv[1] = g;
    const double inv_t = t != 0.0 ? 1.0 / t : 0.0;  // J's scaled entries (unused when t = 0)
    for (int q = 0; q + 1 < P; ++q) st->wa[0][q] = st->s[0][q + 1] * inv_t;
    *skip = beta == 0.0 ? 1 : 0;
  }
  for (int i = threadIdx.x; i < kKrylovMaxDim * kKrylovMaxDim; i += blockDim.x) st->h[i] = 0.0;
}

// After the second pass: hnext = |[w; wa]|; stop on breakdown (1e-12), on the
// last dimension, or (tol > 0) on the a-posteriori estimate
// hnext*|exp(tH)_{d-1,0}| < tol (propagator.rs:271-301).  Otherwise record
// H[j+1,j], the scale and augmented part of V_{j+1} and the next matvec's scalars.
__global__ void k_kry_finish_norm(KrylovDev* st, const double* partials, int nblocks, int j, int* skip) {
  if (*skip) return;
  extern __shared__ double sm[];
  __shared__ double s_hnext;
  __shared__ int s_stop;
  __shared__ int s_break;
  __shared__ double s_sums[kKryRow];
  const int d = j + 1;
  const int P = st->naug;
  const bool reorth = st->reorth != 0;
  if (reorth) sum_partials(partials, nblocks, 0, s_sums);  // uniform
  if (threadIdx.x == 0) {
    double s;
    if (reorth) {
      s = s_sums[kKryNormCol];
      for (int q = 0; q < P; ++q) s += st->wa[2][q] * st->wa[2][q];
    } else {
      s = st->hn2;
    }
    s_hnext = sqrt(s);
    s_break = s_hnext < 1e-12 ? 1 : 0;
    const bool bad = !(s_hnext <= 1.7e308);  // a non-finite vector: stop, never passes
    s_stop = (s_break || bad || d == st->max_dim) ? 1 : 0;
    if (s_break) st->est = 0.0;
    if (bad) {
      st->est = INFINITY;
      s_break = 1;  // no estimate to form
    }
  }
  __syncthreads();
  const double hnext = s_hnext;
  // the estimate is also formed at the last dimension, where it only reports
  if (!s_break && st->tol > 0.0) {
    double* a = sm;
    double* out = a + kKrylovMaxDim * kKrylovMaxDim;
    double* b = out + kKrylovMaxDim * kKrylovMaxDim;
    double* t1 = b + kKrylovMaxDim * kKrylovMaxDim;
    double* t2 = t1 + kKrylovMaxDim * kKrylovMaxDim;
    const double t = st->t;
    for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) {
      const int r = idx / d, c = idx - r * d;
      a[idx] = t * st->h[r * kKrylovMaxDim + c];
    }
    __syncthreads();
    block_expm(a, d, out, b, t1, t2);
    if (threadIdx.x == 0) {
      double est = hnext * fabs(out[(d - 1) * d]);
      if (!(est == est) || isinf(est)) est = INFINITY;  // a non-finite space never passes
      st->est = est;
      if (est < st->tol) s_stop = 1;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (s_stop) {
      st->dim = d;
      st->done = 1;
      *skip = 1;
    } else {
      const double ih = 1.0 / hnext;
      st->h[(j + 1) * kKrylovMaxDim + j] = hnext;
      st->sig[j + 1] = ih;
      double g = 0.0;
      for (int q = 0; q < P; ++q) {
        st->s[j + 1][q] = st->wa[2][q] * ih;
        g += st->c[q] * st->s[j + 1][q];
      }
      st->mv[0] = ih;
      st->mv[1] = g;
      const double inv_t = st->t != 0.0 ? 1.0 / st->t : 0.0;
      for (int q = 0; q < kAugMax; ++q) st->wa[0][q] = q + 1 < P ? st->s[j + 1][q + 1] * inv_t : 0.0;
    }
  }
}

// End of a chunk: coef_i = beta * exp(tH)_{i,0} * sig_i over the final dim.
__global__ void k_kry_finish_coef(KrylovDev* st) {
  extern __shared__ double sm[];
  __shared__ int s_done;
  const int d = st->dim;
  if (threadIdx.x == 0) {
    if (!st->aborted) {
      st->dim_total += d;
      if (st->est < 0.0) {
        st->est_none = 1;
      } else if (st->abort_chunks > 0 && st->est > st->tol) {
        // abort mode: the chunk ran to its dimension without reaching its
        // tolerance, so the step fails whatever the later chunks give; they
        // are skipped and the reported sum is this estimate times the chunk
        // count
        st->aborted = 1;
        st->est_sum = st->est * (double)st->abort_chunks;
      } else {
        st->est_sum += st->est;
      }
    }
    s_done = (d == 0 || st->aborted) ? 1 : 0;
  }
  __syncthreads();
  if (s_done) return;  // uniform: thread 0 decided for the block
  double* a = sm;
  double* out = a + kKrylovMaxDim * kKrylovMaxDim;
  double* b = out + kKrylovMaxDim * kKrylovMaxDim;
  double* t1 = b + kKrylovMaxDim * kKrylovMaxDim;
  double* t2 = t1 + kKrylovMaxDim * kKrylovMaxDim;
  const double t = st->t;
  for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) {
    const int r = idx / d, c = idx - r * d;
    a[idx] = t * st->h[r * kKrylovMaxDim + c];
  }
  __syncthreads();
  block_expm(a, d, out, b, t1, t2);
  for (int i = threadIdx.x; i < d; i += blockDim.x) st->coef[i] = st->beta * out[i * d] * st->sig[i];
}

// Standalone dense expm for tests: a (d*d, global) -> out (global).
__global__ void k_expm_dense(const double* a_g, int d, double* out_g) {
  extern __shared__ double sm[];
  double* a = sm;
  double* out = a + kKrylovMaxDim * kKrylovMaxDim;
  double* b = out + kKrylovMaxDim * kKrylovMaxDim;
  double* t1 = b + kKrylovMaxDim * kKrylovMaxDim;
  double* t2 = t1 + kKrylovMaxDim * kKrylovMaxDim;
  for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) a[idx] = a_g[idx];
  __syncthreads();
  block_expm(a, d, out, b, t1, t2);
  for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) out_g[idx] = out[idx];
}

}  // namespace dgtd
