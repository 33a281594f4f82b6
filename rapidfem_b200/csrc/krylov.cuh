// krylov.cuh -- device-resident Arnoldi / CGS2 for exp(tA)v and the ETD step.
//
// Follows propagator.rs:186-326 (expmv_into) and :338-373 (etd_step_into) and
// the reference GPU chunking of gpu/operator.rs:1175-1483, with every scalar of
// the iteration (Hessenberg H, projections, norms, the augmented component s_j
// of the ETD basis, the stop flag) kept in device memory.  The reference GPU
// path downloads the projections of every CGS pass and the norm partials of
// every step to finish them on the host (gpu/operator.rs:1399-1443); here a
// one-block "finish" kernel does that work, so a chunk runs without a host
// round trip.  Basis, dots and H are f64; the matvec runs through the f32 RHS
// kernel (mode Arnoldi), reading the f64 basis vector and writing f64 w.
//
// Reductions are deterministic: per-warp partials in a fixed order, then a
// fixed-order sum over blocks.
#pragma once
#include <cstdint>

namespace dgtd {

constexpr int kKrylovMaxDim = 64;     // per-chunk Krylov dimension cap (H is 64x64)
constexpr int kKrylovBlocks = 296;    // persistent reduction grid (2 per SM)
constexpr int kKrylovThreads = 256;

// Device-side scalar state of one Arnoldi chunk.
struct KrylovDev {
  double h[kKrylovMaxDim * kKrylovMaxDim];  // H, row-major, stride kKrylovMaxDim
  double proj[kKrylovMaxDim + 1];
  double s[kKrylovMaxDim + 1];              // augmented component of each basis vector (ETD)
  double coef[kKrylovMaxDim];               // final combination coefficients
  double w_s;                               // augmented component of the working vector
  double beta, inv_beta, inv_h, t, tol;
  double est;                               // last a-posteriori estimate (tol > 0), 0 on breakdown
  int dim;                                  // dimension decided so far (the final one when done)
  int done;                                 // 1: stop growing the space
  int aug;                                  // 1: ETD augmented system
  int max_dim;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// partials[b*kKrylovMaxDim + i] = sum over this block's k of V_i[k]*w[k], i < cols.
// Skipped (no writes) when *skip != 0.
__global__ void __launch_bounds__(kKrylovThreads)
k_dots(const double* __restrict__ V, int64_t n, int cols, const double* __restrict__ w,
       double* __restrict__ partials, const int* skip) {
  if (*skip) return;
  __shared__ double acc[kKrylovMaxDim + 1][kKrylovThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < (kKrylovMaxDim + 1) * (kKrylovThreads / 32); i += blockDim.x)
    (&acc[0][0])[i] = 0.0;
  __syncthreads();
  const int64_t wstride = (int64_t)gridDim.x * (kKrylovThreads / 32) * 32;
  for (int64_t k0 = ((int64_t)blockIdx.x * (kKrylovThreads / 32) + warp) * 32; k0 < n; k0 += wstride) {
    const int64_t k = k0 + lane;
    const double wk = k < n ? w[k] : 0.0;
    for (int i = 0; i < cols; ++i) {
      double v = k < n ? V[(int64_t)i * n + k] * wk : 0.0;
      v = warp_sum(v);
      if (lane == 0) acc[i][warp] += v;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < cols; i += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < kKrylovThreads / 32; ++q) s += acc[i][q];
    partials[(int64_t)blockIdx.x * kKrylovMaxDim + i] = s;
  }
}

// w -= sum_i coef[i]*V_i (coef from device), optional partial sum of w^2 into
// partials[b*kKrylovMaxDim + 0].
__global__ void __launch_bounds__(kKrylovThreads)
k_update(const double* __restrict__ V, int64_t n, int cols, const double* __restrict__ coef,
         double* __restrict__ w, double* __restrict__ norm_partials, const int* skip) {
  if (*skip) return;
  __shared__ double c[kKrylovMaxDim];
  __shared__ double acc[kKrylovThreads / 32];
  for (int i = threadIdx.x; i < cols; i += blockDim.x) c[i] = coef[i];
  if (threadIdx.x < kKrylovThreads / 32) acc[threadIdx.x] = 0.0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double sq = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    double wk = w[k];
    for (int i = 0; i < cols; ++i) wk -= c[i] * V[(int64_t)i * n + k];
    w[k] = wk;
    sq += wk * wk;
  }
  if (norm_partials) {
    sq = warp_sum(sq);
    if (lane == 0) acc[warp] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int q = 0; q < kKrylovThreads / 32; ++q) s += acc[q];
      norm_partials[(int64_t)blockIdx.x * kKrylovMaxDim] = s;
    }
  }
}

// partial sums of x^2 (slot 0 of each block's partial row).
__global__ void __launch_bounds__(kKrylovThreads)
k_norm_partials(const double* __restrict__ x, int64_t n, double* __restrict__ partials) {
  __shared__ double acc[kKrylovThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double sq = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    sq += x[k] * x[k];
  sq = warp_sum(sq);
  if (lane == 0) acc[warp] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int q = 0; q < kKrylovThreads / 32; ++q) s += acc[q];
    partials[(int64_t)blockIdx.x * kKrylovMaxDim] = s;
  }
}

// out[k] = x[k] * (*scale)   (skipped when *skip)
__global__ void k_scale(const double* __restrict__ x, int64_t n, const double* scale,
                        double* __restrict__ out, const int* skip) {
  if (skip && *skip) return;
  const double s = *scale;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    out[k] = x[k] * s;
}

// out[k] = sum_{i<dim} coef[i]*V_i[k], dim and coef from the device state.
__global__ void k_lincomb(const double* __restrict__ V, int64_t n, const KrylovDev* st,
                          double* __restrict__ out) {
  __shared__ double c[kKrylovMaxDim];
  const int dim = st->dim;
  for (int i = threadIdx.x; i < dim; i += blockDim.x) c[i] = st->coef[i];
  __syncthreads();
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < dim; ++i) s += c[i] * V[(int64_t)i * n + k];
    out[k] = s;
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

// a: d*d input (shared), out: d*d result (shared), w1..w3 scratch (shared).
__device__ void block_expm(const double* a, int d, double* out, double* b, double* term,
                           double* term2) {
  __shared__ double s_norm;
  __shared__ int s_sq;
  if (threadIdx.x == 0) {
    double nrm = 0.0;
    for (int i = 0; i < d; ++i) {
      double row = 0.0;
      for (int j = 0; j < d; ++j) row += fabs(a[i * d + j]);
      nrm = fmax(nrm, row);
    }
    int sq = 0;
    if (nrm > 0.5) {
      long v = (long)ceil(log2(nrm)) + 1;
      sq = v > 0 ? (int)v : 0;
    }
    s_norm = nrm;
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
  for (int k = 1; k <= 18; ++k) {
    block_matmul(term, b, term2, d);
    __syncthreads();
    const double inv = 1.0 / (double)k;
    for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) {
      const double t2 = term2[idx] * inv;
      out[idx] += t2;
      term[idx] = t2;
    }
    __syncthreads();
  }
  for (int q = 0; q < sq; ++q) {
    block_matmul(out, out, term2, d);
    __syncthreads();
    for (int idx = threadIdx.x; idx < d * d; idx += blockDim.x) out[idx] = term2[idx];
    __syncthreads();
  }
}

constexpr int kExpmThreads = 256;
constexpr size_t kExpmSmem = 5 * kKrylovMaxDim * kKrylovMaxDim * sizeof(double);

// ---------------------------------------------------------------- finishers
// All run as one block of kExpmThreads threads.

// Start of a chunk: beta = sqrt(sum partials (+1 for the augmented [v;1])),
// zero H, s[0] = 1/beta, inv_beta.
__global__ void k_finish_start(KrylovDev* st, const double* partials, int nblocks, double t,
                               double tol, int aug, int max_dim) {
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partials[(int64_t)b * kKrylovMaxDim];
    if (aug) s += 1.0;
    const double beta = sqrt(s);
    st->beta = beta;
    st->inv_beta = beta > 0.0 ? 1.0 / beta : 0.0;
    st->t = t;
    st->tol = tol;
    st->est = beta == 0.0 ? 0.0 : -1.0;  // -1: no estimate formed (tol = 0)
    st->aug = aug;
    st->max_dim = max_dim;
    st->dim = max_dim;
    st->done = beta == 0.0 ? 1 : 0;
    st->w_s = 0.0;
    for (int i = 0; i <= kKrylovMaxDim; ++i) st->s[i] = 0.0;
    st->s[0] = aug ? st->inv_beta : 0.0;
    if (beta == 0.0) st->dim = 0;
  }
  for (int i = threadIdx.x; i < kKrylovMaxDim * kKrylovMaxDim; i += blockDim.x) st->h[i] = 0.0;
}

// After a matvec: the augmented operator's last row is zero (w_s = 0).
// After a dots pass: proj = sum partials (+ s_i*w_s), H[:,j] += proj,
// w_s -= sum proj_i s_i (gpu/operator.rs:1399-1410; propagator.rs:236-270).
__global__ void k_finish_proj(KrylovDev* st, const double* partials, int nblocks, int j,
                              int reset_ws, const int* skip) {
  if (*skip) return;
  __shared__ double proj[kKrylovMaxDim];
  const int cols = j + 1;
  if (reset_ws && threadIdx.x == 0) st->w_s = 0.0;
  __syncthreads();
  const double ws = st->w_s;
  for (int i = threadIdx.x; i < cols; i += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partials[(int64_t)b * kKrylovMaxDim + i];
    if (st->aug) s += st->s[i] * ws;
    proj[i] = s;
    st->proj[i] = s;
    st->h[i * kKrylovMaxDim + j] += s;
  }
  __syncthreads();
  if (threadIdx.x == 0 && st->aug) {
    double d = 0.0;
    for (int i = 0; i < cols; ++i) d += proj[i] * st->s[i];
    st->w_s = ws - d;
  }
}

// After the second pass: hnext = ||[w; w_s]||; stop on breakdown, on the last
// dimension, or (tol > 0) on the a-posteriori estimate
// hnext*|exp(tH)_{d-1,0}| < tol (propagator.rs:271-301).  Otherwise record
// H[j+1,j], inv_h and s[j+1].
__global__ void k_finish_norm(KrylovDev* st, const double* partials, int nblocks, int j,
                              int* skip) {
  if (*skip) return;
  extern __shared__ double sm[];
  __shared__ double s_hnext;
  __shared__ int s_stop;
  __shared__ int s_break;
  const int d = j + 1;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partials[(int64_t)b * kKrylovMaxDim];
    if (st->aug) s += st->w_s * st->w_s;
    s_hnext = sqrt(s);
    s_break = s_hnext < 1e-12 ? 1 : 0;
    s_stop = (s_break || d == st->max_dim) ? 1 : 0;
    if (s_break) st->est = 0.0;
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
      const double est = hnext * fabs(out[(d - 1) * d]);
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
      st->h[(j + 1) * kKrylovMaxDim + j] = hnext;
      st->inv_h = 1.0 / hnext;
      if (st->aug) st->s[j + 1] = st->w_s / hnext;
    }
  }
}

// End of a chunk: coef_i = beta * exp(tH)_{i,0} over the final dim.
__global__ void k_finish_coef(KrylovDev* st) {
  extern __shared__ double sm[];
  const int d = st->dim;
  if (d == 0) return;
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
  for (int i = threadIdx.x; i < d; i += blockDim.x) st->coef[i] = st->beta * out[i * d];
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
