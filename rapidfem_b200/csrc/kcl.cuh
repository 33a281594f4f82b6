// kcl.cuh -- KCL RK4(3)5[2R+]C adaptive transient with the PI step-size
// controller on the device.
//
// The reference (gpu/operator.rs:823-893) runs the stage updates on the GPU
// but reads the embedded-error norm back to the host after every attempted
// substep to accept or reject it.  Here the controller state lives in device
// memory (KclCtl) and one attempt is a fixed sequence of launches:
//
//   k_kcl_begin      back up y, h_try = min(h, dt - t_rel) (session.rs:874)
//   5 x fused RHS + stage launches (mode kModeKcl of the RHS kernels: the
//                    stage update of explicit_adaptive.rs:84-152 in the RHS
//                    epilogue, so the stage derivative never reaches HBM)
//   k_kcl_err        block partials of sum((e / (atol + rtol max(|y0|,|y1|)))^2)
//   k_kcl_control    err_norm, accept / reject, PI factor (session.rs:130-187),
//                    frame bookkeeping, step-collapse check
//   k_kcl_restore    roll y back after a rejection
//   record kernels   the frame's state or functionals when a frame completes
//
// Every kernel of an attempt returns at once when the controller says there
// is nothing to do (run finished, collapsed, or capped), so the host can queue
// attempts in batches and read the status word once per batch instead of once
// per substep.
#pragma once
#include <cstdint>

namespace dgtd {

// KCL RK4(3)5[2R+]C coefficients, Kennedy, Carpenter & Lewis (2000) Table 1
// as constants.rs:151-178 lists them: a[i] = A_{i+1,i}, b, b_hat.
constexpr double kKclA[4] = {
    970286171893.0 / 4311952581923.0,
    6584761158862.0 / 12103376702013.0,
    2251764453980.0 / 15575788980749.0,
    26877169314380.0 / 34165994151039.0,
};
constexpr double kKclB[5] = {
    1153189308089.0 / 22510343858157.0,
    1772645290293.0 / 4653164025191.0,
    -1672844663538.0 / 4480602732383.0,
    2114624349019.0 / 3568978502595.0,
    5198255086312.0 / 14908931495163.0,
};
constexpr double kKclBhat[5] = {
    1016888040809.0 / 7410784769900.0,
    11231460423587.0 / 58533540763752.0,
    -1563879915014.0 / 6823010717585.0,
    606302364029.0 / 971179775848.0,
    1097981568119.0 / 3980877426909.0,
};
constexpr double kKclErrFloor = 1e-12;     // constants.rs:299
constexpr float kKclNonfiniteErr = 10.0f;  // constants.rs:296

enum KclStatus : int { kKclRunning = 0, kKclDone = 1, kKclCollapsed = 2, kKclCapped = 3 };

// One accepted substep of a run: its size and the output frame it belongs to.
struct KclLogEntry {
  float h;
  int frame;
};
constexpr long long kKclLogCap = 1 << 16;  // accepted substeps logged per run

struct KclCtl {
  // controller settings (session.rs:130-143)
  double atol, rtol, safety, growth, shrink, alpha, beta, min_step_factor;
  // state, in the f32 of the reference's GPU path (gpu/operator.rs:836-887)
  float dt, h, h_try, prev_err, t_rel, err_norm, h_min_log, h_max_log;
  long long frame, steps, n_acc, n_rej, attempts_in_frame, attempt_cap;
  KclLogEntry* log;  // accepted substeps, the first kKclLogCap of the run (or null)
  int status;
  int skip;     // nonzero: the attempt in flight does nothing
  int restore;  // the last attempt was rejected
  int record;   // frame row completed by the last attempt, or -1
};

// Controller::factor (session.rs:165-178), in f64.
__device__ inline double kcl_factor(const KclCtl& c, double err_norm, double prev, bool reject) {
  const double err = fmax(err_norm, kKclErrFloor);
  double f = c.safety * pow(err, -c.alpha);
  if (!(reject || prev <= 0.0)) f *= pow(prev, c.beta);
  return reject ? fmax(f, c.shrink) : fmin(fmax(f, c.shrink), c.growth);
}

__global__ void k_kcl_begin(KclCtl* __restrict__ ctl, const float* __restrict__ y, float* __restrict__ ybak,
                            int64_t n) {
  const bool run = ctl->status == kKclRunning && ctl->frame < ctl->steps;
  if (run)
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      ybak[i] = y[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->skip = run ? 0 : 1;
    if (run) ctl->h_try = fminf(ctl->h, ctl->dt - ctl->t_rel);
    ctl->restore = 0;
    ctl->record = -1;
  }
}

// Block partials of the weighted squared embedded error (kcl.cl weighted_err_sq).
__global__ void __launch_bounds__(256) k_kcl_err(const KclCtl* __restrict__ ctl, const float* __restrict__ y_old,
                                                 const float* __restrict__ y_new, const float* __restrict__ err,
                                                 double* __restrict__ partials, int64_t n) {
  if (ctl->skip) return;
  __shared__ float part[8];
  const float atol = (float)ctl->atol, rtol = (float)ctl->rtol;
  float acc = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float sc = atol + rtol * fmaxf(fabsf(y_old[i]), fabsf(y_new[i]));
    const float r = err[i] / sc;
    acc += r * r;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < 8; ++w) t += part[w];
    partials[blockIdx.x] = (double)t;
  }
}

// err_norm = sqrt(sum / n), then the accept / reject decision of
// gpu/operator.rs:848-887 and the frame bookkeeping.
__global__ void __launch_bounds__(256) k_kcl_control(KclCtl* __restrict__ ctl, const double* __restrict__ partials,
                                                     int nb, int64_t n) {
  if (ctl->skip) return;
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += partials[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  KclCtl& c = *ctl;
  const float err = (float)sqrt(red[0] / (double)(n > 0 ? n : 1));
  c.err_norm = err;
  const float h_try = c.h_try;
  const bool accept = isfinite(err) && err <= 1.0f;
  if (accept) {
    if (c.log != nullptr && c.n_acc < kKclLogCap) c.log[c.n_acc] = KclLogEntry{h_try, (int)c.frame};
    c.t_rel += h_try;
    c.n_acc += 1;
    const float factor = (float)kcl_factor(c, (double)err, (double)c.prev_err, false);
    c.h = h_try * factor;
    c.prev_err = fmaxf(err, (float)kKclErrFloor);
    c.h_min_log = fminf(c.h_min_log, c.h);
    c.h_max_log = fmaxf(c.h_max_log, c.h);
  } else {
    c.n_rej += 1;
    c.restore = 1;
    const float probe = isfinite(err) ? err : kKclNonfiniteErr;
    const float factor = (float)kcl_factor(c, (double)probe, (double)c.prev_err, true);
    c.h = h_try * factor;
  }
  c.attempts_in_frame += 1;
  if (c.h < (float)c.min_step_factor * c.dt) {
    c.status = kKclCollapsed;
    return;
  }
  if (accept && !(c.t_rel < c.dt)) {
    c.frame += 1;
    c.record = (int)c.frame;
    c.t_rel = 0.f;
    c.attempts_in_frame = 0;
    if (c.frame >= c.steps) c.status = kKclDone;
  } else if (c.attempts_in_frame >= c.attempt_cap) {
    c.status = kKclCapped;
  }
}

__global__ void k_kcl_restore(const KclCtl* __restrict__ ctl, float* __restrict__ y, const float* __restrict__ ybak,
                              int64_t n) {
  if (ctl->skip || !ctl->restore) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = ybak[i];
}

// Frame record: the SoA state into row `record` of a device trajectory.
__global__ void k_kcl_record_state(const KclCtl* __restrict__ ctl, const float* __restrict__ y,
                                   float* __restrict__ traj, int64_t n) {
  if (ctl->skip || ctl->record < 0) return;
  float* row = traj + (int64_t)ctl->record * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    row[i] = y[i];
}

// Frame record: linear functionals (one block each) into row `record`.
__global__ void __launch_bounds__(256) k_kcl_record_fun(const KclCtl* __restrict__ ctl, const float* __restrict__ y,
                                                        const int64_t* __restrict__ ptr,
                                                        const int64_t* __restrict__ idx,
                                                        const double* __restrict__ w, double* __restrict__ out,
                                                        int64_t n_fun) {
  if (ctl->skip || ctl->record < 0) return;
  __shared__ double part[8];
  const int q = blockIdx.x;
  double s = 0.0;
  for (int64_t k = ptr[q] + threadIdx.x; k < ptr[q + 1]; k += blockDim.x) s += w[k] * (double)y[idx[k]];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < 8; ++i) t += part[i];
    out[(int64_t)ctl->record * n_fun + q] = t;
  }
}

}  // namespace dgtd
