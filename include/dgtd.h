/*
 * dgtd.h -- C ABI of the B200 DGTD hot path (librapidfem_b200.so).
 *
 * The entry points replace rapidfem's OpenCL backend, the `GpuContext` /
 * `GpuOperator` pair of crates/rapidfem-td/src/gpu/{mod.rs,operator.rs}, one
 * for one: plain pointers and sizes, no C++ or torch types.  A Rust host binds
 * them with an `extern "C"` block, a Python host with ctypes.
 *
 * State layout at the boundary is the reference's AoS layout
 * `y[(e*Np + node)*6 + c]`, c = Ex,Ey,Ez,Hx,Hy,Hz (rhs.rs:492-497).  The device
 * keeps its own element-major SoA copy; conversion happens on the device.
 *
 * Every call returns a dgtd_status; on failure `dgtd_last_error` gives the
 * message (thread-local).  There is no CPU fallback: without a usable CUDA
 * device the calls fail with DGTD_ERR_NO_DEVICE.
 *
 * Threading: one op per host thread at a time, like the reference's
 * `unsendable` TdSession (python/src/td.rs:163).  All work of an op is
 * issued on the op's stream (the context's stream by default).
 */
#ifndef DGTD_H
#define DGTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    DGTD_OK = 0,
    DGTD_ERR_BAD_ARG = 1,     /* length / range / shape mismatch (reference: assert! panics) */
    DGTD_ERR_CUDA = 2,        /* a CUDA runtime error (reference: "kernel launch failed: ...") */
    DGTD_ERR_NONFINITE = 3,   /* a NaN/Inf met by a checked run */
    DGTD_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
    DGTD_ERR_NO_DEVICE = 5,   /* no CUDA device (reference: "no OpenCL GPU device found") */
    DGTD_ERR_UNSUPPORTED = 6, /* order / feature outside what the kernels cover */
    DGTD_ERR_OOM = 7,         /* device allocation failed */
    DGTD_ERR_COLLAPSE = 8     /* adaptive step collapsed (reference: "GPU KCL: step size collapsed") */
} dgtd_status;

typedef struct dgtd_ctx dgtd_ctx;
typedef struct dgtd_op dgtd_op;

/* Copy the calling thread's last error message into buf (NUL-terminated): the
 * String the reference returns in its Result<_, String> errors. */
int dgtd_last_error(char *buf, size_t len);

/* Library / build identification: "rapidfem_b200 <version> sm_100a" (no
 * counterpart in the reference). */
const char *dgtd_version(void);

/* ---- context ----------------------------------------------------------
 * Replaces GpuContext::new (crates/rapidfem-td/src/gpu/mod.rs:49): picks the
 * CUDA device, creates the stream the ops run on. */
int dgtd_ctx_create(int device, dgtd_ctx **out);
/* Releases the context (GpuContext is dropped in the reference).  Ops and MLPs
 * made on a context may be destroyed after it (their destructors do not touch
 * the context); any other call on them needs the context alive. */
int dgtd_ctx_destroy(dgtd_ctx *ctx);
/* Device name (GpuContext::device_name, gpu/mod.rs:35). */
int dgtd_ctx_device_name(dgtd_ctx *ctx, char *buf, size_t len);
/* Run subsequent work of this context's ops on an external cudaStream_t
 * (NULL restores the context's own stream).  No counterpart in the reference,
 * whose OpenCL queue is private to GpuContext. */
int dgtd_ctx_set_stream(dgtd_ctx *ctx, void *cuda_stream);
/* Block until the context's stream is idle (no counterpart in the reference). */
int dgtd_ctx_synchronize(dgtd_ctx *ctx);

/* ---- operator ---------------------------------------------------------
 * The arrays GpuOperator::new flattens (gpu/operator.rs:222-292), in f64 as
 * the CPU operator holds them; the device copy is narrowed / split by the
 * library.  Np = (N+1)(N+2)(N+3)/6, Nfp = (N+1)(N+2)/2, K = n_elem. */
typedef struct {
    int32_t order;               /* N, 1..5 */
    int32_t n_elem;              /* K */
    double flux_alpha;           /* 0 central, 1 upwind (session.rs:93-99) */
    const double *diff_r;        /* Np*Np row-major, dg_basis.rs:100-102 */
    const double *diff_s;
    const double *diff_t;
    const double *lift;          /* Np*(4*Nfp) row-major, dg_basis.rs:383 */
    const int32_t *face_nodes;   /* 4*Nfp volume-node ids per face, dg_basis.rs:316-323 */
    const double *jinv;          /* 9K, J^-1[i][k] row-major, geom_factors.rs:81-88 */
    const double *inv_eps;       /* 3K, rhs.rs:900-926 */
    const double *inv_mu;        /* 3K */
    const double *sigma_eps;     /* 3K */
    const double *sigma_mu;      /* 3K */
    const double *face_normal;   /* 12K outward unit normals, topology.rs:64-78 */
    const double *face_fscale;   /* 4K, 2*area/|det J|, rhs.rs:828 */
    const int32_t *face_neighbor;  /* 4K, -1 = boundary */
    const int32_t *face_nbr_local; /* 4K */
    const int32_t *face_port;      /* 4K, -1 = none (non-port boundary = PEC) */
    const int32_t *face_perm;      /* 4K*Nfp neighbour face-node match, rhs.rs:546-566 */
    const double *mass;            /* Np*Np reference mass matrix (dg_basis.rs:95), or NULL;
                                      needed only by the energy entry points */
    const double *dt_scale;        /* K per-element multiplier of the LSERK4 step, or NULL (= 1):
                                      a batch of independent instances in one operator, each
                                      stepping with its own dt (no reference counterpart) */
} dgtd_op_desc;

/* Contraction engine of the stage / RHS / Krylov-matvec kernels.  A new op
 * uses TF32X3 (every order).  The two FP32 engines differ only in the
 * elements per CTA tile (the same arithmetic, so the same results to the
 * bit); batch autotuning picks per order group.
 * (Split-BF16 products were measured at 1-3e-5 relative error per RHS at
 * N = 4, above the 1e-5 bar, and are not offered.) */
typedef enum {
    DGTD_ENGINE_FP32 = 0,      /* FP32 FMA on the CUDA cores, orders 1-5 */
    DGTD_ENGINE_TF32X3 = 1,    /* 3xTF32 split products on tcgen05 tensor cores, FP32 accumulate, orders 1-5 */
    DGTD_ENGINE_FP32_SMALL_TILES = 2  /* DGTD_ENGINE_FP32 with half as many elements per tile */
} dgtd_engine;

/* GpuOperator::new (gpu/operator.rs:207). Uploads the operator once. */
int dgtd_op_create(dgtd_ctx *ctx, const dgtd_op_desc *desc, dgtd_op **out);
/* Releases the op (GpuOperator is dropped in the reference). */
int dgtd_op_destroy(dgtd_op *op);
/* GpuOperator::n_dof (gpu/operator.rs:430): 6*Np*K. */
int dgtd_op_n_dof(const dgtd_op *op, int64_t *n_dof);
/* Select the contraction engine; fails with DGTD_ERR_UNSUPPORTED if this
 * order has no kernel for it.  No counterpart in the reference, which has one
 * OpenCL kernel. */
int dgtd_op_set_engine(dgtd_op *op, int engine);
int dgtd_op_get_engine(const dgtd_op *op, int *engine);
/* Synchronises the op's stream and returns DGTD_ERR_TIMEOUT if a tensor-core
 * kernel of this op gave up one of its bounded waits since the last check
 * (then clears the flag).  The entry points that synchronise check the flag
 * themselves; this is for work queued without a synchronisation
 * (dgtd_run_lserk, dgtd_lserk_stage, dgtd_run_lserk_static).  No counterpart
 * in the reference, whose OpenCL kernels have no bounded waits. */
int dgtd_op_check_error(dgtd_op *op);

/* GpuOperator::apply (gpu/operator.rs:513): dy = A*y, host f32 buffers of
 * n_dof, AoS layout. */
int dgtd_apply(dgtd_op *op, const float *y, float *dy);

/* Drive of a transient, session.rs:107-114 (Drive::{Free,Point,Vector}). */
typedef enum { DGTD_DRIVE_FREE = 0, DGTD_DRIVE_POINT = 1, DGTD_DRIVE_VECTOR = 2 } dgtd_drive;

/* GpuOperator::transient (gpu/operator.rs:906): `steps` frames of `dt`, each
 * `substeps` LSERK4 steps of dt/substeps, the source b*g held per substep
 * with g = g_samples[k*substeps + j] (steps*substeps samples; NULL for a
 * free run).  src_dof is the point DOF (DRIVE_POINT), src_vec the n_dof
 * pattern (DRIVE_VECTOR).  With record != 0, `out` receives the trajectory
 * [(steps+1)*n_dof] (row 0 = y0); else the final state [n_dof]. */
int dgtd_transient(dgtd_op *op, const float *y0, float dt, int64_t steps, int64_t substeps,
                   int drive, int64_t src_dof, const double *src_vec, const float *g_samples,
                   int record, float *out);

/* As dgtd_transient, but recording only the DOFs `probes[n_probes]` per frame
 * into out[(steps+1)*n_probes] and the final state into y_final[n_dof]
 * (either may be NULL).  The session's Record::Dofs (session.rs:117-124). */
int dgtd_transient_probes(dgtd_op *op, const float *y0, float dt, int64_t steps,
                          int64_t substeps, int drive, int64_t src_dof, const double *src_vec,
                          const float *g_samples, const int64_t *probes, int64_t n_probes,
                          float *out, float *y_final);

/* As dgtd_transient, recording per frame n_fun linear functionals of the state
 * on the device, F_q(y) = sum_{k in [fun_ptr[q], fun_ptr[q+1])} fun_w[k] * y[fun_idx[k]]
 * (fun_idx: AoS DOF indices), accumulated in f64, into out[(steps+1)*n_fun];
 * the final state into y_final[n_dof] (may be NULL).  Port modal amplitudes
 * (rhs.rs:1211-1242 as dgtd_host_port_modal_weights) per step without a host
 * trajectory; the reference computes them on the host from a recorded
 * trajectory (session.rs:1041-1054). */
int dgtd_transient_functionals(dgtd_op *op, const float *y0, float dt, int64_t steps,
                               int64_t substeps, int drive, int64_t src_dof, const double *src_vec,
                               const float *g_samples, int64_t n_fun, const int64_t *fun_ptr,
                               const int64_t *fun_idx, const double *fun_w, double *out,
                               float *y_final);

/* Linear functionals of the resident state recorded on the device, for
 * drivers that step the state themselves (ETD tries, stage-level LSERK4).
 * dgtd_op_set_functionals stores n_fun functionals (fun_ptr / fun_idx /
 * fun_w as for dgtd_transient_functionals) and room for max_rows rows;
 * dgtd_record_functionals writes the functionals of the current state into
 * row `row` (stream-ordered, no host synchronisation); dgtd_functional_series
 * copies rows [0, n_rows) to out[n_rows*n_fun] and synchronises.  The
 * reference evaluates port amplitudes on the host from recorded trajectories
 * (session.rs:1041-1054). */
int dgtd_op_set_functionals(dgtd_op *op, int64_t n_fun, const int64_t *fun_ptr, const int64_t *fun_idx,
                            const double *fun_w, int64_t max_rows);
int dgtd_record_functionals(dgtd_op *op, int64_t row);
int dgtd_functional_series(dgtd_op *op, int64_t n_rows, double *out);

/* ---- stage-level stepping for drivers that act between stages
 * (a partitioned run's halo exchange).  One fused LSERK4 stage (0..4) of h on
 * the resident state (explicit.rs:122-133); stage 0 restarts the residual
 * register (a_0 = 0), stage 4 does not write it.  No reference counterpart:
 * the reference steps whole LSERK4 steps only (gpu/operator.rs:906). */
int dgtd_lserk_stage(dgtd_op *op, float h, int32_t stage, int drive, int64_t src_dof, float g);
/* dgtd_lserk_stage on the elements [e_begin, e_end) only, for a partitioned
 * run that overlaps its halo exchange with the elements that do not need the
 * halo: e_begin a multiple of the op's tensor-core tile (20 elements at
 * orders 1-4, 8 at order 5), e_end a multiple of it or n_elem.  flip != 0 makes the stage's output the current state (the
 * last range of a stage); the ranges of one stage read the same input.  No
 * counterpart in the reference. */
int dgtd_lserk_stage_range(dgtd_op *op, float h, int32_t stage, int64_t e_begin, int64_t e_end, int32_t flip,
                           int drive, int64_t src_dof, float g);
/* Copy element blocks (6*Np f32 each, element-major SoA) of the resident
 * state to / from a device buffer: buf[j*6*Np + r] <-> element d_elems[j].
 * d_elems and d_buf are device pointers.  No counterpart in the reference: the
 * halo exchange of a partitioned (multi-GPU) run. */
int dgtd_state_gather_elements(dgtd_op *op, const int64_t *d_elems, int64_t n, float *d_buf);
int dgtd_state_scatter_elements(dgtd_op *op, const int64_t *d_elems, int64_t n, const float *d_buf);
/* The same for any f32 device vector in the state layout (a Krylov basis
 * vector), d_vec a device pointer of at least the state's length. */
int dgtd_vec_gather_elements(dgtd_op *op, const float *d_vec, const int64_t *d_elems, int64_t n, float *d_buf);
int dgtd_vec_scatter_elements(dgtd_op *op, float *d_vec, const int64_t *d_elems, int64_t n, const float *d_buf);

/* ---- partitioned Krylov / ETD (one part of an element partition per rank).
 * The part's operator holds its n_owned owned elements first, then its halo
 * elements.  With the hooks set, every Arnoldi process of the op (dgtd_expmv,
 * dgtd_etd_step*, dgtd_etd_try) reduces its dot products and norms over the
 * owned elements only and calls, on the op's stream order:
 *   halo(user, d_vec)              before each matvec: refresh the halo blocks
 *                                  of the f32 vector d_vec from the peers;
 *   sum(user, d_partials, count)   after each partial-sum kernel: replace the
 *                                  count f64 values at d_partials by their sum
 *                                  over all parts (an allreduce);
 * so that every part forms the same Hessenberg matrix, estimate and step
 * decision.  A hook returns 0, or a nonzero value that the entry point returns
 * as DGTD_ERR_CUDA.  With hooks set, a point drive may name src_dof = -1 (the
 * source lies on another part).  n_owned = 0 and null hooks restore the
 * unpartitioned op.  Requires the f32 Krylov basis and n_owned*6*Np a
 * multiple of 4 (the sweeps read 16-byte vectors).  The reference has no
 * partitioned path; its Arnoldi is propagator.rs:186-326. */
typedef int (*dgtd_halo_hook)(void *user, float *d_vec);
typedef int (*dgtd_sum_hook)(void *user, double *d_partials, int64_t count);
int dgtd_op_set_partition(dgtd_op *op, int64_t n_owned, dgtd_halo_hook halo, dgtd_sum_hook sum, void *user);

/* ---- FP64 path ---------------------------------------------------------
 * The same RHS and LSERK4 stage in f64 on the CUDA cores (f64 operators,
 * element records and state): the arithmetic of the reference's CPU path
 * (rhs.rs, explicit.rs) on the device, for FP64 runs and as the reference
 * solution at sizes the CPU cannot reach.  Host AoS f64 buffers.
 * MaxwellOperator::apply (rhs.rs:1246) in f64: */
int dgtd_apply_f64(dgtd_op *op, const double *y, double *dy);
/* dgtd_transient in f64 (LserkWorkspace::step_into, explicit.rs:100-135, driven
 * as session.rs:107-114): `steps` frames of `dt`, each `substeps` steps,
 * g_samples[steps*substeps] held per substep; with record != 0 `out` receives
 * [(steps+1)*n_dof], else the final state. */
int dgtd_transient_f64(dgtd_op *op, const double *y0, double dt, int64_t steps, int64_t substeps,
                       int drive, int64_t src_dof, const double *src_vec, const double *g_samples,
                       int record, double *out);
/* As dgtd_transient_f64 with the waveform sampled at the five LSERK4 stage
 * times: g_stages[5*q + s] = g(t_q + c_s h), q the substep index, c the stage
 * abscissae of the Carpenter-Kennedy (1994) scheme: c_0 = 0, w_0 = 1,
 * c_{s+1} = c_s + b_s w_s, w_{s+1} = a_{s+1} w_s + 1 (the time y_{s+1} reaches
 * for y' = 1).  No counterpart in the reference (which holds g over a step,
 * first order in h): the fourth-order treatment of a time-dependent source. */
int dgtd_transient_f64_stages(dgtd_op *op, const double *y0, double dt, int64_t steps, int64_t substeps,
                              int drive, int64_t src_dof, const double *src_vec, const double *g_stages,
                              int record, double *out);

/* ---- KCL adaptive transient (gpu/operator.rs:823-893, session.rs:130-187)
 * The KCL RK4(3)5[2R+]C embedded pair with the PI step-size controller, the
 * controller running on the device: attempts are queued in batches and the
 * host reads one status word per batch instead of the error norm of every
 * substep.  g_frames[steps] holds the waveform per output frame (held across
 * the frame's substeps); NULL for a free run. */
typedef struct dgtd_kcl_controller {
    double atol, rtol, safety, growth_limit, shrink_limit, pi_alpha, pi_beta, min_step_factor;
} dgtd_kcl_controller;
typedef struct dgtd_kcl_stats {
    int64_t accepted, rejected;
    float h_min, h_max; /* step sizes in operator time, as the reference logs them */
} dgtd_kcl_stats;
/* One KCL RK4(3)5[2R+]C step of h from the AoS state y (KclWorkspace::step_into,
 * explicit_adaptive.rs:84-152; TdSession::step_adaptive, session.rs:499):
 * y_out = the fourth-order solution, err = the embedded-error vector. */
int dgtd_kcl_step(dgtd_op *op, const double *y, double h, double *y_out, double *err);
/* Controller::default (session.rs:145-158, constants.rs:260-292). */
void dgtd_kcl_controller_default(dgtd_kcl_controller *ctl);
/* With record != 0, out[(steps+1)*n_dof] receives the trajectory (row 0 = y0);
 * else out[n_dof] the final state.  DGTD_ERR_COLLAPSE when the step falls
 * below min_step_factor*dt (the reference's "step size collapsed" error). */
int dgtd_transient_kcl(dgtd_op *op, const float *y0, float dt, int64_t steps, int drive,
                       int64_t src_dof, const double *src_vec, const float *g_frames,
                       const dgtd_kcl_controller *ctl, int record, float *out, dgtd_kcl_stats *stats);
/* As dgtd_transient_kcl, recording per frame the linear functionals of
 * dgtd_transient_functionals into out[(steps+1)*n_fun] (f64) and the final
 * state into y_final (may be NULL). */
int dgtd_transient_kcl_functionals(dgtd_op *op, const float *y0, float dt, int64_t steps, int drive,
                                   int64_t src_dof, const double *src_vec, const float *g_frames,
                                   const dgtd_kcl_controller *ctl, int64_t n_fun,
                                   const int64_t *fun_ptr, const int64_t *fun_idx,
                                   const double *fun_w, double *out, float *y_final,
                                   dgtd_kcl_stats *stats);
/* The accepted substeps of the op's last adaptive run, in order: h[i] (operator
 * time) and the output frame frame[i] it advanced (whose waveform value it
 * held).  Up to `cap` entries are written; *n_total receives the run's accepted
 * count (the device logs the first 65,536).  No counterpart in the reference:
 * it lets a caller replay the run's exact step sequence, e.g. on a CPU path. */
int dgtd_kcl_accepted_steps(dgtd_op *op, float *h, int32_t *frame, int64_t cap, int64_t *n_total);

/* GpuOperator::expmv (gpu/operator.rs:1175): exp(t*A)*v by Arnoldi with CGS2
 * on the device, sub-stepped into chunks of <= 12 (KRYLOV_CHUNK).  The basis
 * is f32 with the matvec on the op's engine and every dot product, norm and
 * the Hessenberg exponential in f64; after dgtd_op_set_krylov_precision(op,
 * 64) the basis and the matvec are f64 (the FP64 path).
 * With tol > 0 each chunk also stops on the a-posteriori estimate
 * h_{j+1,j}*|exp(tH)_{d-1,0}| < tol (propagator.rs:278-294); tol = 0 is the
 * reference GPU's fixed-dimension behaviour.  `dim_used` (may be NULL)
 * receives the summed Krylov dimension. */
int dgtd_expmv(dgtd_op *op, const double *v, double t, int32_t m, double tol, double *out,
               int32_t *dim_used);

/* GpuOperator::etd_step (gpu/operator.rs:1267): exp(hA)y + h*phi1(hA)*b by the
 * augmented Arnoldi, the augmented scalar kept on the device. */
int dgtd_etd_step(dgtd_op *op, const double *y, const double *b, double h, int32_t m,
                  double tol, double *out, int32_t *dim_used);
/* As dgtd_etd_step with tol > 0, also returning the a-posteriori Krylov error
 * estimate h_{d+1,d}*|exp(tH)_{d-1,0}| (propagator.rs:278-294, relative to |y|)
 * summed over the KRYLOV_CHUNK sub-steps, each of the k sub-steps stopping at
 * tol/k; the estimate is formed at the final dimension too, so `est` > tol
 * reports a step whose space was too small.  A sub-step that misses tol/k ends
 * the step: the later sub-steps are skipped and `est` is that sub-step's
 * estimate times k (> tol), so a rejected step costs one sub-step.  The
 * accept/reject test of an adaptive or learned step controller. */
int dgtd_etd_step_est(dgtd_op *op, const double *y, const double *b, double h, int32_t m, double tol,
                      double *out, int32_t *dim_used, double *est);
/* The ETD step with a time-varying source b*g(t0 + tau), g a polynomial over
 * the step: g(t0 + tau) = sum_{k < n_coef} coef[k] tau^k (1 <= n_coef <= 8).
 * Computes exp(hA)y + sum_k h^k phi_k(hA) w_k through the exponential of the
 * (n + n_coef)-augmented matrix [[A, W], [0, J]] (J the nilpotent shift; the
 * reference's etd_step, propagator.rs:338-373, is n_coef = 1, coef = {1}).
 * No counterpart in the reference, which holds the source over the step.  With
 * tol > 0 the sub-steps stop at tol/k and `est` (may be NULL) receives the
 * summed estimate, as dgtd_etd_step_est. */
int dgtd_etd_step_poly(dgtd_op *op, const double *y, const double *b, int32_t n_coef, const double *coef,
                       double h, int32_t m, double tol, double *out, int32_t *dim_used, double *est);
/* Krylov precision of dgtd_expmv / dgtd_etd_step*: 32 (f32 basis, the default)
 * or 64 (f64 basis and FP64 matvec).  No counterpart in the reference (f64
 * basis with an f32 matvec). */
int dgtd_op_set_krylov_precision(dgtd_op *op, int bits);
/* An ETD step on the resident state (f32 basis, the op's engine): the
 * candidate exp(hA)y + sum_k h^k phi_k(hA) w_k, with the source of `drive`
 * (DRIVE_POINT at src_dof, DRIVE_VECTOR with dgtd_set_source_vector's pattern,
 * DRIVE_FREE: coef ignored) times the polynomial coef[n_coef] as in
 * dgtd_etd_step_poly, is written to the op's second state buffer; `dim_used`
 * and `est` (tol > 0; may be NULL) as dgtd_etd_step_est.  dgtd_etd_commit
 * makes the candidate the state (an accepted step, est <= tol); another
 * dgtd_etd_try replaces it (a rejected one, whose candidate is not a valid
 * state: its later sub-steps were skipped).  No counterpart in the reference, whose
 * etd_step copies the state to and from the host every step. */
int dgtd_etd_try(dgtd_op *op, double h, int32_t m, double tol, int32_t n_coef, const double *coef, int drive,
                 int64_t src_dof, int32_t *dim_used, double *est);
int dgtd_etd_commit(dgtd_op *op);

/* ---- device-resident state (no host copies) ---------------------------
 * The op owns a resident f32 state (the reference's device `y` buffer, which
 * GpuOperator keeps private: these calls have no counterpart there and serve
 * callers that keep the state on the device between calls). */
int dgtd_state_upload(dgtd_op *op, const float *y);        /* host AoS -> device state */
int dgtd_state_download(dgtd_op *op, float *y);            /* device state -> host AoS */
int dgtd_state_load_device(dgtd_op *op, const float *d_y); /* device AoS pointer -> state */
int dgtd_state_store_device(dgtd_op *op, float *d_y);      /* state -> device AoS pointer */
/* `steps` LSERK4 steps of `h` on the resident state (the stepping loop of
 * GpuOperator::transient, gpu/operator.rs:906); drive as dgtd_transient with
 * g_samples on the HOST (steps entries, NULL for free). */
int dgtd_run_lserk(dgtd_op *op, float h, int64_t steps, int drive, int64_t src_dof,
                   const float *g_samples);
/* dgtd_run_lserk with the waveform per stage: g_stages[5*k + s] = g(t_k + c_s h)
 * at the LSERK4 stage abscissae c_s (see dgtd_transient_f64_stages); the
 * fourth-order treatment of a time-dependent source (no reference counterpart). */
int dgtd_run_lserk_stages(dgtd_op *op, float h, int64_t steps, int drive, int64_t src_dof,
                          const float *g_stages);
/* Upload the DRIVE_VECTOR pattern (Drive::Vector, session.rs:107-114) used by
 * dgtd_run_lserk. */
int dgtd_set_source_vector(dgtd_op *op, const double *src_vec);
/* dy = A*y on device AoS pointers (f32): GpuOperator::apply (gpu/operator.rs:513)
 * without the host copies. */
int dgtd_apply_device(dgtd_op *op, const float *d_y, float *d_dy);

/* `steps` free LSERK4 steps of `h` from the device AoS state d_y_in into
 * d_y_out (both n_dof floats, may alias), allocating nothing.  No counterpart
 * in the reference: it serves callers that cannot let a library call
 * cudaMalloc (hosts whose framework owns the device memory budget).  The
 * scratch -- two SoA state buffers and the residual register -- is a
 * file-scope device array of 3 x 2,097,152 floats (24 MiB) that every GPU
 * loading the library holds until exit.  The kernels work on whole tiles of
 * 20 elements (8 at order 5), so the limit applies to n_elem rounded up to a
 * multiple of the tile, times 6*Np: an op above it is rejected with DGTD_ERR_BAD_ARG.  The first
 * call on a device takes the array's device address (cudaGetSymbolAddress),
 * so make that first call before any stream capture.  All calls share the one
 * array: calls whose work overlaps on the GPU (other streams, other threads)
 * race.  The work is queued on the op's stream and the call does not
 * synchronise: synchronise before reading d_y_out, then call
 * dgtd_op_check_error, which reports (DGTD_ERR_TIMEOUT) a tensor-core kernel
 * that gave up one of its bounded waits during the run. */
int dgtd_run_lserk_static(dgtd_op *op, const float *d_y_in, float *d_y_out, float h, int64_t steps);

/* ---- session helpers --------------------------------------------------
 * TdSession::cfl_dt (session.rs:514-569) on the device: rho(A) by 40 power
 * iterations from the reference's deterministic start vector (splitmix64 +
 * Box-Muller, seed 0, session.rs:415-431), then the LSERK4 stability bracket
 * z in [3, 15] widened as needed, 7 bisections of 64-step probes from the
 * dominant vector (growth rate <= 1e-3 per step, norm <= 10x).  Outputs the
 * stable step h = 0.8*z/rho (operator time), rho and z; any may be NULL. */
int dgtd_cfl_dt(dgtd_op *op, double *h, double *rho, double *z);
/* Spectral radius only: `iters` power iterations (session.rs:522-534). */
int dgtd_power_rho(dgtd_op *op, int32_t iters, double *rho);
/* field_energy (rhs.rs:1509-1544): 1/2 sum_e |det J_e| sum_c w_c f_c^T M f_c,
 * w = eps (E) or mu (H), accumulated in f64 on the device.  `y` is a host AoS
 * f64 state; dgtd_state_energy uses the resident f32 state.  Needs desc.mass. */
int dgtd_field_energy(dgtd_op *op, const double *y, double *energy);
int dgtd_state_energy(dgtd_op *op, double *energy);

/* ---- statistics -------------------------------------------------------- */
/* Kernel launches issued by this op since creation / the last reset (no
 * counterpart in the reference). */
int dgtd_op_launch_count(const dgtd_op *op, int64_t *count);
int dgtd_op_reset_launch_count(dgtd_op *op);

/* ---- the MLP of the learned ETD step controller (no reference counterpart)
 * n_in -> n_hidden -> n_hidden -> n_out, tanh hidden layers, linear output,
 * mean-squared-error loss, Adam; forward, backward and Adam run as device
 * kernels.  Parameters (f32) in the order W1[H][n_in], b1[H], W2[H][H], b2[H],
 * W3[n_out][H], b3[n_out]; weights start Glorot-uniform from `seed`. */
typedef struct dgtd_mlp dgtd_mlp;
int dgtd_mlp_create(dgtd_ctx *ctx, int32_t n_in, int32_t n_hidden, int32_t n_out, uint64_t seed,
                    dgtd_mlp **out);
void dgtd_mlp_destroy(dgtd_mlp *mlp);
int dgtd_mlp_n_params(const dgtd_mlp *mlp, int64_t *n_params);
int dgtd_mlp_get_params(dgtd_mlp *mlp, float *params);
/* Also resets the Adam moments. */
int dgtd_mlp_set_params(dgtd_mlp *mlp, const float *params);
/* y[batch*n_out] = f(x[batch*n_in]); batch 1..65535, host arrays. */
int dgtd_mlp_forward(dgtd_mlp *mlp, const float *x, int64_t batch, float *y);
/* The gradient of L = mean_b sum_o (f(x_b)_o - t_bo)^2 w.r.t. the parameters
 * (grad[n_params]) and L, without updating. */
int dgtd_mlp_gradient(dgtd_mlp *mlp, const float *x, const float *t, int64_t batch, float *grad,
                      float *loss);
/* `epochs` full-batch Adam steps (beta1 0.9, beta2 0.999, eps 1e-8) at rate lr;
 * losses[epochs] (may be NULL) receives L before each step. */
int dgtd_mlp_train(dgtd_mlp *mlp, const float *x, const float *t, int64_t batch, int32_t epochs, float lr,
                   float *losses);

/* ---- test hooks --------------------------------------------------------
 * Dense exp(A) of a d x d row-major matrix (d <= 64) by the device kernel the
 * Krylov finisher uses (Taylor-18 + scaling and squaring, propagator.rs:69-114). */
int dgtd_debug_expm(dgtd_ctx *ctx, const double *a, int32_t d, double *out);
/* One-CTA tcgen05 GEMM C[M x n] = A[M x k] * B[n x k]^T (row-major f32)
 * through the operand layout, descriptors and TMEM path of the tensor-core RHS
 * kernel.  flags bit 0: 3xTF32 split products (else one tf32 product); bit 1:
 * A operand in TMEM (else shared memory); bit 2: M = 64 (else 128); bit 3
 * (with bit 2): accumulator and TMEM A operand at lane offset o = 16 (else 0).
 * c gets the 128 TMEM lanes x n: at M = 64 row 16 q + r (r < 16) is lane
 * 32 q + o + r.
 * n <= 256 a multiple of 16 (of 8 at M = 64), 8 <= k <= 64 (k % 8 == 0). */
int dgtd_debug_tc_gemm(dgtd_ctx *ctx, const float *a, const float *b, float *c, int32_t n, int32_t k,
                       int32_t flags);
/* The bounded wait of the tensor-core kernels, run by one thread on an
 * mbarrier that nothing arrives on: it gives up after max_polls polls
 * (1 <= max_polls <= 2^19, the kernels' own limit; a failed poll suspends
 * about 4 us, so the kernels' limit is about 2 s), and the call returns
 * DGTD_ERR_TIMEOUT through the same device flag a stage kernel raises, with
 * the time waited in *waited_s.  Nothing faults; the context stays usable. */
int dgtd_debug_wait_timeout(dgtd_ctx *ctx, int64_t max_polls, double *waited_s);
/* Per-phase cycle counters of the tensor-core RHS kernel (8 u64 in device
 * memory, accumulated by thread 0 of every CTA); recorded only by builds
 * compiled with -DDGTD_TC_PHASE_TIMERS, ignored otherwise.  NULL detaches. */
int dgtd_debug_set_phase_clock(dgtd_op *op, void *d_counters);

#ifdef __cplusplus
}
#endif

#endif /* DGTD_H */
