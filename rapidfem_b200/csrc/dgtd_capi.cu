// dgtd_capi.cu -- the C ABI of include/dgtd.h: context, device operator,
// apply / LSERK4 transient / Krylov expmv / ETD step on the B200.
//
// Replaces gpu/mod.rs (GpuContext) and gpu/operator.rs (GpuOperator) of
// crates/rapidfem-td.  The operator arrays are uploaded once
// (gpu/operator.rs:222-292) into the element-major SoA layout described in
// dgtd_common.cuh; every run keeps the state resident and converts to the
// reference's AoS layout only at the boundary.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dgtd.h"
#include "dgtd_common.cuh"
#include "host/errors.h"
#include "krylov.cuh"
#include "rhs_fp32.cuh"
#include "rhs_tc.cuh"
#include "tc_selftest.cuh"
#include "kcl.cuh"
#include "mlp.cuh"

// ------------------------------------------------------------------ errors

namespace dgtd {
static thread_local std::string g_last_error;
int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
}  // namespace dgtd

using dgtd::set_error;

#define CUDA_TRY(expr)                                                                      \
  do {                                                                                      \
    cudaError_t err__ = (expr);                                                             \
    if (err__ != cudaSuccess)                                                               \
      return set_error(err__ == cudaErrorMemoryAllocation ? DGTD_ERR_OOM : DGTD_ERR_CUDA,   \
                       std::string(#expr) + ": " + cudaGetErrorString(err__));              \
  } while (0)

#define DGTD_TRY(expr)            \
  do {                            \
    int st__ = (expr);            \
    if (st__ != DGTD_OK) return st__; \
  } while (0)

extern "C" int dgtd_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return DGTD_ERR_BAD_ARG;
  std::snprintf(buf, len, "%s", dgtd::g_last_error.c_str());
  return DGTD_OK;
}

extern "C" const char* dgtd_version(void) { return "rapidfem_b200 0.1.0 sm_100a"; }

// ------------------------------------------------------------------ context

struct dgtd_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  std::string name;
};

extern "C" int dgtd_ctx_create(int device, dgtd_ctx** out) {
  if (!out) return set_error(DGTD_ERR_BAD_ARG, "ctx_create: null out");
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return set_error(DGTD_ERR_NO_DEVICE, std::string("no CUDA device found") +
                                             (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : ""));
  if (device < 0 || device >= count) return set_error(DGTD_ERR_BAD_ARG, "ctx_create: device index out of range");
  CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return set_error(DGTD_ERR_NO_DEVICE, std::string("device ") + prop.name + " is not sm_100 (built for sm_100a only)");
  auto* c = new dgtd_ctx;
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  c->name = prop.name;
  cudaError_t se = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  if (se != cudaSuccess) {
    delete c;
    return set_error(DGTD_ERR_CUDA, std::string("stream create: ") + cudaGetErrorString(se));
  }
  c->stream = c->own;
  *out = c;
  return DGTD_OK;
}

extern "C" int dgtd_ctx_destroy(dgtd_ctx* c) {
  if (!c) return DGTD_OK;
  cudaSetDevice(c->device);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return DGTD_OK;
}

extern "C" int dgtd_ctx_device_name(dgtd_ctx* c, char* buf, size_t len) {
  if (!c || !buf || !len) return set_error(DGTD_ERR_BAD_ARG, "ctx_device_name: bad argument");
  std::snprintf(buf, len, "%s", c->name.c_str());
  return DGTD_OK;
}

extern "C" int dgtd_ctx_set_stream(dgtd_ctx* c, void* s) {
  if (!c) return set_error(DGTD_ERR_BAD_ARG, "ctx_set_stream: null ctx");
  c->stream = s ? static_cast<cudaStream_t>(s) : c->own;
  return DGTD_OK;
}

extern "C" int dgtd_ctx_synchronize(dgtd_ctx* c) {
  if (!c) return set_error(DGTD_ERR_BAD_ARG, "ctx_synchronize: null ctx");
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return DGTD_OK;
}

// ------------------------------------------------------------------ operator

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  int alloc(size_t count) {
    if (n >= count && p) return DGTD_OK;
    free();
    if (count == 0) return DGTD_OK;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return set_error(DGTD_ERR_OOM, std::string("cudaMalloc(") + std::to_string(count * sizeof(T)) +
                                         " bytes): " + cudaGetErrorString(e));
    }
    n = count;
    return DGTD_OK;
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

struct dgtd_op {
  dgtd_ctx* ctx = nullptr;
  int device = 0;  // the destructor must not read ctx: a host may free the context first
  int order = 0, np = 0, nfp = 0;
  int64_t n_elem = 0, n_dof = 0;
  float alpha = 1.f;
  double alpha64 = 1.0;
  int engine = DGTD_ENGINE_FP32;
  int64_t launches = 0;
  // operator data
  DevBuf<float> meta, dT, liftT;
  DevBuf<uint8_t> fnodes, gtab;
  int n_gather = 0;
  // FP64 path: f64 element records and operators, f64 state (allocated on first use)
  DevBuf<double> meta64, dT64, liftT64, y64[2], p64, src_vec64;
  int cur64 = 0;
  // state
  DevBuf<float> y[2], p, src_vec, aos32;
  int cur = 0;
  bool src_vec_set = false;
  // Krylov
  DevBuf<double> partials, tmp64, vin64;
  DevBuf<float> kbasis32, kvec32[2], kb32;
  DevBuf<double> kbasis64, kvec64[2], kb64, kpoly, kout64;
  bool krylov_fp64 = false;  // host-API Krylov on the FP64 path
  DevBuf<dgtd::KrylovDev> kst;
  DevBuf<int> skip;
  // energy: reference mass matrix (f64) and |det J| per element
  DevBuf<double> mass, absdet;
  bool has_mass = false;
  // tensor-core engine: element count padded to whole tiles, pre-split operands
  int64_t n_elem_pad = 0;
  DevBuf<float> tc_bvol, tc_blift;
  DevBuf<int> err;
  unsigned long long* phase_clk = nullptr;  // instrumented builds: per-phase cycle counters
  // KCL adaptive stepping: controller, backup, embedded error, stage point, RHS, waveform
  DevBuf<dgtd::KclCtl> kcl_ctl;
  DevBuf<dgtd::KclLogEntry> kcl_log;
  int64_t kcl_log_n = 0;  // accepted substeps of the last adaptive run
  DevBuf<float> kcl_bak, kcl_e, kcl_stage, kcl_k, kcl_g;
  DevBuf<double> kcl_part;
  // functionals recorded on the resident state (dgtd_op_set_functionals)
  DevBuf<int64_t> fn_ptr, fn_idx;
  DevBuf<double> fn_w, fn_out;
  int64_t fn_n = 0, fn_rows = 0;
  // partitioned Krylov (dgtd_op_set_partition): owned elements and the hooks
  int64_t part_owned = 0;
  dgtd_halo_hook part_halo = nullptr;
  dgtd_sum_hook part_sum = nullptr;
  void* part_user = nullptr;

  cudaStream_t stream() const { return ctx->stream; }
  ~dgtd_op() {
    cudaSetDevice(device);
    meta.free(); dT.free(); liftT.free(); fnodes.free(); gtab.free();
    meta64.free(); dT64.free(); liftT64.free(); y64[0].free(); y64[1].free(); p64.free(); src_vec64.free();
    y[0].free(); y[1].free(); p.free(); src_vec.free(); aos32.free();
    partials.free(); tmp64.free(); vin64.free();
    kbasis32.free(); kvec32[0].free(); kvec32[1].free(); kb32.free();
    kbasis64.free(); kvec64[0].free(); kvec64[1].free(); kb64.free(); kpoly.free(); kout64.free();
    kst.free(); skip.free(); mass.free(); absdet.free();
    tc_bvol.free(); tc_blift.free(); err.free();
    kcl_ctl.free(); kcl_log.free(); kcl_bak.free(); kcl_e.free(); kcl_stage.free(); kcl_k.free(); kcl_g.free(); kcl_part.free();
    fn_ptr.free(); fn_idx.free(); fn_w.free(); fn_out.free();
  }
};

namespace {

using namespace dgtd;

// ---- layout conversion (AoS y[(e*Np+i)*6+c] <-> SoA y[(e*6+c)*Np+i])
// Element e occupies the same 6*Np consecutive values in both layouts, so a
// conversion permutes values inside element blocks: a CTA stages a chunk of
// kRelayoutElems elements in shared memory with coalesced loads and writes the
// permuted chunk with coalesced stores (32-bit index arithmetic, Np a
// compile-time constant).
constexpr int kRelayoutElems = 8;
template <class TI, class TO, int NP, bool TO_SOA>
__global__ void __launch_bounds__(256) k_relayout(const TI* __restrict__ src, TO* __restrict__ dst, int64_t n_elem) {
  constexpr int PER = 6 * NP, CH = kRelayoutElems * PER;
  __shared__ TI buf[CH];
  const int64_t n_chunks = (n_elem + kRelayoutElems - 1) / kRelayoutElems;
  for (int64_t ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
    const int64_t base = ch * CH;
    const int64_t left = (n_elem - ch * kRelayoutElems) * PER;
    const int len = left < CH ? (int)left : CH;
    for (int k = threadIdx.x; k < len; k += blockDim.x) buf[k] = src[base + k];
    __syncthreads();
    for (int k = threadIdx.x; k < len; k += blockDim.x) {
      const int el = k / PER, r = k - el * PER;
      int from;
      if (TO_SOA) {
        const int c = r / NP, i = r - c * NP;  // destination (c, i) <- source (i, c)
        from = el * PER + i * 6 + c;
      } else {
        const int i = r / 6, c = r - i * 6;  // destination (i, c) <- source (c, i)
        from = el * PER + c * NP + i;
      }
      dst[base + k] = (TO)buf[from];
    }
    __syncthreads();
  }
}
__global__ void k_gather_f32(const float* __restrict__ src, const int64_t* __restrict__ idx,
                             int64_t n, float* __restrict__ out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    out[k] = src[idx[k]];
}

// One block per functional: sum_k w[k] * y[idx[k]] in f64 (fixed order per
// thread and a fixed reduction tree, so the result is deterministic).
__global__ void __launch_bounds__(256) k_functionals(const float* __restrict__ y, const int64_t* __restrict__ ptr,
                                                     const int64_t* __restrict__ idx, const double* __restrict__ w,
                                                     double* __restrict__ out) {
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
    out[q] = t;
  }
}

int grid_for(int64_t n, int threads, int num_sms) {
  int64_t g = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)num_sms * 8));
}

// Length of a device state buffer: whole tensor-core tiles plus 4 floats of slack.
size_t state_len(const dgtd_op* op) { return (size_t)op->n_elem_pad * 6 * op->np + 4; }

int64_t aos_to_soa_index(int64_t dof, int np) {
  const int64_t per = 6LL * np;
  const int64_t e = dof / per;
  const int r = (int)(dof - e * per);
  const int i = r / 6, c = r - i * 6;
  return (e * 6 + c) * np + i;
}

template <class TI, class TO, bool TO_SOA>
int relayout(dgtd_op* op, const TI* src, TO* dst) {
  const int64_t n_elem = op->n_dof / (6 * op->np);
  const int64_t chunks = (n_elem + kRelayoutElems - 1) / kRelayoutElems;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(chunks, (int64_t)op->ctx->num_sms * 16));
  switch (op->np) {
    case np_of(1): k_relayout<TI, TO, np_of(1), TO_SOA><<<grid, 256, 0, op->stream()>>>(src, dst, n_elem); break;
    case np_of(2): k_relayout<TI, TO, np_of(2), TO_SOA><<<grid, 256, 0, op->stream()>>>(src, dst, n_elem); break;
    case np_of(3): k_relayout<TI, TO, np_of(3), TO_SOA><<<grid, 256, 0, op->stream()>>>(src, dst, n_elem); break;
    case np_of(4): k_relayout<TI, TO, np_of(4), TO_SOA><<<grid, 256, 0, op->stream()>>>(src, dst, n_elem); break;
    case np_of(5): k_relayout<TI, TO, np_of(5), TO_SOA><<<grid, 256, 0, op->stream()>>>(src, dst, n_elem); break;
    default: return set_error(DGTD_ERR_UNSUPPORTED, "layout conversion: unsupported order");
  }
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}
template <class TI, class TO>
int to_soa(dgtd_op* op, const TI* aos, TO* soa) {
  return relayout<TI, TO, true>(op, aos, soa);
}
template <class TI, class TO>
int to_aos(dgtd_op* op, const TI* soa, TO* aos) {
  return relayout<TI, TO, false>(op, soa, aos);
}

// ---- RHS kernel dispatch
template <int N, int MODE, int TD>
int launch_rhs_n(dgtd_op* op, const RhsParams& P) {
  using C = Fp32Cfg<N, float, TD>;
  static int blocks_per_sm[8] = {0};
  auto kern = rhs_fp32_kernel<N, MODE, TD>;
  int& bps = blocks_per_sm[op->ctx->device & 7];
  if (bps == 0) {
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, C::THREADS, C::SMEM));
    if (bps < 1) return set_error(DGTD_ERR_CUDA, "rhs kernel does not fit on an SM");
  }
  OpTables T{op->dT.p, op->liftT.p, op->fnodes.p, op->gtab.p, op->n_gather};
  const int64_t tiles = (P.n_elem - P.e_begin + C::E - 1) / C::E;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)op->ctx->num_sms * bps);
  kern<<<grid, C::THREADS, C::SMEM, op->stream()>>>(P, T);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

template <int N, int MODE>
int launch_rhs64_n(dgtd_op* op, const RhsParamsT<double>& P) {
  using C = Fp32Cfg<N, double>;
  static int blocks_per_sm[8] = {0};
  auto kern = rhs_fp64_kernel<N, MODE>;
  int& bps = blocks_per_sm[op->ctx->device & 7];
  if (bps == 0) {
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, C::THREADS, C::SMEM));
    if (bps < 1) return set_error(DGTD_ERR_CUDA, "fp64 rhs kernel does not fit on an SM");
  }
  OpTablesT<double> T{op->dT64.p, op->liftT64.p, op->fnodes.p, op->gtab.p, op->n_gather};
  const int64_t tiles = (P.n_elem - P.e_begin + C::E - 1) / C::E;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)op->ctx->num_sms * bps);
  kern<<<grid, C::THREADS, C::SMEM, op->stream()>>>(P, T);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

// The FP64 path (CUDA cores, f64 throughout), orders 1-5.
template <int MODE>
int launch_rhs64(dgtd_op* op, const RhsParamsT<double>& P) {
  switch (op->order) {
    case 1: return launch_rhs64_n<1, MODE>(op, P);
    case 2: return launch_rhs64_n<2, MODE>(op, P);
    case 3: return launch_rhs64_n<3, MODE>(op, P);
    case 4: return launch_rhs64_n<4, MODE>(op, P);
    case 5: return launch_rhs64_n<5, MODE>(op, P);
    default: return set_error(DGTD_ERR_UNSUPPORTED, "order outside 1..5");
  }
}

template <int N, int MODE>
int launch_rhs_tc_n(dgtd_op* op, const RhsParams& P) {
  using C = TcCfg<N>;
  static bool attr[8] = {false};
  auto kern = rhs_tc_kernel<N, MODE>;
  if (!attr[op->ctx->device & 7]) {
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    attr[op->ctx->device & 7] = true;
  }
  TcTables T{op->tc_bvol.p, op->tc_blift.p, op->fnodes.p, op->gtab.p, op->n_gather};
  // whole tiles: a range ending at the op's last element runs to the padded end
  const int64_t end = P.n_elem >= op->n_elem ? op->n_elem_pad : P.n_elem;
  const int64_t tiles = (end - P.e_begin) / C::E;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)op->ctx->num_sms);
  kern<<<grid, kTcThreadsAll, C::SMEM, op->stream()>>>(P, T, tiles, op->err.p);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

template <int MODE>
int launch_rhs(dgtd_op* op, const RhsParams& P) {
  if constexpr (MODE == kModeApply || MODE == kModeLserk || MODE == kModeKrylov || MODE == kModeKcl) {
    if (op->engine == DGTD_ENGINE_TF32X3) {
      switch (op->order) {
        case 1: return launch_rhs_tc_n<1, MODE>(op, P);
        case 2: return launch_rhs_tc_n<2, MODE>(op, P);
        case 3: return launch_rhs_tc_n<3, MODE>(op, P);
        case 4: return launch_rhs_tc_n<4, MODE>(op, P);
        case 5: return launch_rhs_tc_n<5, MODE>(op, P);
        default: return set_error(DGTD_ERR_UNSUPPORTED, "order outside 1..5");
      }
    }
  }
  if (op->engine == DGTD_ENGINE_FP32_SMALL_TILES) {
    switch (op->order) {
      case 1: return launch_rhs_n<1, MODE, 2>(op, P);
      case 2: return launch_rhs_n<2, MODE, 2>(op, P);
      case 3: return launch_rhs_n<3, MODE, 2>(op, P);
      case 4: return launch_rhs_n<4, MODE, 2>(op, P);
      case 5: return launch_rhs_n<5, MODE, 2>(op, P);
      default: return set_error(DGTD_ERR_UNSUPPORTED, "order outside 1..5");
    }
  }
  switch (op->order) {
    case 1: return launch_rhs_n<1, MODE, 1>(op, P);
    case 2: return launch_rhs_n<2, MODE, 1>(op, P);
    case 3: return launch_rhs_n<3, MODE, 1>(op, P);
    case 4: return launch_rhs_n<4, MODE, 1>(op, P);
    case 5: return launch_rhs_n<5, MODE, 1>(op, P);
    default: return set_error(DGTD_ERR_UNSUPPORTED, "order outside 1..5");
  }
}

RhsParams base_params(dgtd_op* op) {
  RhsParams P;
  std::memset(&P, 0, sizeof(P));
  P.meta = op->meta.p;
  P.n_elem = op->n_elem;
  P.src_idx = -1;
  P.alpha = op->alpha;
  P.phase_clk = op->phase_clk;
  return P;
}

RhsParamsT<double> base_params64(dgtd_op* op) {
  RhsParamsT<double> P;
  std::memset(&P, 0, sizeof(P));
  P.meta = op->meta64.p;
  P.n_elem = op->n_elem;
  P.src_idx = -1;
  P.alpha = op->alpha64;
  return P;
}

const double kLserkA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                           -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kLserkB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                           1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                           2277821191437.0 / 14882151754819.0};

// One LSERK4 step of h on the resident state (explicit.rs:100-135; the
// residual register restarts at zero each step because a_0 = 0).
// g5: the waveform per stage (null: g held over the step, as the reference's
// Source::add_to, explicit.rs:44-56).
int lserk_step(dgtd_op* op, float h, int64_t src_idx, float g, const float* src_vec, const float* g5 = nullptr) {
  for (int s = 0; s < 5; ++s) {
    RhsParams P = base_params(op);
    P.y_in = op->y[op->cur].p;
    P.out = op->y[op->cur ^ 1].p;
    P.p = op->p.p;
    P.a = (float)kLserkA[s];
    P.b = (float)kLserkB[s];
    P.dt = h;
    P.read_p = s > 0;
    P.write_p = s < 4;
    P.src_idx = src_idx;
    P.src_vec = src_vec;
    P.src_g = g5 ? g5[s] : g;
    DGTD_TRY(launch_rhs<kModeLserk>(op, P));
    op->cur ^= 1;
  }
  return DGTD_OK;
}

}  // namespace

extern "C" int dgtd_op_create(dgtd_ctx* ctx, const dgtd_op_desc* d, dgtd_op** out) {
  if (!ctx || !d || !out) return set_error(DGTD_ERR_BAD_ARG, "op_create: null argument");
  if (d->order < 1 || d->order > 5) return set_error(DGTD_ERR_UNSUPPORTED, "op_create: order must be 1..5");
  if (d->n_elem < 1) return set_error(DGTD_ERR_BAD_ARG, "op_create: n_elem must be >= 1");
  if (!d->diff_r || !d->diff_s || !d->diff_t || !d->lift || !d->face_nodes || !d->jinv || !d->inv_eps ||
      !d->inv_mu || !d->sigma_eps || !d->sigma_mu || !d->face_normal || !d->face_fscale ||
      !d->face_neighbor || !d->face_nbr_local || !d->face_port || !d->face_perm)
    return set_error(DGTD_ERR_BAD_ARG, "op_create: a descriptor array is null");
  CUDA_TRY(cudaSetDevice(ctx->device));
  const int N = d->order, np = dgtd::np_of(N), nfp = dgtd::nfp_of(N);
  const int64_t K = d->n_elem;
  // Host-side packing: element records, gather tables.
  const int64_t tile_e = dgtd::tc_tile_e(N);  // tensor-core tile of this order
  const int64_t Kpad = ((K + tile_e - 1) / tile_e) * tile_e;
  std::vector<float> meta((size_t)Kpad * dgtd::kMetaWords, 0.f);
  // the same records in f64 for the FP64 path, integer words as exact values
  std::vector<double> meta64((size_t)Kpad * dgtd::kMetaWords, 0.0);
  {
    // inert padding records: every face a PEC wall with zero normal / scale / metric
    const uint32_t pec = (uint32_t)dgtd::kPec << 8;
    const uint32_t w = pec | (pec << 16);
    const int32_t none = -1;
    for (int64_t e = K; e < Kpad; ++e) {
      float* M = &meta[(size_t)e * dgtd::kMetaWords];
      for (int f = 0; f < 4; ++f) std::memcpy(&M[37 + f], &none, 4);
      std::memcpy(&M[41], &w, 4);
      std::memcpy(&M[42], &w, 4);
      double* M64 = &meta64[(size_t)e * dgtd::kMetaWords];
      for (int f = 0; f < 4; ++f) M64[37 + f] = -1.0;
      M64[41] = (double)w;
      M64[42] = (double)w;
    }
  }
  std::map<std::vector<uint8_t>, int> table_id;
  std::vector<uint8_t> gtab;
  for (int f = 0; f < 4; ++f)
    for (int m = 0; m < nfp; ++m)
      if (d->face_nodes[f * nfp + m] < 0 || d->face_nodes[f * nfp + m] >= np)
        return set_error(DGTD_ERR_BAD_ARG, "op_create: face_nodes entry out of range");
  for (int64_t e = 0; e < K; ++e) {
    float* M = &meta[(size_t)e * dgtd::kMetaWords];
    double* M64 = &meta64[(size_t)e * dgtd::kMetaWords];
    for (int q = 0; q < 9; ++q) M64[q] = d->jinv[9 * e + q];
    for (int q = 0; q < 12; ++q) M64[9 + q] = d->face_normal[12 * e + q];
    for (int q = 0; q < 4; ++q) M64[21 + q] = d->face_fscale[4 * e + q];
    for (int c = 0; c < 3; ++c) {
      M64[25 + c] = d->inv_eps[3 * e + c];
      M64[28 + c] = d->inv_mu[3 * e + c];
      M64[31 + c] = d->sigma_eps[3 * e + c];
      M64[34 + c] = d->sigma_mu[3 * e + c];
    }
    for (int q = 0; q < 9; ++q) M[q] = (float)d->jinv[9 * e + q];
    for (int q = 0; q < 12; ++q) M[9 + q] = (float)d->face_normal[12 * e + q];
    for (int q = 0; q < 4; ++q) M[21 + q] = (float)d->face_fscale[4 * e + q];
    for (int c = 0; c < 3; ++c) {
      M[25 + c] = (float)d->inv_eps[3 * e + c];
      M[28 + c] = (float)d->inv_mu[3 * e + c];
      M[31 + c] = (float)d->sigma_eps[3 * e + c];
      M[34 + c] = (float)d->sigma_mu[3 * e + c];
    }
    uint32_t codes[4];
    for (int f = 0; f < 4; ++f) {
      const int64_t ef = 4 * e + f;
      const int nbr = d->face_neighbor[ef];
      int32_t nb_bits = nbr;
      int kind, id = 0;
      if (d->face_port[ef] >= 0) {
        kind = dgtd::kPort;
      } else if (nbr < 0) {
        kind = dgtd::kPec;
        nb_bits = -1;
      } else {
        if (nbr >= K) return set_error(DGTD_ERR_BAD_ARG, "op_create: face_neighbor out of range");
        const int fn = d->face_nbr_local[ef];
        if (fn < 0 || fn > 3) return set_error(DGTD_ERR_BAD_ARG, "op_create: face_nbr_local out of range");
        kind = dgtd::kInterior;
        std::vector<uint8_t> list(nfp);
        for (int m = 0; m < nfp; ++m) {
          const int pm = d->face_perm[ef * nfp + m];
          if (pm < 0 || pm >= nfp) return set_error(DGTD_ERR_BAD_ARG, "op_create: face_perm out of range");
          list[m] = (uint8_t)d->face_nodes[fn * nfp + pm];
        }
        auto it = table_id.find(list);
        if (it == table_id.end()) {
          if ((int)table_id.size() >= dgtd::kMaxGather)
            return set_error(DGTD_ERR_UNSUPPORTED, "op_create: more than 96 distinct face-node matchings");
          id = (int)table_id.size();
          table_id.emplace(list, id);
          gtab.insert(gtab.end(), list.begin(), list.end());
        } else {
          id = it->second;
        }
      }
      std::memcpy(&M[37 + f], &nb_bits, 4);
      M64[37 + f] = (double)nb_bits;
      codes[f] = (uint32_t)id | ((uint32_t)kind << 8);
    }
    const uint32_t w0 = codes[0] | (codes[1] << 16), w1 = codes[2] | (codes[3] << 16);
    std::memcpy(&M[41], &w0, 4);
    std::memcpy(&M[42], &w1, 4);
    M64[41] = (double)w0;
    M64[42] = (double)w1;
    M[43] = 1.0f;
    M64[43] = 1.0;
    if (d->dt_scale) {
      const double sc = d->dt_scale[e];
      if (!(std::isfinite(sc) && sc > 0.0)) return set_error(DGTD_ERR_BAD_ARG, "op_create: dt_scale must be positive");
      M[43] = (float)sc;
      M64[43] = sc;
    }
  }
  std::vector<float> dT((size_t)3 * np * np), liftT((size_t)4 * nfp * np);
  std::vector<double> dT64(dT.size()), liftT64(liftT.size());
  const double* D[3] = {d->diff_r, d->diff_s, d->diff_t};
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < np; ++i)
      for (int j = 0; j < np; ++j) {
        dT[((size_t)k * np + j) * np + i] = (float)D[k][i * np + j];
        dT64[((size_t)k * np + j) * np + i] = D[k][i * np + j];
      }
  for (int i = 0; i < np; ++i)
    for (int s = 0; s < 4 * nfp; ++s) {
      liftT[(size_t)s * np + i] = (float)d->lift[i * 4 * nfp + s];
      liftT64[(size_t)s * np + i] = d->lift[i * 4 * nfp + s];
    }
  std::vector<uint8_t> fnodes(4 * nfp);
  for (int q = 0; q < 4 * nfp; ++q) fnodes[q] = (uint8_t)d->face_nodes[q];
  if (gtab.empty()) gtab.assign(nfp, 0);

  auto* op = new dgtd_op;
  op->ctx = ctx;
  op->device = ctx->device;
  op->engine = DGTD_ENGINE_TF32X3;
  op->order = N;
  op->np = np;
  op->nfp = nfp;
  op->n_elem = K;
  op->n_dof = 6 * (int64_t)np * K;
  op->alpha = (float)d->flux_alpha;
  op->alpha64 = d->flux_alpha;
  op->n_gather = (int)table_id.size();
  op->n_elem_pad = Kpad;
  const size_t nstate = (size_t)Kpad * 6 * np + 4;
  auto fail = [&](int code) { delete op; return code; };
  int st;
  if ((st = op->meta.alloc(meta.size())) || (st = op->dT.alloc(dT.size())) || (st = op->liftT.alloc(liftT.size())) ||
      (st = op->fnodes.alloc(fnodes.size())) || (st = op->gtab.alloc(gtab.size())) ||
      (st = op->y[0].alloc(nstate)) || (st = op->y[1].alloc(nstate)) || (st = op->p.alloc(nstate)) ||
      (st = op->err.alloc(1)) || (st = op->meta64.alloc(meta64.size())) || (st = op->dT64.alloc(dT64.size())) ||
      (st = op->liftT64.alloc(liftT64.size())))
    return fail(st);
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (!e) e = cudaMemcpyAsync(op->meta.p, meta.data(), meta.size() * 4, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(op->dT.p, dT.data(), dT.size() * 4, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(op->liftT.p, liftT.data(), liftT.size() * 4, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(op->meta64.p, meta64.data(), meta64.size() * 8, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(op->dT64.p, dT64.data(), dT64.size() * 8, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(op->liftT64.p, liftT64.data(), liftT64.size() * 8, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(op->fnodes.p, fnodes.data(), fnodes.size(), cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemcpyAsync(op->gtab.p, gtab.data(), gtab.size(), cudaMemcpyHostToDevice, s);
  if (!e) e = cudaMemsetAsync(op->y[0].p, 0, op->y[0].n * 4, s);
  if (!e) e = cudaMemsetAsync(op->y[1].p, 0, op->y[1].n * 4, s);
  if (!e) e = cudaMemsetAsync(op->p.p, 0, op->p.n * 4, s);
  if (!e) e = cudaMemsetAsync(op->err.p, 0, sizeof(int), s);
  if (!e) {
    // 3xTF32 constant operands: tf32 hi/lo of D_k (rows (k,i), K = node j) and
    // LIFT (rows i, K = face node s), chunk-major K-major layout.
    auto tf32 = [](double x) {
      float f = (float)x;
      uint32_t b;
      std::memcpy(&b, &f, 4);
      if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0x1000u) & 0xffffe000u;
      std::memcpy(&f, &b, 4);
      return f;
    };
    auto build = [&](int R, int Kc, auto value, std::vector<float>& out) {
      out.assign((size_t)2 * R * Kc, 0.f);
      for (int r = 0; r < R; ++r)
        for (int k = 0; k < Kc; ++k) {
          const double v = value(r, k);
          const float h = tf32(v);
          const float l = tf32(v - (double)h);
          const size_t o = dgtd::tc::kmajor_off(r, k, R) / 4;
          out[o] = h;
          out[(size_t)R * Kc + o] = l;
        }
    };
    // LIFT K is laid out per face, each face padded to KLF = Nfp rounded up to 8,
    // so the MMAs of a face pair can start while the other pair's flux is formed.
    const int KV = dgtd::tc_r8(np), NV = dgtd::tc_nv(N), KLF = dgtd::tc_r8(nfp), KL = 4 * KLF;
    const int NL = dgtd::tc_nl(N);
    std::vector<float> bv, bl;
    build(NV, KV, [&](int r, int k) -> double {
      if (r >= 3 * np || k >= np) return 0.0;
      const int kk = r / np, i = r - kk * np;
      return D[kk][i * np + k];
    }, bv);
    // LIFT B operand: hi rows over lo rows in one 2NL-row operand (the kernel's
    // MMA of an A half forms both products at once).
    {
      std::vector<float> hl;
      build(NL, KL, [&](int r, int k) -> double {
        const int f = k / KLF, m = k - f * KLF;
        if (r >= np || m >= nfp) return 0.0;
        return d->lift[r * 4 * nfp + f * nfp + m];
      }, hl);
      bl.assign((size_t)2 * NL * KL, 0.f);
      for (int r = 0; r < NL; ++r)
        for (int k = 0; k < KL; ++k) {
          const size_t src = dgtd::tc::kmajor_off(r, k, NL) / 4;
          bl[dgtd::tc::kmajor_off(r, k, 2 * NL) / 4] = hl[src];
          bl[dgtd::tc::kmajor_off(NL + r, k, 2 * NL) / 4] = hl[(size_t)NL * KL + src];
        }
    }
    if ((st = op->tc_bvol.alloc(bv.size())) || (st = op->tc_blift.alloc(bl.size()))) return fail(st);
    e = cudaMemcpyAsync(op->tc_bvol.p, bv.data(), bv.size() * 4, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(op->tc_blift.p, bl.data(), bl.size() * 4, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaStreamSynchronize(s);
  }
  if (!e && d->mass) {
    // |det J| = 1/|det J^-1| from the f64 J^-1 of the descriptor.
    std::vector<double> absdet((size_t)K);
    for (int64_t q = 0; q < K; ++q) {
      const double* m = d->jinv + 9 * q;
      const double dj = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                        m[2] * (m[3] * m[7] - m[4] * m[6]);
      absdet[q] = 1.0 / std::fabs(dj);
    }
    if ((st = op->mass.alloc((size_t)np * np)) || (st = op->absdet.alloc((size_t)K))) return fail(st);
    e = cudaMemcpyAsync(op->mass.p, d->mass, (size_t)np * np * 8, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(op->absdet.p, absdet.data(), (size_t)K * 8, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaStreamSynchronize(s);
    op->has_mass = true;
  }
  if (!e) e = cudaStreamSynchronize(s);
  if (e) {
    set_error(DGTD_ERR_CUDA, std::string("op_create upload: ") + cudaGetErrorString(e));
    return fail(DGTD_ERR_CUDA);
  }
  *out = op;
  return DGTD_OK;
}

extern "C" int dgtd_op_destroy(dgtd_op* op) {
  delete op;
  return DGTD_OK;
}

extern "C" int dgtd_op_n_dof(const dgtd_op* op, int64_t* n) {
  if (!op || !n) return set_error(DGTD_ERR_BAD_ARG, "op_n_dof: null argument");
  *n = op->n_dof;
  return DGTD_OK;
}

extern "C" int dgtd_op_set_engine(dgtd_op* op, int engine) {
  if (!op) return set_error(DGTD_ERR_BAD_ARG, "op_set_engine: null op");
  if (engine == DGTD_ENGINE_FP32 || engine == DGTD_ENGINE_FP32_SMALL_TILES ||
      engine == DGTD_ENGINE_TF32X3) {
    op->engine = engine;
    return DGTD_OK;
  }
  return set_error(DGTD_ERR_UNSUPPORTED, "op_set_engine: engine not available for this order");
}

extern "C" int dgtd_op_get_engine(const dgtd_op* op, int* engine) {
  if (!op || !engine) return set_error(DGTD_ERR_BAD_ARG, "op_get_engine: null argument");
  *engine = op->engine;
  return DGTD_OK;
}

extern "C" int dgtd_op_launch_count(const dgtd_op* op, int64_t* count) {
  if (!op || !count) return set_error(DGTD_ERR_BAD_ARG, "op_launch_count: null argument");
  *count = op->launches;
  return DGTD_OK;
}

extern "C" int dgtd_op_reset_launch_count(dgtd_op* op) {
  if (!op) return set_error(DGTD_ERR_BAD_ARG, "op_reset_launch_count: null op");
  op->launches = 0;
  return DGTD_OK;
}

// ------------------------------------------------------------------ state

static int ensure_aos32(dgtd_op* op) { return op->aos32.alloc(op->n_dof + 4); }

// A tensor-core kernel that gave up a bounded wait leaves a flag; report it
// (and clear it, so it is reported once).
static int check_kernel_flag(dgtd_op* op) {
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, op->err.p, sizeof(int), cudaMemcpyDeviceToHost, op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  if (h) {
    cudaMemsetAsync(op->err.p, 0, sizeof(int), op->stream());
    return set_error(DGTD_ERR_TIMEOUT, "a tensor-core kernel gave up waiting for its copies / MMAs");
  }
  return DGTD_OK;
}

extern "C" int dgtd_op_check_error(dgtd_op* op) {
  if (!op) return set_error(DGTD_ERR_BAD_ARG, "op_check_error: null op");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  return check_kernel_flag(op);
}

extern "C" int dgtd_state_load_device(dgtd_op* op, const float* d_y) {
  if (!op || !d_y) return set_error(DGTD_ERR_BAD_ARG, "state_load_device: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  return to_soa<float, float>(op, d_y, op->y[op->cur].p);
}

extern "C" int dgtd_state_store_device(dgtd_op* op, float* d_y) {
  if (!op || !d_y) return set_error(DGTD_ERR_BAD_ARG, "state_store_device: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  return to_aos<float, float>(op, op->y[op->cur].p, d_y);
}

extern "C" int dgtd_state_upload(dgtd_op* op, const float* y) {
  if (!op || !y) return set_error(DGTD_ERR_BAD_ARG, "state_upload: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DGTD_TRY(ensure_aos32(op));
  CUDA_TRY(cudaMemcpyAsync(op->aos32.p, y, op->n_dof * 4, cudaMemcpyHostToDevice, op->stream()));
  return to_soa<float, float>(op, op->aos32.p, op->y[op->cur].p);
}

extern "C" int dgtd_state_download(dgtd_op* op, float* y) {
  if (!op || !y) return set_error(DGTD_ERR_BAD_ARG, "state_download: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DGTD_TRY(ensure_aos32(op));
  DGTD_TRY((to_aos<float, float>(op, op->y[op->cur].p, op->aos32.p)));
  CUDA_TRY(cudaMemcpyAsync(y, op->aos32.p, op->n_dof * 4, cudaMemcpyDeviceToHost, op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  return check_kernel_flag(op);
}

extern "C" int dgtd_set_source_vector(dgtd_op* op, const double* src) {
  if (!op || !src) return set_error(DGTD_ERR_BAD_ARG, "set_source_vector: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DGTD_TRY(op->src_vec.alloc(state_len(op)));
  CUDA_TRY(cudaMemsetAsync(op->src_vec.p, 0, state_len(op) * 4, op->stream()));
  DGTD_TRY(op->tmp64.alloc(op->n_dof));
  CUDA_TRY(cudaMemcpyAsync(op->tmp64.p, src, op->n_dof * 8, cudaMemcpyHostToDevice, op->stream()));
  DGTD_TRY((to_soa<double, float>(op, op->tmp64.p, op->src_vec.p)));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  op->src_vec_set = true;
  return DGTD_OK;
}

static int check_drive(dgtd_op* op, int drive, int64_t src_dof, const float* g, int64_t n_samples,
                       int64_t* src_idx) {
  *src_idx = -1;
  if (drive == DGTD_DRIVE_FREE) return DGTD_OK;
  if (!g && n_samples > 0) return set_error(DGTD_ERR_BAD_ARG, "a driven run needs waveform samples");
  if (drive == DGTD_DRIVE_POINT) {
    if (src_dof < 0 || src_dof >= op->n_dof)
      return set_error(DGTD_ERR_BAD_ARG, "source DOF " + std::to_string(src_dof) + " out of range (n_dof = " +
                                             std::to_string(op->n_dof) + ")");
    *src_idx = aos_to_soa_index(src_dof, op->np);
    return DGTD_OK;
  }
  if (drive == DGTD_DRIVE_VECTOR) {
    if (!op->src_vec_set) return set_error(DGTD_ERR_BAD_ARG, "vector drive without a source vector");
    return DGTD_OK;
  }
  return set_error(DGTD_ERR_BAD_ARG, "unknown drive kind");
}

extern "C" int dgtd_run_lserk(dgtd_op* op, float h, int64_t steps, int drive, int64_t src_dof,
                              const float* g) {
  if (!op || steps < 0) return set_error(DGTD_ERR_BAD_ARG, "run_lserk: bad argument");
  if (!(std::isfinite(h) && h > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "run_lserk: step must be positive");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  int64_t src_idx;
  DGTD_TRY(check_drive(op, drive, src_dof, g, steps, &src_idx));
  const float* sv = drive == DGTD_DRIVE_VECTOR ? op->src_vec.p : nullptr;
  for (int64_t k = 0; k < steps; ++k) {
    const float gk = drive == DGTD_DRIVE_FREE ? 0.f : g[k];
    DGTD_TRY(lserk_step(op, h, src_idx, gk, sv));
  }
  return DGTD_OK;
}

extern "C" int dgtd_run_lserk_stages(dgtd_op* op, float h, int64_t steps, int drive, int64_t src_dof,
                                     const float* g_stages) {
  if (!op || steps < 0) return set_error(DGTD_ERR_BAD_ARG, "run_lserk_stages: bad argument");
  if (!(std::isfinite(h) && h > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "run_lserk_stages: step must be positive");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  int64_t src_idx;
  DGTD_TRY(check_drive(op, drive, src_dof, g_stages, steps, &src_idx));
  const float* sv = drive == DGTD_DRIVE_VECTOR ? op->src_vec.p : nullptr;
  static const float zero5[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  for (int64_t k = 0; k < steps; ++k)
    DGTD_TRY(lserk_step(op, h, src_idx, 0.f, sv, drive == DGTD_DRIVE_FREE ? zero5 : g_stages + 5 * k));
  return DGTD_OK;
}

// Element blocks (6*Np f32, contiguous in the element-major SoA state).
__global__ void k_gather_blocks(const float* __restrict__ y, const int64_t* __restrict__ elems, int64_t n,
                                int bs, float* __restrict__ buf) {
  const int64_t total = n * bs;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = t / bs;
    buf[t] = y[elems[j] * bs + (t - j * bs)];
  }
}
__global__ void k_scatter_blocks(float* __restrict__ y, const int64_t* __restrict__ elems, int64_t n, int bs,
                                 const float* __restrict__ buf) {
  const int64_t total = n * bs;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = t / bs;
    y[elems[j] * bs + (t - j * bs)] = buf[t];
  }
}

extern "C" int dgtd_state_gather_elements(dgtd_op* op, const int64_t* d_elems, int64_t n, float* d_buf) {
  if (!op || n < 0 || (n > 0 && (!d_elems || !d_buf)))
    return set_error(DGTD_ERR_BAD_ARG, "state_gather_elements: bad argument");
  if (n == 0) return DGTD_OK;
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  const int bs = 6 * op->np;
  k_gather_blocks<<<grid_for(n * bs, 256, op->ctx->num_sms), 256, 0, op->stream()>>>(op->y[op->cur].p, d_elems, n,
                                                                                      bs, d_buf);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

extern "C" int dgtd_state_scatter_elements(dgtd_op* op, const int64_t* d_elems, int64_t n, const float* d_buf) {
  if (!op || n < 0 || (n > 0 && (!d_elems || !d_buf)))
    return set_error(DGTD_ERR_BAD_ARG, "state_scatter_elements: bad argument");
  if (n == 0) return DGTD_OK;
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  const int bs = 6 * op->np;
  k_scatter_blocks<<<grid_for(n * bs, 256, op->ctx->num_sms), 256, 0, op->stream()>>>(op->y[op->cur].p, d_elems, n,
                                                                                       bs, d_buf);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

extern "C" int dgtd_vec_gather_elements(dgtd_op* op, const float* d_vec, const int64_t* d_elems, int64_t n,
                                        float* d_buf) {
  if (!op || !d_vec || n < 0 || (n > 0 && (!d_elems || !d_buf)))
    return set_error(DGTD_ERR_BAD_ARG, "vec_gather_elements: bad argument");
  if (n == 0) return DGTD_OK;
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  const int bs = 6 * op->np;
  k_gather_blocks<<<grid_for(n * bs, 256, op->ctx->num_sms), 256, 0, op->stream()>>>(d_vec, d_elems, n, bs, d_buf);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

extern "C" int dgtd_vec_scatter_elements(dgtd_op* op, float* d_vec, const int64_t* d_elems, int64_t n,
                                         const float* d_buf) {
  if (!op || !d_vec || n < 0 || (n > 0 && (!d_elems || !d_buf)))
    return set_error(DGTD_ERR_BAD_ARG, "vec_scatter_elements: bad argument");
  if (n == 0) return DGTD_OK;
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  const int bs = 6 * op->np;
  k_scatter_blocks<<<grid_for(n * bs, 256, op->ctx->num_sms), 256, 0, op->stream()>>>(d_vec, d_elems, n, bs, d_buf);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

extern "C" int dgtd_op_set_partition(dgtd_op* op, int64_t n_owned, dgtd_halo_hook halo, dgtd_sum_hook sum,
                                     void* user) {
  if (!op || n_owned < 0 || n_owned > op->n_elem) return set_error(DGTD_ERR_BAD_ARG, "set_partition: bad argument");
  if ((n_owned > 0) != (halo != nullptr && sum != nullptr))
    return set_error(DGTD_ERR_BAD_ARG, "set_partition: give n_owned > 0 with both hooks, or 0 without");
  // the Krylov sweeps read whole 16-byte vectors: the owned prefix must end on one
  if ((n_owned * 6 * op->np) % 4 != 0)
    return set_error(DGTD_ERR_BAD_ARG, "set_partition: the owned DOFs must be a multiple of 4 "
                                       "(an even number of owned elements at order 4)");
  op->part_owned = n_owned;
  op->part_halo = halo;
  op->part_sum = sum;
  op->part_user = user;
  return DGTD_OK;
}

extern "C" int dgtd_lserk_stage(dgtd_op* op, float h, int32_t stage, int drive, int64_t src_dof, float g) {
  if (!op) return set_error(DGTD_ERR_BAD_ARG, "lserk_stage: null op");
  return dgtd_lserk_stage_range(op, h, stage, 0, op->n_elem, 1, drive, src_dof, g);
}

extern "C" int dgtd_lserk_stage_range(dgtd_op* op, float h, int32_t stage, int64_t e_begin, int64_t e_end,
                                      int32_t flip, int drive, int64_t src_dof, float g) {
  if (!op || stage < 0 || stage > 4) return set_error(DGTD_ERR_BAD_ARG, "lserk_stage: stage must be 0..4");
  if (!(std::isfinite(h) && h > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "lserk_stage: step must be positive");
  const int64_t tile = tc_tile_e(op->order);
  if (e_begin < 0 || e_end > op->n_elem || e_begin >= e_end || (e_begin % tile) != 0 ||
      ((e_end % tile) != 0 && e_end != op->n_elem))
    return set_error(DGTD_ERR_BAD_ARG, "lserk_stage_range: need 0 <= e_begin < e_end <= n_elem, e_begin a "
                                       "multiple of the op's tile (" + std::to_string(tile) +
                                       " elements) and e_end one or n_elem");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  int64_t src_idx;
  DGTD_TRY(check_drive(op, drive, src_dof, &g, 1, &src_idx));
  RhsParams P = base_params(op);
  P.e_begin = e_begin;
  P.n_elem = e_end;
  P.y_in = op->y[op->cur].p;
  P.out = op->y[op->cur ^ 1].p;
  P.p = op->p.p;
  P.a = (float)kLserkA[stage];
  P.b = (float)kLserkB[stage];
  P.dt = h;
  P.read_p = stage > 0;
  P.write_p = stage < 4;
  P.src_idx = src_idx;
  P.src_vec = drive == DGTD_DRIVE_VECTOR ? op->src_vec.p : nullptr;
  P.src_g = drive == DGTD_DRIVE_FREE ? 0.f : g;
  DGTD_TRY(launch_rhs<kModeLserk>(op, P));
  if (flip) op->cur ^= 1;
  return DGTD_OK;
}

extern "C" int dgtd_apply_device(dgtd_op* op, const float* d_y, float* d_dy) {
  if (!op || !d_y || !d_dy) return set_error(DGTD_ERR_BAD_ARG, "apply_device: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DGTD_TRY(op->aos32.alloc(op->n_dof + 4));
  // state scratch: y[cur^1] holds the SoA input, p the SoA output (the
  // resident state y[cur] is left untouched).
  DGTD_TRY((to_soa<float, float>(op, d_y, op->y[op->cur ^ 1].p)));
  RhsParams P = base_params(op);
  P.y_in = op->y[op->cur ^ 1].p;
  P.out = op->p.p;
  DGTD_TRY(launch_rhs<kModeApply>(op, P));
  return to_aos<float, float>(op, op->p.p, d_dy);
}

extern "C" int dgtd_apply(dgtd_op* op, const float* y, float* dy) {
  if (!op || !y || !dy) return set_error(DGTD_ERR_BAD_ARG, "apply: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DGTD_TRY(op->tmp64.alloc((op->n_dof + 1) / 2 + 2));  // f32 AoS input staging (reuses f64 scratch)
  float* d_in = reinterpret_cast<float*>(op->tmp64.p);
  DGTD_TRY(op->aos32.alloc(op->n_dof + 4));
  CUDA_TRY(cudaMemcpyAsync(d_in, y, op->n_dof * 4, cudaMemcpyHostToDevice, op->stream()));
  DGTD_TRY(dgtd_apply_device(op, d_in, op->aos32.p));
  CUDA_TRY(cudaMemcpyAsync(dy, op->aos32.p, op->n_dof * 4, cudaMemcpyDeviceToHost, op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  return check_kernel_flag(op);
}

extern "C" int dgtd_transient_probes(dgtd_op* op, const float* y0, float dt, int64_t steps,
                                     int64_t substeps, int drive, int64_t src_dof,
                                     const double* src_vec, const float* g,
                                     const int64_t* probes, int64_t n_probes, float* out,
                                     float* y_final) {
  if (!op || !y0 || steps < 0 || n_probes < 0 || (n_probes > 0 && (!probes || !out)))
    return set_error(DGTD_ERR_BAD_ARG, "transient_probes: bad argument");
  if (!(std::isfinite(dt) && dt > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "dt must be positive");
  substeps = std::max<int64_t>(substeps, 1);
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  if (drive == DGTD_DRIVE_VECTOR) {
    if (!src_vec) return set_error(DGTD_ERR_BAD_ARG, "vector drive without src_vec");
    DGTD_TRY(dgtd_set_source_vector(op, src_vec));
  }
  int64_t src_idx;
  DGTD_TRY(check_drive(op, drive, src_dof, g, steps * substeps, &src_idx));
  DevBuf<int64_t> d_probe;
  DevBuf<float> d_pv;
  std::vector<int64_t> pidx(n_probes);
  for (int64_t q = 0; q < n_probes; ++q) {
    if (probes[q] < 0 || probes[q] >= op->n_dof)
      return set_error(DGTD_ERR_BAD_ARG, "probe DOF " + std::to_string(probes[q]) + " out of range");
    pidx[q] = aos_to_soa_index(probes[q], op->np);
  }
  if (n_probes > 0) {
    DGTD_TRY(d_probe.alloc(n_probes));
    DGTD_TRY(d_pv.alloc((size_t)(steps + 1) * n_probes));
    CUDA_TRY(cudaMemcpyAsync(d_probe.p, pidx.data(), n_probes * 8, cudaMemcpyHostToDevice, op->stream()));
  }
  DGTD_TRY(dgtd_state_upload(op, y0));
  auto record = [&](int64_t row) -> int {
    if (n_probes == 0) return DGTD_OK;
    k_gather_f32<<<grid_for(n_probes, 256, op->ctx->num_sms), 256, 0, op->stream()>>>(
        op->y[op->cur].p, d_probe.p, n_probes, d_pv.p + row * n_probes);
    op->launches++;
    CUDA_TRY(cudaGetLastError());
    return DGTD_OK;
  };
  int st = record(0);
  const float h = dt / (float)substeps;
  const float* sv = drive == DGTD_DRIVE_VECTOR ? op->src_vec.p : nullptr;
  for (int64_t k = 0; k < steps && st == DGTD_OK; ++k) {
    for (int64_t j = 0; j < substeps && st == DGTD_OK; ++j) {
      const float gk = drive == DGTD_DRIVE_FREE ? 0.f : g[k * substeps + j];
      st = lserk_step(op, h, src_idx, gk, sv);
    }
    if (st == DGTD_OK) st = record(k + 1);
  }
  if (st == DGTD_OK && n_probes > 0) {
    cudaError_t e = cudaMemcpyAsync(out, d_pv.p, (size_t)(steps + 1) * n_probes * 4, cudaMemcpyDeviceToHost, op->stream());
    if (e) st = set_error(DGTD_ERR_CUDA, std::string("probe download: ") + cudaGetErrorString(e));
  }
  if (st == DGTD_OK && y_final) st = dgtd_state_download(op, y_final);
  cudaError_t e = cudaStreamSynchronize(op->stream());
  d_probe.free();
  d_pv.free();
  if (st != DGTD_OK) return st;
  CUDA_TRY(e);
  return DGTD_OK;
}

extern "C" int dgtd_transient_functionals(dgtd_op* op, const float* y0, float dt, int64_t steps,
                                          int64_t substeps, int drive, int64_t src_dof,
                                          const double* src_vec, const float* g, int64_t n_fun,
                                          const int64_t* fun_ptr, const int64_t* fun_idx,
                                          const double* fun_w, double* out, float* y_final) {
  if (!op || !y0 || steps < 0 || n_fun < 0 || (n_fun > 0 && (!fun_ptr || !out)))
    return set_error(DGTD_ERR_BAD_ARG, "transient_functionals: bad argument");
  if (n_fun > 65535) return set_error(DGTD_ERR_BAD_ARG, "transient_functionals: at most 65535 functionals");
  if (!(std::isfinite(dt) && dt > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "dt must be positive");
  const int64_t n_terms = n_fun > 0 ? fun_ptr[n_fun] : 0;
  if (n_fun > 0 && fun_ptr[0] != 0) return set_error(DGTD_ERR_BAD_ARG, "fun_ptr[0] must be 0");
  for (int64_t q = 0; q < n_fun; ++q)
    if (fun_ptr[q + 1] < fun_ptr[q]) return set_error(DGTD_ERR_BAD_ARG, "fun_ptr must be non-decreasing");
  if (n_terms > 0 && (!fun_idx || !fun_w)) return set_error(DGTD_ERR_BAD_ARG, "functional terms missing");
  substeps = std::max<int64_t>(substeps, 1);
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  if (drive == DGTD_DRIVE_VECTOR) {
    if (!src_vec) return set_error(DGTD_ERR_BAD_ARG, "vector drive without src_vec");
    DGTD_TRY(dgtd_set_source_vector(op, src_vec));
  }
  int64_t src_idx;
  DGTD_TRY(check_drive(op, drive, src_dof, g, steps * substeps, &src_idx));
  std::vector<int64_t> sidx((size_t)n_terms);
  for (int64_t k = 0; k < n_terms; ++k) {
    if (fun_idx[k] < 0 || fun_idx[k] >= op->n_dof)
      return set_error(DGTD_ERR_BAD_ARG, "functional DOF " + std::to_string(fun_idx[k]) + " out of range");
    sidx[k] = aos_to_soa_index(fun_idx[k], op->np);
  }
  DevBuf<int64_t> d_ptr, d_idx;
  DevBuf<double> d_w, d_out;
  if (n_fun > 0) {
    DGTD_TRY(d_ptr.alloc(n_fun + 1));
    DGTD_TRY(d_idx.alloc(std::max<int64_t>(n_terms, 1)));
    DGTD_TRY(d_w.alloc(std::max<int64_t>(n_terms, 1)));
    DGTD_TRY(d_out.alloc((size_t)(steps + 1) * n_fun));
    CUDA_TRY(cudaMemcpyAsync(d_ptr.p, fun_ptr, (n_fun + 1) * 8, cudaMemcpyHostToDevice, op->stream()));
    if (n_terms > 0) {
      CUDA_TRY(cudaMemcpyAsync(d_idx.p, sidx.data(), n_terms * 8, cudaMemcpyHostToDevice, op->stream()));
      CUDA_TRY(cudaMemcpyAsync(d_w.p, fun_w, n_terms * 8, cudaMemcpyHostToDevice, op->stream()));
    }
  }
  DGTD_TRY(dgtd_state_upload(op, y0));
  auto record = [&](int64_t row) -> int {
    if (n_fun == 0) return DGTD_OK;
    k_functionals<<<(unsigned)n_fun, 256, 0, op->stream()>>>(op->y[op->cur].p, d_ptr.p, d_idx.p, d_w.p,
                                                             d_out.p + row * n_fun);
    op->launches++;
    CUDA_TRY(cudaGetLastError());
    return DGTD_OK;
  };
  int st = record(0);
  const float h = dt / (float)substeps;
  const float* sv = drive == DGTD_DRIVE_VECTOR ? op->src_vec.p : nullptr;
  for (int64_t k = 0; k < steps && st == DGTD_OK; ++k) {
    for (int64_t j = 0; j < substeps && st == DGTD_OK; ++j) {
      const float gk = drive == DGTD_DRIVE_FREE ? 0.f : g[k * substeps + j];
      st = lserk_step(op, h, src_idx, gk, sv);
    }
    if (st == DGTD_OK) st = record(k + 1);
  }
  if (st == DGTD_OK && n_fun > 0) {
    cudaError_t e = cudaMemcpyAsync(out, d_out.p, (size_t)(steps + 1) * n_fun * 8, cudaMemcpyDeviceToHost,
                                    op->stream());
    if (e) st = set_error(DGTD_ERR_CUDA, std::string("functional download: ") + cudaGetErrorString(e));
  }
  if (st == DGTD_OK && y_final) st = dgtd_state_download(op, y_final);
  cudaError_t e = cudaStreamSynchronize(op->stream());
  d_ptr.free(); d_idx.free(); d_w.free(); d_out.free();
  if (st != DGTD_OK) return st;
  CUDA_TRY(e);
  return check_kernel_flag(op);
}

extern "C" int dgtd_op_set_functionals(dgtd_op* op, int64_t n_fun, const int64_t* fun_ptr, const int64_t* fun_idx,
                                       const double* fun_w, int64_t max_rows) {
  if (!op || n_fun < 1 || !fun_ptr || max_rows < 1) return set_error(DGTD_ERR_BAD_ARG, "set_functionals: bad argument");
  if (fun_ptr[0] != 0) return set_error(DGTD_ERR_BAD_ARG, "set_functionals: fun_ptr[0] must be 0");
  for (int64_t q = 0; q < n_fun; ++q)
    if (fun_ptr[q + 1] < fun_ptr[q]) return set_error(DGTD_ERR_BAD_ARG, "set_functionals: fun_ptr must not decrease");
  const int64_t n_terms = fun_ptr[n_fun];
  if (n_terms > 0 && (!fun_idx || !fun_w)) return set_error(DGTD_ERR_BAD_ARG, "set_functionals: terms missing");
  std::vector<int64_t> sidx((size_t)n_terms);
  for (int64_t k = 0; k < n_terms; ++k) {
    if (fun_idx[k] < 0 || fun_idx[k] >= op->n_dof)
      return set_error(DGTD_ERR_BAD_ARG, "set_functionals: DOF " + std::to_string(fun_idx[k]) + " out of range");
    sidx[k] = aos_to_soa_index(fun_idx[k], op->np);
  }
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));  // the old buffers may still be read
  op->fn_ptr.free(); op->fn_idx.free(); op->fn_w.free(); op->fn_out.free();
  op->fn_n = op->fn_rows = 0;
  DGTD_TRY(op->fn_ptr.alloc(n_fun + 1));
  DGTD_TRY(op->fn_idx.alloc(std::max<int64_t>(n_terms, 1)));
  DGTD_TRY(op->fn_w.alloc(std::max<int64_t>(n_terms, 1)));
  DGTD_TRY(op->fn_out.alloc((size_t)max_rows * n_fun));
  CUDA_TRY(cudaMemcpyAsync(op->fn_ptr.p, fun_ptr, (n_fun + 1) * 8, cudaMemcpyHostToDevice, op->stream()));
  if (n_terms > 0) {
    CUDA_TRY(cudaMemcpyAsync(op->fn_idx.p, sidx.data(), n_terms * 8, cudaMemcpyHostToDevice, op->stream()));
    CUDA_TRY(cudaMemcpyAsync(op->fn_w.p, fun_w, n_terms * 8, cudaMemcpyHostToDevice, op->stream()));
  }
  CUDA_TRY(cudaStreamSynchronize(op->stream()));  // sidx leaves scope
  op->fn_n = n_fun;
  op->fn_rows = max_rows;
  return DGTD_OK;
}

extern "C" int dgtd_record_functionals(dgtd_op* op, int64_t row) {
  if (!op || op->fn_n < 1) return set_error(DGTD_ERR_BAD_ARG, "record_functionals: no functionals set");
  if (row < 0 || row >= op->fn_rows) return set_error(DGTD_ERR_BAD_ARG, "record_functionals: row out of range");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  k_functionals<<<(unsigned)op->fn_n, 256, 0, op->stream()>>>(op->y[op->cur].p, op->fn_ptr.p, op->fn_idx.p,
                                                              op->fn_w.p, op->fn_out.p + row * op->fn_n);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

extern "C" int dgtd_functional_series(dgtd_op* op, int64_t n_rows, double* out) {
  if (!op || !out || op->fn_n < 1 || n_rows < 0 || n_rows > op->fn_rows)
    return set_error(DGTD_ERR_BAD_ARG, "functional_series: bad argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  if (n_rows > 0)
    CUDA_TRY(cudaMemcpyAsync(out, op->fn_out.p, (size_t)n_rows * op->fn_n * 8, cudaMemcpyDeviceToHost, op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  return check_kernel_flag(op);
}

extern "C" int dgtd_transient(dgtd_op* op, const float* y0, float dt, int64_t steps, int64_t substeps,
                              int drive, int64_t src_dof, const double* src_vec, const float* g,
                              int record, float* out) {
  if (!op || !y0 || !out || steps < 0) return set_error(DGTD_ERR_BAD_ARG, "transient: bad argument");
  if (!(std::isfinite(dt) && dt > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "dt must be positive");
  substeps = std::max<int64_t>(substeps, 1);
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  if (drive == DGTD_DRIVE_VECTOR) {
    if (!src_vec) return set_error(DGTD_ERR_BAD_ARG, "vector drive without src_vec");
    DGTD_TRY(dgtd_set_source_vector(op, src_vec));
  }
  int64_t src_idx;
  DGTD_TRY(check_drive(op, drive, src_dof, g, steps * substeps, &src_idx));
  DGTD_TRY(dgtd_state_upload(op, y0));
  const float h = dt / (float)substeps;
  const float* sv = drive == DGTD_DRIVE_VECTOR ? op->src_vec.p : nullptr;
  if (record) std::memcpy(out, y0, op->n_dof * 4);
  for (int64_t k = 0; k < steps; ++k) {
    for (int64_t j = 0; j < substeps; ++j) {
      const float gk = drive == DGTD_DRIVE_FREE ? 0.f : g[k * substeps + j];
      DGTD_TRY(lserk_step(op, h, src_idx, gk, sv));
    }
    if (record) DGTD_TRY(dgtd_state_download(op, out + (k + 1) * op->n_dof));
  }
  if (!record) DGTD_TRY(dgtd_state_download(op, out));
  return DGTD_OK;
}

// ------------------------------------------------------------------ FP64 path
//
// The RHS and the LSERK4 stage in f64 on the CUDA cores (rhs_fp64_kernel): the
// reference's CPU arithmetic (rhs.rs, explicit.rs in f64) on the device, for
// FP64 runs and as the reference solution at sizes the CPU cannot reach.

namespace {

int ensure_state64(dgtd_op* op) {
  const size_t len = state_len(op);
  const bool fresh = op->y64[0].n < len || op->y64[1].n < len || op->p64.n < len;
  DGTD_TRY(op->y64[0].alloc(len));
  DGTD_TRY(op->y64[1].alloc(len));
  DGTD_TRY(op->p64.alloc(len));
  DGTD_TRY(op->tmp64.alloc(op->n_dof));
  if (fresh) {  // the padding past n_dof stays zero
    for (int b = 0; b < 2; ++b) CUDA_TRY(cudaMemsetAsync(op->y64[b].p, 0, len * 8, op->stream()));
    CUDA_TRY(cudaMemsetAsync(op->p64.p, 0, len * 8, op->stream()));
  }
  return DGTD_OK;
}

int upload64(dgtd_op* op, const double* y) {
  CUDA_TRY(cudaMemcpyAsync(op->tmp64.p, y, op->n_dof * 8, cudaMemcpyHostToDevice, op->stream()));
  return to_soa<double, double>(op, op->tmp64.p, op->y64[op->cur64].p);
}

int download64(dgtd_op* op, const double* soa, double* y) {
  DGTD_TRY((to_aos<double, double>(op, soa, op->tmp64.p)));
  CUDA_TRY(cudaMemcpyAsync(y, op->tmp64.p, op->n_dof * 8, cudaMemcpyDeviceToHost, op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  return DGTD_OK;
}

int lserk_step64(dgtd_op* op, double h, int64_t src_idx, double g, const double* src_vec,
                 const double* g5 = nullptr) {
  for (int s = 0; s < 5; ++s) {
    RhsParamsT<double> P = base_params64(op);
    P.y_in = op->y64[op->cur64].p;
    P.out = op->y64[op->cur64 ^ 1].p;
    P.p = op->p64.p;
    P.a = kLserkA[s];
    P.b = kLserkB[s];
    P.dt = h;
    P.read_p = s > 0;
    P.write_p = s < 4;
    P.src_idx = src_idx;
    P.src_vec = src_vec;
    P.src_g = g5 ? g5[s] : g;
    DGTD_TRY(launch_rhs64<kModeLserk>(op, P));
    op->cur64 ^= 1;
  }
  return DGTD_OK;
}

}  // namespace

extern "C" int dgtd_apply_f64(dgtd_op* op, const double* y, double* dy) {
  if (!op || !y || !dy) return set_error(DGTD_ERR_BAD_ARG, "apply_f64: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DGTD_TRY(ensure_state64(op));
  DGTD_TRY(upload64(op, y));
  RhsParamsT<double> P = base_params64(op);
  P.y_in = op->y64[op->cur64].p;
  P.out = op->y64[op->cur64 ^ 1].p;
  DGTD_TRY(launch_rhs64<kModeApply>(op, P));
  return download64(op, op->y64[op->cur64 ^ 1].p, dy);
}

namespace {
int transient_f64_impl(dgtd_op* op, const double* y0, double dt, int64_t steps, int64_t substeps, int drive,
                       int64_t src_dof, const double* src_vec, const double* g, bool staged, int record,
                       double* out) {
  if (!op || !y0 || !out || steps < 0) return set_error(DGTD_ERR_BAD_ARG, "transient_f64: bad argument");
  if (!(std::isfinite(dt) && dt > 0.0)) return set_error(DGTD_ERR_BAD_ARG, "transient_f64: dt must be positive");
  substeps = std::max<int64_t>(substeps, 1);
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  int64_t src_idx = -1;
  if (drive == DGTD_DRIVE_POINT) {
    if (src_dof < 0 || src_dof >= op->n_dof)
      return set_error(DGTD_ERR_BAD_ARG, "source DOF " + std::to_string(src_dof) + " out of range");
    src_idx = aos_to_soa_index(src_dof, op->np);
  } else if (drive == DGTD_DRIVE_VECTOR) {
    if (!src_vec) return set_error(DGTD_ERR_BAD_ARG, "vector drive without src_vec");
  } else if (drive != DGTD_DRIVE_FREE) {
    return set_error(DGTD_ERR_BAD_ARG, "unknown drive kind");
  }
  if (drive != DGTD_DRIVE_FREE && !g && steps > 0) return set_error(DGTD_ERR_BAD_ARG, "a driven run needs waveform samples");
  DGTD_TRY(ensure_state64(op));
  const double* sv = nullptr;
  if (drive == DGTD_DRIVE_VECTOR) {
    DGTD_TRY(op->src_vec64.alloc(state_len(op)));
    CUDA_TRY(cudaMemsetAsync(op->src_vec64.p, 0, state_len(op) * 8, op->stream()));
    CUDA_TRY(cudaMemcpyAsync(op->tmp64.p, src_vec, op->n_dof * 8, cudaMemcpyHostToDevice, op->stream()));
    DGTD_TRY((to_soa<double, double>(op, op->tmp64.p, op->src_vec64.p)));
    sv = op->src_vec64.p;
  }
  DGTD_TRY(upload64(op, y0));
  const double h = dt / (double)substeps;
  if (record) std::memcpy(out, y0, op->n_dof * 8);
  for (int64_t k = 0; k < steps; ++k) {
    for (int64_t j = 0; j < substeps; ++j) {
      const int64_t q = k * substeps + j;
      if (staged) {
        static const double zero5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        DGTD_TRY(lserk_step64(op, h, src_idx, 0.0, sv, drive == DGTD_DRIVE_FREE ? zero5 : g + 5 * q));
      } else {
        DGTD_TRY(lserk_step64(op, h, src_idx, drive == DGTD_DRIVE_FREE ? 0.0 : g[q], sv));
      }
    }
    if (record) DGTD_TRY(download64(op, op->y64[op->cur64].p, out + (k + 1) * op->n_dof));
  }
  if (!record) DGTD_TRY(download64(op, op->y64[op->cur64].p, out));
  return DGTD_OK;
}
}  // namespace

extern "C" int dgtd_transient_f64(dgtd_op* op, const double* y0, double dt, int64_t steps, int64_t substeps,
                                  int drive, int64_t src_dof, const double* src_vec, const double* g,
                                  int record, double* out) {
  return transient_f64_impl(op, y0, dt, steps, substeps, drive, src_dof, src_vec, g, false, record, out);
}

extern "C" int dgtd_transient_f64_stages(dgtd_op* op, const double* y0, double dt, int64_t steps,
                                         int64_t substeps, int drive, int64_t src_dof, const double* src_vec,
                                         const double* g_stages, int record, double* out) {
  return transient_f64_impl(op, y0, dt, steps, substeps, drive, src_dof, src_vec, g_stages, true, record, out);
}

// ------------------------------------------------------------------ MLP (learned ETD controller)

struct dgtd_mlp {
  dgtd_ctx* ctx = nullptr;
  int device = 0;  // as dgtd_op: the destructor does not read ctx
  dgtd::MlpShape S{};
  int step = 0;
  DevBuf<float> p, m, v, grad, loss;
  DevBuf<float> x, y, tg, a1, a2, G, lb;
  ~dgtd_mlp() {
    cudaSetDevice(device);
    p.free(); m.free(); v.free(); grad.free(); loss.free();
    x.free(); y.free(); tg.free(); a1.free(); a2.free(); G.free(); lb.free();
  }
};

namespace {

// splitmix64 (Steele, Lea & Flood 2014): the seeded initial weights.
uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int mlp_stage(dgtd_mlp* n, const float* x, const float* t, int64_t batch, bool keep) {
  cudaStream_t s = n->ctx->stream;
  DGTD_TRY(n->x.alloc((size_t)batch * n->S.n_in));
  DGTD_TRY(n->y.alloc((size_t)batch * n->S.n_out));
  CUDA_TRY(cudaMemcpyAsync(n->x.p, x, (size_t)batch * n->S.n_in * 4, cudaMemcpyHostToDevice, s));
  if (t) {
    DGTD_TRY(n->tg.alloc((size_t)batch * n->S.n_out));
    CUDA_TRY(cudaMemcpyAsync(n->tg.p, t, (size_t)batch * n->S.n_out * 4, cudaMemcpyHostToDevice, s));
  }
  if (keep) {
    DGTD_TRY(n->a1.alloc((size_t)batch * n->S.n_hidden));
    DGTD_TRY(n->a2.alloc((size_t)batch * n->S.n_hidden));
    DGTD_TRY(n->G.alloc((size_t)batch * n->S.n_params()));
    DGTD_TRY(n->lb.alloc((size_t)batch));
  }
  return DGTD_OK;
}

int mlp_grad_launch(dgtd_mlp* n, int64_t batch) {
  cudaStream_t s = n->ctx->stream;
  const int th = std::max(32, (n->S.n_hidden + 31) / 32 * 32);
  const int np = n->S.n_params();
  dgtd::k_mlp_forward<<<(unsigned)batch, th, 0, s>>>(n->S, n->p.p, n->x.p, batch, n->y.p, n->a1.p, n->a2.p);
  dgtd::k_mlp_backward<<<(unsigned)batch, th, 0, s>>>(n->S, n->p.p, n->x.p, n->tg.p, n->y.p, n->a1.p, n->a2.p,
                                                      batch, n->G.p, n->lb.p);
  dgtd::k_mlp_reduce<<<(np + 255) / 256, 256, 0, s>>>(n->G.p, batch, np, n->grad.p, n->lb.p, n->loss.p);
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

int mlp_check(dgtd_mlp* n, int64_t batch, const char* what) {
  if (!n || batch < 1 || batch > 65535) return set_error(DGTD_ERR_BAD_ARG, std::string(what) + ": batch must be 1..65535");
  CUDA_TRY(cudaSetDevice(n->ctx->device));
  return DGTD_OK;
}

}  // namespace

extern "C" int dgtd_mlp_create(dgtd_ctx* ctx, int32_t n_in, int32_t n_hidden, int32_t n_out, uint64_t seed,
                               dgtd_mlp** out) {
  if (!ctx || !out || n_in < 1 || n_in > dgtd::kMlpMaxIn || n_hidden < 1 || n_hidden > dgtd::kMlpMaxHidden ||
      n_out < 1 || n_out > dgtd::kMlpMaxOut || n_out > n_hidden)
    return set_error(DGTD_ERR_BAD_ARG, "mlp_create: sizes must be 1..64 in, 1..128 hidden, 1..8 (<= hidden) out");
  CUDA_TRY(cudaSetDevice(ctx->device));
  auto n = std::make_unique<dgtd_mlp>();
  n->ctx = ctx;
  n->device = ctx->device;
  n->S = dgtd::MlpShape{n_in, n_hidden, n_out};
  const int np = n->S.n_params();
  // Glorot-uniform weights, zero biases
  std::vector<float> h(np, 0.f);
  uint64_t st = seed;
  auto fill = [&](int off, int rows, int cols) {
    const double a = std::sqrt(6.0 / (double)(rows + cols));
    for (int q = 0; q < rows * cols; ++q) {
      const double u = (double)(splitmix64(st) >> 11) * (1.0 / 9007199254740992.0);
      h[off + q] = (float)((2.0 * u - 1.0) * a);
    }
  };
  fill(n->S.o_w1(), n_hidden, n_in);
  fill(n->S.o_w2(), n_hidden, n_hidden);
  fill(n->S.o_w3(), n_out, n_hidden);
  DGTD_TRY(n->p.alloc(np));
  DGTD_TRY(n->m.alloc(np));
  DGTD_TRY(n->v.alloc(np));
  DGTD_TRY(n->grad.alloc(np));
  DGTD_TRY(n->loss.alloc(1));
  CUDA_TRY(cudaMemcpyAsync(n->p.p, h.data(), np * 4, cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaMemsetAsync(n->m.p, 0, np * 4, ctx->stream));
  CUDA_TRY(cudaMemsetAsync(n->v.p, 0, np * 4, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *out = n.release();
  return DGTD_OK;
}

extern "C" void dgtd_mlp_destroy(dgtd_mlp* n) { delete n; }

extern "C" int dgtd_mlp_n_params(const dgtd_mlp* n, int64_t* np) {
  if (!n || !np) return set_error(DGTD_ERR_BAD_ARG, "mlp_n_params: null argument");
  *np = n->S.n_params();
  return DGTD_OK;
}

extern "C" int dgtd_mlp_get_params(dgtd_mlp* n, float* out) {
  if (!n || !out) return set_error(DGTD_ERR_BAD_ARG, "mlp_get_params: null argument");
  CUDA_TRY(cudaSetDevice(n->ctx->device));
  CUDA_TRY(cudaMemcpyAsync(out, n->p.p, n->S.n_params() * 4, cudaMemcpyDeviceToHost, n->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(n->ctx->stream));
  return DGTD_OK;
}

extern "C" int dgtd_mlp_set_params(dgtd_mlp* n, const float* in) {
  if (!n || !in) return set_error(DGTD_ERR_BAD_ARG, "mlp_set_params: null argument");
  CUDA_TRY(cudaSetDevice(n->ctx->device));
  CUDA_TRY(cudaMemcpyAsync(n->p.p, in, n->S.n_params() * 4, cudaMemcpyHostToDevice, n->ctx->stream));
  CUDA_TRY(cudaMemsetAsync(n->m.p, 0, n->S.n_params() * 4, n->ctx->stream));
  CUDA_TRY(cudaMemsetAsync(n->v.p, 0, n->S.n_params() * 4, n->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(n->ctx->stream));
  n->step = 0;
  return DGTD_OK;
}

extern "C" int dgtd_mlp_forward(dgtd_mlp* n, const float* x, int64_t batch, float* y) {
  DGTD_TRY(mlp_check(n, batch, "mlp_forward"));
  if (!x || !y) return set_error(DGTD_ERR_BAD_ARG, "mlp_forward: null argument");
  DGTD_TRY(mlp_stage(n, x, nullptr, batch, false));
  const int th = std::max(32, (n->S.n_hidden + 31) / 32 * 32);
  dgtd::k_mlp_forward<<<(unsigned)batch, th, 0, n->ctx->stream>>>(n->S, n->p.p, n->x.p, batch, n->y.p, nullptr,
                                                                  nullptr);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(y, n->y.p, (size_t)batch * n->S.n_out * 4, cudaMemcpyDeviceToHost, n->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(n->ctx->stream));
  return DGTD_OK;
}

extern "C" int dgtd_mlp_gradient(dgtd_mlp* n, const float* x, const float* t, int64_t batch, float* grad,
                                 float* loss) {
  DGTD_TRY(mlp_check(n, batch, "mlp_gradient"));
  if (!x || !t || !grad) return set_error(DGTD_ERR_BAD_ARG, "mlp_gradient: null argument");
  DGTD_TRY(mlp_stage(n, x, t, batch, true));
  DGTD_TRY(mlp_grad_launch(n, batch));
  CUDA_TRY(cudaMemcpyAsync(grad, n->grad.p, n->S.n_params() * 4, cudaMemcpyDeviceToHost, n->ctx->stream));
  if (loss) CUDA_TRY(cudaMemcpyAsync(loss, n->loss.p, 4, cudaMemcpyDeviceToHost, n->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(n->ctx->stream));
  return DGTD_OK;
}

extern "C" int dgtd_mlp_train(dgtd_mlp* n, const float* x, const float* t, int64_t batch, int32_t epochs, float lr,
                              float* losses) {
  DGTD_TRY(mlp_check(n, batch, "mlp_train"));
  if (!x || !t || epochs < 0 || !(lr > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "mlp_train: bad argument");
  DGTD_TRY(mlp_stage(n, x, t, batch, true));
  DevBuf<float> hist;
  DGTD_TRY(hist.alloc(std::max(epochs, 1)));
  cudaStream_t s = n->ctx->stream;
  const int np = n->S.n_params();
  for (int e = 0; e < epochs; ++e) {
    DGTD_TRY(mlp_grad_launch(n, batch));
    ++n->step;
    dgtd::k_mlp_adam<<<(np + 255) / 256, 256, 0, s>>>(n->p.p, n->m.p, n->v.p, n->grad.p, np, lr, 0.9f, 0.999f,
                                                      1e-8f, n->step);
    CUDA_TRY(cudaMemcpyAsync(hist.p + e, n->loss.p, 4, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaGetLastError());
  }
  if (losses && epochs > 0) CUDA_TRY(cudaMemcpyAsync(losses, hist.p, epochs * 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  hist.free();
  return DGTD_OK;
}

// ------------------------------------------------------------------ KCL adaptive

extern "C" void dgtd_kcl_controller_default(dgtd_kcl_controller* c) {
  if (!c) return;
  c->atol = 1e-8;                 // KCL_ATOL
  c->rtol = 1e-4;                 // KCL_RTOL
  c->safety = 0.9;                // KCL_SAFETY
  c->growth_limit = 5.0;          // KCL_GROWTH_LIMIT
  c->shrink_limit = 0.2;          // KCL_SHRINK_LIMIT
  c->pi_alpha = 0.7 / 4.0;        // KCL_PI_ALPHA
  c->pi_beta = 0.4 / 4.0;         // KCL_PI_BETA
  c->min_step_factor = 1e-10;     // KCL_MIN_STEP_FACTOR
}

namespace {

constexpr long long kKclAttemptCap = 10000000;  // per output frame

// The five stages of one KCL attempt as fused RHS + stage launches: stage s
// evaluates the RHS at its point (stage 0: the backup of y the attempt began
// from; later stages: the point the previous stage wrote) and updates y and
// the embedded error in place, writing the next stage's point into the other
// of two stage buffers (explicit_adaptive.rs:84-152).
int kcl_stages(dgtd_op* op, dgtd::KclCtl* dc, float* y, int64_t src_idx, const float* sv, const float* gv) {
  float* stage_buf[2] = {op->kcl_stage.p, op->kcl_k.p};
  for (int st = 0; st < 5; ++st) {
    RhsParams P = base_params(op);
    P.y_in = st == 0 ? op->kcl_bak.p : stage_buf[(st - 1) & 1];
    P.skip = &dc->skip;
    P.src_idx = src_idx;
    P.src_vec = sv;
    P.kcl_y = y;
    P.kcl_e = op->kcl_e.p;
    P.kcl_next = st < 4 ? stage_buf[st & 1] : nullptr;
    P.kcl_h = &dc->h_try;
    P.kcl_frame = &dc->frame;
    P.kcl_g = gv;
    P.kcl_b = (float)dgtd::kKclB[st];
    P.kcl_ew = (float)(dgtd::kKclBhat[st] - dgtd::kKclB[st]);
    P.kcl_amb = st < 4 ? (float)(dgtd::kKclA[st] - dgtd::kKclB[st]) : 0.f;
    P.kcl_stage = st;
    DGTD_TRY(launch_rhs<kModeKcl>(op, P));
  }
  return DGTD_OK;
}

// One adaptive run on the resident state.  Frames are recorded into d_traj
// (SoA rows, may be null) or as functionals into d_fun (may be null).
int kcl_run(dgtd_op* op, float dt, int64_t steps, int drive, int64_t src_dof, const float* g,
            const dgtd_kcl_controller* cin, float* d_traj, int64_t n_fun, const int64_t* d_ptr,
            const int64_t* d_idx, const double* d_w, double* d_fun, dgtd_kcl_stats* stats) {
  using dgtd::KclCtl;
  const int64_t n = op->n_dof;
  cudaStream_t s = op->stream();
  int64_t src_idx;
  DGTD_TRY(check_drive(op, drive, src_dof, g, steps, &src_idx));
  const size_t len = state_len(op);
  DGTD_TRY(op->kcl_ctl.alloc(1));
  DGTD_TRY(op->kcl_log.alloc(dgtd::kKclLogCap));
  op->kcl_log_n = 0;
  const bool fresh = op->kcl_stage.n < len;
  DGTD_TRY(op->kcl_bak.alloc(len));
  DGTD_TRY(op->kcl_e.alloc(len));
  DGTD_TRY(op->kcl_stage.alloc(len));
  DGTD_TRY(op->kcl_k.alloc(len));
  if (fresh) {  // the padding tail of the RHS input must hold finite values
    CUDA_TRY(cudaMemsetAsync(op->kcl_stage.p, 0, len * 4, s));
    CUDA_TRY(cudaMemsetAsync(op->kcl_k.p, 0, len * 4, s));
  }
  const int nt = 256, ng = grid_for(n, nt, op->ctx->num_sms);
  DGTD_TRY(op->kcl_part.alloc(ng));
  const float* gv = nullptr;
  if (drive != DGTD_DRIVE_FREE && steps > 0) {
    DGTD_TRY(op->kcl_g.alloc(steps));
    CUDA_TRY(cudaMemcpyAsync(op->kcl_g.p, g, steps * 4, cudaMemcpyHostToDevice, s));
    gv = op->kcl_g.p;
  }
  KclCtl c;
  std::memset(&c, 0, sizeof(c));
  c.atol = cin->atol; c.rtol = cin->rtol; c.safety = cin->safety; c.growth = cin->growth_limit;
  c.shrink = cin->shrink_limit; c.alpha = cin->pi_alpha; c.beta = cin->pi_beta;
  c.min_step_factor = cin->min_step_factor;
  c.dt = dt; c.h = dt; c.prev_err = 0.f; c.t_rel = 0.f;
  c.h_min_log = INFINITY; c.h_max_log = 0.f;
  c.steps = steps; c.attempt_cap = kKclAttemptCap;
  c.status = steps > 0 ? dgtd::kKclRunning : dgtd::kKclDone;
  c.record = -1;
  c.log = op->kcl_log.p;
  KclCtl* dc = op->kcl_ctl.p;
  CUDA_TRY(cudaMemcpyAsync(dc, &c, sizeof(c), cudaMemcpyHostToDevice, s));
  const float* sv = drive == DGTD_DRIVE_VECTOR ? op->src_vec.p : nullptr;
  float* y = op->y[op->cur].p;
  auto attempt = [&]() -> int {
    dgtd::k_kcl_begin<<<ng, nt, 0, s>>>(dc, y, op->kcl_bak.p, n);
    DGTD_TRY(kcl_stages(op, dc, y, src_idx, sv, gv));
    dgtd::k_kcl_err<<<ng, 256, 0, s>>>(dc, op->kcl_bak.p, y, op->kcl_e.p, op->kcl_part.p, n);
    dgtd::k_kcl_control<<<1, 256, 0, s>>>(dc, op->kcl_part.p, ng, n);
    dgtd::k_kcl_restore<<<ng, nt, 0, s>>>(dc, y, op->kcl_bak.p, n);
    if (d_traj) dgtd::k_kcl_record_state<<<ng, nt, 0, s>>>(dc, y, d_traj, n);
    if (n_fun > 0)
      dgtd::k_kcl_record_fun<<<(unsigned)n_fun, 256, 0, s>>>(dc, y, d_ptr, d_idx, d_w, d_fun, n_fun);
    op->launches += 5;
    CUDA_TRY(cudaGetLastError());
    return DGTD_OK;
  };
  // Batches of attempts; one status read per batch.  The batch is sized from
  // the attempts per frame seen so far; surplus attempts at the end of the
  // run do nothing.
  int64_t batch = 4, attempts = 0;
  while (c.status == dgtd::kKclRunning) {
    for (int64_t b = 0; b < batch; ++b) DGTD_TRY(attempt());
    attempts += batch;
    CUDA_TRY(cudaMemcpyAsync(&c, dc, sizeof(c), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    DGTD_TRY(check_kernel_flag(op));
    if (c.frame > 0) {
      const double per_frame = (double)(c.n_acc + c.n_rej) / (double)c.frame;
      batch = (int64_t)std::ceil(per_frame * (double)(steps - c.frame)) + 1;
    } else {
      batch *= 2;
    }
    batch = std::max<int64_t>(1, std::min<int64_t>(batch, 256));
  }
  (void)attempts;
  op->kcl_log_n = c.n_acc;
  if (stats) {
    stats->accepted = c.n_acc;
    stats->rejected = c.n_rej;
    stats->h_min = c.n_acc ? c.h_min_log : 0.f;
    stats->h_max = c.h_max_log;
  }
  if (c.status == dgtd::kKclCollapsed) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "GPU KCL: step size collapsed below %g*dt after %lld accepted, %lld rejected substeps",
                  cin->min_step_factor, (long long)c.n_acc, (long long)c.n_rej);
    return set_error(DGTD_ERR_COLLAPSE, msg);
  }
  if (c.status == dgtd::kKclCapped)
    return set_error(DGTD_ERR_TIMEOUT, "GPU KCL: more than 1e7 attempts in one output frame");
  return DGTD_OK;
}

int kcl_args(dgtd_op* op, const float* y0, float dt, int64_t steps, int drive, const double* src_vec,
             const dgtd_kcl_controller* ctl, const char* what) {
  if (!op || !y0 || !ctl || steps < 0) return set_error(DGTD_ERR_BAD_ARG, std::string(what) + ": bad argument");
  if (!(std::isfinite(dt) && dt > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "dt must be positive");
  if (!(ctl->atol >= 0.0 && ctl->rtol >= 0.0 && ctl->atol + ctl->rtol > 0.0 && ctl->safety > 0.0 &&
        ctl->shrink_limit > 0.0 && ctl->growth_limit >= ctl->shrink_limit && ctl->min_step_factor >= 0.0))
    return set_error(DGTD_ERR_BAD_ARG, std::string(what) + ": invalid controller settings");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  if (drive == DGTD_DRIVE_VECTOR) {
    if (!src_vec) return set_error(DGTD_ERR_BAD_ARG, "vector drive without src_vec");
    DGTD_TRY(dgtd_set_source_vector(op, src_vec));
  }
  return DGTD_OK;
}

}  // namespace

extern "C" int dgtd_kcl_step(dgtd_op* op, const double* y, double h, double* y_out, double* err) {
  if (!op || !y || !y_out || !err) return set_error(DGTD_ERR_BAD_ARG, "kcl_step: null argument");
  if (!(std::isfinite(h) && h > 0.0)) return set_error(DGTD_ERR_BAD_ARG, "kcl_step: step must be positive");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  cudaStream_t s = op->stream();
  const int64_t n = op->n_dof;
  DGTD_TRY(op->tmp64.alloc(n));
  CUDA_TRY(cudaMemcpyAsync(op->tmp64.p, y, n * 8, cudaMemcpyHostToDevice, s));
  DGTD_TRY((to_soa<double, float>(op, op->tmp64.p, op->y[op->cur].p)));
  const size_t len = state_len(op);
  const bool fresh = op->kcl_stage.n < len;
  DGTD_TRY(op->kcl_ctl.alloc(1));
  DGTD_TRY(op->kcl_bak.alloc(len));
  DGTD_TRY(op->kcl_e.alloc(len));
  DGTD_TRY(op->kcl_stage.alloc(len));
  DGTD_TRY(op->kcl_k.alloc(len));
  if (fresh) {
    CUDA_TRY(cudaMemsetAsync(op->kcl_stage.p, 0, len * 4, s));
    CUDA_TRY(cudaMemsetAsync(op->kcl_k.p, 0, len * 4, s));
  }
  dgtd::KclCtl c;
  std::memset(&c, 0, sizeof(c));
  c.h_try = (float)h;
  c.record = -1;
  dgtd::KclCtl* dc = op->kcl_ctl.p;
  CUDA_TRY(cudaMemcpyAsync(dc, &c, sizeof(c), cudaMemcpyHostToDevice, s));
  float* yd = op->y[op->cur].p;
  CUDA_TRY(cudaMemcpyAsync(op->kcl_bak.p, yd, state_len(op) * 4, cudaMemcpyDeviceToDevice, s));
  DGTD_TRY(kcl_stages(op, dc, yd, -1, nullptr, nullptr));
  DGTD_TRY((to_aos<float, double>(op, yd, op->tmp64.p)));
  CUDA_TRY(cudaMemcpyAsync(y_out, op->tmp64.p, n * 8, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  DGTD_TRY((to_aos<float, double>(op, op->kcl_e.p, op->tmp64.p)));
  CUDA_TRY(cudaMemcpyAsync(err, op->tmp64.p, n * 8, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return check_kernel_flag(op);
}

extern "C" int dgtd_kcl_accepted_steps(dgtd_op* op, float* h, int32_t* frame, int64_t cap, int64_t* n_total) {
  if (!op || cap < 0 || (cap > 0 && (!h || !frame)) || !n_total)
    return set_error(DGTD_ERR_BAD_ARG, "kcl_accepted_steps: bad argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  *n_total = op->kcl_log_n;
  const int64_t n = std::min<int64_t>(std::min<int64_t>(cap, op->kcl_log_n), dgtd::kKclLogCap);
  if (n == 0) return DGTD_OK;
  std::vector<dgtd::KclLogEntry> buf((size_t)n);
  CUDA_TRY(cudaMemcpyAsync(buf.data(), op->kcl_log.p, n * sizeof(dgtd::KclLogEntry), cudaMemcpyDeviceToHost,
                           op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  for (int64_t i = 0; i < n; ++i) {
    h[i] = buf[i].h;
    frame[i] = buf[i].frame;
  }
  return DGTD_OK;
}

extern "C" int dgtd_transient_kcl(dgtd_op* op, const float* y0, float dt, int64_t steps, int drive,
                                  int64_t src_dof, const double* src_vec, const float* g,
                                  const dgtd_kcl_controller* ctl, int record, float* out,
                                  dgtd_kcl_stats* stats) {
  if (!out) return set_error(DGTD_ERR_BAD_ARG, "transient_kcl: null output");
  DGTD_TRY(kcl_args(op, y0, dt, steps, drive, src_vec, ctl, "transient_kcl"));
  DGTD_TRY(dgtd_state_upload(op, y0));
  DevBuf<float> traj;
  if (record) {
    DGTD_TRY(traj.alloc((size_t)(steps + 1) * op->n_dof));
    CUDA_TRY(cudaMemcpyAsync(traj.p, op->y[op->cur].p, op->n_dof * 4, cudaMemcpyDeviceToDevice, op->stream()));
  }
  int st = kcl_run(op, dt, steps, drive, src_dof, g, ctl, record ? traj.p : nullptr, 0, nullptr, nullptr,
                   nullptr, nullptr, stats);
  if (st == DGTD_OK) {
    if (record) {
      std::memcpy(out, y0, op->n_dof * 4);
      DGTD_TRY(op->aos32.alloc(op->n_dof + 4));
      for (int64_t r = 1; r <= steps && st == DGTD_OK; ++r) {
        st = to_aos<float, float>(op, traj.p + r * op->n_dof, op->aos32.p);
        if (st == DGTD_OK) {
          cudaError_t e = cudaMemcpyAsync(out + r * op->n_dof, op->aos32.p, op->n_dof * 4,
                                          cudaMemcpyDeviceToHost, op->stream());
          if (!e) e = cudaStreamSynchronize(op->stream());
          if (e) st = set_error(DGTD_ERR_CUDA, std::string("trajectory download: ") + cudaGetErrorString(e));
        }
      }
    } else {
      st = dgtd_state_download(op, out);
    }
  }
  cudaStreamSynchronize(op->stream());
  traj.free();
  return st;
}

extern "C" int dgtd_transient_kcl_functionals(dgtd_op* op, const float* y0, float dt, int64_t steps, int drive,
                                              int64_t src_dof, const double* src_vec, const float* g,
                                              const dgtd_kcl_controller* ctl, int64_t n_fun,
                                              const int64_t* fun_ptr, const int64_t* fun_idx,
                                              const double* fun_w, double* out, float* y_final,
                                              dgtd_kcl_stats* stats) {
  if (n_fun < 0 || n_fun > 65535 || (n_fun > 0 && (!fun_ptr || !out)))
    return set_error(DGTD_ERR_BAD_ARG, "transient_kcl_functionals: bad functionals");
  DGTD_TRY(kcl_args(op, y0, dt, steps, drive, src_vec, ctl, "transient_kcl_functionals"));
  const int64_t n_terms = n_fun > 0 ? fun_ptr[n_fun] : 0;
  if (n_fun > 0 && fun_ptr[0] != 0) return set_error(DGTD_ERR_BAD_ARG, "fun_ptr[0] must be 0");
  for (int64_t q = 0; q < n_fun; ++q)
    if (fun_ptr[q + 1] < fun_ptr[q]) return set_error(DGTD_ERR_BAD_ARG, "fun_ptr must be non-decreasing");
  if (n_terms > 0 && (!fun_idx || !fun_w)) return set_error(DGTD_ERR_BAD_ARG, "functional terms missing");
  std::vector<int64_t> sidx((size_t)n_terms);
  for (int64_t k = 0; k < n_terms; ++k) {
    if (fun_idx[k] < 0 || fun_idx[k] >= op->n_dof)
      return set_error(DGTD_ERR_BAD_ARG, "functional DOF " + std::to_string(fun_idx[k]) + " out of range");
    sidx[k] = aos_to_soa_index(fun_idx[k], op->np);
  }
  DevBuf<int64_t> d_ptr, d_idx;
  DevBuf<double> d_w, d_out;
  cudaStream_t s = op->stream();
  if (n_fun > 0) {
    DGTD_TRY(d_ptr.alloc(n_fun + 1));
    DGTD_TRY(d_idx.alloc(std::max<int64_t>(n_terms, 1)));
    DGTD_TRY(d_w.alloc(std::max<int64_t>(n_terms, 1)));
    DGTD_TRY(d_out.alloc((size_t)(steps + 1) * n_fun));
    CUDA_TRY(cudaMemcpyAsync(d_ptr.p, fun_ptr, (n_fun + 1) * 8, cudaMemcpyHostToDevice, s));
    if (n_terms > 0) {
      CUDA_TRY(cudaMemcpyAsync(d_idx.p, sidx.data(), n_terms * 8, cudaMemcpyHostToDevice, s));
      CUDA_TRY(cudaMemcpyAsync(d_w.p, fun_w, n_terms * 8, cudaMemcpyHostToDevice, s));
    }
  }
  DGTD_TRY(dgtd_state_upload(op, y0));
  if (n_fun > 0) {
    k_functionals<<<(unsigned)n_fun, 256, 0, s>>>(op->y[op->cur].p, d_ptr.p, d_idx.p, d_w.p, d_out.p);
    CUDA_TRY(cudaGetLastError());
  }
  int st = kcl_run(op, dt, steps, drive, src_dof, g, ctl, nullptr, n_fun, d_ptr.p, d_idx.p, d_w.p, d_out.p, stats);
  if (st == DGTD_OK && n_fun > 0) {
    cudaError_t e = cudaMemcpyAsync(out, d_out.p, (size_t)(steps + 1) * n_fun * 8, cudaMemcpyDeviceToHost, s);
    if (e) st = set_error(DGTD_ERR_CUDA, std::string("functional download: ") + cudaGetErrorString(e));
  }
  if (st == DGTD_OK && y_final) st = dgtd_state_download(op, y_final);
  cudaStreamSynchronize(s);
  d_ptr.free(); d_idx.free(); d_w.free(); d_out.free();
  return st;
}

// ------------------------------------------------------------------ Krylov

namespace {

// Krylov buffers of basis type B: the basis slots 1..chunk, two chunk
// vectors (sub-step input/output) and the source column b, all SoA of
// state_len (whole tensor-core tiles, zero padding).
template <class B>
struct KryBufs {
  DevBuf<B>* basis;
  DevBuf<B>* vec;  // [2]
  DevBuf<B>* b;
};
template <class B>
KryBufs<B> kry_bufs(dgtd_op* op) {
  if constexpr (sizeof(B) == 4)
    return {&op->kbasis32, op->kvec32, &op->kb32};
  else
    return {&op->kbasis64, op->kvec64, &op->kb64};
}

template <class B>
int ensure_krylov(dgtd_op* op, int chunk) {
  if (chunk < 1 || chunk > dgtd::kKryMaxChunk)
    return set_error(DGTD_ERR_UNSUPPORTED, "Krylov chunk dimension outside 1..12");
  const size_t len = state_len(op);
  cudaStream_t s = op->stream();
  KryBufs<B> kb = kry_bufs<B>(op);
  if (kb.basis->n < (size_t)chunk * len) {
    DGTD_TRY(kb.basis->alloc((size_t)chunk * len));
    CUDA_TRY(cudaMemsetAsync(kb.basis->p, 0, kb.basis->n * sizeof(B), s));
  }
  for (int i = 0; i < 2; ++i)
    if (kb.vec[i].n < len) {
      DGTD_TRY(kb.vec[i].alloc(len));
      CUDA_TRY(cudaMemsetAsync(kb.vec[i].p, 0, len * sizeof(B), s));
    }
  if (kb.b->n < len) {
    DGTD_TRY(kb.b->alloc(len));
    CUDA_TRY(cudaMemsetAsync(kb.b->p, 0, len * sizeof(B), s));
  }
  DGTD_TRY(op->partials.alloc((size_t)2 * dgtd::kKrylovBlocks * dgtd::kKryRow));
  DGTD_TRY(op->kst.alloc(1));
  DGTD_TRY(op->skip.alloc(1));
  DGTD_TRY(op->kpoly.alloc(dgtd::kAugMax));
  DGTD_TRY(op->tmp64.alloc(op->n_dof));
  static bool attr[8] = {false};  // kernel attributes are per device
  if (!attr[op->ctx->device & 7]) {
    CUDA_TRY(cudaFuncSetAttribute(dgtd::k_kry_finish_norm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dgtd::kExpmSmem));
    CUDA_TRY(cudaFuncSetAttribute(dgtd::k_kry_finish_coef, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dgtd::kExpmSmem));
    CUDA_TRY(cudaFuncSetAttribute(dgtd::k_expm_dense, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dgtd::kExpmSmem));
    attr[op->ctx->device & 7] = true;
  }
  return DGTD_OK;
}

// w = kry[0] * A v + kry[1] * b on the op's engine (f32 basis) or the FP64 path.
template <class B>
int kry_matvec(dgtd_op* op, const B* v, B* w, const B* bvec, int64_t src_idx, const double* kry, const int* skip) {
  if constexpr (sizeof(B) == 4) {
    RhsParams P = base_params(op);
    P.y_in = v;
    P.out = w;
    P.src_vec = bvec;
    P.src_idx = src_idx;
    P.kry = kry;
    P.skip = skip;
    return launch_rhs<kModeKrylov>(op, P);
  } else {
    RhsParamsT<double> P = base_params64(op);
    P.y_in = v;
    P.out = w;
    P.src_vec = bvec;
    P.src_idx = src_idx;
    P.kry = kry;
    P.skip = skip;
    return launch_rhs64<kModeKrylov>(op, P);
  }
}

// Debug builds (-DDGTD_KRY_TRACE): synchronise after every Krylov launch and
// report it on stderr.
#ifdef DGTD_KRY_TRACE
#define KRY_TRACE(what, j)                                                                       \
  do {                                                                                         \
    cudaError_t e__ = cudaStreamSynchronize(s);                                                \
    std::fprintf(stderr, "kry %s j=%d: %s\n", what, (int)(j), cudaGetErrorString(e__));         \
  } while (0)
#else
#define KRY_TRACE(what, j) \
  do {                     \
  } while (0)
#endif

// One Arnoldi chunk from the SoA vector v (basis slot 0) into `out`: the
// first n components of exp(t*Aug)[v; e_{P-1}/eta] (P > 0, the source
// polynomial's coefficients in op->kpoly, shifted by `delta`) or exp(t*A) v
// (P = 0).  The chunk's dimension and estimate are accumulated on the device
// (KrylovDev::dim_total, est_sum); `first` starts a new accumulation, in
// abort mode when abort_chunks > 0 (see k_kry_finish_coef).
template <class B>
int krylov_chunk(dgtd_op* op, const B* v, double t, int m, double tol, int P, double delta, const B* bvec,
                 int64_t src_idx, B* out, bool first, int abort_chunks) {
  using namespace dgtd;
  cudaStream_t s = op->stream();
  // a part of a partition reduces over its owned elements (the prefix of the
  // element-major layout) and sums its partials with the other parts
  const bool parted = op->part_owned > 0;
  if (parted && sizeof(B) != 4) return set_error(DGTD_ERR_UNSUPPORTED, "partitioned Krylov needs the f32 basis");
  const int64_t n = parted ? op->part_owned * 6 * op->np : op->n_dof;
  const int64_t len = (int64_t)state_len(op);
  const int nb = kKrylovBlocks, nt = kKrylovThreads;
  const int gs = grid_for(n, 256, op->ctx->num_sms);
  KrylovDev* st = op->kst.p;
  B* vb = kry_bufs<B>(op).basis->p;
  double* pa = op->partials.p;
  double* pb = pa + (size_t)kKrylovBlocks * kKryRow;
  const int64_t n_part = (int64_t)kKrylovBlocks * kKryRow;
  auto psum = [&](double* buf) -> int {
    if (parted && op->part_sum(op->part_user, buf, n_part) != 0)
      return set_error(DGTD_ERR_CUDA, "partitioned Krylov: the sum hook failed");
    return DGTD_OK;
  };
  auto phalo = [&](const B* vec) -> int {
    if (parted && op->part_halo(op->part_user, (float*)const_cast<B*>(vec)) != 0)
      return set_error(DGTD_ERR_CUDA, "partitioned Krylov: the halo hook failed");
    return DGTD_OK;
  };
  if (first) {
    struct {
      int dim_total, est_none;
      double est_sum;
      int aborted, abort_chunks;
    } acc = {0, 0, 0.0, 0, abort_chunks};
    static_assert(sizeof(acc) == offsetof(KrylovDev, abort_chunks) + sizeof(int) - offsetof(KrylovDev, dim_total),
                  "accumulator layout");
    CUDA_TRY(cudaMemcpyAsync(&st->dim_total, &acc, sizeof(acc), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));  // acc is on the host stack
  }
  k_kry_norm_partials<B><<<nb, nt, 0, s>>>(v, n, pa);
  KRY_TRACE("norm_partials", -1);
  DGTD_TRY(psum(pa));
  k_kry_start<<<1, kExpmThreads, 0, s>>>(st, pa, nb, t, tol, P, op->kpoly.p, delta, m, op->skip.p);
  KRY_TRACE("start", -1);
  op->launches += 2;
  CUDA_TRY(cudaGetLastError());
  for (int j = 0; j < m; ++j) {
    B* w = vb + (int64_t)j * len;  // slot j + 1
    const B* vj = kry_col(v, (const B*)vb, len, j);
    DGTD_TRY(phalo(vj));
    DGTD_TRY(kry_matvec<B>(op, vj, w, bvec, src_idx, st->mv, op->skip.p));
    KRY_TRACE("matvec", j);
    k_kry_dots<B><<<nb, nt, 0, s>>>(v, vb, len, n, j + 1, w, pa, op->skip.p);
    KRY_TRACE("dots", j);
    DGTD_TRY(psum(pa));
    // the sweeps' register-held columns: the smallest of 4, 8, 12 covering j + 1
    if (j < 4) {
      k_kry_update_dots<B, 4><<<nb, nt, 0, s>>>(st, v, vb, len, n, j, w, pa, nb, pb, op->skip.p);
    } else if (j < 8) {
      k_kry_update_dots<B, 8><<<nb, nt, 0, s>>>(st, v, vb, len, n, j, w, pa, nb, pb, op->skip.p);
    } else {
      k_kry_update_dots<B, kKryCols><<<nb, nt, 0, s>>>(st, v, vb, len, n, j, w, pa, nb, pb, op->skip.p);
    }
    KRY_TRACE("update_dots", j);
    DGTD_TRY(psum(pb));
    if (j < 4) {
      k_kry_update_norm<B, 4><<<nb, nt, 0, s>>>(st, v, vb, len, n, j, w, pb, nb, pa, op->skip.p);
    } else if (j < 8) {
      k_kry_update_norm<B, 8><<<nb, nt, 0, s>>>(st, v, vb, len, n, j, w, pb, nb, pa, op->skip.p);
    } else {
      k_kry_update_norm<B, kKryCols><<<nb, nt, 0, s>>>(st, v, vb, len, n, j, w, pb, nb, pa, op->skip.p);
    }
    KRY_TRACE("update_norm", j);
    DGTD_TRY(psum(pa));
    k_kry_finish_norm<<<1, kExpmThreads, kExpmSmem, s>>>(st, pa, nb, j, op->skip.p);
    KRY_TRACE("finish_norm", j);
    op->launches += 4;
    CUDA_TRY(cudaGetLastError());
  }
  k_kry_finish_coef<<<1, kExpmThreads, kExpmSmem, s>>>(st);
  KRY_TRACE("finish_coef", -1);
  k_kry_lincomb<B><<<nb, nt, 0, s>>>(v, vb, len, n, st, out);
  KRY_TRACE("lincomb", -1);
  op->launches += 2;
  CUDA_TRY(cudaGetLastError());
  return DGTD_OK;
}

// KRYLOV_CHUNK sub-stepping (gpu/operator.rs:1175-1197, :1267-1291): k =
// ceil(m/12) chunks of dimension ceil(m/k), each over t/k.  From the SoA
// vector `in` (not modified) into `out` (may not alias `in`).  With split_tol
// each sub-step runs to tol/k, so that the summed estimate of a step whose
// sub-steps all converged stays within tol, and a sub-step that misses tol/k
// ends the step (the later sub-steps are skipped and the estimate reported is
// that sub-step's times k, above tol): a step that will be rejected costs one
// sub-step.  dim/est (may be null) receive the summed dimension and estimate
// (-1 when no estimate was formed).
template <class B>
int krylov_steps(dgtd_op* op, const B* in, B* out, double t, int m, double tol, int P, const B* bvec,
                 int64_t src_idx, bool split_tol, int* dim, double* est) {
  const int kchunk = 12;
  const int k = std::max(1, (m + kchunk - 1) / kchunk);
  const int chunk = (m + k - 1) / k;
  DGTD_TRY(ensure_krylov<B>(op, chunk));
  B* mid = kry_bufs<B>(op).vec[1].p;
  const double tau = t / (double)k;
  const B* cur = in;
  for (int q = 0; q < k; ++q) {
    B* dst = ((k - 1 - q) % 2 == 0) ? out : mid;
    DGTD_TRY(krylov_chunk<B>(op, cur, tau, chunk, split_tol ? tol / (double)k : tol, P, q * tau, bvec, src_idx, dst,
                             q == 0, split_tol ? k : 0));
    cur = dst;
  }
  if (dim || est) {
    struct {
      int dim_total, est_none;
      double est_sum;
    } acc;
    CUDA_TRY(cudaMemcpyAsync(&acc, &op->kst.p->dim_total, sizeof(acc), cudaMemcpyDeviceToHost, op->stream()));
    CUDA_TRY(cudaStreamSynchronize(op->stream()));
    if (dim) *dim = acc.dim_total;
    if (est) *est = acc.est_none ? -1.0 : acc.est_sum;
  }
  return DGTD_OK;
}

int set_poly(dgtd_op* op, int P, const double* a) {
  if (P < 0 || P > dgtd::kAugMax) return set_error(DGTD_ERR_BAD_ARG, "source polynomial: 0..8 coefficients");
  for (int q = 0; q < P; ++q)
    if (!std::isfinite(a[q])) return set_error(DGTD_ERR_BAD_ARG, "source polynomial: non-finite coefficient");
  double buf[dgtd::kAugMax] = {0};
  for (int q = 0; q < P; ++q) buf[q] = a[q];
  CUDA_TRY(cudaMemcpyAsync(op->kpoly.p, buf, sizeof(buf), cudaMemcpyHostToDevice, op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));  // buf is on the host stack
  return DGTD_OK;
}

// Host API: exp(t*A)v, or the ETD step with the source b*g(t0+tau), g a
// polynomial of P coefficients (host f64 AoS in and out).
template <class B>
int krylov_run_t(dgtd_op* op, const double* v_host, const double* b_host, int P, const double* a, double t, int m,
                 double tol, double* out_host, int* dim_used, double* est_sum, bool split_tol) {
  cudaStream_t s = op->stream();
  const int64_t n = op->n_dof;
  const int k = std::max(1, (m + 11) / 12);
  DGTD_TRY(ensure_krylov<B>(op, (m + k - 1) / k));
  KryBufs<B> kb = kry_bufs<B>(op);
  CUDA_TRY(cudaMemcpyAsync(op->tmp64.p, v_host, n * 8, cudaMemcpyHostToDevice, s));
  DGTD_TRY((to_soa<double, B>(op, op->tmp64.p, kb.vec[0].p)));
  const B* bvec = nullptr;
  if (b_host) {
    CUDA_TRY(cudaStreamSynchronize(s));  // tmp64 is reused
    CUDA_TRY(cudaMemcpyAsync(op->tmp64.p, b_host, n * 8, cudaMemcpyHostToDevice, s));
    DGTD_TRY((to_soa<double, B>(op, op->tmp64.p, kb.b->p)));
    bvec = kb.b->p;
  }
  DGTD_TRY(set_poly(op, b_host ? P : 0, a));
  // the result: a buffer of state_len doubles holds either basis type; it is
  // also an intermediate sub-step's input, so its padding must be zero (and a
  // run of the other basis type may have left values there)
  DGTD_TRY(op->kout64.alloc(state_len(op)));
  CUDA_TRY(cudaMemsetAsync(op->kout64.p, 0, state_len(op) * 8, s));
  B* dst = reinterpret_cast<B*>(op->kout64.p);
  int d = 0;
  double e = -1.0;
  DGTD_TRY(krylov_steps<B>(op, kb.vec[0].p, dst, t, m, tol, b_host ? P : 0, bvec, -1, split_tol, &d, &e));
  DGTD_TRY((to_aos<B, double>(op, dst, op->tmp64.p)));
  CUDA_TRY(cudaMemcpyAsync(out_host, op->tmp64.p, n * 8, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (dim_used) *dim_used = d;
  if (est_sum) *est_sum = e;
  return check_kernel_flag(op);
}

int krylov_run(dgtd_op* op, const double* v_host, const double* b_host, int P, const double* a, double t, int m,
               double tol, double* out_host, int* dim_used, double* est_sum = nullptr, bool split_tol = false) {
  if (m < 1) return set_error(DGTD_ERR_BAD_ARG, "Krylov dimension must be >= 1");
  if (!std::isfinite(t)) return set_error(DGTD_ERR_BAD_ARG, "Krylov time must be finite");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  if (op->krylov_fp64)
    return krylov_run_t<double>(op, v_host, b_host, P, a, t, m, tol, out_host, dim_used, est_sum, split_tol);
  return krylov_run_t<float>(op, v_host, b_host, P, a, t, m, tol, out_host, dim_used, est_sum, split_tol);
}

}  // namespace

extern "C" int dgtd_op_set_krylov_precision(dgtd_op* op, int bits) {
  if (!op || (bits != 32 && bits != 64)) return set_error(DGTD_ERR_BAD_ARG, "set_krylov_precision: 32 or 64");
  op->krylov_fp64 = bits == 64;
  return DGTD_OK;
}

extern "C" int dgtd_expmv(dgtd_op* op, const double* v, double t, int32_t m, double tol, double* out,
                          int32_t* dim_used) {
  if (!op || !v || !out) return set_error(DGTD_ERR_BAD_ARG, "expmv: null argument");
  int d = 0;
  DGTD_TRY(krylov_run(op, v, nullptr, 0, nullptr, t, m, tol, out, &d));
  if (dim_used) *dim_used = d;
  return DGTD_OK;
}

extern "C" int dgtd_etd_step(dgtd_op* op, const double* y, const double* b, double h, int32_t m,
                             double tol, double* out, int32_t* dim_used) {
  if (!op || !y || !b || !out) return set_error(DGTD_ERR_BAD_ARG, "etd_step: null argument");
  const double one = 1.0;
  int d = 0;
  DGTD_TRY(krylov_run(op, y, b, 1, &one, h, m, tol, out, &d));
  if (dim_used) *dim_used = d;
  return DGTD_OK;
}

extern "C" int dgtd_etd_step_est(dgtd_op* op, const double* y, const double* b, double h, int32_t m,
                                 double tol, double* out, int32_t* dim_used, double* est) {
  if (!op || !y || !b || !out || !est) return set_error(DGTD_ERR_BAD_ARG, "etd_step_est: null argument");
  if (!(tol > 0.0)) return set_error(DGTD_ERR_BAD_ARG, "etd_step_est: the estimate needs tol > 0");
  const double one = 1.0;
  int d = 0;
  DGTD_TRY(krylov_run(op, y, b, 1, &one, h, m, tol, out, &d, est, true));
  if (dim_used) *dim_used = d;
  return DGTD_OK;
}

extern "C" int dgtd_etd_step_poly(dgtd_op* op, const double* y, const double* b, int32_t n_coef,
                                  const double* coef, double h, int32_t m, double tol, double* out,
                                  int32_t* dim_used, double* est) {
  if (!op || !y || !b || !out || (n_coef > 0 && !coef) || n_coef < 1)
    return set_error(DGTD_ERR_BAD_ARG, "etd_step_poly: bad argument");
  int d = 0;
  double e = -1.0;
  DGTD_TRY(krylov_run(op, y, b, n_coef, coef, h, m, tol, out, &d, &e, tol > 0.0));
  if (dim_used) *dim_used = d;
  if (est) *est = e;
  return DGTD_OK;
}

// ETD steps on the resident f32 state: the candidate lands in the other state
// buffer and becomes the state on dgtd_etd_commit.
extern "C" int dgtd_etd_try(dgtd_op* op, double h, int32_t m, double tol, int32_t n_coef, const double* coef,
                            int drive, int64_t src_dof, int32_t* dim_used, double* est) {
  if (!op || m < 1 || n_coef < 0 || (n_coef > 0 && !coef)) return set_error(DGTD_ERR_BAD_ARG, "etd_try: bad argument");
  if (!(std::isfinite(h) && h > 0.0)) return set_error(DGTD_ERR_BAD_ARG, "etd_try: step must be positive");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  int64_t src_idx = -1;
  const float* bvec = nullptr;
  int P = n_coef;
  if (drive == DGTD_DRIVE_POINT) {
    // a part of a partition without the source DOF drives nothing locally
    const bool elsewhere = src_dof == -1 && op->part_owned > 0;
    if (!elsewhere && (src_dof < 0 || src_dof >= op->n_dof))
      return set_error(DGTD_ERR_BAD_ARG, "etd_try: source DOF out of range");
    src_idx = elsewhere ? -1 : aos_to_soa_index(src_dof, op->np);
  } else if (drive == DGTD_DRIVE_VECTOR) {
    if (!op->src_vec_set) return set_error(DGTD_ERR_BAD_ARG, "etd_try: vector drive without a source vector");
    bvec = op->src_vec.p;
  } else if (drive == DGTD_DRIVE_FREE) {
    P = 0;
  } else {
    return set_error(DGTD_ERR_BAD_ARG, "etd_try: unknown drive kind");
  }
  if (drive != DGTD_DRIVE_FREE && P < 1) return set_error(DGTD_ERR_BAD_ARG, "etd_try: a driven step needs coefficients");
  const int k = std::max(1, (m + 11) / 12);
  DGTD_TRY(ensure_krylov<float>(op, (m + k - 1) / k));
  DGTD_TRY(set_poly(op, P, coef));
  int d = 0;
  double e = -1.0;
  DGTD_TRY(krylov_steps<float>(op, op->y[op->cur].p, op->y[op->cur ^ 1].p, h, m, tol, P, bvec, src_idx, tol > 0.0,
                               &d, &e));
  if (dim_used) *dim_used = d;
  if (est) *est = e;
  return check_kernel_flag(op);
}

extern "C" int dgtd_etd_commit(dgtd_op* op) {
  if (!op) return set_error(DGTD_ERR_BAD_ARG, "etd_commit: null op");
  op->cur ^= 1;
  return DGTD_OK;
}

// Dense exp(A) on the device (d <= 64), for tests of the Hessenberg exponential.
extern "C" int dgtd_debug_expm(dgtd_ctx* ctx, const double* a, int32_t d, double* out) {
  if (!ctx || !a || !out || d < 1 || d > dgtd::kKrylovMaxDim) return set_error(DGTD_ERR_BAD_ARG, "debug_expm: bad argument");
  CUDA_TRY(cudaSetDevice(ctx->device));
  DevBuf<double> da, dout;
  DGTD_TRY(da.alloc((size_t)d * d));
  DGTD_TRY(dout.alloc((size_t)d * d));
  CUDA_TRY(cudaFuncSetAttribute(dgtd::k_expm_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dgtd::kExpmSmem));
  CUDA_TRY(cudaMemcpyAsync(da.p, a, (size_t)d * d * 8, cudaMemcpyHostToDevice, ctx->stream));
  dgtd::k_expm_dense<<<1, dgtd::kExpmThreads, dgtd::kExpmSmem, ctx->stream>>>(da.p, d, dout.p);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(out, dout.p, (size_t)d * d * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  da.free();
  dout.free();
  return DGTD_OK;
}

// ------------------------------------------------------------------ session helpers

namespace {

__global__ void k_norm2_f32(const float* __restrict__ x, int64_t n, double* __restrict__ partials) {
  __shared__ double acc[8];
  double sq = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double v = x[k];
    sq += v * v;
  }
  sq = dgtd::warp_sum(sq);
  if ((threadIdx.x & 31) == 0) acc[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += acc[q];
    partials[blockIdx.x] = t;
  }
}

__global__ void k_all_finite_f32(const float* __restrict__ x, int64_t n, int* __restrict__ bad) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(x[k])) { *bad = 1; return; }
}

__global__ void k_scale_f32(const float* __restrict__ x, int64_t n, float s, float* __restrict__ out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    out[k] = x[k] * s;
}

// One warp per element: 1/2 |det J| sum_c w_c f_c^T M f_c (rhs.rs:1509-1544).
template <class T>
__global__ void k_energy(const T* __restrict__ y, const double* __restrict__ mass, const double* __restrict__ absdet,
                         const float* __restrict__ meta, int64_t n_elem, int np, double* __restrict__ partials) {
  extern __shared__ double sMass[];
  __shared__ double acc[8];
  for (int i = threadIdx.x; i < np * np; i += blockDim.x) sMass[i] = mass[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double local = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * nw + warp; e < n_elem; e += (int64_t)gridDim.x * nw) {
    const T* Y = y + e * 6 * np;
    const float* M = meta + e * dgtd::kMetaWords;
    double w[6];
    for (int c = 0; c < 3; ++c) {
      w[c] = 1.0 / (double)M[25 + c];
      w[3 + c] = 1.0 / (double)M[28 + c];
    }
    double el = 0.0;
    for (int i = lane; i < np; i += 32)
      for (int c = 0; c < 6; ++c) {
        double t = 0.0;
        for (int j = 0; j < np; ++j) t += sMass[i * np + j] * (double)Y[c * np + j];
        el += w[c] * (double)Y[c * np + i] * t;
      }
    local += absdet[e] * el;
  }
  local = dgtd::warp_sum(local);
  if (lane == 0) acc[warp] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < nw; ++q) t += acc[q];
    partials[blockIdx.x] = t;
  }
}

constexpr int kRedBlocks = 296;

int norm2_f32(dgtd_op* op, const float* x, double* out) {
  DGTD_TRY(op->partials.alloc((size_t)dgtd::kKrylovBlocks * dgtd::kKrylovMaxDim));
  k_norm2_f32<<<kRedBlocks, 256, 0, op->stream()>>>(x, op->n_dof, op->partials.p);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  std::vector<double> h(kRedBlocks);
  CUDA_TRY(cudaMemcpyAsync(h.data(), op->partials.p, kRedBlocks * 8, cudaMemcpyDeviceToHost, op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  double t = 0.0;
  for (double v : h) t += v;
  *out = std::sqrt(t);
  return DGTD_OK;
}

// Deterministic standard normals, splitmix64 + Box-Muller (session.rs:415-431).
void normal_vector(std::vector<double>& out, uint64_t seed) {
  uint64_t state = seed;
  auto uniform = [&]() {
    state += 0x9e3779b97f4a7c15ULL;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return (double(z >> 11) + 0.5) / double(1ULL << 53);
  };
  for (auto& v : out) {
    const double u = uniform(), w = uniform();
    v = std::sqrt(-2.0 * std::log(u)) * std::cos(2.0 * 3.14159265358979323846 * w);
  }
}

// Power iteration on the resident SoA state slot `v` (normalised in place);
// `tmp` receives A v.  Returns rho of the last iteration.
int power_iterate(dgtd_op* op, float* v, float* tmp, int iters, double* rho) {
  double r = 1.0;
  for (int it = 0; it < iters; ++it) {
    RhsParams P = base_params(op);
    P.y_in = v;
    P.out = tmp;
    DGTD_TRY(launch_rhs<kModeApply>(op, P));
    DGTD_TRY(norm2_f32(op, tmp, &r));
    if (!(r > 0.0) || !std::isfinite(r)) return set_error(DGTD_ERR_NONFINITE, "power iteration: norm is zero or non-finite");
    k_scale_f32<<<grid_for(op->n_dof, 256, op->ctx->num_sms), 256, 0, op->stream()>>>(tmp, op->n_dof, (float)(1.0 / r), v);
    op->launches++;
    CUDA_TRY(cudaGetLastError());
  }
  *rho = r;
  return DGTD_OK;
}

int start_vector(dgtd_op* op, float* soa) {
  std::vector<double> v((size_t)op->n_dof);
  normal_vector(v, 0);
  double nrm = 0.0;
  for (double x : v) nrm += x * x;
  nrm = 1.0 / std::sqrt(nrm);
  std::vector<float> f(v.size());
  for (size_t i = 0; i < v.size(); ++i) f[i] = (float)(v[i] * nrm);
  DGTD_TRY(op->aos32.alloc(op->n_dof + 4));
  CUDA_TRY(cudaMemcpyAsync(op->aos32.p, f.data(), op->n_dof * 4, cudaMemcpyHostToDevice, op->stream()));
  DGTD_TRY((to_soa<float, float>(op, op->aos32.p, soa)));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  return DGTD_OK;
}

}  // namespace

extern "C" int dgtd_power_rho(dgtd_op* op, int32_t iters, double* rho) {
  if (!op || !rho || iters < 1) return set_error(DGTD_ERR_BAD_ARG, "power_rho: bad argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DevBuf<float> v, t;
  DGTD_TRY(v.alloc(state_len(op)));
  DGTD_TRY(t.alloc(state_len(op)));
  CUDA_TRY(cudaMemsetAsync(v.p, 0, state_len(op) * 4, op->stream()));
  CUDA_TRY(cudaMemsetAsync(t.p, 0, state_len(op) * 4, op->stream()));
  int st = start_vector(op, v.p);
  if (st == DGTD_OK) st = power_iterate(op, v.p, t.p, iters, rho);
  cudaStreamSynchronize(op->stream());
  v.free();
  t.free();
  return st;
}

extern "C" int dgtd_cfl_dt(dgtd_op* op, double* h_out, double* rho_out, double* z_out) {
  if (!op) return set_error(DGTD_ERR_BAD_ARG, "cfl_dt: null op");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DevBuf<float> probe, tmp;
  DevBuf<int> bad;
  DGTD_TRY(probe.alloc(state_len(op)));
  DGTD_TRY(tmp.alloc(state_len(op)));
  CUDA_TRY(cudaMemsetAsync(probe.p, 0, state_len(op) * 4, op->stream()));
  CUDA_TRY(cudaMemsetAsync(tmp.p, 0, state_len(op) * 4, op->stream()));
  DGTD_TRY(bad.alloc(1));
  double rho = 0.0;
  int st = start_vector(op, probe.p);
  if (st == DGTD_OK) st = power_iterate(op, probe.p, tmp.p, 40, &rho);
  if (st != DGTD_OK) return st;
  double n0 = 0.0;
  DGTD_TRY(norm2_f32(op, probe.p, &n0));
  // Probe: 64 LSERK4 steps of z/rho from the dominant vector on the resident
  // state; stable when finite, norm <= 10 n0 and rate <= 1 + 1e-3.
  auto stable = [&](double z, bool* ok) -> int {
    const float h = (float)(z / rho);
    CUDA_TRY(cudaMemcpyAsync(op->y[op->cur].p, probe.p, op->n_dof * 4, cudaMemcpyDeviceToDevice, op->stream()));
    for (int s = 0; s < 64; ++s) DGTD_TRY(lserk_step(op, h, -1, 0.f, nullptr));
    CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), op->stream()));
    k_all_finite_f32<<<grid_for(op->n_dof, 256, op->ctx->num_sms), 256, 0, op->stream()>>>(op->y[op->cur].p, op->n_dof, bad.p);
    op->launches++;
    CUDA_TRY(cudaGetLastError());
    int hb = 0;
    CUDA_TRY(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, op->stream()));
    CUDA_TRY(cudaStreamSynchronize(op->stream()));
    if (hb) { *ok = false; return DGTD_OK; }
    double nf = 0.0;
    DGTD_TRY(norm2_f32(op, op->y[op->cur].p, &nf));
    if (!std::isfinite(nf) || nf > 10.0 * n0) { *ok = false; return DGTD_OK; }
    const double rate = nf > 0.0 ? std::pow(nf / n0, 1.0 / 64.0) : 0.0;
    *ok = rate <= 1.0 + 1e-3;
    return DGTD_OK;
  };
  double lo = 3.0, hi = 15.0;
  bool ok = false;
  for (;;) { DGTD_TRY(stable(lo, &ok)); if (ok || !(lo > 0.1)) break; lo *= 0.5; }
  for (;;) { DGTD_TRY(stable(hi, &ok)); if (!ok || !(hi < 1e3)) break; hi *= 1.5; }
  for (int it = 0; it < 7; ++it) {
    const double mid = 0.5 * (lo + hi);
    DGTD_TRY(stable(mid, &ok));
    if (ok) lo = mid; else hi = mid;
  }
  probe.free(); tmp.free(); bad.free();
  if (h_out) *h_out = 0.8 * lo / rho;
  if (rho_out) *rho_out = rho;
  if (z_out) *z_out = lo;
  return DGTD_OK;
}

template <class T>
static int energy_of(dgtd_op* op, const T* y_soa, double* energy) {
  if (!op->has_mass) return set_error(DGTD_ERR_UNSUPPORTED, "energy: operator created without the mass matrix");
  DGTD_TRY(op->partials.alloc((size_t)dgtd::kKrylovBlocks * dgtd::kKrylovMaxDim));
  const size_t sm = (size_t)op->np * op->np * 8;
  static bool attr[8] = {false};  // kernel attributes are per device
  if (!attr[op->ctx->device & 7]) {
    CUDA_TRY(cudaFuncSetAttribute(k_energy<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    attr[op->ctx->device & 7] = true;
  }
  k_energy<T><<<kRedBlocks, 256, sm, op->stream()>>>(y_soa, op->mass.p, op->absdet.p, op->meta.p, op->n_elem,
                                                     op->np, op->partials.p);
  op->launches++;
  CUDA_TRY(cudaGetLastError());
  std::vector<double> h(kRedBlocks);
  CUDA_TRY(cudaMemcpyAsync(h.data(), op->partials.p, kRedBlocks * 8, cudaMemcpyDeviceToHost, op->stream()));
  CUDA_TRY(cudaStreamSynchronize(op->stream()));
  double t = 0.0;
  for (double v : h) t += v;
  *energy = 0.5 * t;
  return DGTD_OK;
}

extern "C" int dgtd_field_energy(dgtd_op* op, const double* y, double* energy) {
  if (!op || !y || !energy) return set_error(DGTD_ERR_BAD_ARG, "field_energy: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  DGTD_TRY(op->tmp64.alloc(op->n_dof));
  DGTD_TRY(op->vin64.alloc(op->n_dof));
  CUDA_TRY(cudaMemcpyAsync(op->tmp64.p, y, op->n_dof * 8, cudaMemcpyHostToDevice, op->stream()));
  DGTD_TRY((to_soa<double, double>(op, op->tmp64.p, op->vin64.p)));
  return energy_of<double>(op, op->vin64.p, energy);
}

extern "C" int dgtd_state_energy(dgtd_op* op, double* energy) {
  if (!op || !energy) return set_error(DGTD_ERR_BAD_ARG, "state_energy: null argument");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  return energy_of<float>(op, op->y[op->cur].p, energy);
}

// ------------------------------------------------------------------ no-allocation LSERK4
//
// A variant of the fused LSERK4 stage path for callers that must not have the
// library allocate device memory: hosts whose framework owns the device memory
// budget (a caching allocator that has reserved the GPU, a fixed-budget service
// that forbids allocations after start-up) and so cannot let a library call
// cudaMalloc / cudaFree.  The caller passes the input and output states; the
// scratch this path needs -- two element-major SoA state buffers that the
// stages ping-pong between and the LSERK residual register p -- is the
// file-scope array below.  It is sized for at most kStaticMaxDof degrees of
// freedom, and every GPU that loads this library holds it (24 MiB) until the
// process exits.

namespace {
constexpr int64_t kStaticMaxDof = int64_t(1) << 21;  // 2,097,152 DOFs
static __device__ __align__(256) float g_lserk_scratch[3 * kStaticMaxDof];
std::mutex g_lserk_scratch_mu;
float* g_lserk_scratch_ptr[64] = {nullptr};

// Device address of g_lserk_scratch on the current device.  In host code the
// symbol names a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, taken once per device with that device current.
int lserk_scratch(int device, float** out) {
  if (device < 0 || device >= 64) return set_error(DGTD_ERR_BAD_ARG, "run_lserk_static: device index above 63");
  std::lock_guard<std::mutex> lock(g_lserk_scratch_mu);
  if (!g_lserk_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_lserk_scratch);
    if (e != cudaSuccess || !p)
      return set_error(DGTD_ERR_CUDA, std::string("run_lserk_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_lserk_scratch_ptr[device] = static_cast<float*>(p);
  }
  *out = g_lserk_scratch_ptr[device];
  return DGTD_OK;
}
}  // namespace

extern "C" int dgtd_run_lserk_static(dgtd_op* op, const float* d_y_in, float* d_y_out, float h, int64_t steps) {
  if (!op || !d_y_in || !d_y_out || steps < 0) return set_error(DGTD_ERR_BAD_ARG, "run_lserk_static: bad argument");
  if (!(std::isfinite(h) && h > 0.f)) return set_error(DGTD_ERR_BAD_ARG, "run_lserk_static: step must be positive");
  const int64_t padded = op->n_elem_pad * 6 * op->np;  // the kernels touch whole tiles
  if (padded > kStaticMaxDof)
    return set_error(DGTD_ERR_BAD_ARG, "run_lserk_static: the op's state padded to whole tiles (" +
                                           std::to_string(op->n_elem_pad) + " elements x " +
                                           std::to_string(6 * op->np) + " = " + std::to_string(padded) +
                                           " values, n_dof " + std::to_string(op->n_dof) +
                                           ") exceeds the static scratch limit of " + std::to_string(kStaticMaxDof) +
                                           " values; use dgtd_run_lserk");
  CUDA_TRY(cudaSetDevice(op->ctx->device));
  float* base = nullptr;
  DGTD_TRY(lserk_scratch(op->ctx->device, &base));
  // The residual register is written before it is read in every step (stage
  // 0 has a = 0 and does not read it), so nothing left by an earlier call is
  // ever used and no clearing is needed.
  float* ya = base;
  float* yb = base + kStaticMaxDof;
  float* pr = base + 2 * kStaticMaxDof;
  if (padded > op->n_dof) {
    // the padding of whole tiles must hold finite values (zeros)
    CUDA_TRY(cudaMemsetAsync(ya + op->n_dof, 0, (padded - op->n_dof) * 4, op->stream()));
    CUDA_TRY(cudaMemsetAsync(yb + op->n_dof, 0, (padded - op->n_dof) * 4, op->stream()));
  }
  DGTD_TRY((to_soa<float, float>(op, d_y_in, ya)));
  for (int64_t k = 0; k < steps; ++k)
    for (int s = 0; s < 5; ++s) {
      RhsParams P = base_params(op);
      P.y_in = ya;
      P.out = yb;
      P.p = pr;
      P.a = (float)kLserkA[s];
      P.b = (float)kLserkB[s];
      P.dt = h;
      P.read_p = s > 0;
      P.write_p = s < 4;
      DGTD_TRY(launch_rhs<kModeLserk>(op, P));
      std::swap(ya, yb);
    }
  return to_aos<float, float>(op, ya, d_y_out);
}

// ------------------------------------------------------------------ bounded-wait test hook

extern "C" int dgtd_debug_wait_timeout(dgtd_ctx* ctx, int64_t max_polls, double* waited_s) {
  if (!ctx || max_polls < 1 || max_polls > (int64_t)kTcWaitLimit)
    return set_error(DGTD_ERR_BAD_ARG, "debug_wait_timeout: 1 <= max_polls <= the kernels' own limit (2^19)");
  CUDA_TRY(cudaSetDevice(ctx->device));
  DevBuf<int> d_err;
  DevBuf<unsigned long long> d_ns;
  DGTD_TRY(d_err.alloc(1));
  DGTD_TRY(d_ns.alloc(1));
  CUDA_TRY(cudaMemsetAsync(d_err.p, 0, sizeof(int), ctx->stream));
  k_tc_wait_probe<<<1, 32, 0, ctx->stream>>>((uint32_t)max_polls, d_err.p, d_ns.p);
  CUDA_TRY(cudaGetLastError());
  int h_err = 0;
  unsigned long long h_ns = 0;
  CUDA_TRY(cudaMemcpyAsync(&h_err, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(&h_ns, d_ns.p, sizeof(h_ns), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (waited_s) *waited_s = (double)h_ns * 1e-9;
  if (h_err) return set_error(DGTD_ERR_TIMEOUT, "debug_wait_timeout: the bounded wait gave up (as it should)");
  return DGTD_OK;
}

// ------------------------------------------------------------------ tensor-core self test

extern "C" int dgtd_debug_tc_gemm(dgtd_ctx* ctx, const float* a, const float* b, float* c, int32_t n, int32_t k,
                                  int32_t flags) {
  const int n_step = (flags & 4) ? 8 : 16;  // MMA N granularity at M = 64 / 128
  if (!ctx || !a || !b || !c || n < n_step || n > dgtd::kSelftestMaxN || (n % n_step) || k < 8 ||
      k > dgtd::kSelftestMaxK || (k % 8))
    return set_error(DGTD_ERR_BAD_ARG, "debug_tc_gemm: need N <= 256 a multiple of 16 (of 8 at M = 64), "
                                       "8 <= K <= 64 (K % 8 == 0)");
  CUDA_TRY(cudaSetDevice(ctx->device));
  DevBuf<float> da, db, dc;
  DevBuf<int> derr;
  DGTD_TRY(da.alloc((size_t)128 * k));
  DGTD_TRY(db.alloc((size_t)n * k));
  DGTD_TRY(dc.alloc((size_t)128 * n));
  DGTD_TRY(derr.alloc(1));
  cudaStream_t s = ctx->stream;
  CUDA_TRY(cudaMemcpyAsync(da.p, a, (size_t)128 * k * 4, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(db.p, b, (size_t)n * k * 4, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemsetAsync(dc.p, 0, (size_t)128 * n * 4, s));
  CUDA_TRY(cudaMemsetAsync(derr.p, 0, 4, s));
  const size_t smem = (size_t)(2 * 128 * k + 2 * n * k) * 4;
  CUDA_TRY(cudaFuncSetAttribute(dgtd::k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dgtd::k_tc_selftest<<<1, 128, smem, s>>>(da.p, db.p, dc.p, n, k, flags, derr.p);
  CUDA_TRY(cudaGetLastError());
  int herr = 0;
  CUDA_TRY(cudaMemcpyAsync(c, dc.p, (size_t)128 * n * 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(&herr, derr.p, 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  da.free(); db.free(); dc.free(); derr.free();
  if (herr) return set_error(DGTD_ERR_TIMEOUT, "debug_tc_gemm: MMA completion wait timed out");
  return DGTD_OK;
}

// Point the tensor-core kernel's phase counters (8 x u64, device memory) at
// `d_counters`; only builds compiled with -DDGTD_TC_PHASE_TIMERS record them.
extern "C" int dgtd_debug_set_phase_clock(dgtd_op* op, void* d_counters) {
  if (!op) return set_error(DGTD_ERR_BAD_ARG, "debug_set_phase_clock: null op");
  op->phase_clk = static_cast<unsigned long long*>(d_counters);
  return DGTD_OK;
}

#ifdef DGTD_TC_PHASE_TIMERS
// Instrumented builds only: mbarrier polls of the three timed threads.
extern "C" int dgtd_debug_tc_polls(unsigned long long* host3, int reset) {
  if (reset) {
    unsigned long long z[3] = {0, 0, 0};
    CUDA_TRY(cudaMemcpyToSymbol(dgtd::g_tc_polls, z, sizeof(z)));
    return DGTD_OK;
  }
  CUDA_TRY(cudaMemcpyFromSymbol(host3, dgtd::g_tc_polls, sizeof(unsigned long long) * 3));
  return DGTD_OK;
}
#endif
