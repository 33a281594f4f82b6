// dgtd_common.cuh -- shared device-side definitions of the DGTD kernels.
//
// Device data layout (HBM):
//   state      float  y[K][6][Np]     element-major SoA: component c of node i
//                                     of element e at (e*6 + c)*Np + i, c = Ex,Ey,Ez,Hx,Hy,Hz.
//   element    float  meta[K][kMetaWords] one 176-byte record per element:
//                       [0..9)   J^-1 row-major           (geom_factors.rs:81-88)
//                       [9..21)  4 outward unit normals   (topology.rs:64-78)
//                       [21..25) 4 face scales 2A/|detJ|  (rhs.rs:828)
//                       [25..37) 1/eps, 1/mu, sigma/eps, sigma*/mu (rhs.rs:900-926)
//                       [37..41) 4 neighbour element ids (int bits, -1 boundary)
//                       [41..43) 4 face codes, 16 bits each (faces 0,1 in word 41):
//                                bits 0..7 gather-table id, bits 8..9 kind
//                                (0 interior, 1 PEC wall, 2 port)
//                       [43]     LSERK step multiplier of the element (1, or an
//                                instance's own step in a batched operator)
//   gather tables (per operator, uint8): gtab[id][m] = volume node of the
//                       neighbour that matches this face's node m
//                       (face_nodes[nbr_lf][perm[m]], rhs.rs:1404-1406).
//   face nodes (uint8):  fnodes[f][m] = own volume node of face f node m.
//   operators (f32):     dT[k][j][i] = D_k[i][j] (k = r,s,t), liftT[s][i] = LIFT[i][s].
#pragma once
#include <cstdint>

namespace dgtd {

constexpr int kMetaWords = 44;
constexpr int kMaxGather = 96;
constexpr int kMaxOrder = 5;

enum FaceKind : int { kInterior = 0, kPec = 1, kPort = 2 };

__host__ __device__ constexpr int np_of(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }
__host__ __device__ constexpr int nfp_of(int n) { return (n + 1) * (n + 2) / 2; }

// Epilogue modes of the RHS kernel.
enum RhsMode : int {
  kModeApply = 0,    // out = dy (f32 SoA)
  kModeLserk = 1,    // fused LSERK4 stage: p = a*p + dt*(dy+src); y_out = y_in + b*p
  kModeKrylov = 3,   // Krylov matvec: out = kry[0]*dy + kry[1]*b (state type in and out;
                     // b = src_vec or the point src_idx; kry in device memory)
  kModeKcl = 4,      // fused KCL RK4(3)5 stage: f = h (dy + src); y += b f; e (=|+=) ew f;
                     // next stage point = y + amb f (h, the frame's waveform from device memory)
};

template <class R>
struct OpTablesT {
  const R* dT;            // 3*Np*Np
  const R* liftT;         // 4Nfp*Np
  const uint8_t* fnodes;  // 4*Nfp
  const uint8_t* gtab;    // n_gather*Nfp
  int n_gather;
};
using OpTables = OpTablesT<float>;

// Launch parameters of the RHS kernels; R is the arithmetic type of the state
// (float: the FP32 and tensor-core engines; double: the FP64 path, whose
// element records are the same 44 words stored as doubles, integer words as
// exact double values).
template <class R>
struct RhsParamsT {
  const R* y_in;           // state / stored basis vector
  R* out;                  // Apply: dy ; Lserk: y_out ; Krylov: w
  R* p;                    // Lserk residual register
  const R* meta;
  const R* src_vec;        // DRIVE_VECTOR pattern / Krylov source column b (SoA) or null
  const int* skip;         // device flag: when nonzero the launch does nothing (Arnoldi early stop,
                           // adaptive attempts past the end of a run)
  const double* kry;       // Krylov: device {input scale, source coefficient}
  // KCL stage (kModeKcl): the solution y and embedded error e updated in place,
  // the next stage's evaluation point (null after the last stage), the
  // controller's step and frame in device memory, the per-frame waveform
  R* kcl_y;
  R* kcl_e;
  R* kcl_next;
  const float* kcl_h;
  const long long* kcl_frame;
  const float* kcl_g;
  R kcl_b, kcl_ew, kcl_amb;
  int kcl_stage;
  int64_t n_elem;          // elements [e_begin, n_elem) are computed
  int64_t e_begin;         // first element (a multiple of the tensor-core tile, 20); 0 for the whole op
  int64_t src_idx;         // DRIVE_POINT (Lserk, Krylov): SoA index, or -1
  R src_g;                 // held waveform value of the step
  R a, b, dt;              // LSERK stage coefficients
  int read_p, write_p;     // stage 0 does not read p; the last stage does not write it
  R alpha;                 // flux blend
  unsigned long long* phase_clk;  // per-phase cycle counters (instrumented builds only), or null
};
using RhsParams = RhsParamsT<float>;

}  // namespace dgtd
