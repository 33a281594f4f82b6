// host_op.cpp -- native host side of the DGTD path: structured meshes, the
// nodal reference element and the operator build (f64), behind the C ABI of
// include/dgtd_host.h.  The arrays produced here are what the device operator
// (dgtd_op_create) consumes.
//
// Reference algorithms followed (paths relative to the rapidfem root):
//   mesh_gen.rs:16-139, dg_basis.rs:61-385, geom_factors.rs:33-88,
//   rapidfem-core topology.rs:50-91 + mesh.rs:45-50, rhs.rs:805-1000,
//   rhs.rs:546-770 (periodic pairs), rhs.rs:1030-1066, rhs.rs:1157-1199,
//   waveguide.rs:39-145.
#include <algorithm>
#include <parallel/algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../../include/dgtd_host.h"
#include "errors.h"

namespace dgtd {
namespace host {

using V3 = std::array<double, 3>;

// x.powi(n) as Rust lowers it (binary exponentiation).
static double powi(double a, int b) {
  bool recip = b < 0;
  double r = 1.0;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0 / r : r;
}

static double fact(int n) {
  double p = 1.0;
  for (int k = 1; k <= n; ++k) p *= double(k);
  return p;
}

static V3 cross(const V3& a, const V3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
static double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Dense row-major square/rect helpers.
struct Mat {
  int rows = 0, cols = 0;
  std::vector<double> a;
  Mat() = default;
  Mat(int r, int c) : rows(r), cols(c), a(size_t(r) * c, 0.0) {}
  double& operator()(int i, int j) { return a[size_t(i) * cols + j]; }
  double operator()(int i, int j) const { return a[size_t(i) * cols + j]; }
};

// Gauss-Jordan with partial pivoting (dg_basis.rs:160-206).
static bool gj_inverse(const Mat& src, Mat& inv) {
  const int n = src.rows;
  Mat w = src;
  inv = Mat(n, n);
  for (int i = 0; i < n; ++i) inv(i, i) = 1.0;
  for (int col = 0; col < n; ++col) {
    int piv = col;
    double best = std::fabs(w(col, col));
    for (int r = col + 1; r < n; ++r) {
      double v = std::fabs(w(r, col));
      if (v > best) { best = v; piv = r; }
    }
    if (!(best > 1e-300)) return false;
    if (piv != col)
      for (int k = 0; k < n; ++k) {
        std::swap(w(col, k), w(piv, k));
        std::swap(inv(col, k), inv(piv, k));
      }
    const double d = w(col, col);
    for (int k = 0; k < n; ++k) { w(col, k) /= d; inv(col, k) /= d; }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      const double f = w(r, col);
      if (f == 0.0) continue;
      for (int k = 0; k < n; ++k) {
        w(r, k) -= f * w(col, k);
        inv(r, k) -= f * inv(col, k);
      }
    }
  }
  return true;
}

// A*B skipping zeros of A (dg_basis.rs:213-237).
static Mat mul(const Mat& A, const Mat& B) {
  Mat C(A.rows, B.cols);
  for (int i = 0; i < A.rows; ++i)
    for (int k = 0; k < A.cols; ++k) {
      const double aik = A(i, k);
      if (aik == 0.0) continue;
      for (int j = 0; j < B.cols; ++j) C(i, j) += aik * B(k, j);
    }
  return C;
}

// C^T G C (dg_basis.rs:247-261).
static Mat ctgc(const Mat& C, const Mat& G) {
  const int n = C.rows;
  Mat T(n, n);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) {
      double acc = 0.0;
      for (int m = 0; m < n; ++m) acc += C(m, i) * G(m, k);
      T(i, k) = acc;
    }
  return mul(T, C);
}

// ---------------------------------------------------------------- element

struct RefElement {
  int order = 0, np = 0, nfp = 0;
  std::vector<V3> nodes;
  Mat mass, dr, ds, dt, lift;
  std::vector<int32_t> face_nodes;  // 4*nfp
  std::vector<double> face_w;       // 4*nfp

  bool build(int p) {
    order = p;
    np = (p + 1) * (p + 2) * (p + 3) / 6;
    nfp = (p + 1) * (p + 2) / 2;
    std::vector<std::array<int, 3>> monos, ijk;
    for (int deg = 0; deg <= p; ++deg)
      for (int a = 0; a <= deg; ++a)
        for (int b = 0; b <= deg - a; ++b) monos.push_back({a, b, deg - a - b});
    for (int i = 0; i <= p; ++i)
      for (int j = 0; j <= p - i; ++j)
        for (int k = 0; k <= p - i - j; ++k) ijk.push_back({i, j, k});
    nodes.clear();
    for (auto& c : ijk) nodes.push_back({double(c[0]) / p, double(c[1]) / p, double(c[2]) / p});
    const int n = np;
    Mat V(n, n), G(n, n);
    for (int ni = 0; ni < n; ++ni)
      for (int mi = 0; mi < n; ++mi)
        V(ni, mi) = powi(nodes[ni][0], monos[mi][0]) * powi(nodes[ni][1], monos[mi][1]) *
                    powi(nodes[ni][2], monos[mi][2]);
    Mat Cm;
    if (!gj_inverse(V, Cm)) return false;
    for (int mi = 0; mi < n; ++mi)
      for (int qi = 0; qi < n; ++qi) {
        int a = monos[mi][0] + monos[qi][0], b = monos[mi][1] + monos[qi][1],
            c = monos[mi][2] + monos[qi][2];
        G(mi, qi) = fact(a) * fact(b) * fact(c) / fact(a + b + c + 3);
      }
    mass = ctgc(Cm, G);
    Mat minv;
    if (!gj_inverse(mass, minv)) return false;
    Mat Vd[3] = {Mat(n, n), Mat(n, n), Mat(n, n)};
    for (int ni = 0; ni < n; ++ni)
      for (int mi = 0; mi < n; ++mi)
        for (int ax = 0; ax < 3; ++ax) {
          int e = monos[mi][ax];
          if (e == 0) continue;
          auto d = monos[mi];
          d[ax] -= 1;
          Vd[ax](ni, mi) = double(e) * (powi(nodes[ni][0], d[0]) * powi(nodes[ni][1], d[1]) *
                                        powi(nodes[ni][2], d[2]));
        }
    dr = mul(Vd[0], Cm);
    ds = mul(Vd[1], Cm);
    dt = mul(Vd[2], Cm);

    // Face node sets and LIFT (dg_basis.rs:288-385).
    const int cols = 4 * nfp;
    face_nodes.assign(size_t(4) * nfp, 0);
    face_w.assign(size_t(4) * nfp, 0.0);
    Mat E(n, cols);
    std::vector<std::array<int, 2>> m2;
    for (int deg = 0; deg <= p; ++deg)
      for (int a = 0; a <= deg; ++a) m2.push_back({a, deg - a});
    for (int f = 0; f < 4; ++f) {
      int cnt = 0;
      for (int idx = 0; idx < n; ++idx) {
        const auto& q = ijk[idx];
        bool on = f == 0 ? q[2] == 0 : f == 1 ? q[0] == 0 : f == 2 ? q[1] == 0 : q[0] + q[1] + q[2] == p;
        if (on) {
          if (cnt >= nfp) return false;
          face_nodes[size_t(f) * nfp + cnt++] = idx;
        }
      }
      if (cnt != nfp) return false;
      std::vector<std::array<double, 2>> uv(nfp);
      for (int a = 0; a < nfp; ++a) {
        const auto& q = ijk[face_nodes[size_t(f) * nfp + a]];
        int u = f == 1 ? q[1] : q[0];
        int v = f == 0 || f == 3 ? q[1] : q[2];
        uv[a] = {double(u) / p, double(v) / p};
      }
      Mat V2(nfp, nfp), G2(nfp, nfp), C2;
      for (int i = 0; i < nfp; ++i)
        for (int j = 0; j < nfp; ++j) V2(i, j) = powi(uv[i][0], m2[j][0]) * powi(uv[i][1], m2[j][1]);
      if (!gj_inverse(V2, C2)) return false;
      for (int i = 0; i < nfp; ++i)
        for (int j = 0; j < nfp; ++j) {
          int a = m2[i][0] + m2[j][0], b = m2[i][1] + m2[j][1];
          G2(i, j) = fact(a) * fact(b) / fact(a + b + 2);
        }
      Mat Mf = ctgc(C2, G2);
      for (int a = 0; a < nfp; ++a) {
        int vi = face_nodes[size_t(f) * nfp + a];
        double s = 0.0;
        for (int m = 0; m < nfp; ++m) {
          E(vi, f * nfp + m) = Mf(a, m);
          s += Mf(a, m);
        }
        face_w[size_t(f) * nfp + a] = s;
      }
    }
    lift = mul(minv, E);
    return true;
  }
};

// ---------------------------------------------------------------- operator

static const int kFaceLocal[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 2, 3}};
static const int kPecPlate = -2;  // face_port code of a face of an internal PEC plate
static const int kFaceOpposite[4] = {3, 1, 2, 0};

struct Operator {
  RefElement re;
  int64_t K = 0;
  double alpha = 1.0;
  std::vector<double> origin, jac, jinv, det;      // 3K, 9K, 9K, K
  std::vector<double> normal, fscale;              // 12K, 4K
  std::vector<int32_t> nbr, nbr_lf, port, perm;    // 4K, 4K, 4K, 4K*nfp
  std::vector<double> inv_eps, inv_mu, sig_e, sig_m;

  V3 map(int64_t e, const V3& xi) const {
    V3 x = {origin[3 * e], origin[3 * e + 1], origin[3 * e + 2]};
    const double* J = &jac[9 * e];
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) x[i] += J[i * 3 + k] * xi[k];
    return x;
  }

  std::string build(const double* nodes, int64_t n_nodes, const int32_t* tets, int64_t n_elem,
                    int order, double flux_alpha, const int32_t* face_port, const double* mat) {
    if (order < 1 || order > 5) return "order must be in 1..5";
    if (!re.build(order)) return "reference element construction failed";
    K = n_elem;
    alpha = flux_alpha;
    const int nfp = re.nfp;
    for (int64_t i = 0; i < 4 * K; ++i)
      if (tets[i] < 0 || tets[i] >= n_nodes) return "tet vertex id out of range";
    origin.resize(3 * K); jac.resize(9 * K); jinv.resize(9 * K); det.resize(K);
    // The element and face loops below write only their own element's entries,
    // so they run on all host threads with results identical to a serial run.
    bool degenerate = false;
#pragma omp parallel for schedule(static) reduction(|| : degenerate)
    for (int64_t e = 0; e < K; ++e) {
      const double* v[4];
      for (int q = 0; q < 4; ++q) v[q] = nodes + 3 * size_t(tets[4 * e + q]);
      V3 m[3];
      for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) m[i][k] = v[k + 1][i] - v[0][i];
      V3 adj[3] = {cross(m[1], m[2]), cross(m[2], m[0]), cross(m[0], m[1])};
      const double d = dot(m[0], adj[0]);
      if (d == 0.0 || !std::isfinite(d)) {
        degenerate = true;
        continue;
      }
      const double id = 1.0 / d;
      for (int i = 0; i < 3; ++i) {
        origin[3 * e + i] = v[0][i];
        for (int k = 0; k < 3; ++k) {
          jac[9 * e + i * 3 + k] = m[i][k];
          jinv[9 * e + i * 3 + k] = adj[k][i] * id;
        }
      }
      det[e] = d;
    }
    if (degenerate) return "degenerate tetrahedron";
    // Face topology (topology.rs:50-91) with neighbours from shared vertex sets.
    normal.resize(12 * K); fscale.resize(4 * K);
    nbr.assign(4 * K, -1); nbr_lf.assign(4 * K, -1); port.assign(4 * K, -1);
    perm.assign(size_t(4) * K * nfp, 0);
    std::vector<double> area(4 * K);
    // Faces are matched by their sorted vertex triples: the 4K records are
    // sorted (in parallel) by (triple, face id) and equal neighbours paired.
    // For a triple shared by more than two tets the two lowest face ids, i.e.
    // the first two tets in element order, are kept.
    struct FaceRec {
      int64_t a, b, c, id;
    };
    std::vector<FaceRec> fr(size_t(4) * K);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < K; ++e)
      for (int lf = 0; lf < 4; ++lf) {
        int64_t t3[3] = {tets[4 * e + kFaceLocal[lf][0]], tets[4 * e + kFaceLocal[lf][1]], tets[4 * e + kFaceLocal[lf][2]]};
        std::sort(t3, t3 + 3);
        fr[4 * e + lf] = FaceRec{t3[0], t3[1], t3[2], 4 * e + lf};
      }
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < K; ++e)
      for (int lf = 0; lf < 4; ++lf) {
        auto P = [&](int loc) { const double* p = nodes + 3 * size_t(tets[4 * e + loc]); return V3{p[0], p[1], p[2]}; };
        V3 v0 = P(kFaceLocal[lf][0]), v1 = P(kFaceLocal[lf][1]), v2 = P(kFaceLocal[lf][2]);
        V3 vo = P(kFaceOpposite[lf]);
        V3 n = cross({v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]}, {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]});
        const double len = std::sqrt(dot(n, n));
        area[4 * e + lf] = 0.5 * len;
        for (int k = 0; k < 3; ++k) n[k] /= len;
        if (dot({vo[0] - v0[0], vo[1] - v0[1], vo[2] - v0[2]}, n) > 0.0)
          for (int k = 0; k < 3; ++k) n[k] = -n[k];
        for (int k = 0; k < 3; ++k) normal[12 * e + 3 * lf + k] = n[k];
      }
    const auto rec_less = [](const FaceRec& x, const FaceRec& y) {
      if (x.a != y.a) return x.a < y.a;
      if (x.b != y.b) return x.b < y.b;
      if (x.c != y.c) return x.c < y.c;
      return x.id < y.id;
    };
    __gnu_parallel::sort(fr.begin(), fr.end(), rec_less);
    for (size_t i = 0; i < fr.size();) {
      size_t j = i + 1;
      while (j < fr.size() && fr[j].a == fr[i].a && fr[j].b == fr[i].b && fr[j].c == fr[i].c) ++j;
      if (j - i >= 2) {
        const int64_t fa = fr[i].id, fb = fr[i + 1].id;
        nbr[fa] = int32_t(fb / 4); nbr_lf[fa] = int32_t(fb % 4);
        nbr[fb] = int32_t(fa / 4); nbr_lf[fb] = int32_t(fa % 4);
      }
      i = j;
    }
    // fscale, perm (nearest-node match, tol^2 1e-18 absolute), ports.
    bool unmatched = false;
    double worst = 0.0;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < K; ++e) {
      std::array<V3, 21> here, there;  // Nfp <= 21 (order 5)
      for (int f = 0; f < 4; ++f) {
        const int64_t ef = 4 * e + f;
        fscale[ef] = 2.0 * area[ef] / std::fabs(det[e]);
        if (face_port) port[ef] = face_port[ef];
        if (port[ef] == kPecPlate) {
          // a face of an internal PEC plate: severed from its neighbour (the
          // other side carries the code too), the PEC ghost state applies
          // (rhs.rs:862-880)
          port[ef] = -1;
          nbr[ef] = -1;
          nbr_lf[ef] = 0;
        }
        if (nbr[ef] < 0) continue;
        const int64_t en = nbr[ef];
        const int fn = nbr_lf[ef];
        for (int m = 0; m < nfp; ++m) {
          here[m] = map(e, re.nodes[re.face_nodes[size_t(f) * nfp + m]]);
          there[m] = map(en, re.nodes[re.face_nodes[size_t(fn) * nfp + m]]);
        }
        for (int m = 0; m < nfp; ++m) {
          double best = std::numeric_limits<double>::max();
          int bm = 0;
          for (int m2 = 0; m2 < nfp; ++m2) {
            double d = powi(here[m][0] - there[m2][0], 2) + powi(here[m][1] - there[m2][1], 2) +
                       powi(here[m][2] - there[m2][2], 2);
            if (d < best) { best = d; bm = m2; }
          }
          if (!(best < 1e-18)) {
#pragma omp critical(dgtd_unmatched)
            {
              unmatched = true;
              if (!(best <= worst)) worst = best;
            }
          }
          perm[size_t(ef) * nfp + m] = bm;
        }
      }
    }
    if (unmatched) return "unmatched face node (best distance " + std::to_string(std::sqrt(worst)) + ")";
    inv_eps.resize(3 * K); inv_mu.resize(3 * K); sig_e.resize(3 * K); sig_m.resize(3 * K);
    for (int64_t e = 0; e < K; ++e) {
      double eps[3] = {1, 1, 1}, mu[3] = {1, 1, 1}, sg = 0.0, sm = 0.0;
      if (mat) {
        for (int c = 0; c < 3; ++c) { eps[c] = mat[8 * e + c]; mu[c] = mat[8 * e + 3 + c]; }
        sg = mat[8 * e + 6]; sm = mat[8 * e + 7];
      }
      for (int c = 0; c < 3; ++c) {
        inv_eps[3 * e + c] = 1.0 / eps[c];
        inv_mu[3 * e + c] = 1.0 / mu[c];
        sig_e[3 * e + c] = sg / eps[c];
        sig_m[3 * e + c] = sm / mu[c];
      }
    }
    return "";
  }
};

}  // namespace host
}  // namespace dgtd

struct dgtd_host_op {
  dgtd::host::Operator op;
};

using dgtd::host::V3;
using dgtd::host::cross;
using dgtd::host::dot;
using dgtd::set_error;

// ------------------------------------------------------------------ meshes

static const int kKuhn[6][4] = {{0, 1, 3, 7}, {0, 3, 2, 7}, {0, 2, 6, 7},
                                {0, 6, 4, 7}, {0, 4, 5, 7}, {0, 5, 1, 7}};

static void kuhn_tets(int nx, int ny, int nz, int32_t* tets) {
  const int nxp = nx + 1, nyp = ny + 1;
  size_t t = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        for (const auto& kt : kKuhn) {
          int32_t v[4];
          for (int q = 0; q < 4; ++q) {
            const int c = kt[q];
            v[q] = ((k + ((c >> 2) & 1)) * nyp + (j + ((c >> 1) & 1))) * nxp + (i + (c & 1));
          }
          std::sort(v, v + 4);
          std::memcpy(tets + 4 * t, v, sizeof(v));
          ++t;
        }
}

extern "C" int dgtd_mesh_box(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                             double* nodes, int32_t* tets) {
  if (nx < 1 || ny < 1 || nz < 1 || !nodes || !tets) return set_error(DGTD_ERR_BAD_ARG, "box: bad arguments");
  size_t c = 0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i, ++c) {
        nodes[3 * c] = lx * double(i) / double(nx);
        nodes[3 * c + 1] = ly * double(j) / double(ny);
        nodes[3 * c + 2] = lz * double(k) / double(nz);
      }
  kuhn_tets(nx, ny, nz, tets);
  return DGTD_OK;
}

static double jitter_mix(uint64_t x) {
  x *= 0x9E3779B97F4A7C15ULL;
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ULL;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBULL;
  x ^= x >> 31;
  return (double(x) / double(UINT64_MAX)) * 2.0 - 1.0;
}

extern "C" int dgtd_mesh_box_jittered(int32_t nx, int32_t ny, int32_t nz, double lx, double ly,
                                      double lz, double amplitude, uint64_t seed, double* nodes,
                                      int32_t* tets) {
  if (nx < 1 || ny < 1 || nz < 1 || !nodes || !tets) return set_error(DGTD_ERR_BAD_ARG, "box: bad arguments");
  const double hx = lx / nx, hy = ly / ny, hz = lz / nz;
  size_t c = 0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i, ++c) {
        double p[3] = {hx * double(i), hy * double(j), hz * double(k)};
        const uint64_t base = seed + uint64_t(i) * 0x01000193ULL + uint64_t(j) * 0x00000100000001B3ULL +
                              uint64_t(k) * 0xC2B2AE3D27D4EB4FULL;
        const double off[3] = {jitter_mix(base), jitter_mix(base ^ 0xAAAA), jitter_mix(base ^ 0x5555)};
        if (i != 0 && i != nx) p[0] += amplitude * hx * off[0];
        if (j != 0 && j != ny) p[1] += amplitude * hy * off[1];
        if (k != 0 && k != nz) p[2] += amplitude * hz * off[2];
        std::memcpy(nodes + 3 * c, p, sizeof(p));
      }
  kuhn_tets(nx, ny, nz, tets);
  return DGTD_OK;
}

extern "C" int dgtd_mesh_box_graded_z(int32_t nx, int32_t ny, int32_t nz, double lx, double ly,
                                      double lz, double ratio, double* nodes, int32_t* tets) {
  if (nx < 1 || ny < 1 || nz < 1 || !nodes || !tets || !(ratio > 0.0))
    return set_error(DGTD_ERR_BAD_ARG, "graded box: bad arguments");
  // Geometric spacing h_k = h0*q^k, q^(nz-1) = ratio, sum h_k = lz.
  std::vector<double> z(nz + 1, 0.0);
  const double q = nz > 1 ? std::pow(ratio, 1.0 / double(nz - 1)) : 1.0;
  double s = 0.0, h = 1.0;
  for (int k = 0; k < nz; ++k) { s += h; h *= q; }
  h = lz / s;
  for (int k = 0; k < nz; ++k) { z[k + 1] = z[k] + h; h *= q; }
  z[nz] = lz;
  size_t c = 0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i, ++c) {
        nodes[3 * c] = lx * double(i) / double(nx);
        nodes[3 * c + 1] = ly * double(j) / double(ny);
        nodes[3 * c + 2] = z[k];
      }
  kuhn_tets(nx, ny, nz, tets);
  return DGTD_OK;
}

// ---------------------------------------------------------------- operator

extern "C" int dgtd_host_op_build(const double* nodes, int64_t n_nodes, const int32_t* tets,
                                  int64_t n_elem, int32_t order, double flux_alpha,
                                  const int32_t* face_port, const double* materials,
                                  dgtd_host_op** out) {
  if (!nodes || !tets || !out || n_elem < 1 || n_nodes < 4)
    return set_error(DGTD_ERR_BAD_ARG, "host_op_build: bad arguments");
  if (n_elem > (int64_t(1) << 29)) return set_error(DGTD_ERR_BAD_ARG, "host_op_build: too many elements");
  auto* h = new (std::nothrow) dgtd_host_op;
  if (!h) return set_error(DGTD_ERR_OOM, "host_op_build: out of memory");
  std::string err;
  try {
    err = h->op.build(nodes, n_nodes, tets, n_elem, order, flux_alpha, face_port, materials);
  } catch (const std::bad_alloc&) {
    delete h;
    return set_error(DGTD_ERR_OOM, "host_op_build: out of memory");
  }
  if (!err.empty()) {
    delete h;
    return set_error(order < 1 || order > 5 ? DGTD_ERR_UNSUPPORTED : DGTD_ERR_BAD_ARG, "host_op_build: " + err);
  }
  *out = h;
  return DGTD_OK;
}

extern "C" int dgtd_host_op_destroy(dgtd_host_op* op) {
  delete op;
  return DGTD_OK;
}

// ------------------------------------------------------- periodic face pairs

namespace {

const double kPeriodicRelTol = 1e-9;     // PERIODIC_MATCH_REL_TOL (constants.rs:216)
const double kPeriodicAbsFloor = 1e-12;  // PERIODIC_MATCH_ABS_FLOOR (constants.rs:222)
const V3 kRefVertex[4] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

struct FaceGeom {
  V3 centroid;
  double area;
};

FaceGeom face_geom(const dgtd::host::Operator& o, int64_t ef) {
  const int64_t e = ef / 4;
  const int lf = int(ef % 4);
  V3 v[3];
  for (int q = 0; q < 3; ++q) v[q] = o.map(e, kRefVertex[dgtd::host::kFaceLocal[lf][q]]);
  const V3 n = cross({v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]},
                     {v[2][0] - v[0][0], v[2][1] - v[0][1], v[2][2] - v[0][2]});
  FaceGeom g;
  g.area = 0.5 * std::sqrt(dot(n, n));
  for (int k = 0; k < 3; ++k) g.centroid[k] = (v[0][k] + v[1][k] + v[2][k]) / 3.0;
  return g;
}

std::string sci(double v) {
  char buf[32];
  std::snprintf(buf, sizeof buf, "%.3e", v);
  return buf;
}

double dist2(const V3& a, const V3& b) {
  return dgtd::host::powi(a[0] - b[0], 2) + dgtd::host::powi(a[1] - b[1], 2) +
         dgtd::host::powi(a[2] - b[2], 2);
}

// match_face_nodes (rhs.rs:546-568): perm[m] = the node of face `there`
// nearest to node m of face `here` shifted by `shift`; false if one is
// farther than sqrt(tol2).
bool match_nodes(const dgtd::host::Operator& o, int64_t here, int64_t there, const V3& shift, double tol2,
                 int32_t* perm, double* worst) {
  const int nfp = o.re.nfp;
  std::array<V3, 21> ph, pt;  // Nfp <= 21 (order 5)
  for (int m = 0; m < nfp; ++m) {
    ph[m] = o.map(here / 4, o.re.nodes[o.re.face_nodes[size_t(here % 4) * nfp + m]]);
    pt[m] = o.map(there / 4, o.re.nodes[o.re.face_nodes[size_t(there % 4) * nfp + m]]);
  }
  bool ok = true;
  for (int m = 0; m < nfp; ++m) {
    const V3 target = {ph[m][0] + shift[0], ph[m][1] + shift[1], ph[m][2] + shift[2]};
    double best = std::numeric_limits<double>::max();
    int bm = 0;
    for (int m2 = 0; m2 < nfp; ++m2) {
      const double d = dist2(target, pt[m2]);
      if (d < best) { best = d; bm = m2; }
    }
    if (!(best < tol2)) {
      ok = false;
      *worst = std::max(*worst, std::sqrt(best));
    }
    perm[m] = bm;
  }
  return ok;
}

}  // namespace

// link_periodic_faces (rhs.rs:616-770) on face ids e*4+lf.  Everything is
// checked before the operator changes, so a failed call leaves it as it was.
extern "C" int dgtd_host_op_link_periodic(dgtd_host_op* h, const int64_t* faces_a, int64_t n_a,
                                          const int64_t* faces_b, int64_t n_b) {
  if (!h || !faces_a || !faces_b || n_a < 1 || n_b < 1)
    return set_error(DGTD_ERR_BAD_ARG, "link_periodic: bad arguments");
  auto& o = h->op;
  if (n_a != n_b)
    return set_error(DGTD_ERR_BAD_ARG, "link_periodic: periodic pair has different triangle counts on each side: A has " +
                                           std::to_string(n_a) + ", B has " + std::to_string(n_b));
  const int64_t n = n_a;
  for (int side = 0; side < 2; ++side)
    for (int64_t i = 0; i < n; ++i) {
      const int64_t ef = (side ? faces_b : faces_a)[i];
      if (ef < 0 || ef >= 4 * o.K) return set_error(DGTD_ERR_BAD_ARG, "link_periodic: face id out of range");
      if (o.port[ef] >= 0)
        return set_error(DGTD_ERR_BAD_ARG, "link_periodic: face " + std::to_string(ef) + " is marked both port and periodic");
      if (o.nbr[ef] >= 0)
        return set_error(DGTD_ERR_BAD_ARG, "link_periodic: face " + std::to_string(ef) + " is not on the domain boundary");
    }
  // Period translation from the area-weighted side centroids (rhs.rs:588-614).
  std::vector<FaceGeom> ga(n), gb(n);
  V3 ca = {0, 0, 0}, cb = {0, 0, 0};
  double wa = 0.0, wb = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    ga[i] = face_geom(o, faces_a[i]);
    gb[i] = face_geom(o, faces_b[i]);
    for (int k = 0; k < 3; ++k) {
      ca[k] += ga[i].area * ga[i].centroid[k];
      cb[k] += gb[i].area * gb[i].centroid[k];
    }
    wa += ga[i].area;
    wb += gb[i].area;
  }
  if (!(wa > 0.0) || !(wb > 0.0)) return set_error(DGTD_ERR_BAD_ARG, "link_periodic: periodic face has zero total area");
  V3 trans;
  for (int k = 0; k < 3; ++k) trans[k] = cb[k] / wb - ca[k] / wa;
  const double mag = std::sqrt(dot(trans, trans));
  const double tol = std::max(kPeriodicRelTol * mag, kPeriodicAbsFloor);
  const double tol2 = tol * tol;
  // Triangle partners: nearest translated centroid.  B's centroids are sorted
  // by x, so each A triangle scans only the B triangles within tol in x; the
  // nearest of those (lowest B index on a tie) is the nearest of all whenever
  // one lies within tol.
  std::vector<int64_t> bx(n);
  for (int64_t i = 0; i < n; ++i) bx[i] = i;
  std::sort(bx.begin(), bx.end(), [&](int64_t p, int64_t q) {
    return gb[p].centroid[0] < gb[q].centroid[0] || (gb[p].centroid[0] == gb[q].centroid[0] && p < q);
  });
  std::vector<double> xs(n);
  for (int64_t i = 0; i < n; ++i) xs[i] = gb[bx[i]].centroid[0];
  std::vector<int64_t> a_to_b(n, -1), b_to_a(n, -1);
  for (int64_t i = 0; i < n; ++i) {
    const V3 t = {ga[i].centroid[0] + trans[0], ga[i].centroid[1] + trans[1], ga[i].centroid[2] + trans[2]};
    auto lo = std::lower_bound(xs.begin(), xs.end(), t[0] - tol);
    double best = std::numeric_limits<double>::max();
    int64_t bi = -1;
    for (auto it = lo; it != xs.end() && *it <= t[0] + tol; ++it) {
      const int64_t j = bx[it - xs.begin()];
      const double d = dist2(t, gb[j].centroid);
      if (d < best || (d == best && j < bi)) { best = d; bi = j; }
    }
    if (bi < 0 || !(best < tol2))
      return set_error(DGTD_ERR_BAD_ARG, "link_periodic: periodic face " + std::to_string(faces_a[i]) +
                                             " on side A has no partner on side B within tolerance " + sci(tol));
    if (b_to_a[bi] >= 0)
      return set_error(DGTD_ERR_BAD_ARG, "link_periodic: periodic side-B face " + std::to_string(faces_b[bi]) +
                                             " matched by two side-A faces; a periodic pair must be a bijection");
    a_to_b[i] = bi;
    b_to_a[bi] = i;
  }
  const int nfp = o.re.nfp;
  const V3 back = {-trans[0], -trans[1], -trans[2]};
  std::vector<int32_t> perm_a(size_t(n) * nfp), perm_b(size_t(n) * nfp);
  double worst = 0.0;
  bool ok = true;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t fa = faces_a[i], fb = faces_b[a_to_b[i]];
    ok &= match_nodes(o, fa, fb, trans, tol2, &perm_a[size_t(i) * nfp], &worst);
    ok &= match_nodes(o, fb, fa, back, tol2, &perm_b[size_t(i) * nfp], &worst);
  }
  if (!ok)
    return set_error(DGTD_ERR_BAD_ARG, "link_periodic: periodic face node found no partner within tolerance " +
                                           sci(tol) + " (best " + sci(worst) + ")");
  for (int64_t i = 0; i < n; ++i) {
    const int64_t fa = faces_a[i], fb = faces_b[a_to_b[i]];
    o.nbr[fa] = int32_t(fb / 4); o.nbr_lf[fa] = int32_t(fb % 4);
    o.nbr[fb] = int32_t(fa / 4); o.nbr_lf[fb] = int32_t(fa % 4);
    std::memcpy(&o.perm[size_t(fa) * nfp], &perm_a[size_t(i) * nfp], sizeof(int32_t) * nfp);
    std::memcpy(&o.perm[size_t(fb) * nfp], &perm_b[size_t(i) * nfp], sizeof(int32_t) * nfp);
  }
  return DGTD_OK;
}

extern "C" int dgtd_host_op_desc(const dgtd_host_op* h, dgtd_op_desc* d) {
  if (!h || !d) return set_error(DGTD_ERR_BAD_ARG, "host_op_desc: null argument");
  const auto& o = h->op;
  *d = dgtd_op_desc{};  // optional arrays (dt_scale) start unset
  d->order = o.re.order;
  d->n_elem = int32_t(o.K);
  d->flux_alpha = o.alpha;
  d->diff_r = o.re.dr.a.data();
  d->diff_s = o.re.ds.a.data();
  d->diff_t = o.re.dt.a.data();
  d->lift = o.re.lift.a.data();
  d->face_nodes = o.re.face_nodes.data();
  d->jinv = o.jinv.data();
  d->inv_eps = o.inv_eps.data();
  d->inv_mu = o.inv_mu.data();
  d->sigma_eps = o.sig_e.data();
  d->sigma_mu = o.sig_m.data();
  d->face_normal = o.normal.data();
  d->face_fscale = o.fscale.data();
  d->face_neighbor = o.nbr.data();
  d->face_nbr_local = o.nbr_lf.data();
  d->face_port = o.port.data();
  d->face_perm = o.perm.data();
  d->mass = o.re.mass.a.data();
  return DGTD_OK;
}

extern "C" int dgtd_host_op_info(const dgtd_host_op* h, int32_t* np, int32_t* nfp, int64_t* n_elem,
                                 int64_t* n_dof) {
  if (!h) return set_error(DGTD_ERR_BAD_ARG, "host_op_info: null op");
  if (np) *np = h->op.re.np;
  if (nfp) *nfp = h->op.re.nfp;
  if (n_elem) *n_elem = h->op.K;
  if (n_dof) *n_dof = 6 * int64_t(h->op.re.np) * h->op.K;
  return DGTD_OK;
}

template <class T>
static void copy_out(const std::vector<T>& v, double* out) {
  for (size_t i = 0; i < v.size(); ++i) out[i] = double(v[i]);
}

extern "C" int dgtd_host_op_get(const dgtd_host_op* h, const char* name, double* out) {
  if (!h || !name || !out) return set_error(DGTD_ERR_BAD_ARG, "host_op_get: null argument");
  const auto& o = h->op;
  const std::string n(name);
  if (n == "nodes") { for (size_t i = 0; i < o.re.nodes.size(); ++i) for (int k = 0; k < 3; ++k) out[3 * i + k] = o.re.nodes[i][k]; }
  else if (n == "mass") copy_out(o.re.mass.a, out);
  else if (n == "dr") copy_out(o.re.dr.a, out);
  else if (n == "ds") copy_out(o.re.ds.a, out);
  else if (n == "dt") copy_out(o.re.dt.a, out);
  else if (n == "lift") copy_out(o.re.lift.a, out);
  else if (n == "face_nodes") copy_out(o.re.face_nodes, out);
  else if (n == "face_w") copy_out(o.re.face_w, out);
  else if (n == "jinv") copy_out(o.jinv, out);
  else if (n == "jac") copy_out(o.jac, out);
  else if (n == "origin") copy_out(o.origin, out);
  else if (n == "det") copy_out(o.det, out);
  else if (n == "normal") copy_out(o.normal, out);
  else if (n == "fscale") copy_out(o.fscale, out);
  else if (n == "nbr") copy_out(o.nbr, out);
  else if (n == "nbr_lf") copy_out(o.nbr_lf, out);
  else if (n == "port") copy_out(o.port, out);
  else if (n == "perm") copy_out(o.perm, out);
  else if (n == "inv_eps") copy_out(o.inv_eps, out);
  else if (n == "inv_mu") copy_out(o.inv_mu, out);
  else if (n == "sigma_eps") copy_out(o.sig_e, out);
  else if (n == "sigma_mu") copy_out(o.sig_m, out);
  else return set_error(DGTD_ERR_BAD_ARG, "host_op_get: unknown array '" + n + "'");
  return DGTD_OK;
}

extern "C" int dgtd_host_node_coords(const dgtd_host_op* h, double* out) {
  if (!h || !out) return set_error(DGTD_ERR_BAD_ARG, "node_coords: null argument");
  const auto& o = h->op;
  for (int64_t e = 0; e < o.K; ++e)
    for (int i = 0; i < o.re.np; ++i) {
      V3 x = o.map(e, o.re.nodes[i]);
      std::memcpy(out + 3 * (size_t(e) * o.re.np + i), x.data(), sizeof(double) * 3);
    }
  return DGTD_OK;
}

extern "C" int dgtd_host_nearest_node_dof(const dgtd_host_op* h, const double* point, int32_t field,
                                          int32_t comp, int64_t* dof) {
  if (!h || !point || !dof || field < 0 || field > 1 || comp < 0 || comp > 2)
    return set_error(DGTD_ERR_BAD_ARG, "nearest_node_dof: bad arguments");
  const auto& o = h->op;
  double best_d = std::numeric_limits<double>::max();
  int64_t best = 0;
  for (int64_t e = 0; e < o.K; ++e)
    for (int node = 0; node < o.re.np; ++node) {
      V3 p = o.map(e, o.re.nodes[node]);
      double d = dgtd::host::powi(p[0] - point[0], 2) + dgtd::host::powi(p[1] - point[1], 2) +
                 dgtd::host::powi(p[2] - point[2], 2);
      if (d < best_d) { best_d = d; best = (e * o.re.np + node) * 6 + field * 3 + comp; }
    }
  *dof = best;
  return DGTD_OK;
}

extern "C" int dgtd_host_port_n_faces(const dgtd_host_op* h, int32_t port, int64_t* n_faces) {
  if (!h || !n_faces) return set_error(DGTD_ERR_BAD_ARG, "port_n_faces: null argument");
  int64_t c = 0;
  for (int32_t p : h->op.port) c += (p == port);
  *n_faces = c;
  return DGTD_OK;
}

extern "C" int dgtd_host_rect_port_profiles(const dgtd_host_op* h, int32_t port,
                                            const double* inward_normal, int32_t mode_m,
                                            int32_t mode_n, double* out) {
  if (!h || !inward_normal || !out || (mode_m == 0 && mode_n == 0) || mode_m < 0 || mode_n < 0)
    return set_error(DGTD_ERR_BAD_ARG, "rect_port_profiles: bad arguments");
  const auto& o = h->op;
  const int nfp = o.re.nfp;
  // Port face nodes (the frame fit only needs their extents; mesh vertices and
  // DG face nodes span the same rectangle).
  std::vector<V3> pts;
  for (int64_t e = 0; e < o.K; ++e)
    for (int f = 0; f < 4; ++f)
      if (o.port[4 * e + f] == port)
        for (int m = 0; m < nfp; ++m) pts.push_back(o.map(e, o.re.nodes[o.re.face_nodes[size_t(f) * nfp + m]]));
  if (pts.empty()) return set_error(DGTD_ERR_BAD_ARG, "rect_port_profiles: port has no faces");
  // FaceFrame::fit (waveguide.rs:39-81).
  int k = 0;
  for (int i = 1; i < 3; ++i)
    if (std::fabs(inward_normal[i]) > std::fabs(inward_normal[k])) k = i;
  const double s = inward_normal[k] >= 0.0 ? 1.0 : -1.0;
  int others[2], oc = 0;
  for (int i = 0; i < 3; ++i) if (i != k) others[oc++] = i;
  auto extent = [&](int ax, double& lo, double& ext) {
    double l = std::numeric_limits<double>::max(), hi = std::numeric_limits<double>::lowest();
    for (auto& p : pts) { l = std::min(l, p[ax]); hi = std::max(hi, p[ax]); }
    lo = l; ext = hi - l;
  };
  double lo0, ext0, lo1, ext1;
  extent(others[0], lo0, ext0);
  extent(others[1], lo1, ext1);
  int wide, narrow;
  double a, b, lo_w, lo_n;
  if (ext0 >= ext1) { wide = others[0]; narrow = others[1]; a = ext0; b = ext1; lo_w = lo0; lo_n = lo1; }
  else { wide = others[1]; narrow = others[0]; a = ext1; b = ext0; lo_w = lo1; lo_n = lo0; }
  V3 u{0, 0, 0}, v{0, 0, 0}, w{0, 0, 0}, org{0, 0, 0};
  u[wide] = 1.0; v[narrow] = 1.0; w[k] = s;
  org[wide] = lo_w; org[k] = pts[0][k];
  if (dot(cross(u, v), w) >= 0.0) org[narrow] = lo_n;
  else { v[narrow] = -1.0; org[narrow] = lo_n + b; }
  const double mm = mode_m, nn = mode_n, PI = 3.14159265358979323846;
  size_t idx = 0;
  for (auto& x : pts) {
    V3 d{x[0] - org[0], x[1] - org[1], x[2] - org[2]};
    const double uu = dot(d, u), vv = dot(d, v);
    const double mu = mm * PI / a, nv = nn * PI / b;
    double eu = (nn / b) * std::cos(mu * uu) * std::sin(nv * vv);
    double ev = -(mm / a) * std::sin(mu * uu) * std::cos(nv * vv);
    const double scale = std::max(std::max(mm / a, nn / b), std::numeric_limits<double>::min());
    eu /= scale; ev /= scale;
    V3 et{eu * u[0] + ev * v[0], eu * u[1] + ev * v[1], eu * u[2] + ev * v[2]};
    V3 ht = cross(w, et);
    for (int q = 0; q < 3; ++q) { out[6 * idx + q] = et[q]; out[6 * idx + 3 + q] = ht[q]; }
    ++idx;
  }
  return DGTD_OK;
}

// The modal projections of port_modal_projections (rhs.rs:1211-1242) as linear
// functionals of the AoS state: P_e = sum_k w[k] y[idx[k]] over the E components
// of the port face nodes (which = 0), P_h over the H components (which = 1).
// n_faces * nfp * 3 terms, in port-face order.  A zero-norm profile gives zero
// weights (the reference returns 0 then).
extern "C" int dgtd_host_port_modal_weights(const dgtd_host_op* h, int32_t port, const double* profiles,
                                            int32_t which, int64_t* idx, double* w) {
  if (!h || !profiles || !idx || !w || (which != 0 && which != 1))
    return set_error(DGTD_ERR_BAD_ARG, "port_modal_weights: bad arguments");
  const auto& o = h->op;
  const int np = o.re.np, nfp = o.re.nfp;
  double norm = 0.0;
  size_t fi = 0, k = 0;
  for (int64_t e = 0; e < o.K; ++e)
    for (int f = 0; f < 4; ++f) {
      const int64_t ef = 4 * e + f;
      if (o.port[ef] != port) continue;
      const double area = o.fscale[ef] * std::fabs(o.det[e]) / 2.0;
      for (int m = 0; m < nfp; ++m) {
        const double* pr = profiles + 6 * (fi * nfp + m) + 3 * which;
        const double wn = 2.0 * area * o.re.face_w[size_t(f) * nfp + m];
        const int vi = o.re.face_nodes[size_t(f) * nfp + m];
        const int64_t base = (e * np + vi) * 6 + 3 * which;
        norm += wn * (pr[0] * pr[0] + pr[1] * pr[1] + pr[2] * pr[2]);
        for (int c = 0; c < 3; ++c) {
          idx[k] = base + c;
          w[k] = wn * pr[c];
          ++k;
        }
      }
      ++fi;
    }
  const double inv = norm > 0.0 ? 1.0 / norm : 0.0;
  for (size_t q = 0; q < k; ++q) w[q] *= inv;
  return DGTD_OK;
}

extern "C" int dgtd_host_port_source(const dgtd_host_op* h, int32_t port, const double* profiles,
                                     double* b) {
  if (!h || !profiles || !b) return set_error(DGTD_ERR_BAD_ARG, "port_source: null argument");
  const auto& o = h->op;
  const int np = o.re.np, nfp = o.re.nfp, cols = 4 * nfp;
  std::memset(b, 0, sizeof(double) * size_t(6) * np * o.K);
  size_t fi = 0;
  for (int64_t e = 0; e < o.K; ++e)
    for (int f = 0; f < 4; ++f) {
      const int64_t ef = 4 * e + f;
      if (o.port[ef] != port) continue;
      const V3 n{o.normal[3 * ef], o.normal[3 * ef + 1], o.normal[3 * ef + 2]};
      const double coef = 0.5 * o.fscale[ef];
      for (int m = 0; m < nfp; ++m) {
        const double* pr = profiles + 6 * (fi * nfp + m);
        const V3 et{pr[0], pr[1], pr[2]}, ht{pr[3], pr[4], pr[5]};
        const V3 nxe = cross(n, et), nxh = cross(n, ht);
        const V3 nne = cross(n, nxe), nnh = cross(n, nxh);
        const V3 sde{nxh[0] - nne[0], nxh[1] - nne[1], nxh[2] - nne[2]};
        const V3 sdh{-nxe[0] - nnh[0], -nxe[1] - nnh[1], -nxe[2] - nnh[2]};
        for (int i = 0; i < np; ++i) {
          const double wgt = coef * o.re.lift(i, f * nfp + m);
          const size_t base = (size_t(e) * np + i) * 6;
          for (int c = 0; c < 3; ++c) {
            b[base + c] += o.inv_eps[3 * e + c] * wgt * sde[c];
            b[base + 3 + c] += o.inv_mu[3 * e + c] * wgt * sdh[c];
          }
        }
      }
      ++fi;
    }
  return DGTD_OK;
}
