/*
 * dgtd_oracle.c -- CPU restatement of rapidfem's DGTD path, f64.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed
 * CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * legs load it, and only as the checker: nothing in rapidfem_b200/ links,
 * imports or calls it.
 *
 * Every function restates the reference algorithm step by step (same loop
 * order, same formulas) so that its f64 results track the reference's own
 * f64 CPU path to rounding.  Each block cites the reference file:line it
 * follows (paths relative to the rapidfem project root).
 *
 * Build: oracle/Makefile  ->  oracle/_build/libdgtd_oracle.so
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_NONE (-1)

/* ------------------------------------------------------------------------
 * Small helpers
 * --------------------------------------------------------------------- */

/* Integer power by binary exponentiation, the lowering of Rust's `powi`
 * (compiler-rt __powidf2).  Used wherever the reference calls `powi`. */
static double powi_d(double a, int b) {
    int recip = b < 0;
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

static double factorial(int n) {
    double p = 1.0;
    for (int k = 1; k <= n; k++) p *= (double)k;
    return p;
}

static void cross3(const double *a, const double *b, double *o) {
    double x = a[1] * b[2] - a[2] * b[1];
    double y = a[2] * b[0] - a[0] * b[2];
    double z = a[0] * b[1] - a[1] * b[0];
    o[0] = x; o[1] = y; o[2] = z;
}
static double dot3(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* Gauss-Jordan inverse with partial pivoting.
 * crates/rapidfem-td/src/dg_basis.rs:160-206 (`invert`). */
static int invert(const double *src, int n, double *inv) {
    double *a = (double *)malloc(sizeof(double) * n * n);
    memcpy(a, src, sizeof(double) * n * n);
    memset(inv, 0, sizeof(double) * n * n);
    for (int i = 0; i < n; i++) inv[i * n + i] = 1.0;
    for (int col = 0; col < n; col++) {
        int piv = col;
        double best = fabs(a[col * n + col]);
        for (int r = col + 1; r < n; r++) {
            double v = fabs(a[r * n + col]);
            if (v > best) { best = v; piv = r; }
        }
        if (!(best > 1e-300)) { free(a); return -1; }
        if (piv != col) {
            for (int k = 0; k < n; k++) {
                double t = a[col * n + k]; a[col * n + k] = a[piv * n + k]; a[piv * n + k] = t;
                t = inv[col * n + k]; inv[col * n + k] = inv[piv * n + k]; inv[piv * n + k] = t;
            }
        }
        double d = a[col * n + col];
        for (int k = 0; k < n; k++) { a[col * n + k] /= d; inv[col * n + k] /= d; }
        for (int r = 0; r < n; r++) {
            if (r == col) continue;
            double f = a[r * n + col];
            if (f == 0.0) continue;
            for (int k = 0; k < n; k++) {
                a[r * n + k] -= f * a[col * n + k];
                inv[r * n + k] -= f * inv[col * n + k];
            }
        }
    }
    free(a);
    return 0;
}

/* out = A*B skipping zero entries of A.  dg_basis.rs:213-237 (`matmul_into`). */
static void matmul_into(const double *a, const double *b, int rows, int inner,
                        int cols, double *out) {
    memset(out, 0, sizeof(double) * rows * cols);
    for (int i = 0; i < rows; i++)
        for (int k = 0; k < inner; k++) {
            double aik = a[i * inner + k];
            if (aik == 0.0) continue;
            for (int j = 0; j < cols; j++) out[i * cols + j] += aik * b[k * cols + j];
        }
}

/* C^T G C.  dg_basis.rs:247-261 (`triple_product`). */
static void triple_product(const double *c, const double *g, int n, double *out) {
    double *ctg = (double *)malloc(sizeof(double) * n * n);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < n; k++) {
            double acc = 0.0;
            for (int m = 0; m < n; m++) acc += c[m * n + i] * g[m * n + k];
            ctg[i * n + k] = acc;
        }
    matmul_into(ctg, c, n, n, n, out);
    free(ctg);
}

/* ------------------------------------------------------------------------
 * Reference element.  dg_basis.rs:61-119 (`ReferenceElement::new`),
 * :123-134 (`monomials`), :265-279 (`equispaced_ijk`), :288-385 (`build_lift`).
 * --------------------------------------------------------------------- */

typedef struct {
    int order, np, nfp;
    double *nodes;      /* np*3, (r,s,t) */
    double *mass;       /* np*np */
    double *dr, *ds, *dt;
    int *face_nodes;    /* 4*nfp */
    double *lift;       /* np*4nfp */
    double *face_w;     /* 4*nfp */
} orc_refelem;

static int orc_refelem_build(int p, orc_refelem *re) {
    int n = (p + 1) * (p + 2) * (p + 3) / 6;
    int nfp = (p + 1) * (p + 2) / 2;
    re->order = p; re->np = n; re->nfp = nfp;
    int (*monos)[3] = malloc(sizeof(int) * 3 * n);
    int (*ijk)[3] = malloc(sizeof(int) * 3 * n);
    int c = 0;
    for (int deg = 0; deg <= p; deg++)
        for (int a = 0; a <= deg; a++)
            for (int b = 0; b <= deg - a; b++) {
                monos[c][0] = a; monos[c][1] = b; monos[c][2] = deg - a - b; c++;
            }
    c = 0;
    for (int i = 0; i <= p; i++)
        for (int j = 0; j <= p - i; j++)
            for (int k = 0; k <= p - i - j; k++) {
                ijk[c][0] = i; ijk[c][1] = j; ijk[c][2] = k; c++;
            }
    re->nodes = malloc(sizeof(double) * 3 * n);
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) re->nodes[i * 3 + d] = (double)ijk[i][d] / (double)p;

    double *V = malloc(sizeof(double) * n * n), *C = malloc(sizeof(double) * n * n);
    double *G = malloc(sizeof(double) * n * n);
    for (int ni = 0; ni < n; ni++)
        for (int mi = 0; mi < n; mi++) {
            const double *x = re->nodes + 3 * ni;
            V[ni * n + mi] = powi_d(x[0], monos[mi][0]) * powi_d(x[1], monos[mi][1]) *
                             powi_d(x[2], monos[mi][2]);
        }
    if (invert(V, n, C)) return -1;
    for (int mi = 0; mi < n; mi++)
        for (int qi = 0; qi < n; qi++) {
            int a = monos[mi][0] + monos[qi][0], b = monos[mi][1] + monos[qi][1],
                cc = monos[mi][2] + monos[qi][2];
            G[mi * n + qi] = factorial(a) * factorial(b) * factorial(cc) / factorial(a + b + cc + 3);
        }
    re->mass = malloc(sizeof(double) * n * n);
    triple_product(C, G, n, re->mass);
    double *minv = malloc(sizeof(double) * n * n);
    if (invert(re->mass, n, minv)) return -1;

    double *Vd[3];
    for (int ax = 0; ax < 3; ax++) Vd[ax] = malloc(sizeof(double) * n * n);
    for (int ni = 0; ni < n; ni++)
        for (int mi = 0; mi < n; mi++) {
            const double *x = re->nodes + 3 * ni;
            for (int ax = 0; ax < 3; ax++) {
                int e = monos[mi][ax];
                double v = 0.0;
                if (e != 0) {
                    int d[3] = {monos[mi][0], monos[mi][1], monos[mi][2]};
                    d[ax] -= 1;
                    v = (double)e * (powi_d(x[0], d[0]) * powi_d(x[1], d[1]) * powi_d(x[2], d[2]));
                }
                Vd[ax][ni * n + mi] = v;
            }
        }
    re->dr = malloc(sizeof(double) * n * n);
    re->ds = malloc(sizeof(double) * n * n);
    re->dt = malloc(sizeof(double) * n * n);
    matmul_into(Vd[0], C, n, n, n, re->dr);
    matmul_into(Vd[1], C, n, n, n, re->ds);
    matmul_into(Vd[2], C, n, n, n, re->dt);

    /* build_lift */
    int cols = 4 * nfp;
    re->face_nodes = malloc(sizeof(int) * 4 * nfp);
    re->face_w = malloc(sizeof(double) * 4 * nfp);
    double *emat = calloc((size_t)n * cols, sizeof(double));
    int (*monos2)[2] = malloc(sizeof(int) * 2 * nfp);
    c = 0;
    for (int deg = 0; deg <= p; deg++)
        for (int a = 0; a <= deg; a++) { monos2[c][0] = a; monos2[c][1] = deg - a; c++; }
    double *v2 = malloc(sizeof(double) * nfp * nfp), *c2 = malloc(sizeof(double) * nfp * nfp);
    double *g2 = malloc(sizeof(double) * nfp * nfp), *mf = malloc(sizeof(double) * nfp * nfp);
    double (*xy)[2] = malloc(sizeof(double) * 2 * nfp);
    for (int f = 0; f < 4; f++) {
        int cnt = 0;
        for (int idx = 0; idx < n; idx++) {
            const int *q = ijk[idx];
            int on = (f == 0) ? q[2] == 0 : (f == 1) ? q[0] == 0 : (f == 2) ? q[1] == 0
                                                                 : (q[0] + q[1] + q[2] == p);
            if (on) re->face_nodes[f * nfp + cnt++] = idx;
        }
        if (cnt != nfp) return -2;
        for (int a = 0; a < nfp; a++) {
            const int *q = ijk[re->face_nodes[f * nfp + a]];
            int u, v;
            switch (f) {
            case 0: u = q[0]; v = q[1]; break;
            case 1: u = q[1]; v = q[2]; break;
            case 2: u = q[0]; v = q[2]; break;
            default: u = q[0]; v = q[1]; break;
            }
            xy[a][0] = (double)u / (double)p;
            xy[a][1] = (double)v / (double)p;
        }
        for (int i = 0; i < nfp; i++)
            for (int j = 0; j < nfp; j++)
                v2[i * nfp + j] = powi_d(xy[i][0], monos2[j][0]) * powi_d(xy[i][1], monos2[j][1]);
        if (invert(v2, nfp, c2)) return -1;
        for (int i = 0; i < nfp; i++)
            for (int j = 0; j < nfp; j++) {
                int a = monos2[i][0] + monos2[j][0], b = monos2[i][1] + monos2[j][1];
                g2[i * nfp + j] = factorial(a) * factorial(b) / factorial(a + b + 2);
            }
        triple_product(c2, g2, nfp, mf);
        for (int a = 0; a < nfp; a++) {
            int vi = re->face_nodes[f * nfp + a];
            for (int m = 0; m < nfp; m++) emat[(size_t)vi * cols + f * nfp + m] = mf[a * nfp + m];
        }
        for (int a = 0; a < nfp; a++) {
            double s = 0.0;
            for (int m = 0; m < nfp; m++) s += mf[a * nfp + m];
            re->face_w[f * nfp + a] = s;
        }
    }
    re->lift = malloc(sizeof(double) * n * cols);
    matmul_into(minv, emat, n, n, cols, re->lift);

    free(monos); free(ijk); free(V); free(C); free(G); free(minv);
    for (int ax = 0; ax < 3; ax++) free(Vd[ax]);
    free(emat); free(monos2); free(v2); free(c2); free(g2); free(mf); free(xy);
    return 0;
}

static void orc_refelem_free(orc_refelem *re) {
    free(re->nodes); free(re->mass); free(re->dr); free(re->ds); free(re->dt);
    free(re->face_nodes); free(re->lift); free(re->face_w);
}

/* ------------------------------------------------------------------------
 * Structured meshes.  crates/rapidfem-td/src/mesh_gen.rs:16-76 (Kuhn box),
 * :86-139 (jittered box, `jitter_offset`).
 * --------------------------------------------------------------------- */

static const int KUHN[6][4] = {
    {0, 1, 3, 7}, {0, 3, 2, 7}, {0, 2, 6, 7}, {0, 6, 4, 7}, {0, 4, 5, 7}, {0, 5, 1, 7}};

static int cmp_int(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* Tets of an nx*ny*nz cell grid, each tet's vertex ids sorted ascending. */
void orc_kuhn_tets(int nx, int ny, int nz, int *tets) {
    int nxp = nx + 1, nyp = ny + 1;
    size_t t = 0;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
                for (int kt = 0; kt < 6; kt++) {
                    int v[4];
                    for (int q = 0; q < 4; q++) {
                        int cc = KUHN[kt][q];
                        int ii = i + (cc & 1), jj = j + ((cc >> 1) & 1), kk = k + ((cc >> 2) & 1);
                        v[q] = (kk * nyp + jj) * nxp + ii;
                    }
                    qsort(v, 4, sizeof(int), cmp_int);
                    for (int q = 0; q < 4; q++) tets[t * 4 + q] = v[q];
                    t++;
                }
}

/* Node coordinates of the box [0,lx]x[0,ly]x[0,lz], k outer, i inner. */
void orc_box_nodes(int nx, int ny, int nz, double lx, double ly, double lz, double *nodes) {
    size_t c = 0;
    for (int k = 0; k <= nz; k++)
        for (int j = 0; j <= ny; j++)
            for (int i = 0; i <= nx; i++) {
                nodes[c * 3 + 0] = lx * (double)i / (double)nx;
                nodes[c * 3 + 1] = ly * (double)j / (double)ny;
                nodes[c * 3 + 2] = lz * (double)k / (double)nz;
                c++;
            }
}

static double jitter_mix(uint64_t x) {
    x *= 0x9E3779B97F4A7C15ULL;
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ULL;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBULL;
    x ^= x >> 31;
    return ((double)x / (double)UINT64_MAX) * 2.0 - 1.0;
}

/* Jittered box nodes.  mesh_gen.rs:86-139. */
void orc_box_nodes_jittered(int nx, int ny, int nz, double lx, double ly, double lz,
                            double amplitude, uint64_t seed, double *nodes) {
    double hx = lx / nx, hy = ly / ny, hz = lz / nz;
    size_t c = 0;
    for (int k = 0; k <= nz; k++)
        for (int j = 0; j <= ny; j++)
            for (int i = 0; i <= nx; i++) {
                double p[3] = {hx * (double)i, hy * (double)j, hz * (double)k};
                uint64_t base = seed + (uint64_t)i * 0x01000193ULL + (uint64_t)j * 0x00000100000001B3ULL +
                                (uint64_t)k * 0xC2B2AE3D27D4EB4FULL;
                double off[3] = {jitter_mix(base), jitter_mix(base ^ 0xAAAA), jitter_mix(base ^ 0x5555)};
                if (i != 0 && i != nx) p[0] += amplitude * hx * off[0];
                if (j != 0 && j != ny) p[1] += amplitude * hy * off[1];
                if (k != 0 && k != nz) p[2] += amplitude * hz * off[2];
                nodes[c * 3 + 0] = p[0]; nodes[c * 3 + 1] = p[1]; nodes[c * 3 + 2] = p[2];
                c++;
            }
}

/* ------------------------------------------------------------------------
 * Operator.  crates/rapidfem-td/src/rhs.rs:805-1000 (`MaxwellOperator::new`),
 * geom_factors.rs:33-88, rapidfem-core topology.rs:50-91, mesh.rs:45-50.
 * --------------------------------------------------------------------- */

typedef struct {
    orc_refelem re;
    int n_elem;
    double flux_alpha;
    double *origin, *jac, *jinv, *det;         /* 3K, 9K, 9K, K */
    double *normal, *fscale;                   /* 12K, 4K */
    int *nbr, *nbr_lf, *port, *perm;           /* 4K, 4K, 4K, 4K*nfp */
    double *inv_eps, *inv_mu, *sig_e, *sig_m;  /* 3K each */
} orc_op;

static const int TET_FACE_LOCAL[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 2, 3}};
static const int TET_FACE_OPPOSITE[4] = {3, 1, 2, 0};

/* Face-key hash table: sorted vertex triple -> first (e,f) seen. */
typedef struct { int64_t key[3]; int ef; int ef2; } face_slot;

static uint64_t hash3(const int64_t *k) {
    uint64_t h = (uint64_t)k[0] * 0x9E3779B97F4A7C15ULL;
    h ^= (uint64_t)k[1] * 0xC2B2AE3D27D4EB4FULL + (h << 6) + (h >> 2);
    h ^= (uint64_t)k[2] * 0x165667B19E3779F9ULL + (h << 6) + (h >> 2);
    return h;
}

/* Affine map of reference point xi on element e.  geom_factors.rs:52-60. */
static void map_point(const orc_op *op, int e, const double *xi, double *x) {
    const double *J = op->jac + 9 * e;
    for (int i = 0; i < 3; i++) {
        x[i] = op->origin[3 * e + i];
        for (int k = 0; k < 3; k++) x[i] += J[i * 3 + k] * xi[k];
    }
}

#define ORC_PEC_PLATE (-2)
/* Build the operator.  `face_port` (4K, -1 = none, -2 = a face of an internal
 * PEC plate, severed from its neighbour on both sides) tags port faces; it may
 * be NULL.  `mat` (K*8: eps[3], mu[3], sigma, sigma_m) may be NULL (vacuum). */
orc_op *orc_op_build(const double *nodes, int n_nodes, const int *tets, int n_elem, int order,
                     double flux_alpha, const int *face_port, const double *mat) {
    (void)n_nodes;
    orc_op *op = (orc_op *)calloc(1, sizeof(orc_op));
    if (orc_refelem_build(order, &op->re)) { free(op); return NULL; }
    int K = n_elem, nfp = op->re.nfp;
    op->n_elem = K;
    op->flux_alpha = flux_alpha;
    op->origin = malloc(sizeof(double) * 3 * K);
    op->jac = malloc(sizeof(double) * 9 * K);
    op->jinv = malloc(sizeof(double) * 9 * K);
    op->det = malloc(sizeof(double) * K);
    op->normal = malloc(sizeof(double) * 12 * K);
    op->fscale = malloc(sizeof(double) * 4 * K);
    op->nbr = malloc(sizeof(int) * 4 * K);
    op->nbr_lf = malloc(sizeof(int) * 4 * K);
    op->port = malloc(sizeof(int) * 4 * K);
    op->perm = calloc((size_t)4 * K * nfp, sizeof(int));
    op->inv_eps = malloc(sizeof(double) * 3 * K);
    op->inv_mu = malloc(sizeof(double) * 3 * K);
    op->sig_e = malloc(sizeof(double) * 3 * K);
    op->sig_m = malloc(sizeof(double) * 3 * K);

    /* Geometric factors: J columns v_{k+1}-v0, closed-form inverse. */
    for (int e = 0; e < K; e++) {
        const double *v[4];
        for (int q = 0; q < 4; q++) v[q] = nodes + 3 * (size_t)tets[4 * e + q];
        double c[3][3];
        for (int k = 0; k < 3; k++)
            for (int i = 0; i < 3; i++) c[k][i] = v[k + 1][i] - v[0][i];
        double m[3][3];
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++) m[i][k] = c[k][i];
        double adj[3][3];
        cross3(m[1], m[2], adj[0]);
        cross3(m[2], m[0], adj[1]);
        cross3(m[0], m[1], adj[2]);
        double det = dot3(m[0], adj[0]);
        double id = 1.0 / det;
        for (int i = 0; i < 3; i++) {
            op->origin[3 * e + i] = v[0][i];
            for (int k = 0; k < 3; k++) {
                op->jac[9 * e + i * 3 + k] = m[i][k];
                op->jinv[9 * e + i * 3 + k] = adj[k][i] * id;
            }
        }
        op->det[e] = det;
    }

    /* Face topology: outward normals, area, neighbour by shared vertex set. */
    double *area = malloc(sizeof(double) * 4 * K);
    for (int e = 0; e < K; e++)
        for (int lf = 0; lf < 4; lf++) {
            const double *v0 = nodes + 3 * (size_t)tets[4 * e + TET_FACE_LOCAL[lf][0]];
            const double *v1 = nodes + 3 * (size_t)tets[4 * e + TET_FACE_LOCAL[lf][1]];
            const double *v2 = nodes + 3 * (size_t)tets[4 * e + TET_FACE_LOCAL[lf][2]];
            const double *vo = nodes + 3 * (size_t)tets[4 * e + TET_FACE_OPPOSITE[lf]];
            double a[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
            double b[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
            double n[3];
            cross3(a, b, n);
            double len = sqrt(dot3(n, n));
            area[4 * e + lf] = 0.5 * len;
            for (int k = 0; k < 3; k++) n[k] /= len;
            double d[3] = {vo[0] - v0[0], vo[1] - v0[1], vo[2] - v0[2]};
            if (dot3(d, n) > 0.0)
                for (int k = 0; k < 3; k++) n[k] = -n[k];
            for (int k = 0; k < 3; k++) op->normal[12 * e + 3 * lf + k] = n[k];
        }
    size_t cap = 1;
    while (cap < (size_t)8 * K) cap <<= 1;
    face_slot *tab = (face_slot *)malloc(sizeof(face_slot) * cap);
    for (size_t i = 0; i < cap; i++) tab[i].ef = -1;
    for (int e = 0; e < K; e++)
        for (int lf = 0; lf < 4; lf++) {
            int64_t k3[3];
            for (int q = 0; q < 3; q++) k3[q] = tets[4 * e + TET_FACE_LOCAL[lf][q]];
            /* sort */
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2 - a; b++)
                    if (k3[b] > k3[b + 1]) { int64_t t = k3[b]; k3[b] = k3[b + 1]; k3[b + 1] = t; }
            size_t h = hash3(k3) & (cap - 1);
            for (;;) {
                if (tab[h].ef < 0) {
                    memcpy(tab[h].key, k3, sizeof(k3));
                    tab[h].ef = 4 * e + lf;
                    tab[h].ef2 = -1;
                    break;
                }
                if (!memcmp(tab[h].key, k3, sizeof(k3))) {
                    if (tab[h].ef2 < 0) tab[h].ef2 = 4 * e + lf; /* keeps the first two */
                    break;
                }
                h = (h + 1) & (cap - 1);
            }
        }
    for (int i = 0; i < 4 * K; i++) { op->nbr[i] = ORC_NONE; op->nbr_lf[i] = ORC_NONE; }
    for (size_t i = 0; i < cap; i++) {
        if (tab[i].ef < 0 || tab[i].ef2 < 0) continue;
        int a = tab[i].ef, b = tab[i].ef2;
        op->nbr[a] = b / 4; op->nbr_lf[a] = b % 4;
        op->nbr[b] = a / 4; op->nbr_lf[b] = a % 4;
    }
    free(tab);

    /* Per (e,f): fscale, perm by nearest-node match (tol^2 = 1e-18 absolute),
     * port tag.  rhs.rs:825-854, rhs.rs:546-566. */
    int np = op->re.np;
    double *here = malloc(sizeof(double) * 3 * nfp), *there = malloc(sizeof(double) * 3 * nfp);
    int bad = 0;
    for (int e = 0; e < K; e++)
        for (int f = 0; f < 4; f++) {
            int ef = 4 * e + f;
            op->fscale[ef] = 2.0 * area[ef] / fabs(op->det[e]);
            op->port[ef] = face_port ? face_port[ef] : ORC_NONE;
            if (op->port[ef] == ORC_PEC_PLATE) {
                /* internal PEC plate: sever the face on this side, the PEC
                 * ghost state applies (rhs.rs:862-880) */
                op->port[ef] = ORC_NONE;
                op->nbr[ef] = ORC_NONE;
                op->nbr_lf[ef] = 0;
            }
            if (op->nbr[ef] == ORC_NONE) continue;
            int en = op->nbr[ef], fn = op->nbr_lf[ef];
            for (int m = 0; m < nfp; m++) {
                map_point(op, e, op->re.nodes + 3 * op->re.face_nodes[f * nfp + m], here + 3 * m);
                map_point(op, en, op->re.nodes + 3 * op->re.face_nodes[fn * nfp + m], there + 3 * m);
            }
            for (int m = 0; m < nfp; m++) {
                double best = 1.79769313486231570e+308;
                int bm = 0;
                for (int m2 = 0; m2 < nfp; m2++) {
                    double d = powi_d(here[3 * m] - there[3 * m2], 2) +
                               powi_d(here[3 * m + 1] - there[3 * m2 + 1], 2) +
                               powi_d(here[3 * m + 2] - there[3 * m2 + 2], 2);
                    if (d < best) { best = d; bm = m2; }
                }
                if (!(best < 1e-18)) bad = 1;
                op->perm[(size_t)ef * nfp + m] = bm;
            }
        }
    (void)np;
    free(here); free(there); free(area);
    if (bad) return NULL;

    /* Materials.  rhs.rs:900-926. */
    for (int e = 0; e < K; e++) {
        double eps[3] = {1, 1, 1}, mu[3] = {1, 1, 1}, sg = 0.0, sm = 0.0;
        if (mat) {
            for (int c = 0; c < 3; c++) { eps[c] = mat[8 * e + c]; mu[c] = mat[8 * e + 3 + c]; }
            sg = mat[8 * e + 6]; sm = mat[8 * e + 7];
        }
        for (int c = 0; c < 3; c++) {
            op->inv_eps[3 * e + c] = 1.0 / eps[c];
            op->inv_mu[3 * e + c] = 1.0 / mu[c];
            op->sig_e[3 * e + c] = sg / eps[c];
            op->sig_m[3 * e + c] = sm / mu[c];
        }
    }
    return op;
}

void orc_op_free(orc_op *op) {
    if (!op) return;
    orc_refelem_free(&op->re);
    free(op->origin); free(op->jac); free(op->jinv); free(op->det);
    free(op->normal); free(op->fscale);
    free(op->nbr); free(op->nbr_lf); free(op->port); free(op->perm);
    free(op->inv_eps); free(op->inv_mu); free(op->sig_e); free(op->sig_m);
    free(op);
}

int orc_op_np(const orc_op *op) { return op->re.np; }
int orc_op_nfp(const orc_op *op) { return op->re.nfp; }
int orc_op_n_elem(const orc_op *op) { return op->n_elem; }
long orc_op_n_dof(const orc_op *op) { return 6L * op->re.np * op->n_elem; }

/* Copy-out accessors for the tests.  `which` names the array. */
int orc_op_get(const orc_op *op, const char *which, double *out) {
    int K = op->n_elem, np = op->re.np, nfp = op->re.nfp;
#define CPYD(name, src, cnt) if (!strcmp(which, name)) { for (size_t i = 0; i < (size_t)(cnt); i++) out[i] = (double)(src)[i]; return 0; }
    CPYD("nodes", op->re.nodes, 3 * np)
    CPYD("mass", op->re.mass, np * np)
    CPYD("dr", op->re.dr, np * np)
    CPYD("ds", op->re.ds, np * np)
    CPYD("dt", op->re.dt, np * np)
    CPYD("lift", op->re.lift, np * 4 * nfp)
    CPYD("face_nodes", op->re.face_nodes, 4 * nfp)
    CPYD("face_w", op->re.face_w, 4 * nfp)
    CPYD("jinv", op->jinv, 9 * K)
    CPYD("jac", op->jac, 9 * K)
    CPYD("origin", op->origin, 3 * K)
    CPYD("det", op->det, K)
    CPYD("normal", op->normal, 12 * K)
    CPYD("fscale", op->fscale, 4 * K)
    CPYD("nbr", op->nbr, 4 * K)
    CPYD("nbr_lf", op->nbr_lf, 4 * K)
    CPYD("port", op->port, 4 * K)
    CPYD("perm", op->perm, (size_t)4 * K * nfp)
    CPYD("inv_eps", op->inv_eps, 3 * K)
    CPYD("inv_mu", op->inv_mu, 3 * K)
    CPYD("sigma_eps", op->sig_e, 3 * K)
    CPYD("sigma_mu", op->sig_m, 3 * K)
#undef CPYD
    return -1;
}

/* Retag face (e,f) -- used for internal PEC plates / ports after the build. */
void orc_op_set_port(orc_op *op, int ef, int port) { op->port[ef] = port; }

/* ------------------------------------------------------------------------
 * Periodic face pairs.  rhs.rs:546-568 (`match_face_nodes`), rhs.rs:588-614
 * (`periodic_face_centroid`), rhs.rs:616-770 (`link_periodic_faces`), with
 * PERIODIC_MATCH_REL_TOL = 1e-9 and PERIODIC_MATCH_ABS_FLOOR = 1e-12
 * (constants.rs:216-222).  Faces are ids e*4+lf; triangle coordinates come
 * from the mesh nodes, as in the reference.  Returns 0, or: 1 counts differ,
 * 2 a port face, 3 a face with a neighbour, 4 zero area, 5 a side-A face
 * without partner, 6 not a bijection, 7 an unmatched face node.  Matching is
 * the reference's all-pairs nearest search; the operator changes only when
 * every check passed.
 * --------------------------------------------------------------------- */

static void tri_xyz(const double *nodes, const int *tets, int ef, double v[3][3]) {
    for (int q = 0; q < 3; q++)
        for (int k = 0; k < 3; k++)
            v[q][k] = nodes[3 * (size_t)tets[4 * (ef / 4) + TET_FACE_LOCAL[ef % 4][q]] + k];
}

static int match_face_nodes(const orc_op *op, int here, int there, const double *shift, double tol2,
                            int *perm) {
    int nfp = op->re.nfp;
    double ph[21 * 3], pt[21 * 3];
    for (int m = 0; m < nfp; m++) {
        map_point(op, here / 4, op->re.nodes + 3 * op->re.face_nodes[(here % 4) * nfp + m], ph + 3 * m);
        map_point(op, there / 4, op->re.nodes + 3 * op->re.face_nodes[(there % 4) * nfp + m], pt + 3 * m);
    }
    for (int m = 0; m < nfp; m++) {
        double t[3] = {ph[3 * m] + shift[0], ph[3 * m + 1] + shift[1], ph[3 * m + 2] + shift[2]};
        double best = 1.79769313486231570e+308;
        int bm = 0;
        for (int m2 = 0; m2 < nfp; m2++) {
            double d = powi_d(t[0] - pt[3 * m2], 2) + powi_d(t[1] - pt[3 * m2 + 1], 2) +
                       powi_d(t[2] - pt[3 * m2 + 2], 2);
            if (d < best) { best = d; bm = m2; }
        }
        if (!(best < tol2)) return 1;
        perm[m] = bm;
    }
    return 0;
}

int orc_link_periodic(orc_op *op, const double *nodes, const int *tets, const long *faces_a, int n_a,
                      const long *faces_b, int n_b) {
    if (n_a != n_b) return 1;
    int n = n_a, nfp = op->re.nfp;
    for (int i = 0; i < 2 * n; i++) {
        long ef = i < n ? faces_a[i] : faces_b[i - n];
        if (op->port[ef] != ORC_NONE) return 2;
        if (op->nbr[ef] != ORC_NONE) return 3;
    }
    double *cen = malloc(sizeof(double) * 6 * (size_t)n);  /* A then B triangle centroids */
    double side[2][3] = {{0, 0, 0}, {0, 0, 0}}, total[2] = {0, 0};
    for (int i = 0; i < 2 * n; i++) {
        int s = i >= n;
        double v[3][3], e1[3], e2[3], nn[3];
        tri_xyz(nodes, tets, (int)(s ? faces_b[i - n] : faces_a[i]), v);
        for (int k = 0; k < 3; k++) { e1[k] = v[1][k] - v[0][k]; e2[k] = v[2][k] - v[0][k]; }
        cross3(e1, e2, nn);
        double area = 0.5 * sqrt(dot3(nn, nn));
        for (int k = 0; k < 3; k++) {
            side[s][k] += area * (v[0][k] + v[1][k] + v[2][k]) / 3.0;
            cen[3 * (size_t)i + k] = (v[0][k] + v[1][k] + v[2][k]) / 3.0;
        }
        total[s] += area;
    }
    int rc = 0;
    int *a2b = malloc(sizeof(int) * (size_t)n), *b2a = malloc(sizeof(int) * (size_t)n);
    int *perm = malloc(sizeof(int) * 2 * (size_t)n * nfp);
    if (!(total[0] > 0.0) || !(total[1] > 0.0)) { rc = 4; goto done; }
    double trans[3], back[3];
    for (int k = 0; k < 3; k++) {
        trans[k] = side[1][k] / total[1] - side[0][k] / total[0];
        back[k] = -trans[k];
    }
    double mag = sqrt(dot3(trans, trans));
    double tol = 1e-9 * mag > 1e-12 ? 1e-9 * mag : 1e-12;
    double tol2 = tol * tol;
    for (int i = 0; i < n; i++) b2a[i] = -1;
    for (int i = 0; i < n; i++) {
        double t[3] = {cen[3 * i] + trans[0], cen[3 * i + 1] + trans[1], cen[3 * i + 2] + trans[2]};
        double best = 1.79769313486231570e+308;
        int bi = -1;
        for (int j = 0; j < n; j++) {
            const double *c = cen + 3 * ((size_t)n + j);
            double d = powi_d(t[0] - c[0], 2) + powi_d(t[1] - c[1], 2) + powi_d(t[2] - c[2], 2);
            if (d < best) { best = d; bi = j; }
        }
        if (!(best < tol2)) { rc = 5; goto done; }
        if (b2a[bi] >= 0) { rc = 6; goto done; }
        a2b[i] = bi;
        b2a[bi] = i;
    }
    for (int i = 0; i < n; i++) {
        int fa = (int)faces_a[i], fb = (int)faces_b[a2b[i]];
        if (match_face_nodes(op, fa, fb, trans, tol2, perm + (size_t)(2 * i) * nfp) ||
            match_face_nodes(op, fb, fa, back, tol2, perm + (size_t)(2 * i + 1) * nfp)) { rc = 7; goto done; }
    }
    for (int i = 0; i < n; i++) {
        int fa = (int)faces_a[i], fb = (int)faces_b[a2b[i]];
        op->nbr[fa] = fb / 4; op->nbr_lf[fa] = fb % 4;
        op->nbr[fb] = fa / 4; op->nbr_lf[fb] = fa % 4;
        memcpy(op->perm + (size_t)fa * nfp, perm + (size_t)(2 * i) * nfp, sizeof(int) * nfp);
        memcpy(op->perm + (size_t)fb * nfp, perm + (size_t)(2 * i + 1) * nfp, sizeof(int) * nfp);
    }
done:
    free(cen); free(a2b); free(b2a); free(perm);
    return rc;
}

/* ------------------------------------------------------------------------
 * The RHS.  rhs.rs:39-85 (`element_curl`), rhs.rs:1341-1473 (`apply_element`),
 * rhs.rs:1262-1325 (`apply_into`, contiguous element runs per task).
 * --------------------------------------------------------------------- */

/* Physical curl of field (node-major [node*3+comp]) into out.  rhs.rs:39-85. */
void orc_element_curl(const orc_op *op, int np, const double *dr, const double *ds,
                      const double *dt, const double *jinv, const double *field, double *out,
                      double *rd, double *pd) {
    (void)op;
    int n = np;
    const double *dref[3] = {dr, ds, dt};
    for (int comp = 0; comp < 3; comp++) {
        for (int k = 0; k < 3; k++) {
            const double *d = dref[k];
            for (int i = 0; i < n; i++) {
                double acc = 0.0;
                for (int j = 0; j < n; j++) acc += d[i * n + j] * field[j * 3 + comp];
                rd[k * n + i] = acc;
            }
        }
        for (int phys = 0; phys < 3; phys++) {
            double j0 = jinv[0 * 3 + phys], j1 = jinv[1 * 3 + phys], j2 = jinv[2 * 3 + phys];
            int base = (phys * 3 + comp) * n;
            for (int i = 0; i < n; i++) pd[base + i] = j0 * rd[i] + j1 * rd[n + i] + j2 * rd[2 * n + i];
        }
    }
#define IDX(p, c, i) (((p) * 3 + (c)) * n + (i))
    for (int i = 0; i < n; i++) {
        out[i * 3] = pd[IDX(1, 2, i)] - pd[IDX(2, 1, i)];
        out[i * 3 + 1] = pd[IDX(2, 0, i)] - pd[IDX(0, 2, i)];
        out[i * 3 + 2] = pd[IDX(0, 1, i)] - pd[IDX(1, 0, i)];
    }
#undef IDX
}

/* Stand-alone curl on one element given its Jacobian inverse (golden test). */
int orc_curl_single(int order, const double *jinv, const double *field, double *out) {
    orc_refelem re;
    if (orc_refelem_build(order, &re)) return -1;
    int n = re.np;
    double *rd = malloc(sizeof(double) * 3 * n), *pd = malloc(sizeof(double) * 9 * n);
    orc_element_curl(NULL, n, re.dr, re.ds, re.dt, jinv, field, out, rd, pd);
    free(rd); free(pd);
    orc_refelem_free(&re);
    return 0;
}

typedef struct { double *ee, *hh, *de, *dh, *rd, *pd; } orc_scratch;

static void apply_element(const orc_op *op, int e, const double *y, double *out, orc_scratch *s) {
    int np = op->re.np, nfp = op->re.nfp, cols = 4 * nfp;
    size_t base = (size_t)e * np * 6;
    for (int node = 0; node < np; node++)
        for (int c = 0; c < 3; c++) {
            s->ee[node * 3 + c] = y[base + node * 6 + c];
            s->hh[node * 3 + c] = y[base + node * 6 + 3 + c];
        }
    const double *jinv = op->jinv + 9 * e;
    orc_element_curl(op, np, op->re.dr, op->re.ds, op->re.dt, jinv, s->hh, s->de, s->rd, s->pd);
    orc_element_curl(op, np, op->re.dr, op->re.ds, op->re.dt, jinv, s->ee, s->dh, s->rd, s->pd);
    for (int i = 0; i < 3 * np; i++) s->dh[i] = -s->dh[i];

    for (int f = 0; f < 4; f++) {
        int ef = 4 * e + f;
        const double *n = op->normal + 3 * ef;
        double coef = 0.5 * op->fscale[ef];
        int port = op->port[ef], nbr = op->nbr[ef];
        for (int m = 0; m < nfp; m++) {
            int vi = op->re.face_nodes[f * nfp + m];
            double em[3] = {s->ee[vi * 3], s->ee[vi * 3 + 1], s->ee[vi * 3 + 2]};
            double hm[3] = {s->hh[vi * 3], s->hh[vi * 3 + 1], s->hh[vi * 3 + 2]};
            double je[3], jh[3];
            if (port != ORC_NONE) {
                for (int k = 0; k < 3; k++) { je[k] = em[k]; jh[k] = hm[k]; }
            } else if (nbr == ORC_NONE) {
                double edn = dot3(n, em), hdn = dot3(n, hm);
                for (int k = 0; k < 3; k++) {
                    je[k] = 2.0 * (em[k] - edn * n[k]);
                    jh[k] = 2.0 * hdn * n[k];
                }
            } else {
                int vj = op->re.face_nodes[op->nbr_lf[ef] * nfp + op->perm[(size_t)ef * nfp + m]];
                size_t nbb = (size_t)nbr * np * 6;
                for (int k = 0; k < 3; k++) {
                    je[k] = em[k] - y[nbb + vj * 6 + k];
                    jh[k] = hm[k] - y[nbb + vj * 6 + 3 + k];
                }
            }
            double nxjh[3], nxje[3], t[3], pe[3], ph[3];
            cross3(n, jh, nxjh);
            cross3(n, je, nxje);
            double a = (port != ORC_NONE) ? 1.0 : op->flux_alpha;
            cross3(n, je, t); cross3(n, t, pe);
            cross3(n, jh, t); cross3(n, t, ph);
            for (int i = 0; i < np; i++) {
                double w = coef * op->re.lift[i * cols + f * nfp + m];
                for (int c = 0; c < 3; c++) {
                    s->de[i * 3 + c] += w * (-nxjh[c] + a * pe[c]);
                    s->dh[i * 3 + c] += w * (nxje[c] + a * ph[c]);
                }
            }
        }
    }
    const double *ie = op->inv_eps + 3 * e, *im = op->inv_mu + 3 * e;
    const double *se = op->sig_e + 3 * e, *sm = op->sig_m + 3 * e;
    for (int node = 0; node < np; node++)
        for (int c = 0; c < 3; c++) {
            out[node * 6 + c] = ie[c] * s->de[node * 3 + c] - se[c] * s->ee[node * 3 + c];
            out[node * 6 + 3 + c] = im[c] * s->dh[node * 3 + c] - sm[c] * s->hh[node * 3 + c];
        }
}

static int g_threads = 0; /* 0 = OpenMP default */

void orc_set_threads(int t) { g_threads = t; }
int orc_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* dy = A*y over all elements, contiguous runs of n_elem/(4*threads)
 * elements per task.  rhs.rs:1262-1294. */
void orc_apply(const orc_op *op, const double *y, double *dy) {
    int K = op->n_elem, np = op->re.np;
    int threads = orc_get_threads();
    int chunk = K / (4 * threads);
    if (chunk < 1) chunk = 1;
    int nchunks = (K + chunk - 1) / chunk;
#pragma omp parallel num_threads(threads)
    {
        orc_scratch s;
        s.ee = malloc(sizeof(double) * 3 * np); s.hh = malloc(sizeof(double) * 3 * np);
        s.de = malloc(sizeof(double) * 3 * np); s.dh = malloc(sizeof(double) * 3 * np);
        s.rd = malloc(sizeof(double) * 3 * np); s.pd = malloc(sizeof(double) * 9 * np);
#pragma omp for schedule(dynamic, 1)
        for (int ci = 0; ci < nchunks; ci++) {
            int e1 = (ci + 1) * chunk;
            if (e1 > K) e1 = K;
            for (int e = ci * chunk; e < e1; e++) apply_element(op, e, y, dy + (size_t)e * np * 6, &s);
        }
        free(s.ee); free(s.hh); free(s.de); free(s.dh); free(s.rd); free(s.pd);
    }
}

/* ------------------------------------------------------------------------
 * LSERK4.  explicit.rs:100-135, constants.rs:106-122.
 * --------------------------------------------------------------------- */

static const double LSERK4_A[5] = {
    0.0,
    -567301805773.0 / 1357537059087.0,
    -2404267990393.0 / 2016746695238.0,
    -3550918686646.0 / 2091501179385.0,
    -1275806237668.0 / 842570457699.0,
};
static const double LSERK4_B[5] = {
    1432997174477.0 / 9575080441755.0,
    5161836677717.0 / 13612068292357.0,
    1720146321549.0 / 2090206949498.0,
    3134564353537.0 / 4481467310338.0,
    2277821191437.0 / 14882151754819.0,
};

void orc_lserk_coeffs(double *a, double *b) {
    for (int i = 0; i < 5; i++) { a[i] = LSERK4_A[i]; b[i] = LSERK4_B[i]; }
}

/* `steps` LSERK4 steps of dy/dt = A y + b, source held per step.
 * src_kind: 0 none, 1 point (src_dof, vals[step]), 2 vector (src_vec * vals[step]).
 * explicit.rs:44-56 (Source::add_to), :100-135 (step_into). */
void orc_lserk_steps(const orc_op *op, double *y, double dt, int steps, int src_kind,
                     long src_dof, const double *src_vec, const double *vals) {
    size_t n = (size_t)orc_op_n_dof(op);
    double *p = malloc(sizeof(double) * n), *k = malloc(sizeof(double) * n);
    int threads = orc_get_threads();
    for (int st = 0; st < steps; st++) {
        memset(p, 0, sizeof(double) * n);
        for (int stage = 0; stage < 5; stage++) {
            orc_apply(op, y, k);
            if (src_kind == 1) {
                if (src_dof >= 0 && (size_t)src_dof < n) k[src_dof] += vals[st];
            } else if (src_kind == 2) {
                double g = vals[st];
#pragma omp parallel for num_threads(threads)
                for (long i = 0; i < (long)n; i++) k[i] += src_vec[i] * g;
            }
            double a = LSERK4_A[stage], b = LSERK4_B[stage];
#pragma omp parallel for num_threads(threads)
            for (long i = 0; i < (long)n; i++) {
                p[i] = a * p[i] + dt * k[i];
                y[i] += b * p[i];
            }
        }
    }
    free(p); free(k);
}

/* ------------------------------------------------------------------------
 * KCL RK4(3)5[2R+]C.  explicit_adaptive.rs:84-152, constants.rs:151-178.
 * --------------------------------------------------------------------- */

static const double KCL_A[4] = {
    970286171893.0 / 4311952581923.0,
    6584761158862.0 / 12103376702013.0,
    2251764453980.0 / 15575788980749.0,
    26877169314380.0 / 34165994151039.0,
};
static const double KCL_B[5] = {
    1153189308089.0 / 22510343858157.0,
    1772645290293.0 / 4653164025191.0,
    -1672844663538.0 / 4480602732383.0,
    2114624349019.0 / 3568978502595.0,
    5198255086312.0 / 14908931495163.0,
};
static const double KCL_BHAT[5] = {
    1016888040809.0 / 7410784769900.0,
    11231460423587.0 / 58533540763752.0,
    -1563879915014.0 / 6823010717585.0,
    606302364029.0 / 971179775848.0,
    1097981568119.0 / 3980877426909.0,
};

void orc_kcl_coeffs(double *a4, double *b5, double *bhat5) {
    for (int i = 0; i < 4; i++) a4[i] = KCL_A[i];
    for (int i = 0; i < 5; i++) { b5[i] = KCL_B[i]; bhat5[i] = KCL_BHAT[i]; }
}

/* One KCL step in place; err receives the embedded-error vector.
 * src_kind as in orc_lserk_steps, with the single held value `g`. */
void orc_kcl_step(const orc_op *op, double *y, double *err, double dt, int src_kind, long src_dof,
                  const double *src_vec, double g) {
    size_t n = (size_t)orc_op_n_dof(op);
    double *k = malloc(sizeof(double) * n), *stg = malloc(sizeof(double) * n);
    orc_apply(op, y, k);
    if (src_kind == 1) k[src_dof] += g;
    else if (src_kind == 2) for (size_t i = 0; i < n; i++) k[i] += src_vec[i] * g;
    double b0 = KCL_B[0], e0 = KCL_BHAT[0] - b0;
    for (size_t i = 0; i < n; i++) {
        double f = dt * k[i];
        k[i] = f;
        y[i] += b0 * f;
        err[i] = e0 * f;
    }
    for (int stage = 1; stage < 5; stage++) {
        double amb = KCL_A[stage - 1] - KCL_B[stage - 1];
        for (size_t i = 0; i < n; i++) stg[i] = y[i] + amb * k[i];
        orc_apply(op, stg, k);
        if (src_kind == 1) k[src_dof] += g;
        else if (src_kind == 2) for (size_t i = 0; i < n; i++) k[i] += src_vec[i] * g;
        double b = KCL_B[stage], ew = KCL_BHAT[stage] - b;
        for (size_t i = 0; i < n; i++) {
            double f = dt * k[i];
            k[i] = f;
            y[i] += b * f;
            err[i] += ew * f;
        }
    }
    free(k); free(stg);
}

/* ------------------------------------------------------------------------
 * Dense expm and the Krylov propagator.  propagator.rs:69-114 (expm_into),
 * :186-326 (expmv_into, CGS2 + a-posteriori stop), :338-373 (etd_step_into),
 * constants.rs:58-99.
 * --------------------------------------------------------------------- */

#define EXPM_SCALE_THRESHOLD 0.5
#define EXPM_TAYLOR_TERMS 18
#define ARNOLDI_BREAKDOWN 1e-12

void orc_expm(const double *a, int n, double *out) {
    int nn = n * n;
    double *b = malloc(sizeof(double) * nn), *res = malloc(sizeof(double) * nn);
    double *term = malloc(sizeof(double) * nn), *term2 = malloc(sizeof(double) * nn);
    double *tmp = malloc(sizeof(double) * nn);
    double norm = 0.0;
    for (int i = 0; i < n; i++) {
        double row = 0.0;
        for (int j = 0; j < n; j++) row += fabs(a[i * n + j]);
        norm = fmax(norm, row);
    }
    unsigned sq = 0;
    if (norm > EXPM_SCALE_THRESHOLD) {
        long v = (long)ceil(log2(norm)) + 1;
        sq = v > 0 ? (unsigned)v : 0;
    }
    double scale = powi_d(2.0, (int)sq);
    for (int k = 0; k < nn; k++) b[k] = a[k] / scale;
    memset(res, 0, sizeof(double) * nn);
    memset(term, 0, sizeof(double) * nn);
    for (int i = 0; i < n; i++) { res[i * n + i] = 1.0; term[i * n + i] = 1.0; }
    for (int k = 1; k <= EXPM_TAYLOR_TERMS; k++) {
        matmul_into(term, b, n, n, n, term2);
        double inv = 1.0 / (double)k;
        for (int q = 0; q < nn; q++) term2[q] *= inv;
        for (int q = 0; q < nn; q++) res[q] += term2[q];
        memcpy(term, term2, sizeof(double) * nn);
    }
    for (unsigned s = 0; s < sq; s++) {
        matmul_into(res, res, n, n, n, tmp);
        memcpy(res, tmp, sizeof(double) * nn);
    }
    memcpy(out, res, sizeof(double) * nn);
    free(b); free(res); free(term); free(term2); free(tmp);
}

/* Generic matvec callback: ax = A x over vectors of length n. */
typedef void (*orc_matvec_fn)(void *ctx, const double *x, double *ax);

static double norm2(const double *a, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += a[i] * a[i];
    return sqrt(s);
}

/* exp(t A) v; returns the Krylov dimension used.  propagator.rs:186-326. */
int orc_expmv_cb(orc_matvec_fn mv, void *ctx, const double *v, size_t n, double t, int max_dim,
                 double tol, double *out) {
    double beta = norm2(v, n);
    if (beta == 0.0) { memset(out, 0, sizeof(double) * n); return 0; }
    double *basis = malloc(sizeof(double) * (size_t)(max_dim + 1) * n);
    double *w = malloc(sizeof(double) * n);
    double *proj = malloc(sizeof(double) * (max_dim + 1));
    double *h = calloc((size_t)max_dim * max_dim, sizeof(double));
    double *th = malloc(sizeof(double) * max_dim * max_dim);
    double *eth = malloc(sizeof(double) * max_dim * max_dim);
    double inv_beta = 1.0 / beta;
    for (size_t k = 0; k < n; k++) basis[k] = v[k] * inv_beta;
    int threads = orc_get_threads();
    int dim = max_dim;
    for (int j = 0; j < max_dim; j++) {
        mv(ctx, basis + (size_t)j * n, w);
        int cols = j + 1;
        for (int pass = 0; pass < 2; pass++) {
#pragma omp parallel for num_threads(threads)
            for (int i = 0; i < cols; i++) {
                const double *bi = basis + (size_t)i * n;
                double s = 0.0;
                for (size_t k = 0; k < n; k++) s += bi[k] * w[k];
                proj[i] = s;
            }
#pragma omp parallel for num_threads(threads)
            for (long k = 0; k < (long)n; k++) {
                double wk = w[k];
                for (int i = 0; i < cols; i++) wk -= proj[i] * basis[(size_t)i * n + k];
                w[k] = wk;
            }
            for (int i = 0; i < cols; i++) h[i * max_dim + j] += proj[i];
        }
        double hnext = norm2(w, n);
        int d = j + 1;
        if (hnext < ARNOLDI_BREAKDOWN || d == max_dim) { dim = d; break; }
        if (tol > 0.0) {
            for (int a = 0; a < d; a++)
                for (int b = 0; b < d; b++) th[a * d + b] = t * h[a * max_dim + b];
            orc_expm(th, d, eth);
            if (hnext * fabs(eth[(d - 1) * d]) < tol) { dim = d; break; }
        }
        h[(j + 1) * max_dim + j] = hnext;
        double inv = 1.0 / hnext;
        double *dst = basis + (size_t)(j + 1) * n;
        for (size_t k = 0; k < n; k++) dst[k] = w[k] * inv;
    }
    for (int i = 0; i < dim; i++)
        for (int j = 0; j < dim; j++) th[i * dim + j] = t * h[i * max_dim + j];
    orc_expm(th, dim, eth);
    memset(out, 0, sizeof(double) * n);
    for (int i = 0; i < dim; i++) {
        double c = beta * eth[i * dim];
        const double *bi = basis + (size_t)i * n;
        for (size_t k = 0; k < n; k++) out[k] += c * bi[k];
    }
    free(basis); free(w); free(proj); free(h); free(th); free(eth);
    return dim;
}

/* Dense-matrix matvec, for the propagator golden (a 6x6 operator). */
typedef struct { const double *a; size_t n; } dense_ctx;
static void dense_mv(void *c, const double *x, double *ax) {
    dense_ctx *d = (dense_ctx *)c;
    for (size_t i = 0; i < d->n; i++) {
        double s = 0.0;
        for (size_t j = 0; j < d->n; j++) s += d->a[i * d->n + j] * x[j];
        ax[i] = s;
    }
}
int orc_expmv_dense(const double *a, size_t n, const double *v, double t, int m, double tol,
                    double *out) {
    dense_ctx c = {a, n};
    return orc_expmv_cb(dense_mv, &c, v, n, t, m, tol, out);
}

static void op_mv(void *c, const double *x, double *ax) { orc_apply((const orc_op *)c, x, ax); }

int orc_expmv(const orc_op *op, const double *v, double t, int m, double tol, double *out) {
    return orc_expmv_cb(op_mv, (void *)op, v, (size_t)orc_op_n_dof(op), t, m, tol, out);
}

/* Augmented operator [[A, b],[0, 0]].  propagator.rs:338-373. */
typedef struct { const orc_op *op; const double *b; size_t n; } aug_ctx;
static void aug_mv(void *c, const double *z, double *o) {
    aug_ctx *a = (aug_ctx *)c;
    orc_apply(a->op, z, o);
    double xi = z[a->n];
    for (size_t k = 0; k < a->n; k++) o[k] += xi * a->b[k];
    o[a->n] = 0.0;
}

int orc_etd_step(const orc_op *op, const double *y, const double *b, double h, int m, double tol,
                 double *out) {
    size_t n = (size_t)orc_op_n_dof(op);
    double *z = malloc(sizeof(double) * (n + 1)), *r = malloc(sizeof(double) * (n + 1));
    memcpy(z, y, sizeof(double) * n);
    z[n] = 1.0;
    aug_ctx c = {op, b, n};
    int dim = orc_expmv_cb(aug_mv, &c, z, n + 1, h, m, tol, r);
    memcpy(out, r, sizeof(double) * n);
    free(z); free(r);
    return dim;
}

/* ------------------------------------------------------------------------
 * Energy, spectral radius, port source / projections.
 * rhs.rs:1509-1544 (field_energy), session.rs:415-431 (normal_vector),
 * session.rs:514-569 (cfl_dt), rhs.rs:1157-1242 (port_source, projections).
 * --------------------------------------------------------------------- */

double orc_field_energy(const orc_op *op, const double *y) {
    int K = op->n_elem, np = op->re.np;
    double half = 0.0;
#pragma omp parallel for reduction(+ : half) num_threads(orc_get_threads())
    for (int e = 0; e < K; e++) {
        double scale = fabs(op->det[e]);
        double w6[6];
        for (int c = 0; c < 3; c++) {
            w6[c] = 1.0 / op->inv_eps[3 * e + c];
            w6[3 + c] = 1.0 / op->inv_mu[3 * e + c];
        }
        size_t base = (size_t)e * np * 6;
        double acc = 0.0;
        for (int ni = 0; ni < np; ni++)
            for (int nj = 0; nj < np; nj++) {
                double mij = scale * op->re.mass[ni * np + nj];
                if (mij == 0.0) continue;
                for (int c = 0; c < 6; c++)
                    acc += w6[c] * mij * y[base + ni * 6 + c] * y[base + nj * 6 + c];
            }
        half += acc;
    }
    return 0.5 * half;
}

void orc_normal_vector(size_t n, uint64_t seed, double *out) {
    uint64_t state = seed;
    for (size_t i = 0; i < n; i++) {
        double uv[2];
        for (int q = 0; q < 2; q++) {
            state += 0x9e3779b97f4a7c15ULL;
            uint64_t z = state;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            z ^= z >> 31;
            uv[q] = ((double)(z >> 11) + 0.5) / (double)(1ULL << 53);
        }
        out[i] = sqrt(-2.0 * log(uv[0])) * cos(2.0 * 3.14159265358979323846 * uv[1]);
    }
}

/* Spectral radius by `iters` power iterations from normal_vector(seed 0);
 * returns rho and leaves the final iterate in `v` (n).  session.rs:522-534. */
double orc_power_rho(const orc_op *op, int iters, double *v) {
    size_t n = (size_t)orc_op_n_dof(op);
    orc_normal_vector(n, 0, v);
    double s = 1.0 / norm2(v, n);
    for (size_t i = 0; i < n; i++) v[i] *= s;
    double *av = malloc(sizeof(double) * n);
    double rho = 1.0;
    for (int it = 0; it < iters; it++) {
        orc_apply(op, v, av);
        rho = norm2(av, n);
        for (size_t i = 0; i < n; i++) v[i] = av[i] / rho;
    }
    free(av);
    return rho;
}

/* The bracketed LSERK4 stability limit z* (before CFL_SAFETY) and rho.
 * session.rs:514-569 with constants.rs:233-258. */
double orc_cfl_z(const orc_op *op, double *rho_out) {
    size_t n = (size_t)orc_op_n_dof(op);
    double *probe = malloc(sizeof(double) * n), *y = malloc(sizeof(double) * n);
    double rho = orc_power_rho(op, 40, probe);
    double n0 = norm2(probe, n);
#define STABLE(z, res)                                                              \
    do {                                                                            \
        double h_ = (z) / rho;                                                      \
        memcpy(y, probe, sizeof(double) * n);                                       \
        orc_lserk_steps(op, y, h_, 64, 0, 0, NULL, NULL);                           \
        int fin_ = 1;                                                               \
        for (size_t i_ = 0; i_ < n; i_++) if (!isfinite(y[i_])) { fin_ = 0; break; } \
        if (!fin_) { res = 0; break; }                                              \
        double nf_ = norm2(y, n);                                                   \
        if (nf_ > 10.0 * n0) { res = 0; break; }                                    \
        double rate_ = nf_ > 0.0 ? pow(nf_ / n0, 1.0 / 64.0) : 0.0;                 \
        res = rate_ <= 1.0 + 1e-3;                                                  \
    } while (0)
    double lo = 3.0, hi = 15.0;
    int st;
    for (;;) { STABLE(lo, st); if (st || !(lo > 0.1)) break; lo *= 0.5; }
    for (;;) { STABLE(hi, st); if (!st || !(hi < 1e3)) break; hi *= 1.5; }
    for (int it = 0; it < 7; it++) {
        double mid = 0.5 * (lo + hi);
        STABLE(mid, st);
        if (st) lo = mid; else hi = mid;
    }
#undef STABLE
    free(probe); free(y);
    if (rho_out) *rho_out = rho;
    return lo;
}

/* Physical coordinates of every DG node, [e*np+node][3].  rhs.rs:1055-1066. */
void orc_node_coords(const orc_op *op, double *out) {
    int K = op->n_elem, np = op->re.np;
    for (int e = 0; e < K; e++)
        for (int i = 0; i < np; i++) map_point(op, e, op->re.nodes + 3 * i, out + 3 * ((size_t)e * np + i));
}

/* Incident-field source vector of a port, given the (e_t, h_t) profile at
 * every port face node (face order: (e,f) ascending, m inner; 6 doubles each).
 * rhs.rs:1157-1199. */
void orc_port_source(const orc_op *op, int port, const double *profiles, double *b) {
    int K = op->n_elem, np = op->re.np, nfp = op->re.nfp, cols = 4 * nfp;
    memset(b, 0, sizeof(double) * (size_t)orc_op_n_dof(op));
    size_t fi = 0;
    for (int e = 0; e < K; e++)
        for (int f = 0; f < 4; f++) {
            int ef = 4 * e + f;
            if (op->port[ef] != port) continue;
            const double *n = op->normal + 3 * ef;
            double coef = 0.5 * op->fscale[ef];
            const double *ie = op->inv_eps + 3 * e, *im = op->inv_mu + 3 * e;
            for (int m = 0; m < nfp; m++) {
                const double *et = profiles + 6 * (fi * nfp + m), *ht = et + 3;
                double nxe[3], nxh[3], nne[3], nnh[3];
                cross3(n, et, nxe); cross3(n, ht, nxh);
                cross3(n, nxe, nne); cross3(n, nxh, nnh);
                double s_de[3], s_dh[3];
                for (int c = 0; c < 3; c++) {
                    s_de[c] = nxh[c] - nne[c];
                    s_dh[c] = -nxe[c] - nnh[c];
                }
                for (int i = 0; i < np; i++) {
                    double w = coef * op->re.lift[i * cols + f * nfp + m];
                    size_t base = ((size_t)e * np + i) * 6;
                    for (int c = 0; c < 3; c++) {
                        b[base + c] += ie[c] * w * s_de[c];
                        b[base + 3 + c] += im[c] * w * s_dh[c];
                    }
                }
            }
            fi++;
        }
}

/* Modal projections (P_e, P_h) of state y on a port.  rhs.rs:1211-1242. */
void orc_port_projections(const orc_op *op, int port, const double *profiles, const double *y,
                          double *pe_ph) {
    int K = op->n_elem, np = op->re.np, nfp = op->re.nfp;
    double e_dot = 0, e_norm = 0, h_dot = 0, h_norm = 0;
    size_t fi = 0;
    for (int e = 0; e < K; e++)
        for (int f = 0; f < 4; f++) {
            int ef = 4 * e + f;
            if (op->port[ef] != port) continue;
            double area = op->fscale[ef] * fabs(op->det[e]) / 2.0;
            for (int m = 0; m < nfp; m++) {
                int vi = op->re.face_nodes[f * nfp + m];
                const double *et = profiles + 6 * (fi * nfp + m), *ht = et + 3;
                double w = 2.0 * area * op->re.face_w[f * nfp + m];
                size_t base = ((size_t)e * np + vi) * 6;
                e_dot += w * dot3(y + base, et);
                e_norm += w * dot3(et, et);
                h_dot += w * dot3(y + base + 3, ht);
                h_norm += w * dot3(ht, ht);
            }
            fi++;
        }
    pe_ph[0] = e_norm > 0.0 ? e_dot / e_norm : 0.0;
    pe_ph[1] = h_norm > 0.0 ? h_dot / h_norm : 0.0;
}
