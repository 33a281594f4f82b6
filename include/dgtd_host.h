/*
 * dgtd_host.h -- C ABI of the native host side of the DGTD path
 * (librapidfem_b200.so): structured meshes and the operator build that
 * feeds dgtd_op_desc.
 *
 * These replace the Rust host pieces the reference's GPU operator consumes:
 *   crates/rapidfem-td/src/mesh_gen.rs        (structured Kuhn boxes)
 *   crates/rapidfem-td/src/dg_basis.rs        (ReferenceElement::new)
 *   crates/rapidfem-td/src/geom_factors.rs    (all_geometric_factors)
 *   crates/rapidfem-core/src/topology.rs      (FaceTopology::build)
 *   crates/rapidfem-td/src/rhs.rs:805-1000    (MaxwellOperator::new)
 *   crates/rapidfem-td/src/rhs.rs:546-770     (periodic face pairs)
 *   crates/rapidfem-td/src/rhs.rs:1157-1242   (port_source, port projections)
 *   crates/rapidfem-td/src/waveguide.rs:90-152 (RectPort TE_mn profiles)
 * All arithmetic here is f64, as in the reference.
 */
#ifndef DGTD_HOST_H
#define DGTD_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "dgtd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dgtd_host_op dgtd_host_op;

/* structured_box (mesh_gen.rs:54-76): nodes[(nx+1)(ny+1)(nz+1)*3],
 * tets[6*nx*ny*nz*4], vertex ids of each tet sorted ascending. */
int dgtd_mesh_box(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                  double *nodes, int32_t *tets);
/* structured_box_jittered (mesh_gen.rs:86-139): interior node components
 * displaced by amplitude*h*U[-1,1] from the reference's hash of (i,j,k,seed). */
int dgtd_mesh_box_jittered(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                           double amplitude, uint64_t seed, double *nodes, int32_t *tets);
/* A box graded geometrically along z: z_k spacing ratio `ratio` = h_last/h_first
 * (so ratio 20 grades 20:1 with the fine end at z = 0).  No reference
 * counterpart; same Kuhn split as structured_box. */
int dgtd_mesh_box_graded_z(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                           double ratio, double *nodes, int32_t *tets);

/* MaxwellOperator::new (rhs.rs:805-1000) on a tet mesh.
 * face_port: 4K ints or NULL: a port index (>= 0), -1 none, or -2 for a face
 * of an internal PEC plate (OperatorOptions::pec_plates: the face is severed
 * from its neighbour and gets the PEC ghost state, rhs.rs:862-880; both sides
 * of the plate carry the code); materials: K*8 doubles (eps_xyz, mu_xyz,
 * sigma, sigma_m) or NULL for vacuum. */
int dgtd_host_op_build(const double *nodes, int64_t n_nodes, const int32_t *tets, int64_t n_elem,
                       int32_t order, double flux_alpha, const int32_t *face_port,
                       const double *materials, dgtd_host_op **out);
/* A periodic face pair (PeriodicSpec, rhs.rs:253-270; link_periodic_faces,
 * rhs.rs:616-770): the domain-boundary faces faces_a[n_a] and faces_b[n_b]
 * (face ids e*4 + local face) are wired to one another as interior faces
 * across the translation between the two sides' area-weighted centroids.
 * Each side-A face takes the side-B face whose centroid is nearest its own
 * translated centroid (within max(1e-9 |T|, 1e-12)), the pairing must be a
 * bijection, and the face-node permutations are nearest-node matches in the
 * translated frame (both directions).  Port faces and faces that already have
 * a neighbour are rejected; on any error the operator is left unchanged.
 * Call once per pair, after dgtd_host_op_build and before dgtd_host_op_desc. */
int dgtd_host_op_link_periodic(dgtd_host_op *op, const int64_t *faces_a, int64_t n_a,
                               const int64_t *faces_b, int64_t n_b);
/* Releases the host operator (MaxwellOperator is dropped in the reference). */
int dgtd_host_op_destroy(dgtd_host_op *op);
/* Fill a dgtd_op_desc whose pointers stay valid while `op` lives: the arrays
 * GpuOperator::new flattens (gpu/operator.rs:222-292). */
int dgtd_host_op_desc(const dgtd_host_op *op, dgtd_op_desc *desc);
/* Np, Nfp, K and n_dof of the operator (no counterpart in the reference). */
int dgtd_host_op_info(const dgtd_host_op *op, int32_t *np, int32_t *nfp, int64_t *n_elem,
                      int64_t *n_dof);
/* Copy a named array out as doubles (no counterpart in the reference; a test
 * and inspection aid): nodes, mass, dr, ds, dt, lift, face_nodes,
 * face_w, jinv, jac, origin, det, normal, fscale, nbr, nbr_lf, port, perm,
 * inv_eps, inv_mu, sigma_eps, sigma_mu. */
int dgtd_host_op_get(const dgtd_host_op *op, const char *name, double *out);
/* Physical coordinates of all DG nodes, [K*Np*3] (rhs.rs:1055-1066). */
int dgtd_host_node_coords(const dgtd_host_op *op, double *out);
/* nearest_node_dof (rhs.rs:1030-1051): field 0=E 1=H, comp 0..2. */
int dgtd_host_nearest_node_dof(const dgtd_host_op *op, const double *point, int32_t field,
                               int32_t comp, int64_t *dof);
/* Number of (e,f) faces on port `port`, in (e,f) ascending order (the face
 * set port_source and port_modal_projections walk, rhs.rs:1157-1242). */
int dgtd_host_port_n_faces(const dgtd_host_op *op, int32_t port, int64_t *n_faces);
/* RectPort TE_mn (waveguide.rs:124-145) profiles at every node of port
 * `port`'s faces: out[n_faces*Nfp*6] = (e_t xyz, h_t xyz).  The frame is
 * FaceFrame::fit (waveguide.rs:39-81) of the port nodes with `inward_normal`. */
int dgtd_host_rect_port_profiles(const dgtd_host_op *op, int32_t port, const double *inward_normal,
                                 int32_t mode_m, int32_t mode_n, double *out);
/* The modal projections P_e (which = 0) or P_h (which = 1) of a port as linear
 * functionals of the AoS state (rhs.rs:1211-1242, port_modal_projections):
 * P = sum_k w[k] * y[idx[k]], with n_faces*nfp*3 terms written to idx / w.
 * profiles as for dgtd_host_port_source. */
int dgtd_host_port_modal_weights(const dgtd_host_op *op, int32_t port, const double *profiles,
                                 int32_t which, int64_t *idx, double *w);
/* port_source (rhs.rs:1157-1199) from per-node profiles: b[n_dof]. */
int dgtd_host_port_source(const dgtd_host_op *op, int32_t port, const double *profiles,
                          double *b);

#ifdef __cplusplus
}
#endif

#endif /* DGTD_HOST_H */
