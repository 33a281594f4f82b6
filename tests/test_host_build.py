"""The native host build (include/dgtd_host.h) against the oracle, on the CPU.

The product's MaxwellOperator (rhs.rs:805-1000 restated in C++) must produce
the same f64 arrays as the oracle's restatement, bit for bit, on regular,
jittered and graded meshes, with ports and materials.
"""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import operator as O
from rapidfem_b200._native import DgtdError

ARRAYS = ["mass", "dr", "ds", "dt", "lift", "face_nodes", "face_w", "jinv", "jac", "origin", "det",
          "normal", "fscale", "nbr", "nbr_lf", "port", "perm", "inv_eps", "inv_mu", "sigma_eps",
          "sigma_mu"]


def _same(prod, orc):
    for k in ARRAYS:
        a, b = prod.get(k), orc.get(k)
        assert np.array_equal(a, b), k


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_box_operator_matches_oracle(order):
    m = O.structured_box(2, 2, 3, 1.0, 1.0, 1.5)
    nodes, tets = R.box_mesh(2, 2, 3, 1.0, 1.0, 1.5)
    assert np.array_equal(m.nodes, nodes) and np.array_equal(m.tets, tets)
    _same(O.MaxwellOperator(m, order, 1.0), R.Operator(nodes, tets, order, 1.0))


def test_jittered_box_with_ports_and_materials_matches_oracle():
    m = O.structured_box_jittered(4, 3, 3, 1.0, 0.8, 0.9, 0.1, 42)
    nodes, tets = R.box_mesh_jittered(4, 3, 3, 1.0, 0.8, 0.9, 0.1, 42)
    assert np.array_equal(m.nodes, nodes)
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    port[O.boundary_faces_on_plane(m, 2, 0.9)] = 1
    K = m.n_tets
    rng = np.random.default_rng(3)
    mat = O.isotropic_materials(rng.uniform(1, 4, K), rng.uniform(1, 2, K), rng.uniform(0, 1, K))
    _same(O.MaxwellOperator(m, 3, 1.0, face_port=port, materials=mat),
          R.Operator(nodes, tets, 3, 1.0, face_port=port, materials=mat))


def test_graded_box_spacing():
    m = O.structured_box_graded_z(2, 2, 24, 1.0, 1.0, 1.0, 20.0)
    z = np.unique(np.round(m.nodes[:, 2], 14))
    h = np.diff(z)
    assert z[0] == 0.0 and abs(z[-1] - 1.0) < 1e-15
    assert abs(h[-1] / h[0] - 20.0) < 1e-9
    op = O.MaxwellOperator(m, 3)
    assert np.all(np.isfinite(op.get("jinv")))


def test_box_counts_and_volume():
    m = O.structured_box(3, 2, 2)
    assert m.n_tets == 3 * 2 * 2 * 6
    v = m.nodes[m.tets]
    vol = np.abs(np.einsum("ij,ij->i", v[:, 1] - v[:, 0], np.cross(v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]))).sum() / 6
    assert abs(vol - 1.0) < 1e-12


def test_interior_faces_are_paired_and_boundary_is_pec():
    op = O.MaxwellOperator(O.structured_box(2, 2, 2), 2)
    nbr = op.get("nbr").astype(int).reshape(-1, 4)
    lf = op.get("nbr_lf").astype(int).reshape(-1, 4)
    for e in range(nbr.shape[0]):
        for f in range(4):
            if nbr[e, f] >= 0:
                assert nbr[nbr[e, f], lf[e, f]] == e
    n_boundary = (nbr < 0).sum()
    assert n_boundary == 6 * 2 * 2 * 2  # 2 triangles per boundary cell face


def test_bad_order_is_rejected():
    with pytest.raises(DgtdError):
        O.MaxwellOperator(O.structured_box(1, 1, 1), 6)


def test_degenerate_tet_is_rejected():
    m = O.Mesh(np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 0, 1.0]]), np.array([[0, 1, 2, 3]], dtype=np.int32))
    with pytest.raises(DgtdError):
        O.MaxwellOperator(m, 2)


def test_nearest_node_dof_and_coords():
    op = O.MaxwellOperator(O.structured_box(2, 2, 2), 2)
    xyz = op.node_coords()
    dof = op.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    node = dof // 6
    assert np.allclose(xyz[node], [0.5, 0.5, 0.5])
    assert dof % 6 == 2


def test_port_source_matches_oracle():
    m = O.structured_box(3, 2, 4, 2.0, 1.0, 3.0)
    nodes, tets = R.box_mesh(3, 2, 4, 2.0, 1.0, 3.0)
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    prod = O.MaxwellOperator(m, 2, face_port=port)
    orc = R.Operator(nodes, tets, 2, face_port=port)
    prof = prod.rect_port_profiles(0, [0, 0, 1.0], (1, 0))
    assert prof.shape == (prod.port_n_faces(0) * prod.nfp, 6)
    # TE10 on a 2x1 cross-section: E along the narrow axis, sin(pi x / 2)
    assert np.max(np.abs(prof[:, 0])) < 1e-12 and np.max(np.abs(prof[:, 1])) > 0.9
    b = prod.port_source(0, prof)
    assert np.array_equal(b, orc.port_source(0, prof))
    assert np.linalg.norm(b) > 0


def test_port_modal_weights_match_oracle_projections():
    """P_e, P_h as sparse functionals equal port_modal_projections (rhs.rs:1211-1242)."""
    nodes, tets = R.box_mesh_jittered(3, 2, 4, 1.0, 0.6, 1.2, 0.1, 11)
    m = O.Mesh(nodes, tets)
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    port[O.boundary_faces_on_plane(m, 2, 1.2)] = 1
    prod = O.MaxwellOperator(m, 3, face_port=port)
    orc = R.Operator(nodes, tets, 3, face_port=port)
    rng = np.random.default_rng(5)
    y = rng.normal(size=prod.n_dof)
    for p in (0, 1):
        prof = prod.rect_port_profiles(p, [0, 0, 1.0 if p == 0 else -1.0], (1, 0))
        ie, we = prod.port_modal_weights(p, prof, "E")
        ih, wh = prod.port_modal_weights(p, prof, "H")
        assert ie.size == prod.port_n_faces(p) * prod.nfp * 3
        assert np.all(ie % 6 < 3) and np.all(ih % 6 >= 3)
        pe, ph = orc.port_projections(p, prof, y)
        assert abs(y[ie] @ we - pe) <= 1e-12 * max(1.0, abs(pe))
        assert abs(y[ih] @ wh - ph) <= 1e-12 * max(1.0, abs(ph))
    with pytest.raises(ValueError):
        prod.port_modal_weights(0, prof, "X")
