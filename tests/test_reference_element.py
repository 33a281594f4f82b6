"""The reference's reference-element and geometric-factor unit tests
(dg_basis.rs:396-495, geom_factors.rs tests) on the CPU, for both host
builds: the oracle's restatement and the product's C++ host build
(rapidfem_b200.operator.MaxwellOperator), at orders 1-5 where the reference
checks 1-4 (order 5 is on the path here).  The element matrices are those of
the unit tet (0,0,0), (1,0,0), (0,1,0), (0,0,1): on it the physical operator
arrays are the reference ones."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import operator as O

REF_TET = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
ONE_TET = np.array([[0, 1, 2, 3]], dtype=np.int32)
SHEARED = np.array([[1.0, 2.0, -1.0], [3.0, 2.5, -1.0], [1.5, 5.0, 0.5], [2.0, 2.0, 4.0]])


def _ops(nodes, order, tets=ONE_TET):
    """The oracle's and the product's host operator on one tet."""
    return (R.Operator(nodes, tets, order),
            O.MaxwellOperator(O.Mesh(np.ascontiguousarray(nodes), np.ascontiguousarray(tets)), order, 1.0))


def _np(p):
    return (p + 1) * (p + 2) * (p + 3) // 6


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_node_counts_mass_and_inverse(p):
    """node_counts, mass_is_partition_of_unity (sum M = 1/6, the unit tet's
    volume), mass_is_symmetric, mass_inverse_is_correct (dg_basis.rs:396-450).
    The reference checks orders 1-4 with symmetry to 1e-13; at order 5 the
    monomial Vandermonde of the equispaced nodes is worse conditioned
    (dg_basis.rs:496-521 tracks it) and the same construction is symmetric to
    1.6e-13, so order 5 is held to 1e-12."""
    for op in _ops(REF_TET, p):
        n = _np(p)
        assert op.node_coords().shape == (n, 3)
        m = op.get("mass").reshape(n, n)
        assert abs(m.sum() - 1.0 / 6.0) < 1e-11
        assert np.max(np.abs(m - m.T)) < (1e-13 if p <= 4 else 1e-12)
        assert np.max(np.abs(m @ np.linalg.inv(m) - np.eye(n))) < 1e-9


def _poly(p):
    """A polynomial of degree p in (r, s, t) and its gradient: the reference's
    degree-3 case (dg_basis.rs:468-476) plus terms up to degree p."""
    def u(r, s, t):
        v = 1.0 + 2.0 * r + 3.0 * s - t
        if p >= 2:
            v = v + r * s
        if p >= 3:
            v = v + r * t * t + s ** 3
        if p >= 4:
            v = v + r * r * s * t
        if p >= 5:
            v = v + t ** 5 - r * s ** 4
        return v

    def grad(r, s, t):
        dr = 2.0 + (s if p >= 2 else 0.0) + (t * t if p >= 3 else 0.0)
        ds = 3.0 + (r if p >= 2 else 0.0) + (3.0 * s * s if p >= 3 else 0.0)
        dt = -1.0 + (2.0 * r * t if p >= 3 else 0.0)
        if p >= 4:
            dr, ds, dt = dr + 2.0 * r * s * t, ds + r * r * t, dt + r * r * s
        if p >= 5:
            dr, ds, dt = dr - s ** 4, ds - 4.0 * r * s ** 3, dt + 5.0 * t ** 4
        return dr, ds, dt

    return u, grad


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_diff_is_exact_on_polynomials(p):
    """diff_is_exact_on_polynomials (dg_basis.rs:464-495): Dr, Ds, Dt
    differentiate a degree-p polynomial exactly at the nodes."""
    u, grad = _poly(p)
    n = _np(p)
    for op in _ops(REF_TET, p):
        x = op.node_coords()
        un = u(x[:, 0], x[:, 1], x[:, 2])
        want = grad(x[:, 0], x[:, 1], x[:, 2])
        for k, name in enumerate(("dr", "ds", "dt")):
            d = op.get(name).reshape(n, n)
            assert np.max(np.abs(d @ un - want[k])) < 1e-8 * max(1.0, np.max(np.abs(want[k])))


def test_reference_tet_is_identity():
    """geom_factors.rs reference_tet_is_identity."""
    for op in _ops(REF_TET, 1):
        assert abs(op.get("det")[0] - 1.0) < 1e-14
        assert np.max(np.abs(op.get("jac") - np.eye(3).ravel())) < 1e-14
        assert np.max(np.abs(op.get("jinv") - np.eye(3).ravel())) < 1e-14


def test_jacobian_inverse_and_determinant():
    """inverse_jacobian_is_consistent, det_matches_triple_product (J's columns
    are v1 - v0, v2 - v0, v3 - v0; det J is six times the volume) and
    det_flips_with_orientation (geom_factors.rs tests)."""
    a, b, c = SHEARED[1] - SHEARED[0], SHEARED[2] - SHEARED[0], SHEARED[3] - SHEARED[0]
    for op in _ops(SHEARED, 2):
        jac, jinv = op.get("jac").reshape(3, 3), op.get("jinv").reshape(3, 3)
        assert np.array_equal(jac, np.column_stack([a, b, c]))
        assert np.max(np.abs(jac @ jinv - np.eye(3))) < 1e-12
        det = op.get("det")[0]
        assert det > 0.0 and abs(det - a @ np.cross(b, c)) < 1e-12
    swapped = np.array([[0, 2, 1, 3]], dtype=np.int32)
    for op in _ops(REF_TET, 1, swapped):
        assert abs(op.get("det")[0] + 1.0) < 1e-14


def test_physical_derivatives_are_exact():
    """physical_derivatives_are_exact (geom_factors.rs): the reference
    operators and the metric give d/dx, d/dy, d/dz of u = x y + 2 x + z^2
    exactly at the nodes of a sheared order-2 element,
    (D_x u)_i = sum_k Jinv[k][axis] (D_k u)_i."""
    v = np.array([[1.0, 0.0, 0.0], [2.0, 0.0, 0.0], [1.0, 1.0, 0.0], [1.0, 0.0, 3.0]])
    n = _np(2)
    for op in _ops(v, 2):
        x = op.node_coords()
        un = x[:, 0] * x[:, 1] + 2.0 * x[:, 0] + x[:, 2] ** 2
        exact = (x[:, 1] + 2.0, x[:, 0], 2.0 * x[:, 2])
        jinv = op.get("jinv").reshape(3, 3)
        ref = [op.get(k).reshape(n, n) @ un for k in ("dr", "ds", "dt")]
        for axis in range(3):
            got = sum(jinv[k, axis] * ref[k] for k in range(3))
            assert np.max(np.abs(got - exact[axis])) < 1e-9
