"""The reference's propagator tests (propagator.rs:488-625) on the device
Krylov path with the f64 basis (dgtd_op_set_krylov_precision(op, 64)): a
central-flux run conserves the field energy, the adaptive expmv meets its
tolerance against the dense exponential, and a tighter tolerance takes at
least as many Krylov dimensions."""
import numpy as np
import pytest
from scipy.linalg import expm

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O

from .test_physics import dense

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def _unit_cube(ctx, alpha):
    mesh = O.structured_box(1, 1, 1)
    op = O.MaxwellOperator(mesh, 2, alpha)
    gop = G.GpuOperator(ctx, op)
    gop.set_krylov_precision(64)
    return mesh, op, gop


def test_central_flux_propagation_conserves_energy(ctx):
    """propagator.rs:561-589: 30 expmv steps of 0.02 (m = 40), drift < 1e-7."""
    mesh, op, gop = _unit_cube(ctx, 0.0)
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 0.0)
    y = np.sin(0.2 + 0.013 * np.arange(op.n_dof))
    e0 = orc.field_energy(y)
    for _ in range(30):
        y, _ = gop.expmv(y, 0.02, 40)
    assert abs(orc.field_energy(y) - e0) / e0 < 1e-7


def test_adaptive_krylov_dimension_meets_tolerance(ctx):
    """propagator.rs:488-534, :591-625: expmv at tol 1e-9 within 1e-7 of
    the dense exponential with fewer dimensions than the state; a tighter
    tolerance takes at least as many."""
    mesh, op, gop = _unit_cube(ctx, 1.0)
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 1.0)
    n, t = op.n_dof, 0.05
    v = np.sin(0.3 + 0.017 * np.arange(n))
    want = expm(t * dense(orc.apply, n)) @ v
    got, dim = gop.expmv(v, t, 200, 1e-9)
    assert np.linalg.norm(got - want) < 1e-7 * np.linalg.norm(want)
    assert 0 < dim < n
    _, dim_tight = gop.expmv(v, t, 200, 1e-13)
    assert dim_tight >= dim
