"""The FP64 path (rhs_fp64_kernel: f64 operators, element records and state on
the CUDA cores) against the f64 oracle: one RHS to 1e-12 relative L2 on every
order and boundary kind, LSERK4 transients free and driven to 1e-11, and the
plain-DGTD FP64 cavity configuration (8^3 x 6 PEC cube, N = 3, TM110, CFL 0.5,
1000 steps) against the oracle and the analytic mode.  Bounds: both sides are
f64 with different summation orders, so they agree to ~1e-14 per RHS; the
transient bound leaves room for the rounding to grow with the step count."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200 import workloads as W

from .conftest import rel_l2

pytestmark = pytest.mark.gpu

RHS_TOL64 = 1e-12
RUN_TOL64 = 1e-11


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def _pair(mesh, order, alpha=1.0, face_port=None, materials=None):
    prod = O.MaxwellOperator(mesh, order, alpha, face_port=face_port, materials=materials)
    orc = R.Operator(mesh.nodes, mesh.tets, order, alpha, face_port=face_port, materials=materials)
    return prod, orc


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_apply_f64_matches_oracle(ctx, order):
    m = O.structured_box_jittered(4, 3, 5, 1.0, 0.8, 1.1, 0.1, 5)
    cen = m.nodes[m.tets].mean(axis=1)
    rng = np.random.default_rng(order)
    K = m.n_tets
    mat = O.isotropic_materials(np.where(cen[:, 0] > 0.5, 4.0, 1.0), rng.uniform(1, 2, K), rng.uniform(0, 3, K),
                                rng.uniform(0, 1, K))
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    for alpha in (1.0, 0.0):
        prod, orc = _pair(m, order, alpha, face_port=port, materials=mat)
        gop = G.GpuOperator(ctx, prod)
        y = np.sin(0.3 + 0.017 * np.arange(gop.n_dof()))
        assert rel_l2(gop.apply_f64(y), orc.apply(y)) < RHS_TOL64


def test_transient_f64_free_and_driven(ctx):
    m = O.structured_box(3, 3, 3)
    prod, orc = _pair(m, 3)
    gop = G.GpuOperator(ctx, prod)
    n = gop.n_dof()
    y0 = np.sin(0.2 + 0.011 * np.arange(n))
    dt = 1.0 / orc.power_rho(30)[0]
    steps = 200
    assert rel_l2(gop.transient_f64(y0, dt, steps), orc.lserk(y0, dt, steps)) < RUN_TOL64
    # point source, waveform held per substep
    dof = prod.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    sub = 2
    g = np.exp(-((np.arange(steps * sub) - 60.0) / 20.0) ** 2)
    got = gop.transient_f64(np.zeros(n), dt, steps, sub, drive=("point", dof), g=g, record=True)
    want = np.zeros(n)
    for k in range(steps):
        want = orc.lserk(want, dt / sub, sub, src_dof=dof, vals=g[k * sub:(k + 1) * sub])
        if k in (0, steps // 2):
            assert rel_l2(got[k + 1], want) < RUN_TOL64
    assert rel_l2(got[-1], want) < RUN_TOL64
    # vector source
    b = np.cos(0.05 * np.arange(n))
    got = gop.transient_f64(np.zeros(n), dt, 40, 1, drive=("vector", b), g=g[:40])
    want = orc.lserk(np.zeros(n), dt, 40, src_vec=b, vals=g[:40])
    assert rel_l2(got, want) < RUN_TOL64


def test_c1_fp64_cavity_1000_steps(ctx):
    """Plain DGTD in FP64: TM110 of the 8^3 x 6 PEC cube, N = 3, vacuum, upwind,
    LSERK4 at dt = 0.5 * 2.8 / rho for 1000 steps."""
    wl = W.cavity_tm110(8, 3)
    op = wl.build()
    nodes, tets = R.box_mesh(8, 8, 8, 1.0, 1.0, 1.0)
    orc = R.Operator(nodes, tets, 3, 1.0)
    rho, _ = orc.power_rho(40)
    dt = 0.5 * 2.8 / rho
    steps = 1000
    y0 = wl.y0(op)
    want = orc.lserk(y0, dt, steps)
    gop = G.GpuOperator(ctx, op)
    got = gop.transient_f64(y0, dt, steps)
    assert rel_l2(got, want) < RUN_TOL64
    exact = W.tm110_exact(op, steps * dt)
    assert rel_l2(got, exact) < 1e-2  # the N = 3, h = 1/8 discretisation error of the mode
