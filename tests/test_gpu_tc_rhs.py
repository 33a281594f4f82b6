"""The tensor-core (tcgen05, 3xTF32) RHS engine against the oracle and against
the FP32 CUDA-core engine, through the C ABI.  Same tolerances as the FP32
parity tests: one RHS < 1e-5, LSERK4 transients < 1e-4 (relative L2)."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import _native
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O

from .conftest import rel_l2

pytestmark = pytest.mark.gpu
TF32X3 = _native.ENGINE_TF32X3


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def _ops(ctx, mesh, order, alpha=1.0, face_port=None, materials=None):
    prod = O.MaxwellOperator(mesh, order, alpha, face_port=face_port, materials=materials)
    orc = R.Operator(mesh.nodes, mesh.tets, order, alpha, face_port=face_port, materials=materials)
    gop = G.GpuOperator(ctx, prod)
    gop.set_engine(TF32X3)
    return prod, orc, gop


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("cells", [(3, 3, 4), (3, 3, 3)], ids=["whole_tiles", "ragged"])
def test_tc_apply_matches_oracle(ctx, order, cells):
    """216 tets fill whole tiles at order 5 (8 elements) but not at orders 1-4
    (20); 162 tets fill neither."""
    prod, orc, gop = _ops(ctx, O.structured_box(*cells), order)
    y32 = np.sin(0.3 + 0.017 * np.arange(gop.n_dof())).astype(np.float32)
    assert rel_l2(gop.apply(y32), orc.apply(y32.astype(np.float64))) < 1e-5


def test_tc_apply_jittered_sphere_ports_lossy(ctx):
    m = O.structured_box_jittered(6, 5, 7, 1.0, 0.9, 1.2, 0.1, 11)
    cen = m.nodes[m.tets].mean(axis=1)
    K = m.n_tets
    eps = np.where(np.linalg.norm(cen - [0.5, 0.45, 0.6], axis=1) < 0.25, 4.0, 1.0)
    rng = np.random.default_rng(5)
    mat = O.isotropic_materials(eps, rng.uniform(1, 2, K), rng.uniform(0, 2, K), rng.uniform(0, 1, K))
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    port[O.boundary_faces_on_plane(m, 2, 1.2)] = 1
    for order in (3, 4, 5):
        for alpha in (1.0, 0.0):
            prod, orc, gop = _ops(ctx, m, order, alpha, face_port=port, materials=mat)
            y32 = np.sin(0.1 + 0.0123 * np.arange(gop.n_dof())).astype(np.float32)
            assert rel_l2(gop.apply(y32), orc.apply(y32.astype(np.float64))) < 1e-5


def test_tc_matches_fp32_engine(ctx):
    m = O.structured_box_jittered(7, 7, 7, 1.0, 1.0, 1.0, 0.1, 3)
    prod = O.MaxwellOperator(m, 4, 1.0)
    a = G.GpuOperator(ctx, prod)
    a.set_engine(_native.ENGINE_FP32)
    b = G.GpuOperator(ctx, prod)
    b.set_engine(TF32X3)
    x = prod.node_coords()
    y = np.zeros((x.shape[0], 6), dtype=np.float32)
    y[:, 2] = np.exp(-((x - [0.3, 0.4, 0.5]) ** 2).sum(1) / (2 * 0.1 ** 2))
    y = y.ravel()
    assert rel_l2(b.apply(y), a.apply(y)) < 1e-5


def test_tc_transient_matches_oracle(ctx):
    prod, orc, gop = _ops(ctx, O.structured_box(3, 3, 3), 3)
    y0 = np.sin(0.2 + 0.011 * np.arange(gop.n_dof()))
    rho, _ = orc.power_rho(30)
    dt = 1.0 / rho
    got = gop.transient(y0, dt, 150, 1)
    want = orc.lserk(y0.astype(np.float32).astype(np.float64), dt, 150)
    assert rel_l2(got, want) < 1e-4


def test_tc_driven_transient_matches_oracle(ctx):
    m = O.structured_box(4, 3, 3)
    prod, orc, gop = _ops(ctx, m, 4)
    n = gop.n_dof()
    dof = prod.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    rho, _ = orc.power_rho(20)
    dt = 1.0 / rho
    steps = 60
    t = np.arange(steps) * dt
    g = np.exp(-((t - 20 * dt) / (6 * dt)) ** 2)
    got = gop.transient(np.zeros(n), dt, steps, 1, drive=("point", dof), g=g)
    want = orc.lserk(np.zeros(n), dt, steps, src_dof=dof, vals=g.astype(np.float32).astype(np.float64))
    assert rel_l2(got, want) < 1e-4


def test_tc_order5_matches_fp32_engine(ctx):
    m = O.structured_box_jittered(4, 4, 4, 1.0, 1.0, 1.0, 0.1, 3)
    prod = O.MaxwellOperator(m, 5, 1.0)
    a = G.GpuOperator(ctx, prod)
    a.set_engine(_native.ENGINE_FP32)
    b = G.GpuOperator(ctx, prod)
    b.set_engine(TF32X3)
    x = prod.node_coords()
    y = np.zeros((x.shape[0], 6), dtype=np.float32)
    y[:, 1] = np.exp(-((x - [0.4, 0.5, 0.5]) ** 2).sum(1) / (2 * 0.12 ** 2))
    y = y.ravel()
    assert rel_l2(b.apply(y), a.apply(y)) < 1e-5


def test_tc_order5_transients_match_oracle(ctx):
    """LSERK4 free and point-driven, on a mesh whose 162 tets are not whole
    8-element tiles."""
    m = O.structured_box_jittered(3, 3, 3, 1.0, 1.0, 1.0, 0.1, 8)
    prod, orc, gop = _ops(ctx, m, 5)
    n = gop.n_dof()
    rho, _ = orc.power_rho(30)
    dt = 1.0 / rho
    y0 = np.sin(0.2 + 0.011 * np.arange(n))
    got = gop.transient(y0, dt, 100, 1)
    want = orc.lserk(y0.astype(np.float32).astype(np.float64), dt, 100)
    assert rel_l2(got, want) < 1e-4
    dof = prod.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    steps = 60
    t = np.arange(steps) * dt
    g = np.exp(-((t - 20 * dt) / (6 * dt)) ** 2)
    got = gop.transient(np.zeros(n), dt, steps, 1, drive=("point", dof), g=g)
    want = orc.lserk(np.zeros(n), dt, steps, src_dof=dof, vals=g.astype(np.float32).astype(np.float64))
    assert rel_l2(got, want) < 1e-4


def test_tc_order5_krylov_and_kcl_match_oracle(ctx):
    """The Krylov-matvec and KCL-stage modes of the order-5 kernel."""
    m = O.structured_box_jittered(3, 3, 2, 1.0, 1.0, 0.7, 0.1, 4)
    cen = m.nodes[m.tets].mean(axis=1)
    slab = cen[:, 2] < 0.3
    mat = O.isotropic_materials(np.where(slab, 2.2, 1.0), sigma=np.where(slab, 5.0, 0.0))
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.7), 0, -1)
    prod, orc, gop = _ops(ctx, m, 5, face_port=port, materials=mat)
    n = gop.n_dof()
    rho, _ = orc.power_rho(30)
    v = np.sin(0.3 + 0.017 * np.arange(n))
    t = 6.0 / rho
    want, _ = orc.expmv(v, t, 36, 0.0)
    got, _ = gop.expmv(v, t, 36)
    assert rel_l2(got, want) < 1e-4
    h = 1.0 / rho
    y_gpu, _ = gop.kcl_step(v, h)
    y_ref, _ = orc.kcl_step(v.astype(np.float32).astype(np.float64), h)
    assert rel_l2(y_gpu, y_ref) < 1e-5
