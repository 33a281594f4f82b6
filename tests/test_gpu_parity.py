"""GPU parity: the CUDA path through the C ABI against the f64 oracle.

Tolerances (relative L2), from the DGTD parity targets and the reference's
own budget (constants.rs:43-50, GPU_REL_TOL = 1e-3):
  * one RHS evaluation:         < 1e-5 against the oracle on the same f32 input
  * LSERK4 transients:          < 1e-4 at the final frame
  * Krylov expmv / ETD (f64 basis, f32 matvec): < 1e-4
Fixtures follow gpu/operator.rs:1515-1950: structured boxes, y_i =
sin(0.3 + 0.017 i), dt = 1/rho(A).
"""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200._native import DgtdError

from .conftest import rel_l2

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-5
RUN_TOL = 1e-4
KRY_TOL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def _pair(mesh, order, alpha=1.0, face_port=None, materials=None):
    prod = O.MaxwellOperator(mesh, order, alpha, face_port=face_port, materials=materials)
    orc = R.Operator(mesh.nodes, mesh.tets, order, alpha, face_port=face_port, materials=materials)
    return prod, orc


def _y(n, a=0.3, b=0.017):
    return np.sin(a + b * np.arange(n))


def _rho(orc, iters=30):
    rho, _ = orc.power_rho(iters)
    return rho


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_apply_matches_oracle_vacuum(ctx, order):
    prod, orc = _pair(O.structured_box(3, 3, 3), order)
    gop = G.GpuOperator(ctx, prod)
    y32 = _y(gop.n_dof()).astype(np.float32)
    got = gop.apply(y32)
    want = orc.apply(y32.astype(np.float64))
    assert rel_l2(got, want) < RHS_TOL


def test_apply_matches_oracle_dielectric_lossy_central(ctx):
    m = O.structured_box(3, 3, 3)
    K = m.n_tets
    rng = np.random.default_rng(0)
    mat = O.isotropic_materials(np.full(K, 4.0), rng.uniform(1, 2, K), rng.uniform(0, 3, K), rng.uniform(0, 1, K))
    for alpha in (1.0, 0.0):
        prod, orc = _pair(m, 2, alpha, materials=mat)
        gop = G.GpuOperator(ctx, prod)
        y32 = _y(gop.n_dof()).astype(np.float32)
        assert rel_l2(gop.apply(y32), orc.apply(y32.astype(np.float64))) < RHS_TOL


def test_apply_matches_oracle_jittered_sphere_ports(ctx):
    m = O.structured_box_jittered(5, 5, 6, 1.0, 1.0, 1.2, 0.1, 7)
    cen = m.nodes[m.tets].mean(axis=1)
    eps = np.where(np.linalg.norm(cen - [0.5, 0.5, 0.6], axis=1) < 0.25, 4.0, 1.0)
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    port[O.boundary_faces_on_plane(m, 2, 1.2)] = 1
    for order in (3, 4):
        prod, orc = _pair(m, order, 1.0, face_port=port, materials=O.isotropic_materials(eps))
        gop = G.GpuOperator(ctx, prod)
        y32 = _y(gop.n_dof(), 0.1, 0.0123).astype(np.float32)
        assert rel_l2(gop.apply(y32), orc.apply(y32.astype(np.float64))) < RHS_TOL


def test_apply_on_smooth_field_matches_f64_input(ctx):
    # Same initial data in f64 (not pre-rounded): the f32 path within 1e-5.
    m = O.structured_box(4, 4, 4)
    prod, orc = _pair(m, 3)
    gop = G.GpuOperator(ctx, prod)
    x = prod.node_coords()
    y = np.zeros((x.shape[0], 6))
    y[:, 2] = np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1])
    y[:, 3] = 0.3 * np.cos(np.pi * x[:, 2])
    y = y.ravel()
    assert rel_l2(gop.apply(y), orc.apply(y)) < RHS_TOL


def test_transient_matches_oracle(ctx):
    prod, orc = _pair(O.structured_box(3, 3, 3), 2)
    gop = G.GpuOperator(ctx, prod)
    n = gop.n_dof()
    y0 = _y(n, 0.2, 0.011)
    dt = 1.0 / _rho(orc)
    steps = 200
    got = gop.transient(y0, dt, steps, 1)
    want = orc.lserk(y0.astype(np.float32).astype(np.float64), dt, steps)
    assert rel_l2(got, want) < RUN_TOL


def test_transient_record_and_substeps(ctx):
    prod, orc = _pair(O.structured_box(2, 2, 2), 3)
    gop = G.GpuOperator(ctx, prod)
    y0 = _y(gop.n_dof())
    dt = 2.0 / _rho(orc)
    traj = gop.transient(y0, dt, 4, substeps=2, record=True)
    assert traj.shape == (5, gop.n_dof())
    assert np.array_equal(traj[0], y0.astype(np.float32))
    want = y0.astype(np.float32).astype(np.float64)
    for k in range(4):
        want = orc.lserk(want, dt / 2, 2)
        assert rel_l2(traj[k + 1], want) < RUN_TOL


def test_driven_point_transient_matches_oracle(ctx):
    prod, orc = _pair(O.structured_box(3, 3, 3), 2)
    gop = G.GpuOperator(ctx, prod)
    n = gop.n_dof()
    dof = prod.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    dt = 1.0 / _rho(orc)
    steps = 150
    t = np.arange(steps) * dt
    g = np.exp(-((t - 40 * dt) / (12 * dt)) ** 2)
    got = gop.transient(np.zeros(n), dt, steps, 1, drive=("point", dof), g=g)
    want = orc.lserk(np.zeros(n), dt, steps, src_dof=dof, vals=g.astype(np.float32).astype(np.float64))
    assert rel_l2(got, want) < RUN_TOL


def test_driven_vector_transient_matches_oracle(ctx):
    m = O.structured_box(2, 2, 4, 1.0, 0.5, 2.0)
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    port[O.boundary_faces_on_plane(m, 2, 2.0)] = 1
    prod, orc = _pair(m, 2, 1.0, face_port=port)
    prof = prod.rect_port_profiles(0, [0, 0, 1.0], (1, 0))
    b = prod.port_source(0, prof)
    gop = G.GpuOperator(ctx, prod)
    dt = 1.0 / _rho(orc)
    steps = 120
    t = np.arange(steps) * dt
    g = np.exp(-((t - 30 * dt) / (10 * dt)) ** 2) * np.cos(2 * np.pi * 1.5 * t)
    got = gop.transient(np.zeros(gop.n_dof()), dt, steps, 1, drive=("vector", b), g=g)
    want = orc.lserk(np.zeros(gop.n_dof()), dt, steps, src_vec=b.astype(np.float32).astype(np.float64),
                     vals=g.astype(np.float32).astype(np.float64))
    assert rel_l2(got, want) < RUN_TOL


def test_transient_probes(ctx):
    prod, orc = _pair(O.structured_box(2, 2, 2), 2)
    gop = G.GpuOperator(ctx, prod)
    y0 = _y(gop.n_dof())
    dt = 1.0 / _rho(orc)
    probes = [0, 5, gop.n_dof() - 1]
    series, yf = gop.transient_probes(y0, dt, 10, 1, probes=probes)
    traj = gop.transient(y0, dt, 10, 1, record=True)
    assert np.array_equal(series, traj[:, probes])
    assert np.array_equal(yf, traj[-1])
    # a caller-owned output array receives the same final state
    out = np.full(gop.n_dof(), np.nan, dtype=np.float32)
    series2, yf2 = gop.transient_probes(y0, dt, 10, 1, probes=probes, y_final=out)
    assert yf2 is out and np.array_equal(out, yf) and np.array_equal(series2, series)
    with pytest.raises(ValueError):
        gop.transient_probes(y0, dt, 1, 1, probes=probes, y_final=np.empty(3, dtype=np.float32))


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_state_layout_round_trip(ctx, order):
    # AoS -> device SoA -> AoS is the identity, including a final chunk of
    # fewer elements than the conversion kernel stages at once (162 = 8*20 + 2).
    prod = O.MaxwellOperator(O.structured_box(3, 3, 3), order, 1.0)
    gop = G.GpuOperator(ctx, prod)
    y = _y(gop.n_dof()).astype(np.float32)
    gop.upload(y)
    assert np.array_equal(gop.download(), y)


def test_expmv_matches_oracle(ctx):
    # gpu/operator.rs:1839: m = 40, t = 0.02 against the CPU propagator.
    prod, orc = _pair(O.structured_box(3, 3, 3), 2)
    gop = G.GpuOperator(ctx, prod)
    v = _y(gop.n_dof())
    want, _ = orc.expmv(v, 0.02, 40, 0.0)
    got, dim = gop.expmv(v, 0.02, 40)
    assert rel_l2(got, want) < KRY_TOL
    assert dim == 40
    got_a, dim_a = gop.expmv(v, 0.02, 40, tol=1e-10)
    assert rel_l2(got_a, want) < KRY_TOL
    assert dim_a <= 40


def test_etd_step_matches_oracle(ctx):
    prod, orc = _pair(O.structured_box(3, 3, 3), 2)
    gop = G.GpuOperator(ctx, prod)
    n = gop.n_dof()
    y = _y(n, 0.1, 0.007)
    b = np.zeros(n)
    b[prod.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)] = 0.7
    h = 0.05
    want, _ = orc.etd_step(y, b, h, 40, 0.0)
    got, dim = gop.etd_step(y, b, h, 24)
    assert rel_l2(got, want) < KRY_TOL


def test_device_expm_matches_oracle(ctx):
    rng = np.random.default_rng(1)
    for d in (1, 5, 23, 64):
        a = rng.normal(size=(d, d)) * (3.0 / np.sqrt(d))
        assert rel_l2(ctx.expm(a), R.expm(a)) < 1e-12


def test_bad_arguments_raise(ctx):
    prod, _ = _pair(O.structured_box(1, 1, 1), 2)
    gop = G.GpuOperator(ctx, prod)
    with pytest.raises(ValueError):
        gop.apply(np.zeros(3))
    with pytest.raises(DgtdError):
        gop.transient(np.zeros(gop.n_dof()), 0.01, 2, 1, drive=("point", gop.n_dof() + 5), g=np.ones(2))
    with pytest.raises(DgtdError):
        gop.transient(np.zeros(gop.n_dof()), -1.0, 2)
    assert gop.launch_count() >= 0


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_single_cell_mesh_one_padded_tile(ctx, order, engine):
    # 6 tets: fewer elements than one tile of either kernel, so most of the tile
    # is inert padding; every face of the cube is a PEC boundary face
    prod, orc = _pair(O.structured_box(1, 1, 1), order)
    gop = G.GpuOperator(ctx, prod)
    gop.set_engine(engine)
    y32 = _y(gop.n_dof()).astype(np.float32)
    assert rel_l2(gop.apply(y32), orc.apply(y32.astype(np.float64))) < RHS_TOL
    dt = 0.5 / _rho(orc)
    got = gop.transient(y32, dt, 5)
    want = orc.lserk(y32.astype(np.float64), dt, 5)
    assert rel_l2(got, want) < RUN_TOL


@pytest.mark.parametrize("engine", [0, 1])
def test_zero_steps_and_empty_probe_list(ctx, engine):
    prod, orc = _pair(O.structured_box(2, 2, 2), 3)
    gop = G.GpuOperator(ctx, prod)
    gop.set_engine(engine)
    y32 = _y(gop.n_dof()).astype(np.float32)
    dt = 0.5 / _rho(orc)
    # no steps: the final state is the initial one, the record is one frame
    assert np.array_equal(gop.transient(y32, dt, 0), y32)
    traj = gop.transient(y32, dt, 0, record=True)
    assert traj.shape == (1, gop.n_dof()) and np.array_equal(traj[0], y32)
    # no probes: an empty series and the same final state as a plain transient
    series, yf = gop.transient_probes(y32, dt, 4, 1, probes=())
    assert series.shape == (5, 0)
    assert np.array_equal(yf, gop.transient(y32, dt, 4))


@pytest.mark.parametrize("engine", [0, 1])
def test_zero_state_has_zero_rhs(ctx, engine):
    prod, _ = _pair(O.structured_box(3, 3, 3), 4)
    gop = G.GpuOperator(ctx, prod)
    gop.set_engine(engine)
    assert not np.any(gop.apply(np.zeros(gop.n_dof(), dtype=np.float32)))


@pytest.mark.parametrize("engine", [0, 1])
def test_rhs_linearity_at_size(ctx, engine):
    # a property that needs no oracle, at a size the oracle would be slow on:
    # A(a x + b z) = a A x + b A z to f32 rounding (16^3 x 6 tets, 5.2 M DOFs)
    from rapidfem_b200 import workloads as W

    wl = W.sphere_pulse(16, 4)
    gop = G.GpuOperator(ctx, wl.build())
    gop.set_engine(engine)
    n = gop.n_dof()
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n).astype(np.float32)
    z = rng.standard_normal(n).astype(np.float32)
    a, b = np.float32(0.75), np.float32(-1.25)
    lhs = gop.apply((a * x + b * z).astype(np.float32)).astype(np.float64)
    rhs = a * gop.apply(x).astype(np.float64) + b * gop.apply(z).astype(np.float64)
    assert rel_l2(lhs, rhs) < 1e-5


def test_cfl_dt_matches_oracle(ctx):
    # session.rs:514-569: 40 power iterations from the same seeded start vector,
    # then a bisection of the LSERK4 stability point z; h = 0.8 z / rho
    import ctypes as C

    from rapidfem_b200 import _native as nat

    prod, orc = _pair(O.structured_box(3, 3, 3), 3)
    gop = G.GpuOperator(ctx, prod)
    h, rho, z = C.c_double(), C.c_double(), C.c_double()
    nat.check(nat.lib.dgtd_cfl_dt(gop.handle, C.byref(h), C.byref(rho), C.byref(z)))
    z_ref, rho_ref = orc.cfl_z()
    assert abs(rho.value - rho_ref) < 1e-4 * rho_ref
    assert abs(z.value - z_ref) < 0.25  # within two steps of the bisection's final bracket
    assert abs(h.value - 0.8 * z.value / rho.value) < 1e-12 * h.value + 1e-15


def test_field_energy_matches_oracle(ctx):
    import ctypes as C

    from rapidfem_b200 import _native as nat

    m = O.structured_box_jittered(3, 3, 3, 1.0, 1.0, 1.0, 0.1, 5)
    K = m.n_tets
    rng = np.random.default_rng(2)
    mat = O.isotropic_materials(rng.uniform(1, 4, K), rng.uniform(1, 2, K))
    prod, orc = _pair(m, 3, materials=mat)
    gop = G.GpuOperator(ctx, prod)
    y = _y(gop.n_dof())
    e = C.c_double()
    nat.check(nat.lib.dgtd_field_energy(gop.handle, np.ascontiguousarray(y, dtype=np.float64), C.byref(e)))
    want = orc.field_energy(y)
    assert abs(e.value - want) < 1e-6 * abs(want)
