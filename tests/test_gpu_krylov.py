"""The Krylov / ETD path on the device (f32 basis with f64 dot products, fused
CGS2 sweeps, the matvec on either stage engine; or the FP64 path) against
independent references:

  * the oracle's f64 Arnoldi (propagator.rs:186-326) for expmv and the
    held-source ETD step (propagator.rs:338-373);
  * the dense exponential of the (n + P)-augmented matrix [[A, W], [0, J]] of a
    small operator (A assembled column by column from the oracle's apply,
    scipy's expm) for the polynomial-source step;
  * the resident-state step (dgtd_etd_try / commit) against the host-API step.

Tolerances: 1e-4 relative L2 with the f32 basis (the Krylov parity bar), 1e-10
on the FP64 path against the oracle's Arnoldi over the same sub-steps.
"""
import numpy as np
import pytest
import scipy.linalg

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200._native import ENGINE_FP32, ENGINE_TF32X3

from .conftest import rel_l2

pytestmark = pytest.mark.gpu

KRY_TOL = 1e-4
KRY_TOL64 = 1e-10


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def _pair(mesh, order, face_port=None, materials=None):
    prod = O.MaxwellOperator(mesh, order, 1.0, face_port=face_port, materials=materials)
    orc = R.Operator(mesh.nodes, mesh.tets, order, 1.0, face_port=face_port, materials=materials)
    return prod, orc


def _lossy_box():
    m = O.structured_box_jittered(3, 3, 2, 1.0, 1.0, 0.7, 0.1, 4)
    cen = m.nodes[m.tets].mean(axis=1)
    slab = cen[:, 2] < 0.3
    mat = O.isotropic_materials(np.where(slab, 2.2, 1.0), sigma=np.where(slab, 5.0, 0.0))
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.7), 0, -1)
    return m, port, mat


@pytest.mark.parametrize("engine", [ENGINE_FP32, ENGINE_TF32X3], ids=["fp32", "tf32x3"])
def test_expmv_and_etd_step_match_oracle(ctx, engine):
    m, port, mat = _lossy_box()
    prod, orc = _pair(m, 3, port, mat)
    gop = G.GpuOperator(ctx, prod)
    gop.set_engine(engine)
    n = prod.n_dof
    rho, _ = orc.power_rho(30)
    v = np.sin(0.3 + 0.017 * np.arange(n))
    t = 6.0 / rho
    want, _ = orc.expmv(v, t, 36, 0.0)
    got, dim = gop.expmv(v, t, 36)
    assert dim == 36 and rel_l2(got, want) < KRY_TOL
    b = np.cos(0.05 * np.arange(n))
    want, _ = orc.etd_step(v, b, t, 24, 0.0)
    got, dim = gop.etd_step(v, b, t, 24)
    assert rel_l2(got, want) < KRY_TOL


def test_fp64_krylov_matches_oracle(ctx):
    m, port, mat = _lossy_box()
    prod, orc = _pair(m, 2, port, mat)
    gop = G.GpuOperator(ctx, prod)
    gop.set_krylov_precision(64)
    n = prod.n_dof
    rho, _ = orc.power_rho(30)
    v = np.sin(0.3 + 0.017 * np.arange(n))
    b = np.cos(0.05 * np.arange(n))
    t = 8.0 / rho
    # m = 40 runs as 4 sub-steps of dimension 10 over t/4 (KRYLOV_CHUNK,
    # gpu/operator.rs:1175-1197); the oracle's CPU Arnoldi does not sub-step,
    # so it is composed over the same sub-steps (exact for the held source)
    want = v
    for _ in range(4):
        want, _ = orc.expmv(want, t / 4, 10, 0.0)
    got, _ = gop.expmv(v, t, 40)
    assert rel_l2(got, want) < KRY_TOL64
    want = v
    for _ in range(4):
        want, _ = orc.etd_step(want, b, t / 4, 10, 0.0)
    got, _ = gop.etd_step(v, b, t, 40)
    assert rel_l2(got, want) < KRY_TOL64


def _dense_a(orc):
    n = orc.n_dof
    a = np.zeros((n, n))
    e = np.zeros(n)
    for j in range(n):
        e[j] = 1.0
        a[:, j] = orc.apply(e)
        e[j] = 0.0
    return a


def _poly_reference(a, y, b, coef, h):
    """First n components of expm(h [[A, W], [0, J]]) [y; e_{P-1}], W's column q
    = coef[P-1-q] (P-1-q)! b (the exact solution of y' = A y + b g(t) with g the
    polynomial)."""
    n, P = a.shape[0], len(coef)
    big = np.zeros((n + P, n + P))
    big[:n, :n] = a
    fact = 1.0
    for k in range(P):
        if k:
            fact *= k
        big[:n, n + P - 1 - k] = coef[k] * fact * b
    for q in range(P - 1):
        big[n + q, n + q + 1] = 1.0
    z = np.concatenate([y, np.zeros(P)])
    z[n + P - 1] = 1.0
    return (scipy.linalg.expm(h * big) @ z)[:n]


@pytest.mark.parametrize("precision", [32, 64])
def test_etd_poly_matches_dense_augmented_exponential(ctx, precision):
    m = O.structured_box(1, 1, 2)
    mat = O.isotropic_materials(np.array([1.0, 2.0] * 6), sigma=np.array([0.0, 3.0] * 6))
    prod, orc = _pair(m, 2, materials=mat)
    gop = G.GpuOperator(ctx, prod)
    gop.set_krylov_precision(precision)
    a = _dense_a(orc)
    n = prod.n_dof
    rng = np.random.default_rng(1)
    y = rng.normal(size=n)
    b = np.zeros(n)
    b[prod.nearest_node_dof([0.5, 0.5, 1.0], 0, 2)] = 1.0
    rho = np.max(np.abs(np.linalg.eigvals(a)))
    h = 3.0 / rho
    tol = KRY_TOL if precision == 32 else KRY_TOL64
    for coef in ([1.0], [0.3, -2.0], [0.1, 1.5, -40.0, 200.0], [0.5, -3.0, 25.0, -60.0, 900.0, -2e3, 1e4, -3e4]):
        want = _poly_reference(a, y, b, coef, h)
        got, dim, _ = gop.etd_step_poly(y, b, coef, h, 36, 0.0)
        assert rel_l2(got, want) < tol, (coef, rel_l2(got, want))
    # P = 1 with coef 1 is the reference's held-source step
    got1, _ = gop.etd_step(y, b, h, 36)
    want1, _ = orc.etd_step(y, b, h, 36, 0.0)
    assert rel_l2(got1, want1) < tol


@pytest.mark.parametrize("engine", [ENGINE_FP32, ENGINE_TF32X3], ids=["fp32", "tf32x3"])
def test_resident_etd_step_matches_host_api(ctx, engine):
    m, port, mat = _lossy_box()
    prod, orc = _pair(m, 3, port, mat)
    gop = G.GpuOperator(ctx, prod)
    gop.set_engine(engine)
    n = prod.n_dof
    rho, _ = orc.power_rho(30)
    dof = prod.nearest_node_dof([0.5, 0.5, 0.35], 0, 2)
    b = np.zeros(n)
    b[dof] = 1.0
    y0 = (0.1 * np.sin(0.3 + 0.017 * np.arange(n))).astype(np.float32)
    coef = [0.2, 3.0, -10.0]
    gop.upload(y0)
    # a step too long for its space is rejected (est > tol) after its first
    # sub-step; halve it until one passes
    h = 12.0 / rho
    d1, e1 = gop.etd_try(h, 30, 1e-6, coef=coef, drive=("point", dof))
    tries = 1
    while e1 > 1e-6:
        assert d1 <= 10 and tries < 8  # a rejected step stopped after one sub-step of <= 10
        h *= 0.5
        d1, e1 = gop.etd_try(h, 30, 1e-6, coef=coef, drive=("point", dof))
        tries += 1
    assert tries > 1  # the first try was rejected
    d2, e2 = gop.etd_try(h, 30, 1e-6, coef=coef, drive=("point", dof))  # a retry replaces the candidate
    assert (d1, e1) == (d2, e2) and 0 <= e1 <= 1e-6
    gop.etd_commit()
    got = gop.download()
    want, dw, ew = gop.etd_step_poly(y0.astype(np.float64), b, coef, h, 30, 1e-6)
    assert rel_l2(got, want) < 1e-5
    # and against the exact solution by the f64 oracle's fine LSERK4 with the polynomial source
    sub = 400
    dt = h / sub
    tt = (np.arange(sub) + 0.5) * dt
    g = coef[0] + coef[1] * tt + coef[2] * tt ** 2
    ref = orc.lserk(y0.astype(np.float64), dt, sub, src_dof=dof, vals=g)
    assert rel_l2(got, ref) < 1e-3  # the held-per-substep source is first order in dt
