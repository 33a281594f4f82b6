"""The oracle pinned against the reference's own golden vectors and analytic
tests (CPU only).

Golden fixtures in tests/golden/ come from crates/rapidfem-td/tests/*.rs
(see tests/golden/make_golden.py).  The analytic checks restate
rhs.rs:1830-1868 (central flux skew), rhs.rs:2113-2148 (cavity pi*sqrt 2),
dg_basis.rs:524-557 (LIFT integrates face traces) and
tests/lserk4_convergence_test.rs (fourth order).
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as R

from .conftest import rel_l2

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF_TET = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
ONE_TET = np.array([[0, 1, 2, 3]], dtype=np.int32)


def _max_rel_err(got, want):
    want = np.asarray(want)
    return np.max(np.abs(np.asarray(got) - want)) / max(np.max(np.abs(want)), 1e-300)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_dg_basis_matches_golden(p):
    tab = json.load(open(os.path.join(GOLD, "dg_basis.json")))["tables"]
    op = R.Operator(REF_TET, ONE_TET, p)
    for arr, key in (("mass", "MASS"), ("dr", "DR"), ("ds", "DS"), ("dt", "DT")):
        assert _max_rel_err(op.get(arr), tab[f"{key}_P{p}"]) < 1e-9, (arr, p)


def test_curl_matches_golden():
    g = json.load(open(os.path.join(GOLD, "rhs_curl.json")))
    tet = np.array(g["tet"]).reshape(4, 3)
    op = R.Operator(tet, ONE_TET, g["order"])
    got = R.curl_single(g["order"], op.get("jinv"), g["field"])
    assert _max_rel_err(got, g["curl"]) < 1e-9


def test_expmv_matches_golden():
    g = json.load(open(os.path.join(GOLD, "propagator_expm.json")))
    a = np.array(g["a"]).reshape(g["n"], g["n"])
    for h, ref in g["cases"]:
        got, dim = R.expmv_dense(a, g["v0"], h, 12, 0.0)
        assert rel_l2(got, ref) < 1e-10
        assert dim <= 6  # lucky breakdown inside the 6-dim space


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_lift_integrates_face_traces(p):
    op = R.Operator(REF_TET, ONE_TET, p)
    np_, nfp = op.np, op.nfp
    lift = op.get("lift").reshape(np_, 4 * nfp)
    mass = op.get("mass").reshape(np_, np_)
    for f in range(4):
        tr = np.zeros(4 * nfp)
        tr[f * nfp:(f + 1) * nfp] = 1.0
        assert abs(np.sum(mass @ (lift @ tr)) - 0.5) < 1e-9


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_diff_rows_sum_to_zero(p):
    op = R.Operator(REF_TET, ONE_TET, p)
    for k in ("dr", "ds", "dt"):
        d = op.get(k).reshape(op.np, op.np)
        assert np.max(np.abs(d.sum(axis=1))) < 1e-8


def _dense(op):
    n = op.n_dof
    a = np.zeros((n, n))
    e = np.zeros(n)
    for j in range(n):
        e[j] = 1.0
        a[:, j] = op.apply(e)
        e[j] = 0.0
    return a


def _energy_mass(op):
    np_ = op.np
    mass = op.get("mass").reshape(np_, np_)
    det = np.abs(op.get("det"))
    ie = op.get("inv_eps").reshape(-1, 3)
    im = op.get("inv_mu").reshape(-1, 3)
    n = op.n_dof
    m = np.zeros((n, n))
    for e in range(op.n_elem):
        w = np.concatenate([1 / ie[e], 1 / im[e]])
        for c in range(6):
            idx = (e * np_ + np.arange(np_)) * 6 + c
            m[np.ix_(idx, idx)] = w[c] * det[e] * mass
    return m


def test_central_flux_is_skew_in_energy_norm():
    nodes, tets = R.box_mesh(1, 1, 1)
    op = R.Operator(nodes, tets, 2, flux_alpha=0.0)
    ma = _energy_mass(op) @ _dense(op)
    assert np.max(np.abs(ma + ma.T)) < 1e-9 * max(np.max(np.abs(ma)), 1.0)


def test_cavity_fundamental_is_pi_sqrt2():
    nodes, tets = R.box_mesh(2, 2, 2)
    op = R.Operator(nodes, tets, 2, flux_alpha=1.0)
    ev = np.linalg.eigvals(_dense(op))
    phys = ev[np.abs(ev.imag) > 1.0]
    fund = phys[np.argmax(phys.real)]
    want = np.pi * np.sqrt(2.0)
    assert fund.real < 0.0
    assert abs(abs(fund.imag) - want) / want < 0.05


def test_lserk4_is_fourth_order_on_the_dg_operator():
    nodes, tets = R.box_mesh(1, 1, 1)
    op = R.Operator(nodes, tets, 2, flux_alpha=1.0)
    a = _dense(op)
    y0 = np.sin(0.3 + 0.017 * np.arange(op.n_dof))
    t = 0.4
    w, v = np.linalg.eig(a * t)
    exact = np.real(v @ (np.exp(w) * np.linalg.solve(v, y0)))
    errs = []
    for steps in (40, 80, 160):
        errs.append(rel_l2(op.lserk(y0, t / steps, steps), exact))
    orders = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(orders > 3.5), orders


def test_krylov_matches_lserk_on_the_dg_operator():
    # explicit.rs:173-208: one LSERK4 step of 1e-3 vs expmv (m = 40), < 1e-9.
    nodes, tets = R.box_mesh(2, 2, 2)
    op = R.Operator(nodes, tets, 2, flux_alpha=1.0)
    y0 = np.sin(0.3 + 0.017 * np.arange(op.n_dof))
    h = 1e-3
    ref = op.lserk(y0, h, 1)
    got, dim = op.expmv(y0, h, 40, 0.0)
    assert rel_l2(got, ref) < 1e-9
    got_adaptive, dim = op.expmv(y0, h, 40, 1e-10)
    assert rel_l2(got_adaptive, ref) < 1e-9
    assert dim < 40


def test_kcl_matches_the_exponential_propagator_below_cfl():
    # explicit_adaptive.rs:219-255: one KCL RK4(3)5 step of 1e-3 vs expmv, < 1e-9.
    nodes, tets = R.box_mesh(2, 2, 2)
    op = R.Operator(nodes, tets, 2, flux_alpha=1.0)
    y0 = np.sin(0.3 + 0.017 * np.arange(op.n_dof))
    got, _ = op.kcl_step(y0, 1e-3)
    want, _ = op.expmv(y0, 1e-3, 40, 0.0)
    assert rel_l2(got, want) < 1e-9


def test_kcl_and_lserk4_driven_match_etd_below_cfl():
    # explicit.rs:265-313, explicit_adaptive.rs:257-300: one driven step of 1e-3
    # (a point source of 0.7, a spread vector source) vs the ETD step, < 1e-9.
    nodes, tets = R.box_mesh(2, 2, 2)
    op = R.Operator(nodes, tets, 2, flux_alpha=1.0)
    n = op.n_dof
    y0 = np.sin(0.2 + 0.019 * np.arange(n))
    sdof = n // 3
    point = np.zeros(n)
    point[sdof] = 0.7
    spread = 0.4 * np.cos(0.11 * np.arange(n))
    for b, kw in ((point, dict(src_dof=sdof)), (spread, dict(src_vec=spread))):
        g = 0.7 if "src_dof" in kw else 1.0
        want, _ = op.etd_step(y0, b, 1e-3, 40)
        kcl, _ = op.kcl_step(y0, 1e-3, g=g, **kw)
        assert rel_l2(kcl, want) < 1e-9
        rk = op.lserk(y0, 1e-3, 1, vals=np.array([g]), **kw)
        assert rel_l2(rk, want) < 1e-9


def test_etd_step_matches_augmented_dense():
    nodes, tets = R.box_mesh(1, 1, 1)
    op = R.Operator(nodes, tets, 2, flux_alpha=1.0)
    n = op.n_dof
    a = _dense(op)
    y = np.cos(0.1 + 0.013 * np.arange(n))
    b = np.zeros(n)
    b[7] = 1.0
    h = 0.05
    aug = np.zeros((n + 1, n + 1))
    aug[:n, :n] = a
    aug[:n, n] = b
    ref = R.expm(aug * h)[:n] @ np.concatenate([y, [1.0]])
    got, _ = op.etd_step(y, b, h, 40, 0.0)
    assert rel_l2(got, ref) < 1e-9


def test_expm_identities():
    z = R.expm(np.zeros((3, 3)))
    assert np.allclose(z, np.eye(3))
    a = np.array([[0.0, 1.0], [-1.0, 0.0]]) * 3.0
    e = R.expm(a)
    assert np.allclose(e, [[np.cos(3), np.sin(3)], [-np.sin(3), np.cos(3)]], atol=1e-13)


def test_lserk4_is_fourth_order_on_a_linear_ode():
    """explicit.rs:143-170: the oracle's LSERK4 coefficient table (the one the
    product's stage-time table in sources.py matches exactly) integrates the
    rotation dy/dt = [[0, -w], [w, 0]] y, w = 1.3, to T = 1.7 at fourth order:
    halving the step from T/20 to T/40 cuts the error more than 12-fold."""
    from rapidfem_b200 import sources as S

    a, b = R.lserk_coeffs()
    assert np.array_equal(a, S.LSERK_A) and np.array_equal(b, S.LSERK_B)
    w, t_end = 1.3, 1.7
    amat = np.array([[0.0, -w], [w, 0.0]])

    def err(nsteps):
        dt = t_end / nsteps
        y, p = np.array([1.0, 0.4]), np.zeros(2)
        for _ in range(nsteps):
            for s in range(5):
                p = a[s] * p + dt * (amat @ y)
                y = y + b[s] * p
        c, sn = np.cos(w * t_end), np.sin(w * t_end)
        return float(np.linalg.norm(y - [c - 0.4 * sn, sn + 0.4 * c]))

    assert err(20) / err(40) > 12.0


def test_etd_step_matches_analytic_linear_ode():
    """propagator.rs:536-559: dy/dt = A y + b with A the rotation (w = 1.3),
    b = (0.4, -0.7), y0 = (1, 0.5), h = 0.6: the augmented exponential
    exp(h [[A, b], [0, 0]]) [y0; 1] (the oracle's dense Krylov, m = 8 >= 3,
    exact) gives exp(hA)(y0 + A^-1 b) - A^-1 b to 1e-12."""
    w, h = 1.3, 0.6
    amat = np.array([[0.0, -w], [w, 0.0]])
    b, y0 = np.array([0.4, -0.7]), np.array([1.0, 0.5])
    aug = np.zeros((3, 3))
    aug[:2, :2], aug[:2, 2] = amat, b
    got, _ = R.expmv_dense(aug, np.array([y0[0], y0[1], 1.0]), h, 8, 0.0)
    ainv_b = np.array([b[1] / w, -b[0] / w])
    c, s = np.cos(w * h), np.sin(w * h)
    sh = y0 + ainv_b
    want = np.array([c * sh[0] - s * sh[1], s * sh[0] + c * sh[1]]) - ainv_b
    assert np.max(np.abs(got[:2] - want)) < 1e-12 and abs(got[2] - 1.0) < 1e-12


def test_kcl_orders_on_the_dg_operator():
    """explicit_adaptive.rs:160-217 (fourth order; the embedded error third
    order), restated on the DG operator (2^3 box, N = 2, upwind) with the
    exact step exp(hA) y from the oracle's Krylov: halving h = 0.1 / rho cuts
    the one-step error of the KCL RK4(3)5 step by about 2^5 (> 24) and the
    embedded error estimate by about 2^4 (> 12, the reference's bound 10)."""
    nodes, tets = R.box_mesh(2, 2, 2)
    orc = R.Operator(nodes, tets, 2, 1.0)
    rho, _ = orc.power_rho(40)
    y = np.sin(0.3 + 0.017 * np.arange(orc.n_dof))
    step_err, est = [], []
    for h in (0.1 / rho, 0.05 / rho):
        yk, e = orc.kcl_step(y, h)
        exact, _ = orc.expmv(y, h, 40, 0.0)
        step_err.append(np.linalg.norm(yk - exact))
        est.append(np.linalg.norm(e))
    assert step_err[0] / step_err[1] > 24.0
    assert est[0] / est[1] > 12.0
