"""The reference's operator physics tests (rhs.rs:1995-2030, :2366-2520; see
tests/test_physics.py for the oracle runs) on the device path: the operator
assembled by TdSession.state_space (FP64 device RHS), the propagation by the
device Krylov expmv."""
import numpy as np
import pytest

from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200 import td as TD

from .test_physics import _port_column, energy_mass, least_damped_re

pytestmark = pytest.mark.gpu


def _dense(sess):
    n, row_ptr, col_idx, vals = sess.state_space()
    a = np.zeros((n, n))
    a[np.repeat(np.arange(n), np.diff(row_ptr)), col_idx] = vals
    return a


def test_conductivity_damps_at_the_analytic_rate_device():
    mesh = O.structured_box(1, 1, 1)
    res = []
    for sigma in (0.0, 0.2):
        mat = O.isotropic_materials(np.ones(mesh.n_tets), sigma=np.full(mesh.n_tets, sigma))
        sess = TD.TdSession(O.MaxwellOperator(mesh, 2, 1.0, materials=mat))
        res.append(least_damped_re(_dense(sess)))
    delta, want = res[1] - res[0], -0.2 / 2.0
    assert abs(delta - want) / abs(want) < 0.1


def test_port_operator_only_dissipates_device():
    mesh, port = _port_column(2, 2.0, 1.0, True)
    op = O.MaxwellOperator(mesh, 2, 0.0, face_port=port)
    a = _dense(TD.TdSession(op))
    ma = energy_mass(op) @ a  # the host operator carries the same arrays as the oracle
    ev = np.linalg.eigvalsh(ma + ma.T)
    scale = np.max(np.abs(ma))
    assert ev.max() < 1e-7 * scale and ev.min() < -1e-3 * scale


def test_port_face_drains_field_energy_device():
    ctx = G.GpuContext(0)
    kept = {}
    for with_port in (False, True):
        mesh, port = _port_column(10, 5.0, 0.5, with_port)
        op = O.MaxwellOperator(mesh, 2, 0.0, face_port=port)
        sess = TD.TdSession(op)
        gop = G.GpuOperator(ctx, op)
        xyz = op.node_coords()
        y = np.zeros(op.n_dof)
        y[0::6] = np.exp(-((xyz[:, 2] - 2.5) / 0.5) ** 2)
        e0 = sess.field_energy(y)
        for _ in range(900):
            y, _ = gop.expmv(y, 0.06, 24)
        kept[with_port] = sess.field_energy(y) / e0
    assert kept[False] > 0.95 and kept[True] < 0.5


def test_port_injects_a_mode_at_the_group_velocity_device():
    from .test_physics import group_velocity_check, guide

    _, _, op, _, _ = guide()
    gop = G.GpuOperator(G.GpuContext(0), op)
    group_velocity_check(lambda y, b, h, m: gop.etd_step(y, b, h, m)[0], op)


def test_port_extracts_the_incident_amplitude_device():
    from .test_physics import guide, incident_amplitude_check

    _, _, op, _, funcs = guide()
    gop = G.GpuOperator(G.GpuContext(0), op)
    incident_amplitude_check(lambda y, b, h, m: gop.etd_step(y, b, h, m)[0], funcs)


def test_cavity_fundamental_on_an_irregular_mesh_device():
    from .test_physics import WANT_FUNDAMENTAL, fundamental

    mesh = O.structured_box_jittered(2, 2, 2, 1.0, 1.0, 1.0, 0.25, 7)
    re, im = fundamental(_dense(TD.TdSession(O.MaxwellOperator(mesh, 2, 1.0))))
    assert re < 0.0 and abs(im - WANT_FUNDAMENTAL) / WANT_FUNDAMENTAL < 0.08


def test_cavity_fundamental_converges_device():
    from .test_physics import WANT_FUNDAMENTAL, fundamental

    err = []
    for cells in (1, 2):
        sess = TD.TdSession(O.MaxwellOperator(O.structured_box(cells, cells, cells), 2, 1.0))
        err.append(abs(fundamental(_dense(sess))[1] - WANT_FUNDAMENTAL) / WANT_FUNDAMENTAL)
    assert err[1] < err[0] and err[1] < 1e-3


def test_anisotropic_central_flux_conserves_energy_device():
    from .test_physics import anisotropic_box, skew_defect

    mesh, mat = anisotropic_box()
    op = O.MaxwellOperator(mesh, 2, 0.0, materials=mat)
    assert skew_defect(_dense(TD.TdSession(op)), energy_mass(op)) < 1e-12
