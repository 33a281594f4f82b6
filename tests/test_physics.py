"""The reference's operator physics tests (rhs.rs:1995-2030 conductivity
damping, :2366-2445 a port face drains energy, :2447-2520 the port operator
only dissipates) on the f64 oracle; tests/test_gpu_physics.py runs them on
the device path."""
import numpy as np

from oracle import oracle as R
from rapidfem_b200 import operator as O


def dense(apply, n):
    """A column by column from a matrix-free apply (assemble_dense, rhs.rs:1477)."""
    a = np.zeros((n, n))
    e = np.zeros(n)
    for j in range(n):
        e[j] = 1.0
        a[:, j] = apply(e)
        e[j] = 0.0
    return a


def energy_mass(orc):
    """The block-diagonal energy mass M~ of the AoS state (rhs.rs:1550):
    |det J_e| M_ref weighted by eps_c / mu_c (field_energy = y' M~ y / 2)."""
    K, np_ = orc.n_elem, orc.np
    det = np.abs(orc.get("det"))
    mref = orc.get("mass").reshape(np_, np_)
    w = np.concatenate([1.0 / orc.get("inv_eps").reshape(K, 3), 1.0 / orc.get("inv_mu").reshape(K, 3)], axis=1)
    m = np.zeros((orc.n_dof, orc.n_dof))
    for e in range(K):
        for c in range(6):
            idx = (e * np_ + np.arange(np_)) * 6 + c
            m[np.ix_(idx, idx)] = det[e] * w[e, c] * mref
    return m


def least_damped_re(a):
    ev = np.linalg.eigvals(a)
    return float(np.max(ev.real[np.abs(ev.imag) > 1.0]))


def test_conductivity_damps_at_the_analytic_rate():
    """rhs.rs:1995-2030: sigma = 0.2 shifts the least-damped physical mode's
    real part by -sigma / (2 eps) within 10 % (unit box, N = 2, upwind)."""
    mesh = O.structured_box(1, 1, 1)
    res = []
    for sigma in (0.0, 0.2):
        mat = O.isotropic_materials(np.ones(mesh.n_tets), sigma=np.full(mesh.n_tets, sigma))
        orc = R.Operator(mesh.nodes, mesh.tets, 2, 1.0, materials=mat)
        res.append(least_damped_re(dense(orc.apply, orc.n_dof)))
    delta, want = res[1] - res[0], -0.2 / 2.0
    assert abs(delta - want) / abs(want) < 0.1


def _port_column(nz, lz, lxy, with_port):
    mesh = O.structured_box(1, 1, nz, lxy, lxy, lz)
    port = np.where(O.boundary_faces_on_plane(mesh, 2, lz), 0, -1) if with_port else None
    return mesh, port


def test_port_operator_only_dissipates():
    """rhs.rs:2447-2520: with a characteristic port face (central flux) the
    symmetric part M~A + A'M~ has no positive eigenvalue and a clearly
    negative one."""
    mesh, port = _port_column(2, 2.0, 1.0, True)
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 0.0, face_port=port)
    a = dense(orc.apply, orc.n_dof)
    ma = energy_mass(orc) @ a
    s = ma + ma.T
    ev = np.linalg.eigvalsh(s)
    scale = np.max(np.abs(ma))
    assert ev.max() < 1e-7 * scale and ev.min() < -1e-3 * scale


def test_port_face_drains_field_energy():
    """rhs.rs:2366-2445: a pulse in a PEC channel keeps its energy (> 0.95,
    central flux); with a port at the far end most of it leaves (< 0.5)."""
    kept = {}
    for with_port in (False, True):
        mesh, port = _port_column(10, 5.0, 0.5, with_port)
        orc = R.Operator(mesh.nodes, mesh.tets, 2, 0.0, face_port=port)
        xyz = orc.node_coords()
        y = np.zeros(orc.n_dof)
        y[0::6] = np.exp(-((xyz[:, 2] - 2.5) / 0.5) ** 2)
        e0 = orc.field_energy(y)
        for _ in range(900):
            y, _ = orc.expmv(y, 0.06, 24)
        kept[with_port] = orc.field_energy(y) / e0
    assert kept[False] > 0.95 and kept[True] < 0.5
