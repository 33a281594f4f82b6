"""The reference's operator physics tests on the f64 oracle (whose host
arrays the product's host build matches bit for bit): element curl exactness,
dielectric and absorber spectra, energy conservation, the soft source,
conductivity damping (rhs.rs:1995-2030), port dissipation (:2366-2520) and the
waveguide port (:2522-2735); tests/test_gpu_physics.py runs the operator-level
ones on the device path."""
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


# ---- the rectangular waveguide port (rhs.rs:2522-2735): TE10 injected at
# z = 0 of a 1 x 0.5 x 9 guide (N = 2, central flux), a Gaussian-modulated sine
OMEGA0 = 1.6 * np.pi


def guide():
    """(mesh, host operator with the TE10 port at z = 0, port source b,
    P_e / P_h functionals)."""
    mesh = O.structured_box(2, 1, 18, 1.0, 0.5, 9.0)
    port = np.where(O.boundary_faces_on_plane(mesh, 2, 0.0), 0, -1)
    op = O.MaxwellOperator(mesh, 2, 0.0, face_port=port)
    prof = op.rect_port_profiles(0, [0.0, 0.0, 1.0], (1, 0))
    return mesh, port, op, op.port_source(0, prof), (op.port_modal_weights(0, prof, "E"),
                                                     op.port_modal_weights(0, prof, "H"))


def pulse(t):
    return np.exp(-((t - 7.0) / 2.5) ** 2) * np.sin(OMEGA0 * (t - 7.0))


def group_velocity_check(etd_step, op):
    """rhs.rs:2522-2623: the packet's peaks at z = 3.5 and 6.5 (E_y at the
    guide's centre) travel at the TE10 group velocity sqrt(1 - (pi/a/w0)^2)
    within 15 %; 850 ETD steps of 0.02 with the source held per step."""
    b = guide()[3]
    p1 = op.nearest_node_dof([0.5, 0.25, 3.5], 0, 1)
    p2 = op.nearest_node_dof([0.5, 0.25, 6.5], 0, 1)
    y = np.zeros(op.n_dof)
    pk = [[0.0, 0.0], [0.0, 0.0]]
    for s in range(850):
        t = s * 0.02
        y = etd_step(y, b * pulse(t), 0.02, 20)
        for k, p in enumerate((p1, p2)):
            if abs(y[p]) > pk[k][0]:
                pk[k] = [abs(y[p]), t]
    assert np.all(np.isfinite(y)) and pk[0][0] > 1e-3 and pk[1][0] > 1e-3
    v = 3.0 / (pk[1][1] - pk[0][1])
    vg = np.sqrt(1.0 - (np.pi / OMEGA0) ** 2)
    assert abs(v - vg) / vg < 0.15


def incident_amplitude_check(etd_step, funcs):
    """rhs.rs:2623-2735: from the port's P_e, P_h series the incident wave
    A = (P_e + Z P_h) / 2 dominates the reflected B = (P_e - Z P_h) / 2
    (|B/A| < 0.06, Z = w / sqrt(w^2 - (pi/a)^2) the TE10 impedance) at three
    frequencies of the band; 700 steps."""
    b = guide()[3]
    (ie, we), (ih, wh) = funcs
    y = np.zeros(b.size)
    pe, ph = [], []
    dt = 0.02
    for s in range(700):
        y = etd_step(y, b * pulse(s * dt), dt, 20)
        pe.append(we @ y[ie])
        ph.append(wh @ y[ih])
    t = np.arange(700) * dt
    for w in (1.45 * np.pi, 1.6 * np.pi, 1.75 * np.pi):
        ker = np.exp(-1j * w * t) * dt
        fe, fh = np.dot(pe, ker), np.dot(ph, ker)
        z = w / np.sqrt(w * w - np.pi ** 2)
        a_inc, b_ref = 0.5 * (fe + z * fh), 0.5 * (fe - z * fh)
        assert abs(a_inc) > 1e-3 and abs(b_ref) / abs(a_inc) < 0.06


def test_port_injects_a_mode_at_the_group_velocity():
    mesh, port, op, _, _ = guide()
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 0.0, face_port=port)
    group_velocity_check(lambda y, b, h, m: orc.etd_step(y, b, h, m)[0], op)


def test_port_extracts_the_incident_amplitude():
    mesh, port, op, _, funcs = guide()
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 0.0, face_port=port)
    incident_amplitude_check(lambda y, b, h, m: orc.etd_step(y, b, h, m)[0], funcs)


# ---- cavity modes and energy conservation (rhs.rs:1830-1945, :2113-2222)
WANT_FUNDAMENTAL = np.pi * np.sqrt(2.0)  # TE/TM110 of the unit PEC cube, c = 1


def fundamental(a):
    """(Re, |Im|) of the least-damped physical mode (|Im| > 1)."""
    ev = np.linalg.eigvals(a)
    ev = ev[np.abs(ev.imag) > 1.0]
    z = ev[np.argmax(ev.real)]
    return float(z.real), float(abs(z.imag))


def anisotropic_box():
    mesh = O.structured_box_jittered(2, 1, 1, 1.0, 0.6, 0.7, 0.2, 5)
    K = mesh.n_tets
    mat = np.zeros((K, 8))
    i = np.arange(K)
    mat[:, 0], mat[:, 1], mat[:, 2] = 2.0 + (i % 3), 3.0, 1.5
    mat[:, 3], mat[:, 4], mat[:, 5] = 1.0, 1.2 + 0.3 * (i % 2), 2.0
    return mesh, mat


def skew_defect(a, m):
    """|M~A + A'M~| / |M~A| (central flux, no loss, PEC: exactly skew)."""
    ma = m @ a
    return float(np.linalg.norm(ma + ma.T) / np.linalg.norm(ma))


def test_cavity_fundamental_on_an_irregular_mesh():
    """rhs.rs:2151-2185: jittered 2^3 cube (amplitude 0.25, seed 7), N = 2,
    upwind: the fundamental is damped (Re < 0) and within 8 % of pi sqrt 2."""
    mesh = O.structured_box_jittered(2, 2, 2, 1.0, 1.0, 1.0, 0.25, 7)
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 1.0)
    re, im = fundamental(dense(orc.apply, orc.n_dof))
    assert re < 0.0 and abs(im - WANT_FUNDAMENTAL) / WANT_FUNDAMENTAL < 0.08


def test_cavity_fundamental_converges():
    """rhs.rs:2187-2222: N = 2 on the 1^3 and 2^3 cubes: the error falls and is
    below 1e-3 on the finer mesh."""
    err = []
    for cells in (1, 2):
        mesh = O.structured_box(cells, cells, cells)
        orc = R.Operator(mesh.nodes, mesh.tets, 2, 1.0)
        err.append(abs(fundamental(dense(orc.apply, orc.n_dof))[1] - WANT_FUNDAMENTAL) / WANT_FUNDAMENTAL)
    assert err[1] < err[0] and err[1] < 1e-3


def test_anisotropic_central_flux_conserves_energy():
    """rhs.rs:2031-2075: diagonal anisotropic eps and mu varying by element,
    central flux, jittered mesh: M~A is skew to rounding."""
    mesh, mat = anisotropic_box()
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 0.0, materials=mat)
    assert skew_defect(dense(orc.apply, orc.n_dof), energy_mass(orc)) < 1e-12


# ---- element curl, dielectric and absorber physics, soft source (rhs.rs:1778-2110, :2223-2260)
SHEARED_TET = np.array([[0.3, -0.2, 0.1], [1.4, 0.1, -0.2], [0.2, 1.3, 0.4], [-0.1, 0.2, 1.6]])
ONE_TET = np.array([[0, 1, 2, 3]], dtype=np.int32)


def test_curl_of_polynomial_field_is_exact():
    """rhs.rs:1778-1813: on a sheared element the discrete curl of
    F = (y z, 2 z x, 3 x y) is curl F = (x, -2 y, z) at the nodes (N = 2; the
    field is in every higher order's space too, so N = 3..5 as well)."""
    for order in (2, 3, 4, 5):
        orc = R.Operator(SHEARED_TET, ONE_TET, order)
        p = orc.node_coords()
        field = np.stack([p[:, 1] * p[:, 2], 2.0 * p[:, 2] * p[:, 0], 3.0 * p[:, 0] * p[:, 1]], axis=1)
        curl = R.curl_single(order, orc.get("jinv"), field).reshape(-1, 3)
        want = np.stack([p[:, 0], -2.0 * p[:, 1], p[:, 2]], axis=1)
        assert np.max(np.abs(curl - want)) < 1e-9, order


def test_curl_of_constant_field_vanishes():
    """rhs.rs:1815-1828: a constant field has zero curl (N = 3, and N = 5)."""
    ref = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    for order in (3, 5):
        orc = R.Operator(ref, ONE_TET, order)
        curl = R.curl_single(order, orc.get("jinv"), np.full(3 * orc.np, 0.7))
        assert np.max(np.abs(curl)) < 1e-10


def test_uniform_dielectric_shifts_cavity_resonance():
    """rhs.rs:1870-1898: filling the unit cube with eps_r = 4 scales the
    fundamental to pi sqrt 2 / sqrt(eps_r) within 2 % (2^3 mesh, N = 2, upwind)."""
    mesh = O.structured_box(2, 2, 2)
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 1.0, materials=O.isotropic_materials(np.full(mesh.n_tets, 4.0)))
    ev = np.linalg.eigvals(dense(orc.apply, orc.n_dof))
    ev = ev[np.abs(ev.imag) > 0.5]
    im = float(abs(ev[np.argmax(ev.real)].imag))
    assert abs(im - WANT_FUNDAMENTAL / 2.0) / (WANT_FUNDAMENTAL / 2.0) < 0.02


def test_heterogeneous_central_flux_conserves_energy():
    """rhs.rs:1899-1943: isotropic eps = 1 + 0.7 i, mu = 1 + 0.3 i by element
    (unit cube, N = 2, central flux): M~A is skew to 1e-9 of its largest entry."""
    mesh = O.structured_box(1, 1, 1)
    i = np.arange(mesh.n_tets)
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 0.0, materials=O.isotropic_materials(1.0 + 0.7 * i, 1.0 + 0.3 * i))
    ma = energy_mass(orc) @ dense(orc.apply, orc.n_dof)
    assert np.max(np.abs(ma + ma.T)) < 1e-9 * max(np.max(np.abs(ma)), 1.0)


def test_matched_absorber_damps_at_the_full_rate():
    """rhs.rs:2075-2110: an impedance-matched loss (sigma / eps = sigma* / mu =
    nu = 0.15) shifts the least-damped mode's real part by -nu within 8 %,
    twice an electric-only loss (unit cube, N = 2, upwind)."""
    mesh = O.structured_box(1, 1, 1)
    ones = np.ones(mesh.n_tets)
    res = []
    for mat in (O.isotropic_materials(ones), O.isotropic_materials(ones, ones, 0.15 * ones, 0.15 * ones)):
        orc = R.Operator(mesh.nodes, mesh.tets, 2, 1.0, materials=mat)
        res.append(least_damped_re(dense(orc.apply, orc.n_dof)))
    assert abs((res[1] - res[0]) + 0.15) / 0.15 < 0.08


def test_soft_source_injects_energy():
    """rhs.rs:2223-2260: a Gaussian pulse (t0 = 0.3, tau = 0.08) at the E_z DOF of
    the unit cube's centre node, 80 ETD steps of 0.01 (m = 30) from rest,
    leaves finite fields with energy > 1e-6."""
    mesh = O.structured_box(1, 1, 1)
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 1.0)
    sdof = O.MaxwellOperator(mesh, 2, 1.0).nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    y = np.zeros(orc.n_dof)
    for k in range(80):
        b = np.zeros(orc.n_dof)
        b[sdof] = np.exp(-(((k * 0.01) - 0.3) / 0.08) ** 2)
        y, _ = orc.etd_step(y, b, 0.01, 30)
    assert np.all(np.isfinite(y))
    assert float(y @ energy_mass(orc) @ y) > 1e-6
