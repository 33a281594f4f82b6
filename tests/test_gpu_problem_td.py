"""The user-facing Problem API (ProblemTD, problem/td.py:195-750) on the
device: box construction, rhs, and transients by the reference's three
methods against the f64 oracle on the same mesh."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import operator as O
from rapidfem_b200.td import GaussianPulse, ProblemTD

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


def _problem():
    p = ProblemTD.box(size=(1.0, 1.0, 1.0), cells=(2, 2, 2), order=2)
    mesh = O.structured_box(2, 2, 2, 1.0, 1.0, 1.0)
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 1.0)
    y0 = np.sin(0.3 + 0.017 * np.arange(p.n_dofs))
    return p, orc, y0


def test_problem_rhs_and_sizes():
    p, orc, y0 = _problem()
    assert p.n_tets == 48 and p.n_dofs == orc.n_dof
    assert rel_l2(p.rhs(y0), orc.apply(y0.astype(np.float32).astype(np.float64))) < 1e-5


# explicit: the same LSERK4 steps as the oracle's; exponential: Krylov steps,
# exact in time, against the oracle's LSERK4 at dt/16 (time error ~1e-8 per
# step even on the highest modes of this rough field); adaptive: KCL RK4(3)5
# with the default controller (rtol 1e-4 per step) against the same reference
@pytest.mark.parametrize("method,tol", [("explicit", 1e-4), ("exponential", 1e-4), ("adaptive", 1e-3)])
def test_problem_transient_methods_match_oracle(method, tol):
    p, orc, y0 = _problem()
    dt = 0.5 * p.cfl_dt()
    steps = 6
    frames = np.asarray(p.transient(y0, dt=dt, steps=steps, method=method, verbose=False), dtype=np.float64)
    assert frames.shape == (steps + 1, p.n_dofs)
    assert rel_l2(frames[0], y0) < 1e-7
    y32 = y0.astype(np.float32).astype(np.float64)
    want = orc.lserk(y32, dt, steps) if method == "explicit" else orc.lserk(y32, dt / 16, 16 * steps)
    assert rel_l2(frames[-1], want) < tol


def test_problem_driven_transient_shapes():
    p, _, _ = _problem()
    dt = 0.5 * p.cfl_dt()
    t, series = p.driven_transient(source=((0.3, 0.5, 0.5), "E", "z"), waveform=GaussianPulse(t0=0.5, tau=0.2, f0=1.0),
                                   probes=[((0.7, 0.5, 0.5), "E", "z"), ((0.5, 0.5, 0.5), "H", "x")], dt=dt,
                                   steps=20, verbose=False)
    assert t.shape == (21,) and series.shape == (2, 21)
    assert np.all(np.isfinite(series)) and np.abs(series).max() > 0


def test_stepper_ode_and_trajectory():
    """ProblemTD.stepper / ode and the TdTrajectory return type
    (problem/td.py:47-98, :170-192, :381, :487)."""
    from rapidfem_b200 import td as TD

    p = TD.ProblemTD.box(size=(1, 1, 1), cells=(2, 2, 2), order=2)
    n = p.n_dofs
    y0 = np.sin(0.3 + 0.017 * np.arange(n))
    dt = 0.5 * p.cfl_dt()
    traj = p.transient(y0, dt=dt, steps=3, method="explicit", verbose=False)
    assert isinstance(traj, TD.TdTrajectory) and traj.shape == (4, n) and traj._dt == dt
    st = p.stepper(dt, method="explicit")
    y = y0
    for _ in range(3):
        y = st(y)
    assert np.allclose(y, traj[-1], rtol=0, atol=1e-6 * np.max(np.abs(traj[-1])))
    ode = p.ode()
    assert ode.n_dofs == n
    assert np.array_equal(ode.rhs(0.0, y0), p.rhs(y0))
    jac = ode.jacobian()
    assert jac.shape == (n, n)
    assert np.linalg.norm(jac @ y0 - p.rhs(y0)) <= 1e-5 * np.linalg.norm(p.rhs(y0))
    with pytest.raises(ValueError):
        p.stepper(dt, method="adaptive")
    ex = p.stepper(2 * dt, krylov_dim=24)(y0)
    assert np.linalg.norm(ex - p.step(y0, 2 * dt, krylov_dim=24)) <= 1e-5 * np.linalg.norm(ex)


def test_state_space_matches_the_oracle():
    """assemble_sparse (rhs.rs:1621-1700, its tests :2260-2330): the probed CSR
    against the f64 oracle's matrix-free apply, within the stencil bound and
    genuinely sparse, on an operator with a port face and materials."""
    from rapidfem_b200 import td as TD

    m = O.structured_box(3, 3, 3)
    nodes, tets = R.box_mesh(3, 3, 3, 1.0, 1.0, 1.0)
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    eps = np.where(m.nodes[m.tets].mean(axis=1)[:, 0] > 0.5, 4.0, 1.0)
    mat = O.isotropic_materials(eps, sigma=np.where(eps > 1, 0.3, 0.0))
    sess = TD.TdSession(O.MaxwellOperator(m, 2, 1.0, face_port=port, materials=mat))
    orc = R.Operator(nodes, tets, 2, 1.0, face_port=port, materials=mat)
    n, row_ptr, col_idx, vals = sess.state_space()
    assert n == orc.n_dof and row_ptr[-1] == vals.size
    assert np.all(np.diff(row_ptr) >= 0)
    for r in range(0, n, 97):  # columns ascend within a row
        assert np.all(np.diff(col_idx[row_ptr[r]:row_ptr[r + 1]]) > 0)
    stride = 6 * 10
    assert vals.size <= 5 * stride * n and vals.size < n * n // 4
    from scipy.sparse import csr_matrix
    a = csr_matrix((vals, col_idx, row_ptr), shape=(n, n))
    v = np.cos(1.0 + 0.07 * np.arange(n))
    want = orc.apply(v)
    assert np.linalg.norm(a @ v - want) <= 1e-12 * np.linalg.norm(want)


def test_resonance_of_the_unit_cube():
    """session.rs:1373-1382: TE/TM 110 of the unit PEC cube (2x2x2, N = 2,
    c = 1) at sqrt(2)/2 within 2 %, three ascending values."""
    from rapidfem_b200 import td as TD

    p = TD.ProblemTD.box(size=(1, 1, 1), cells=(2, 2, 2), order=2, c=1.0)
    f = p.resonances(n=3)
    want = np.sqrt(2.0) / 2.0
    assert f.size == 3 and abs(f[0] - want) / want < 0.02
    assert np.all(np.diff(f) > 0)


def test_driven_transient_from_a_model_port():
    """python/tests/test_td_model.py:34-78 on a model-built guide: a port-driven
    run starts at zero and injects the pulse, the GaussianPulse object and a
    Python callable of it drive the same run to the bit, the port signal has a
    row per frame, and a name that is not a port is refused."""
    from rapidfem_b200 import model as M
    from rapidfem_b200 import td as TD

    tm = M.box_tagged(3, 2, 6, 22.86e-3, 10.16e-3, 60e-3)
    p = TD.ProblemTD.from_model(tm, M.Model(faces=[M.RectangularPort(5, (1, 0)), M.AbcFace(6)]),
                                order=1, flux="upwind")
    pulse = TD.GaussianPulse(t0=90e-12, tau=22e-12, f0=10e9)
    t = np.linspace(0.0, 200e-12, 9)
    ref = np.exp(-((t - 90e-12) / 22e-12) ** 2) * np.cos(2 * np.pi * 10e9 * (t - 90e-12))
    assert np.allclose(pulse(t), ref, rtol=0.0, atol=1e-15) and pulse(90e-12) == 1.0
    run = dict(port=5, dt=3e-12, steps=20, method="explicit", verbose=False)
    native = p.transient(waveform=pulse, **run)
    python = p.transient(waveform=lambda s: pulse(s), **run)
    amp = np.linalg.norm(np.asarray(native), axis=1)
    assert np.all(np.isfinite(native)) and amp[0] == 0.0 and amp.max() > 0.0
    assert np.array_equal(native, python)
    _, rows = p.port_signals(native, [5])
    assert rows.shape == (1, 21) and np.abs(rows).max() > 0.0
    with pytest.raises(ValueError, match="not a port"):
        p.transient(port=99, waveform=pulse, dt=3e-12, steps=1, verbose=False)


def test_transfer_function_matches_the_oracle():
    """ProblemTD.transfer_function (problem/td.py:549-598, session.rs:985-999):
    the probe series of the driven run it makes equals the reference's LSERK4
    run on the oracle with the source held per step, and H is the transfer of
    that series with the pulse sampled at the frame times."""
    from rapidfem_b200 import td as TD

    p, orc, _ = _problem()
    dt = 0.5 * p.cfl_dt()  # one LSERK4 step per frame
    steps = 200
    pulse = GaussianPulse(t0=1.0, tau=0.25, f0=0.8)
    source, probe = ((0.3, 0.5, 0.5), "E", "z"), ((0.7, 0.5, 0.5), "E", "z")
    tf = p.transfer_function(source=source, probe=probe, pulse=pulse, dt=dt, steps=steps, verbose=False)
    assert isinstance(tf, TD.TdTransfer) and tf.source_label == "E_z @ (0.3, 0.5, 0.5)"
    f, h = tf
    assert f.shape == h.shape == ((steps + 1) // 2 + 1,)
    t, series = p.driven_transient(source=source, waveform=pulse, probes=[probe], dt=dt, steps=steps, verbose=False)
    f_ref, h_ref = TD.transfer(pulse(t), series[0], dt)
    assert np.array_equal(f, f_ref) and np.array_equal(h, h_ref)
    src = p.probe_dof(source[0], field="E", component="z")
    pr = p.probe_dof(probe[0], field="E", component="z")
    g32 = np.asarray(pulse(t), dtype=np.float32).astype(np.float64)
    y = np.zeros(p.n_dofs)
    want = [0.0]
    for k in range(steps):
        y = orc.lserk(y, dt, 1, src_dof=src, vals=g32[k:k + 1])
        want.append(y[pr])
    want = np.array(want)
    assert rel_l2(series[0], want) < 1e-4
    _, h_orc = TD.transfer(pulse(t), want, dt)
    band = h_orc != 0
    assert band.sum() > 5 and np.all(h[~band] == 0)
    assert np.linalg.norm(h[band] - h_orc[band]) < 1e-3 * np.linalg.norm(h_orc[band])
