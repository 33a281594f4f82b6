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
    with pytest.raises(NotImplementedError):
        ode.jacobian()
    with pytest.raises(ValueError):
        p.stepper(dt, method="adaptive")
    ex = p.stepper(2 * dt, krylov_dim=24)(y0)
    assert np.linalg.norm(ex - p.step(y0, 2 * dt, krylov_dim=24)) <= 1e-5 * np.linalg.norm(ex)
