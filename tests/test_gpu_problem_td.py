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
