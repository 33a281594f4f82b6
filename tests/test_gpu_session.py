"""The reference's session tests (session.rs:1289-1350) on TdSession: the
three integrators agree on free and driven runs, warm-up and probe recording,
and the cached, stable CFL step.  (The run hook of session.rs:1335 has no
counterpart: a device run is not interrupted between frames.)"""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import td as TD

pytestmark = pytest.mark.gpu


def session():
    """session.rs:1268-1271: the 2^3 unit cube, N = 2, upwind, c = 1."""
    return TD.TdSession.box_cavity(2, 2, 2, 1.0, 1.0, 1.0, 2, "upwind", 1.0)


def pulse(t):
    return np.exp(-((np.asarray(t) - 1.0) / 0.3) ** 2)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def test_integrators_agree_on_free_and_driven_runs():
    s = session()
    n = s.n_dofs()
    y0 = R.normal_vector(n, 7)
    d = s.nearest_node_dof([0.4, 0.5, 0.5], "E", "z")
    for driven in (False, True):
        kw = dict(dt=0.05, steps=12, verbose=False)
        if driven:
            kw.update(y0=None, source_dof=d, waveform=pulse)
        else:
            kw.update(y0=y0)
        exp, _ = s.transient(method="exponential", **kw)
        assert exp.shape == (13, n)
        for method in ("explicit", "adaptive"):
            r, stats = s.transient(method=method, **kw)
            tol = {(False, "explicit"): 1e-2, (False, "adaptive"): 1e-4,
                   (True, "explicit"): 5e-2, (True, "adaptive"): 0.5}[(driven, method)]
            assert rel(r[-1], exp[-1]) < tol, (driven, method)
            if method == "adaptive":
                assert stats[0] >= 12


def test_warmup_and_probes():
    s = session()
    n = s.n_dofs()
    y0 = R.normal_vector(n, 3)
    full, _ = s.transient(y0, dt=0.05, steps=12, method="explicit", warmup=3, verbose=False)
    p, _ = s.transient(y0, dt=0.05, steps=12, method="explicit", warmup=3, probes=[5, 17], verbose=False)
    assert p.shape == (13, 2)
    assert np.array_equal(p[:, 0], full[:, 5]) and np.array_equal(p[:, 1], full[:, 17])
    with pytest.raises(ValueError):
        s.transient(None, dt=0.05, steps=2, method="adaptive", warmup=1, verbose=False)


def test_cfl_step_is_stable_and_cached():
    s = session()
    h = s.cfl_dt()
    assert 0.0 < h < np.inf and s.cfl_dt() == h
    y = R.normal_vector(s.n_dofs(), 1)
    n0 = np.linalg.norm(y)
    for _ in range(500):
        y = s.step_explicit(y, h)
    assert np.linalg.norm(y) <= 1.01 * n0
