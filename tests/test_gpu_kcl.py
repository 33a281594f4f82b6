"""KCL RK4(3)5[2R+]C adaptive stepping on the GPU with the PI controller on
the device (explicit_adaptive.rs:84-152, session.rs:130-187,
gpu/operator.rs:823-893): one step against the f64 oracle, a controlled run
against a host replica of the reference controller over oracle steps, the
device-recorded functionals against the recorded trajectory, and the
step-collapse error."""
import math

import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200 import td as T
from rapidfem_b200._native import DGTD_ERR_COLLAPSE, ENGINE_FP32, ENGINE_TF32X3, DgtdError

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def _cavity(order=3, cells=3):
    m = O.structured_box(cells, cells, cells)
    nodes, tets = R.box_mesh(cells, cells, cells, 1.0, 1.0, 1.0)
    prod = O.MaxwellOperator(m, order, 1.0)
    orc = R.Operator(nodes, tets, order, 1.0)
    xyz = orc.node_coords()
    y0 = np.zeros(prod.n_dof)
    y0[2::6] = np.sin(np.pi * xyz[:, 0]) * np.sin(np.pi * xyz[:, 1])  # TM110 E_z
    return prod, orc, y0


def _err_norm(ctl, y_old, y_new, err):
    if not np.all(np.isfinite(y_new)):
        return math.inf
    sc = ctl.atol + ctl.rtol * np.maximum(np.abs(y_old), np.abs(y_new))
    return float(np.sqrt(np.mean((err / sc) ** 2)))


def _factor(ctl, err_norm, prev, reject):
    err = max(err_norm, 1e-12)
    f = ctl.safety * err ** (-ctl.pi_alpha)
    if not (reject or prev <= 0.0):
        f *= prev ** ctl.pi_beta
    return max(f, ctl.shrink_limit) if reject else min(max(f, ctl.shrink_limit), ctl.growth_limit)


def _host_kcl(orc, y0, dt, steps, ctl):
    """The reference's host loop (gpu/operator.rs:836-887) over f64 oracle steps,
    with the controller scalars in f32 as the reference keeps them."""
    f32 = np.float32
    y = y0.copy()
    h, prev, dtf = f32(dt), f32(0.0), f32(dt)
    acc = rej = 0
    for _ in range(steps):
        t_rel = f32(0.0)
        while t_rel < dtf:
            h_try = min(h, f32(dtf - t_rel))
            y_new, err = orc.kcl_step(y, float(h_try))
            en = f32(_err_norm(ctl, y, y_new, err))
            if math.isfinite(en) and en <= 1.0:
                t_rel = f32(t_rel + h_try)
                acc += 1
                h = f32(h_try * f32(_factor(ctl, float(en), float(prev), False)))
                prev = f32(max(en, f32(1e-12)))
                y = y_new
            else:
                rej += 1
                probe = en if math.isfinite(en) else f32(10.0)
                h = f32(h_try * f32(_factor(ctl, float(probe), float(prev), True)))
            assert h >= f32(ctl.min_step_factor) * dtf
    return y, acc, rej


def _replay(gop, orc, y0, steps, src_dof=None, g=None):
    """The device run's own accepted substeps (h, frame) replayed on the f64
    oracle from the same f32 initial state, the waveform held per frame as
    the device holds it; returns the frames [steps+1, n]."""
    h, fr = gop.kcl_accepted_steps()
    assert h.size > 0 and np.all(np.diff(fr) >= 0) and fr[-1] == steps - 1
    y = np.asarray(y0, dtype=np.float32).astype(np.float64)
    frames = [y]
    for hk, f in zip(h, fr):
        gk = 0.0 if g is None else float(np.float32(g[f]))
        y, _ = orc.kcl_step(y, float(hk), src_dof=src_dof, g=gk)
        if len(frames) <= f + 1:
            frames.append(y)
        else:
            frames[f + 1] = y
    assert len(frames) == steps + 1
    return np.array(frames)


def test_kcl_step_matches_oracle(ctx):
    prod, orc, y0 = _cavity()
    gop = G.GpuOperator(ctx, prod)
    rho, _ = orc.power_rho(30)
    h = 1.0 / rho
    y_gpu, e_gpu = gop.kcl_step(y0, h)
    y_ref, e_ref = orc.kcl_step(y0.astype(np.float32).astype(np.float64), h)
    assert rel_l2(y_gpu, y_ref) < 1e-5
    # The embedded error is a small sum of O(|y|) stage terms, so its f32 value
    # carries f32 cancellation: bound it against the state, and relative to
    # itself well inside what the controller's rtol = 1e-4 weighting resolves.
    assert np.linalg.norm(e_gpu - e_ref) < 1e-6 * np.linalg.norm(y_ref)
    assert rel_l2(e_gpu, e_ref) < 2e-2


@pytest.mark.parametrize("engine,slack", [(ENGINE_FP32, 2), (ENGINE_TF32X3, 6)], ids=["fp32", "tf32x3"])
def test_kcl_run_matches_host_controller(ctx, engine, slack):
    """Two checks.  (1) The device's own accepted step sequence, replayed on the
    f64 oracle, gives every recorded frame within 1e-4.  (2) The reference's
    host loop, run on f64 oracle states, takes about the same decisions: it
    decides on f64 states and the device on f32 ones (FP32 kernel: the
    reference's own f32 path), so decisions near the err_norm = 1 threshold
    may differ by a few."""
    prod, orc, y0 = _cavity()
    gop = G.GpuOperator(ctx, prod)
    gop.set_engine(engine)
    rho, _ = orc.power_rho(30)
    dt = 4.0 / rho  # frames longer than the stability limit: the controller must cut the step
    steps = 6
    ctl = G.GpuOperator.kcl_controller()
    traj, st = gop.transient_kcl(y0, dt, steps, controller=ctl, record=True)
    y_host, acc, rej = _host_kcl(orc, y0.astype(np.float32).astype(np.float64), dt, steps, ctl)
    assert st["accepted"] + st["rejected"] > steps
    assert abs(st["accepted"] - acc) <= slack and abs(st["rejected"] - rej) <= slack
    assert rel_l2(traj[-1], y_host) < 1e-3  # a different step sequence: agreement to the controller tolerance
    want = _replay(gop, orc, y0, steps)
    assert len(gop.kcl_accepted_steps()[0]) == st["accepted"]
    for k in range(steps + 1):
        assert rel_l2(traj[k], want[k]) < 1e-4, k
    assert 0 < st["h_min"] <= st["h_max"]
    assert np.array_equal(traj[0], y0.astype(np.float32))


def test_kcl_functionals_match_trajectory(ctx):
    prod, orc, y0 = _cavity()
    gop = G.GpuOperator(ctx, prod)
    rho, _ = orc.power_rho(30)
    dt = 2.0 / rho
    steps = 8
    dof = prod.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    rng = np.random.default_rng(3)
    idx = rng.choice(prod.n_dof, 50, replace=False)
    w = rng.normal(size=50)
    traj, st1 = gop.transient_kcl(y0, dt, steps, record=True)
    series, yf, st2 = gop.transient_kcl_functionals(y0, dt, steps, functionals=[(np.array([dof]), np.ones(1)),
                                                                                (idx, w)])
    assert st1 == st2
    t64 = traj.astype(np.float64)
    assert np.array_equal(series[:, 0], t64[:, dof])
    assert np.max(np.abs(series[:, 1] - t64[:, idx] @ w)) <= 1e-12 * np.max(np.abs(t64[:, idx] @ w))
    assert np.array_equal(yf, traj[-1])


def test_kcl_driven_point_source(ctx):
    prod, orc, _ = _cavity(order=2)
    gop = G.GpuOperator(ctx, prod)
    n = prod.n_dof
    rho, _ = orc.power_rho(30)
    dt = 1.0 / rho
    steps = 30
    dof = prod.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    g = np.exp(-((np.arange(steps) * dt - 10 * dt) / (4 * dt)) ** 2)
    traj, st = gop.transient_kcl(np.zeros(n), dt, steps, drive=("point", dof), g=g, record=True)
    # the device's accepted steps replayed on the oracle, the source held per frame
    want = _replay(gop, orc, np.zeros(n), steps, src_dof=dof, g=g)
    assert rel_l2(traj[-1], want[-1]) < 1e-4
    for k in range(1, steps + 1):
        assert rel_l2(traj[k], want[k]) < 1e-4, k
    # the same held source through LSERK4 with a small fixed step agrees to the controller tolerance
    ref = np.zeros(n)
    sub = 8
    for k in range(steps):
        ref = orc.lserk(ref, dt / sub, sub, src_dof=dof, vals=np.full(sub, float(np.float32(g[k]))))
    assert rel_l2(traj[-1], ref) < 2e-3
    assert np.max(np.abs(traj[-1])) > 0


def test_kcl_collapse_is_an_error(ctx):
    prod, orc, y0 = _cavity(order=2)
    gop = G.GpuOperator(ctx, prod)
    rho, _ = orc.power_rho(30)
    ctl = G.GpuOperator.kcl_controller(atol=1e-30, rtol=1e-30, min_step_factor=0.5)
    with pytest.raises(DgtdError) as ei:
        gop.transient_kcl(y0, 1.0 / rho, 3, controller=ctl, record=False)
    assert ei.value.code == DGTD_ERR_COLLAPSE
    assert "collapsed" in str(ei.value)


def test_session_adaptive_method(ctx):
    s = T.TdSession.box_cavity(2, 2, 2, 1.0, 1.0, 1.0, 2)
    n = s.n_dofs()
    y0 = np.sin(0.3 + 0.017 * np.arange(n))
    dt = 2.0 * s.cfl_dt()
    rows, stats = s.transient(y0, dt=dt, steps=4, method="adaptive", verbose=False)
    assert rows.shape == (5, n) and len(stats) == 4 and stats[0] >= 4
    p = [0, 7, n - 1]
    rows_p, stats_p = s.transient(y0, dt=dt, steps=4, method="adaptive", probes=p, verbose=False)
    assert stats_p == stats
    assert np.array_equal(rows_p, rows[:, p])
    with pytest.raises(ValueError):
        s.transient(y0, dt=dt, steps=4, method="adaptive", warmup=1, verbose=False)
    y1, err = s.step_adaptive(y0, 0.5 * s.cfl_dt())
    assert y1.shape == (n,) and err.shape == (n,) and np.all(np.isfinite(err))
