"""Port modal probes on the GPU: the per-frame modal amplitudes P_e, P_h
(rhs.rs:1211-1242) computed on the device as linear functionals of the state,
against the host projections of a recorded trajectory (the reference's
port_signals, session.rs:1041-1054) and against the f64 oracle."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200 import td as T

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def _guide():
    m = O.structured_box(2, 2, 4, 1.0, 0.5, 2.0)
    nodes, tets = R.box_mesh(2, 2, 4, 1.0, 0.5, 2.0)
    port = np.where(O.boundary_faces_on_plane(m, 2, 0.0), 0, -1)
    port[O.boundary_faces_on_plane(m, 2, 2.0)] = 1
    prod = O.MaxwellOperator(m, 2, 1.0, face_port=port)
    orc = R.Operator(nodes, tets, 2, 1.0, face_port=port)
    return m, port, prod, orc


def _drive(prod, orc, steps):
    prof0 = prod.rect_port_profiles(0, [0, 0, 1.0], (1, 0))
    prof1 = prod.rect_port_profiles(1, [0, 0, -1.0], (1, 0))
    b = prod.port_source(0, prof0)
    dt = 0.5 / orc.power_rho(40)[0]
    t = np.arange(steps) * dt
    g = np.exp(-((t - 30 * dt) / (10 * dt)) ** 2) * np.cos(2 * np.pi * 1.5 * t)
    return prof0, prof1, b, dt, g


def test_functionals_equal_host_projections_of_trajectory(ctx):
    _, _, prod, orc = _guide()
    steps = 80
    prof0, prof1, b, dt, g = _drive(prod, orc, steps)
    gop = G.GpuOperator(ctx, prod)
    n = gop.n_dof()
    dof = prod.nearest_node_dof([0.5, 0.25, 1.0], 0, 1)
    funcs = [prod.port_modal_weights(0, prof0, "E"), prod.port_modal_weights(0, prof0, "H"),
             prod.port_modal_weights(1, prof1, "E"), (np.array([dof]), np.ones(1))]
    series, yf = gop.transient_functionals(np.zeros(n), dt, steps, 1, drive=("vector", b), g=g, functionals=funcs)
    traj = gop.transient(np.zeros(n), dt, steps, 1, drive=("vector", b), g=g, record=True).astype(np.float64)
    want = np.stack([traj[:, i] @ w for i, w in funcs], axis=1)
    assert series.shape == (steps + 1, 4)
    assert np.array_equal(yf.astype(np.float64), traj[-1])
    assert np.array_equal(series[:, 3], traj[:, dof])
    assert np.max(np.abs(series - want)) <= 1e-12 * np.max(np.abs(want))
    assert np.max(np.abs(series[:, 2])) > 0  # the pulse reaches the far port


def test_port_amplitude_series_matches_oracle(ctx):
    _, _, prod, orc = _guide()
    steps = 80
    prof0, prof1, b, dt, g = _drive(prod, orc, steps)
    gop = G.GpuOperator(ctx, prod)
    n = gop.n_dof()
    funcs = [prod.port_modal_weights(0, prof0, "E"), prod.port_modal_weights(1, prof1, "E")]
    series, _ = gop.transient_functionals(np.zeros(n), dt, steps, 1, drive=("vector", b), g=g, functionals=funcs)
    y = np.zeros(n)
    b64 = b.astype(np.float32).astype(np.float64)
    g64 = g.astype(np.float32).astype(np.float64)
    want = [[orc.port_projections(0, prof0, y)[0], orc.port_projections(1, prof1, y)[0]]]
    for k in range(steps):
        y = orc.lserk(y, dt, 1, src_vec=b64, vals=g64[k:k + 1])
        want.append([orc.port_projections(0, prof0, y)[0], orc.port_projections(1, prof1, y)[0]])
    want = np.array(want)
    assert rel_l2(series[:, 0], want[:, 0]) < 1e-4
    assert rel_l2(series[:, 1], want[:, 1]) < 1e-4


def test_session_port_probes_match_port_signals(ctx):
    m, port, _, _ = _guide()
    faces0 = port == 0
    faces1 = port == 1
    ports = {"in": {"faces": faces0, "inward_normal": (0, 0, 1.0), "mode": (1, 0)},
             "out": {"faces": faces1, "inward_normal": (0, 0, -1.0), "mode": (1, 0)}}
    s = T.TdSession.from_mesh(m, 2, ports=ports)
    dt = s.cfl_dt()
    wave = T.GaussianPulse(20 * dt, 8 * dt, 1.0)
    steps = 40
    dof = s.nearest_node_dof((0.5, 0.25, 1.0), "E", "y")
    rows, _ = s.transient(None, dt=dt, steps=steps, port="in", waveform=wave, probes=[dof],
                          port_probes=["in", "out"], method="explicit", verbose=False)
    traj, _ = s.transient(None, dt=dt, steps=steps, port="in", waveform=wave, method="explicit", verbose=False)
    assert rows.shape == (steps + 1, 3)
    sig = s.port_signals(traj, ["in", "out"])
    assert np.array_equal(rows[:, 0], traj[:, dof])
    assert np.max(np.abs(rows[:, 1:] - sig.T)) <= 1e-12 * np.max(np.abs(sig))
    with pytest.raises(ValueError):
        s.port_signals(traj[:, :-1], ["in"])


def test_recorded_functionals_on_resident_state(ctx):
    """dgtd_record_functionals between stage-level LSERK4 calls equals the
    per-step series of dgtd_transient_functionals, and an ETD run records the
    same functionals at each accepted step (its last row equals the host
    projection of its final state)."""
    from rapidfem_b200 import etd as ETD

    _, _, prod, orc = _guide()
    steps = 40
    prof0, prof1, b, dt, g = _drive(prod, orc, steps)
    gop = G.GpuOperator(ctx, prod)
    n = gop.n_dof()
    funcs = [prod.port_modal_weights(0, prof0, "E"), prod.port_modal_weights(1, prof1, "E")]
    want, _ = gop.transient_functionals(np.zeros(n), dt, steps, 1, drive=("vector", b), g=g, functionals=funcs)
    gop.upload(np.zeros(n, dtype=np.float32))
    gop.set_source_vector(b)
    gop.set_functionals(funcs, steps + 1)
    gop.record_functionals(0)
    for k in range(steps):
        # a held sample per step: the 5 stage values all equal g[k]
        gop.run_lserk_stages(dt, 1, drive=("vector", None), g_stages=np.full(5, g[k], dtype=np.float32))
        gop.record_functionals(k + 1)
    got = gop.functional_series(steps + 1)
    assert np.array_equal(got, want)
    with pytest.raises(Exception):
        gop.record_functionals(steps + 1)  # past the rows set aside

    t0, tau = 30 * dt, 10 * dt
    wave = lambda t: np.exp(-((np.asarray(t) - t0) / tau) ** 2) * np.cos(2 * np.pi * 1.5 * np.asarray(t))
    y, st = ETD.run_etd(gop, np.zeros(n), b, wave, steps * dt, 4 * dt, ETD.PlainEtd(1e-7, 24),
                        functionals=funcs)
    assert st.series.shape == (st.accepted + 1, 2) and st.times[0] == 0.0
    assert abs(st.times[-1] - steps * dt) < 1e-9 * steps * dt
    host = np.array([np.dot(y[i], w) for i, w in funcs])
    assert np.allclose(st.series[-1], host, rtol=1e-5, atol=1e-9 * np.max(np.abs(want)))
