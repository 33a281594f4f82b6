"""The learned ETD controller's pieces on the device: the MLP's forward,
gradient and Adam kernels against the numpy restatement, and the ETD step's
a-posteriori estimate."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import etd as E
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O

from .conftest import rel_l2
from .mlp_ref import forward, loss_and_grad

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def test_mlp_forward_and_gradient_match_numpy(ctx):
    mlp = E.Mlp(ctx, 16, 64, 2, seed=3)
    rng = np.random.default_rng(4)
    x = rng.normal(size=(40, 16)).astype(np.float32)
    t = rng.normal(size=(40, 2)).astype(np.float32)
    p = mlp.params.astype(np.float64)
    y_ref, _ = forward(p, x, 16, 64, 2)
    assert rel_l2(mlp.forward(x), y_ref) < 1e-5
    g, loss = mlp.gradient(x, t)
    loss_ref, g_ref = loss_and_grad(p, x, t, 16, 64, 2)
    assert abs(loss - loss_ref) < 1e-5 * loss_ref
    assert np.max(np.abs(g - g_ref)) < 1e-4 * np.max(np.abs(g_ref))
    # the same gradient again (fixed-order reduction)
    g2, _ = mlp.gradient(x, t)
    assert np.array_equal(g, g2)


def test_mlp_adam_training(ctx):
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=(256, 16)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) * x[:, 1], 0.5 * x[:, 2] - x[:, 3] ** 2], axis=1).astype(np.float32)
    a = E.Mlp(ctx, seed=7)
    b = E.Mlp(ctx, seed=7)
    la = a.train(x, t, epochs=600, lr=3e-3)
    lb = b.train(x, t, epochs=600, lr=3e-3)
    assert np.array_equal(la, lb) and np.array_equal(a.params, b.params)  # deterministic
    assert la[-1] < 0.05 * la[0]
    # one Adam step against the numpy restatement
    c = E.Mlp(ctx, seed=9)
    p0 = c.params.astype(np.float64)
    c.train(x[:32], t[:32], epochs=1, lr=1e-2)
    _, g = loss_and_grad(p0, x[:32], t[:32], 16, 64, 2)
    m = 0.1 * g
    v = 0.001 * g * g
    p1 = p0 - 1e-2 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.max(np.abs(c.params - p1)) < 1e-5


def test_etd_step_estimate(ctx):
    m = O.structured_box(3, 3, 3)
    nodes, tets = R.box_mesh(3, 3, 3, 1.0, 1.0, 1.0)
    prod = O.MaxwellOperator(m, 2, 1.0)
    orc = R.Operator(nodes, tets, 2, 1.0)
    gop = G.GpuOperator(ctx, prod)
    n = prod.n_dof
    y = np.sin(0.3 + 0.017 * np.arange(n))
    b = np.cos(0.1 + 0.03 * np.arange(n))
    rho, _ = orc.power_rho(30)
    h = 1.0 / rho
    # one Krylov sub-step (m <= 12): its Arnoldi stops once the estimate is below tol
    out, dim, est = gop.etd_step_est(y, b, h, 12, 1e-8)
    assert 0 <= est <= 1e-8 and dim <= 12
    want, _ = orc.etd_step(y, b, h, 60, 0.0)
    assert rel_l2(out, want) < 1e-4
    # m = 48 runs four sub-steps; the estimate is their sum
    out4, dim4, est4 = gop.etd_step_est(y, b, 4 * h, 48, 1e-8)
    assert 0 <= est4 <= 1e-8 and dim4 <= 48  # each sub-step ran to tol / 4
    want4, _ = orc.etd_step(y, b, 4 * h, 60, 0.0)
    assert rel_l2(out4, want4) < 1e-4
    # a space far too small for the step reports an estimate above tol
    _, dim2, est2 = gop.etd_step_est(y, b, 20.0 * h, 4, 1e-8)
    assert est2 > 1e-8 and dim2 == 4


def test_learned_controller_gain(ctx):
    """The MLP, trained on the device on the plain controller's traces of three
    pulses, steers a held-out pulse: every step still passes the Krylov
    estimate, the result matches the plain controller's and the LSERK4
    reference, and it takes fewer Krylov matvecs than the plain controller."""
    import ctypes as C

    from rapidfem_b200 import _native as nat
    from rapidfem_b200 import workloads as W

    op = W.graded_slab(6, 2).build()
    gop = G.GpuOperator(ctx, op)
    rho = C.c_double()
    nat.check(nat.lib.dgtd_power_rho(gop.handle, 40, C.byref(rho)))
    dt_cfl = 2.8 / rho.value
    x = op.node_coords()

    def pulse(c):
        y = np.zeros((x.shape[0], 6))
        y[:, 2] = np.exp(-((x - np.array(c)) ** 2).sum(axis=1) / (2 * 0.08 ** 2))
        return y.ravel()

    T = 1.0
    plain = E.PlainEtd(tol=1e-7, m_max=48)
    logs = []
    for c in ([0.3, 0.4, 0.5], [0.6, 0.5, 0.4], [0.5, 0.3, 0.6]):
        E.run_etd(gop, pulse(c), None, None, T, 4 * dt_cfl, plain, log=logs)
    mlp = E.Mlp(ctx, seed=1)
    losses = E.train_controller(mlp, logs, epochs=3000, lr=3e-3)
    assert losses[-1] < 0.05 * losses[0]
    held = [0.45, 0.55, 0.45]
    yp, sp = E.run_etd(gop, pulse(held), None, None, T, 4 * dt_cfl, plain)
    yl, sl = E.run_etd(gop, pulse(held), None, None, T, 4 * dt_cfl, plain, learned=E.LearnedEtd(mlp, plain))
    ref = gop.transient(pulse(held), T, 1, int(np.ceil(T / (0.25 * dt_cfl))), record=False).astype(np.float64)
    assert all(e <= plain.tol for _, _, e in sl.history)
    assert rel_l2(yl, yp) < 1e-5
    assert rel_l2(yl, ref) < 1e-5 and rel_l2(yp, ref) < 1e-5
    gain = sp.matvecs / sl.matvecs
    print(f"learned ETD controller: {sl.matvecs} matvecs in {sl.accepted} steps "
          f"({sl.proposals_kept} proposals kept, {sl.proposals_failed} failed) vs plain {sp.matvecs} in "
          f"{sp.accepted} steps: {gain:.2f}x fewer matvecs")
    assert sl.matvecs < sp.matvecs
