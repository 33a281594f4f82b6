"""Periodic face pairs on the device: a periodic operator is an ordinary
operator whose linked boundary faces carry a neighbour and a face-node
permutation (rhs.rs:253-270), so every engine runs it unchanged.  The RHS of
a warped, fully periodic box on the FP32, tensor-core and FP64 paths against
the f64 oracle with the same links, and a plane wave crossing a box periodic
in x and z, run through ProblemTD.from_model and against the oracle's run and
the exact travelling wave."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import model as M
from rapidfem_b200 import td as T
from rapidfem_b200._native import ENGINE_FP32, ENGINE_TF32X3

from .conftest import rel_l2
from .test_periodic import _linked, _plane_wave, _tagged

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


@pytest.mark.parametrize("engine", [ENGINE_FP32, ENGINE_TF32X3], ids=["fp32", "tf32x3"])
@pytest.mark.parametrize("order", [3, 4])
def test_periodic_apply_matches_oracle(ctx, engine, order):
    tm = _tagged(3, 2, 4, 1.5, 1.0, 2.0, 0.2)
    op, orc = _linked(tm, order, [(1, 2), (3, 4), (5, 6)])
    gop = G.GpuOperator(ctx, op)
    gop.set_engine(engine)
    y = np.sin(0.3 + 0.017 * np.arange(op.n_dof))
    want = orc.apply(y)
    assert rel_l2(gop.apply(y.astype(np.float32)), want) < 1e-5
    assert rel_l2(gop.apply_f64(y), want) < 1e-12
    # the links change the operator
    walls = R.Operator(tm.mesh.nodes, tm.mesh.tets, order)
    assert rel_l2(walls.apply(y), want) > 1e-2


def test_periodic_plane_wave_device(ctx):
    lx, ly, lz = 1.0, 0.5, 0.5
    tm = _tagged(4, 2, 2, lx, ly, lz)
    pairs = [(1, 2), (5, 6)]
    _, orc = _linked(tm, 3, pairs)
    prob = T.ProblemTD.from_model(tm, M.Model(periodic=pairs), order=3, c=1.0)
    xyz = orc.node_coords()
    t_end, steps = 0.5, 250
    y0 = _plane_wave(xyz, 0.0, lx)
    traj = prob.transient(y0, dt=t_end / steps, steps=steps, method="explicit", verbose=False)
    got = np.asarray(traj)[-1]
    want = orc.lserk(y0, t_end / steps, steps)
    assert rel_l2(got, want) < 1e-4
    assert rel_l2(got, _plane_wave(xyz, t_end, lx)) < 5e-3
    # the FP64 device path follows the oracle to rounding
    gop = G.GpuOperator(ctx, M.operator_from_model(tm, M.Model(periodic=pairs), 3).op)
    assert rel_l2(gop.transient_f64(y0, t_end / steps, steps), want) < 1e-10


def test_periodic_column_passes_plane_wave_device(ctx):
    """The reference's periodic plane-wave test (rhs.rs:3261-3436) with the
    device ETD step (f32 basis, tensor-core matvec): energy within 5e-3,
    forward coherence > 0.85, and > 0.3 above the PEC-walled column."""
    from .test_periodic import _column, _packet, coherence

    lz = 4.0
    op_per, orc = _column(1, 1, 16, 0.5, 0.5, lz, [(1, 2), (3, 4), (5, 6)])
    op_pec, _ = _column(1, 1, 16, 0.5, 0.5, lz, [(1, 2), (3, 4)])
    g_per, g_pec = G.GpuOperator(ctx, op_per), G.GpuOperator(ctx, op_pec)
    y0 = _packet(orc.node_coords(), lz)
    zero = np.zeros_like(y0)
    yp, yc = y0.copy(), y0.copy()
    for _ in range(250):
        yp, _ = g_per.etd_step(yp, zero, 0.04, 24)
        yc, _ = g_pec.etd_step(yc, zero, 0.04, 24)
    e0 = orc.field_energy(y0)
    assert abs(orc.field_energy(yp) - e0) / e0 < 5e-3
    assert coherence(yp) > 0.85 and coherence(yp) - coherence(yc) > 0.3


def test_periodic_box_is_translation_invariant_device(ctx):
    """The reference's translation-invariance test (rhs.rs:3437-3620) with the
    device ETD step on the FP64 path (f64 basis and matvec)."""
    from .test_periodic import _column

    op_all, _ = _column(1, 1, 4, 0.5, 0.5, 1.5, [(1, 2), (3, 4), (5, 6)])
    op_z, _ = _column(1, 1, 4, 0.5, 0.5, 1.5, [(1, 2), (3, 4)])
    g_all, g_z = G.GpuOperator(ctx, op_all), G.GpuOperator(ctx, op_z)
    for g in (g_all, g_z):
        g.set_krylov_precision(64)
    y0 = np.zeros(op_all.n_dof)
    y0[0::6] = 1.0
    zero = np.zeros_like(y0)
    ya, yz = y0.copy(), y0.copy()
    for _ in range(80):
        ya, _ = g_all.etd_step(ya, zero, 0.05, 18)
        yz, _ = g_z.etd_step(yz, zero, 0.05, 18)
    s_all, s_z = float(np.std(ya[0::6])), float(np.std(yz[0::6]))
    assert s_all < 1e-9 and s_z > 100.0 * s_all
