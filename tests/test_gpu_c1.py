"""The plain-DGTD cavity case: the PEC unit cube as 8^3 hexes x 6 tets, N = 3,
vacuum, upwind flux, the analytic TM110 mode as initial field, LSERK4 at
CFL 0.5 (dt = 0.5 * 2.8 / rho(A)) for 1000 steps, on both stage kernels
against the f64 oracle and against the analytic mode."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import workloads as W
from rapidfem_b200._native import ENGINE_FP32, ENGINE_TF32X3

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_tm110_cavity_1000_steps():
    wl = W.cavity_tm110(8, 3)
    op = wl.build()
    nodes, tets = R.box_mesh(8, 8, 8, 1.0, 1.0, 1.0)
    orc = R.Operator(nodes, tets, 3, 1.0)
    R.set_threads(R.threads())
    rho, _ = orc.power_rho(40)
    dt = 0.5 * 2.8 / rho
    steps = 1000
    y0 = wl.y0(op)
    y32 = y0.astype(np.float32).astype(np.float64)
    ref = orc.lserk(y32, dt, steps)
    exact = W.tm110_exact(op, steps * dt)
    ctx = G.GpuContext(0)
    for eng in (ENGINE_FP32, ENGINE_TF32X3):
        gop = G.GpuOperator(ctx, op)
        gop.set_engine(eng)
        gop.upload(y0)
        gop.run_lserk(dt, steps)
        got = gop.download().astype(np.float64)
        assert rel_l2(got, ref) < 1e-4
        assert rel_l2(got, exact) < 1e-2  # the N = 3, h = 1/8 discretisation error of the mode
    assert rel_l2(ref, exact) < 1e-2
