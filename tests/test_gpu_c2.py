"""The C2 workload at its full size (48^3 x 6 jittered sphere_pulse box,
663,552 tets, N = 4, 139 M DOFs): the FP32 and tensor-core LSERK4 engines
against the FP64 device path run from the same f32 state (the reference at a
size the CPU oracle cannot reach; the FP64 path itself is pinned to the f64
oracle in tests/test_gpu_fp64.py), and a size-independent property: with
upwind flux and PEC walls the discrete field energy does not grow."""
import ctypes as C

import numpy as np
import pytest

from rapidfem_b200 import _native as nat
from rapidfem_b200 import gpu as G
from rapidfem_b200 import workloads as W
from rapidfem_b200._native import ENGINE_FP32, ENGINE_TF32X3

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


def _energy(gop, y):
    e = C.c_double()
    nat.check(nat.lib.dgtd_field_energy(gop.handle, np.ascontiguousarray(y, dtype=np.float64), C.byref(e)))
    return e.value


def test_c2_full_size_against_fp64():
    ctx = G.GpuContext(0)
    wl = W.sphere_pulse(48, 4)
    op = wl.build()
    assert op.n_dof == 139_345_920
    gop = G.GpuOperator(ctx, op)
    y0 = wl.y0(op).astype(np.float32)
    rho = C.c_double()
    nat.check(nat.lib.dgtd_power_rho(gop.handle, 20, C.byref(rho)))
    dt = 0.5 * 2.8 / rho.value
    steps = 200
    ref = gop.transient_f64(y0.astype(np.float64), dt, steps)
    e0, e_ref = _energy(gop, y0), _energy(gop, ref)
    assert 0.0 < e_ref <= e0 * (1 + 1e-9)
    for engine in (ENGINE_FP32, ENGINE_TF32X3):
        gop.set_engine(engine)
        gop.upload(y0)
        gop.run_lserk(dt, steps)
        got = gop.download()
        assert rel_l2(got, ref) < 1e-5
        assert _energy(gop, got) <= e0 * (1 + 1e-6)
