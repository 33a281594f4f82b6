"""The reference's LSERK4 tests (explicit.rs:173-313) on the device FP64
path: one step agrees with the exponential propagator (f64 Krylov) to 1e-9,
free and driven by a point or a vector source, and the scheme is stable at
2 / rho and diverges at 12 / rho."""
import ctypes as C

import numpy as np
import pytest

from rapidfem_b200 import _native as nat
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cube():
    """explicit.rs:178-180: the 2^3 unit cube, N = 2, upwind."""
    op = O.MaxwellOperator(O.structured_box(2, 2, 2), 2, 1.0)
    gop = G.GpuOperator(G.GpuContext(0), op)
    gop.set_krylov_precision(64)
    return op, gop


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_lserk4_matches_the_exponential_propagator_below_cfl(cube):
    op, gop = cube
    y0 = np.sin(0.3 + 0.017 * np.arange(op.n_dof))
    rk = gop.transient_f64(y0, 1e-3, 1)
    ex, _ = gop.expmv(y0, 1e-3, 40)
    assert rel(rk, ex) < 1e-9


def test_lserk4_driven_matches_etd_below_cfl(cube):
    op, gop = cube
    n = op.n_dof
    y0 = np.sin(0.2 + 0.019 * np.arange(n))
    sdof = n // 3
    point = np.zeros(n)
    point[sdof] = 0.7
    spread = 0.4 * np.cos(0.11 * np.arange(n))
    for drive, g, b in ((("point", sdof), [0.7], point), (("vector", spread), [1.0], spread)):
        rk = gop.transient_f64(y0, 1e-3, 1, drive=drive, g=g)
        etd, _ = gop.etd_step(y0, b, 1e-3, 40)
        assert rel(rk, etd) < 1e-9, drive[0]


def test_lserk4_is_stable_below_cfl_and_diverges_above(cube):
    op, gop = cube
    rho = C.c_double()
    nat.check(nat.lib.dgtd_power_rho(gop.handle, 60, C.byref(rho)))
    y0 = np.cos(0.05 * np.arange(op.n_dof))
    stable = np.linalg.norm(gop.transient_f64(y0, 2.0 / rho.value, 400))
    assert np.isfinite(stable) and stable < 1e3
    unstable = np.linalg.norm(gop.transient_f64(y0, 12.0 / rho.value, 400))
    assert not np.isfinite(unstable) or unstable > 1e6
