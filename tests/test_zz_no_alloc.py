"""The no-allocation LSERK4 entry point against the allocating one.

`dgtd_run_lserk_static` is for callers that cannot let the library call
cudaMalloc -- hosts whose framework owns the device memory budget.  Its scratch
is a file-scope device array shared by every call, so this test checks two
calls in a row (the second starts from the first's output, over scratch the
first call left behind) against `dgtd_transient`, which allocates its own
buffers, within the transient tolerance of the parity tests.  The file is named
to be collected last.
"""
import ctypes

import numpy as np
import pytest

from rapidfem_b200 import _native
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O

from .conftest import rel_l2

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-4
STATIC_MAX_DOF = 1 << 21


def _static(gop, d_in, d_out, h, steps):
    lib = ctypes.CDLL(_native.LIB_PATH)
    lib.dgtd_run_lserk_static.restype = ctypes.c_int
    lib.dgtd_run_lserk_static.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_float, ctypes.c_int64]
    return lib.dgtd_run_lserk_static(gop.handle, d_in, d_out, h, steps)


@pytest.mark.parametrize("cells,engine", [((5, 4, 4), None), ((3, 3, 3), _native.ENGINE_FP32),
                                          ((3, 3, 3), _native.ENGINE_TF32X3)],
                         ids=["whole-tiles", "padded-fp32", "padded-tf32x3"])
def test_static_lserk_matches_allocating_entry_point_twice(cells, engine):
    """(5,4,4): 480 tets, whole 20-element tiles.  (3,3,3): 162 tets, so the
    last tile is padded and the call clears the padding of its scratch."""
    import torch

    ctx = G.GpuContext(0)
    op = O.MaxwellOperator(O.structured_box(*cells), 3, 1.0)
    gop = G.GpuOperator(ctx, op)
    if engine is not None:
        gop.set_engine(engine)
    n = gop.n_dof()
    assert n <= STATIC_MAX_DOF
    y0 = np.sin(0.3 + 0.017 * np.arange(n)).astype(np.float32)
    h, steps = 2e-3, 7

    want1 = gop.transient(y0, h, steps, 1)
    want2 = gop.transient(want1, h, steps, 1)

    dev = torch.device("cuda", 0)
    d_in = torch.from_numpy(y0).to(dev)
    d_mid = torch.empty(n, device=dev, dtype=torch.float32)
    d_out = torch.empty(n, device=dev, dtype=torch.float32)
    torch.cuda.synchronize()
    _native.check(_static(gop, d_in.data_ptr(), d_mid.data_ptr(), h, steps))
    ctx.synchronize()
    gop.check_error()  # no bounded wait of the run gave up
    got1 = d_mid.cpu().numpy()
    _native.check(_static(gop, d_mid.data_ptr(), d_out.data_ptr(), h, steps))
    ctx.synchronize()
    gop.check_error()
    got2 = d_out.cpu().numpy()

    assert rel_l2(got1, want1) < RUN_TOL
    assert rel_l2(got2, want2) < RUN_TOL


def test_static_lserk_rejects_sizes_above_its_scratch():
    import torch

    ctx = G.GpuContext(0)
    op = O.MaxwellOperator(O.structured_box(15, 15, 15), 3, 1.0)
    assert op.n_dof > STATIC_MAX_DOF
    gop = G.GpuOperator(ctx, op)
    d = torch.zeros(8, device="cuda", dtype=torch.float32)
    st = _static(gop, d.data_ptr(), d.data_ptr(), 1e-3, 1)
    assert st == 1
    assert "static scratch limit" in _native.last_error()
