"""tcgen05 building blocks: a one-CTA GEMM through the tensor-core RHS kernel's
operand layout, descriptors and TMEM path (A from shared memory or from TMEM),
against numpy in f64."""
import numpy as np
import pytest

from rapidfem_b200 import _native
from rapidfem_b200 import gpu as G

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("a_tmem", [0, 2], ids=["a_smem", "a_tmem"])
@pytest.mark.parametrize("n,k", [(16, 8), (32, 16), (112, 40), (48, 64), (176, 56), (256, 64)])
def test_tc_gemm_3xtf32(n, k, a_tmem):
    ctx = G.GpuContext(0)
    rng = np.random.default_rng(n * 100 + k)
    a = rng.normal(size=(128, k)).astype(np.float32)
    b = rng.normal(size=(n, k)).astype(np.float32)
    c = np.zeros((128, n), dtype=np.float32)
    _native.check(_native.lib.dgtd_debug_tc_gemm(ctx.handle, a.ravel(), b.ravel(), c.ravel(), n, k, 1 | a_tmem))
    want = a.astype(np.float64) @ b.astype(np.float64).T
    assert rel_l2(c, want) < 2e-6
    c1 = np.zeros((128, n), dtype=np.float32)
    _native.check(_native.lib.dgtd_debug_tc_gemm(ctx.handle, a.ravel(), b.ravel(), c1.ravel(), n, k, a_tmem))
    e1 = rel_l2(c1, want)
    assert 1e-5 < e1 < 5e-3  # one tf32 product: ~2^-11 relative


@pytest.mark.parametrize("off", [0, 16], ids=["lanes0", "lanes16"])
@pytest.mark.parametrize("a_tmem", [0, 2], ids=["a_smem", "a_tmem"])
@pytest.mark.parametrize("n,k", [(16, 8), (168, 56), (112, 48)])
def test_tc_gemm_m64_lane_layout(n, k, a_tmem, off):
    """64-row MMAs (the order-5 stage kernel's shape): row 16 q + r of the
    accumulator, and of an A operand in TMEM, is TMEM lane 32 q + off + r,
    with the accumulator (and the TMEM A operand) at lane offset off = 0 or 16
    (the kernel's two accumulator sets)."""
    ctx = G.GpuContext(0)
    rng = np.random.default_rng(7 * n + k)
    a = rng.normal(size=(128, k)).astype(np.float32)
    b = rng.normal(size=(n, k)).astype(np.float32)
    c = np.zeros((128, n), dtype=np.float32)
    flags = 1 | a_tmem | 4 | (8 if off else 0)
    _native.check(_native.lib.dgtd_debug_tc_gemm(ctx.handle, a.ravel(), b.ravel(), c.ravel(), n, k, flags))
    want = a[:64].astype(np.float64) @ b.astype(np.float64).T
    lanes = np.array([32 * (r // 16) + off + r % 16 for r in range(64)])
    assert rel_l2(c[lanes], want) < 2e-6
