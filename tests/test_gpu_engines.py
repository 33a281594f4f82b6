"""The small-tile FP32 engine (DGTD_ENGINE_FP32_SMALL_TILES) runs the FP32
engine's arithmetic on half as many elements per CTA tile, so every element's
result is the same to the bit: RHS and LSERK4 steps at every order, on a mesh
whose element count is not a multiple of either tile."""
import numpy as np
import pytest

from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200._native import ENGINE_FP32, ENGINE_FP32_SMALL_TILES

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_small_tiles_bit_identical(ctx, order):
    mesh = O.structured_box_jittered(3, 3, 2, 1.0, 1.0, 0.7, 0.1, 11)  # 108 tets
    eps = np.where(mesh.nodes[mesh.tets].mean(axis=1)[:, 0] > 0.5, 3.0, 1.0)
    op = O.MaxwellOperator(mesh, order, 1.0, materials=O.isotropic_materials(eps))
    gop = G.GpuOperator(ctx, op)
    y = np.sin(0.3 + 0.017 * np.arange(op.n_dof)).astype(np.float32)
    out = {}
    for eng in (ENGINE_FP32, ENGINE_FP32_SMALL_TILES):
        gop.set_engine(eng)
        assert gop.engine == eng
        dy = gop.apply(y)
        gop.upload(y)
        gop.run_lserk(1e-3, 3)
        out[eng] = (dy, gop.download())
    assert np.array_equal(out[ENGINE_FP32][0], out[ENGINE_FP32_SMALL_TILES][0])
    assert np.array_equal(out[ENGINE_FP32][1], out[ENGINE_FP32_SMALL_TILES][1])
