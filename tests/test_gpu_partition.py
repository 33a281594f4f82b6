"""The partitioned path on the device: all parts of a partition on one GPU
(LoopbackLserk over GpuEngine, exchanges as device copies, one fused stage
launch per part and stage) against the undivided run.  Each element's update
depends only on its own and its neighbours' data, so the FP32 engine's result
is the same to the bit; the tensor-core engine to f32 rounding."""
import numpy as np
import pytest
import torch

from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200 import partition as PT
from rapidfem_b200._native import ENGINE_FP32, ENGINE_TF32X3

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


@pytest.mark.parametrize("engine", [ENGINE_FP32, ENGINE_TF32X3], ids=["fp32", "tf32x3"])
def test_loopback_partition_matches_single_domain(ctx, engine):
    mesh = O.structured_box_jittered(6, 5, 4, 1.0, 0.8, 0.7, 0.1, 3)
    port = np.where(O.boundary_faces_on_plane(mesh, 2, 0.0), 0, -1)
    eps = np.where(mesh.nodes[mesh.tets].mean(axis=1)[:, 1] > 0.4, 3.0, 1.0)
    mat = O.isotropic_materials(eps)
    order = 3
    full = O.MaxwellOperator(mesh, order, 1.0, face_port=port, materials=mat)
    g_full = G.GpuOperator(ctx, full)
    g_full.set_engine(engine)
    n = full.n_dof
    y0 = np.sin(0.3 + 0.017 * np.arange(n)).astype(np.float32)
    h = 0.002
    g_full.upload(y0)
    g_full.run_lserk(h, 3)
    want = g_full.download()

    parts = PT.build_parts(mesh, PT.morton_partition(mesh, 3), face_port=port, materials=mat)
    dev = torch.device("cuda", 0)
    engines = []
    for p in parts:
        gop = G.GpuOperator(ctx, O.MaxwellOperator(p.mesh, order, 1.0, face_port=p.face_port,
                                                   materials=p.materials))
        gop.set_engine(engine)
        engines.append(PT.GpuEngine(gop, dev))
    for e, yl in zip(engines, PT.split_state(parts, y0, full.np)):
        e.load(yl)
    PT.LoopbackLserk(parts, engines).step(h, 3)
    got = PT.join_state(parts, [e.state() for e in engines], full.np)
    if engine == ENGINE_FP32:
        assert np.array_equal(got, want)
    else:
        assert rel_l2(got, want) < 1e-6


@pytest.mark.parametrize("engine", [ENGINE_FP32, ENGINE_TF32X3], ids=["fp32", "tf32x3"])
def test_loopback_split_stages_match_single_domain(ctx, engine):
    """Stages split as in an overlapped sharded run: the interior elements'
    update (dgtd_lserk_stage_range on [0, n_interior)) before the halo scatter,
    the boundary and halo elements' after it."""
    mesh = O.structured_box_jittered(8, 6, 5, 1.0, 0.8, 0.7, 0.1, 5)
    order = 3
    full = O.MaxwellOperator(mesh, order, 1.0)
    g_full = G.GpuOperator(ctx, full)
    g_full.set_engine(engine)
    y0 = np.sin(0.3 + 0.017 * np.arange(full.n_dof)).astype(np.float32)
    h = 0.002
    g_full.upload(y0)
    g_full.run_lserk(h, 3)
    want = g_full.download()
    parts = PT.build_parts(mesh, PT.morton_partition(mesh, 3))
    assert all(p.n_interior >= 2 * PT.TILE for p in parts)
    dev = torch.device("cuda", 0)
    ctx2 = G.GpuContext(0)  # the engines bind their own streams to this context
    engines = []
    for p in parts:
        gop = G.GpuOperator(ctx2, O.MaxwellOperator(p.mesh, order, 1.0))
        gop.set_engine(engine)
        engines.append(PT.GpuEngine(gop, dev))
    for e, yl in zip(engines, PT.split_state(parts, y0, full.np)):
        e.load(yl)
    PT.LoopbackLserk(parts, engines, split=True).step(h, 3)
    got = PT.join_state(parts, [e.state() for e in engines], full.np)
    if engine == ENGINE_FP32:
        assert np.array_equal(got, want)
    else:
        assert rel_l2(got, want) < 1e-6


def test_stage_range_arguments(ctx):
    op = O.MaxwellOperator(O.structured_box(3, 3, 3), 2, 1.0)  # 162 elements
    gop = G.GpuOperator(ctx, op)
    from rapidfem_b200._native import DgtdError
    for b, e in ((10, 40), (0, 150), (40, 20), (0, 200)):
        with pytest.raises(DgtdError):
            gop.lserk_stage_range(1e-3, 0, b, e, False)
    gop.lserk_stage_range(1e-3, 0, 0, 160, False)
    gop.lserk_stage_range(1e-3, 0, 160, 162, True)
