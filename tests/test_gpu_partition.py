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


def _krylov_setup(ctx, n_parts=2):
    mesh = O.structured_box_jittered(6, 5, 4, 1.0, 0.8, 0.7, 0.1, 3)
    order = 3  # 120 DOFs per element: every owned prefix ends on a 16-byte vector
    full = O.MaxwellOperator(mesh, order, 1.0)
    g_full = G.GpuOperator(ctx, full)
    parts = PT.build_parts(mesh, PT.morton_partition(mesh, n_parts))
    dev = torch.device("cuda", 0)
    ctx2 = G.GpuContext(0)  # the parts share this context's stream
    engines = [PT.GpuEngine(G.GpuOperator(ctx2, O.MaxwellOperator(p.mesh, order, 1.0)), dev) for p in parts]
    y0 = np.sin(0.3 + 0.017 * np.arange(full.n_dof))
    dof = full.nearest_node_dof([0.5, 0.4, 0.35], 0, 2)
    return mesh, full, g_full, parts, engines, y0, dof


def test_loopback_krylov_etd_tries_match_single_domain(ctx):
    """dgtd_etd_try over a 2-part partition (one host thread per part, halo
    hooks and all-reduced partial sums) against the undivided op: the same
    Krylov dimensions, the state to f32 rounding of the reordered sums."""
    mesh, full, g_full, parts, engines, y0, dof = _krylov_setup(ctx)
    coef = np.array([1.0, 0.5, -0.2])
    h, m = 0.02, 24
    g_full.upload(y0.astype(np.float32))
    want_dims = []
    for _ in range(3):
        d, _ = g_full.etd_try(h, m, 0.0, coef=coef, drive=("point", dof))
        g_full.etd_commit()
        want_dims.append(d)
    want = g_full.download()
    lk = PT.LoopbackKrylov(parts, engines)
    locs = PT.split_state(parts, y0, full.np)

    def body(r):
        gop = engines[r].gop
        gop.upload(locs[r].astype(np.float32))
        dims = []
        ldof = PT.local_dof(parts[r], full.np, dof)
        for _ in range(3):
            d, _ = gop.etd_try(h, m, 0.0, coef=coef, drive=("point", ldof))
            gop.etd_commit()
            dims.append(d)
        return gop.download(), dims

    res = lk.run(body)
    lk.close()
    assert sum(PT.local_dof(p, full.np, dof) >= 0 for p in parts) == 1
    assert all(dims == want_dims for _, dims in res)
    got = PT.join_state(parts, [y for y, _ in res], full.np)
    assert rel_l2(got, want) < 1e-5


def test_loopback_krylov_etd_run_matches_single_domain(ctx):
    """etd.run_etd with the plain controller on every part (one thread each):
    the parts take the same steps, and the joined state matches the
    undivided run."""
    from rapidfem_b200 import etd as E

    mesh, full, g_full, parts, engines, y0, dof = _krylov_setup(ctx)
    wave = lambda t: np.sin(2 * np.pi * 1.5 * np.asarray(t)) * np.exp(-((np.asarray(t) - 0.3) / 0.15) ** 2)
    plain = E.PlainEtd(tol=1e-7, m_max=36)
    want, st = E.run_etd(g_full, y0, None, wave, 0.3, 0.01, plain, point_dof=dof)
    lk = PT.LoopbackKrylov(parts, engines)
    locs = PT.split_state(parts, y0, full.np)

    def body(r):
        ldof = PT.local_dof(parts[r], full.np, dof)
        return E.run_etd(engines[r].gop, locs[r], None, wave, 0.3, 0.01, plain, point_dof=ldof)

    res = lk.run(body)
    lk.close()
    steps = [s.accepted for _, s in res]
    assert len(set(steps)) == 1 and len({s.matvecs for _, s in res}) == 1
    assert abs(steps[0] - st.accepted) <= 1
    got = PT.join_state(parts, [y for y, _ in res], full.np)
    assert rel_l2(got, want) < 1e-4


def test_loopback_periodic_partition_matches_single_domain(ctx):
    """A box periodic in x and z split in three parts on the device (links
    across the period as halo exchanges) against the undivided periodic run,
    bit-identical on the FP32 engine."""
    from rapidfem_b200 import model as M

    tm = M.box_tagged(6, 2, 4, 1.0, 0.5, 0.8)
    model = M.Model(periodic=[(1, 2), (5, 6)])
    order = 3
    glob = M.operator_from_model(tm, model, order).op
    g_full = G.GpuOperator(ctx, glob)
    g_full.set_engine(ENGINE_FP32)
    y0 = np.sin(0.3 + 0.017 * np.arange(glob.n_dof)).astype(np.float32)
    h = 0.002
    g_full.upload(y0)
    g_full.run_lserk(h, 3)
    want = g_full.download()
    links = PT.periodic_links(glob, M.periodic_faces_of(tm, model))
    parts = PT.build_parts(tm.mesh, PT.morton_partition(tm.mesh, 3), links=links)
    dev = torch.device("cuda", 0)
    ctx2 = G.GpuContext(0)
    engines = []
    for p in parts:
        gop = G.GpuOperator(ctx2, p.operator(order))
        gop.set_engine(ENGINE_FP32)
        engines.append(PT.GpuEngine(gop, dev))
    for e, yl in zip(engines, PT.split_state(parts, y0, glob.np)):
        e.load(yl)
    PT.LoopbackLserk(parts, engines).step(h, 3)
    got = PT.join_state(parts, [e.state() for e in engines], glob.np)
    assert np.array_equal(got, want)


def test_loopback_krylov_vector_source_on_periodic_box(ctx):
    """Partitioned ETD tries with a vector source on a box periodic in x and z
    (links across the period as halo blocks of the Krylov vectors) against the
    undivided op."""
    from rapidfem_b200 import model as M

    tm = M.box_tagged(6, 2, 4, 1.0, 0.5, 0.8)
    model = M.Model(periodic=[(1, 2), (5, 6)])
    order = 3
    glob = M.operator_from_model(tm, model, order).op
    g_full = G.GpuOperator(ctx, glob)
    n = glob.n_dof
    y0 = np.sin(0.3 + 0.017 * np.arange(n))
    b = np.cos(0.1 + 0.003 * np.arange(n))
    coef = np.array([0.5, -1.0, 0.25])
    h, m = 0.02, 24
    g_full.set_source_vector(b)
    g_full.upload(y0.astype(np.float32))
    want_dims = []
    for _ in range(2):
        d, _ = g_full.etd_try(h, m, 0.0, coef=coef, drive=("vector", None))
        g_full.etd_commit()
        want_dims.append(d)
    want = g_full.download()
    links = PT.periodic_links(glob, M.periodic_faces_of(tm, model))
    parts = PT.build_parts(tm.mesh, PT.morton_partition(tm.mesh, 2), links=links)
    dev = torch.device("cuda", 0)
    ctx2 = G.GpuContext(0)
    engines = [PT.GpuEngine(G.GpuOperator(ctx2, p.operator(order)), dev) for p in parts]
    lk = PT.LoopbackKrylov(parts, engines)
    ys, bs = PT.split_state(parts, y0, glob.np), PT.split_state(parts, b, glob.np)

    def body(r):
        gop = engines[r].gop
        gop.set_source_vector(bs[r])
        gop.upload(ys[r].astype(np.float32))
        dims = []
        for _ in range(2):
            d, _ = gop.etd_try(h, m, 0.0, coef=coef, drive=("vector", None))
            gop.etd_commit()
            dims.append(d)
        return gop.download(), dims

    res = lk.run(body)
    lk.close()
    assert all(dims == want_dims for _, dims in res)
    got = PT.join_state(parts, [y for y, _ in res], glob.np)
    assert rel_l2(got, want) < 1e-5
