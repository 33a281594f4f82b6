"""Element partition with one halo exchange per stage (the multi-GPU path):
partition invariants, an in-process run of all parts, and a world_size-2 gloo
run on CPU, each against the single-domain oracle.  The oracle stands in for
the device engine of each rank here; tests/test_gpu_partition.py runs the
device engine."""
import os
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as R
from rapidfem_b200 import operator as O
from rapidfem_b200 import partition as PT


class OracleEngine:
    """The per-part compute of a partitioned run on the f64 oracle."""

    def __init__(self, part: PT.Part, order: int):
        self.orc = R.Operator(part.mesh.nodes, part.mesh.tets, order, 1.0, face_port=part.face_port,
                              materials=part.materials)
        for a, b in part.links:
            self.orc.link_periodic(a, b)
        self.bs = 6 * self.orc.np
        self.a, self.b = R.lserk_coeffs()
        self.y = None
        self.p = None
        self._out = None

    def new_buffer(self, n_elem):
        return torch.empty(n_elem * self.bs, dtype=torch.float64)

    def gather(self, ids, buf):
        buf.copy_(torch.from_numpy(self.y.reshape(-1, self.bs)[ids].ravel()))

    def scatter(self, ids, buf):
        self.y.reshape(-1, self.bs)[ids] = buf.numpy().reshape(-1, self.bs)

    def stage(self, h, s):
        k = self.orc.apply(self.y)
        self.p = h * k if s == 0 else self.a[s] * self.p + h * k
        self.y = self.y + self.b[s] * self.p

    def stage_range(self, h, s, e_begin, e_end, flip):
        """The stage on elements [e_begin, e_end) only; the ranges of a stage
        read the same input, the last one (flip) makes the output current."""
        if self._out is None:
            self._out = (self.y.copy(), np.zeros_like(self.y) if self.p is None else self.p.copy())
        y_out, p_out = self._out
        k = self.orc.apply(self.y)
        r = slice(e_begin * self.bs, e_end * self.bs)
        p_out[r] = h * k[r] if s == 0 else self.a[s] * self.p[r] + h * k[r]
        y_out[r] = self.y[r] + self.b[s] * p_out[r]
        if flip:
            self.y, self.p = y_out, p_out
            self._out = None

    def sync(self):
        pass

    def load(self, y):
        self.y = np.array(y, dtype=np.float64)

    def state(self):
        return self.y


def _problem():
    mesh = O.structured_box_jittered(4, 3, 3, 1.0, 0.8, 0.9, 0.1, 7)
    port = np.where(O.boundary_faces_on_plane(mesh, 2, 0.0), 0, -1)
    eps = np.where(mesh.nodes[mesh.tets].mean(axis=1)[:, 0] > 0.5, 4.0, 1.0)
    mat = O.isotropic_materials(eps)
    return mesh, port, mat


def test_parts_are_consistent():
    mesh, port, mat = _problem()
    part = PT.morton_partition(mesh, 3)
    counts = np.bincount(part, minlength=3)
    assert counts.size == 3 and counts.max() - counts.min() <= 1  # equal shares
    parts = PT.build_parts(mesh, part, face_port=port, materials=mat)
    nbr = PT.face_neighbours(mesh.tets)
    assert np.array_equal(np.sort(np.concatenate([p.owned for p in parts])), np.arange(mesh.n_tets))
    for p in parts:
        need = nbr[p.owned].ravel()
        need = np.unique(need[need >= 0])
        assert np.array_equal(np.setdiff1d(need, p.owned), p.halo)
        for q, ids in p.send.items():
            r_ids = parts[q].recv[p.rank]
            assert np.array_equal(p.owned[ids], parts[q].elements[r_ids])
        assert set(p.recv) == {q for q in range(3) if p.rank in parts[q].send}
        # the interior run: whole tiles of elements with no face neighbour elsewhere
        assert p.n_interior % PT.TILE == 0
        inner = nbr[p.owned[:p.n_interior]].ravel()
        assert np.all(np.isin(inner[inner >= 0], p.owned))


def _global_run(mesh, port, mat, order, y0, h, steps):
    orc = R.Operator(mesh.nodes, mesh.tets, order, 1.0, face_port=port, materials=mat)
    return orc.lserk(y0, h, steps), orc


def test_loopback_partition_matches_single_domain():
    mesh, port, mat = _problem()
    order = 2
    orc = R.Operator(mesh.nodes, mesh.tets, order, 1.0, face_port=port, materials=mat)
    y0 = np.sin(0.3 + 0.017 * np.arange(orc.n_dof))
    h = 0.5 / orc.power_rho(30)[0]
    want = orc.lserk(y0, h, 4)
    parts = PT.build_parts(mesh, PT.morton_partition(mesh, 3), face_port=port, materials=mat)
    engines = [OracleEngine(p, order) for p in parts]
    for e, yl in zip(engines, PT.split_state(parts, y0, orc.np)):
        e.load(yl)
    PT.LoopbackLserk(parts, engines).step(h, 4)
    got = PT.join_state(parts, [e.state() for e in engines], orc.np)
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))


def _rank_main(rank, world, port_no, tmp):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port_no}", rank=rank, world_size=world)
    try:
        mesh, port, mat = _problem()
        order = 2
        parts = PT.build_parts(mesh, PT.morton_partition(mesh, world), face_port=port, materials=mat)
        me = parts[rank]
        eng = OracleEngine(me, order)
        n = 6 * eng.orc.np * mesh.n_tets
        y0 = np.sin(0.3 + 0.017 * np.arange(n))
        eng.load(PT.split_state(parts, y0, eng.orc.np)[rank])
        h = float(np.load(os.path.join(tmp, "h.npy")))
        PT.ShardedLserk(me, eng, PT.TorchTransport()).step(h, 3)
        np.save(os.path.join(tmp, f"y{rank}.npy"), eng.state())
    finally:
        dist.destroy_process_group()


def test_gloo_world2_matches_single_domain():
    mesh, port, mat = _problem()
    order = 2
    orc = R.Operator(mesh.nodes, mesh.tets, order, 1.0, face_port=port, materials=mat)
    y0 = np.sin(0.3 + 0.017 * np.arange(orc.n_dof))
    h = 0.5 / orc.power_rho(30)[0]
    want = orc.lserk(y0, h, 3)
    with tempfile.TemporaryDirectory() as tmp:
        np.save(os.path.join(tmp, "h.npy"), np.array(h))
        port_no = 29500 + (os.getpid() % 2000)
        mp.spawn(_rank_main, args=(2, port_no, tmp), nprocs=2, join=True)
        parts = PT.build_parts(mesh, PT.morton_partition(mesh, 2), face_port=port, materials=mat)
        got = PT.join_state(parts, [np.load(os.path.join(tmp, f"y{r}.npy")) for r in range(2)], orc.np)
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))


def test_loopback_split_stages_match_single_domain():
    """Each stage as [interior elements | halo scatter | boundary and halo
    elements], the order of an overlapped sharded run."""
    mesh = O.structured_box_jittered(6, 5, 4, 1.0, 0.8, 0.9, 0.1, 9)
    order = 2
    orc = R.Operator(mesh.nodes, mesh.tets, order, 1.0)
    y0 = np.sin(0.3 + 0.017 * np.arange(orc.n_dof))
    h = 0.5 / orc.power_rho(30)[0]
    want = orc.lserk(y0, h, 3)
    parts = PT.build_parts(mesh, PT.morton_partition(mesh, 2))
    assert all(p.n_interior >= 2 * PT.TILE for p in parts)
    engines = [OracleEngine(p, order) for p in parts]
    for e, yl in zip(engines, PT.split_state(parts, y0, orc.np)):
        e.load(yl)
    PT.LoopbackLserk(parts, engines, split=True).step(h, 3)
    got = PT.join_state(parts, [e.state() for e in engines], orc.np)
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))


@pytest.mark.parametrize("n_parts", [1, 8])
def test_loopback_one_and_many_parts(n_parts):
    # one part: no halo and no exchange at all; eight parts of ~27 tets: most
    # elements sit on a cut, so every part exchanges with several peers
    mesh, port, mat = _problem()
    order = 2
    orc = R.Operator(mesh.nodes, mesh.tets, order, 1.0, face_port=port, materials=mat)
    y0 = np.sin(0.3 + 0.017 * np.arange(orc.n_dof))
    h = 0.5 / orc.power_rho(30)[0]
    want = orc.lserk(y0, h, 3)
    parts = PT.build_parts(mesh, PT.morton_partition(mesh, n_parts), face_port=port, materials=mat)
    assert len(parts) == n_parts
    if n_parts == 1:
        assert parts[0].halo.size == 0 and not parts[0].send and not parts[0].recv
    else:
        assert all(len(p.send) >= 2 for p in parts)
    engines = [OracleEngine(p, order) for p in parts]
    for e, yl in zip(engines, PT.split_state(parts, y0, orc.np)):
        e.load(yl)
    PT.LoopbackLserk(parts, engines).step(h, 3)
    got = PT.join_state(parts, [e.state() for e in engines], orc.np)
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))


def test_partition_rejects_bad_part_count():
    mesh, _, _ = _problem()
    with pytest.raises(ValueError):
        PT.morton_partition(mesh, 0)


class CpuVecEngine:
    """Vectors and partial sums of a partitioned Krylov run as CPU tensors,
    addressed by their data pointers as the device hooks address device
    memory: the host side of ShardedKrylov without a device."""

    class _Gop:
        def __init__(self):
            self.n_owned, self.hooks = 0, None

        def set_partition(self, n_owned, halo=None, reduce=None):
            self.n_owned, self.hooks = n_owned, (halo, reduce)

    def __init__(self, bs):
        self.bs = bs
        self.reg = {}
        self.gop = self._Gop()

    def register(self, t):
        self.reg[t.data_ptr()] = t
        return t.data_ptr()

    def new_buffer(self, n_elem):
        return torch.empty(n_elem * self.bs, dtype=torch.float64)

    def gather_vec(self, d_vec, ids, buf):
        buf.copy_(self.reg[d_vec].view(-1, self.bs)[torch.from_numpy(ids)].reshape(-1))

    def scatter_vec(self, d_vec, ids, buf):
        self.reg[d_vec].view(-1, self.bs)[torch.from_numpy(ids)] = buf.view(-1, self.bs)

    def view_f64(self, d_buf, count):
        return self.reg[d_buf][:count]

    def reduce_context(self):
        import contextlib

        return contextlib.nullcontext()


def _krylov_rank_main(rank, world, port_no, tmp):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port_no}", rank=rank, world_size=world)
    try:
        mesh, port, mat = _problem()
        parts = PT.build_parts(mesh, PT.morton_partition(mesh, world), face_port=port, materials=mat)
        me = parts[rank]
        bs = 6 * 10  # order 2
        eng = CpuVecEngine(bs)
        sk = PT.ShardedKrylov(me, eng, PT.TorchTransport())
        assert eng.gop.n_owned == me.n_owned
        # a Krylov vector: owned blocks hold the global vector, halo blocks are stale
        g = np.sin(0.3 + 0.017 * np.arange(mesh.n_tets * bs))
        v = torch.from_numpy(PT.split_state(parts, g, 10)[rank].copy())
        v.view(-1, bs)[me.n_owned:] = float("nan")
        halo, reduce = eng.gop.hooks
        halo(eng.register(v))
        # partial sums: each part's own, summed over the parts in place
        part_sums = torch.arange(16, dtype=torch.float64) * (rank + 1)
        reduce(eng.register(part_sums), 12)
        np.save(os.path.join(tmp, f"v{rank}.npy"), v.numpy())
        np.save(os.path.join(tmp, f"s{rank}.npy"), part_sums.numpy())
        sk.close()
        assert eng.gop.n_owned == 0
    finally:
        dist.destroy_process_group()


def test_gloo_world2_krylov_hooks():
    """The host side of the partitioned Krylov path on two gloo ranks: the halo
    hook refreshes a vector's halo blocks from the peer's owned blocks, the
    sum hook all-reduces the partial sums in place (only `count` values)."""
    mesh, port, mat = _problem()
    bs = 60
    g = np.sin(0.3 + 0.017 * np.arange(mesh.n_tets * bs))
    with tempfile.TemporaryDirectory() as tmp:
        port_no = 29500 + ((os.getpid() + 7) % 2000)
        mp.spawn(_krylov_rank_main, args=(2, port_no, tmp), nprocs=2, join=True)
        parts = PT.build_parts(mesh, PT.morton_partition(mesh, 2), face_port=port, materials=mat)
        for r, p in enumerate(parts):
            v = np.load(os.path.join(tmp, f"v{r}.npy")).reshape(-1, bs)
            assert np.array_equal(v, g.reshape(-1, bs)[p.elements])
            s = np.load(os.path.join(tmp, f"s{r}.npy"))
            assert np.array_equal(s[:12], np.arange(12) * 3.0) and np.array_equal(s[12:], np.arange(12, 16) * (r + 1))


def test_local_dof():
    mesh, port, mat = _problem()
    parts = PT.build_parts(mesh, PT.morton_partition(mesh, 3))
    bs = 6 * 4  # order 1
    for dof in (0, 7 * bs + 5, (mesh.n_tets - 1) * bs + 23):
        hits = [PT.local_dof(p, 4, dof) for p in parts]
        assert sum(h >= 0 for h in hits) == 1
        r = next(i for i, h in enumerate(hits) if h >= 0)
        assert parts[r].elements[hits[r] // bs] == dof // bs and hits[r] % bs == dof % bs


def test_loopback_periodic_partition_matches_single_domain():
    """A box periodic in x and z, split in three: the periodic links join the
    neighbour relation (halo elements across the period), each part links the
    pairs it holds both sides of, and the run matches the undivided one."""
    from rapidfem_b200 import model as M

    tm = M.box_tagged(6, 2, 4, 1.0, 0.5, 0.8)
    pairs = M.periodic_faces_of(tm, M.Model(periodic=[(1, 2), (5, 6)]))
    order = 2
    glob = M.operator_from_model(tm, M.Model(periodic=[(1, 2), (5, 6)]), order).op
    links = PT.periodic_links(glob, pairs)
    orc = R.Operator(tm.mesh.nodes, tm.mesh.tets, order, 1.0)
    for a, b in links:
        orc.link_periodic(a, b)
    y0 = np.sin(0.3 + 0.017 * np.arange(orc.n_dof))
    h = 0.5 / orc.power_rho(30)[0]
    want = orc.lserk(y0, h, 3)
    parts = PT.build_parts(tm.mesh, PT.morton_partition(tm.mesh, 3), links=links)
    assert any(p.links for p in parts)
    for p in parts:
        # halo: every face neighbour, across the period too
        nbr = PT.face_neighbours(tm.mesh.tets).reshape(-1)
        for a, b in links:
            nbr[a], nbr[b] = b // 4, a // 4
        need = nbr.reshape(-1, 4)[p.owned].ravel()
        assert np.array_equal(np.setdiff1d(np.unique(need[need >= 0]), p.owned), p.halo)
        # the host build links what the oracle links
        eng_nbr = p.operator(order).get("nbr")
        loc = R.Operator(p.mesh.nodes, p.mesh.tets, order, 1.0)
        for a, b in p.links:
            loc.link_periodic(a, b)
        assert np.array_equal(eng_nbr, loc.get("nbr"))
    engines = [OracleEngine(p, order) for p in parts]
    for e, yl in zip(engines, PT.split_state(parts, y0, orc.np)):
        e.load(yl)
    PT.LoopbackLserk(parts, engines).step(h, 3)
    got = PT.join_state(parts, [e.state() for e in engines], orc.np)
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))
