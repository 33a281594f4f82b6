"""Element partition of the DGTD path across ranks, with one halo exchange per
RHS stage.

The RHS of an element reads its own state and the face traces of its four face
neighbours (rhs.rs:1370-1441), so a run split by elements needs, before every
stage, the current state of the neighbour elements that other ranks own.  Each
rank holds a local operator over its owned elements followed by its halo
elements (the face neighbours it does not own); the local build makes the
halo's outer faces boundary faces, which only changes halo rows, and those are
overwritten by the next exchange.  The exchange moves whole element blocks
(6*Np values, contiguous in both the AoS boundary layout and the device SoA
layout).

Pieces:
  * morton_partition / build_parts: the partition and the per-rank pieces
    (local mesh, face ports, materials, send and receive lists per peer);
  * ShardedLserk: LSERK4 steps as [exchange, fused stage] x 5 per step over an
    engine (GpuEngine: the device operator; any object with the same methods)
    and a transport (TorchTransport: torch.distributed point-to-point, NCCL on
    GPUs, gloo on CPUs);
  * LoopbackLserk: all parts in one process, exchanges as device copies.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .operator import Mesh


def face_neighbours(tets: np.ndarray) -> np.ndarray:
    """nbr[K, 4]: the element across local face f (faces opposite vertex 3, 1,
    2, 0 in the TET_FACE_LOCAL order of core/mesh.rs:45-50), -1 on the boundary.
    Matching is by the sorted vertex triple of the face."""
    tets = np.asarray(tets, dtype=np.int64)
    K = tets.shape[0]
    local = np.array([[0, 1, 2], [0, 2, 3], [0, 3, 1], [1, 2, 3]])
    faces = np.sort(tets[:, local].reshape(-1, 3), axis=1)  # [4K, 3]
    order = np.lexsort((faces[:, 2], faces[:, 1], faces[:, 0]))
    fs = faces[order]
    same = np.all(fs[1:] == fs[:-1], axis=1)
    nbr = -np.ones(4 * K, dtype=np.int64)
    a, b = order[:-1][same], order[1:][same]
    nbr[a] = b // 4
    nbr[b] = a // 4
    return nbr.reshape(K, 4)


def _morton_key(xyz: np.ndarray, bits: int = 21) -> np.ndarray:
    lo, hi = xyz.min(axis=0), xyz.max(axis=0)
    span = np.where(hi > lo, hi - lo, 1.0)
    q = np.minimum(((xyz - lo) / span * ((1 << bits) - 1)).astype(np.uint64), (1 << bits) - 1)
    key = np.zeros(xyz.shape[0], dtype=np.uint64)
    for b in range(bits):
        for ax in range(3):
            key |= ((q[:, ax] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + ax)
    return key


def morton_partition(mesh: Mesh, n_parts: int) -> np.ndarray:
    """part[K]: contiguous runs of the Morton order of the element centroids,
    as equal in size as possible (a space-filling-curve partition)."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    cen = mesh.nodes[np.asarray(mesh.tets, dtype=np.int64)].mean(axis=1)
    order = np.argsort(_morton_key(cen), kind="stable")
    part = np.empty(mesh.n_tets, dtype=np.int32)
    bounds = np.linspace(0, mesh.n_tets, n_parts + 1).round().astype(np.int64)
    for r in range(n_parts):
        part[order[bounds[r]:bounds[r + 1]]] = r
    return part


TILE = 40  # a whole number of tensor-core tiles (20 elements, 8 at order 5): stage ranges start on one


@dataclass
class Part:
    """One rank's piece: local element k < n_owned is owned[k], local element
    n_owned + j is halo[j] (global ids).  The owned elements come in two runs:
    the first n_interior (a multiple of TILE) have no face neighbour in the
    halo, so their stage update needs no exchange and can overlap it; the
    rest (and the halo rows, whose updates are discarded) follow once the
    halo has arrived."""

    rank: int
    owned: np.ndarray
    halo: np.ndarray
    mesh: Mesh
    face_port: np.ndarray | None
    materials: np.ndarray | None
    send: dict = field(default_factory=dict)  # peer -> local ids of owned elements to send
    recv: dict = field(default_factory=dict)  # peer -> local ids of halo slots to fill
    n_interior: int = 0
    links: list = field(default_factory=list)  # periodic face pairs between local elements, local face ids

    def operator(self, order: int, flux_alpha: float = 1.0):
        """The part's host operator (MaxwellOperator over the local mesh, face
        codes and materials) with its periodic links applied."""
        from .operator import MaxwellOperator

        op = MaxwellOperator(self.mesh, order, flux_alpha, face_port=self.face_port, materials=self.materials)
        for a, b in self.links:
            op.link_periodic(a, b)
        return op

    @property
    def n_owned(self) -> int:
        return int(self.owned.size)

    @property
    def n_local(self) -> int:
        return int(self.owned.size + self.halo.size)

    @property
    def elements(self) -> np.ndarray:
        return np.concatenate([self.owned, self.halo])


def periodic_links(op, pairs) -> list:
    """The face pairs of periodic links as linked in a global host operator:
    for each (faces_a, faces_b) of `pairs` (face ids e*4 + local face, as
    model.periodic_faces_of gives them), (faces_a, the partner of each)."""
    nbr = op.get("nbr").astype(np.int64)
    lf = op.get("nbr_lf").astype(np.int64)
    out = []
    for a, _ in pairs:
        a = np.asarray(a, dtype=np.int64)
        if np.any(nbr[a] < 0):
            raise ValueError("a periodic face of the pair is not linked in the operator")
        out.append((a, nbr[a] * 4 + lf[a]))
    return out


def build_parts(mesh: Mesh, part: np.ndarray, face_port=None, materials=None, links=None) -> list[Part]:
    """The per-rank pieces of a partition `part[K]` (rank ids 0..R-1).  Owned
    elements are ordered interior first (no face neighbour owned elsewhere;
    the interior run is cut to a multiple of TILE, the cut-off interior
    elements join the boundary run), each run in ascending global id.  Send
    and receive lists of a pair of ranks list the same global elements in the
    same (ascending global id) order.  `links` (periodic_links) adds the
    periodic face pairs to the neighbour relation; each part keeps, in
    Part.links, the pairs whose two elements are both local, in local face
    ids (Part.operator applies them).  A halo element's link to an element
    that is not local stays a boundary face, which only changes halo rows."""
    part = np.asarray(part, dtype=np.int64)
    K = mesh.n_tets
    if part.shape != (K,):
        raise ValueError("part must have one rank id per element")
    R = int(part.max()) + 1
    nbr = face_neighbours(mesh.tets)
    links = [(np.asarray(a, dtype=np.int64), np.asarray(b, dtype=np.int64)) for a, b in (links or [])]
    for a, b in links:
        if a.shape != b.shape:
            raise ValueError("periodic link sides differ in length")
        flat = nbr.reshape(-1)
        flat[a] = b // 4
        flat[b] = a // 4
    tets = np.asarray(mesh.tets, dtype=np.int64)
    fp = None if face_port is None else np.asarray(face_port, dtype=np.int32).reshape(K, 4)
    mat = None if materials is None else np.asarray(materials, dtype=np.float64).reshape(K, -1)
    # an element is on the cut if a face neighbour belongs to another rank
    nbr_part = np.where(nbr >= 0, part[np.maximum(nbr, 0)], -1)
    on_cut = np.any((nbr >= 0) & (nbr_part != part[:, None]), axis=1)
    parts = []
    for r in range(R):
        mine = np.flatnonzero(part == r)
        inner = mine[~on_cut[mine]]
        n_int = (inner.size // TILE) * TILE
        owned = np.concatenate([inner[:n_int], np.sort(np.concatenate([inner[n_int:], mine[on_cut[mine]]]))])
        nb = nbr[owned].ravel()
        nb = nb[nb >= 0]
        halo = np.unique(nb[part[nb] != r])
        elems = np.concatenate([owned, halo])
        verts, inv = np.unique(tets[elems].ravel(), return_inverse=True)
        local = Mesh(np.ascontiguousarray(mesh.nodes[verts]), inv.reshape(-1, 4).astype(np.int32))
        loc = -np.ones(K, dtype=np.int64)
        loc[elems] = np.arange(elems.size)
        plinks = []
        for a, b in links:
            both = (loc[a // 4] >= 0) & (loc[b // 4] >= 0)
            if np.any(both):
                plinks.append((loc[a[both] // 4] * 4 + a[both] % 4, loc[b[both] // 4] * 4 + b[both] % 4))
        parts.append(Part(r, owned, halo, local, None if fp is None else np.ascontiguousarray(fp[elems]),
                          None if mat is None else np.ascontiguousarray(mat[elems]), n_interior=n_int,
                          links=plinks))
    for r, pr in enumerate(parts):
        elems = pr.elements
        order = np.argsort(elems, kind="stable")
        srt = elems[order]

        def local_ids(glob):  # local index of each global id (all present)
            return order[np.searchsorted(srt, glob)].astype(np.int64)

        for q in range(R):
            if q == r:
                continue
            # elements r owns that q keeps as halo: what r sends to q
            s_glob = parts[q].halo[part[parts[q].halo] == r]
            if s_glob.size:
                pr.send[q] = local_ids(s_glob)
            # elements q owns that r keeps as halo: what r receives from q
            r_glob = pr.halo[part[pr.halo] == q]
            if r_glob.size:
                pr.recv[q] = local_ids(r_glob)
    return parts


def split_state(parts: list[Part], y: np.ndarray, np_: int) -> list[np.ndarray]:
    """The local AoS states of a global AoS state (owned and halo blocks)."""
    bs = 6 * np_
    yb = np.asarray(y).reshape(-1, bs)
    return [np.ascontiguousarray(yb[p.elements].ravel()) for p in parts]


def join_state(parts: list[Part], locals_: list[np.ndarray], np_: int) -> np.ndarray:
    """The global AoS state from the owned blocks of the local states."""
    bs = 6 * np_
    K = sum(p.n_owned for p in parts)
    out = np.empty((K, bs), dtype=np.asarray(locals_[0]).dtype)
    for p, y in zip(parts, locals_):
        out[p.owned] = np.asarray(y).reshape(-1, bs)[: p.n_owned]
    return out.ravel()


class GpuEngine:
    """The device operator of one part, for ShardedLserk / LoopbackLserk.

    The operator's kernels run on one torch CUDA stream (`stream`) that the
    operator's context is bound to; the transport's collectives and the halo
    scatter run on a second stream (`comm_stream`).  The ordering is by
    stream waits, so an exchange needs no host synchronisation:
    `begin_exchange` makes the communication stream wait for the gathers
    queued on the compute stream, and `end_exchange` makes the compute stream
    wait for the scatters.  NCCL point-to-point operations issued under
    `comm()` wait for the work queued on the communication stream, and
    `req.wait()` makes that stream wait for their completion.  Engines whose
    operators share a context (all parts on one device) share its streams:
    the first engine of a context binds them, the others reuse them."""

    def __init__(self, gop, device, stream=None):
        import torch

        self.torch = torch
        self.gop = gop
        self.device = device
        bound = getattr(gop.ctx, "_engine_stream", None)
        if bound is None:
            bound = stream if stream is not None else torch.cuda.Stream(device=device)
            gop.ctx.set_stream(bound.cuda_stream)
            gop.ctx._engine_stream = bound
            gop.ctx._engine_comm_stream = torch.cuda.Stream(device=device)
        elif stream is not None and stream is not bound:
            raise ValueError("engines of one context must share its stream")
        self.stream = bound
        self.comm_stream = gop.ctx._engine_comm_stream
        self.bs = 6 * gop.host_op.np
        self._idx = {}

    def _index(self, ids: np.ndarray):
        hit = self._idx.get(id(ids))
        if hit is None:
            with self.torch.cuda.stream(self.stream):
                t = self.torch.from_numpy(np.ascontiguousarray(ids, dtype=np.int64)).to(self.device)
            self.stream.synchronize()  # the index list is copied before its first use
            hit = (ids, t)
            self._idx[id(ids)] = hit  # the list stays referenced, so its id is not reused
        return hit[1]

    def new_buffer(self, n_elem: int):
        with self.torch.cuda.stream(self.stream):
            return self.torch.empty(n_elem * self.bs, dtype=self.torch.float32, device=self.device)

    def comm(self):
        """Context in which the transport issues its operations (the communication stream)."""
        return self.torch.cuda.stream(self.comm_stream)

    def begin_exchange(self) -> None:
        """The communication stream waits for what the compute stream queued (the gathers)."""
        self.comm_stream.wait_stream(self.stream)

    def end_exchange(self) -> None:
        """The compute stream waits for the communication stream (received and scattered halo)."""
        self.stream.wait_stream(self.comm_stream)

    def gather(self, ids: np.ndarray, buf) -> None:
        self.gop.gather_elements(self._index(ids).data_ptr(), ids.size, buf.data_ptr())

    def scatter(self, ids: np.ndarray, buf) -> None:
        """Received blocks into the halo rows, on the communication stream."""
        ctx = self.gop.ctx
        ctx.set_stream(self.comm_stream.cuda_stream)
        try:
            self.gop.scatter_elements(self._index(ids).data_ptr(), ids.size, buf.data_ptr())
        finally:
            ctx.set_stream(self.stream.cuda_stream)

    def gather_vec(self, d_vec: int, ids: np.ndarray, buf) -> None:
        """Element blocks of a device vector (a Krylov basis vector) into `buf`."""
        self.gop.gather_vec_elements(d_vec, self._index(ids).data_ptr(), ids.size, buf.data_ptr())

    def scatter_vec(self, d_vec: int, ids: np.ndarray, buf) -> None:
        """Received blocks into a device vector's halo rows, on the communication stream."""
        ctx = self.gop.ctx
        ctx.set_stream(self.comm_stream.cuda_stream)
        try:
            self.gop.scatter_vec_elements(d_vec, self._index(ids).data_ptr(), ids.size, buf.data_ptr())
        finally:
            ctx.set_stream(self.stream.cuda_stream)

    def view_f64(self, d_buf: int, count: int):
        """A torch view of `count` f64 values of device memory at `d_buf`."""
        return device_view(self.torch, d_buf, count, "<f8", self.device)

    def reduce_context(self):
        """Context in which a collective on the partial sums is issued (the compute stream)."""
        return self.torch.cuda.stream(self.stream)

    def stage(self, h: float, s: int) -> None:
        self.gop.lserk_stage(h, s)

    def stage_range(self, h: float, s: int, e_begin: int, e_end: int, flip: bool) -> None:
        self.gop.lserk_stage_range(h, s, e_begin, e_end, flip)

    def sync(self) -> None:
        self.stream.synchronize()
        self.comm_stream.synchronize()

    def load(self, y_local) -> None:
        self.gop.upload(np.asarray(y_local, dtype=np.float32))

    def state(self) -> np.ndarray:
        return self.gop.download()


class TorchTransport:
    """Halo exchange over torch.distributed point-to-point operations (NCCL for
    CUDA buffers, gloo for CPU buffers), all pairs in one batch."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group

    def exchange(self, sends: dict, recvs: dict) -> None:
        ops = []
        for q, buf in sends.items():
            ops.append(self.dist.P2POp(self.dist.isend, buf, q, group=self.group))
        for q, buf in recvs.items():
            ops.append(self.dist.P2POp(self.dist.irecv, buf, q, group=self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()


class ShardedLserk:
    """LSERK4 on one part (explicit.rs:100-135 with a halo exchange before each
    RHS).  With `overlap` (and an engine with stage ranges) a stage is
    [gather | exchange + scatter on the communication stream | the interior
    elements' update on the compute stream | wait | the boundary and halo
    elements' update], so the exchange runs under the interior update;
    otherwise [exchange, fused stage]."""

    def __init__(self, part: Part, engine, transport, overlap: bool = True):
        self.part = part
        self.engine = engine
        self.transport = transport
        self.sbuf = {q: engine.new_buffer(ids.size) for q, ids in part.send.items()}
        self.rbuf = {q: engine.new_buffer(ids.size) for q, ids in part.recv.items()}
        self.overlap = bool(overlap) and hasattr(engine, "stage_range") and part.n_interior > 0

    def begin_exchange(self) -> None:
        """Gather the blocks peers need, move them, scatter the received ones.
        A device engine queues the gathers on its compute stream and the rest
        on its communication stream (no host wait); an engine without `comm()`
        works synchronously on the host."""
        for q, ids in self.part.send.items():
            self.engine.gather(ids, self.sbuf[q])
        comm = getattr(self.engine, "comm", None)
        if comm is None:
            self.transport.exchange(self.sbuf, self.rbuf)
        else:
            self.engine.begin_exchange()
            with comm():
                self.transport.exchange(self.sbuf, self.rbuf)
        for q, ids in self.part.recv.items():
            self.engine.scatter(ids, self.rbuf[q])

    def end_exchange(self) -> None:
        if hasattr(self.engine, "end_exchange"):
            self.engine.end_exchange()

    def exchange(self) -> None:
        self.begin_exchange()
        self.end_exchange()

    def step(self, h: float, steps: int = 1) -> None:
        n_int, n_loc = self.part.n_interior, self.part.n_local
        for _ in range(int(steps)):
            for s in range(5):
                if self.overlap:
                    self.begin_exchange()
                    self.engine.stage_range(h, s, 0, n_int, False)
                    self.end_exchange()
                    self.engine.stage_range(h, s, n_int, n_loc, True)
                else:
                    self.exchange()
                    self.engine.stage(h, s)


class LoopbackLserk:
    """All parts of a partition in one process (one device or the CPU): the
    exchange copies each pair's blocks through a buffer of the sender.  With
    `split` (and engines with stage ranges) each stage updates the interior
    elements before the scatter and the rest after it, as an overlapped
    sharded run does."""

    def __init__(self, parts: list[Part], engines: list, split: bool = False):
        self.parts = parts
        self.engines = engines
        self.split = bool(split)
        self.bufs = {(r, q): engines[r].new_buffer(ids.size) for r, p in enumerate(parts) for q, ids in p.send.items()}

    def exchange(self) -> None:
        for r, p in enumerate(self.parts):
            for q, ids in p.send.items():
                self.engines[r].gather(ids, self.bufs[(r, q)])
        for e in self.engines:
            e.sync()
        for r, p in enumerate(self.parts):
            for q, ids in p.recv.items():
                self.engines[r].scatter(ids, self.bufs[(q, r)])
        for e in self.engines:
            e.sync()

    def step(self, h: float, steps: int = 1) -> None:
        for _ in range(int(steps)):
            for s in range(5):
                if not self.split:
                    self.exchange()
                    for e in self.engines:
                        e.stage(h, s)
                    continue
                for r, p in enumerate(self.parts):
                    for q, ids in p.send.items():
                        self.engines[r].gather(ids, self.bufs[(r, q)])
                for e in self.engines:
                    e.sync()
                for e, p in zip(self.engines, self.parts):
                    if p.n_interior > 0:
                        e.stage_range(h, s, 0, p.n_interior, False)
                for r, p in enumerate(self.parts):
                    for q, ids in p.recv.items():
                        self.engines[r].scatter(ids, self.bufs[(q, r)])
                for e in self.engines:
                    e.sync()
                for e, p in zip(self.engines, self.parts):
                    e.stage_range(h, s, p.n_interior, p.n_local, True)


# --------------------------------------------------------------- Krylov / ETD

class _CudaBuffer:
    """Device memory described by the CUDA array interface (no copy)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2}


def device_view(torch, ptr: int, n: int, typestr: str, device):
    """A torch tensor over `n` values of device memory at `ptr` (no copy)."""
    return torch.as_tensor(_CudaBuffer(ptr, n, typestr), device=device)


def local_dof(part: Part, np_: int, dof: int) -> int:
    """The local AoS DOF of the global AoS DOF `dof` ((e*Np + node)*6 + c) on
    this part, or -1 when another part owns element e."""
    bs = 6 * np_
    e, r = divmod(int(dof), bs)
    k = np.flatnonzero(part.owned == e)
    return int(k[0]) * bs + r if k.size else -1


class ShardedKrylov:
    """The Arnoldi process of one part's device operator over a partition
    (dgtd_op_set_partition): before each matvec the Krylov vector's halo blocks
    are exchanged with the peers over the transport (as ShardedLserk exchanges
    the state), and after each partial-sum kernel the f64 partials (the CGS
    dots and norms, at most (m+1) per pass and one norm) are all-reduced, so
    every part forms the same Hessenberg matrix, estimate and step decision.
    The engine's gop then runs dgtd_expmv / dgtd_etd_try (etd.run_etd) as on
    one domain, with the part's local state and source."""

    def __init__(self, part: Part, engine, transport, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.part = part
        self.engine = engine
        self.transport = transport
        self.sbuf = {q: engine.new_buffer(ids.size) for q, ids in part.send.items()}
        self.rbuf = {q: engine.new_buffer(ids.size) for q, ids in part.recv.items()}
        engine.gop.set_partition(part.n_owned, self.halo, self.reduce)

    def halo(self, d_vec: int) -> None:
        for q, ids in self.part.send.items():
            self.engine.gather_vec(d_vec, ids, self.sbuf[q])
        comm = getattr(self.engine, "comm", None)
        if comm is None:
            self.transport.exchange(self.sbuf, self.rbuf)
        else:
            self.engine.begin_exchange()
            with comm():
                self.transport.exchange(self.sbuf, self.rbuf)
        for q, ids in self.part.recv.items():
            self.engine.scatter_vec(d_vec, ids, self.rbuf[q])
        if hasattr(self.engine, "end_exchange"):
            self.engine.end_exchange()

    def reduce(self, d_buf: int, count: int) -> None:
        t = self.engine.view_f64(d_buf, count)
        with self.engine.reduce_context():
            self.dist.all_reduce(t, group=self.group)

    def close(self) -> None:
        self.engine.gop.set_partition(0)


class LoopbackKrylov:
    """All parts of a partition on one device, each part's Krylov / ETD run in
    its own host thread (`run`): the hooks of the parts meet at a barrier, the
    halo blocks of each Krylov vector are copied from the peers' vectors, and
    part 0 sums the parts' partials in a fixed order (all on the shared stream
    of the parts' context, so no host wait is needed between the copies and
    the kernels).  A part whose thread fails breaks the barrier (and every
    wait on it ends after `timeout` seconds), so the other parts fail too."""

    def __init__(self, parts: list[Part], engines: list, timeout: float = 120.0):
        import threading

        self.torch = engines[0].torch
        self.parts = parts
        self.engines = engines
        self.stream = engines[0].stream
        if any(e.stream is not self.stream for e in engines):
            raise ValueError("the parts' operators must share one context (one stream)")
        self.barrier = threading.Barrier(len(parts), timeout=timeout)
        self.slot = [0] * len(parts)
        self.bufs = {(q, r): engines[q].new_buffer(ids.size) for r, p in enumerate(parts) for q, ids in p.recv.items()}
        # index lists on the device before any thread runs
        self.ids = {}
        for r, p in enumerate(parts):
            for q, ids in p.recv.items():
                self.ids[("recv", r, q)] = engines[r]._index(ids)
                self.ids[("send", q, r)] = engines[q]._index(parts[q].send[r])
        for r, (p, e) in enumerate(zip(parts, engines)):
            e.gop.set_partition(p.n_owned, lambda d, r=r: self._halo(r, d),
                                lambda d, c, r=r: self._reduce(r, d, c))

    def _halo(self, r: int, d_vec: int) -> None:
        self.slot[r] = d_vec
        self.barrier.wait()
        for q, ids in self.parts[r].recv.items():
            buf = self.bufs[(q, r)]
            src = self.ids[("send", q, r)]
            self.engines[q].gop.gather_vec_elements(self.slot[q], src.data_ptr(), src.numel(), buf.data_ptr())
            dst = self.ids[("recv", r, q)]
            self.engines[r].gop.scatter_vec_elements(d_vec, dst.data_ptr(), dst.numel(), buf.data_ptr())
        self.barrier.wait()

    def _reduce(self, r: int, d_buf: int, count: int) -> None:
        self.slot[r] = d_buf
        self.barrier.wait()
        if r == 0:
            dev = self.engines[0].device
            with self.torch.cuda.stream(self.stream):
                views = [device_view(self.torch, p, count, "<f8", dev) for p in self.slot]
                total = views[0].clone()
                for v in views[1:]:
                    total += v
                for v in views:
                    v.copy_(total)
        self.barrier.wait()

    def run(self, fn) -> list:
        """fn(r) for every part r, each in its own thread; returns the results
        in part order and re-raises the first failure."""
        import threading

        out, err = [None] * len(self.parts), [None] * len(self.parts)

        def body(r):
            try:
                out[r] = fn(r)
            except BaseException as e:  # noqa: BLE001 - re-raised below
                err[r] = e
                self.barrier.abort()

        ts = [threading.Thread(target=body, args=(r,)) for r in range(len(self.parts))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        def from_barrier(e):  # a part stopped because another part failed
            return isinstance(e, threading.BrokenBarrierError) or \
                isinstance(getattr(e, "__cause__", None), threading.BrokenBarrierError)

        first = next((e for e in err if e is not None and not from_barrier(e)), None)
        first = first or next((e for e in err if e is not None), None)
        if first is not None:
            raise first
        return out

    def close(self) -> None:
        for e in self.engines:
            e.gop.set_partition(0)

