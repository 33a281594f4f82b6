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


@dataclass
class Part:
    """One rank's piece: local element k < n_owned is owned[k], local element
    n_owned + j is halo[j] (global ids)."""

    rank: int
    owned: np.ndarray
    halo: np.ndarray
    mesh: Mesh
    face_port: np.ndarray | None
    materials: np.ndarray | None
    send: dict = field(default_factory=dict)  # peer -> local ids of owned elements to send
    recv: dict = field(default_factory=dict)  # peer -> local ids of halo slots to fill

    @property
    def n_owned(self) -> int:
        return int(self.owned.size)

    @property
    def n_local(self) -> int:
        return int(self.owned.size + self.halo.size)

    @property
    def elements(self) -> np.ndarray:
        return np.concatenate([self.owned, self.halo])


def build_parts(mesh: Mesh, part: np.ndarray, face_port=None, materials=None) -> list[Part]:
    """The per-rank pieces of a partition `part[K]` (rank ids 0..R-1).  Send and
    receive lists of a pair of ranks list the same global elements in the same
    (ascending global id) order."""
    part = np.asarray(part, dtype=np.int64)
    K = mesh.n_tets
    if part.shape != (K,):
        raise ValueError("part must have one rank id per element")
    R = int(part.max()) + 1
    nbr = face_neighbours(mesh.tets)
    tets = np.asarray(mesh.tets, dtype=np.int64)
    fp = None if face_port is None else np.asarray(face_port, dtype=np.int32).reshape(K, 4)
    mat = None if materials is None else np.asarray(materials, dtype=np.float64).reshape(K, -1)
    parts = []
    for r in range(R):
        owned = np.flatnonzero(part == r)
        nb = nbr[owned].ravel()
        nb = nb[nb >= 0]
        halo = np.unique(nb[part[nb] != r])
        elems = np.concatenate([owned, halo])
        verts, inv = np.unique(tets[elems].ravel(), return_inverse=True)
        local = Mesh(np.ascontiguousarray(mesh.nodes[verts]), inv.reshape(-1, 4).astype(np.int32))
        parts.append(Part(r, owned, halo, local, None if fp is None else np.ascontiguousarray(fp[elems]),
                          None if mat is None else np.ascontiguousarray(mat[elems])))
    for r, pr in enumerate(parts):
        for q in range(R):
            if q == r:
                continue
            # elements r owns that q keeps as halo: what r sends to q
            s_glob = parts[q].halo[part[parts[q].halo] == r]
            if s_glob.size:
                pr.send[q] = np.searchsorted(pr.owned, s_glob).astype(np.int64)
            # elements q owns that r keeps as halo: what r receives from q
            r_glob = pr.halo[part[pr.halo] == q]
            if r_glob.size:
                pr.recv[q] = (pr.n_owned + np.searchsorted(pr.halo, r_glob)).astype(np.int64)
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

    Every kernel of the operator, the exchange buffers and the transport's
    collectives run on ONE torch CUDA stream, which the operator's context is
    bound to.  NCCL point-to-point operations issued under `comm()` wait for
    the gathers queued before them on that stream, and their completion is
    waited for on that stream before the scatters that follow, so an exchange
    needs no host synchronisation.  Engines whose operators share a context
    (all parts on one device) share its stream: the first engine of a context
    binds it (`stream`, or a new torch stream), the others reuse it."""

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
        elif stream is not None and stream is not bound:
            raise ValueError("engines of one context must share its stream")
        self.stream = bound
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
        """Context in which the transport issues its operations (this engine's stream)."""
        return self.torch.cuda.stream(self.stream)

    def gather(self, ids: np.ndarray, buf) -> None:
        self.gop.gather_elements(self._index(ids).data_ptr(), ids.size, buf.data_ptr())

    def scatter(self, ids: np.ndarray, buf) -> None:
        self.gop.scatter_elements(self._index(ids).data_ptr(), ids.size, buf.data_ptr())

    def stage(self, h: float, s: int) -> None:
        self.gop.lserk_stage(h, s)

    def sync(self) -> None:
        self.stream.synchronize()

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
    """LSERK4 on one part: per stage, the halo exchange, then one fused stage of
    the local operator (explicit.rs:100-135 with the exchange before each RHS)."""

    def __init__(self, part: Part, engine, transport):
        self.part = part
        self.engine = engine
        self.transport = transport
        self.sbuf = {q: engine.new_buffer(ids.size) for q, ids in part.send.items()}
        self.rbuf = {q: engine.new_buffer(ids.size) for q, ids in part.recv.items()}

    def exchange(self) -> None:
        """Gather the blocks peers need, move them, scatter the received ones.
        A device engine orders the three on its stream (no host wait); an
        engine without `comm()` works synchronously on the host."""
        for q, ids in self.part.send.items():
            self.engine.gather(ids, self.sbuf[q])
        comm = getattr(self.engine, "comm", None)
        if comm is None:
            self.transport.exchange(self.sbuf, self.rbuf)
        else:
            with comm():
                self.transport.exchange(self.sbuf, self.rbuf)
        for q, ids in self.part.recv.items():
            self.engine.scatter(ids, self.rbuf[q])

    def step(self, h: float, steps: int = 1) -> None:
        for _ in range(int(steps)):
            for s in range(5):
                self.exchange()
                self.engine.stage(h, s)


class LoopbackLserk:
    """All parts of a partition in one process (one device or the CPU): the
    exchange copies each pair's blocks through a buffer of the sender."""

    def __init__(self, parts: list[Part], engines: list):
        self.parts = parts
        self.engines = engines
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
                self.exchange()
                for e in self.engines:
                    e.stage(h, s)
