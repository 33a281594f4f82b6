"""Host side of the DGTD path: structured meshes and the f64 operator build.

Python face of ``include/dgtd_host.h``.  ``MaxwellOperator`` mirrors
crates/rapidfem-td/src/rhs.rs:805-1000 (``MaxwellOperator::new``): it holds the
reference element, geometric factors, face topology, neighbour permutations,
port tags and material reciprocals that the device operator consumes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from ._native import check, lib


@dataclass
class Mesh:
    """A tetrahedral mesh: node coordinates [n,3] (f64), tets [K,4] (i32)."""

    nodes: np.ndarray
    tets: np.ndarray

    @property
    def n_tets(self) -> int:
        return int(self.tets.shape[0])


def structured_box(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0) -> Mesh:
    """mesh_gen.rs:54-76: the Kuhn 6-tets-per-hex box [0,lx]x[0,ly]x[0,lz]."""
    nodes = np.zeros(((nx + 1) * (ny + 1) * (nz + 1), 3))
    tets = np.zeros((6 * nx * ny * nz, 4), dtype=np.int32)
    check(lib.dgtd_mesh_box(nx, ny, nz, lx, ly, lz, nodes.ravel(), tets.ravel()))
    return Mesh(nodes, tets)


def structured_box_jittered(nx, ny, nz, lx, ly, lz, amplitude, seed) -> Mesh:
    """mesh_gen.rs:86-139: the box with interior nodes displaced by up to
    `amplitude` cells along each axis, deterministic in `seed`."""
    nodes = np.zeros(((nx + 1) * (ny + 1) * (nz + 1), 3))
    tets = np.zeros((6 * nx * ny * nz, 4), dtype=np.int32)
    check(lib.dgtd_mesh_box_jittered(nx, ny, nz, lx, ly, lz, amplitude, seed, nodes.ravel(), tets.ravel()))
    return Mesh(nodes, tets)


def structured_box_graded_z(nx, ny, nz, lx, ly, lz, ratio) -> Mesh:
    """A box graded geometrically along z, the largest to smallest cell height
    `ratio`, fine at z = 0."""
    nodes = np.zeros(((nx + 1) * (ny + 1) * (nz + 1), 3))
    tets = np.zeros((6 * nx * ny * nz, 4), dtype=np.int32)
    check(lib.dgtd_mesh_box_graded_z(nx, ny, nz, lx, ly, lz, ratio, nodes.ravel(), tets.ravel()))
    return Mesh(nodes, tets)


def isotropic_materials(eps, mu=None, sigma=None, sigma_m=None):
    """Per-element material table [K,8] from per-element scalars."""
    eps = np.asarray(eps, dtype=np.float64)
    K = eps.size
    mu = np.ones(K) if mu is None else np.broadcast_to(np.asarray(mu, dtype=np.float64), (K,))
    sigma = np.zeros(K) if sigma is None else np.broadcast_to(np.asarray(sigma, dtype=np.float64), (K,))
    sigma_m = np.zeros(K) if sigma_m is None else np.broadcast_to(np.asarray(sigma_m, dtype=np.float64), (K,))
    m = np.zeros((K, 8))
    m[:, 0:3] = eps[:, None]
    m[:, 3:6] = mu[:, None]
    m[:, 6] = sigma
    m[:, 7] = sigma_m
    return m


def boundary_faces_on_plane(mesh: Mesh, axis: int, value: float, tol: float = 1e-9):
    """Boolean [K,4]: local faces (rhs.rs TET_FACE_LOCAL order) whose three
    vertices lie on the plane x[axis] == value."""
    local = np.array([[0, 1, 2], [0, 2, 3], [0, 3, 1], [1, 2, 3]])
    coords = mesh.nodes[mesh.tets][:, :, axis]  # [K,4]
    on = np.abs(coords - value) < tol
    return on[:, local].all(axis=2)


class MaxwellOperator:
    """The f64 DG operator on a tet mesh (rhs.rs:805-1000), built natively.

    face_port: optional int [K,4] port index per face (-1 none); materials:
    optional [K,8] (eps_xyz, mu_xyz, sigma, sigma_m).
    """

    def __init__(self, mesh: Mesh, order: int, flux_alpha: float = 1.0, face_port=None,
                 materials=None):
        self.mesh = mesh
        self.order = int(order)
        self.flux_alpha = float(flux_alpha)
        nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64)
        tets = np.ascontiguousarray(mesh.tets, dtype=np.int32)
        self._fp = None if face_port is None else np.ascontiguousarray(face_port, dtype=np.int32).ravel()
        self._mat = None if materials is None else np.ascontiguousarray(materials, dtype=np.float64).ravel()
        if self._fp is not None and self._fp.size != 4 * tets.shape[0]:
            raise ValueError("face_port must have 4 entries per tet")
        if self._mat is not None and self._mat.size != 8 * tets.shape[0]:
            raise ValueError("materials must have 8 entries per tet")
        h = C.c_void_p()
        check(lib.dgtd_host_op_build(nodes.ravel(), nodes.shape[0], tets.ravel(), tets.shape[0],
                                     self.order, self.flux_alpha, nat.ptr(self._fp), nat.ptr(self._mat),
                                     C.byref(h)))
        self._h = h
        np_, nfp, ne, nd = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
        check(lib.dgtd_host_op_info(h, C.byref(np_), C.byref(nfp), C.byref(ne), C.byref(nd)))
        self.np, self.nfp, self.n_elem, self.n_dof = np_.value, nfp.value, ne.value, nd.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:  # lib is None at interpreter shutdown
            lib.dgtd_host_op_destroy(h)
            self._h = C.c_void_p()

    @property
    def handle(self):
        return self._h

    _SIZES = {
        "nodes": lambda s: 3 * s.np, "mass": lambda s: s.np * s.np, "dr": lambda s: s.np * s.np,
        "ds": lambda s: s.np * s.np, "dt": lambda s: s.np * s.np, "lift": lambda s: s.np * 4 * s.nfp,
        "face_nodes": lambda s: 4 * s.nfp, "face_w": lambda s: 4 * s.nfp,
        "jinv": lambda s: 9 * s.n_elem, "jac": lambda s: 9 * s.n_elem, "origin": lambda s: 3 * s.n_elem,
        "det": lambda s: s.n_elem, "normal": lambda s: 12 * s.n_elem, "fscale": lambda s: 4 * s.n_elem,
        "nbr": lambda s: 4 * s.n_elem, "nbr_lf": lambda s: 4 * s.n_elem, "port": lambda s: 4 * s.n_elem,
        "perm": lambda s: 4 * s.n_elem * s.nfp, "inv_eps": lambda s: 3 * s.n_elem,
        "inv_mu": lambda s: 3 * s.n_elem, "sigma_eps": lambda s: 3 * s.n_elem,
        "sigma_mu": lambda s: 3 * s.n_elem,
    }

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self._SIZES[name](self))
        check(lib.dgtd_host_op_get(self._h, name.encode(), out))
        return out

    def link_periodic(self, faces_a, faces_b) -> None:
        """Wire a periodic face pair (link_periodic_faces, rhs.rs:616-770):
        the domain-boundary faces `faces_a` and `faces_b` (ids e*4 + local
        face) become interior faces across the translation between the two
        sides' centroids.  Raises (and leaves the operator unchanged) when a
        face is a port or not on the boundary, the counts differ, or a face
        or face node finds no partner."""
        a = np.ascontiguousarray(faces_a, dtype=np.int64).ravel()
        b = np.ascontiguousarray(faces_b, dtype=np.int64).ravel()
        if a.size == 0 or b.size == 0:
            raise ValueError("periodic pair: a side has no faces")
        check(lib.dgtd_host_op_link_periodic(self._h, a, a.size, b, b.size))

    def desc(self) -> nat.OpDesc:
        d = nat.OpDesc()
        check(lib.dgtd_host_op_desc(self._h, C.byref(d)))
        return d

    def node_coords(self) -> np.ndarray:
        out = np.zeros((self.n_elem * self.np, 3))
        check(lib.dgtd_host_node_coords(self._h, out.ravel()))
        return out

    def nearest_node_dof(self, point, field: int, comp: int) -> int:
        d = C.c_int64()
        check(lib.dgtd_host_nearest_node_dof(self._h, np.asarray(point, dtype=np.float64), field, comp, C.byref(d)))
        return d.value

    def port_n_faces(self, port: int) -> int:
        n = C.c_int64()
        check(lib.dgtd_host_port_n_faces(self._h, port, C.byref(n)))
        return n.value

    def rect_port_profiles(self, port: int, inward_normal, mode=(1, 0)) -> np.ndarray:
        nf = self.port_n_faces(port)
        out = np.zeros((nf * self.nfp, 6))
        check(lib.dgtd_host_rect_port_profiles(self._h, port, np.asarray(inward_normal, dtype=np.float64),
                                               int(mode[0]), int(mode[1]), out.ravel()))
        return out

    def port_modal_weights(self, port: int, profiles, which: str = "E"):
        """P_e (which="E") or P_h ("H") of `port` as a linear functional of the
        AoS state (rhs.rs:1211-1242): returns (idx, w) with P = w @ y[idx]."""
        if which not in ("E", "H"):
            raise ValueError("which must be 'E' or 'H'")
        nt = self.port_n_faces(port) * self.nfp * 3
        idx = np.empty(nt, dtype=np.int64)
        w = np.empty(nt, dtype=np.float64)
        check(lib.dgtd_host_port_modal_weights(self._h, port, np.ascontiguousarray(profiles, dtype=np.float64).ravel(),
                                               0 if which == "E" else 1, idx, w))
        return idx, w

    def port_source(self, port: int, profiles) -> np.ndarray:
        b = np.zeros(self.n_dof)
        check(lib.dgtd_host_port_source(self._h, port, np.ascontiguousarray(profiles, dtype=np.float64).ravel(), b))
        return b
