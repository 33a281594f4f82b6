"""The time-domain operator of a model on a tagged mesh: the B200 path's
counterpart of crates/rapidfem-td/src/build.rs:74-259 (``operator_from_model``).

A model names volume regions and face groups by integer tags of a tagged mesh
(tet volume tags, and boundary or interior triangles grouped by face tag, as
rapidfem's meshes carry them) and attaches to them:

* materials (build.rs:84-105): diagonal eps and mu, conductivity, per volume
  tag; everything else is vacuum;
* PML regions (build.rs:109-118): graded impedance-matched absorbing layers,
  sigma = nu eps, sigma* = nu mu with nu = nu_max (depth/thickness)^2 and
  nu_max = ABSORBER_LOSS_BUDGET / thickness (build.rs:36-68);
* ports (build.rs:121-231), numbered in the reference's order: rectangular
  modal ports, then absorbing (ABC) faces; every port face is a
  characteristic (Silver-Mueller) boundary, and a rectangular port carries
  its TE_mn profile for injection and modal probes;
* PEC plates (build.rs:244-247): interior faces severed from their neighbour,
  each side a PEC wall; boundary faces are PEC anyway;
* periodic pairs (build.rs:235-240): two boundary face groups wired to one
  another across the period translation (MaxwellOperator.link_periodic).

Kinds the DG path of this library does not carry are rejected with the
reference's wording where the reference rejects them (lumped ports) and with
a clear error otherwise (Debye dispersion: the reference's GPU path excludes
it too, gpu/operator.rs:211-215; coaxial, Floquet and numerical wave-port
profiles).  Frequency-domain-only face conditions are
ignored with a warning, as the reference does (build.rs:216-229).
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass, field

import numpy as np

from .operator import MaxwellOperator, Mesh

ABSORBER_LOSS_BUDGET = 24.0  # build.rs:36-40: round-trip loss nu_max * thickness

_FACE_LOCAL = np.array([[0, 1, 2], [0, 2, 3], [0, 3, 1], [1, 2, 3]])  # core/mesh.rs:45-50
PEC_PLATE = -2  # face_port code of a severed interior face (include/dgtd_host.h)


@dataclass
class TaggedMesh:
    """A tet mesh with volume tags per tet and face groups: face_tags[tag] is
    an [T, 3] array of node-id triangles (any vertex order)."""

    mesh: Mesh
    volume_tags: np.ndarray
    face_tags: dict = field(default_factory=dict)

    @property
    def n_tets(self) -> int:
        return self.mesh.n_tets

    def tets_of(self, tag: int) -> np.ndarray:
        return np.flatnonzero(np.asarray(self.volume_tags) == tag)

    def faces_of(self, tag: int) -> np.ndarray:
        """Boolean [K, 4]: the local faces (TET_FACE_LOCAL order) whose
        triangle belongs to face group `tag` (both sides of an interior face)."""
        tris = self.face_tags.get(tag)
        if tris is None or len(tris) == 0:
            raise ValueError(f"face tag {tag} has no triangles")
        return _faces_matching(self.mesh, np.asarray(tris))


def _tri_keys(tris: np.ndarray, base: int) -> np.ndarray:
    t = np.sort(np.asarray(tris, dtype=np.int64), axis=1)
    return (t[:, 0] * base + t[:, 1]) * base + t[:, 2]


def _faces_matching(mesh: Mesh, tris: np.ndarray) -> np.ndarray:
    tets = np.asarray(mesh.tets, dtype=np.int64)
    base = int(mesh.nodes.shape[0]) + 1
    faces = tets[:, _FACE_LOCAL].reshape(-1, 3)
    keys = _tri_keys(faces, base)
    want = np.unique(_tri_keys(tris, base))
    hit = np.isin(keys, want).reshape(-1, 4)
    return hit


# ---------------------------------------------------------------- model parts

@dataclass
class Material:
    """A material on a volume tag (rapidfem_core Model materials): relative
    permittivity / permeability (scalar or diagonal) and conductivity (in the
    operator's units).  `debye` (eps_inf, eps_static, tau) is not carried on
    this path."""

    volume_tag: int
    er: float = 1.0
    ur: float = 1.0
    er_diag: tuple | None = None
    ur_diag: tuple | None = None
    conductivity: float = 0.0
    debye: tuple | None = None


@dataclass
class Pml:
    """A PML region: the tets of `volume_tag` behind the plane
    x[axis] = inner_face, `direction` pointing out of the domain, `thickness` deep."""

    volume_tag: int
    direction: tuple
    inner_face: float
    thickness: float


@dataclass
class RectangularPort:
    """A rectangular waveguide port (TE_mn, mode != (0, 0)) on face group `tag`."""

    tag: int
    mode: tuple = (1, 0)


@dataclass
class AbcFace:
    """An absorbing (first-order Silver-Mueller) boundary on face group `tag`."""

    tag: int


@dataclass
class OtherFace:
    """A face condition this path does not model: kind in {"lumped", "coax",
    "floquet", "wave", "surface_impedance", "lumped_element", "user_defined",
    "pmc"}."""

    tag: int
    kind: str


@dataclass
class Model:
    materials: list = field(default_factory=list)
    pml: list = field(default_factory=list)
    faces: list = field(default_factory=list)
    pec_tags: list = field(default_factory=list)
    periodic: list = field(default_factory=list)
    far_field_tag: int | None = None


@dataclass
class ModelOperator:
    """The result of operator_from_model: the host operator, the face tag of
    each port in port order, the per-tet material table [K, 8] and the
    face codes [K, 4] it was built from."""

    op: MaxwellOperator
    port_tags: list
    port_modes: list
    materials: np.ndarray
    face_port: np.ndarray


# ---------------------------------------------------------------- the mapping

def absorber_rate(mesh: Mesh, tets: np.ndarray, axis: int, low: bool, inner: float, thickness: float,
                  nu_max: float) -> np.ndarray:
    """build.rs:52-68: nu_max (depth/thickness)^2 by tet centroid, NaN in front
    of the layer (depth <= 0)."""
    cen = mesh.nodes[np.asarray(mesh.tets)[tets]][:, :, axis].sum(axis=1) / 4.0
    depth = (inner - cen) if low else (cen - inner)
    frac = np.clip(depth / thickness, 0.0, 1.0)
    return np.where(depth > 0.0, nu_max * frac * frac, np.nan)


def materials_of(tm: TaggedMesh, model: Model) -> np.ndarray:
    """The per-tet material table [K, 8] (eps_xyz, mu_xyz, sigma, sigma_m)."""
    K = tm.n_tets
    mat = np.zeros((K, 8))
    mat[:, 0:6] = 1.0
    for m in model.materials:
        if m.debye is not None:
            raise NotImplementedError(
                f"volume tag {m.volume_tag}: Debye dispersion is not carried by the device path "
                "(the reference's GPU path excludes dispersion as well)")
        eps = m.er_diag if m.er_diag is not None else (m.er,) * 3
        mu = m.ur_diag if m.ur_diag is not None else (m.ur,) * 3
        t = tm.tets_of(m.volume_tag)
        mat[t, 0:3] = eps
        mat[t, 3:6] = mu
        mat[t, 6] = m.conductivity
        mat[t, 7] = 0.0
    for p in model.pml:
        d = np.asarray(p.direction, dtype=np.float64)
        axis = int(np.argmax(np.abs(d)))
        low = d[axis] < 0.0
        nu_max = ABSORBER_LOSS_BUDGET / p.thickness if p.thickness > 0.0 else 0.0
        t = tm.tets_of(p.volume_tag)
        nu = absorber_rate(tm.mesh, t, axis, low, p.inner_face, p.thickness, nu_max)
        ok = ~np.isnan(nu)
        tt = t[ok]
        mat[tt, 6] = nu[ok] * mat[tt, 0]
        mat[tt, 7] = nu[ok] * mat[tt, 3]
    return mat


def face_codes_of(tm: TaggedMesh, model: Model):
    """(face_port [K, 4], port_tags, port_modes): port indices in the
    reference's order (rectangular, then ABC), -2 on PEC plate faces."""
    K = tm.n_tets
    code = -np.ones((K, 4), dtype=np.int32)
    tags, modes = [], []
    for f in model.faces:
        if isinstance(f, RectangularPort):
            if tuple(f.mode) == (0, 0):
                raise ValueError(f"rectangular port tag {f.tag}: mode (0, 0) carries no TE field, "
                                 "use (m, n) with m or n nonzero")
            code[tm.faces_of(f.tag)] = len(tags)
            tags.append(f.tag)
            modes.append(tuple(f.mode))
    for f in model.faces:
        if isinstance(f, OtherFace) and f.kind in ("coax", "floquet", "wave"):
            raise NotImplementedError(f"{f.kind} port tag {f.tag}: its modal profile is not carried by the "
                                      "device path (rectangular ports and ABC faces are)")
    for f in model.faces:
        if isinstance(f, AbcFace):
            code[tm.faces_of(f.tag)] = len(tags)
            tags.append(f.tag)
            modes.append(None)
        elif isinstance(f, OtherFace):
            if f.kind == "lumped":
                raise ValueError("LumpedPort is not supported by the time-domain backend. Use a modal port "
                                 "(RectWaveguidePort, CoaxPort) for waveguide / TEM geometries, or a WavePort "
                                 "(2D cross-section eigensolve) for microstrip-class lines. The "
                                 "frequency-domain backend still supports LumpedPort.")
            if f.kind in ("surface_impedance", "lumped_element", "user_defined", "pmc"):
                warnings.warn(f"TD: face tag {f.tag} carries a frequency-domain-only condition, ignored")
    if model.far_field_tag is not None:
        warnings.warn(f"TD: far-field surface tag {model.far_field_tag} ignored, the near-to-far-field "
                      "transform is frequency-domain only")
    for tag in model.pec_tags:
        code[tm.faces_of(tag)] = PEC_PLATE
    return code, tags, modes


def operator_from_model(tm: TaggedMesh, model: Model, order: int, flux_alpha: float = 1.0,
                        c: float = 1.0) -> ModelOperator:
    """build.rs:74-259: the host operator of `model` on `tm` (order, flux blend
    1 upwind / 0 central; `c` the speed of light in the mesh's length unit,
    which the reference uses only for dispersion and wave-port wavenumbers,
    neither carried here), with the face tag of each port in port order."""
    del c
    mat = materials_of(tm, model)
    code, tags, modes = face_codes_of(tm, model)
    pairs = periodic_faces_of(tm, model)
    op = MaxwellOperator(tm.mesh, order, flux_alpha, face_port=code, materials=mat)
    for a, b in pairs:
        op.link_periodic(a, b)
    return ModelOperator(op, tags, modes, mat, code)


def periodic_faces_of(tm: TaggedMesh, model: Model) -> list:
    """build.rs:235-240: per periodic pair (tag_a, tag_b), the face ids
    (e*4 + local face) of each side's triangles."""
    out = []
    for a, b in model.periodic:
        ta, tb = tm.face_tags.get(a), tm.face_tags.get(b)
        if ta is None or tb is None or len(ta) == 0 or len(tb) == 0:
            raise ValueError(f"periodic pair ({a}, {b}): a face tag has no triangles")
        out.append((np.flatnonzero(tm.faces_of(a).ravel()), np.flatnonzero(tm.faces_of(b).ravel())))
    return out


def box_tagged(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0) -> TaggedMesh:
    """The structured Kuhn box with the six boundary planes as face groups
    1..6 (x = 0, x = lx, y = 0, y = ly, z = 0, z = lz) and volume tag 1."""
    from .operator import boundary_faces_on_plane, structured_box

    mesh = structured_box(nx, ny, nz, lx, ly, lz)
    tets = np.asarray(mesh.tets)
    groups = {}
    for k, (axis, value) in enumerate(((0, 0.0), (0, lx), (1, 0.0), (1, ly), (2, 0.0), (2, lz))):
        on = boundary_faces_on_plane(mesh, axis, value)
        e, f = np.nonzero(on)
        groups[k + 1] = tets[e[:, None], _FACE_LOCAL[f]]
    return TaggedMesh(mesh, np.ones(mesh.n_tets, dtype=np.int32), groups)


def plane_triangles(mesh: Mesh, axis: int, value: float, lo=None, hi=None, tol=1e-9) -> np.ndarray:
    """Triangles of the mesh's faces lying on the plane x[axis] = value (interior
    or boundary), optionally restricted to the rectangle lo <= x <= hi of the
    other two axes: a face group for an internal plate or a port."""
    tets = np.asarray(mesh.tets, dtype=np.int64)
    tri = tets[:, _FACE_LOCAL].reshape(-1, 3)
    x = mesh.nodes[tri]  # [4K, 3, 3]
    on = np.all(np.abs(x[:, :, axis] - value) < tol, axis=1)
    if lo is not None or hi is not None:
        cen = x.mean(axis=1)
        lo = np.asarray(lo if lo is not None else [-np.inf] * 3, dtype=np.float64)
        hi = np.asarray(hi if hi is not None else [np.inf] * 3, dtype=np.float64)
        on &= np.all((cen >= lo - tol) & (cen <= hi + tol), axis=1)
    t = np.unique(np.sort(tri[on], axis=1), axis=0)
    return t
