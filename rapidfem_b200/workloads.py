"""Synthetic workloads with the shapes of the DGTD benchmark configurations.

No dataset is involved: every mesh, material map and initial field here is
generated from the configuration's stated sizes and a seed.

  cavity_tm110   8^3 x 6 unit PEC cavity, N=3, vacuum, TM110 mode at the nodes
  sphere_pulse   48^3 x 6 jittered (+-10% h) box, N=4, eps_r=4 sphere r=0.25 at
                 the centre, Gaussian E_z pulse (sigma 0.05) at (0.3,0.4,0.5)
  graded_slab    24^3 x 6 box graded 20:1 toward z=0, N=3, lossy slab z<0.2
                 (eps_r 2.2, sigma 5), point E_z source at the centre
  waveguide_post 22.86 x 10.16 x 60 mm WR-90 section as 39x17x101 hex x6 tets,
                 N=3, dielectric post r=1.5 mm, TE10 port at z=0, absorbing z=60 mm
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import operator as O


@dataclass
class Workload:
    name: str
    mesh: O.Mesh
    order: int
    materials: np.ndarray | None
    face_port: np.ndarray | None
    y0_fn: object
    info: dict = field(default_factory=dict)

    def build(self, flux_alpha: float = 1.0) -> O.MaxwellOperator:
        return O.MaxwellOperator(self.mesh, self.order, flux_alpha, face_port=self.face_port,
                                 materials=self.materials)

    def y0(self, op: O.MaxwellOperator) -> np.ndarray:
        return self.y0_fn(op)


def _centroids(mesh):
    return mesh.nodes[mesh.tets].mean(axis=1)


def cavity_tm110(n: int = 8, order: int = 3) -> Workload:
    mesh = O.structured_box(n, n, n)

    def y0(op):
        x = op.node_coords()
        y = np.zeros((x.shape[0], 6))
        y[:, 2] = np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1])
        return y.ravel()

    return Workload("cavity_tm110", mesh, order, None, None, y0,
                    {"cells": f"{n}^3", "tets": mesh.n_tets, "order": order})


def tm110_exact(op, t):
    """TM110 of the unit PEC cube at time t (omega = pi*sqrt 2, c = 1)."""
    x = op.node_coords()
    w = np.pi * np.sqrt(2.0)
    y = np.zeros((x.shape[0], 6))
    y[:, 2] = np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1]) * np.cos(w * t)
    y[:, 3] = -(np.pi / w) * np.sin(np.pi * x[:, 0]) * np.cos(np.pi * x[:, 1]) * np.sin(w * t)
    y[:, 4] = (np.pi / w) * np.cos(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1]) * np.sin(w * t)
    return y.ravel()


def sphere_pulse(n: int = 48, order: int = 4, seed: int = 2024) -> Workload:
    mesh = O.structured_box_jittered(n, n, n, 1.0, 1.0, 1.0, 0.10, seed)
    cen = _centroids(mesh)
    eps = np.where(np.linalg.norm(cen - 0.5, axis=1) < 0.25, 4.0, 1.0)

    def y0(op):
        x = op.node_coords()
        y = np.zeros((x.shape[0], 6))
        r2 = ((x - np.array([0.3, 0.4, 0.5])) ** 2).sum(axis=1)
        y[:, 2] = np.exp(-r2 / (2 * 0.05 ** 2))
        return y.ravel()

    return Workload("sphere_pulse", mesh, order, O.isotropic_materials(eps), None, y0,
                    {"cells": f"{n}^3", "tets": mesh.n_tets, "order": order, "jitter": 0.10,
                     "seed": seed, "sphere_eps": 4.0})


def graded_slab(n: int = 24, order: int = 3) -> Workload:
    mesh = O.structured_box_graded_z(n, n, n, 1.0, 1.0, 1.0, 20.0)
    cen = _centroids(mesh)
    slab = cen[:, 2] < 0.2
    eps = np.where(slab, 2.2, 1.0)
    sigma = np.where(slab, 5.0, 0.0)

    def y0(op):
        return np.zeros(op.n_dof)

    return Workload("graded_slab", mesh, order, O.isotropic_materials(eps, sigma=sigma), None, y0,
                    {"cells": f"{n}^3", "tets": mesh.n_tets, "order": order, "grading": 20.0})


def gaussian_sine(t, t0, sigma_t, f0):
    """Gaussian-modulated sine g(t) = exp(-(t-t0)^2/(2 sigma^2)) sin(2 pi f0 (t-t0))."""
    return np.exp(-((t - t0) ** 2) / (2 * sigma_t ** 2)) * np.sin(2 * np.pi * f0 * (t - t0))


def waveguide_post(eps_post: float = 6.0, order: int = 3, cells=(39, 17, 101)) -> Workload:
    a, b, L = 22.86e-3, 10.16e-3, 60e-3
    mesh = O.structured_box(cells[0], cells[1], cells[2], a, b, L)
    cen = _centroids(mesh)
    post = np.hypot(cen[:, 0] - a / 2, cen[:, 2] - L / 2) < 1.5e-3
    eps = np.where(post, eps_post, 1.0)
    port = np.where(O.boundary_faces_on_plane(mesh, 2, 0.0), 0, -1)
    port[O.boundary_faces_on_plane(mesh, 2, L)] = 1

    def y0(op):
        return np.zeros(op.n_dof)

    return Workload("waveguide_post", mesh, order, O.isotropic_materials(eps), port, y0,
                    {"cells": "x".join(map(str, cells)), "tets": mesh.n_tets, "order": order,
                     "eps_post": eps_post})
