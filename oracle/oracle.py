"""ctypes binding of the CPU oracle (``oracle/dgtd_oracle.c``).

TEST INFRASTRUCTURE ONLY: the f64 CPU restatement of rapidfem's DGTD path
(crates/rapidfem-td/src/{dg_basis,geom_factors,rhs,explicit,
explicit_adaptive,propagator,session}.rs).  Imported by ``tests/``,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` as the checker;
the product package ``rapidfem_b200`` never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libdgtd_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "dgtd_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-B" if force else "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    L.orc_op_build.restype = C.c_void_p
    L.orc_op_build.argtypes = [_dp, C.c_int, _ip, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    L.orc_op_free.argtypes = [C.c_void_p]
    for f in ("orc_op_np", "orc_op_nfp", "orc_op_n_elem"):
        getattr(L, f).restype = C.c_int
        getattr(L, f).argtypes = [C.c_void_p]
    L.orc_op_n_dof.restype = C.c_long
    L.orc_op_n_dof.argtypes = [C.c_void_p]
    L.orc_op_get.restype = C.c_int
    L.orc_op_get.argtypes = [C.c_void_p, C.c_char_p, _dp]
    L.orc_apply.argtypes = [C.c_void_p, _dp, _dp]
    L.orc_lserk_steps.argtypes = [C.c_void_p, _dp, C.c_double, C.c_int, C.c_int, C.c_long,
                                  C.c_void_p, C.c_void_p]
    L.orc_kcl_step.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_int, C.c_long, C.c_void_p,
                               C.c_double]
    L.orc_expm.argtypes = [_dp, C.c_int, _dp]
    L.orc_expmv.restype = C.c_int
    L.orc_expmv.argtypes = [C.c_void_p, _dp, C.c_double, C.c_int, C.c_double, _dp]
    L.orc_expmv_dense.restype = C.c_int
    L.orc_expmv_dense.argtypes = [_dp, C.c_size_t, _dp, C.c_double, C.c_int, C.c_double, _dp]
    L.orc_etd_step.restype = C.c_int
    L.orc_etd_step.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_int, C.c_double, _dp]
    L.orc_field_energy.restype = C.c_double
    L.orc_field_energy.argtypes = [C.c_void_p, _dp]
    L.orc_power_rho.restype = C.c_double
    L.orc_power_rho.argtypes = [C.c_void_p, C.c_int, _dp]
    L.orc_cfl_z.restype = C.c_double
    L.orc_cfl_z.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.orc_curl_single.restype = C.c_int
    L.orc_curl_single.argtypes = [C.c_int, _dp, _dp, _dp]
    L.orc_kuhn_tets.argtypes = [C.c_int, C.c_int, C.c_int, _ip]
    L.orc_box_nodes.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _dp]
    L.orc_box_nodes_jittered.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_uint64, _dp]
    L.orc_normal_vector.argtypes = [C.c_size_t, C.c_uint64, _dp]
    L.orc_node_coords.argtypes = [C.c_void_p, _dp]
    L.orc_port_source.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    L.orc_port_projections.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_get_threads.restype = C.c_int
    L.orc_lserk_coeffs.argtypes = [_dp, _dp]
    _lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
    L.orc_link_periodic.restype = C.c_int
    L.orc_link_periodic.argtypes = [C.c_void_p, _dp, _ip, _lp, C.c_int, _lp, C.c_int]
    L.orc_kcl_coeffs.argtypes = [_dp, _dp, _dp]
    _lib = L
    return L


def set_threads(t: int) -> None:
    lib().orc_set_threads(int(t))


def threads() -> int:
    return int(lib().orc_get_threads())


# --------------------------------------------------------------------------
# meshes (mesh_gen.rs restated)
# --------------------------------------------------------------------------

def box_mesh(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0):
    L = lib()
    nodes = np.zeros(((nx + 1) * (ny + 1) * (nz + 1), 3))
    tets = np.zeros((nx * ny * nz * 6, 4), dtype=np.int32)
    L.orc_box_nodes(nx, ny, nz, lx, ly, lz, nodes)
    L.orc_kuhn_tets(nx, ny, nz, tets)
    return nodes, tets


def box_mesh_jittered(nx, ny, nz, lx, ly, lz, amplitude, seed):
    L = lib()
    nodes = np.zeros(((nx + 1) * (ny + 1) * (nz + 1), 3))
    tets = np.zeros((nx * ny * nz * 6, 4), dtype=np.int32)
    L.orc_box_nodes_jittered(nx, ny, nz, lx, ly, lz, amplitude, seed, nodes)
    L.orc_kuhn_tets(nx, ny, nz, tets)
    return nodes, tets


def normal_vector(n, seed=0):
    out = np.zeros(n)
    lib().orc_normal_vector(n, seed, out)
    return out


def lserk_coeffs():
    a = np.zeros(5)
    b = np.zeros(5)
    lib().orc_lserk_coeffs(a, b)
    return a, b


def expm(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    out = np.zeros_like(a)
    lib().orc_expm(a.ravel(), n, out.ravel())
    return out


def expmv_dense(a, v, t, m, tol=0.0):
    a = np.ascontiguousarray(a, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    out = np.zeros_like(v)
    dim = lib().orc_expmv_dense(a.ravel(), v.size, v, t, m, tol, out)
    return out, dim


def curl_single(order, jinv, field):
    jinv = np.ascontiguousarray(jinv, dtype=np.float64).ravel()
    field = np.ascontiguousarray(field, dtype=np.float64).ravel()
    out = np.zeros_like(field)
    if lib().orc_curl_single(order, jinv, field, out):
        raise RuntimeError("curl_single failed")
    return out


class Operator:
    """The f64 operator of rhs.rs:805-1000 built on a tet mesh.

    face_port: optional int32 [K,4] (-1 none); materials: optional [K, 8]
    float64 (eps_x,eps_y,eps_z, mu_x,mu_y,mu_z, sigma, sigma_m).
    """

    def __init__(self, nodes, tets, order, flux_alpha=1.0, face_port=None, materials=None):
        L = lib()
        self._L = L
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        tets = np.ascontiguousarray(tets, dtype=np.int32)
        fp = None
        mp = None
        if face_port is not None:
            self._fp = np.ascontiguousarray(face_port, dtype=np.int32).ravel()
            fp = self._fp.ctypes.data
        if materials is not None:
            self._mat = np.ascontiguousarray(materials, dtype=np.float64).ravel()
            mp = self._mat.ctypes.data
        h = L.orc_op_build(nodes.ravel(), nodes.shape[0], tets.ravel(), tets.shape[0], int(order),
                           float(flux_alpha), fp, mp)
        if not h:
            raise RuntimeError("oracle operator build failed (unmatched face node?)")
        self.h = C.c_void_p(h)
        self.np = L.orc_op_np(self.h)
        self.nfp = L.orc_op_nfp(self.h)
        self.n_elem = L.orc_op_n_elem(self.h)
        self.n_dof = int(L.orc_op_n_dof(self.h))
        self.order = order
        self.flux_alpha = flux_alpha
        self._nodes, self._tets = nodes, tets

    _PERIODIC_ERRORS = {1: "different face counts on the two sides", 2: "a port face", 3: "a face with a neighbour",
                        4: "zero total area", 5: "a side-A face without partner", 6: "not a bijection",
                        7: "an unmatched face node"}

    def link_periodic(self, faces_a, faces_b):
        """link_periodic_faces (rhs.rs:616-770) on face ids e*4+lf."""
        a = np.ascontiguousarray(faces_a, dtype=np.int64)
        b = np.ascontiguousarray(faces_b, dtype=np.int64)
        rc = self._L.orc_link_periodic(self.h, self._nodes.ravel(), self._tets.ravel(), a, a.size, b, b.size)
        if rc:
            raise ValueError(f"periodic pair: {self._PERIODIC_ERRORS.get(rc, rc)}")

    def __del__(self):
        try:
            self._L.orc_op_free(self.h)
        except Exception:
            pass

    _SIZES = {
        "nodes": lambda s: 3 * s.np, "mass": lambda s: s.np * s.np, "dr": lambda s: s.np * s.np,
        "ds": lambda s: s.np * s.np, "dt": lambda s: s.np * s.np,
        "lift": lambda s: s.np * 4 * s.nfp, "face_nodes": lambda s: 4 * s.nfp,
        "face_w": lambda s: 4 * s.nfp, "jinv": lambda s: 9 * s.n_elem, "jac": lambda s: 9 * s.n_elem,
        "origin": lambda s: 3 * s.n_elem, "det": lambda s: s.n_elem,
        "normal": lambda s: 12 * s.n_elem, "fscale": lambda s: 4 * s.n_elem,
        "nbr": lambda s: 4 * s.n_elem, "nbr_lf": lambda s: 4 * s.n_elem,
        "port": lambda s: 4 * s.n_elem, "perm": lambda s: 4 * s.n_elem * s.nfp,
        "inv_eps": lambda s: 3 * s.n_elem, "inv_mu": lambda s: 3 * s.n_elem,
        "sigma_eps": lambda s: 3 * s.n_elem, "sigma_mu": lambda s: 3 * s.n_elem,
    }

    def get(self, which):
        out = np.zeros(self._SIZES[which](self))
        if self._L.orc_op_get(self.h, which.encode(), out):
            raise KeyError(which)
        return out

    def apply(self, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        dy = np.zeros_like(y)
        self._L.orc_apply(self.h, y, dy)
        return dy

    def lserk(self, y, dt, steps, src_dof=None, src_vec=None, vals=None):
        y = np.array(y, dtype=np.float64, copy=True)
        kind, dof, vp, gp = 0, 0, None, None
        if src_dof is not None:
            kind, dof = 1, int(src_dof)
        elif src_vec is not None:
            kind = 2
            self._sv = np.ascontiguousarray(src_vec, dtype=np.float64)
            vp = self._sv.ctypes.data
        if kind:
            self._vals = np.ascontiguousarray(vals, dtype=np.float64)
            gp = self._vals.ctypes.data
        self._L.orc_lserk_steps(self.h, y, float(dt), int(steps), kind, dof, vp, gp)
        return y

    def kcl_step(self, y, dt, src_dof=None, src_vec=None, g=0.0):
        y = np.array(y, dtype=np.float64, copy=True)
        err = np.zeros_like(y)
        kind, dof, vp = 0, 0, None
        if src_dof is not None:
            kind, dof = 1, int(src_dof)
        elif src_vec is not None:
            kind = 2
            self._sv = np.ascontiguousarray(src_vec, dtype=np.float64)
            vp = self._sv.ctypes.data
        self._L.orc_kcl_step(self.h, y, err, float(dt), kind, dof, vp, float(g))
        return y, err

    def expmv(self, v, t, m, tol=0.0):
        v = np.ascontiguousarray(v, dtype=np.float64)
        out = np.zeros_like(v)
        dim = self._L.orc_expmv(self.h, v, float(t), int(m), float(tol), out)
        return out, dim

    def etd_step(self, y, b, h, m, tol=0.0):
        y = np.ascontiguousarray(y, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        out = np.zeros_like(y)
        dim = self._L.orc_etd_step(self.h, y, b, float(h), int(m), float(tol), out)
        return out, dim

    def field_energy(self, y):
        return float(self._L.orc_field_energy(self.h, np.ascontiguousarray(y, dtype=np.float64)))

    def power_rho(self, iters=40):
        v = np.zeros(self.n_dof)
        rho = self._L.orc_power_rho(self.h, int(iters), v)
        return float(rho), v

    def cfl_z(self):
        rho = C.c_double(0.0)
        z = self._L.orc_cfl_z(self.h, C.byref(rho))
        return float(z), float(rho.value)

    def node_coords(self):
        out = np.zeros((self.n_elem * self.np, 3))
        self._L.orc_node_coords(self.h, out.ravel())
        return out

    def port_source(self, port, profiles):
        b = np.zeros(self.n_dof)
        self._L.orc_port_source(self.h, int(port), np.ascontiguousarray(profiles, dtype=np.float64).ravel(), b)
        return b

    def port_projections(self, port, profiles, y):
        out = np.zeros(2)
        self._L.orc_port_projections(self.h, int(port),
                                     np.ascontiguousarray(profiles, dtype=np.float64).ravel(),
                                     np.ascontiguousarray(y, dtype=np.float64), out)
        return out
