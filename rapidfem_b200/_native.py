"""ctypes binding of ``_lib/librapidfem_b200.so`` (the C ABI of include/dgtd.h
and include/dgtd_host.h).

There is no fallback: if the library is missing or cannot be loaded, importing
this module raises, naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("DGTD_LIB_PATH") or os.path.join(_PKG, "_lib", "librapidfem_b200.so")

DGTD_OK = 0
DGTD_ERR_COLLAPSE = 8
ERR_NAMES = {
    1: "BAD_ARG", 2: "CUDA", 3: "NONFINITE", 4: "TIMEOUT", 5: "NO_DEVICE", 6: "UNSUPPORTED",
    7: "OOM", 8: "COLLAPSE",
}

DRIVE_FREE, DRIVE_POINT, DRIVE_VECTOR = 0, 1, 2
ENGINE_FP32, ENGINE_TF32X3, ENGINE_FP32_SMALL_TILES = 0, 1, 2


class DgtdError(RuntimeError):
    """An error status returned by the native library."""

    def __init__(self, code, msg):
        super().__init__(f"[{ERR_NAMES.get(code, code)}] {msg}")
        self.code = code


class NoDeviceError(DgtdError):
    pass


if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"rapidfem_b200 native library not found at {LIB_PATH}; build it with "
        "`python -m rapidfem_b200.build` (there is no CPU fallback)")

lib = C.CDLL(LIB_PATH)

_vp = C.c_void_p
_i32, _i64, _u64, _f32, _f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_float, C.c_double
_pd = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_pf = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_pi = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_pl = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


class OpDesc(C.Structure):
    _fields_ = [
        ("order", _i32), ("n_elem", _i32), ("flux_alpha", _f64),
        ("diff_r", _vp), ("diff_s", _vp), ("diff_t", _vp), ("lift", _vp), ("face_nodes", _vp),
        ("jinv", _vp), ("inv_eps", _vp), ("inv_mu", _vp), ("sigma_eps", _vp), ("sigma_mu", _vp),
        ("face_normal", _vp), ("face_fscale", _vp), ("face_neighbor", _vp),
        ("face_nbr_local", _vp), ("face_port", _vp), ("face_perm", _vp), ("mass", _vp), ("dt_scale", _vp),
    ]


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("dgtd_last_error", C.c_int, C.c_char_p, C.c_size_t)
_sig("dgtd_version", C.c_char_p)
_sig("dgtd_ctx_create", C.c_int, C.c_int, C.POINTER(_vp))
_sig("dgtd_ctx_destroy", C.c_int, _vp)
_sig("dgtd_ctx_device_name", C.c_int, _vp, C.c_char_p, C.c_size_t)
_sig("dgtd_ctx_set_stream", C.c_int, _vp, _vp)
_sig("dgtd_ctx_synchronize", C.c_int, _vp)
_sig("dgtd_op_create", C.c_int, _vp, C.POINTER(OpDesc), C.POINTER(_vp))
_sig("dgtd_op_destroy", C.c_int, _vp)
_sig("dgtd_op_n_dof", C.c_int, _vp, C.POINTER(_i64))
_sig("dgtd_op_set_engine", C.c_int, _vp, C.c_int)
_sig("dgtd_op_get_engine", C.c_int, _vp, C.POINTER(C.c_int))
_sig("dgtd_op_check_error", C.c_int, _vp)
_sig("dgtd_apply", C.c_int, _vp, _pf, _pf)
_sig("dgtd_transient", C.c_int, _vp, _pf, _f32, _i64, _i64, C.c_int, _i64, _vp, _vp, C.c_int, _pf)
_sig("dgtd_apply_f64", C.c_int, _vp, _pd, _pd)
_sig("dgtd_transient_f64", C.c_int, _vp, _pd, _f64, _i64, _i64, C.c_int, _i64, _vp, _vp, C.c_int, _pd)
_sig("dgtd_transient_f64_stages", C.c_int, _vp, _pd, _f64, _i64, _i64, C.c_int, _i64, _vp, _vp, C.c_int, _pd)
_sig("dgtd_transient_probes", C.c_int, _vp, _pf, _f32, _i64, _i64, C.c_int, _i64, _vp, _vp, _vp,
     _i64, _vp, _vp)
class KclController(C.Structure):
    """dgtd_kcl_controller (session.rs:130-143)."""
    _fields_ = [(k, C.c_double) for k in ("atol", "rtol", "safety", "growth_limit", "shrink_limit",
                                           "pi_alpha", "pi_beta", "min_step_factor")]


class KclStats(C.Structure):
    _fields_ = [("accepted", C.c_int64), ("rejected", C.c_int64), ("h_min", C.c_float), ("h_max", C.c_float)]


lib.dgtd_kcl_controller_default.argtypes = [C.POINTER(KclController)]
lib.dgtd_kcl_controller_default.restype = None
_sig("dgtd_mlp_create", C.c_int, _vp, _i32, _i32, _i32, C.c_uint64, C.POINTER(_vp))
lib.dgtd_mlp_destroy.argtypes = [_vp]
lib.dgtd_mlp_destroy.restype = None
_sig("dgtd_mlp_n_params", C.c_int, _vp, C.POINTER(_i64))
_sig("dgtd_mlp_get_params", C.c_int, _vp, _pf)
_sig("dgtd_mlp_set_params", C.c_int, _vp, _pf)
_sig("dgtd_mlp_forward", C.c_int, _vp, _pf, _i64, _pf)
_sig("dgtd_mlp_gradient", C.c_int, _vp, _pf, _pf, _i64, _pf, C.POINTER(_f32))
_sig("dgtd_mlp_train", C.c_int, _vp, _pf, _pf, _i64, _i32, _f32, _pf)
_sig("dgtd_etd_step_est", C.c_int, _vp, _pd, _pd, _f64, _i32, _f64, _pd, C.POINTER(_i32), C.POINTER(_f64))
_sig("dgtd_lserk_stage", C.c_int, _vp, _f32, _i32, C.c_int, _i64, _f32)
_sig("dgtd_lserk_stage_range", C.c_int, _vp, _f32, _i32, _i64, _i64, _i32, C.c_int, _i64, _f32)
_sig("dgtd_state_gather_elements", C.c_int, _vp, _vp, _i64, _vp)
_sig("dgtd_state_scatter_elements", C.c_int, _vp, _vp, _i64, _vp)
_sig("dgtd_kcl_step", C.c_int, _vp, _pd, _f64, _pd, _pd)
_sig("dgtd_transient_kcl", C.c_int, _vp, _pf, _f32, _i64, C.c_int, _i64, _vp, _vp, C.POINTER(KclController),
     C.c_int, _vp, C.POINTER(KclStats))
_sig("dgtd_transient_kcl_functionals", C.c_int, _vp, _pf, _f32, _i64, C.c_int, _i64, _vp, _vp,
     C.POINTER(KclController), _i64, _vp, _vp, _vp, _vp, _vp, C.POINTER(KclStats))
_sig("dgtd_kcl_accepted_steps", C.c_int, _vp, _pf, _pi, _i64, C.POINTER(_i64))
_sig("dgtd_transient_functionals", C.c_int, _vp, _pf, _f32, _i64, _i64, C.c_int, _i64, _vp, _vp, _i64,
     _vp, _vp, _vp, _vp, _vp)
_sig("dgtd_expmv", C.c_int, _vp, _pd, _f64, _i32, _f64, _pd, C.POINTER(_i32))
_sig("dgtd_etd_step", C.c_int, _vp, _pd, _pd, _f64, _i32, _f64, _pd, C.POINTER(_i32))
_sig("dgtd_etd_step_poly", C.c_int, _vp, _pd, _pd, _i32, _pd, _f64, _i32, _f64, _pd, C.POINTER(_i32),
     C.POINTER(_f64))
_sig("dgtd_op_set_krylov_precision", C.c_int, _vp, C.c_int)
_sig("dgtd_etd_try", C.c_int, _vp, _f64, _i32, _f64, _i32, _vp, C.c_int, _i64, C.POINTER(_i32), C.POINTER(_f64))
_sig("dgtd_etd_commit", C.c_int, _vp)
HALO_HOOK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p)
SUM_HOOK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64)
_sig("dgtd_op_set_partition", C.c_int, _vp, _i64, _vp, _vp, _vp)
_sig("dgtd_vec_gather_elements", C.c_int, _vp, _vp, _vp, _i64, _vp)
_sig("dgtd_vec_scatter_elements", C.c_int, _vp, _vp, _vp, _i64, _vp)
_sig("dgtd_op_set_functionals", C.c_int, _vp, _i64, _pl, _vp, _vp, _i64)
_sig("dgtd_record_functionals", C.c_int, _vp, _i64)
_sig("dgtd_functional_series", C.c_int, _vp, _i64, _pd)
_sig("dgtd_state_upload", C.c_int, _vp, _pf)
_sig("dgtd_state_download", C.c_int, _vp, _pf)
_sig("dgtd_state_load_device", C.c_int, _vp, _vp)
_sig("dgtd_state_store_device", C.c_int, _vp, _vp)
_sig("dgtd_run_lserk", C.c_int, _vp, _f32, _i64, C.c_int, _i64, _vp)
_sig("dgtd_run_lserk_stages", C.c_int, _vp, _f32, _i64, C.c_int, _i64, _vp)
_sig("dgtd_set_source_vector", C.c_int, _vp, _pd)
_sig("dgtd_apply_device", C.c_int, _vp, _vp, _vp)
_sig("dgtd_op_launch_count", C.c_int, _vp, C.POINTER(_i64))
_sig("dgtd_op_reset_launch_count", C.c_int, _vp)
_sig("dgtd_debug_expm", C.c_int, _vp, _pd, _i32, _pd)
_sig("dgtd_debug_tc_gemm", C.c_int, _vp, _pf, _pf, _pf, _i32, _i32, _i32)
_sig("dgtd_debug_wait_timeout", C.c_int, _vp, _i64, C.POINTER(_f64))
_sig("dgtd_cfl_dt", C.c_int, _vp, C.POINTER(_f64), C.POINTER(_f64), C.POINTER(_f64))
_sig("dgtd_power_rho", C.c_int, _vp, _i32, C.POINTER(_f64))
_sig("dgtd_field_energy", C.c_int, _vp, _pd, C.POINTER(_f64))
_sig("dgtd_state_energy", C.c_int, _vp, C.POINTER(_f64))
# host side
_sig("dgtd_mesh_box", C.c_int, _i32, _i32, _i32, _f64, _f64, _f64, _pd, _pi)
_sig("dgtd_mesh_box_jittered", C.c_int, _i32, _i32, _i32, _f64, _f64, _f64, _f64, _u64, _pd, _pi)
_sig("dgtd_mesh_box_graded_z", C.c_int, _i32, _i32, _i32, _f64, _f64, _f64, _f64, _pd, _pi)
_sig("dgtd_host_op_build", C.c_int, _pd, _i64, _pi, _i64, _i32, _f64, _vp, _vp, C.POINTER(_vp))
_sig("dgtd_host_op_destroy", C.c_int, _vp)
_sig("dgtd_host_op_link_periodic", C.c_int, _vp, _pl, _i64, _pl, _i64)
_sig("dgtd_host_op_desc", C.c_int, _vp, C.POINTER(OpDesc))
_sig("dgtd_host_op_info", C.c_int, _vp, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i64), C.POINTER(_i64))
_sig("dgtd_host_op_get", C.c_int, _vp, C.c_char_p, _pd)
_sig("dgtd_host_node_coords", C.c_int, _vp, _pd)
_sig("dgtd_host_nearest_node_dof", C.c_int, _vp, _pd, _i32, _i32, C.POINTER(_i64))
_sig("dgtd_host_port_n_faces", C.c_int, _vp, _i32, C.POINTER(_i64))
_sig("dgtd_host_rect_port_profiles", C.c_int, _vp, _i32, _pd, _i32, _i32, _pd)
_sig("dgtd_host_port_source", C.c_int, _vp, _i32, _pd, _pd)
_sig("dgtd_host_port_modal_weights", C.c_int, _vp, _i32, _pd, _i32, _pl, _pd)


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib.dgtd_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != DGTD_OK:
        msg = last_error()
        if status == 5:
            raise NoDeviceError(status, msg)
        raise DgtdError(status, msg)


def version() -> str:
    return lib.dgtd_version().decode()


def ptr(a) -> int | None:
    return None if a is None else a.ctypes.data
