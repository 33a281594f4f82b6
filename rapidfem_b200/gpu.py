"""The device operator: Python face of include/dgtd.h.

``GpuContext`` and ``GpuOperator`` keep the names, argument meaning and error
behaviour of crates/rapidfem-td/src/gpu/mod.rs:49-135 and
gpu/operator.rs:207-1486 (``new``, ``n_dof``, ``apply``, ``transient``,
``expmv``, ``etd_step``).  Where the reference returns ``Err(String)`` these
raise :class:`rapidfem_b200._native.DgtdError`; length mismatches the reference
asserts on raise ``ValueError``.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import check, lib
from .operator import MaxwellOperator


class GpuContext:
    """GpuContext::new (gpu/mod.rs:49): the CUDA device and its stream."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.dgtd_ctx_create(int(device), C.byref(h)))
        self._h = h
        buf = C.create_string_buffer(256)
        check(lib.dgtd_ctx_device_name(h, buf, 256))
        self.device_name = buf.value.decode()
        self.device = device
        self.fp64 = True

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:  # lib is None at interpreter shutdown
            lib.dgtd_ctx_destroy(h)
            self._h = C.c_void_p()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_handle: int | None) -> None:
        """Issue work on an external cudaStream_t (e.g. torch's ``stream.cuda_stream``)."""
        check(lib.dgtd_ctx_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None))

    def synchronize(self) -> None:
        check(lib.dgtd_ctx_synchronize(self._h))

    def expm(self, a) -> np.ndarray:
        """Dense exp(A), d <= 64, on the device (the Krylov finisher's kernel)."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        out = np.zeros_like(a)
        check(lib.dgtd_debug_expm(self._h, a.ravel(), a.shape[0], out.ravel()))
        return out

    def wait_timeout_probe(self, max_polls: int) -> float:
        """Run the kernels' bounded wait on a barrier nothing arrives on
        (dgtd_debug_wait_timeout); raises DgtdError (TIMEOUT) once it gives
        up after `max_polls` polls, with the seconds waited as `waited_s` on
        the exception."""
        waited = C.c_double(0.0)
        st = lib.dgtd_debug_wait_timeout(self._h, int(max_polls), C.byref(waited))
        try:
            check(st)
        except nat.DgtdError as e:
            e.waited_s = waited.value
            raise
        return waited.value


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32).ravel()


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64).ravel()


class GpuOperator:
    """GpuOperator::new (gpu/operator.rs:207): the operator resident on the device."""

    def __init__(self, ctx: GpuContext, op: MaxwellOperator, dt_scale=None, inv_eps=None):
        """`dt_scale[K]` (optional): a per-element multiplier of the LSERK4 step,
        for a batch of independent instances that step with their own dt.
        `inv_eps[K,3]` (optional): replaces the host operator's 1/eps, for
        lossless material variants of one mesh (the host operator's sigma/eps
        is kept as it is)."""
        self.ctx = ctx
        self.host_op = op
        d = op.desc()
        if dt_scale is not None:
            ds = np.ascontiguousarray(dt_scale, dtype=np.float64).ravel()
            if ds.size != op.n_elem:
                raise ValueError("dt_scale needs one entry per element")
            d.dt_scale = ds.ctypes.data
        if inv_eps is not None:
            ie = np.ascontiguousarray(inv_eps, dtype=np.float64).ravel()
            if ie.size != 3 * op.n_elem:
                raise ValueError("inv_eps needs three entries per element")
            d.inv_eps = ie.ctypes.data
        h = C.c_void_p()
        check(lib.dgtd_op_create(ctx.handle, C.byref(d), C.byref(h)))
        self._h = h
        n = C.c_int64()
        check(lib.dgtd_op_n_dof(h, C.byref(n)))
        self._n = n.value
        self.order = op.order

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:  # lib is None at interpreter shutdown
            lib.dgtd_op_destroy(h)
            self._h = C.c_void_p()

    @property
    def handle(self):
        return self._h

    def n_dof(self) -> int:
        return self._n

    def set_engine(self, engine: int) -> None:
        check(lib.dgtd_op_set_engine(self._h, int(engine)))

    @property
    def engine(self) -> int:
        e = C.c_int()
        check(lib.dgtd_op_get_engine(self._h, C.byref(e)))
        return e.value

    def check_error(self) -> None:
        """Synchronise and raise DgtdError (TIMEOUT) if a tensor-core kernel of
        this op gave up a bounded wait since the last check."""
        check(lib.dgtd_op_check_error(self._h))

    def launch_count(self) -> int:
        c = C.c_int64()
        check(lib.dgtd_op_launch_count(self._h, C.byref(c)))
        return c.value

    def reset_launch_count(self) -> None:
        check(lib.dgtd_op_reset_launch_count(self._h))

    def _check_len(self, what, a):
        if a.size != self._n:
            raise ValueError(f"{what} has {a.size} entries, expected n_dof = {self._n}")

    def apply(self, y) -> np.ndarray:
        """dy = A*y in f32 (gpu/operator.rs:513)."""
        y = _f32(y)
        self._check_len("state", y)
        dy = np.empty_like(y)
        check(lib.dgtd_apply(self._h, y, dy))
        return dy

    def apply_f64(self, y) -> np.ndarray:
        """dy = A*y in f64 on the device (the FP64 path; rhs.rs:1246's arithmetic)."""
        y = _f64(y)
        self._check_len("state", y)
        dy = np.empty_like(y)
        check(lib.dgtd_apply_f64(self._h, y, dy))
        return dy

    def transient_f64(self, y0, dt, steps, substeps=1, drive=None, g=None, record=False) -> np.ndarray:
        """LSERK4 transient in f64 on the device (explicit.rs:100-135): as
        `transient`, with f64 state, step and waveform."""
        y0 = _f64(y0)
        self._check_len("state", y0)
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            self._check_len("source", vec)
        substeps = max(int(substeps), 1)
        gs = None
        if kind != nat.DRIVE_FREE:
            gs = _f64(g)
            if gs.size != steps * substeps:
                raise ValueError("wrong number of waveform samples")
        out = np.empty(((steps + 1) * self._n) if record else self._n, dtype=np.float64)
        check(lib.dgtd_transient_f64(self._h, y0, float(dt), int(steps), substeps, kind, dof, nat.ptr(vec),
                                     nat.ptr(gs), 1 if record else 0, out))
        return out.reshape(steps + 1, self._n) if record else out

    def transient_f64_stages(self, y0, dt, steps, substeps=1, drive=None, g=None, record=False) -> np.ndarray:
        """As transient_f64 with g sampled at the LSERK4 stage times: 5 samples
        per substep (sources.stage_samples)."""
        y0 = _f64(y0)
        self._check_len("state", y0)
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            self._check_len("source", vec)
        substeps = max(int(substeps), 1)
        gs = None
        if kind != nat.DRIVE_FREE:
            gs = _f64(g)
            if gs.size != 5 * steps * substeps:
                raise ValueError("need 5 waveform samples per substep")
        out = np.empty(((steps + 1) * self._n) if record else self._n, dtype=np.float64)
        check(lib.dgtd_transient_f64_stages(self._h, y0, float(dt), int(steps), substeps, kind, dof, nat.ptr(vec),
                                            nat.ptr(gs), 1 if record else 0, out))
        return out.reshape(steps + 1, self._n) if record else out

    @staticmethod
    def _drive(drive):
        """drive: None | ('point', dof) | ('vector', b)."""
        if drive is None:
            return nat.DRIVE_FREE, 0, None
        kind, arg = drive
        if kind == "point":
            return nat.DRIVE_POINT, int(arg), None
        if kind == "vector":
            return nat.DRIVE_VECTOR, 0, None if arg is None else _f64(arg)
        raise ValueError(f"unknown drive {kind!r}")

    def transient(self, y0, dt, steps, substeps=1, drive=None, g=None, record=False) -> np.ndarray:
        """LSERK4 transient (gpu/operator.rs:906): `steps` frames of `dt`, each
        `substeps` steps of dt/substeps, source held per substep."""
        y0 = _f32(y0)
        self._check_len("state", y0)
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            self._check_len("source", vec)
        substeps = max(int(substeps), 1)
        gs = None
        if kind != nat.DRIVE_FREE:
            gs = _f32(g)
            if gs.size != steps * substeps:
                raise ValueError("wrong number of waveform samples")
        out = np.empty(((steps + 1) * self._n) if record else self._n, dtype=np.float32)
        check(lib.dgtd_transient(self._h, y0, float(dt), int(steps), substeps, kind, dof, nat.ptr(vec),
                                 nat.ptr(gs), 1 if record else 0, out))
        return out.reshape(steps + 1, self._n) if record else out

    def transient_probes(self, y0, dt, steps, substeps=1, drive=None, g=None, probes=(), y_final=None):
        """As transient, recording `probes` per frame; returns (series[steps+1, P], y_final).
        `y_final`, if given, is a caller-owned contiguous float32 array of n_dof
        values that receives the final state (page-locked memory makes the
        download a direct DMA)."""
        y0 = _f32(y0)
        self._check_len("state", y0)
        kind, dof, vec = self._drive(drive)
        substeps = max(int(substeps), 1)
        gs = None
        if kind != nat.DRIVE_FREE:
            gs = _f32(g)
            if gs.size != steps * substeps:
                raise ValueError("wrong number of waveform samples")
        pr = np.ascontiguousarray(probes, dtype=np.int64)
        series = np.empty((steps + 1) * max(pr.size, 1), dtype=np.float32)
        if y_final is None:
            yf = np.empty(self._n, dtype=np.float32)
        else:
            yf = y_final
            if not (isinstance(yf, np.ndarray) and yf.dtype == np.float32 and yf.flags.c_contiguous
                    and yf.size == self._n):
                raise ValueError(f"y_final must be a contiguous float32 array of {self._n} values")
        check(lib.dgtd_transient_probes(self._h, y0, float(dt), int(steps), substeps, kind, dof, nat.ptr(vec),
                                        nat.ptr(gs), nat.ptr(pr) if pr.size else None, pr.size,
                                        series.ctypes.data, yf.ctypes.data))
        return series[: (steps + 1) * pr.size].reshape(steps + 1, pr.size), yf

    def transient_functionals(self, y0, dt, steps, substeps=1, drive=None, g=None, functionals=()):
        """As transient, recording per frame the linear functionals
        `functionals = [(idx, w), ...]` (F(y) = sum w[k] y[idx[k]], AoS DOF
        indices) on the device in f64; returns (series[steps+1, F], y_final)."""
        y0 = _f32(y0)
        self._check_len("state", y0)
        kind, dof, vec = self._drive(drive)
        substeps = max(int(substeps), 1)
        gs = None
        if kind != nat.DRIVE_FREE:
            gs = _f32(g)
            if gs.size != steps * substeps:
                raise ValueError("wrong number of waveform samples")
        idx = [np.ascontiguousarray(i, dtype=np.int64).ravel() for i, _ in functionals]
        wts = [np.ascontiguousarray(w, dtype=np.float64).ravel() for _, w in functionals]
        for i, w in zip(idx, wts):
            if i.size != w.size:
                raise ValueError("functional index and weight arrays differ in length")
        nf = len(idx)
        ptr = np.zeros(nf + 1, dtype=np.int64)
        ptr[1:] = np.cumsum([i.size for i in idx]) if nf else []
        all_i = np.concatenate(idx) if nf else np.zeros(0, dtype=np.int64)
        all_w = np.concatenate(wts) if nf else np.zeros(0, dtype=np.float64)
        series = np.empty((steps + 1) * max(nf, 1), dtype=np.float64)
        yf = np.empty(self._n, dtype=np.float32)
        check(lib.dgtd_transient_functionals(self._h, y0, float(dt), int(steps), substeps, kind, dof, nat.ptr(vec),
                                             nat.ptr(gs), nf, nat.ptr(ptr) if nf else None,
                                             nat.ptr(all_i) if all_i.size else None,
                                             nat.ptr(all_w) if all_w.size else None,
                                             series.ctypes.data, yf.ctypes.data))
        return series[: (steps + 1) * nf].reshape(steps + 1, nf), yf

    def etd_step_est(self, y, b, h, m, tol):
        """ETD step with its a-posteriori Krylov estimate: (out, dim_used, est)."""
        y = _f64(y)
        b = _f64(b)
        self._check_len("state", y)
        self._check_len("source", b)
        out = np.empty_like(y)
        dim = C.c_int32()
        est = C.c_double()
        self._hook_check(lib.dgtd_etd_step_est(self._h, y, b, float(h), int(m), float(tol), out, C.byref(dim),
                                               C.byref(est)))
        return out, dim.value, est.value

    def lserk_stage(self, h, stage, drive=None, g=0.0):
        """One fused LSERK4 stage on the resident state (drivers that act between
        stages, e.g. a partitioned run's halo exchange)."""
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            raise ValueError("set a vector drive with set_source_vector first and pass ('vector', None)")
        check(lib.dgtd_lserk_stage(self._h, float(h), int(stage), kind, dof, float(g)))

    def lserk_stage_range(self, h, stage, e_begin, e_end, flip, drive=None, g=0.0):
        """One fused LSERK4 stage on elements [e_begin, e_end) of the resident
        state (dgtd_lserk_stage_range); `flip` on the last range of a stage."""
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            raise ValueError("set a vector drive with set_source_vector first and pass ('vector', None)")
        check(lib.dgtd_lserk_stage_range(self._h, float(h), int(stage), int(e_begin), int(e_end),
                                         1 if flip else 0, kind, dof, float(g)))

    def gather_elements(self, d_elems: int, n: int, d_buf: int) -> None:
        """Element blocks (6*Np f32) of the resident state into a device buffer."""
        check(lib.dgtd_state_gather_elements(self._h, d_elems, int(n), d_buf))

    def scatter_elements(self, d_elems: int, n: int, d_buf: int) -> None:
        """A device buffer of element blocks into the resident state."""
        check(lib.dgtd_state_scatter_elements(self._h, d_elems, int(n), d_buf))

    def gather_vec_elements(self, d_vec: int, d_elems: int, n: int, d_buf: int) -> None:
        """Element blocks of a device vector in the state layout into a device buffer."""
        check(lib.dgtd_vec_gather_elements(self._h, d_vec, d_elems, int(n), d_buf))

    def scatter_vec_elements(self, d_vec: int, d_elems: int, n: int, d_buf: int) -> None:
        """A device buffer of element blocks into a device vector in the state layout."""
        check(lib.dgtd_vec_scatter_elements(self._h, d_vec, d_elems, int(n), d_buf))

    def set_partition(self, n_owned: int, halo=None, reduce=None) -> None:
        """Make the op one part of an element partition for its Krylov / ETD
        entry points (dgtd_op_set_partition): dots and norms over the first
        n_owned elements, `halo(d_vec)` refreshing a device vector's halo blocks
        before each matvec and `reduce(d_partials, count)` summing f64 partials
        over all parts in place.  n_owned = 0 restores the undivided op.  An
        exception in a hook fails the entry point that called it and is
        re-raised there."""
        if int(n_owned) == 0:
            check(lib.dgtd_op_set_partition(self._h, 0, None, None, None))
            self._part_hooks = None
            return
        errors = []

        def on_halo(_user, d_vec):
            try:
                halo(int(d_vec))
                return 0
            except BaseException as e:  # noqa: BLE001 - carried to the caller
                errors.append(e)
                return 1

        def on_sum(_user, d_buf, count):
            try:
                reduce(int(d_buf), int(count))
                return 0
            except BaseException as e:  # noqa: BLE001
                errors.append(e)
                return 1

        hooks = (nat.HALO_HOOK(on_halo), nat.SUM_HOOK(on_sum), errors)
        check(lib.dgtd_op_set_partition(self._h, int(n_owned), C.cast(hooks[0], C.c_void_p),
                                        C.cast(hooks[1], C.c_void_p), None))
        self._part_hooks = hooks  # the C side keeps the function pointers

    def _hook_check(self, status: int) -> None:
        hooks = getattr(self, "_part_hooks", None)
        if status != nat.DGTD_OK and hooks is not None and hooks[2]:
            err = hooks[2].pop(0)
            hooks[2].clear()
            raise RuntimeError("a partition hook failed") from err
        check(status)

    def kcl_step(self, y, h):
        """One KCL RK4(3)5 step (explicit_adaptive.rs:84-152): (y_new, err)."""
        y = _f64(y)
        self._check_len("state", y)
        out = np.empty_like(y)
        err = np.empty_like(y)
        check(lib.dgtd_kcl_step(self._h, y, float(h), out, err))
        return out, err

    @staticmethod
    def kcl_controller(**overrides):
        """Controller::default (session.rs:145-158) with keyword overrides."""
        c = nat.KclController()
        lib.dgtd_kcl_controller_default(C.byref(c))
        for k, v in overrides.items():
            if not hasattr(c, k):
                raise ValueError(f"unknown controller setting {k!r}")
            setattr(c, k, float(v))
        return c

    def _kcl_common(self, y0, steps, drive, g, controller):
        y0 = _f32(y0)
        self._check_len("state", y0)
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            self._check_len("source", vec)
        gs = None
        if kind != nat.DRIVE_FREE:
            gs = _f32(g)
            if gs.size != steps:
                raise ValueError("a KCL run takes one waveform sample per output frame")
        ctl = controller if controller is not None else self.kcl_controller()
        return y0, kind, dof, vec, gs, ctl

    def transient_kcl(self, y0, dt, steps, drive=None, g=None, controller=None, record=True):
        """KCL RK4(3)5 adaptive transient (gpu/operator.rs:823) with the PI
        controller on the device.  Returns (trajectory[steps+1, n] or final
        state, stats dict with accepted, rejected, h_min, h_max)."""
        y0, kind, dof, vec, gs, ctl = self._kcl_common(y0, steps, drive, g, controller)
        out = np.empty(((steps + 1) if record else 1) * self._n, dtype=np.float32)
        st = nat.KclStats()
        check(lib.dgtd_transient_kcl(self._h, y0, float(dt), int(steps), kind, dof, nat.ptr(vec), nat.ptr(gs),
                                     C.byref(ctl), 1 if record else 0, out.ctypes.data, C.byref(st)))
        stats = {"accepted": st.accepted, "rejected": st.rejected, "h_min": st.h_min, "h_max": st.h_max}
        return (out.reshape(steps + 1, self._n) if record else out), stats

    def kcl_accepted_steps(self):
        """The accepted substeps of the last adaptive run: (h[n], frame[n]),
        the step sizes in order and the output frame each one advanced."""
        n = C.c_int64()
        check(lib.dgtd_kcl_accepted_steps(self._h, np.zeros(1, np.float32), np.zeros(1, np.int32), 0,
                                          C.byref(n)))
        cap = min(n.value, 1 << 16)
        h = np.zeros(max(cap, 1), dtype=np.float32)
        fr = np.zeros(max(cap, 1), dtype=np.int32)
        check(lib.dgtd_kcl_accepted_steps(self._h, h, fr, cap, C.byref(n)))
        if n.value > cap:
            raise RuntimeError(f"the run accepted {n.value} substeps; the device log holds {cap}")
        return h[:cap], fr[:cap]

    def transient_kcl_functionals(self, y0, dt, steps, drive=None, g=None, controller=None, functionals=()):
        """As transient_kcl, recording per frame the linear functionals
        [(idx, w), ...] on the device; returns (series[steps+1, F], y_final, stats)."""
        y0, kind, dof, vec, gs, ctl = self._kcl_common(y0, steps, drive, g, controller)
        idx = [np.ascontiguousarray(i, dtype=np.int64).ravel() for i, _ in functionals]
        wts = [np.ascontiguousarray(w, dtype=np.float64).ravel() for _, w in functionals]
        nf = len(idx)
        ptr = np.zeros(nf + 1, dtype=np.int64)
        ptr[1:] = np.cumsum([i.size for i in idx]) if nf else []
        all_i = np.concatenate(idx) if nf else np.zeros(0, dtype=np.int64)
        all_w = np.concatenate(wts) if nf else np.zeros(0, dtype=np.float64)
        series = np.empty((steps + 1) * max(nf, 1), dtype=np.float64)
        yf = np.empty(self._n, dtype=np.float32)
        st = nat.KclStats()
        check(lib.dgtd_transient_kcl_functionals(self._h, y0, float(dt), int(steps), kind, dof, nat.ptr(vec),
                                                 nat.ptr(gs), C.byref(ctl), nf, nat.ptr(ptr) if nf else None,
                                                 nat.ptr(all_i) if all_i.size else None,
                                                 nat.ptr(all_w) if all_w.size else None,
                                                 series.ctypes.data, yf.ctypes.data, C.byref(st)))
        stats = {"accepted": st.accepted, "rejected": st.rejected, "h_min": st.h_min, "h_max": st.h_max}
        return series[: (steps + 1) * nf].reshape(steps + 1, nf), yf, stats

    def expmv(self, v, t, m, tol=0.0):
        """exp(t*A)*v (gpu/operator.rs:1175); returns (out, dim_used)."""
        v = _f64(v)
        self._check_len("state", v)
        if m < 1:
            raise ValueError("Krylov dimension must be >= 1")
        out = np.empty_like(v)
        dim = C.c_int32()
        self._hook_check(lib.dgtd_expmv(self._h, v, float(t), int(m), float(tol), out, C.byref(dim)))
        return out, dim.value

    def etd_step(self, y, b, h, m, tol=0.0):
        """exp(hA)y + h*phi1(hA)b (gpu/operator.rs:1267); returns (out, dim_used)."""
        y = _f64(y)
        b = _f64(b)
        self._check_len("state", y)
        self._check_len("source", b)
        if m < 1:
            raise ValueError("Krylov dimension must be >= 1")
        out = np.empty_like(y)
        dim = C.c_int32()
        self._hook_check(lib.dgtd_etd_step(self._h, y, b, float(h), int(m), float(tol), out, C.byref(dim)))
        return out, dim.value

    def etd_step_poly(self, y, b, coef, h, m, tol=0.0):
        """ETD step with the source b*g(t0+tau), g(t0+tau) = sum_k coef[k] tau^k:
        (out, dim_used, est)."""
        y = _f64(y)
        b = _f64(b)
        a = _f64(coef)
        self._check_len("state", y)
        self._check_len("source", b)
        out = np.empty_like(y)
        dim = C.c_int32()
        est = C.c_double()
        self._hook_check(lib.dgtd_etd_step_poly(self._h, y, b, a.size, a, float(h), int(m), float(tol), out,
                                                C.byref(dim), C.byref(est)))
        return out, dim.value, est.value

    def set_krylov_precision(self, bits: int) -> None:
        """32: f32 basis on the op's engine (default); 64: f64 basis and FP64 matvec."""
        check(lib.dgtd_op_set_krylov_precision(self._h, int(bits)))

    def etd_try(self, h, m, tol=0.0, coef=None, drive=None):
        """ETD step candidate from the resident state (see dgtd_etd_try):
        returns (dim_used, est); `etd_commit` accepts it."""
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            raise ValueError("set a vector drive with set_source_vector first and pass ('vector', None)")
        a = None if coef is None else _f64(coef)
        dim = C.c_int32()
        est = C.c_double()
        self._hook_check(lib.dgtd_etd_try(self._h, float(h), int(m), float(tol), 0 if a is None else a.size,
                                          nat.ptr(a), kind, dof, C.byref(dim), C.byref(est)))
        return dim.value, est.value

    def etd_commit(self) -> None:
        check(lib.dgtd_etd_commit(self._h))

    # ---- device-resident state
    def upload(self, y) -> None:
        y = _f32(y)
        self._check_len("state", y)
        check(lib.dgtd_state_upload(self._h, y))

    def download(self) -> np.ndarray:
        out = np.empty(self._n, dtype=np.float32)
        check(lib.dgtd_state_download(self._h, out))
        return out

    def load_device(self, dptr: int) -> None:
        check(lib.dgtd_state_load_device(self._h, C.c_void_p(dptr)))

    def store_device(self, dptr: int) -> None:
        check(lib.dgtd_state_store_device(self._h, C.c_void_p(dptr)))

    def set_source_vector(self, b) -> None:
        b = _f64(b)
        self._check_len("source", b)
        check(lib.dgtd_set_source_vector(self._h, b))

    def run_lserk(self, h, steps, drive=None, g=None) -> None:
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            self.set_source_vector(vec)
        gs = None
        if kind != nat.DRIVE_FREE:
            gs = _f32(g)
            if gs.size != steps:
                raise ValueError("wrong number of waveform samples")
        check(lib.dgtd_run_lserk(self._h, float(h), int(steps), kind, dof, nat.ptr(gs)))

    def run_lserk_stages(self, h, steps, drive=None, g_stages=None) -> None:
        """`steps` LSERK4 steps on the resident state with the waveform sampled
        at the stage times (5 per step, sources.stage_samples)."""
        kind, dof, vec = self._drive(drive)
        if vec is not None:
            self.set_source_vector(vec)
        gs = None
        if kind != nat.DRIVE_FREE:
            gs = _f32(g_stages)
            if gs.size != 5 * steps:
                raise ValueError("need 5 waveform samples per step")
        check(lib.dgtd_run_lserk_stages(self._h, float(h), int(steps), kind, dof, nat.ptr(gs)))

    def set_functionals(self, functionals, max_rows: int) -> None:
        """Functionals [(idx, w), ...] (F(y) = sum w[k] y[idx[k]], AoS DOF
        indices) to record on the resident state, with room for max_rows rows."""
        idx = [np.ascontiguousarray(i, dtype=np.int64).ravel() for i, _ in functionals]
        wts = [np.ascontiguousarray(w, dtype=np.float64).ravel() for _, w in functionals]
        if not idx:
            raise ValueError("no functionals")
        for i, w in zip(idx, wts):
            if i.size != w.size:
                raise ValueError("functional index and weight arrays differ in length")
        ptr = np.zeros(len(idx) + 1, dtype=np.int64)
        ptr[1:] = np.cumsum([i.size for i in idx])
        self._fn_keep = (np.concatenate(idx), np.concatenate(wts))
        self._n_fun = len(idx)
        check(lib.dgtd_op_set_functionals(self._h, len(idx), ptr, nat.ptr(self._fn_keep[0]),
                                          nat.ptr(self._fn_keep[1]), int(max_rows)))

    def record_functionals(self, row: int) -> None:
        """The functionals of the current state into row `row` (no synchronisation)."""
        check(lib.dgtd_record_functionals(self._h, int(row)))

    def functional_series(self, n_rows: int) -> np.ndarray:
        out = np.empty(int(n_rows) * self._n_fun, dtype=np.float64)
        check(lib.dgtd_functional_series(self._h, int(n_rows), out))
        return out.reshape(int(n_rows), self._n_fun)

    def apply_device(self, d_y: int, d_dy: int) -> None:
        check(lib.dgtd_apply_device(self._h, C.c_void_p(d_y), C.c_void_p(d_dy)))
