"""The time-domain session and problem API on the B200 path.

``TdSession`` mirrors ``PyTdSession`` (python/src/td.rs:163-426) and
``ProblemTD`` mirrors rapidfem.problem.td.ProblemTD (problem/td.py:195-750)
for the parts on the DGTD hot path: the operator, ``apply``, the Krylov
``step``, ``step_explicit``, ``cfl_dt``, ``nearest_node_dof``, ``field_energy``
and ``transient`` with point / port drives and probes, for the exponential and
explicit (LSERK4) integrators.  Runs go to the GPU; ``device="cpu"`` is refused
(there is no CPU path in this package).  The run logic follows
TdSession::transient (crates/rapidfem-td/src/session.rs:620-777): LSERK4 is
sub-stepped to the CFL limit with the source held per substep, the exponential
integrator takes one ETD step per frame with the source held per frame.
"""
from __future__ import annotations

import math
import sys

import numpy as np

from . import gpu as G
from . import operator as O

C_LIGHT = 299_792_458.0
RESONANCE_STATIC_FRACTION = 1e-3  # constants.rs:305: modes below this share of max |Im| are static
RESONANCE_MERGE_REL = 1e-3        # constants.rs:308: resonances this close (relative) are one
TRANSFER_BAND_FRACTION = 1e-2     # constants.rs:313: H is zero where |G| is below this share of its peak
KRYLOV_TOL = 1e-10
_CTX = {}


def _log(verbose, msg):
    if verbose:
        print(f"  [rapidfem-td] {msg}", file=sys.stderr, flush=True)


def _ctx(device_index=0):
    if device_index not in _CTX:
        _CTX[device_index] = G.GpuContext(device_index)
    return _CTX[device_index]


def flux_alpha(flux: str) -> float:
    """session.rs:93-99."""
    if flux == "upwind":
        return 1.0
    if flux == "central":
        return 0.0
    raise ValueError(f"flux must be one of ['central', 'upwind'], got {flux!r}")


class GaussianPulse:
    """g(t) = exp(-((t-t0)/tau)^2) * cos(2 pi f0 (t-t0)) (session.rs:242-261)."""

    def __init__(self, t0, tau, f0=None):
        self.t0, self.tau, self.f0 = float(t0), float(tau), None if f0 is None else float(f0)

    def __call__(self, t):
        t = np.asarray(t, dtype=np.float64)
        x = (t - self.t0) / self.tau
        env = np.exp(-(x * x))
        if self.f0 is None:
            return env
        return env * np.cos(2.0 * np.pi * self.f0 * (t - self.t0))


def _sample(waveform, t):
    try:
        v = waveform(np.asarray(t, dtype=np.float64))
        v = np.asarray(v, dtype=np.float64)
        if v.shape == np.shape(t):
            return v
    except Exception:
        pass
    return np.array([float(waveform(float(x))) for x in np.ravel(t)])


def transfer(g, r, dt):
    """The frequency response of a drive series g and a response series r of
    equal length sampled every dt (session.rs:1238-1261): the one-sided
    spectra of both (forward real FFT, length n // 2 + 1), frequencies
    k / (n dt), and H = R / G where |G| exceeds TRANSFER_BAND_FRACTION of its
    peak, zero elsewhere."""
    g = np.asarray(g, dtype=np.float64).ravel()
    r = np.asarray(r, dtype=np.float64).ravel()
    if g.size != r.size:
        raise ValueError("drive and response lengths differ")
    n = g.size
    if n == 0:
        return np.zeros(0), np.zeros(0, dtype=np.complex128)
    sg, sr = np.fft.rfft(g), np.fft.rfft(r)
    peak = float(np.max(np.abs(sg)))
    freqs = np.arange(sg.size) / (n * dt)
    band = np.abs(sg) > TRANSFER_BAND_FRACTION * peak
    h = np.zeros(sg.size, dtype=np.complex128)
    h[band] = sr[band] / sg[band]
    return freqs, h


def _distance2_colors(nbr: np.ndarray) -> np.ndarray:
    """Greedy colouring of the elements such that two elements that are face
    neighbours, or share a face neighbour, differ in colour."""
    K = nbr.shape[0]
    adj = [[int(x) for x in row if x >= 0] for row in nbr]
    color = -np.ones(K, dtype=np.int64)
    for e in range(K):
        used = set()
        for a in adj[e]:
            used.add(int(color[a]))
            for b in adj[a]:
                used.add(int(color[b]))
        k = 0
        while k in used:
            k += 1
        color[e] = k
    return color


class TdSession:
    """The DGTD operator on the GPU with its steppers and runs (td.rs:163)."""

    def __init__(self, op: O.MaxwellOperator, c: float = 1.0, device: int = 0, ports=None):
        self.op = op
        self.c = float(c)
        self.ctx = _ctx(device)
        self.gop = G.GpuOperator(self.ctx, op)
        self._cfl_h = None
        self._ports = ports or {}

    # ---- construction (td.rs:191-208)
    @staticmethod
    def box_cavity(nx, ny, nz, lx, ly, lz, order, flux="upwind", c=1.0):
        mesh = O.structured_box(nx, ny, nz, lx, ly, lz)
        return TdSession(O.MaxwellOperator(mesh, order, flux_alpha(flux)), c)

    @staticmethod
    def from_mesh(mesh: O.Mesh, order, flux="upwind", c=1.0, materials=None, ports=None):
        """An operator on an arbitrary tet mesh.  `ports` maps a port name to
        {"faces": bool [K,4], "inward_normal": (x,y,z), "mode": (m,n) or None}."""
        face_port = None
        port_ids = {}
        if ports:
            face_port = -np.ones((mesh.n_tets, 4), dtype=np.int32)
            for k, (name, spec) in enumerate(ports.items()):
                face_port[np.asarray(spec["faces"], dtype=bool)] = k
                port_ids[name] = (k, spec)
        op = O.MaxwellOperator(mesh, order, flux_alpha(flux), face_port=face_port, materials=materials)
        return TdSession(op, c, ports=port_ids)

    @staticmethod
    def from_model(tagged_mesh, model, order, flux="upwind", c=1.0):
        """TdSession::from_model (td.rs:203, build.rs:74-259): the operator of a
        `model.Model` on a `model.TaggedMesh`.  Ports are named by their face
        tag; a rectangular port's inward normal is the mean inward normal of
        its faces."""
        from . import model as M

        mo = M.operator_from_model(tagged_mesh, model, order, flux_alpha(flux), c)
        normals = mo.op.get("normal").reshape(-1, 4, 3)
        ports = {}
        for k, (tag, mode) in enumerate(zip(mo.port_tags, mo.port_modes)):
            faces = mo.face_port == k
            n_out = normals[faces].mean(axis=0)
            n_in = -n_out / max(np.linalg.norm(n_out), 1e-300)
            ports[tag] = (k, {"faces": faces, "inward_normal": tuple(n_in), "mode": mode})
        sess = TdSession(mo.op, c, ports=ports)
        sess.model_operator = mo
        return sess

    # ---- sizes
    def n_dofs(self) -> int:
        return self.op.n_dof

    def n_tets(self) -> int:
        return self.op.n_elem

    def gpu_available(self) -> bool:
        return True

    def _check(self, what, y):
        y = np.ascontiguousarray(y, dtype=np.float64).ravel()
        if y.size != self.n_dofs():
            raise ValueError(f"{what} has {y.size} entries, expected n_dof = {self.n_dofs()}")
        return y

    # ---- the ODE
    def apply(self, y) -> np.ndarray:
        """A*y (f32 on the device, returned as f64)."""
        return self.gop.apply(self._check("y", y)).astype(np.float64)

    def field_energy(self, y) -> float:
        from ._native import check, lib
        import ctypes as C
        e = C.c_double()
        check(lib.dgtd_field_energy(self.gop.handle, self._check("y", y), C.byref(e)))
        return e.value

    # ---- the assembled operator and its spectrum
    def state_space(self):
        """A as CSR (n, row_ptr, col_idx, values), td.rs:382 over
        assemble_sparse (rhs.rs:1621-1700): the operator couples an element
        only to itself and its face neighbours, so its columns are probed
        with unit vectors, the same local column of every element of one
        distance-2 colour at once (no two elements of one colour share a
        neighbour, so each output block comes from one probe), each probe one
        FP64 RHS on the device (dgtd_apply_f64); exact zeros are dropped and
        each row's columns ascend.  Memory O(nnz); n_colours * 6 Np probes."""
        nbr = self.op.get("nbr").astype(np.int64).reshape(-1, 4)
        K, bs, n = nbr.shape[0], 6 * self.op.np, self.n_dofs()
        color = _distance2_colors(nbr)
        rows, cols, vals = [], [], []
        il = np.arange(bs, dtype=np.int64)
        for col_id in range(int(color.max()) + 1):
            src = np.flatnonzero(color == col_id)
            # (output element, probed element) pairs of this colour's stencils
            sten = np.concatenate([src[:, None], nbr[src]], axis=1)
            dst = sten.ravel()
            owner = np.repeat(src, 5)
            keep = dst >= 0
            dst, owner = dst[keep], owner[keep]
            for jl in range(bs):
                probe = np.zeros(n)
                probe[src * bs + jl] = 1.0
                blk = self.gop.apply_f64(probe).reshape(K, bs)[dst]
                nz = blk != 0.0
                rows.append((dst[:, None] * bs + il[None, :])[nz])
                cols.append(np.broadcast_to((owner * bs + jl)[:, None], blk.shape)[nz])
                vals.append(blk[nz])
        r = np.concatenate(rows)
        c = np.concatenate(cols)
        v = np.concatenate(vals)
        order = np.lexsort((c, r))
        r, c, v = r[order], c[order], v[order]
        row_ptr = np.zeros(n + 1, dtype=np.int64)
        np.add.at(row_ptr, r + 1, 1)
        return n, np.cumsum(row_ptr), c.astype(np.int64), v

    def resonances(self, n: int = 8) -> np.ndarray:
        """The n lowest distinct resonances (session.rs:1007-1031): the dense
        spectrum of A, near-static modes (|Im| <= 1e-3 max |Im|) dropped, the
        least damped first, f = c |Im lambda| / 2 pi, values within 1e-3 of a
        kept one merged, returned ascending.  Dense, so for modest meshes."""
        m, row_ptr, col_idx, vals = self.state_space()
        a = np.zeros((m, m))
        a[np.repeat(np.arange(m), np.diff(row_ptr)), col_idx] = vals
        ev = np.linalg.eigvals(a)
        w_max = float(np.max(np.abs(ev.imag))) if ev.size else 0.0
        phys = ev[np.abs(ev.imag) > RESONANCE_STATIC_FRACTION * w_max]
        phys = phys[np.argsort(-phys.real, kind="stable")]
        out = []
        for z in phys:
            f = abs(z.imag) * self.c / (2.0 * math.pi)
            if any(abs(f - g) <= RESONANCE_MERGE_REL * g for g in out):
                continue
            out.append(f)
            if len(out) >= n:
                break
        return np.sort(np.array(out))

    # ---- steps
    def step(self, y, h, krylov_dim=40, tol=None):
        """exp(h A) y by the device Krylov propagator (td.rs:235-239)."""
        tol = KRYLOV_TOL if tol is None else float(tol)
        out, _ = self.gop.expmv(self._check("y", y), self.c * float(h), int(krylov_dim), tol)
        return out

    def step_explicit(self, y, h):
        """One LSERK4 step of h (td.rs:242-244)."""
        return self.gop.transient(self._check("y", y), self.c * float(h), 1, 1).astype(np.float64)

    def step_adaptive(self, y, h):
        """One KCL RK4(3)5 step of h (session.rs:499): (y_new, embedded error)."""
        out, err = self.gop.kcl_step(self._check("y", y), self.c * float(h))
        return out, err

    def cfl_dt(self, recompute=False) -> float:
        """The largest stable LSERK4 step in physical time (session.rs:514-569)."""
        if self._cfl_h is None or recompute:
            from ._native import check, lib
            import ctypes as C
            h = C.c_double()
            check(lib.dgtd_cfl_dt(self.gop.handle, C.byref(h), None, None))
            self._cfl_h = h.value
        return self._cfl_h / self.c

    def nearest_node_dof(self, point, field, component) -> int:
        f = {"E": 0, "H": 1}.get(field)
        if f is None:
            raise ValueError(f"field must be 'E' or 'H', got {field!r}")
        cpt = {"x": 0, "y": 1, "z": 2}.get(component)
        if cpt is None:
            raise ValueError(f"component must be 'x', 'y' or 'z', got {component!r}")
        return self.op.nearest_node_dof(point, f, cpt)

    def _port(self, name):
        """(index, spec) of a port of this problem; a name that is not one is
        refused (python/tests/test_td_model.py:72-78)."""
        hit = self._ports.get(name)
        if hit is None:
            raise ValueError(f"{name!r} is not a port of this problem")
        return hit

    def port_source(self, name):
        k, spec = self._port(name)
        if spec.get("mode") is None:
            return np.zeros(self.n_dofs())
        prof = self.op.rect_port_profiles(k, spec["inward_normal"], spec["mode"])
        return self.op.port_source(k, prof)

    def port_functional(self, name, which="E"):
        """P_e (or P_h) of a modal port as (idx, w) over the AoS state
        (rhs.rs:1211-1242)."""
        if name not in self._ports:
            raise ValueError(f"no port named {name!r}")
        k, spec = self._port(name)
        if spec.get("mode") is None:
            raise ValueError(f"port {name!r} is an absorbing boundary, not a modal port")
        prof = self.op.rect_port_profiles(k, spec["inward_normal"], spec["mode"])
        return self.op.port_modal_weights(k, prof, which)

    def port_signals(self, states, ports):
        """The modal amplitude P_e of each port over a row-major trajectory,
        [ports, rows] (session.rs:1041-1054)."""
        n = self.n_dofs()
        states = np.asarray(states, dtype=np.float64)
        if states.size == 0 or states.size % n:
            raise ValueError(f"the trajectory length {states.size} is not a multiple of n_dof = {n}")
        rows = states.reshape(-1, n)
        out = np.empty((len(ports), rows.shape[0]))
        for q, name in enumerate(ports):
            idx, w = self.port_functional(name)
            out[q] = rows[:, idx] @ w
        return out

    def transfer_function(self, source_dof, probe_dof, pulse, dt, steps, method=None, device="gpu",
                          krylov_dim=40, verbose=True):
        """(frequencies, H) of the field at probe_dof driven by the soft point
        source `pulse` at source_dof (td.rs:331-350, session.rs:985-999): one
        driven transient of `steps` frames from rest recording the probe, the
        drive sampled at the frame times k dt, k = 0..steps, then `transfer`."""
        frames, _ = self.transient(None, dt=dt, steps=steps, source_dof=source_dof, waveform=pulse,
                                   probes=[probe_dof], method=method, device=device, krylov_dim=krylov_dim,
                                   verbose=verbose)
        g = _sample(pulse, np.arange(steps + 1) * float(dt))
        return transfer(g, frames[:, 0], float(dt))

    # ---- runs
    def transient(self, y0=None, *, dt, steps, source_dof=None, port=None, waveform=None, probes=None,
                  port_probes=None, method=None, device="gpu", krylov_dim=40, warmup=0, verbose=True):
        """A run of `steps` frames of `dt` (td.rs:281-324, session.rs:620-777).
        Returns (frames [steps+1, n_dof, or len(probes) + len(port_probes)], None).
        `port_probes` names modal ports whose amplitude P_e is recorded per frame
        (on the device in the explicit path) after the point probes."""
        if device not in ("gpu", "cuda"):
            raise ValueError("rapidfem_b200 runs the DGTD path on the GPU only (device='gpu')")
        method = method or "explicit"
        if method not in ("exponential", "explicit", "adaptive"):
            raise ValueError("method must be 'exponential', 'explicit', or 'adaptive'")
        if method == "adaptive" and warmup > 0:
            raise ValueError("warmup is not supported with method='adaptive' (the controller "
                             "stabilises itself in the first few frames)")
        if not (math.isfinite(dt) and dt > 0.0):
            raise ValueError(f"dt must be positive, got {dt}")
        if source_dof is not None and port is not None:
            raise ValueError("pass either source= (point) or port= (modal port), not both")
        n = self.n_dofs()
        if source_dof is not None and not 0 <= source_dof < n:
            raise ValueError(f"source DOF {source_dof} out of range (n_dof = {n})")
        drive = None
        if source_dof is not None:
            drive = ("point", int(source_dof))
        elif port is not None:
            drive = ("vector", self.port_source(port))
        if drive is not None and waveform is None:
            raise ValueError("a driven run needs a waveform")
        if probes is not None:
            probes = [int(p) for p in probes]
            bad = [p for p in probes if not 0 <= p < n]
            if bad:
                raise ValueError(f"probe DOF {bad[0]} out of range (n_dof = {n})")
        funcs = [self.port_functional(p) for p in (port_probes or [])]
        if funcs and probes is None:
            probes = []
        warmup = min(int(warmup), steps)
        y = np.zeros(n) if y0 is None else self._check("y0", y0)

        def sample(v):
            v = np.asarray(v, dtype=np.float64)
            if probes is None:
                return v.copy()
            return np.concatenate([v[probes], [v[i] @ w for i, w in funcs]])

        rows = [sample(y)]

        def push(v):
            rows.append(sample(v))

        if method == "adaptive":
            # KCL RK4(3)5 with the PI controller on the device (session.rs:940-970)
            _log(verbose, "transient: KCL adaptive on the GPU (atol=1e-08, rtol=1e-04)")
            g = None
            if drive is not None:
                g = _sample(waveform, np.arange(steps) * dt)
            if probes is not None:
                fun = [(np.array([p], dtype=np.int64), np.ones(1)) for p in probes] + funcs
                series, _, st = self.gop.transient_kcl_functionals(y, self.c * dt, steps, drive=drive, g=g,
                                                                   functionals=fun)
                rows.extend(list(series[1:]))
            else:
                traj, st = self.gop.transient_kcl(y, self.c * dt, steps, drive=drive, g=g, record=True)
                rows.extend(list(traj[1:].astype(np.float64)))
            stats = (st["accepted"], st["rejected"], st["h_min"] / self.c, st["h_max"] / self.c)
            return np.array(rows), stats

        exp_frames = steps if method == "exponential" else warmup
        for k in range(exp_frames):
            g = 0.0 if drive is None else float(_sample(waveform, np.array([k * dt]))[0])
            if drive is None:
                y, _ = self.gop.expmv(y, self.c * dt, krylov_dim, KRYLOV_TOL)
            else:
                b = np.zeros(n)
                if drive[0] == "point":
                    b[drive[1]] = g
                else:
                    b = drive[1] * g
                y, _ = self.gop.etd_step(y, b, self.c * dt, krylov_dim, KRYLOV_TOL)
            push(y)
        if method == "explicit" and warmup < steps:
            nsub = max(1, math.ceil(dt / self.cfl_dt()))
            _log(verbose, f"transient: explicit LSERK4 on the GPU ({nsub} substeps/step)")
            h_sub = dt / nsub
            kk = steps - warmup
            g = None
            if drive is not None:
                t = (warmup * nsub + np.arange(kk * nsub)) * h_sub
                g = _sample(waveform, t)
            if funcs:
                fun = [(np.array([p], dtype=np.int64), np.ones(1)) for p in probes] + funcs
                series, yf = self.gop.transient_functionals(y, self.c * dt, kk, nsub, drive=drive, g=g,
                                                            functionals=fun)
                rows.extend(list(series[1:]))
                y = yf.astype(np.float64)
            elif probes is not None:
                series, yf = self.gop.transient_probes(y, self.c * dt, kk, nsub, drive=drive, g=g, probes=probes)
                rows.extend(list(series[1:].astype(np.float64)))
                y = yf.astype(np.float64)
            else:
                traj = self.gop.transient(y, self.c * dt, kk, nsub, drive=drive, g=g, record=True)
                rows.extend(list(traj[1:].astype(np.float64)))
                y = traj[-1].astype(np.float64)
        return np.array(rows), None


class TdTransfer:
    """A field-to-field frequency response (problem/td.py:140-167): iterates
    as (frequencies, H); the labels name the source and probe points."""

    def __init__(self, frequencies, H, *, source_label="", probe_label=""):
        self.frequencies = np.asarray(frequencies)
        self.H = np.asarray(H)
        self.source_label = source_label
        self.probe_label = probe_label

    def __iter__(self):
        return iter((self.frequencies, self.H))

    def __repr__(self):
        return f"TdTransfer(n_freq={self.frequencies.size})"


def _point_label(spec):
    """'E_z @ (x, y, z)' for a (point, field, component) spec (problem/td.py:101-106)."""
    p, f, c = spec
    coords = ", ".join(f"{v:g}" for v in np.asarray(p, dtype=float).ravel())
    return f"{f}_{c} @ ({coords})"


class TdTrajectory(np.ndarray):
    """A field trajectory [n_snapshot, n_dofs] (problem/td.py:170-192): an
    ndarray that also carries the problem and the frame step."""

    def __new__(cls, data, *, problem=None, dt=None):
        obj = np.ascontiguousarray(data, dtype=np.float64).view(cls)
        obj._problem = problem
        obj._dt = dt
        return obj

    def __array_finalize__(self, obj):
        if obj is None:
            return
        self._problem = getattr(obj, "_problem", None)
        self._dt = getattr(obj, "_dt", None)


class TdODE:
    """The problem as the linear ODE dy/dt = A y for an external integrator
    (problem/td.py:47-72): `rhs(t, y)` has scipy's solve_ivp signature and
    runs on the device; `jacobian()` is the assembled sparse A."""

    def __init__(self, problem):
        self._p = problem
        self.n_dofs = problem.n_dofs

    def rhs(self, t, y):
        return self._p._op.apply(y)

    def jacobian(self, t=None, y=None):
        return self._p.state_space()

    def __repr__(self):
        return f"TdODE(n_dofs={self.n_dofs})"


class TdStepper:
    """A one-step propagator bound to a fixed dt (problem/td.py:75-98): the
    exponential step, or LSERK4 sub-stepped to its stability limit."""

    def __init__(self, problem, dt, krylov_dim, method="exponential"):
        self._p = problem
        self.dt = float(dt)
        self.krylov_dim = int(krylov_dim)
        self.method = method

    def __call__(self, y):
        frames, _ = self._p._op.transient(np.asarray(y, dtype=np.float64), dt=self.dt, steps=1,
                                          method=self.method, krylov_dim=self.krylov_dim, verbose=False)
        return frames[-1]

    def __repr__(self):
        return f"TdStepper(dt={self.dt:g}, method={self.method!r})"


class ProblemTD:
    """problem/td.py:195-750 on the B200 path (box cavities and tet meshes)."""

    def __init__(self, mesh: O.Mesh, *, order=2, flux="upwind", c=C_LIGHT, materials=None, ports=None):
        self.c = float(c)
        self._op = TdSession.from_mesh(mesh, order, flux, self.c, materials, ports)
        self.order = order
        self.flux = flux

    @classmethod
    def from_model(cls, tagged_mesh, model, *, order=2, flux="upwind", c=C_LIGHT):
        """ProblemTD(g) of problem/td.py:256-283 for a model on a tagged mesh
        (this package has no geometry / meshing layer): materials, PML
        absorbers, rectangular / ABC ports, PEC plates and periodic pairs of `model`."""
        obj = cls.__new__(cls)
        obj.c = float(c)
        obj._op = TdSession.from_model(tagged_mesh, model, order, flux, obj.c)
        obj.order, obj.flux = order, flux
        return obj

    @classmethod
    def box(cls, *, size, cells, order=2, flux="upwind", c=1.0):
        lx, ly, lz = size
        nx, ny, nz = cells
        obj = cls.__new__(cls)
        obj._op = TdSession.box_cavity(nx, ny, nz, lx, ly, lz, order, flux, float(c))
        obj.order, obj.flux, obj.c = order, flux, float(c)
        obj.size, obj.cells = tuple(size), tuple(cells)
        return obj

    @property
    def n_dofs(self):
        return self._op.n_dofs()

    @property
    def n_tets(self):
        return self._op.n_tets()

    def rhs(self, y):
        return self._op.apply(y)

    def field_energy(self, state):
        return self._op.field_energy(state)

    def step(self, y, h, krylov_dim=40, tol=None):
        return self._op.step(y, float(h), int(krylov_dim), tol)

    def step_explicit(self, y, h):
        return self._op.step_explicit(y, float(h))

    def step_adaptive(self, y, h):
        return self._op.step_adaptive(y, float(h))

    def cfl_dt(self, *, recompute=False):
        return self._op.cfl_dt(recompute)

    def state_space(self):
        """The operator A as a scipy.sparse.csr_matrix (problem/td.py:367-379)."""
        try:
            from scipy.sparse import csr_matrix
        except ImportError as e:
            raise ImportError("scipy is required for state_space() and jacobian()") from e
        n, row_ptr, col_idx, values = self._op.state_space()
        return csr_matrix((values, col_idx, row_ptr), shape=(n, n))

    def resonances(self, *, n=8):
        """Cavity resonant frequencies from the operator's spectrum
        (problem/td.py:391-399; session.rs:1007-1031).  Dense: modest meshes only."""
        return np.asarray(self._op.resonances(n))

    def ode(self):
        """The problem as dy/dt = A y for an external integrator (problem/td.py:381)."""
        return TdODE(self)

    def stepper(self, dt, *, krylov_dim=40, method="exponential"):
        """A reusable one-step propagator bound to `dt` (problem/td.py:487)."""
        if method not in ("exponential", "explicit"):
            raise ValueError("method must be 'exponential' or 'explicit'")
        return TdStepper(self, dt, krylov_dim, method)

    def probe_dof(self, point, *, field="E", component="z"):
        return self._op.nearest_node_dof(tuple(float(x) for x in point), field, component)

    def driven_transient(self, *, source, waveform, probes, dt, steps, krylov_dim=40, device="gpu",
                         method="explicit", verbose=True):
        src = self.probe_dof(source[0], field=source[1], component=source[2])
        pr = [self.probe_dof(p[0], field=p[1], component=p[2]) for p in probes]
        frames, _ = self._op.transient(None, dt=float(dt), steps=int(steps), source_dof=src, waveform=waveform,
                                       probes=pr, device=device, method=method, krylov_dim=int(krylov_dim),
                                       verbose=verbose)
        return np.arange(steps + 1) * dt, frames.T

    def transfer_function(self, *, source, probe, pulse, dt, steps, krylov_dim=40, device="gpu", verbose=True):
        """Field-to-field frequency response H(f) = R(f) / G(f) from one run
        driven by the broadband `pulse` at `source` and recorded at `probe`,
        both (point, field, component) (problem/td.py:549-598).  A TdTransfer:
        the steps + 1 frames give frequencies k / ((steps + 1) dt),
        k = 0 .. (steps + 1) // 2, and H is zero outside the pulse's band."""
        freqs, h = self._op.transfer_function(
            self.probe_dof(source[0], field=source[1], component=source[2]),
            self.probe_dof(probe[0], field=probe[1], component=probe[2]), pulse,
            dt=float(dt), steps=int(steps), device=device, krylov_dim=int(krylov_dim), verbose=verbose)
        return TdTransfer(freqs, h, source_label=_point_label(source), probe_label=_point_label(probe))

    def transient(self, y0=None, *, dt, steps, source=None, waveform=None, port=None, krylov_dim=40,
                  method="exponential", warmup=0, device="gpu", verbose=True, port_probes=None):
        src = None if source is None else self.probe_dof(source[0], field=source[1], component=source[2])
        frames, _ = self._op.transient(y0, dt=float(dt), steps=int(steps), source_dof=src, port=port,
                                       waveform=waveform, method=method, device=device,
                                       krylov_dim=int(krylov_dim), warmup=int(warmup), verbose=verbose,
                                       port_probes=port_probes)
        return TdTrajectory(frames, problem=self, dt=float(dt))

    def port_signals(self, traj, ports, *, dt=None):
        """Modal amplitude P_e(t) of each port over a trajectory (problem/td.py:612):
        returns (t, rows [ports, n_snapshot])."""
        traj = np.ascontiguousarray(traj, dtype=np.float64)
        rows = self._op.port_signals(traj, list(ports))
        n_rows = rows.shape[1]
        return np.arange(n_rows) * (1.0 if dt is None else float(dt)), rows
