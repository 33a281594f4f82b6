"""Adaptive exponential (ETD) time stepping on the device with an a-posteriori
Krylov error check, and a learned step proposer.

A step of dy/dt = A y + b g(t) is the exponential of the system augmented
with the step's source polynomial (dgtd_etd_try; with one coefficient held at
the step start it is the reference's exp(h [[A, b g_n],[0, 0]]) [y; 1],
propagator.rs:338-373); the device Arnoldi reports its a-posteriori estimate
h_{d+1,d}|exp(tH)_{d-1,0}| (propagator.rs:278-294), and a step is accepted when
the estimate is at most `tol`.  The state stays on the device between steps.

PlainEtd is the adaptive controller: after a step it scales h by
0.9 (tol/est)^(1/(d+1)) (d the Krylov dimension per sub-step), clipped to
[1/2, 2] after an accepted step and to [1/4, 1/2] after a rejected one, with
the Krylov dimension capped at m_max.

LearnedEtd asks a small MLP (16 -> 64 -> 64 -> 2, trained on traces the plain
controller logged) for the next step size and Krylov cap from the history of
the last four accepted steps; the proposed step is never below the plain
controller's own next step, it is tried and kept only if its estimate passes,
otherwise the plain controller decides the step (and its estimate alone decides
acceptance).  A proposal within 5 % of the plain step is not tried on its own;
after a failed proposal the next attempt is the plain controller's, and after
k failed proposals in a row the next 2^(k-1) (at most 32) are.  The training target of a logged step is what its
run says in hindsight: the largest step the plain controller itself took
within the next LOOKAHEAD accepted steps (a step size it reached and passed
from a similar state), relative to the previous step, and that step's Krylov
dimension relative to m_max.  The network so learns to skip the plain
controller's slow growth.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np

from ._native import check, lib

N_FEATURES = 16
N_HIDDEN = 64
N_OUT = 2
HISTORY = 4
LOOKAHEAD = 5


class Mlp:
    """The device MLP (dgtd_mlp_*): forward, gradient and Adam training run as
    the library's own kernels."""

    def __init__(self, ctx, n_in=N_FEATURES, n_hidden=N_HIDDEN, n_out=N_OUT, seed=0):
        self.ctx = ctx
        self.n_in, self.n_hidden, self.n_out = n_in, n_hidden, n_out
        h = C.c_void_p()
        check(lib.dgtd_mlp_create(ctx.handle, n_in, n_hidden, n_out, C.c_uint64(seed), C.byref(h)))
        self._h = h
        n = C.c_int64()
        check(lib.dgtd_mlp_n_params(h, C.byref(n)))
        self.n_params = n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.dgtd_mlp_destroy(h)
            self._h = C.c_void_p()

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        check(lib.dgtd_mlp_get_params(self._h, out))
        return out

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters")
        check(lib.dgtd_mlp_set_params(self._h, p))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float32)
        y = np.empty((x.shape[0], self.n_out), dtype=np.float32)
        check(lib.dgtd_mlp_forward(self._h, x, x.shape[0], y))
        return y

    def gradient(self, x, t):
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float32)
        t = np.ascontiguousarray(np.atleast_2d(t), dtype=np.float32)
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_float()
        check(lib.dgtd_mlp_gradient(self._h, x, t, x.shape[0], g, C.byref(loss)))
        return g, loss.value

    def train(self, x, t, epochs=2000, lr=3e-3) -> np.ndarray:
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float32)
        t = np.ascontiguousarray(np.atleast_2d(t), dtype=np.float32)
        losses = np.empty(max(int(epochs), 1), dtype=np.float32)
        check(lib.dgtd_mlp_train(self._h, x, t, x.shape[0], int(epochs), float(lr), losses))
        return losses[: int(epochs)]


@dataclass
class StepRecord:
    h: float
    dim: int
    est: float
    rejected_before: int


@dataclass
class EtdStats:
    accepted: int = 0
    rejected: int = 0
    proposals_kept: int = 0
    proposals_failed: int = 0
    matvecs: int = 0
    seconds: float = 0.0
    history: list = field(default_factory=list)
    times: np.ndarray | None = None   # t of each recorded row (0 and every accepted step)
    series: np.ndarray | None = None  # [rows, n_fun] functionals of the state at `times`


def features(hist: list, tol: float, m_max: int, h_ref: float) -> np.ndarray:
    """16 features from the last four accepted steps (most recent first; zero
    padding before there are four): log10(est/tol)/8, log(h_k/h_{k-1})/2,
    d_k/m_max, rejections before step k / 4."""
    f = np.zeros(N_FEATURES, dtype=np.float32)
    for q in range(HISTORY):
        k = len(hist) - 1 - q
        if k < 0:
            break
        r = hist[k]
        prev_h = hist[k - 1].h if k > 0 else h_ref
        est = max(r.est, 1e-30)
        f[4 * q + 0] = math.log10(est / tol) / 8.0
        f[4 * q + 1] = math.log(r.h / prev_h) / 2.0
        f[4 * q + 2] = r.dim / m_max
        f[4 * q + 3] = r.rejected_before / 4.0
    return f


class PlainEtd:
    """The adaptive controller (see the module docstring)."""

    def __init__(self, tol=1e-7, m_max=48, safety=0.9):
        self.tol, self.m_max, self.safety = float(tol), int(m_max), float(safety)

    def _factor(self, est, dim, m, accepted):
        chunks = max(1, math.ceil(m / 12))
        d = max(1.0, dim / chunks)
        est = max(est, 1e-300)
        f = self.safety * (self.tol / est) ** (1.0 / (d + 1.0))
        return min(max(f, 0.5), 2.0) if accepted else min(max(f, 0.25), 0.5)

    def next_after(self, h, est, dim, m, accepted):
        return h * self._factor(est, dim, m, accepted), self.m_max


class LearnedEtd:
    """MLP proposals, kept only when their estimate passes (else PlainEtd)."""

    def __init__(self, mlp: Mlp, plain: PlainEtd, m_min=10):
        self.mlp, self.plain, self.m_min = mlp, plain, int(m_min)

    def propose(self, hist, h_ref):
        x = features(hist, self.plain.tol, self.plain.m_max, h_ref)
        out = self.mlp.forward(x[None, :])[0]
        h_prev = hist[-1].h if hist else h_ref
        h = h_prev * math.exp(float(np.clip(out[0], -1.4, 1.4)))
        # The Krylov cap sets the number of <= 12-dimensional sub-steps, so a
        # cap below the predicted dimension starves every sub-step: the
        # predicted dimension is rounded up to whole sub-steps with a margin.
        d = float(np.clip(out[1], 0.0, 1.0)) * self.plain.m_max
        m = int(min(self.plain.m_max, max(self.m_min, 12 * math.ceil((1.25 * d + 1) / 12))))
        return h, m


def run_etd(gop, y0, b, waveform, t_end, h0, plain: PlainEtd, learned: LearnedEtd | None = None,
            log: list | None = None, max_attempts=100000, point_dof=None, n_coef=8, src_tol=None,
            functionals=None, max_rows=1 << 16):
    """ETD from t = 0 to t_end on the device-resident state; returns (y, EtdStats).

    The source is b*g(t) (b a vector, or the unit vector of `point_dof`), g =
    `waveform` (None: a free run).  Over each step g is replaced by its
    degree-(n_coef-1) interpolant at the step's Chebyshev points
    (sources.step_polynomial) and the step is the exponential of the
    polynomial-augmented system (dgtd_etd_try); a step whose interpolant
    deviates from g by more than `src_tol` (default: plain.tol) is shortened
    before it is tried.  n_coef = 1 with the value at the step start is the
    reference's held source (propagator.rs:338-373).  The state stays on the
    device: each try reads back only the Krylov dimension and estimate.
    `log`, if given, gets a (features, target) pair per accepted step of the
    plain controller for training (the look-ahead target of the module
    docstring).  `functionals` [(idx, w), ...] (F(y) = sum w[k] y[idx[k]],
    e.g. port modal amplitudes) are recorded on the device at t = 0 and after
    every accepted step, into EtdStats.times / series (at most max_rows rows)."""
    from . import sources as S

    driven = waveform is not None and (b is not None or point_dof is not None)
    drive = None
    if driven:
        if point_dof is not None:
            drive = ("point", int(point_dof))
        else:
            gop.set_source_vector(np.asarray(b, dtype=np.float64))
            drive = ("vector", None)
    src_tol = plain.tol if src_tol is None else float(src_tol)
    gop.upload(np.asarray(y0, dtype=np.float32))
    st = EtdStats()
    times = [0.0]
    if functionals:
        gop.set_functionals(functionals, max_rows)
        gop.record_functionals(0)

    def recorded(t_now):
        if functionals:
            if len(times) >= max_rows:
                raise RuntimeError("ETD run exceeded the functional rows")
            gop.record_functionals(len(times))
            times.append(t_now)
    pending = []  # (features, index of the accepted step, previous step) awaiting look-ahead targets
    hist: list[StepRecord] = []
    t, h, m = 0.0, float(h0), plain.m_max
    rejects = 0
    w0 = time.perf_counter()
    attempts = 0
    skip, streak = 0, 0  # proposals still to skip; consecutive failed proposals

    def coef_for(t0, hh):
        """(coef, hh): the step's source polynomial, hh shortened until it fits."""
        if not driven:
            return None, hh
        for _ in range(60):
            if n_coef == 1:
                return np.array([float(waveform(t0))]), hh
            c, err = S.step_polynomial(waveform, t0, hh, n_coef)
            if err * hh <= src_tol:
                return c, hh
            hh *= 0.5
        raise RuntimeError("source polynomial does not converge")

    def attempt(hh, mm):
        c, hh = coef_for(t, hh)
        dim, est = gop.etd_try(hh, mm, plain.tol, coef=c, drive=drive)
        st.matvecs += dim
        return hh, dim, est

    while t < t_end * (1 - 1e-12):
        attempts += 1
        if attempts > max_attempts:
            raise RuntimeError("ETD run exceeded the attempt limit")
        feat = features(hist, plain.tol, plain.m_max, h0)
        tried_learned = False
        hp = mp = None
        if learned is not None and skip > 0:
            skip -= 1
        elif learned is not None:
            hp, mp = learned.propose(hist, h0)
            # never below the plain controller's own next step: the network
            # can only skip ahead of it; a proposal no longer than that step
            # is the plain step, which is tried below anyway
            hp = min(max(hp, h), t_end - t)
            if hp <= 1.05 * min(h, t_end - t):
                hp = None
        if hp is not None:
            hp, dim, est = attempt(hp, mp)
            tried_learned = True
            if est <= plain.tol:
                gop.etd_commit()
                streak = 0
                st.proposals_kept += 1
                st.accepted += 1
                t += hp
                recorded(t)
                hist.append(StepRecord(hp, dim, est, rejects))
                rejects = 0
                h, m = plain.next_after(hp, est, dim, mp, True)
                continue
            st.proposals_failed += 1
            # the next attempts are the plain controller's alone: one after an
            # isolated failure, doubling with each further failure in a row
            streak += 1
            skip = min(1 << (streak - 1), 32)
        h_try = min(h, t_end - t)
        h_try, dim, est = attempt(h_try, m)
        if est <= plain.tol:
            gop.etd_commit()
            st.accepted += 1
            if log is not None and not tried_learned:
                pending.append((feat, len(hist), hist[-1].h if hist else h0))
            t += h_try
            recorded(t)
            hist.append(StepRecord(h_try, dim, est, rejects))
            rejects = 0
            h, m = plain.next_after(h_try, est, dim, m, True)
        else:
            st.rejected += 1
            rejects += 1
            h, m = plain.next_after(h_try, est, dim, m, False)
    y = gop.download().astype(np.float64)
    st.seconds = time.perf_counter() - w0
    if functionals:
        st.times = np.array(times)
        st.series = gop.functional_series(len(times))
    st.history = [(r.h, r.dim, r.est) for r in hist]
    if log is not None:
        for feat, k, prev in pending:
            window = hist[k:k + LOOKAHEAD]
            best = max(window, key=lambda r: r.h)
            log.append((feat, np.array([math.log(best.h / prev), best.dim / plain.m_max], dtype=np.float32)))
    return y, st


def train_controller(mlp: Mlp, logs: list, epochs=3000, lr=3e-3) -> np.ndarray:
    """Fit the MLP to logged (features, target) pairs with the device Adam."""
    x = np.stack([f for f, _ in logs]).astype(np.float32)
    t = np.stack([g for _, g in logs]).astype(np.float32)
    return mlp.train(x, t, epochs=epochs, lr=lr)
