"""A batch of independent DGTD instances stepped together on one GPU: many
small PEC cavities of mixed order (the batched multi-instance configuration:
256 cavities, n x n x n Kuhn boxes with n in 4..20, orders 2..5, a dielectric
block, a Gaussian-pulse initial field, LSERK4 steps).

Instances of one order are concatenated into one operator.  The union shares
no vertex ids, and faces are matched by vertex ids, so no face couples two
instances (they may overlap in space) and each instance evolves exactly as it
would alone: its geometric factors are computed from the same coordinates.
Every element carries its instance's own LSERK4 step as a per-element
multiplier of the stage step (element record word 43), so one fused stage
launch per order group steps every instance with its own dt.  An autotuner
times the stage kernels for each group (tensor cores, FP32 CUDA cores with
the full or the half tile) and keeps the fastest; the steps are then captured into a
CUDA graph (an even number per graph, so that the ping-pong state buffers end
where they started) and replayed.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from . import gpu as G
from . import operator as O

CFL = 0.5            # fraction of the LSERK4 stability bound |z| ~ 2.8 of h * rho
LSERK_Z = 2.8
REF_CELLS = 4        # reference cavity for the spectral radius of each order


@dataclass
class Instance:
    """One cavity: a unit Kuhn box of n^3 cells, order, per-element materials
    [K, 8], a Gaussian E pulse (centre, width, component) as initial field."""

    cells: int
    order: int
    materials: np.ndarray
    pulse_center: np.ndarray
    pulse_width: float
    pulse_component: int
    dt: float = 0.0


def random_cavities(count: int, seed: int, cells=(4, 20), orders=(2, 5), eps=(1.0, 10.0)) -> list[Instance]:
    """Seeded instances: n ~ U{cells}, order ~ U{orders}, an axis-aligned block
    (by element centroid) with eps_r ~ U[eps], a pulse at a random interior
    point on a random E component."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(cells[0], cells[1] + 1))
        order = int(rng.integers(orders[0], orders[1] + 1))
        mesh = O.structured_box(n, n, n)
        cen = mesh.nodes[mesh.tets].mean(axis=1)
        lo = rng.uniform(0.0, 0.6, 3)
        hi = lo + rng.uniform(0.2, 0.4, 3)
        inside = np.all((cen >= lo) & (cen <= hi), axis=1)
        eps_r = float(rng.uniform(eps[0], eps[1]))
        mat = O.isotropic_materials(np.where(inside, eps_r, 1.0))
        out.append(Instance(n, order, mat, rng.uniform(0.25, 0.75, 3), float(rng.uniform(0.06, 0.15)),
                            int(rng.integers(0, 3))))
    return out


@dataclass
class BatchGroup:
    """The instances of one order as one operator."""

    order: int
    members: list
    op: O.MaxwellOperator
    elem_off: np.ndarray           # [members + 1] element offsets
    dt_scale: np.ndarray           # [K] per-element step
    y0: np.ndarray = field(default=None)  # AoS f32

    @property
    def n_dof(self) -> int:
        return self.op.n_dof

    def dof_slice(self, j: int) -> slice:
        bs = 6 * self.op.np
        return slice(int(self.elem_off[j]) * bs, int(self.elem_off[j + 1]) * bs)


def build_groups(instances: list[Instance]) -> list[BatchGroup]:
    """Concatenate the instances of each order (vertex ids offset per instance)."""
    groups = []
    for order in sorted({ins.order for ins in instances}):
        members = [i for i, ins in enumerate(instances) if ins.order == order]
        nodes, tets, mats, offs = [], [], [], [0]
        nbase = 0
        for j, i in enumerate(members):
            m = O.structured_box(instances[i].cells, instances[i].cells, instances[i].cells)
            nodes.append(m.nodes)
            tets.append(m.tets + nbase)
            nbase += m.nodes.shape[0]
            mats.append(instances[i].materials)
            offs.append(offs[-1] + m.n_tets)
        mesh = O.Mesh(np.ascontiguousarray(np.concatenate(nodes)), np.ascontiguousarray(np.concatenate(tets)))
        op = O.MaxwellOperator(mesh, order, 1.0, materials=np.concatenate(mats))
        groups.append(BatchGroup(order, members, op, np.array(offs, dtype=np.int64),
                                 np.ones(mesh.n_tets)))
    return groups


def initial_fields(groups: list[BatchGroup], instances: list[Instance]) -> None:
    """Each group's AoS f32 initial state from its instances' pulses."""
    for g in groups:
        xyz = g.op.node_coords()  # [K*Np, 3]
        y = np.zeros(g.n_dof, dtype=np.float32)
        np_ = g.op.np
        for j, i in enumerate(g.members):
            ins = instances[i]
            a, b = int(g.elem_off[j]) * np_, int(g.elem_off[j + 1]) * np_
            x = xyz[a:b]
            r2 = np.sum((x - ins.pulse_center) ** 2, axis=1)
            y[a * 6 + ins.pulse_component:b * 6:6] = np.exp(-r2 / (2.0 * ins.pulse_width ** 2))
        g.y0 = y


def assign_steps(ctx: G.GpuContext, groups: list[BatchGroup], instances: list[Instance], iters: int = 40) -> dict:
    """dt of every instance: CFL * 2.8 / rho, with rho the spectral radius of the
    order's reference cavity (REF_CELLS^3, vacuum; device power iteration)
    scaled by n / REF_CELLS: the elements of an n-cell box are the reference
    box's elements shrunk by REF_CELLS / n, and eps_r >= 1 only slows waves."""
    import ctypes as C

    rho_ref = {}
    for g in groups:
        ref = O.MaxwellOperator(O.structured_box(REF_CELLS, REF_CELLS, REF_CELLS), g.order, 1.0)
        gop = G.GpuOperator(ctx, ref)
        rho = C.c_double()
        nat.check(nat.lib.dgtd_power_rho(gop.handle, iters, C.byref(rho)))
        rho_ref[g.order] = rho.value
        del gop
        for j, i in enumerate(g.members):
            ins = instances[i]
            ins.dt = CFL * LSERK_Z / (rho_ref[g.order] * ins.cells / REF_CELLS)
            g.dt_scale[g.elem_off[j]:g.elem_off[j + 1]] = ins.dt
    return rho_ref


class BatchRunner:
    """The groups on the device: one operator per order group with its
    per-element steps, the autotuned stage kernel, and a CUDA graph of
    `steps_per_graph` LSERK4 steps of every group.  Each group runs on its own
    context and torch stream; the graph forks from the runner's stream
    (`self.stream`) to the group streams and joins back, so the groups' stage
    launches overlap (one group's launch tails are filled by the others).
    Time it with events on `self.stream`."""

    def __init__(self, ctx: G.GpuContext, groups: list[BatchGroup], device=0):
        import torch

        self.torch = torch
        self.ctx = ctx
        self.groups = groups
        self.device = device
        self.stream = torch.cuda.Stream(device=device)
        ctx.set_stream(self.stream.cuda_stream)
        # one context (and stream) per group, so that the groups can overlap
        self.ctxs = [G.GpuContext(ctx.device) for _ in groups]
        self.streams = [torch.cuda.Stream(device=device) for _ in groups]
        for c, st in zip(self.ctxs, self.streams):
            c.set_stream(st.cuda_stream)
        self.gops = [G.GpuOperator(c, g.op, dt_scale=g.dt_scale) for c, g in zip(self.ctxs, groups)]
        self.graph = None
        self.steps_per_graph = 0
        self.tuning = []

    def _fork(self):
        """Group streams wait for the runner's stream."""
        for st in self.streams:
            st.wait_stream(self.stream)

    def _join(self):
        """The runner's stream waits for every group stream."""
        for st in self.streams:
            self.stream.wait_stream(st)

    @property
    def n_dof(self) -> int:
        return sum(g.n_dof for g in self.groups)

    def load_device(self, ptrs) -> None:
        """Each group's AoS state from a device pointer, ordered after the work
        queued on the runner's stream and before what follows it."""
        self._fork()
        for gop, ptr in zip(self.gops, ptrs):
            gop.load_device(ptr)
        self._join()

    def store_device(self, ptrs) -> None:
        """Each group's AoS state to a device pointer (ordered as load_device)."""
        self._fork()
        for gop, ptr in zip(self.gops, ptrs):
            gop.store_device(ptr)
        self._join()

    def load(self) -> None:
        self._fork()
        for g, gop in zip(self.groups, self.gops):
            gop.upload(g.y0)
        self._join()

    def _time_steps(self, k: int, steps: int) -> float:
        st = self.streams[k]
        t0 = self.torch.cuda.Event(enable_timing=True)
        t1 = self.torch.cuda.Event(enable_timing=True)
        t0.record(st)
        self.gops[k].run_lserk(1.0, steps)
        t1.record(st)
        st.synchronize()
        return t0.elapsed_time(t1) / steps

    def autotune(self, trial_steps: int = 2) -> list:
        """Time each available stage kernel per group (after one warm-up step)
        and keep the fastest.  Leaves the initial states loaded."""
        self.tuning = []
        self.stream.synchronize()
        for k, (g, gop) in enumerate(zip(self.groups, self.gops)):
            cands = [nat.ENGINE_FP32, nat.ENGINE_FP32_SMALL_TILES, nat.ENGINE_TF32X3]
            times = {}
            for eng in cands:
                gop.set_engine(eng)
                gop.upload(g.y0)
                gop.run_lserk(1.0, 1)
                times[eng] = self._time_steps(k, trial_steps)
            best = min(times, key=times.get)
            gop.set_engine(best)
            name = {nat.ENGINE_FP32: "fp32", nat.ENGINE_FP32_SMALL_TILES: "fp32_small_tiles",
                    nat.ENGINE_TF32X3: "tf32x3"}
            self.tuning.append({"order": g.order, "instances": len(g.members), "n_dof": g.n_dof,
                                "ms_per_step": {name[k]: round(v, 4) for k, v in times.items()},
                                "engine": name[best]})
        self.load()
        self.stream.synchronize()
        return self.tuning

    def capture(self, steps_per_graph: int = 10) -> None:
        """Capture `steps_per_graph` (even) LSERK4 steps of every group into one
        CUDA graph.  Leaves the initial states loaded."""
        torch = self.torch
        if steps_per_graph < 2 or steps_per_graph % 2:
            raise ValueError("steps_per_graph must be even (the state buffers ping-pong 5 times per step)")
        self._fork()
        for gop in self.gops:  # kernel attributes are set on the first launch, outside the capture
            gop.run_lserk(1.0, 2)
        self._join()
        self.load()
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            # fork from the capture stream to the group streams, join back
            for st in self.streams:
                st.wait_stream(self.stream)
            for gop in self.gops:
                gop.run_lserk(1.0, steps_per_graph)
            for st in self.streams:
                self.stream.wait_stream(st)
        self.graph = g
        self.steps_per_graph = steps_per_graph

    def run(self, steps: int) -> None:
        """`steps` LSERK4 steps of every instance on `self.stream` (graph
        replays when a graph is captured: steps must be a multiple of it)."""
        if self.graph is None:
            self._fork()
            for gop in self.gops:
                gop.run_lserk(1.0, steps)
            self._join()
            return
        if steps % self.steps_per_graph:
            raise ValueError("steps must be a multiple of steps_per_graph")
        with self.torch.cuda.stream(self.stream):
            for _ in range(steps // self.steps_per_graph):
                self.graph.replay()

    def states(self, instances: list[Instance]) -> list[np.ndarray]:
        """The AoS f32 state of every instance, in instance order."""
        self.stream.synchronize()
        for st in self.streams:
            st.synchronize()
        out = [None] * len(instances)
        for g, gop in zip(self.groups, self.gops):
            y = gop.download()
            for j, i in enumerate(g.members):
                out[i] = y[g.dof_slice(j)].copy()
        return out
