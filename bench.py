#!/usr/bin/env python
"""DGTD throughput benchmark: DOF-stage-updates/s of the fused LSERK4 step.

Workload (the single-GPU configuration the metric is quoted on): the
48^3 x 6 = 663,552-tet jittered box (+-10% h, seed 2024), order N=4 (Np=35),
eps_r=4 sphere r=0.25 at the centre, Gaussian E_z pulse (sigma 0.05) at
(0.3,0.4,0.5), upwind flux, PEC walls, LSERK4.  A step is one LSERK4 step (5
RHS stages) over the whole mesh; n_dof = 139,345,920, so every step streams
~2.3 GB per stage, far above the 126 MB L2 (no L2 flush is needed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

`--impl reference` times the CPU restatement of the reference's CPU path
(oracle/, f64, all host threads) on the same workload within a time budget.
Under torchrun (N > 1 ranks) the workload is partitioned across the ranks
with a halo exchange per stage over NCCL (strong scaling); `--replicas` runs
N independent replicas instead (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_DOF_STAGE = {2: 18.8, 3: 17.4, 4: 16.8, 5: 16.5}
FLOPS_PER_DOF_STAGE = {n: 6 * (n + 1) * (n + 2) * (n + 3) // 6 + 8 * (n + 1) * (n + 2) // 2 for n in range(1, 6)}
METRIC = "DOF-stage-updates/s"


def _rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(kernel, order, n_dof):
    """DRAM bytes per launch of the stage kernel (dram__bytes_read.sum +
    dram__bytes_write.sum from the ncu capture summarised in profiles/, scaled
    from bytes per DOF to this workload's n_dof), or None when no capture exists."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p)).get(f"{kernel}/N{order}")
    if not d:
        return None
    return float(d["bytes_per_dof_stage_avg"]) * n_dof


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def sphere_pulse_config(cells, order, n_dof, world):
    """The workload description shared by both arms' JSON lines."""
    return {"workload": f"sphere_pulse: jittered {cells}^3x6 box ({6 * cells ** 3:,} tets), N={order}, eps_r=4 "
                        "sphere r=0.25, Gaussian Ez pulse sigma=0.05 at (0.3,0.4,0.5), upwind, PEC, LSERK4",
            "cells": f"{cells}^3", "order": order, "n_dof": n_dof,
            "l2": "state 4*n_dof bytes per buffer >> 126 MB L2; no flush",
            "parallelism": f"replica x{world}" if world > 1 else "single GPU"}


def _oracle_sphere_pulse(R, n_cells, order):
    """The sphere_pulse workload built by the oracle alone (mesh_gen.rs jitter,
    seed 2024, +-10% h; eps_r = 4 for element centroids within 0.25 of the
    centre; the Gaussian E_z pulse at the oracle's nodes): the reference arm
    and the CPU baseline load no product code."""
    nodes, tets = R.box_mesh_jittered(n_cells, n_cells, n_cells, 1.0, 1.0, 1.0, 0.10, 2024)
    cen = nodes[tets].mean(axis=1)
    eps = np.where(np.linalg.norm(cen - 0.5, axis=1) < 0.25, 4.0, 1.0)
    mat = np.zeros((eps.size, 8))
    mat[:, 0:3] = eps[:, None]
    mat[:, 3:6] = 1.0
    orc = R.Operator(nodes, tets, order, 1.0, materials=mat)
    x = orc.node_coords()
    y = np.zeros((x.shape[0], 6))
    y[:, 2] = np.exp(-((x - np.array([0.3, 0.4, 0.5])) ** 2).sum(axis=1) / (2 * 0.05 ** 2))
    return orc, y.ravel()


def _oracle_dt(R, n_cells, order):
    """LSERK4 step 0.5 * 2.8 / rho, rho from 20 power iterations of the oracle
    at 12^3 scaled by n_cells / 12 (rho grows as 1/h); the step only has to keep
    a timing run stable."""
    orc, _ = _oracle_sphere_pulse(R, 12, order)
    rho, _ = orc.power_rho(20)
    return 0.5 * 2.8 / (rho * n_cells / 12.0)


def cpu_reference_rate(steps, warmup, n_cells=24, order=4, threads=None, budget_s=None):
    """Oracle (f64 CPU restatement of explicit.rs:100-135 over rhs.rs:1262-1473,
    OpenMP over all host threads) on the sphere_pulse workload at n_cells^3;
    returns (DOF-stage/s, info).  With budget_s, at most one warm-up step is
    run and the timed steps are capped so that they take about budget_s."""
    from oracle import oracle as R

    if threads:
        R.set_threads(threads)
    orc, y = _oracle_sphere_pulse(R, n_cells, order)
    dt = _oracle_dt(R, n_cells, order)
    t_warm = None
    if budget_s is not None:
        warmup = min(warmup, 1)
    if warmup:
        t0 = time.perf_counter()
        y = orc.lserk(y, dt, warmup)
        t_warm = (time.perf_counter() - t0) / warmup
    timed = steps
    if budget_s is not None and t_warm:
        timed = max(1, min(steps, int(budget_s / t_warm)))
    t0 = time.perf_counter()
    y = orc.lserk(y, dt, timed)
    el = time.perf_counter() - t0
    rate = orc.n_dof * 5 * timed / el
    return rate, {"cores": R.threads(), "seconds": el, "n_dof": orc.n_dof, "steps": timed, "warmup": warmup,
                  "dt": dt, "finite": bool(np.all(np.isfinite(y))),
                  "sample": f"sphere_pulse at {n_cells}^3 x 6 = {6 * n_cells ** 3} tets, N={order}, "
                            f"{timed} timed LSERK4 steps after {warmup} warm-up (f64, OpenMP, "
                            f"{R.threads()} threads)"}


def run_reference(args):
    rank, world, _ = _rank()
    if rank != 0:
        return 0
    steps, warmup = args.steps, args.warmup
    rate, info = cpu_reference_rate(steps, warmup, n_cells=args.cells, budget_s=args.ref_budget)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "DOF-stage/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": warmup, "ms_per_step": info["seconds"] / info["steps"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": sphere_pulse_config(args.cells, 4, info["n_dof"], world),
        "cpu_baseline": {"value": rate, "unit": "DOF-stage/s", "cores": info["cores"], "kind": "port",
                         "sample": info["sample"]},
        "e2e": {"value": rate, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "steps_timed": info["steps"], "warmup_run": info["warmup"], "finite": info["finite"],
        "note": "The reference's Rust CPU path cannot be built here (no Rust toolchain); timed is the "
                "oracle's C restatement of explicit.rs:100-135 over rhs.rs:1262-1473 on the full workload, "
                "one warm-up step and as many of the requested steps as fit the time budget "
                f"({args.ref_budget:.0f} s).",
    }
    print(json.dumps(line), flush=True)
    return 0


def _init_nccl(local, seconds):
    """The NCCL process group of this rank on cuda:`local`, its communicator
    created at once (a barrier), with file descriptor 1 pointed at stderr
    meanwhile: NCCL's version banner and init log lines go to stderr, so
    stdout carries only the JSON line."""
    import datetime

    import torch

    torch.cuda.set_device(local)
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=seconds),
                                             device_id=torch.device("cuda", local))
        torch.distributed.barrier()
        torch.cuda.synchronize()
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)


def run_sharded(args):
    """The 48^3 sphere_pulse workload partitioned across the N ranks (strong
    scaling): a Morton element partition, one local operator per rank over its
    owned elements and halo, LSERK4 stages with one halo exchange each over
    NCCL point-to-point, the interior elements' update overlapping the
    exchange (partition.ShardedLserk).  `value` counts the global DOFs."""
    import torch

    from rapidfem_b200 import gpu as G
    from rapidfem_b200 import operator as O
    from rapidfem_b200 import partition as PT
    from rapidfem_b200 import workloads as W

    rank, world, local = _rank()
    if world == 1:  # a one-rank group outside torchrun
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", str(29400 + os.getpid() % 1000))
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    dev = torch.device("cuda", local)
    _init_nccl(local, 120)
    wl = W.sphere_pulse(args.cells, 4)
    parts = PT.build_parts(wl.mesh, PT.morton_partition(wl.mesh, world), materials=wl.materials)
    me = parts[rank]
    op = O.MaxwellOperator(me.mesh, 4, 1.0, materials=me.materials)
    ctx = G.GpuContext(local)
    gop = G.GpuOperator(ctx, op)
    gop.set_engine({"fp32": 0, "tf32x3": 1}[args.engine])
    eng = PT.GpuEngine(gop, dev)
    y_local = wl.y0(op).astype(np.float32)  # the pulse at this rank's nodes (owned and halo)
    n_global = 6 * op.np * wl.mesh.n_tets

    # spectral radius: power iteration on the local operator, max over ranks
    with torch.cuda.stream(eng.stream):
        g = torch.Generator(device=dev).manual_seed(rank)
        v = torch.randn(op.n_dof, device=dev, dtype=torch.float32, generator=g)
        v /= v.norm()
        av = torch.empty_like(v)
        rho = 1.0
        for _ in range(args.power_iters):
            gop.apply_device(v.data_ptr(), av.data_ptr())
            rho = float(av.norm())
            v = av / rho
    t = torch.tensor([rho], device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    dt = 0.5 * 2.8 / float(t)

    sharded = PT.ShardedLserk(me, eng, PT.TorchTransport(), overlap=True)
    eng.load(y_local)
    torch.distributed.barrier()
    sharded.step(dt, args.warmup)
    eng.sync()
    torch.distributed.barrier()
    gop.reset_launch_count()
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    eng.sync()
    torch.distributed.barrier()
    t_start.record(eng.stream)
    sharded.step(dt, args.steps)
    t_end.record(eng.stream)
    eng.sync()
    torch.distributed.barrier()
    ms = t_start.elapsed_time(t_end)
    ck = clocks.stop()
    launches = gop.launch_count()
    finite = bool(np.isfinite(eng.state()).all())
    t = torch.tensor([ms], device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms = float(t)
    value = n_global * 5 * args.steps / (ms * 1e-3)
    stage_ms = ms / (5 * args.steps)
    peak, peak_kind = _peaks()
    achieved = BYTES_PER_DOF_STAGE[4] * n_global / world / (stage_ms * 1e-3) / 1e9  # per GPU

    # end to end: this rank's part from page-locked host memory, the run, the part back
    y_host = torch.from_numpy(y_local).pin_memory()
    y_out = torch.empty(op.n_dof, dtype=torch.float32).pin_memory()
    y_dev = torch.empty(op.n_dof, dtype=torch.float32, device=dev)
    eng.sync()
    torch.distributed.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(eng.stream)
    with torch.cuda.stream(eng.stream):
        y_dev.copy_(y_host, non_blocking=True)
        gop.load_device(y_dev.data_ptr())
        sharded.step(dt, args.steps)
        gop.store_device(y_dev.data_ptr())
        y_out.copy_(y_dev, non_blocking=True)
    e1.record(eng.stream)
    eng.sync()
    e2e_ms = e0.elapsed_time(e1)
    t = torch.tensor([e2e_ms], device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    e2e_ms = float(t)
    line = {
        "metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(sphere_pulse_config(args.cells, 4, n_global, world),
                       parallelism=f"element partition x{world} (Morton), one halo exchange per stage over "
                                   "NCCL point-to-point, the interior update overlapping it"),
        "run": {"dt": dt, "engine": args.engine, "halo_elements_max": int(max(p.halo.size for p in parts)),
                "interior_fraction_min": float(min(p.n_interior / p.n_owned for p in parts))},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "stage kernel, per GPU", "stage_ms": stage_ms, "peak_kind": peak_kind},
        "clocks": ck,
        "e2e": {"value": n_global * 5 * args.steps / (e2e_ms * 1e-3), "unit": "DOF-stage/s",
                "h2d_bytes_per_step": op.n_dof * 4 / args.steps, "d2h_bytes_per_step": op.n_dof * 4 / args.steps,
                "steps": args.steps, "api": "load_device / ShardedLserk.step / store_device per rank"},
        "finite": finite,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    del sharded, eng, gop
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()
    return 0


def run_b200(args):
    import torch

    from rapidfem_b200 import gpu as G
    from rapidfem_b200 import workloads as W

    rank, world, local = _rank()
    dist = world > 1
    if dist:
        _init_nccl(local, 120)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    wl = W.sphere_pulse(args.cells, 4)
    op = wl.build()
    order = wl.order
    ctx = G.GpuContext(local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    gop = G.GpuOperator(ctx, op)
    gop.set_engine({"fp32": 0, "tf32x3": 1}[args.engine])
    n = gop.n_dof()
    y0 = wl.y0(op).astype(np.float32)

    # spectral radius by power iteration on the device, dt = 0.5 * 2.8 / rho
    with torch.cuda.stream(stream):
        g = torch.Generator(device=dev).manual_seed(0)
        v = torch.randn(n, device=dev, dtype=torch.float32, generator=g)
        v /= v.norm()
        av = torch.empty_like(v)
        rho = 1.0
        for _ in range(args.power_iters):
            gop.apply_device(v.data_ptr(), av.data_ptr())
            rho = float(av.norm())
            v = av / rho
    torch.cuda.synchronize()
    dt = 0.5 * 2.8 / rho

    y_dev = torch.from_numpy(y0).to(dev)
    gop.load_device(y_dev.data_ptr())
    gop.run_lserk(dt, args.warmup)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    gop.reset_launch_count()
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    t_start.record(stream)
    gop.run_lserk(dt, args.steps)
    t_end.record(stream)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    ms = t_start.elapsed_time(t_end)
    ck = clocks.stop()
    launches = gop.launch_count()
    yf = torch.empty(n, device=dev, dtype=torch.float32)
    gop.store_device(yf.data_ptr())
    torch.cuda.synchronize()
    finite = bool(torch.isfinite(yf).all())
    if dist:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t)

    total_units = n * 5 * args.steps * world
    value = total_units / (ms * 1e-3)
    stage_ms = ms / (5 * args.steps)
    alg_bytes = BYTES_PER_DOF_STAGE[order] * n
    peak, peak_kind = _peaks()
    achieved = alg_bytes / (stage_ms * 1e-3) / 1e9
    traffic = _traffic("rhs_fp32_lserk" if gop.engine == 0 else "rhs_tc_lserk", order, n)

    # end to end through the public API with pinned host buffers
    e2e_steps = args.steps
    y_host = torch.from_numpy(y0).pin_memory().numpy()
    y_out = torch.empty(n, dtype=torch.float32).pin_memory().numpy()  # final state, page-locked like the input
    probes = np.array([op.nearest_node_dof([0.5, 0.5, 0.5], 0, 2), op.nearest_node_dof([0.7, 0.4, 0.5], 1, 1)])
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    series, yfin = gop.transient_probes(y_host, dt, e2e_steps, 1, probes=probes, y_final=y_out)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t)
    e2e_value = n * 5 * e2e_steps * world / (e2e_ms * 1e-3)
    h2d = n * 4
    d2h = n * 4 + series.nbytes

    line = {
        "metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": sphere_pulse_config(args.cells, order, n, world),
        "run": {"dt": dt, "engine": ["fp32", "tf32x3"][gop.engine]},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "rhs_fp32_kernel<N,LSERK>" if gop.engine == 0 else "rhs_tc_kernel<N,LSERK>",
                     "alg_bytes_per_dof_stage": BYTES_PER_DOF_STAGE[order],
                     "stage_ms": stage_ms, "peak_kind": peak_kind,
                     "flops_per_dof_stage": FLOPS_PER_DOF_STAGE[order],
                     "achieved_tflops": FLOPS_PER_DOF_STAGE[order] * n / (stage_ms * 1e-3) / 1e12},
        "clocks": ck,
        "e2e": {"value": e2e_value, "unit": "DOF-stage/s", "h2d_bytes_per_step": h2d / e2e_steps,
                "d2h_bytes_per_step": d2h / e2e_steps, "steps": e2e_steps,
                "api": "GpuOperator.transient_probes (dgtd_transient_probes): y0 in, probe series + final state out"},
        "finite": finite,
    }
    if rank == 0 and world == 1 and not args.no_cpu:  # the CPU baseline is an N = 1 figure
        rate, info = cpu_reference_rate(args.cpu_steps, 1, n_cells=args.ref_cells)
        line["cpu_baseline"] = {"value": rate, "unit": "DOF-stage/s", "cores": info["cores"], "kind": "port",
                                "sample": info["sample"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del gop
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_c4(args):
    """The batched multi-instance configuration: 256 PEC cavities (n^3 Kuhn
    boxes, n ~ U{4..20}, orders ~ U{2..5}, a dielectric block eps_r ~ U[1,10],
    a Gaussian pulse), LSERK4 with each cavity's own dt, autotuned stage kernel
    per order group, steps replayed from a CUDA graph."""
    import torch

    from rapidfem_b200 import batch as B
    from rapidfem_b200 import gpu as G

    rank, world, local = _rank()
    dist = world > 1
    if dist:
        _init_nccl(local, 300)
    torch.cuda.set_device(local)
    inst = B.random_cavities(args.instances, seed=20250)
    groups = B.build_groups(inst)
    B.initial_fields(groups, inst)
    ctx = G.GpuContext(local)
    B.assign_steps(ctx, groups, inst)
    runner = B.BatchRunner(ctx, groups, device=local)
    tuning = runner.autotune(trial_steps=2)
    gs = args.graph_steps
    runner.capture(gs)
    warm = -(-args.warmup // gs) * gs
    steps = -(-args.steps // gs) * gs
    runner.run(warm)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    t0.record(runner.stream)
    runner.run(steps)
    t1.record(runner.stream)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    ms = t0.elapsed_time(t1)
    ck = clocks.stop()
    states = runner.states(inst)
    finite = all(bool(np.isfinite(y).all()) for y in states)
    if dist:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t)
    n = runner.n_dof
    value = n * 5 * steps * world / (ms * 1e-3)
    stage_ms = ms / (5 * steps)
    alg_bytes = sum(BYTES_PER_DOF_STAGE[g.order] * g.n_dof for g in groups)
    peak, peak_kind = _peaks()
    achieved = alg_bytes / (stage_ms * 1e-3) / 1e9

    # end to end: every group's initial state from pinned host memory, the run,
    # every group's final state back to the host
    hosts = [torch.from_numpy(g.y0).pin_memory() for g in groups]
    outs = [torch.empty(g.n_dof, dtype=torch.float32).pin_memory() for g in groups]
    devs = [torch.empty(g.n_dof, dtype=torch.float32, device="cuda") for g in groups]
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(runner.stream)
    with torch.cuda.stream(runner.stream):
        for h, d in zip(hosts, devs):
            d.copy_(h, non_blocking=True)
        runner.load_device([d.data_ptr() for d in devs])
        runner.run(steps)
        runner.store_device([d.data_ptr() for d in devs])
        for o, d in zip(outs, devs):
            o.copy_(d, non_blocking=True)
    e1.record(runner.stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t)
    e2e_value = n * 5 * steps * world / (e2e_ms * 1e-3)

    line = {
        "metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": steps,
        "warmup": warm, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.instances} PEC cavities: n^3 Kuhn boxes n~U{{4..20}}, order~U{{2..5}}, "
                               "dielectric block eps_r~U[1,10], Gaussian E pulse; LSERK4, each cavity its own "
                               "dt (0.5 * 2.8 / rho); one stage launch per order group, the groups on concurrent streams "
                               "in one CUDA graph",
                   "instances": args.instances, "n_dof": n, "graph_steps": gs, "autotune": tuning,
                   "l2": "state 4*n_dof bytes per buffer >> 126 MB L2; no flush",
                   "parallelism": f"replica x{world}" if world > 1 else "single GPU"},
        "gpu_launches": len(groups) * 5 * steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "kernel": "stage kernels of all order groups",
                     "alg_bytes_per_stage": alg_bytes, "stage_ms": stage_ms, "peak_kind": peak_kind},
        "clocks": ck,
        "e2e": {"value": e2e_value, "unit": "DOF-stage/s", "h2d_bytes_per_step": n * 4 / steps,
                "d2h_bytes_per_step": n * 4 / steps, "steps": steps,
                "api": "GpuOperator.load_device/store_device + BatchRunner.run (graph replays)"},
        "finite": finite,
    }
    if rank == 0 and world == 1 and not args.no_cpu:  # the CPU baseline is an N = 1 figure
        rate, info = cpu_batch_rate(inst, groups)
        line["cpu_baseline"] = {"value": rate, "unit": "DOF-stage/s", "cores": info["cores"], "kind": "port",
                                "sample": info["sample"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del runner
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_c2_accuracy(args):
    """Accuracy of the f32-class engines over the C2 run length: the
    sphere_pulse workload, LSERK4 at dt = 0.5 * 2.8 / rho (the bench's rule),
    `--acc-steps` steps (2000 by default) on the FP32 and the tensor-core
    engines, each compared with the FP64 path on the device run from the same
    f32 initial state.  At `--acc-cells`^3 (16 by default) all three are also
    compared with the f64 oracle on the host's cores (which validates the FP64
    path); at the full 48^3 size (139 M DOFs, where the f64 oracle would take
    hours) the FP64 path is the reference."""
    import ctypes as C

    import torch

    from oracle import oracle as R
    from rapidfem_b200 import _native as nat
    from rapidfem_b200 import gpu as G
    from rapidfem_b200 import workloads as W

    rank, world, local = _rank()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    steps = args.acc_steps
    ctx = G.GpuContext(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    out = {}
    for cells in (args.acc_cells, args.cells):
        wl = W.sphere_pulse(cells, 4)
        op = wl.build()
        gop = G.GpuOperator(ctx, op)
        y0 = wl.y0(op).astype(np.float32)
        rho = C.c_double()
        nat.check(nat.lib.dgtd_power_rho(gop.handle, 40, C.byref(rho)))
        dt = 0.5 * 2.8 / rho.value
        finals, secs = {}, {}
        for name, eng in (("fp32", 0), ("tf32x3", 1)):
            gop.set_engine(eng)
            gop.upload(y0)
            t0 = time.perf_counter()
            gop.run_lserk(dt, steps)
            ctx.synchronize()
            secs[name] = time.perf_counter() - t0
            finals[name] = gop.download().astype(np.float64)
        # the FP64 path on the device from the same f32 initial state: the
        # reference at sizes the CPU oracle cannot reach
        t0 = time.perf_counter()
        ref64 = gop.transient_f64(y0.astype(np.float64), dt, steps)
        secs["fp64"] = time.perf_counter() - t0
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        rec = {"n_dof": int(gop.n_dof()), "dt": dt, "steps": steps, "gpu_seconds": secs,
               "tf32x3_vs_fp32": rel(finals["tf32x3"], finals["fp32"]),
               "fp32_vs_fp64_device": rel(finals["fp32"], ref64),
               "tf32x3_vs_fp64_device": rel(finals["tf32x3"], ref64)}
        if cells == args.acc_cells:
            orc = R.Operator(wl.mesh.nodes, wl.mesh.tets, 4, 1.0, materials=wl.materials)
            t0 = time.perf_counter()
            ref = orc.lserk(y0.astype(np.float64), dt, steps)
            rec["oracle_seconds"] = time.perf_counter() - t0
            rec["oracle_threads"] = R.threads()
            rec["fp32_vs_f64"] = rel(finals["fp32"], ref)
            rec["tf32x3_vs_f64"] = rel(finals["tf32x3"], ref)
            rec["fp64_device_vs_f64"] = rel(ref64, ref)
        out[f"{cells}^3"] = rec
        del gop
    big = out[f"{args.cells}^3"]
    line = {"metric": "relative L2 error after the C2 run length vs f64", "value": big["tf32x3_vs_fp64_device"],
            "unit": "relative L2", "n_gpus": 1, "higher_is_better": False, "dtype": "f32 / tf32x3",
            "data": "synthetic", "config": {"workload": "sphere_pulse (jittered box, N=4, eps_r=4 sphere, "
                                                        "Gaussian Ez pulse), LSERK4", "runs": out}}
    print(json.dumps(line))
    return 0


def run_time_to_t(args):
    """The stiff driven configuration, time to T at <= 1e-4 relative L2 against
    an FP64 reference: the 24^3 x 6 box graded 20:1 toward z = 0, N = 3, a lossy
    slab z < 0.2 (eps_r 2.2, sigma 5), a soft E_z point source at the centre
    with the Gaussian-modulated sine g(t) = exp(-(t-t0)^2/(2 sigma_t^2))
    sin(2 pi f (t-t0)) (f = 2, sigma_t = 0.5, t0 = 5 sigma_t), T = 10.

    Methods: plain FP32 LSERK4 (the FP32 CUDA-core stage kernel at CFL 0.5, the
    source sampled at the stage times), the same on the tensor-core stage
    kernel, and the exponential integrator on the tensor-core matvec with the
    plain adaptive and the learned step controllers (Krylov dimension 10-60,
    the source as a degree-7 polynomial per step).  The reference solution is
    the FP64 path (dgtd_transient_f64_stages) at half the LSERK4 step; it is
    itself checked against the f64 CPU oracle on a coarser mesh of the same
    configuration (`oracle_check`).  The headline value is the learned ETD
    time; each method's ratio to the plain FP32 LSERK4 time is in
    `config.methods`."""
    import ctypes as C

    import torch

    from rapidfem_b200 import _native as nat
    from rapidfem_b200 import etd as E
    from rapidfem_b200 import gpu as G
    from rapidfem_b200 import sources as S
    from rapidfem_b200 import workloads as W

    rank, world, local = _rank()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    n_cells, order, T = args.ttt_cells, 3, args.ttt_time
    f0, sigma_t = 2.0, 0.5
    t0 = 5.0 * sigma_t

    def g(t):
        return S.gaussian_sine(t, t0, sigma_t, f0)

    def problem(cells):
        wl = W.graded_slab(cells, order)
        op = wl.build()
        dof = op.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
        return wl, op, dof

    ctx = G.GpuContext(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)

    def rho_of(gop):
        r = C.c_double()
        nat.check(nat.lib.dgtd_power_rho(gop.handle, 40, C.byref(r)))
        return r.value

    # ---- the FP64 reference path against the CPU oracle at a size the oracle finishes
    oracle_check = None
    if args.ttt_check_cells > 0:
        from oracle import oracle as R
        wl_c, op_c, dof_c = problem(args.ttt_check_cells)
        gop_c = G.GpuOperator(ctx, op_c)
        dt_c = 0.5 * 2.8 / rho_of(gop_c)
        t_chk = min(T, args.ttt_check_time)
        steps_c = int(np.ceil(t_chk / dt_c))
        dt_c = t_chk / steps_c
        gst = S.stage_samples(g, 0.0, dt_c, steps_c)
        # the same discretisation on both sides: LSERK4 with the source held per
        # step (explicit.rs:44-56), the f64 device path against the f64 oracle
        g_held = g(np.arange(steps_c) * dt_c)
        y64 = gop_c.transient_f64(np.zeros(op_c.n_dof), dt_c, steps_c, 1, drive=("point", dof_c), g=g_held)
        R.set_threads(os.cpu_count() or 1)
        orc = R.Operator(wl_c.mesh.nodes, wl_c.mesh.tets, order, 1.0, materials=wl_c.materials)
        yo = orc.lserk(np.zeros(op_c.n_dof), dt_c, steps_c, src_dof=dof_c, vals=g_held)
        oracle_check = {"cells": f"{args.ttt_check_cells}^3", "t": t_chk, "steps": steps_c,
                        "rel_l2_fp64_vs_oracle": float(np.linalg.norm(y64 - yo) / np.linalg.norm(yo))}
        del gop_c

    wl, op, dof = problem(n_cells)
    gop = G.GpuOperator(ctx, op)
    rho = rho_of(gop)
    dt_cfl = 2.8 / rho
    steps = int(np.ceil(T / (0.5 * dt_cfl)))
    dt = T / steps
    n = op.n_dof

    # FP64 reference at half the step, source at the stage times
    w = time.perf_counter()
    g_ref = S.stage_samples(g, 0.0, dt / 2, 2 * steps)
    ref = gop.transient_f64_stages(np.zeros(n), dt / 2, 2 * steps, 1, drive=("point", dof), g=g_ref)
    ref_s = time.perf_counter() - w
    ref_norm = float(np.linalg.norm(ref))

    def rel(a):
        return float(np.linalg.norm(np.asarray(a, dtype=np.float64) - ref) / ref_norm)

    methods = {}
    g_st = S.stage_samples(g, 0.0, dt, steps).astype(np.float32)
    for name, eng in (("lserk4_fp32", nat.ENGINE_FP32), ("lserk4_tf32x3", nat.ENGINE_TF32X3)):
        gop.set_engine(eng)
        gop.upload(np.zeros(n, dtype=np.float32))
        gop.run_lserk_stages(dt, 2, ("point", dof), g_st[:10])  # warm
        gop.upload(np.zeros(n, dtype=np.float32))
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        gop.run_lserk_stages(dt, steps, ("point", dof), g_st)
        e1.record(stream)
        stream.synchronize()
        methods[name] = {"seconds": e0.elapsed_time(e1) * 1e-3, "rel_l2": rel(gop.download()), "steps": steps,
                         "matvecs": 5 * steps, "dt": dt}
    gop.set_engine(nat.ENGINE_TF32X3)
    plain = E.PlainEtd(tol=args.ttt_tol, m_max=60)
    h0 = 8 * dt_cfl
    # controller training: the plain controller's traces on the same mesh with
    # other sources (positions and carrier frequencies), to T / 2
    logs = []
    w = time.perf_counter()
    for c, fq in (([0.3, 0.4, 0.5], 1.5), ([0.6, 0.5, 0.6], 2.5), ([0.5, 0.7, 0.4], 2.0)):
        d_tr = op.nearest_node_dof(c, 0, 2)
        E.run_etd(gop, np.zeros(n), None, lambda t, fq=fq: S.gaussian_sine(t, t0, sigma_t, fq), T / 2, h0, plain,
                  log=logs, point_dof=d_tr)
    trace_s = time.perf_counter() - w
    mlp = E.Mlp(ctx, seed=1)
    w = time.perf_counter()
    losses = E.train_controller(mlp, logs, epochs=3000, lr=3e-3)
    train_s = time.perf_counter() - w
    for name, learned in (("etd_plain", None), ("etd_learned", E.LearnedEtd(mlp, plain))):
        E.run_etd(gop, np.zeros(n), None, g, 4 * h0, h0, plain, learned=learned, point_dof=dof)  # warm
        yf, st = E.run_etd(gop, np.zeros(n), None, g, T, h0, plain, learned=learned, point_dof=dof)
        methods[name] = {"seconds": st.seconds, "rel_l2": rel(yf), "steps": st.accepted, "rejected": st.rejected,
                         "matvecs": st.matvecs, "proposals_kept": st.proposals_kept,
                         "proposals_failed": st.proposals_failed,
                         "h_mean": T / max(st.accepted, 1)}
    base = methods["lserk4_fp32"]["seconds"]
    for m in methods.values():
        m["speedup_vs_lserk4_fp32"] = base / m["seconds"]
        m["within_1e-4"] = m["rel_l2"] <= 1e-4
    line = {
        "metric": "time-to-T at <= 1e-4 relative L2 vs the FP64 reference", "value": methods["etd_learned"]["seconds"],
        "unit": "s", "n_gpus": 1, "steps": methods["etd_learned"]["steps"], "warmup": 1,
        "higher_is_better": False, "scaling": "none", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"graded slab {n_cells}^3 x 6 tets (20:1 toward z=0), N={order}, lossy slab z<0.2 "
                               f"eps_r 2.2 sigma 5, soft E_z point source at the centre, Gaussian-modulated sine "
                               f"f={f0} sigma_t={sigma_t} t0={t0}, T={T}",
                   "n_dof": n, "rho": rho, "dt_cfl": dt_cfl, "methods": methods,
                   "etd": {"tol": plain.tol, "m_max": plain.m_max, "source_terms": 8, "engine": "tf32x3"},
                   "controller_training": {"traces": len(logs), "trace_seconds": trace_s, "epochs": 3000,
                                           "seconds": train_s, "loss_first": float(losses[0]),
                                           "loss_last": float(losses[-1])},
                   "reference": {"kind": "FP64 path (device), LSERK4 at dt/2, source at the stage times",
                                 "seconds": ref_s, "oracle_check": oracle_check}},
        "e2e": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def _c5_setup(args, local):
    """The waveguide-post study's operator, port source and probes, step and
    variants (shared by the LSERK4 and the ETD runs)."""
    import ctypes as C

    import torch

    from rapidfem_b200 import _native as nat
    from rapidfem_b200 import gpu as G
    from rapidfem_b200 import td as T
    from rapidfem_b200 import workloads as W

    c_light = 299792458.0
    a, b_w, L = 22.86e-3, 10.16e-3, 60e-3
    cells = tuple(args.c5_cells)
    wl = W.waveguide_post(6.0, order=3, cells=cells)
    op = wl.build()
    cen = wl.mesh.nodes[wl.mesh.tets].mean(axis=1)
    post = np.hypot(cen[:, 0] - a / 2, cen[:, 2] - L / 2) < 1.5e-3
    prof_in = op.rect_port_profiles(0, [0, 0, 1.0], (1, 0))
    prof_out = op.rect_port_profiles(1, [0, 0, -1.0], (1, 0))
    src = op.port_source(0, prof_in)
    funcs = [op.port_modal_weights(1, prof_out, "E"), op.port_modal_weights(0, prof_in, "E")]
    ctx = G.GpuContext(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    vac = G.GpuOperator(ctx, op, inv_eps=np.ones(3 * op.n_elem))
    rho = C.c_double()
    nat.check(nat.lib.dgtd_power_rho(vac.handle, 40, C.byref(rho)))
    del vac
    dt = 0.5 * 2.8 / rho.value  # operator time c*t; eps_r >= 1 only slows waves
    tau = 2.0 * np.sqrt(np.log(2.0)) / (np.pi * 4e9) * c_light
    t0 = 3.0 * tau
    t_end = t0 + 3.0 * tau + L / 0.7
    steps = int(np.ceil(t_end / dt)) if args.c5_steps <= 0 else args.c5_steps
    V = args.c5_variants
    return {"op": op, "post": post, "src": src, "funcs": funcs, "ctx": ctx, "stream": stream, "rho": rho.value,
            "dt": dt, "steps": steps, "cells": cells, "V": V, "t0": t0, "tau": tau,
            "wave": T.GaussianPulse(t0, tau, 10e9 / c_light),
            "eps_list": [2.0 + 8.0 * k / max(V - 1, 1) for k in range(V)]}


def run_c5_etd(args):
    """The waveguide study under the exponential integrator: the first and last
    post variants (eps_r 2 and 10) run by ETD with the learned step controller
    (tensor-core Krylov matvec, m <= 60, the port source as a polynomial over
    each step), the transmitted and reflected modal amplitudes recorded on the
    device at every accepted step, against plain FP32 LSERK4 (CUDA-core stage
    kernel, the source sampled at the stage times, amplitudes every step).  The
    controller is trained on the plain controller's traces of the middle
    variant (eps_r 6), which is not one of the two checked."""
    import torch

    from rapidfem_b200 import _native as nat
    from rapidfem_b200 import etd as E
    from rapidfem_b200 import gpu as G
    from rapidfem_b200 import sources as S

    rank, world, local = _rank()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    cfg = _c5_setup(args, local)
    op, post, src, funcs, ctx, stream = cfg["op"], cfg["post"], cfg["src"], cfg["funcs"], cfg["ctx"], cfg["stream"]
    dt, steps, wave = cfg["dt"], cfg["steps"], cfg["wave"]
    t_end = steps * dt
    eps_checked = [2.0, 10.0]
    plain = E.PlainEtd(tol=args.ttt_tol, m_max=60)
    h0 = 8 * dt

    def operator(eps):
        gop = G.GpuOperator(ctx, op, inv_eps=np.repeat(np.where(post, 1.0 / eps, 1.0), 3))
        gop.set_source_vector(src)
        return gop

    # training traces: the plain controller on the middle variant
    logs = []
    gop = operator(6.0)
    gop.set_engine(nat.ENGINE_TF32X3)
    _, st_tr = E.run_etd(gop, np.zeros(op.n_dof), src, wave, t_end, h0, plain, log=logs)
    trace = {"eps_r": 6.0, "seconds": st_tr.seconds, "steps": st_tr.accepted, "rejected": st_tr.rejected,
             "matvecs": st_tr.matvecs, "traces": len(logs)}
    del gop
    mlp = E.Mlp(ctx, seed=1)
    w = time.perf_counter()
    losses = E.train_controller(mlp, logs, epochs=3000, lr=3e-3)
    train_s = time.perf_counter() - w
    learned = E.LearnedEtd(mlp, plain)
    g_st = S.stage_samples(wave, 0.0, dt, steps).astype(np.float32)
    variants = []
    for eps in eps_checked:
        gop = operator(eps)
        # plain FP32 LSERK4: amplitudes after every step, recorded on the device
        gop.set_engine(nat.ENGINE_FP32)
        gop.upload(np.zeros(op.n_dof, dtype=np.float32))
        gop.set_functionals(funcs, steps + 1)
        gop.record_functionals(0)
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(steps):
            gop.run_lserk_stages(dt, 1, ("vector", None), g_st[5 * k:5 * k + 5])
            gop.record_functionals(k + 1)
        e1.record(stream)
        stream.synchronize()
        lserk_s = e0.elapsed_time(e1) * 1e-3
        ref = gop.functional_series(steps + 1)
        t_ref = np.arange(steps + 1) * dt
        # learned ETD on the tensor-core matvec
        gop.set_engine(nat.ENGINE_TF32X3)
        _, st = E.run_etd(gop, np.zeros(op.n_dof), src, wave, t_end, h0, plain, learned=learned,
                          functionals=funcs)

        def rel_series(run):
            at = np.stack([np.interp(run.times, t_ref, ref[:, q]) for q in range(ref.shape[1])], axis=1)
            return [float(np.linalg.norm(run.series[:, q] - at[:, q]) / np.linalg.norm(at[:, q]))
                    for q in range(ref.shape[1])]

        rel = rel_series(st)
        plain_run = None
        if eps == eps_checked[0]:
            # the plain controller alone on the same variant
            _, sp = E.run_etd(gop, np.zeros(op.n_dof), src, wave, t_end, h0, plain, functionals=funcs)
            rp = rel_series(sp)
            plain_run = {"seconds": sp.seconds, "steps": sp.accepted, "rejected": sp.rejected,
                         "matvecs": sp.matvecs, "rel_l2_transmitted_Pe": rp[0], "rel_l2_reflected_Pe": rp[1]}
        variants.append({"eps_r": eps, "lserk4_fp32_seconds": lserk_s, "lserk4_steps": steps,
                         "etd_plain": plain_run,
                         "etd_learned_seconds": st.seconds, "etd_steps": st.accepted, "etd_rejected": st.rejected,
                         "etd_matvecs": st.matvecs, "proposals_kept": st.proposals_kept,
                         "proposals_failed": st.proposals_failed,
                         "rel_l2_transmitted_Pe": rel[0], "rel_l2_reflected_Pe": rel[1],
                         "peak_transmitted_Pe": {"lserk4": float(np.max(np.abs(ref[:, 0]))),
                                                 "etd": float(np.max(np.abs(st.series[:, 0])))},
                         "speedup_vs_lserk4_fp32": lserk_s / st.seconds})
        del gop
    line = {
        "metric": "seconds per waveguide variant (learned ETD) with port probes vs plain FP32 LSERK4",
        "value": float(np.mean([v["etd_learned_seconds"] for v in variants])), "unit": "s", "n_gpus": 1,
        "steps": int(np.mean([v["etd_steps"] for v in variants])), "warmup": 0, "higher_is_better": False,
        "scaling": "none", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"WR-90 post variants eps_r {eps_checked} ({op.n_elem} tets, N=3, "
                               f"{op.n_dof} DOFs), TE10 pulse injected at z=0, T={t_end:.5g} (operator time)",
                   "etd": {"tol": plain.tol, "m_max": plain.m_max, "source_terms": 8, "engine": "tf32x3"},
                   "lserk4": {"engine": "fp32", "dt": dt, "source": "sampled at the stage times"},
                   "controller_training": dict(trace, train_seconds=train_s, epochs=3000,
                                               loss_first=float(losses[0]), loss_last=float(losses[-1])),
                   "variants": variants},
        "e2e": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_etd_try(args):
    """One exponential step of the stiff driven configuration timed alone: the
    graded slab (--ttt-cells), N = 3, a soft E_z point source at the centre
    whose Gaussian-modulated sine (f = 2, sigma_t = 0.5, t0 = 2.5) enters as an
    8-term polynomial over the step, h = 0.01, Krylov cap 48 (4 sub-steps of
    12), tol 1e-6, tensor-core matvec.  `--warmup` committed steps from rest,
    then the next step's candidate tried `--steps` times (not committed, so
    every timed try does the same work); reports ms per try and per Arnoldi
    step."""
    import torch

    from rapidfem_b200 import gpu as G
    from rapidfem_b200 import sources as S
    from rapidfem_b200 import workloads as W

    rank, world, local = _rank()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    ctx = G.GpuContext(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    op = W.graded_slab(args.ttt_cells, 3).build()
    gop = G.GpuOperator(ctx, op)
    dof = op.nearest_node_dof([0.5, 0.5, 0.5], 0, 2)
    coef, _ = S.step_polynomial(lambda t: S.gaussian_sine(t, 2.5, 0.5, 2.0), 2.0, 0.01, 8)
    gop.upload(np.zeros(op.n_dof, dtype=np.float32))
    for _ in range(args.warmup):  # committed: the timed tries start from a driven field
        gop.etd_try(0.01, 48, args.ttt_tol, coef=coef, drive=("point", dof))
        gop.etd_commit()
    stream.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dims = []
    for _ in range(args.steps):
        d, est = gop.etd_try(0.01, 48, args.ttt_tol, coef=coef, drive=("point", dof))
        dims.append(d)
    e1.record(stream)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    line = {"metric": "ms per ETD try", "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "scaling": "none", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"graded slab {args.ttt_cells}^3 x 6, N=3, point source, h=0.01, m<=48, "
                                   f"tol {args.ttt_tol}, tensor-core matvec", "n_dof": op.n_dof,
                       "arnoldi_steps_per_try": dims[-1], "est": est,
                       "ms_per_arnoldi_step": ms / max(dims[-1], 1)},
            "e2e": None}
    print(json.dumps(line), flush=True)
    return 0


def run_c5(args):
    """The waveguide study: a 22.86 x 10.16 x 60 mm guide (39 x 17 x 101 hex x 6
    tets), N = 3, a centred dielectric post (r = 1.5 mm) with eps_r spread over
    2-10 in `--c5-variants` variants, a TE10 Gaussian-modulated pulse (10 GHz,
    4 GHz FWHM bandwidth) injected by incident-field flux at z = 0, an absorbing
    port at z = 60 mm, PEC walls; LSERK4 on the tensor-core stage kernel with
    the modal amplitudes P_e of both ports recorded per step on the device, and
    the first and last variants' series checked against the FP32 stage kernel."""
    import torch

    from rapidfem_b200 import _native as nat
    from rapidfem_b200 import gpu as G

    rank, world, local = _rank()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    cfg = _c5_setup(args, local)
    op, post, src, funcs, ctx, stream = cfg["op"], cfg["post"], cfg["src"], cfg["funcs"], cfg["ctx"], cfg["stream"]
    dt, steps, cells, V, eps_list = cfg["dt"], cfg["steps"], cfg["cells"], cfg["V"], cfg["eps_list"]
    g = cfg["wave"](np.arange(steps) * dt).astype(np.float32)

    def run(eps, engine):
        ie = np.repeat(np.where(post, 1.0 / eps, 1.0), 3)
        gop = G.GpuOperator(ctx, op, inv_eps=ie)
        gop.set_engine(engine)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        series, _ = gop.transient_functionals(np.zeros(op.n_dof), dt, steps, 1, drive=("vector", src), g=g,
                                              functionals=funcs)
        e1.record(stream)
        stream.synchronize()
        return series, e0.elapsed_time(e1) * 1e-3

    series, secs = [], []
    for eps in eps_list:
        s_, t_ = run(eps, nat.ENGINE_TF32X3)
        series.append(s_)
        secs.append(t_)
    checks = []
    for k in sorted({0, V - 1}):
        ref, _ = run(eps_list[k], nat.ENGINE_FP32)
        checks.append({"eps_r": eps_list[k],
                       "rel_l2_out": float(np.linalg.norm(series[k][:, 0] - ref[:, 0]) / np.linalg.norm(ref[:, 0])),
                       "rel_l2_in": float(np.linalg.norm(series[k][:, 1] - ref[:, 1]) / np.linalg.norm(ref[:, 1]))})
    total = sum(secs)
    value = V * op.n_dof * 5 * steps / total
    line = {
        "metric": METRIC, "value": value, "unit": "DOF-stage/s", "n_gpus": 1, "steps": steps, "warmup": 0,
        "ms_per_step": total / (V * steps) * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"WR-90 section 22.86x10.16x60 mm, {cells[0]}x{cells[1]}x{cells[2]} hex x 6 = "
                               f"{op.n_elem} tets, N=3, dielectric post r=1.5 mm eps_r in 2..10 ({V} variants), "
                               "TE10 pulse 10 GHz / 4 GHz FWHM injected at z=0, absorbing port at z=60 mm, PEC "
                               "walls; LSERK4 (tensor-core stage kernel), port modal amplitudes per step on the device",
                   "n_dof_per_variant": op.n_dof, "dt_operator": dt, "variants": V,
                   "series_vs_fp32_engine": checks,
                   "peak_transmitted_Pe": [float(np.max(np.abs(s_[:, 0]))) for s_ in series],
                   "seconds_per_variant": secs},
        "gpu_launches": V * 5 * steps + V * (steps + 1),
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_batch_rate(inst, groups, n_inst=4, steps=2):
    """The oracle (f64, OpenMP) on the first instances of the batch."""
    from oracle import oracle as R
    from rapidfem_b200 import operator as O

    R.build()
    cores = os.cpu_count() or 1
    R.set_threads(cores)
    units, secs = 0, 0.0
    for i in range(n_inst):
        g = next(gr for gr in groups if i in gr.members)
        j = g.members.index(i)
        m = O.structured_box(inst[i].cells, inst[i].cells, inst[i].cells)
        orc = R.Operator(m.nodes, m.tets, inst[i].order, 1.0, materials=inst[i].materials)
        y = g.y0[g.dof_slice(j)].astype(np.float64)
        t = time.perf_counter()
        orc.lserk(y, inst[i].dt, steps)
        secs += time.perf_counter() - t
        units += orc.n_dof * 5 * steps
    return units / secs, {"cores": cores, "sample": f"first {n_inst} cavities of the batch, {steps} LSERK4 steps "
                                                   "each (f64 oracle, OpenMP)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cells", type=int, default=48)
    ap.add_argument("--engine", default="tf32x3", choices=["fp32", "tf32x3"],
                    help="stage kernel: FP32 CUDA cores, or the tcgen05 tensor-core kernel (3xTF32 products)")
    ap.add_argument("--power-iters", type=int, default=20)
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--ref-cells", type=int, default=24, help="mesh of the b200 arm's bounded CPU baseline sample")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="seconds of timed steps of the reference arm (full workload)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1 ranks: N independent replicas instead of the partitioned run")
    ap.add_argument("--sharded", action="store_true",
                    help="the partitioned run even on one rank (a one-part partition)")
    ap.add_argument("--workload", default="sphere",
                    choices=["sphere", "c4", "c5", "c5-etd", "time-to-t", "c2-accuracy", "etd-try"],
                    help="sphere: the 48^3 N=4 single-instance workload; c4: the batched cavities; "
                         "c5: the waveguide post variants with port probes; "
                         "c5-etd: two of those variants under the learned ETD controller against FP32 LSERK4; "
                         "etd-try: one exponential step of the time-to-t configuration timed alone; "
                         "time-to-t: LSERK4 vs adaptive / learned ETD to a final time against the oracle")
    ap.add_argument("--c5-variants", type=int, default=32)
    ap.add_argument("--c5-cells", type=int, nargs=3, default=[39, 17, 101])
    ap.add_argument("--c5-steps", type=int, default=0, help="0: long enough for the pulse to cross the guide")
    ap.add_argument("--ttt-cells", type=int, default=24)
    ap.add_argument("--ttt-tol", type=float, default=1e-6, help="ETD a-posteriori Krylov tolerance per step")
    ap.add_argument("--ttt-check-cells", type=int, default=8,
                    help="mesh of the FP64-path-against-oracle check (0: skip)")
    ap.add_argument("--ttt-check-time", type=float, default=10.0)
    ap.add_argument("--acc-cells", type=int, default=16)
    ap.add_argument("--acc-steps", type=int, default=2000)
    ap.add_argument("--ttt-time", type=float, default=10.0)
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--graph-steps", type=int, default=10)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "c4":
        return run_c4(args)
    if args.workload == "time-to-t":
        return run_time_to_t(args)
    if args.workload == "c2-accuracy":
        return run_c2_accuracy(args)
    if args.workload == "c5":
        return run_c5(args)
    if args.workload == "c5-etd":
        return run_c5_etd(args)
    if args.workload == "etd-try":
        return run_etd_try(args)
    if (_rank()[1] > 1 and not args.replicas) or args.sharded:
        return run_sharded(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
