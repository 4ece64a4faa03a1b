#!/usr/bin/env python3
"""Benchmark of the assemble + ILU(0)/IC(0) + Krylov hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl reference]

One step = one pass of the hot path over one synthetic problem: value
assembly into the resident CSR pattern, ILU(0) (IC(0)) factorisation and a
BiCGStab (CG) solve to rtol = atol = 1e-8, all FP64.  At N GPUs every rank
solves its own seeded problem (independent replicas, weak scaling, no
data-path collective); `value` is the solves/s of the whole job, timed on the
device with CUDA events between barriers and taken as the max over ranks.

`--impl reference` times the CPU arm instead: the reference crate cannot be
built here (no Rust toolchain, no MPI), so the arm runs the oracle's C
restatement of the reference's MPI algorithm (block-Jacobi ILU/IC over
contiguous partitions, one OpenMP thread per rank) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "finite-volumes-rs_b200"))

METRIC = "solves/s and DOF-iters/s vs plain FP64 at rel err <=1e-8; p50/p99 solve latency"

WORKLOADS = {
    # plain FP64 3D convection-diffusion, 128^3 hexes x 6 tets (the headline problem)
    "cube128_convdiff": dict(kind="3d", n=128, jitter=0.15, sigma=0.5, velocity=(1.0, 0.5, 0.25), solver="bicgstab"),
    # the CPU-runnable 2D case: 256x256 squares x 2 triangles, lognormal(0,1)
    "square256_diffusion": dict(kind="2d", n=256, jitter=0.2, sigma=1.0, solver="cg"),
    # smaller versions (profiling captures, smoke runs); cube64 still exceeds L2
    # mixed precision: the 3D case with FP32 BiCGStab + FP32 ILU(0)
    # inside FP64 reliable updates, to |b - A x| / |b| <= 1e-10
    "cube128_convdiff_mixed": dict(kind="3d", n=128, jitter=0.15, sigma=0.5, velocity=(1.0, 0.5, 0.25),
                                   solver="bicgstab", precision="mixed"),
    "cube96_convdiff": dict(kind="3d", n=96, jitter=0.15, sigma=0.5, velocity=(1.0, 0.5, 0.25), solver="bicgstab"),
    "cube96_convdiff_mixed": dict(kind="3d", n=96, jitter=0.15, sigma=0.5, velocity=(1.0, 0.5, 0.25),
                                  solver="bicgstab", precision="mixed"),
    "cube64_convdiff": dict(kind="3d", n=64, jitter=0.15, sigma=0.5, velocity=(1.0, 0.5, 0.25), solver="bicgstab"),
    "cube32_convdiff": dict(kind="3d", n=32, jitter=0.15, sigma=0.5, velocity=(1.0, 0.5, 0.25), solver="bicgstab"),
    # batched: 1,024 2D diffusion problems of uneven sizes
    "batch1024_diffusion": dict(kind="batch"),
    # served: a Poisson stream of requests, continuous batching
    "serve_mixed": dict(kind="serve"),
    # the time loop of the crate's examples on the config-1 mesh: implicit Euler,
    # per step value-only re-assembly, ILU(0) refactorisation, BiCGStab from
    # the previous solution
    "cube128_transient": dict(kind="transient", n=128, jitter=0.15, sigma=0.5, velocity=(1.0, 0.5, 0.25),
                              dt=2e-3),
}
RTOL = 1e-8


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_problem(fv, wl, seed, on_device=False):
    if wl["kind"] == "3d":
        m = fv.Mesh.cube(wl["n"], wl["jitter"], seed, on_device=on_device)
        kappa0 = float(np.linalg.norm(wl["velocity"])) * (1.0 / wl["n"]) / 3.0
        kf, fl, sc = m.fields(seed, kappa0, wl["sigma"], velocity=wl["velocity"], source_uniform=True)
        coef = (-1.0, 1.0, -1.0)
    else:
        m = fv.Mesh.square(wl["n"], wl["jitter"], seed, on_device=on_device)
        kf, _, sc = m.fields(seed, 1.0, wl["sigma"], source_const=1.0)
        fl = None
        coef = (-1.0, 0.0, -1.0)
    nb = m.n_boundary_faces
    return dict(mesh=m, kappa=kf, flux=fl, source=sc, bndi=np.zeros(nb), bnde=np.zeros(nb), coef=coef)


def device_mesh_build_s(fv, wl, seed):
    """Wall time of fv_mesh_build_cube / _square: the element list generated on
    the host, then faces, geometry and gradient coefficients on the GPU, no
    read back."""
    import ctypes as C

    import torch

    from fvb200._lib import check, lib
    from fvb200.streams import stream_handle
    h = C.c_void_p()
    fn = lib().fv_mesh_build_cube if wl["kind"] == "3d" else lib().fv_mesh_build_square
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    check(fn(wl["n"], wl["jitter"], seed, stream_handle(None), C.byref(h), None), "fv_mesh_build")
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    lib().fv_mesh_destroy(h)
    return t


def equation(fv, prob, tensors):
    lap = fv.laplacian(fv.Orthogonal(), tensors["kappa"])
    src = fv.source(tensors["source"])
    if prob["coef"][1] != 0.0:
        return fv.convection(fv.Upwind(tensors["flux"]), tensors["flux"]) - lap - src
    return -lap - src


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, tag: str = ""):
        self.index = index
        self.tag = tag
        self.proc = None
        self.path = None

    def start(self):
        try:
            # raw samples go to FV_BENCH_CLOCKS_DIR when set (kept for inspection), else a temporary folder
            out = Path(os.environ.get("FV_BENCH_CLOCKS_DIR") or tempfile.mkdtemp(prefix="fv_clocks_"))
            out.mkdir(parents=True, exist_ok=True)
            self.path = out / f"clocks_rank{self.index}{self.tag}.csv"
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
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
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def sweep_schedule(P):
    """Which sweep schedule the preconditioner uses, with its box-tile plan."""
    if P.perm is not None:
        return {"kind": "reordered factorisation: contiguous levels, block tickets (k_sweep_seq)"}
    act, st = P.schedule()
    if act == 3:
        return {"kind": "level chunks, next chunk prefetched"}
    if act == 4:
        return {"kind": "permuted system: rows sorted by level, consecutive rows, block tickets (k_sweep_seq)"}
    if act != 2:
        return {"kind": "level chunks"}
    return {"kind": "box tiles", "box_edge_cells": float(st[0]), "boxes": int(st[1]),
            "lane_use": [round(float(st[2]), 3), round(float(st[3]), 3)],
            "ring_share": [round(float(st[4]), 3), round(float(st[5]), 3)]}


def time_kernel(torch, fn, reps, stream):
    """Average device time of fn() over reps launches, CUDA events on `stream`."""
    for _ in range(2):
        fn()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps / 1e3


def setup_single(args, wl, rank, world, local_rank):
    """Build the library, the seeded problem of a single-problem workload on
    the device and its equation; returns the shared context."""
    import torch
    torch.cuda.set_device(local_rank)
    from fvb200.build import build
    if rank == 0:
        build()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    build()
    import fvb200 as fv
    t0 = time.time()
    prob = make_problem(fv, wl, seed=1000 + rank, on_device=True)
    t_mesh = time.time() - t0
    t_mesh_dev = device_mesh_build_s(fv, wl, 1000 + rank)
    dev = torch.device("cuda", local_rank)
    T = {k: torch.as_tensor(prob[k], device=dev) for k in ("kappa", "source", "bndi", "bnde")}
    T["flux"] = torch.as_tensor(prob["flux"], device=dev) if prob["flux"] is not None else None
    return dict(fv=fv, torch=torch, wl=wl, prob=prob, mesh=prob["mesh"], T=T, eq=equation(fv, prob, T),
                bc=(T["bndi"], T["bnde"]), t_mesh=t_mesh, t_mesh_dev=t_mesh_dev, dev=dev, world=world,
                local_rank=local_rank, A=None)


def measure_single(ctx, ordering, steps, warmup, precision="fp64", e2e=True, kernels=True, tol=None,
                   reorder="system"):
    """Time `steps` steps (after `warmup`) of one single-problem workload:
    value assembly into the resident pattern, refactorisation and a solve from
    x0 = 0 (BiCGStab + ILU(0) in 3D, CG + IC(0) in 2D) to rtol = atol = 1e-8
    (FP64), or the FP32 Krylov + FP32 factors inside FP64 reliable updates to
    |b - Ax|/|b| <= 1e-10 (precision "mixed").  ordering None = the
    reference's natural order; "boxes" = the box-colour order, either as the
    permuted system (reorder "system": B = Q A Q^T factorised and solved in
    its own numbering, b permuted in and x back every step) or as the
    reordered factorisation applied in A's numbering (reorder "precond").  tol
    replaces the target: rtol = atol (FP64) or the outer tolerance (mixed)."""
    fv, torch, wl = ctx["fv"], ctx["torch"], ctx["wl"]
    from fvb200._lib import lib
    world, local_rank = ctx["world"], ctx["local_rank"]
    mesh, eq, bc, T, prob = ctx["mesh"], ctx["eq"], ctx["bc"], ctx["T"], ctx["prob"]
    stream = torch.cuda.current_stream()
    Pcls = fv.IncompleteLowerUpper if wl["solver"] == "bicgstab" else fv.IncompleteCholesky
    solve = fv.bi_conjugate_gradient_stab if wl["solver"] == "bicgstab" else fv.conjugate_gradient
    opts = fv.LinearSolverOptions(tol or RTOL, tol or RTOL, 10000)
    outer_tol = tol or 1e-10
    N = mesh.n_cells

    # first pass builds the resident pattern, symbolic analysis and factor storage
    if ctx["A"] is None:
        ctx["A"], _ = fv.assemble(eq, bc, mesh)
    A = ctx["A"]
    _, b = fv.assemble(eq, bc, mesh, lhs=A)
    system = ordering is not None and reorder == "system"
    t0 = time.perf_counter()
    order_info = None
    if system:
        perm, order_info = fv.order_boxes(A)
        S = A.permuted(perm)  # the system solved: Q A Q^T
        P = Pcls.from_matrix(S, 0)
        bq = fv.DistributedVector.from_size(N)
        y = fv.DistributedVector.from_size(N)
    else:
        S = A
        P = Pcls.from_matrix(A, 0, ordering=ordering)
        order_info = P.order_info
    torch.cuda.synchronize()
    t_factor_setup = time.perf_counter() - t0
    x = fv.DistributedVector.from_size(N)

    mixed = precision == "mixed"
    if mixed:
        from types import SimpleNamespace

        from fvb200.batch import BatchCG
        single = BatchCG(S, [0, N], 2048)

    # one step: value assembly (new rhs), refactorisation, solve from x0 = 0
    def step_b(marks=None):
        nonlocal b
        _, b = fv.assemble(eq, bc, mesh, lhs=A)
        if marks is not None:
            marks.append(torch.cuda.Event(enable_timing=True))
            marks[-1].record(stream)
        if system:
            S.refresh_permuted()
        P.refactor()
        if marks is not None:
            marks.append(torch.cuda.Event(enable_timing=True))
            marks[-1].record(stream)
        rhs, sol = (bq, y) if system else (b, x)
        if system:
            S.to_permuted(b, bq)
        sol.data.zero_()
        if mixed:
            o = single.solve(P, rhs, sol, precision="mixed", outer_tolerance=outer_tol,
                             inner_relative_tolerance=ctx.get("mixed_delta", 1e-2),
                             max_iterations=20000, solver=wl["solver"])
            out = SimpleNamespace(iterations=int(o["iterations"][0]), refinements=int(o["outer_steps"][0]),
                                  fallback=int(o["fp64_fallback"][0]), final=float(o["final_residual"][0]))
        else:
            out = solve(sol, S, rhs, P, None, opts)
        if system:
            S.from_permuted(y, x)
        return out

    for _ in range(warmup):
        info = step_b()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    clk = Clocks(local_rank, f"_{ordering or 'natural'}_{precision}")
    clk.start()
    torch.cuda.synchronize()
    L0 = lib().fv_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    lat, iters, phases = [], [], []
    e0.record(stream)
    for _ in range(steps):
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        marks = []
        info = step_b(marks)
        s1.record(stream)
        iters.append(info.iterations)
        lat.append((s0, s1))
        phases.append((s0, marks, s1))
    e1.record(stream)
    torch.cuda.synchronize()
    # assembly / refactorisation / solve of every step (ms)
    phase_ms = [[round(s0.elapsed_time(m[0]), 2), round(m[0].elapsed_time(m[1]), 2), round(m[1].elapsed_time(s1), 2)]
                for s0, m, s1 in phases]
    launches = lib().fv_launch_count() - L0
    clocks = clk.stop()
    elapsed = e0.elapsed_time(e1) / 1e3
    lat_ms = [a.elapsed_time(c) for a, c in lat]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([elapsed], device=ctx["dev"], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    # correctness of the last step: true residual, and error against a tight FP64 solve
    r = fv.DistributedVector.from_size(N)
    A.imul(r, x)
    relres = float(torch.linalg.norm(r.data - b.data) / torch.linalg.norm(b.data))
    if ctx.get("x_tight") is None:
        Pn = Pcls.from_matrix(A, 0)
        xt = fv.DistributedVector.from_size(N)
        solve(xt, A, b, Pn, None, fv.LinearSolverOptions(1e-13, 1e-13, 20000))
        ctx["x_tight"] = xt
        del Pn
    xt = ctx["x_tight"]
    err_tight = float(torch.linalg.norm(x.data - xt.data) / torch.linalg.norm(xt.data))
    mixed_info = None
    if mixed:
        mixed_info = {"refinement_steps": info.refinements, "fp64_fallback": info.fallback,
                      "final_fp64_residual": info.final}
    res = dict(elapsed=elapsed, steps=steps, N=N, nnz=A.shape()[2], iters=iters, lat_ms=lat_ms, relres=relres,
               err_tight=err_tight, launches=launches, clocks=clocks, phase_ms=phase_ms, mixed_info=mixed_info,
               order_info=order_info, levels=P.levels()[2:], schedule=sweep_schedule(P),
               reorder=(reorder if ordering is not None else None),
               factor_setup_s=round(t_factor_setup, 3), x=x.numpy())

    if e2e:
        # ---- end to end through the public API with host buffers
        pin = {k: torch.empty(len(prob[k]), dtype=torch.float64).pin_memory()
               for k in ("kappa", "source", "bndi", "bnde") + (("flux",) if prob["flux"] is not None else ())}
        for k, t in pin.items():
            t.copy_(torch.from_numpy(prob[k]))
        x_host = torch.empty(N, dtype=torch.float64).pin_memory()
        h2d = sum(t.numel() * 8 for t in pin.values())

        def e2e_step():
            for k, t in pin.items():
                T[k].copy_(t, non_blocking=True)
            step_b()
            x_host.copy_(x.data, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        clk2 = Clocks(local_rank, "_e2e")
        clk2.start()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2e_lat = []
        e2.record(stream)
        for _ in range(steps):
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            e2e_step()
            s1.record(stream)
            e2e_lat.append((s0, s1))
        e3.record(stream)
        torch.cuda.synchronize()
        e2e_clocks = clk2.stop()
        e2e_elapsed = e2.elapsed_time(e3) / 1e3
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([e2e_elapsed], device=ctx["dev"], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_elapsed = float(t.item())
        res.update(e2e_elapsed=e2e_elapsed, h2d=h2d, d2h=N * 8,
                   e2e_lat_ms=[round(a.elapsed_time(c), 1) for a, c in e2e_lat], e2e_clocks=e2e_clocks)

    if kernels:
        # ---- per-kernel timing of the hot kernels (roofline)
        nnz = res["nnz"]
        yk = fv.DistributedVector.from_size(N)
        zk = fv.DistributedVector.from_size(N)
        hbm, peak_kind = peaks()
        t_spmv = time_kernel(torch, lambda: S.imul(yk, x), 20, stream)  # the solved system's matrix
        t_prec = time_kernel(torch, lambda: P.precondition(zk, b), 10, stream)
        # the assembly kernel alone: the fv_assemble C call with prebuilt descriptors into a preallocated rhs
        from fvb200.linalg import assembly_launcher
        b_fixed = fv.DistributedVector.from_size(N)
        t_asm = time_kernel(torch, assembly_launcher(eq, bc, mesh, A, b_fixed), 10, stream)
        t_fac = time_kernel(torch, lambda: P.refactor(), 3, stream)
        F, Fb = mesh.n_faces, mesh.n_boundary_faces
        bytes_spmv = 12 * nnz + 20 * N
        # ILU(0) apply: 12 nnz + 40 N; IC(0): 2 (12 (nnz + N) / 2 + 28 N); the reordered
        # factorisation applied in A's numbering also reads the permutation twice (8 N)
        bytes_prec = (12 * nnz + 40 * N) if wl["solver"] == "bicgstab" else (12 * (nnz + N) + 56 * N)
        if ordering is not None and not system:
            bytes_prec += 8 * N
        # assembly (Orthogonal scheme, the mesh's cached geometry): per face area, kappa, flux, 1/|d| and the
        # owner/neighbour pair; per boundary face the two constraint values; per cell volume and source;
        # the values and the right-hand side written
        bytes_asm = 40 * F + 16 * Fb + 16 * N + 8 * nnz + 8 * N
        it_mean = float(np.mean(iters))
        per_it = 2 if wl["solver"] == "bicgstab" else 1
        step_s = elapsed / steps
        share = {
            "precond_apply": t_prec * per_it * it_mean / step_s,
            "spmv": t_spmv * per_it * it_mean / step_s,
            "assembly": t_asm / step_s,
            "factor": t_fac / step_s,
        }
        kern = {"precond_apply": (bytes_prec, t_prec), "spmv": (bytes_spmv, t_spmv), "assembly": (bytes_asm, t_asm)}
        dom = max(("precond_apply", "spmv", "assembly"), key=lambda k: share[k])
        bts, tk = kern[dom]
        ach = bts / tk / 1e9
        res.update(
            roofline={"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                      "frac": round(ach / hbm, 4), "peak_kind": peak_kind, "algorithmic_bytes": int(bts),
                      "launch_ms": round(tk * 1e3, 4)},
            kernels={k: {"achieved_gbs": round(kern[k][0] / kern[k][1] / 1e9, 1),
                         "frac": round(kern[k][0] / kern[k][1] / 1e9 / hbm, 4),
                         "launch_ms": round(kern[k][1] * 1e3, 4), "algorithmic_bytes": int(kern[k][0])}
                     for k in kern},
            share={k: round(v, 4) for k, v in share.items()}, t_factor_ms=round(t_fac * 1e3, 3))
    del P
    return res


def single_summary(res, world, label):
    """A sub-object of the JSON line for one measured single-problem mode."""
    K = res["steps"]
    value = K * world / res["elapsed"]
    lat = sorted(res["lat_ms"])
    out = {"label": label, "value": round(value, 4), "unit": "solves/s", "steps": K,
           "ms_per_step": round(res["elapsed"] / K * 1e3, 3), "iterations": res["iters"],
           "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
           "dof_iters_per_s": round(res["N"] * float(np.mean(res["iters"])) * value, 1),
           "true_rel_residual": res["relres"], "rel_err_vs_tight_fp64": res["err_tight"],
           "levels_fwd_bwd": list(res["levels"]), "ordering_info": res["order_info"],
           "step_phase_ms_last": res["phase_ms"][-1], "clocks": res["clocks"], "gpu_launches": int(res["launches"])}
    if res.get("kernels"):
        out["kernels"] = res["kernels"]
        out["roofline"] = res["roofline"]
    if res.get("mixed_info"):
        out["mixed"] = res["mixed_info"]
    return out


def cpu_full_solve(prob, wl):
    """One complete solve of the workload by the oracle on one host thread
    (one reference rank): assembly (pattern + values), ILU(0) / IC(0)
    factorisation and the Krylov solve to rtol = atol = 1e-8, all timed."""
    import oracle
    m = prob["mesh"]
    c = prob["coef"]
    kind = "ilu" if wl["solver"] == "bicgstab" else "ic"
    solver = oracle.bicgstab if wl["solver"] == "bicgstab" else oracle.cg
    t0 = time.perf_counter()
    ptr, cols, vals, rhs = oracle.assemble(m, c[0], c[1], c[2], kappa=prob["kappa"], flux=prob["flux"],
                                           source=prob["source"], bndi=prob["bndi"], bnde=prob["bnde"])
    t1 = time.perf_counter()
    pc = oracle.Precond(kind, ptr, cols, vals)
    t2 = time.perf_counter()
    x, info = solver(ptr, cols, vals, pc, rhs, rtol=RTOL, atol=RTOL, maxit=10000)
    t3 = time.perf_counter()
    sample = (f"oracle (1 thread): one complete solve -- assembly + {kind.upper()}(0) + {wl['solver']} to rtol "
              f"{RTOL} ({info['iterations']} iterations) -- timed, no extrapolation")
    return dict(t_solve=t3 - t0, t_asm=t1 - t0, t_fac=t2 - t1, t_krylov=t3 - t2, iters=int(info["iterations"]),
                sample=sample, x=x)


def oracle_problem(wl, seed):
    """The workload's inputs generated by the oracle itself (oracle/oracle_mesh.c:
    the same mesh and fields as make_problem, bit for bit), so that the
    reference arm never loads the product library."""
    from oracle import gen
    if wl["kind"] == "3d":
        m = gen.Mesh.cube(wl["n"], wl["jitter"], seed)
        kappa0 = float(np.linalg.norm(wl["velocity"])) * (1.0 / wl["n"]) / 3.0
        kf, fl, sc = m.fields(seed, kappa0, wl["sigma"], velocity=wl["velocity"], source_uniform=True)
        coef = (-1.0, 1.0, -1.0)
    else:
        m = gen.Mesh.square(wl["n"], wl["jitter"], seed)
        kf, _, sc = m.fields(seed, 1.0, wl["sigma"], source_const=1.0)
        fl = None
        coef = (-1.0, 0.0, -1.0)
    nb = m.n_boundary_faces
    return dict(mesh=m, kappa=kf, flux=fl, source=sc, bndi=np.zeros(nb), bnde=np.zeros(nb), coef=coef)


# wall-clock bound of the whole reference arm (the driver allows 1,800 s per step)
REFERENCE_BUDGET_S = 1500.0


def reference_arm(args, rank, world):
    """The CPU reference arm: the oracle's C restatement of what the crate
    computes on P MPI ranks (oracle/oracle_mpi.c: contiguous partitions, one
    OpenMP thread per rank, every rank assembling its own rows, block-Jacobi
    ILU(0)/IC(0) of its square block, halo = shared vector, reduce_add = sum
    in rank order), on all host cores.  Every warm-up and timed step is one
    complete solve of the workload: assembly (pattern + values),
    factorisation and the Krylov solve to rtol = atol = 1e-8.  Inputs come
    from the oracle's own generator; the product library is not loaded."""
    if rank != 0:
        return
    import oracle
    from oracle import mpi as ompi
    t_start = time.time()
    wl = WORKLOADS[args.workload]
    if wl["kind"] not in ("2d", "3d"):
        print(json.dumps({"impl": "reference", "unavailable": f"the reference arm covers the single-problem "
                          f"workloads; {args.workload} has none"}), flush=True)
        return
    oracle.lib()
    prob = oracle_problem(wl, seed=1000)
    t_gen = time.time() - t_start
    threads = os.cpu_count() or 1
    m, c = prob["mesh"], prob["coef"]
    kind = "ilu" if wl["solver"] == "bicgstab" else "ic"

    def step():
        t0 = time.perf_counter()
        ptr, cols, vals, rhs = ompi.assemble(m, c[0], c[1], c[2], prob["kappa"], prob["flux"], prob["source"],
                                             prob["bndi"], prob["bnde"], threads)
        bj = ompi.BlockJacobi(kind, ptr, cols, vals, threads)
        x, info = ompi.solve(wl["solver"], ptr, cols, vals, bj, rhs, RTOL, RTOL, 10000)
        return time.perf_counter() - t0, info, x, (ptr, cols, vals, rhs)

    warm = []
    for _ in range(args.warmup):
        warm.append(step()[0])
    # timed steps: all K unless the wall budget would run out (then as many as fit, reported)
    per = warm[-1] if warm else None
    steps = args.steps
    if per:
        left = REFERENCE_BUDGET_S - (time.time() - t_start)
        steps = max(1, min(args.steps, int(left / per)))
    times, iters = [], []
    last = None
    for _ in range(steps):
        t, info, x, sysm = step()
        times.append(t)
        iters.append(int(info["iterations"]))
        last = (x, sysm)
    x, (ptr, cols, vals, rhs) = last
    r = oracle.spmv(ptr, cols, vals, x) - rhs
    relres = float(np.linalg.norm(r) / np.linalg.norm(rhs))
    total = float(np.sum(times))
    value = len(times) / total
    N = m.n_cells
    nnz = int(len(cols))
    lat = sorted(t * 1e3 for t in times)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "solves/s", "n_gpus": args.gpus,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": round(total / len(times) * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(args, wl, N, nnz),
        "dof_iters_per_s": round(N * float(np.mean(iters)) * value, 1),
        "iterations": iters, "p50_ms": round(float(np.percentile(lat, 50)), 1),
        "p99_ms": round(float(np.percentile(lat, 99)), 1), "true_rel_residual": relres,
        "warmup_ms": [round(t * 1e3, 1) for t in warm],
        "cpu_baseline": {"value": round(value, 6), "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"every step one complete solve: assembly on {threads} ranks + block-Jacobi "
                                   f"{kind.upper()}(0) over {threads} contiguous partitions + {wl['solver']} to "
                                   f"rtol {RTOL}, timed (no extrapolation)"},
        "e2e": {"value": round(value, 6), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "input_generation_s": round(t_gen, 1),
        "note": "reference crate not buildable here (no Rust toolchain, no MPI): C restatement of its MPI "
                "block-Jacobi algorithm on all host cores; inputs from the oracle's own generator (the product "
                "library is not loaded)",
    }
    if steps < args.steps:
        line["steps_requested"] = args.steps
        line["steps_note"] = f"timed steps capped so the arm ends within {REFERENCE_BUDGET_S:.0f} s of wall time"
    print(json.dumps(line), flush=True)


def config_of(args, wl, N, nnz):
    return {"workload": args.workload, "cells": N, "nnz": nnz, "dim": 3 if wl["kind"] == "3d" else 2,
            "solver": f"{wl['solver']}+{'ilu0' if wl['solver'] == 'bicgstab' else 'ic0'}", "rtol": RTOL,
            "atol": RTOL, "precision": "fp64", "l2": "inputs larger than L2 (no flush needed)"
            if N > 1_000_000 else "working set fits L2; reported as effective bandwidth",
            "parallelism": f"replicas x{args.gpus}"}


def transient_arm(args, rank, world, local_rank):
    """Implicit-Euler time loop on the config-1 problem (what every example of
    the crate runs): time(Euler(u, dt)) + convection(Upwind(F), F)
    - laplacian(Orthogonal, kappa) - source(f), u0 = 0.  One step = value-only
    re-assembly into the resident pattern, ILU(0) refactorisation, BiCGStab to
    rtol 1e-8 from the previous solution.  Metric: time steps per second."""
    import torch
    torch.cuda.set_device(local_rank)
    from fvb200.build import build
    build()
    import fvb200 as fv
    from fvb200._lib import lib
    wl = WORKLOADS[args.workload]
    prob = make_problem(fv, dict(wl, kind="3d"), seed=1000 + rank, on_device=True)
    mesh = prob["mesh"]
    dev = torch.device("cuda", local_rank)
    T = {k: torch.as_tensor(prob[k], device=dev) for k in ("kappa", "flux", "source", "bndi", "bnde")}
    bc = (T["bndi"], T["bnde"])
    N = mesh.n_cells
    u = torch.zeros(N, dtype=torch.float64, device=dev)
    opts = fv.LinearSolverOptions(RTOL, RTOL, 10000)
    stream = torch.cuda.current_stream()
    A = P = S = None
    system = args.ordering != "natural" and args.reorder == "system"
    bq = y = None

    def step():
        nonlocal A, P, S, u, bq, y
        eq = (fv.time(fv.Euler(u, wl["dt"])) + fv.convection(fv.Upwind(T["flux"]), T["flux"])
              - fv.laplacian(fv.Orthogonal(), T["kappa"]) - fv.source(T["source"]))
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        if A is None:
            A, b = fv.assemble(eq, bc, mesh)
            ev[1].record(stream)
            if system:  # the box order as the permuted system, solved in its own numbering
                perm, _ = fv.order_boxes(A)
                S = A.permuted(perm)
                P = fv.IncompleteLowerUpper.from_matrix(S, 0)
                bq = fv.DistributedVector.from_size(N)
                y = fv.DistributedVector.from_size(N)
                S.to_permuted(u, y)
            else:
                P = fv.IncompleteLowerUpper.from_matrix(A, 0, ordering=None if args.ordering == "natural"
                                                        else args.ordering)
        else:
            _, b = fv.assemble(eq, bc, mesh, lhs=A)
            ev[1].record(stream)
            if system:
                S.refresh_permuted()
            P.refactor()
        ev[2].record(stream)
        if system:  # from the previous solution, kept in the permuted numbering
            S.to_permuted(b, bq)
            info = fv.bi_conjugate_gradient_stab(y, S, bq, P, None, opts)
            x = fv.DistributedVector.from_size(N)
            S.from_permuted(y, x)
        else:
            x = fv.DistributedVector(u.clone())
            info = fv.bi_conjugate_gradient_stab(x, A, b, P, None, opts)
        ev[3].record(stream)
        u = x.data
        return info.iterations, ev

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clk = Clocks(local_rank)
    clk.start()
    L0 = lib().fv_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    its, phases = [], []
    for _ in range(args.steps):
        n_it, ev = step()
        its.append(int(n_it))
        phases.append(ev)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    launches = lib().fv_launch_count() - L0
    elapsed = e0.elapsed_time(e1) / 1e3
    ph = [[round(ev[0].elapsed_time(ev[1]), 2), round(ev[1].elapsed_time(ev[2]), 2), round(ev[2].elapsed_time(ev[3]), 2)]
          for ev in phases]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([elapsed], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    line = {
        "metric": "implicit-Euler time steps/s (re-assembly + ILU(0) refactorisation + BiCGStab to rtol 1e-8)",
        "value": round(args.steps * world / elapsed, 4), "unit": "time steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(elapsed / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "cells": N, "dt": wl["dt"], "solver": "bicgstab+ilu0",
                   "ordering": args.ordering, "reorder": args.reorder if args.ordering != "natural" else None,
                   "rtol": RTOL, "parallelism": f"replicas x{world}"},
        "iterations": its, "step_phase_ms": ph, "phase_names": ["assemble", "refactor", "solve"],
        "gpu_launches": int(launches), "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def batch_problems(fv, count, seed, rank):
    """The batched workload: `count` 2D diffusion problems built as the
    256x256 case, sides log-uniform in [32, 512], per-problem sigma ~ U(0.5, 2),
    seeds seed+k.  Meshes are generated on all host cores."""
    from concurrent.futures import ThreadPoolExecutor
    rng = np.random.default_rng(seed + 7919 * rank)
    sides = np.rint(np.exp(rng.uniform(np.log(32), np.log(512), count))).astype(int)
    sigmas = rng.uniform(0.5, 2.0, count)

    def one(k):
        m = fv.Mesh.square(int(sides[k]), 0.2, seed + k)
        kf, _, sc = m.fields(seed + k, 1.0, float(sigmas[k]), source_const=1.0)
        return m, kf, sc

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        probs = list(ex.map(one, range(count)))
    return probs, sides, sigmas


def batch_arm(args, rank, world, local_rank):
    """Batched CG + IC(0) over 1,024 independent 2D problems, FP64 or FP32 inner
    with FP64 refinement (the faster of the two in a warm-up trial by default)."""
    import torch
    torch.cuda.set_device(local_rank)
    from fvb200.build import build
    build()
    import fvb200 as fv
    from fvb200._lib import lib
    from fvb200.batch import BatchCG, MeshBatch, autotune_schedule, autotune_tile
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    t0 = time.time()
    probs, sides, sigmas = batch_problems(fv, args.batch_count, 5000, rank)
    mb = MeshBatch([p[0] for p in probs])
    kf = torch.as_tensor(mb.face_field([p[1] for p in probs]), device=dev)
    sc = torch.as_tensor(mb.cell_field([p[2] for p in probs]), device=dev)
    t_mesh = time.time() - t0
    nb = mb.n_boundary_faces
    bc = (torch.zeros(nb, dtype=torch.float64, device=dev), torch.zeros(nb, dtype=torch.float64, device=dev))
    eq = -fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
    A, b = fv.assemble(eq, bc, mb)
    ordering = None if args.ordering == "natural" else args.ordering
    t0 = time.time()
    P = fv.IncompleteCholesky.from_matrix(A, 0, ordering=ordering, offsets=mb.cell_offsets if ordering else None)
    t_factor_setup = time.time() - t0
    x = fv.DistributedVector.from_size(mb.n_cells)
    tile, tile_times = autotune_tile(A, mb.cell_offsets, P, b, x)
    sched, sched_times = autotune_schedule(P, b, x) if ordering is None else (None, {})
    solver = BatchCG(A, mb.cell_offsets, tile)
    # both precisions reach the same FP64 target |b - A x| / |b| <= 1e-10 per problem
    opts_by = {"mixed": dict(precision="mixed", outer_tolerance=BATCH_OUTER_TOL, inner_relative_tolerance=1e-2,
                             max_outer=30, max_iterations=20000),
               "fp64": dict(precision="fp64", relative_tolerance=BATCH_OUTER_TOL,
                            absolute_tolerance=BATCH_OUTER_TOL, max_iterations=20000)}
    choice = args.batch_precision if args.batch_precision != "auto" else "mixed"

    def step(prec=None):
        nonlocal b
        _, b = fv.assemble(eq, bc, mb, lhs=A)
        P.refactor()
        return solver.solve(P, b, x, **opts_by[prec or choice])

    # precision autotune: one warm-up step of each, the faster one is timed
    trial = {}
    for k in range(args.warmup):
        prec = None
        if args.batch_precision == "auto" and k < 2:
            prec = ("mixed", "fp64")[k]
        w0 = torch.cuda.Event(enable_timing=True)
        w1 = torch.cuda.Event(enable_timing=True)
        w0.record(stream)
        out = step(prec)
        w1.record(stream)
        torch.cuda.synchronize()
        if prec:
            trial[prec] = w0.elapsed_time(w1) / 1e3
            if len(trial) == 2:
                choice = min(trial, key=trial.get)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    clk = Clocks(local_rank)
    clk.start()
    torch.cuda.synchronize()
    L0 = lib().fv_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    outs = []
    for _ in range(args.steps):
        outs.append(step())
    e1.record(stream)
    torch.cuda.synchronize()
    launches = lib().fv_launch_count() - L0
    clocks = clk.stop()
    elapsed = e0.elapsed_time(e1) / 1e3
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    out = outs[-1]
    # the other precision, one timed step (the same accuracy target)
    other = "fp64" if choice == "mixed" else "mixed"
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    xo = fv.DistributedVector.from_size(mb.n_cells)
    f0.record(stream)
    _, b = fv.assemble(eq, bc, mb, lhs=A)
    P.refactor()
    out_other = solver.solve(P, b, xo, **opts_by[other])
    f1.record(stream)
    torch.cuda.synchronize()
    t_other = f0.elapsed_time(f1) / 1e3
    del xo
    # accuracy: every problem's true FP64 residual; error against a tight FP64
    # solve on a sample of problems (each solved alone, plain FP64 path)
    rng = np.random.default_rng(11)
    sample = sorted(rng.choice(args.batch_count, size=min(args.plain_sample, args.batch_count), replace=False))
    xs = x.numpy()
    errs, plain_t = [], []
    for k in sample:
        m, kfk, sck = probs[k]
        nbk = m.n_boundary_faces
        eqk = -fv.laplacian(fv.Orthogonal(), kfk) - fv.source(sck)
        zb = (np.zeros(nbk), np.zeros(nbk))
        torch.cuda.synchronize()
        s0 = time.perf_counter()
        Ak, bk = fv.assemble(eqk, zb, m)
        Pk = fv.IncompleteCholesky.from_matrix(Ak, 0)
        xk = fv.DistributedVector.from_size(m.n_cells)
        fv.conjugate_gradient(xk, Ak, bk, Pk, None, fv.LinearSolverOptions(RTOL, RTOL, 20000))
        torch.cuda.synchronize()
        plain_t.append(time.perf_counter() - s0)
        # tight reference for the error
        xt = fv.DistributedVector.from_size(m.n_cells)
        fv.conjugate_gradient(xt, Ak, bk, Pk, None, fv.LinearSolverOptions(1e-13, 1e-13, 40000))
        r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
        xr = xt.numpy()
        errs.append(float(np.linalg.norm(xs[r0:r1] - xr) / np.linalg.norm(xr)))
    # plain FP64 per-request throughput on this batch: the sample's mean time
    # per cell-iteration scaled to the batch is not needed -- requests are
    # drawn from the same distribution, so solves/s = 1 / mean(time)
    plain_solves = 1.0 / float(np.mean(plain_t))
    return dict(elapsed=elapsed, out=out, launches=launches, clocks=clocks, t_mesh=t_mesh, N=mb.n_cells,
                choice=choice, trial=trial, other=other, t_other=t_other,
                other_it_max=int(np.max(out_other["iterations"])),
                nnz=A.shape()[2], tile=tile, tile_times=tile_times, errs=errs, plain_solves=plain_solves,
                sample=len(sample), sides=sides, levels=P.levels()[2:], schedule=sweep_schedule(P),
                sched_times=sched_times, order_info=P.order_info, factor_setup_s=round(t_factor_setup, 2))


BATCH_OUTER_TOL = 1e-10


def serve_arm(args, rank, world, local_rank):
    """Served configuration: Poisson arrivals mixing 2D diffusion and 3D
    convection-diffusion requests (sizes lognormal, 1st/99th percentiles
    10k / 2M cells), admission by device memory, continuous batching."""
    import torch
    torch.cuda.set_device(local_rank)
    from fvb200.build import build
    build()
    import fvb200 as fv
    from fvb200._lib import lib
    from fvb200.serve import MeshCache, Server, request_fields, request_stream
    from concurrent.futures import ThreadPoolExecutor
    reqs = request_stream(rate=args.serve_rate, duration=args.serve_duration, seed=2024 + rank)
    # sizes quantised so the host builds a bounded set of meshes up front
    for r in reqs:
        if r.kind == "2d":
            r.side = max(16, int(round(r.side / 16.0)) * 16)
            r.cells = 2 * r.side ** 2
        else:
            r.side = max(4, int(round(r.side / 4.0)) * 4)
            r.cells = 6 * r.side ** 3
    import functools

    from fvb200.serve import solve_wave
    from fvb200.serve import WaveRun
    ordering = None if args.ordering == "natural" else args.ordering
    # a refill holds the old and the rebuilt wave on the device for a moment: half-size waves
    wave_cells = args.serve_wave_cells or (24_000_000 if args.serve_refill else 48_000_000)
    srv = Server(fv, workers=args.serve_workers, max_wave_cells=wave_cells,
                 max_wave_requests=args.serve_wave_requests, wave_order=args.serve_wave_order,
                 solve_fn=functools.partial(solve_wave, precision=args.serve_precision, ordering=ordering),
                 refill=bool(args.serve_refill),
                 run_fn=functools.partial(WaveRun, precision=args.serve_precision, ordering=ordering))
    t0 = time.time()
    keys = sorted({(r.kind, r.side) for r in reqs})
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(lambda k: srv.cache.get(*k), keys))
    t_mesh = time.time() - t0
    clk = Clocks(local_rank)
    clk.start()
    L0 = lib().fv_launch_count()
    cap = args.serve_time_limit if args.serve_time_limit > 0 else args.serve_duration + 15.0
    stats = srv.run(reqs, time_limit=cap, drain=False)
    launches = lib().fv_launch_count() - L0
    clocks = clk.stop()
    # the same server below its capacity: latency of a request that does not queue behind thousands
    sustain = None
    if args.serve_sustain_rate > 0:
        sreqs = request_stream(rate=args.serve_sustain_rate, duration=args.serve_sustain_duration,
                               seed=4048 + rank)
        for r in sreqs:
            if r.kind == "2d":
                r.side = max(16, int(round(r.side / 16.0)) * 16)
                r.cells = 2 * r.side ** 2
            else:
                r.side = max(4, int(round(r.side / 4.0)) * 4)
                r.cells = 6 * r.side ** 3
        srv2 = Server(fv, workers=args.serve_workers, max_wave_cells=wave_cells,
                      max_wave_requests=args.serve_wave_requests, wave_order=args.serve_wave_order,
                      solve_fn=functools.partial(solve_wave, precision=args.serve_precision, ordering=ordering),
                      refill=bool(args.serve_refill),
                      run_fn=functools.partial(WaveRun, precision=args.serve_precision, ordering=ordering))
        srv2.cache = srv.cache
        clk2 = Clocks(local_rank, "_sustain")
        clk2.start()
        s2 = srv2.run(sreqs, time_limit=args.serve_sustain_duration + 60.0, warm=False, drain=True)
        sustain = {"arrival_rate_per_s": args.serve_sustain_rate, "arrival_window_s": args.serve_sustain_duration,
                   "requests": len(sreqs), "completed": s2["completed"], "failed": s2["failed"],
                   "backlog": s2["backlog"], "solves_per_s": round(s2["solves_per_s"], 3),
                   "p50_ms": round(s2["p50_ms"], 1) if s2["p50_ms"] is not None else None,
                   "p99_ms": round(s2["p99_ms"], 1) if s2["p99_ms"] is not None else None,
                   "waves": s2["waves"], "refills": s2["refills"], "clocks": clk2.stop()}
    # plain FP64 per-request path on a sample of the same requests, stratified by
    # size: per kind, the requests at evenly spaced quantiles of the cell count
    sample = []
    for kind in ("2d", "3d"):
        rk = sorted((r for r in reqs if r.kind == kind), key=lambda r: r.cells)
        m = min(max(1, args.plain_sample // 2), len(rk))
        sample += [rk[int((j + 0.5) * len(rk) / m)] for j in range(m)] if rk else []
    plain = []
    for r in sample:
        m = srv.cache.get(r.kind, r.side)
        kf, fl, sc = request_fields(m, r)
        nb = m.n_boundary_faces
        zb = (np.zeros(nb), np.zeros(nb))
        torch.cuda.synchronize()
        s0 = time.perf_counter()
        if r.kind == "2d":
            Ak, bk = fv.assemble(-fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc), zb, m)
            Pk = fv.IncompleteCholesky.from_matrix(Ak, 0)
            xk = fv.DistributedVector.from_size(m.n_cells)
            fv.conjugate_gradient(xk, Ak, bk, Pk, None, fv.LinearSolverOptions(RTOL, RTOL, 20000))
        else:
            eqk = fv.convection(fv.Upwind(fl), fl) - fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
            Ak, bk = fv.assemble(eqk, zb, m)
            Pk = fv.IncompleteLowerUpper.from_matrix(Ak, 0)
            xk = fv.DistributedVector.from_size(m.n_cells)
            fv.bi_conjugate_gradient_stab(xk, Ak, bk, Pk, None, fv.LinearSolverOptions(RTOL, RTOL, 20000))
        torch.cuda.synchronize()
        plain.append(time.perf_counter() - s0)
    plain_rate = 1.0 / float(np.mean(plain))
    line = {
        "metric": METRIC, "value": round(stats["solves_per_s"], 3), "unit": "solves/s", "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": round(stats["wall_s"] * 1e3, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-inner/f64-refinement" if args.serve_precision == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "arrival_rate_per_s": args.serve_rate,
                   "precision": args.serve_precision, "ordering": args.ordering,
                   "arrival_window_s": args.serve_duration, "requests": len(reqs),
                   "mix": "50% 2D diffusion (CG+IC0) / 50% 3D convection-diffusion (BiCGStab+ILU0)",
                   "sizes": "lognormal, 1st/99th pct 10k/2M cells, clipped; 2D sides x16, 3D sides x4",
                   "workers": args.serve_workers, "max_wave_cells": wave_cells,
                   "max_wave_requests": args.serve_wave_requests,
                   "batching": ("slot refill: finished requests leave at once, waiting ones join the running "
                                "wave, whose running requests carry their state over" if args.serve_refill
                                else f"whole waves ({args.serve_wave_order} order)"),
                   "outer_tolerance": 1e-10},
        "p50_ms": round(stats["p50_ms"], 1) if stats["p50_ms"] is not None else None,
        "p99_ms": round(stats["p99_ms"], 1) if stats["p99_ms"] is not None else None,
        "completed": stats["completed"], "offered": stats["offered"], "backlog_at_cap": stats["backlog"],
        "arrived_by_cap": stats["arrived_by_cap"], "wall_cap_s": cap, "failed": stats["failed"],
        "waves": stats["waves"], "refills": stats["refills"], "cells_per_s": round(stats["cells_per_s"], 1),
        "max_final_residual": stats["max_residual"],
        "plain_fp64_solves_per_s": round(plain_rate, 3),
        "plain_sample": f"{len(sample)} requests at evenly spaced size quantiles per kind, one at a time, rtol 1e-8",
        "speedup_vs_plain_fp64": round(stats["solves_per_s"] / plain_rate, 2) if plain_rate > 0 else None,
        "below_capacity": sustain,
        "gpu_launches": int(launches), "clocks": clocks, "mesh_build_s": round(t_mesh, 1),
    }
    return line


def main_batch(args, rank, world, local_rank):
    res = batch_arm(args, rank, world, local_rank)
    K = args.steps
    solves = K * args.batch_count * world
    value = solves / res["elapsed"]
    out = res["out"]
    its = out["iterations"]
    cells = np.diff(np.asarray([0] + list(np.cumsum([2 * int(s) ** 2 for s in res["sides"]]))))
    mixed = res["choice"] == "mixed"
    prec_name = {"mixed": "FP32 CG + FP32 IC(0) inside FP64 refinement", "fp64": "FP64 CG + IC(0)"}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "solves/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(res["elapsed"] / K * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-inner/f64-refinement" if mixed else "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "problems": args.batch_count, "cells_total": res["N"],
                   "nnz": res["nnz"], "sides": "log-uniform [32,512]", "solver": "batched CG+IC(0)",
                   "precision": prec_name[res["choice"]], "precision_choice": args.batch_precision,
                   "target": f"|b-Ax|/|b| <= {BATCH_OUTER_TOL} per problem",
                   "tile_rows": res["tile"], "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
        "precision_trial_s": {k: round(v, 3) for k, v in res["trial"].items()},
        f"{res['other']}_batched_solves_per_s": round(args.batch_count / res["t_other"], 3),
        f"{res['other']}_batched_iterations_max": res["other_it_max"],
        "dof_iters_per_s": round(float(np.sum(cells * its)) * K * world / res["elapsed"], 1),
        "max_rel_err_vs_fp64": max(res["errs"]) if res["errs"] else None, "err_sample": res["sample"],
        "max_final_residual": float(np.max(out["final_residual"])),
        "plain_fp64_solves_per_s": round(res["plain_solves"], 4),
        "speedup_vs_plain_fp64": round(value / res["plain_solves"] / world, 2),
        "outer_steps_max": int(np.max(out["outer_steps"])), "iterations_max": int(np.max(its)),
        "fp64_fallback_problems": int(np.sum(out["fp64_fallback"])),
        "launched_iterations": int(out["launched_iterations"]), "levels_fwd_bwd": list(res["levels"]),
        "sweep_schedule": res["schedule"], "ordering": args.ordering, "ordering_info": res["order_info"],
        "factor_setup_s": res["factor_setup_s"],
        "autotune_tile_s": {str(k): round(v, 4) for k, v in res["tile_times"].items()},
        "autotune_sweep_schedule_ms": {str(k): round(v, 3) for k, v in res["sched_times"].items()},
        "gpu_launches": int(res["launches"]), "clocks": res["clocks"], "mesh_build_s": round(res["t_mesh"], 2),
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="cube128_convdiff", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reorder", default="system", choices=["system", "precond"],
                    help="box order as the permuted system Q A Q^T (default) or as the reordered factorisation "
                         "applied in A's numbering")
    ap.add_argument("--mixed-delta", type=float, default=1e-2,
                    help="mixed precision: FP32 residual reduction that triggers an FP64 residual replacement")
    ap.add_argument("--ordering", default="boxes", choices=["boxes", "natural"],
                    help="factorisation order of the single-problem workloads: the reordered perf mode (boxes) "
                         "or the reference's natural order")
    ap.add_argument("--no-configs", action="store_true", help="only the headline workload (no sub-configs)")
    ap.add_argument("--batch-count", type=int, default=1024)
    ap.add_argument("--plain-sample", type=int, default=8)
    ap.add_argument("--batch-precision", default="auto", choices=["auto", "mixed", "fp64"])
    ap.add_argument("--serve-precision", default="fp64", choices=["mixed", "fp64"])
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-duration", type=float, default=60.0)
    ap.add_argument("--serve-workers", type=int, default=2)
    ap.add_argument("--serve-wave-cells", type=int, default=0,
                    help="cells per wave (0: 24M with slot refill, 48M with whole waves)")
    ap.add_argument("--serve-wave-requests", type=int, default=512)
    ap.add_argument("--serve-wave-order", default="size", choices=["size", "fifo"])
    ap.add_argument("--serve-sustain-rate", type=float, default=20.0,
                    help="a second served run at this arrival rate (below capacity) for unqueued latency; 0: skip")
    ap.add_argument("--serve-sustain-duration", type=float, default=30.0)
    ap.add_argument("--serve-refill", type=int, default=1, choices=[0, 1],
                    help="1: slot refill (running waves take newly admitted requests); 0: whole waves")
    ap.add_argument("--serve-time-limit", type=float, default=0.0,
                    help="wall cap of the served run (0: arrival window + 15 s); at the cap admission stops, "
                         "running waves finish, the rest is reported as backlog")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    import torch
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if WORKLOADS[args.workload]["kind"] in ("batch", "serve", "transient"):
        kind = WORKLOADS[args.workload]["kind"]
        line = {"batch": main_batch, "serve": serve_arm, "transient": transient_arm}[kind](args, rank, world,
                                                                                         local_rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    wl = WORKLOADS[args.workload]
    ordering = None if args.ordering == "natural" else args.ordering
    precision = wl.get("precision", "fp64")
    ctx = setup_single(args, wl, rank, world, local_rank)
    ctx["mixed_delta"] = args.mixed_delta
    res = measure_single(ctx, ordering, args.steps, args.warmup, precision=precision, e2e=True, kernels=True,
                         reorder=args.reorder)
    K = args.steps
    solves = K * world
    value = solves / res["elapsed"]
    it_mean = float(np.mean(res["iters"]))
    N = res["N"]
    lat = sorted(res["lat_ms"])
    cfg = config_of(args, wl, N, res["nnz"])
    cfg["ordering"] = args.ordering
    if ordering is not None:
        cfg["reorder"] = {"system": "permuted system Q A Q^T solved in its own numbering",
                          "precond": "reordered factorisation applied in A's numbering"}[args.reorder]
    line = {
        "metric": METRIC, "value": round(value, 6), "unit": "solves/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(res["elapsed"] / K * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "dof_iters_per_s": round(N * it_mean * solves / res["elapsed"], 1),
        "iterations": res["iters"], "step_phase_ms": res["phase_ms"],
        "p50_ms": round(float(np.percentile(lat, 50)), 3),
        "p99_ms": round(float(np.percentile(lat, 99)), 3), "true_rel_residual": res["relres"],
        "rel_err_vs_tight_fp64": res["err_tight"],
        "roofline": res["roofline"], "kernels": res["kernels"], "time_share": res["share"],
        "factor_ms": res["t_factor_ms"], "levels_fwd_bwd": list(res["levels"]), "ordering_info": res["order_info"],
        "factor_setup_s": res["factor_setup_s"], "sweep_schedule": res["schedule"],
        "e2e": {"value": round(solves / res["e2e_elapsed"], 6), "unit": "solves/s",
                "h2d_bytes_per_step": res["h2d"], "d2h_bytes_per_step": res["d2h"],
                "step_ms": res["e2e_lat_ms"], "clocks": res["e2e_clocks"]},
        "gpu_launches": int(res["launches"]),
        "clocks": res["clocks"],
        "mesh_build_s": round(ctx["t_mesh"], 2),
        "mesh_build": {"where": "device (fv_mesh_build_*)", "with_read_back_and_fields_s": round(ctx["t_mesh"], 2),
                       "elements_then_device_build_s": round(ctx["t_mesh_dev"], 3)},
    }
    if res.get("mixed_info"):
        line["dtype"] = "f32-inner/f64-refinement"
        line["config"]["precision"] = "FP32 Krylov + FP32 factors, FP64 reliable updates to |b-Ax|/|b| <= 1e-10"
        line["mixed"] = res["mixed_info"]
    x_gpu = {args.ordering: res["x"]}
    if world == 1 and not args.no_configs:
        # the same problem in the other ordering, and the FP32/FP64 form (config "mixed")
        other = "natural" if ordering is not None else "boxes"
        ro = measure_single(ctx, None if other == "natural" else other, max(3, K // 4), 2, e2e=False, kernels=True)
        x_gpu[other] = ro["x"]
        head_label = f"{wl['solver']}, {args.ordering} order" + (
            " as the permuted system" if ordering is not None and args.reorder == "system" else "") + ", FP64"
        line["orderings"] = {args.ordering: single_summary(res, world, head_label),
                             other: single_summary(ro, world, f"{wl['solver']}, {other} order, FP64")}
        del ro
        if ordering is not None:  # the box order's other form
            alt = "precond" if args.reorder == "system" else "system"
            ra = measure_single(ctx, ordering, max(3, K // 4), 2, e2e=False, kernels=True, reorder=alt)
            line["orderings"][f"{args.ordering}_{alt}"] = single_summary(
                ra, world, f"{wl['solver']}, {args.ordering} order as the "
                + ("reordered factorisation applied in A's numbering" if alt == "precond" else "permuted system")
                + ", FP64")
            del ra
        if precision == "fp64":
            rm = measure_single(ctx, ordering, max(3, K // 4), 2, precision="mixed", e2e=False, kernels=False)
            line["configs"] = {f"{args.workload}_mixed": single_summary(
                rm, world, "FP32 Krylov + FP32 factors inside FP64 reliable updates to |b-Ax|/|b| <= 1e-10, "
                f"{args.ordering} order")}
            # FP64 to the same target as the mixed form: the comparison at equal accuracy
            rf = measure_single(ctx, ordering, max(3, K // 4), 2, e2e=False, kernels=False, tol=1e-10)
            sm = line["configs"][f"{args.workload}_mixed"]
            sf = single_summary(rf, world, f"FP64 {wl['solver']} to rtol = atol = 1e-10, {args.ordering} order "
                                "(the mixed form's target)")
            sm["fp64_same_target"] = {k: sf[k] for k in ("label", "value", "ms_per_step", "iterations",
                                                         "true_rel_residual", "rel_err_vs_tight_fp64", "clocks")}
            sm["speedup_vs_fp64_same_target"] = round(sm["value"] / sf["value"], 3)
            del rf
            del rm
        if args.workload == "cube128_convdiff":
            line.setdefault("configs", {}).update(square_configs(args))
            from types import SimpleNamespace
            sub = SimpleNamespace(**vars(args))
            sub.workload = "batch1024_diffusion"
            sub.steps, sub.warmup, sub.plain_sample = 1, 2, 4
            line["configs"]["batch1024_diffusion"] = main_batch(sub, rank, world, local_rank)
            sub = SimpleNamespace(**vars(args))
            sub.workload = "serve_mixed"
            sub.plain_sample = 4
            line["configs"]["serve_mixed"] = serve_arm(sub, rank, world, local_rank)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cs = cpu_full_solve(ctx["prob"], wl)
            cpu = {"value": round(1.0 / cs["t_solve"], 6), "unit": "solves/s", "cores": 1, "kind": "port",
                   "sample": cs["sample"], "iterations": cs["iters"],
                   "phase_s": {"assemble": round(cs["t_asm"], 2), "factor": round(cs["t_fac"], 2),
                               "krylov": round(cs["t_krylov"], 2)}}
            # the oracle's natural-order solution against the GPU's (the same algorithm)
            if "natural" in x_gpu:
                xo = cs["x"]
                cpu["rel_err_gpu_natural_vs_oracle"] = float(np.linalg.norm(x_gpu["natural"] - xo) / np.linalg.norm(xo))
        except Exception as e:  # pragma: no cover - reported, not fatal
            cpu = {"value": None, "unit": "solves/s", "cores": 1, "kind": "port", "sample": f"failed: {e}"}
    line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def square_configs(args):
    """Config "square256_diffusion" (the CPU-runnable 2D case) on the GPU in
    both orderings, with the GPU solutions checked against the oracle's."""
    wl = WORKLOADS["square256_diffusion"]
    ctx = setup_single(args, wl, 0, 1, 0)
    out = {}
    import oracle
    c = ctx["prob"]["coef"]
    p = ctx["prob"]
    ptr, cols, vals, rhs = oracle.assemble(p["mesh"], c[0], c[1], c[2], kappa=p["kappa"], flux=p["flux"],
                                           source=p["source"], bndi=p["bndi"], bnde=p["bnde"])
    for name, ordering in (("natural", None), ("boxes", "boxes")):
        r = measure_single(ctx, ordering, args.steps, args.warmup, e2e=False, kernels=True, reorder=args.reorder)
        sm = single_summary(r, 1, f"cg+ic0, {name} order, FP64")
        if ordering is None:
            pc = oracle.Precond("ic", ptr, cols, vals)
        else:
            perm = ctx["fv"].IncompleteCholesky.from_matrix(ctx["A"], 0, ordering="boxes").perm
            pc = oracle.Precond.reordered("ic", ptr, cols, vals, perm)
        xo, io = oracle.cg(ptr, cols, vals, pc, rhs, rtol=RTOL, atol=RTOL, maxit=20000)
        sm["oracle_iterations"] = int(io["iterations"])
        sm["rel_err_vs_oracle_same_ordering"] = float(np.linalg.norm(r["x"] - xo) / np.linalg.norm(xo))
        out[f"square256_diffusion_{name}"] = sm
    return out


if __name__ == "__main__":
    main()
