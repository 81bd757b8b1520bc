#!/usr/bin/env python
"""Benchmark of the closed-form matting hot path on B200.

Workload (one "step"): a seeded synthetic 1920x1080 image with ~10%
scribbles (eps = 1e-5, gamma = 100) goes through the hot path: FP64 Levin
Laplacian assembly into the FP16 symmetric band store, then the fused
persistent mixed-precision CG to relative residual 1e-6 (FP64 true-residual
replacement every 50 iterations, max 5000).  The metric is Mpix * CG
iterations per second over the whole job; ms_per_step is the time to
relative residual 1e-6.

  value   device-resident inputs, CUDA events on the launching stream, L2
          flushed (256 MB write) between timed steps.
  e2e     the same step through the C ABI from pinned HOST buffers: H2D of the
          RGB8 image, scribbles and initial alpha, assembly, solve, D2H alpha.
  plain   (N=1, rank 0) the plain FP32 method on the same image: 25-band FP32
          reference-layout store, fused CG, same stopping rule.
  pcg, mg (N=1, rank 0) the same step with Jacobi-preconditioned CG and with
          the multigrid-preconditioned CG.
  solvers (N=1, rank 0) CG, steepest descent and Jacobi to 1e-6, mixed and
          plain, and CG / Jacobi PCG / multigrid PCG to 1e-10 (alpha within
          1e-4 of FP64).
  slab    (N=1, rank 0) the row-slab split of the same image, its slabs held
          by one process on this GPU (gpumatting_b200/slab.py).

Multi-GPU: one process per GPU (torchrun); every rank solves its own image
(seed = rank), no data-path collective; time is the max over ranks.

--impl reference times the reference's own CPU path (hostLevinLaplacian +
gaussSeidel_host from oracle/_ref, compiled from the reference sources) on the
same image with all host threads, one independent image per thread.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpix·CG-iter/s and time to rel-residual 1e-6 at 1080p, mixed vs FP32, 1 B200"
UNIT = "Mpix·CG-iter/s"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "source": "fallback"}

# Algorithmic bytes per pixel: Krylov sweep of the FP16
# symmetric store = 12 planes x 2 B + gamma 4 B + read r,q,p 12 B + write
# r,p,q 12 B + solution increment read/write 8 B.
KRYLOV_BYTES = {"fp16": 60, "bf16": 60, "fp32": 84, "ref25": 132}
REPLACE_BYTES = {"sym_mixed": 92, "ref25": 124}
IMPORT_BYTES = {"sym_mixed": 36, "ref25": 20}


def load_peaks(path: str | None = None):
    """The HBM roofline denominator: `hbm_gbs` of the per-pod measured-peaks
    file when it holds a positive number there, else the fallback (the
    reason kept in `source`)."""
    p = path or os.path.join(ROOT, "MEASURED_PEAKS.json")
    if not os.path.exists(p):
        return dict(FALLBACK_PEAKS)
    try:
        with open(p) as f:
            d = json.load(f)
        v = float(d["hbm_gbs"])
    except (OSError, ValueError, TypeError, KeyError) as e:
        return dict(FALLBACK_PEAKS, source=f"fallback ({os.path.basename(p)} unreadable: {type(e).__name__})")
    if not v > 0.0:
        return dict(FALLBACK_PEAKS, source=f"fallback ({os.path.basename(p)} hbm_gbs = {v})")
    d["hbm_gbs"] = v
    d["source"] = "measured"
    return d


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", self.gpu_id], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def allreduce_max(x: float, world: int) -> float:
    from gpumatting_b200.shard import max_over_ranks

    return x if world == 1 else max_over_ranks(x)


def allreduce_sum(x: float, world: int) -> float:
    from gpumatting_b200.shard import sum_over_ranks

    return x if world == 1 else sum_over_ranks(x)


def barrier(world: int):
    import torch

    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own CPU path
# ---------------------------------------------------------------------------
def reference_cpu_path(prob, sweeps: int, threads: int, steps: int = 1):
    """hostLevinLaplacian + `sweeps` gaussSeidel_host sweeps per image, one
    image per thread; returns (seconds per step list, kind, assembly_s)."""
    import numpy as np

    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    W, H = prob.W, prob.H
    N = W * H
    im4 = prob.image_float4()
    offs = O.levin_offsets(W)

    def one(out: list):
        t0 = time.perf_counter()
        if kind == "reference":
            a, b = O.ref_levin(im4, prob.scribbles, prob.eps)
        else:
            a, b = O.levin_ref32(im4, prob.scribbles, prob.eps, 1.0)
        t1 = time.perf_counter()
        x = np.full(N, 0.5, np.float32)
        O.gs_host(a, offs, b, x, sweeps, use_ref=(kind == "reference"))
        t2 = time.perf_counter()
        out.append((t1 - t0, t2 - t1))

    times, asm = [], []
    for _ in range(steps):
        outs: list = []
        ths = [threading.Thread(target=one, args=(outs,)) for _ in range(threads)]
        t0 = time.perf_counter()
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        times.append(time.perf_counter() - t0)
        asm.append(statistics.mean(o[0] for o in outs))
    return times, kind, statistics.mean(asm)


def calibrate_sweeps(prob, target_s: float) -> int:
    """Gauss-Seidel sweeps that take about target_s on one core."""
    import numpy as np

    from oracle import oracle as O

    W, H = prob.W, prob.H
    a, b = O.levin_ref32(prob.image_float4(), prob.scribbles, prob.eps, 1.0)
    x = np.full(W * H, 0.5, np.float32)
    t0 = time.perf_counter()
    O.gs_host(a, O.levin_offsets(W), b, x, 2)
    per = (time.perf_counter() - t0) / 2
    return max(1, int(target_s / max(per, 1e-6)))


def oracle_cg_rate(prob, target_s: float) -> dict:
    """The project's own FP64 CPU CG (the oracle's orc_cg64, OpenMP over the
    host cores) on the headline problem, over a bounded number of iterations.
    The reference has no CPU CG (its CPU solvers are Gauss-Seidel and
    Jacobi); this figure is labelled as this project's code, not the
    reference's."""
    import numpy as np

    from oracle import oracle as O

    W, H = prob.W, prob.H
    w = O.levin_sym64(prob.image.astype(np.float64) / 255.0, prob.eps)
    g = prob.gamma.ravel().astype(np.float64)
    b = (prob.gamma * prob.s).ravel().astype(np.float64)
    op = O.Operator(W=W, H=H, w=w, gamma=g)
    x0 = np.full(W * H, 0.5)
    t0 = time.perf_counter()
    op.cg(b, x0, rtol=0.0, maxit=5)
    per = (time.perf_counter() - t0) / 5
    iters = max(5, int(target_s / max(per, 1e-6)))
    t0 = time.perf_counter()
    _, done, _ = op.cg(b, x0, rtol=0.0, maxit=iters)
    dt = time.perf_counter() - t0
    threads = int(O.lib().orc_num_threads())
    return {"value": W * H * done / 1e6 / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{W}x{H}: {done} FP64 CG iterations of the oracle (symmetric FP64 operator, "
                      f"{threads} OpenMP threads); the project's own CPU CG, not the reference's"}


def cpu_threads_for(W: int, H: int) -> int:
    n = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_AVPHYS_PAGES")
    except (ValueError, OSError):
        avail = 16 << 30
    per = 40 * W * H * 4  # bands, rhs, x, image per thread
    return max(1, min(n, int(0.5 * avail // per)))


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from gpumatting_b200.synth import make_problem

    prob = make_problem(args.W, args.H, 0)
    threads = cpu_threads_for(args.W, args.H)
    sweeps = calibrate_sweeps(prob, args.ref_seconds)
    reference_cpu_path(prob, sweeps, threads, steps=args.warmup)
    times, kind, asm = reference_cpu_path(prob, sweeps, threads, steps=args.steps)
    N = args.W * args.H
    total = sum(times)
    value = threads * N * sweeps * args.steps / 1e6 / total
    sample = (f"{args.W}x{args.H} image per thread: hostLevinLaplacian ({asm:.2f} s) + {sweeps} gaussSeidel_host "
              f"sweeps, {threads} independent images on {threads} threads")
    conv = reference_convergence(prob, sweeps)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": reference_config_dict(args, sweeps, threads),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "time_to_rtol": conv,
            "note": "units differ from the GPU arm: iterations here are Gauss-Seidel sweeps (Solve.cpp:3-33), "
                    "the reference has no CPU CG; time_to_rtol gives the residual the sweeps reach"}
    print(json.dumps(line), flush=True)


def reference_convergence(prob, sweeps: int) -> dict:
    """How far the reference's CPU path gets towards rel-residual 1e-6: the
    true FP64 relative residual ||b - A x|| / ||b|| of its own 25-band system
    after `sweeps` gaussSeidel_host sweeps from alpha = 0.5 (one image, one
    core), with the time those sweeps took.  Gauss-Seidel on this
    ill-conditioned system does not reach 1e-6 in any affordable sample."""
    import numpy as np

    from oracle import oracle as O

    W, H = prob.W, prob.H
    im4 = prob.image_float4()
    use_ref = O.ref_available()
    a, b = O.ref_levin(im4, prob.scribbles, prob.eps) if use_ref else O.levin_ref32(im4, prob.scribbles, prob.eps, 1.0)
    offs = O.levin_offsets(W)
    op = O.Operator(W=W, H=H, bands=a.astype(np.float64), offs=offs)
    b64 = b.astype(np.float64)
    x = np.full(W * H, 0.5, np.float32)
    rel0 = float(np.linalg.norm(b64 - op.apply(x.astype(np.float64))) / np.linalg.norm(b64))
    t0 = time.perf_counter()
    x = O.gs_host(a, offs, b, x, sweeps, use_ref=use_ref)
    dt = time.perf_counter() - t0
    rel = float(np.linalg.norm(b64 - op.apply(x.astype(np.float64))) / np.linalg.norm(b64))
    return {"target_rel_residual": 1e-6, "reached": rel <= 1e-6, "sweeps": sweeps, "seconds": dt,
            "rel_residual_start": rel0, "rel_residual_reached": rel, "cores": 1}


def config_dict(args) -> dict:
    return {"workload": f"{args.W}x{args.H} synthetic matting solve (seeded), eps=1e-5, gamma=100, ~10% scribbles; "
                        f"{args.precision.upper()} symmetric band store, fused mixed CG to rel-residual 1e-6 "
                        f"(FP64 replacement every 50, max 5000)",
            "W": args.W, "H": args.H, "precision": args.precision, "rtol": 1e-6,
            "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{args.gpus}"}


def reference_config_dict(args, sweeps: int, threads: int) -> dict:
    """What the reference arm runs: the reference's CPU solve path on the same
    synthetic image, a fixed number of Gauss-Seidel sweeps (it has no CPU CG
    and no stopping rule), one independent image per host thread."""
    return {"workload": f"{args.W}x{args.H} synthetic matting solve (seeded), eps=1e-5, gamma=1 (Matting.cu:48), "
                        f"~10% scribbles; reference CPU path: hostLevinLaplacian into 25 FP32 bands, then "
                        f"{sweeps} gaussSeidel_host sweeps (Solve.cpp:3-33), fixed count",
            "W": args.W, "H": args.H, "precision": "fp32 (25 bands)", "sweeps": sweeps, "threads": threads,
            "parallelism": f"{threads} independent images on {threads} host threads"}


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import numpy as np
    import torch

    from gpumatting_b200 import _lib as L
    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    world, rank, local = dist_setup()
    W, H = args.W, args.H
    N = W * H
    prob = make_problem(W, H, rank)
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    img_h = torch.from_numpy(prob.image).pin_memory()
    scr_h = torch.from_numpy(prob.scribbles).pin_memory()
    a0_h = torch.full((H, W), 0.5, dtype=torch.float32).pin_memory()
    out_h = torch.empty((H, W), dtype=torch.float32).pin_memory()
    img_d = img_h.to(dev)
    scr_d = scr_h.to(dev)
    a0_d = a0_h.to(dev)
    alpha = torch.empty((H, W), dtype=torch.float32, device=dev)
    store = api.LevinStore(W, H, args.precision)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)  # 256 MB > L2
    params = dict(rtol=1e-6, max_iters=5000, replace_every=args.replace_every, ctas_per_sm=args.ctas_per_sm,
                  strip_width=args.strip_width)
    if args.fixed_iters:
        params.update(rtol=0.0, max_iters=args.fixed_iters)

    def step_device():
        store.assemble(img_d, scr_d, eps=prob.eps, gamma_value=100.0)
        alpha.copy_(a0_d, non_blocking=True)
        return store.solve(alpha, args.solver, **params)

    def step_e2e():
        img_d.copy_(img_h, non_blocking=True)
        scr_d.copy_(scr_h, non_blocking=True)
        alpha.copy_(a0_h, non_blocking=True)
        store.assemble(img_d, scr_d, eps=prob.eps, gamma_value=100.0)
        r = store.solve(alpha, args.solver, **params)
        out_h.copy_(alpha, non_blocking=True)
        return r

    def timed(fn, k):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        res = []
        for i in range(k):
            flush.fill_(float(i))
            ev[i][0].record(stream)
            res.append(fn())
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev], res

    for _ in range(args.warmup):
        r = step_device()
        assert r.status == 0, r
    gpu_id = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(gpu_id)
    barrier(world)
    clocks.start()
    ms, res = timed(step_device, args.steps)
    barrier(world)
    clk = clocks.stop()
    for r in res:
        assert r.status == 0 and (args.fixed_iters or r.rel_residual <= 1e-6), r
    iters = sum(r.iters for r in res)
    reps = sum(r.replacements for r in res)
    kern_ms = sum(r.kernel_ms for r in res)
    t_local = sum(ms) / 1000.0
    t_max = allreduce_max(t_local, world)
    work = allreduce_sum(N * iters, world)
    value = work / 1e6 / t_max

    # e2e through the C ABI with host buffers
    if args.no_e2e:
        ms_e, res_e = ms, res
    else:
        for _ in range(max(1, args.warmup // 2)):
            step_e2e()
        barrier(world)
        ms_e, res_e = timed(step_e2e, args.steps)
        barrier(world)
    iters_e = sum(r.iters for r in res_e)
    te_max = allreduce_max(sum(ms_e) / 1000.0, world)
    e2e_value = allreduce_sum(N * iters_e, world) / 1e6 / te_max

    peaks = load_peaks()
    kb = KRYLOV_BYTES[args.precision]
    alg_bytes = N * (iters * kb + reps * REPLACE_BYTES["sym_mixed"] + args.steps * IMPORT_BYTES["sym_mixed"])
    achieved = alg_bytes / (kern_ms / 1000.0) / 1e9
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "solver_traffic.json")
    if os.path.exists(tr_path):
        tr = json.load(open(tr_path))
        if tr.get("precision") == args.precision and tr.get("W") == W and tr.get("H") == H:
            traffic = tr["dram_bytes_per_px_iter"] * N * iters / args.steps
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.precision + " bands / f32 vectors / f64 residual",
            "data": "synthetic", "config": config_dict(args),
            "time_to_rtol_ms": 1000 * t_max / args.steps,
            "iters_per_solve": iters / args.steps, "replacements_per_solve": reps / args.steps,
            "solver_kernel_ms": kern_ms / args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                         "peak_source": peaks.get("source"),
                         "alg_bytes_per_launch": alg_bytes / args.steps,
                         "kernel": "gm::solver_kernel (fused persistent CG)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": N * (3 + 1 + 4),
                    "d2h_bytes_per_step": N * 4, "ms_per_step": 1000 * te_max / args.steps},
            "gpu_launches": 3 * args.steps,  # per step: levin_sym_kernel, levin_diag_kernel, solver_kernel
            "clocks": clk}
    def timed_solve(solver, k, **extra):
        """Solve-only times (assembly outside the events, L2 flushed before
        each solve), for comparisons with the plain arm, which is timed the
        same way."""
        out_ms, out_res = [], []
        for i in range(k):
            store.assemble(img_d, scr_d, eps=prob.eps, gamma_value=100.0)
            alpha.copy_(a0_d, non_blocking=True)
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = store.solve(alpha, solver, **dict(params, **extra))
            e1.record(stream)
            torch.cuda.synchronize()
            out_ms.append(e0.elapsed_time(e1))
            out_res.append(r)
        assert all(r.status == 0 and (args.fixed_iters or r.rel_residual <= 1e-6) for r in out_res), out_res
        return statistics.mean(out_ms), out_res

    if rank == 0 and world == 1:
        line["solve_only_ms"] = timed_solve(args.solver, args.steps)[0]
    if rank == 0 and world == 1 and not args.no_pcg:
        # the same step with Jacobi-preconditioned mixed CG, to the same true rel-res
        def step_pcg():
            store.assemble(img_d, scr_d, eps=prob.eps, gamma_value=100.0)
            alpha.copy_(a0_d, non_blocking=True)
            return store.solve(alpha, "pcg", **params)

        for _ in range(2):
            step_pcg()
        ms_p, res_p = timed(step_pcg, args.steps)
        assert all(r.status == 0 and (args.fixed_iters or r.rel_residual <= 1e-6) for r in res_p), res_p
        it_p = sum(r.iters for r in res_p)
        line["pcg"] = {"solver": "Jacobi-preconditioned mixed CG (FP16 store, FP64 replacement every 50)",
                       "ms_per_step": sum(ms_p) / args.steps, "iters_per_solve": it_p / args.steps,
                       "replacements_per_solve": sum(r.replacements for r in res_p) / args.steps,
                       "rel_residual_max": max(r.rel_residual for r in res_p),
                       "mpix_iter_s": N * it_p / 1e6 / (sum(ms_p) / 1000),
                       "solver_kernel_ms": sum(r.kernel_ms for r in res_p) / args.steps,
                       "solve_only_ms": timed_solve("pcg", args.steps)[0]}
    if rank == 0 and world == 1 and not args.no_mg:
        # the same step with the multigrid-preconditioned CG, to the same true rel-res
        def step_mg():
            store.assemble(img_d, scr_d, eps=prob.eps, gamma_value=100.0)
            alpha.copy_(a0_d, non_blocking=True)
            return store.solve(alpha, "mg", **params)

        for _ in range(2):
            step_mg()
        ms_m, res_m = timed(step_mg, args.steps)
        assert all(r.status == 0 and (args.fixed_iters or r.rel_residual <= 1e-6) for r in res_m), res_m
        it_m = sum(r.iters for r in res_m)
        line["mg"] = {"solver": "multigrid-preconditioned CG (2x2 aggregation V-cycle on the FP16 planes, FP32 "
                                "outer operator, FP64 solution and replacement every 50), one graph launch per solve",
                      "ms_per_step": sum(ms_m) / args.steps, "iters_per_solve": it_m / args.steps,
                      "levels": res_m[0].grid,
                      "replacements_per_solve": sum(r.replacements for r in res_m) / args.steps,
                      "rel_residual_max": max(r.rel_residual for r in res_m),
                      "solve_ms": sum(r.kernel_ms for r in res_m) / args.steps,
                      "speedup_vs_cg": (1000 * t_max / args.steps) / (sum(ms_m) / args.steps),
                      "solve_only_ms": timed_solve("mg", args.steps)[0]}
        # end to end through the public API from pinned host buffers, like `e2e`
        def step_mg_e2e():
            img_d.copy_(img_h, non_blocking=True)
            scr_d.copy_(scr_h, non_blocking=True)
            alpha.copy_(a0_h, non_blocking=True)
            store.assemble(img_d, scr_d, eps=prob.eps, gamma_value=100.0)
            r = store.solve(alpha, "mg", **params)
            out_h.copy_(alpha, non_blocking=True)
            return r

        step_mg_e2e()
        ms_me, res_me = timed(step_mg_e2e, args.steps)
        assert all(r.status == 0 and (args.fixed_iters or r.rel_residual <= 1e-6) for r in res_me), res_me
        line["mg"]["e2e_ms"] = sum(ms_me) / args.steps
        # the fastest time to rel-res 1e-6 of this step (the headline value stays the CG's)
        line["time_to_rtol_mg_ms"] = line["mg"]["ms_per_step"]
        # the same multigrid solve with the V-cycle on the FP32 planes (use_low = 0)
        ms32, res32 = timed_solve("mg", args.steps, use_low=0)
        line["mg"]["fp32_planes"] = {"solve_only_ms": ms32, "iters": res32[0].iters,
                                     "rel_residual": res32[0].rel_residual}
        # algorithmic bytes per pixel-iteration of the store's precision
        mg_bpp = MG_BYTES_PER_PX_ITER[args.precision]
        mg_bytes = N * mg_bpp * (it_m / args.steps)
        mg_gbs = mg_bytes / (line["mg"]["solve_ms"] / 1000.0) / 1e9
        line["mg"]["roofline"] = {"bound": "hbm", "achieved": mg_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                  "frac": mg_gbs / peaks["hbm_gbs"], "bytes_per_px_iter": mg_bpp,
                                  "peak_source": peaks.get("source")}
    if rank == 0 and world == 1 and not args.no_plain:
        # speed-ups on equal footing: solve-only time of each arm, from alpha = 0.5
        # to the same true rel-res (the plain arm's 25 bands are assembled once,
        # outside its timing); the *_step_* ratios put the mixed arm's assembly
        # on its side only (conservative)
        def mixed_once(i):
            store.assemble(img_d, scr_d, eps=prob.eps, gamma_value=100.0)
            alpha.copy_(a0_d, non_blocking=True)
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = store.solve(alpha, args.solver, **params)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1), r

        pl = run_plain(args, prob, img_d, scr_d, flush, stream, mixed_once)
        pl["speedup_mixed_vs_plain"] = pl["speedup_median"]
        pl["speedup_mixed_step_vs_plain_solve"] = pl["ms_per_solve"] / line["ms_per_step"]
        # the mixed-vs-plain target numbers, where a reader of the line sees them first
        line["speedup_mixed_vs_plain"] = pl["speedup_median"]
        line["speedup_mixed_vs_plain_range"] = [pl["speedup_per_round_min"], pl["speedup_per_round_max"]]
        line["plain_fp32_ms"] = pl["ms_per_solve"]
        line["mixed_cg_solve_ms"] = pl["mixed_ms_per_solve"]
        if "pcg" in line:
            pl["speedup_mixed_pcg_vs_plain"] = pl["ms_per_solve"] / line["pcg"]["solve_only_ms"]
        if "mg" in line:
            pl["speedup_mixed_mg_vs_plain"] = pl["ms_per_solve"] / line["mg"]["solve_only_ms"]
            pl["speedup_mixed_mg_step_vs_plain_solve"] = pl["ms_per_solve"] / line["mg"]["ms_per_step"]
        line["plain_fp32"] = pl
    if rank == 0 and world == 1 and not args.no_solvers:
        line["solvers"] = supplementary("solvers", lambda: run_solvers(args, prob, img_d, scr_d, store, flush, stream))
    if args.batch_count > 0:
        line["batch"] = run_batch(args, stream, world, rank)
    if rank == 0 and world == 1 and args.large_size > 0:
        line["large"] = supplementary("large", lambda: run_large(args, stream, peaks))
    if rank == 0 and world == 1 and args.spmv_size > 0:
        line["spmv"] = supplementary("spmv", lambda: run_spmv(args, stream, peaks))
    if rank == 0 and world == 1 and args.slabs:
        line["slab"] = supplementary("slab", lambda: run_slab(args, prob, img_d, scr_d, stream))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sweeps = calibrate_sweeps(prob, args.cpu_seconds)
        times, kind, asm = reference_cpu_path(prob, sweeps, 1, steps=1)
        v = N * sweeps / 1e6 / times[0]
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": kind,
                                "sample": f"{W}x{H}: hostLevinLaplacian ({asm:.2f} s) + {sweeps} gaussSeidel_host "
                                          f"sweeps on 1 core (iterations are Gauss-Seidel sweeps)"}
        line["cpu_oracle_cg"] = supplementary("cpu_oracle_cg", lambda: oracle_cg_rate(prob, args.cpu_seconds / 3))
    if rank == 0:
        print(json.dumps(ordered_line(line)), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# Keys printed first: the contract's, then the headline target numbers; the
# supplementary sections follow in the order they ran.
LEAD_KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
             "vs_baseline", "dtype", "data", "config", "time_to_rtol_ms", "speedup_mixed_vs_plain",
             "speedup_mixed_vs_plain_range", "plain_fp32_ms", "mixed_cg_solve_ms", "time_to_rtol_mg_ms", "roofline",
             "e2e", "gpu_launches", "clocks", "cpu_baseline")


def ordered_line(line: dict) -> dict:
    out = {k: line[k] for k in LEAD_KEYS if k in line}
    out.update((k, v) for k, v in line.items() if k not in out)
    return out


# Multigrid PCG on an FP16 store, algorithmic bytes per pixel-iteration:
# SpMV 44 (FP16 planes 24, d, z and p read, p and q written), update 24 (FP32
# solution increment read/write, p, q, r read, r written), level-0
# restriction 33 and prolongation 37 (FP16 planes 24, r, 1/d, the coarse
# side, z written), coarse levels 18 (54 B per coarse cell, a third of a
# pixel).  A BF16 or FP32 store's SpMV reads the FP32 planes: 68.
MG_BYTES_PER_PX_ITER = {"fp16": 44 + 24 + 33 + 37 + 18, "bf16": 68 + 24 + 33 + 37 + 18,
                        "fp32": 68 + 24 + 57 + 61 + 18}  # FP32 planes 48 in restriction / prolongation

# Algorithmic bytes per pixel of one SpMV pass: band planes + diagonal plane
# + x read once + y written once.
SPMV_BYTES = {"fp16": 12 * 2 + 4 + 8, "bf16": 12 * 2 + 4 + 8, "fp32": 12 * 4 + 4 + 8, "true_fp32": 12 * 4 + 4 + 8,
              "ref25": 25 * 4 + 8}


_PROBLEMS = {}


def cached_problem(W: int, H: int, seed: int):
    from gpumatting_b200.synth import make_problem

    key = (W, H, seed)
    if key not in _PROBLEMS:
        _PROBLEMS[key] = make_problem(W, H, seed)
    return _PROBLEMS[key]


def supplementary(name: str, fn) -> dict:
    """Runs one single-rank section after the headline numbers exist; a
    failure there is reported in its own key instead of losing the line."""
    import traceback

    try:
        return fn()
    except Exception as e:  # noqa: BLE001 - any failure of an extra section
        traceback.print_exc(file=sys.stderr)
        return {"error": f"{type(e).__name__}: {e}"[:300], "section": name}


def run_large(args, stream, peaks) -> dict:
    """The large single solve: args.large_size^2 (generator smoothing x4,
    ~5 % scribbles, eps 1e-7), FP16 store, mixed CG to rel-res 1e-6 from
    alpha = 0.5, then the adjoint of loss = mean((alpha - alpha_gt)^2) (one
    more solve for lambda + the window back-propagation)."""
    import numpy as np
    import torch

    from gpumatting_b200 import api

    S = args.large_size
    N = S * S
    prob = cached_problem(S, S, 0)
    dev = torch.device("cuda", torch.cuda.current_device())
    img = torch.from_numpy(prob.image).to(dev)
    scr = torch.from_numpy(prob.scribbles).to(dev)
    gt = torch.from_numpy(prob.alpha_gt.astype(np.float32)).to(dev)
    st = api.LevinStore(S, S, "fp16")
    alpha = torch.empty((S, S), device=dev)

    def ev():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    out = {"size": f"{S}x{S}", "eps": prob.eps, "precision": "fp16"}
    for rep in range(2):  # the first run warms caches and the workspace
        e0, e1 = ev()
        e0.record(stream)
        st.assemble(img, scr, eps=prob.eps, gamma_value=100.0, stream=stream)
        e1.record(stream)
        alpha.fill_(0.5)
        r = st.solve(alpha, "cg", rtol=1e-6, max_iters=5000, stream=stream)
        torch.cuda.synchronize()
    alg = N * (r.iters * KRYLOV_BYTES["fp16"] + r.replacements * REPLACE_BYTES["sym_mixed"]
               + IMPORT_BYTES["sym_mixed"])
    out.update({"assemble_ms": e0.elapsed_time(e1), "solve_status": r.status, "iters": r.iters,
                "replacements": r.replacements, "rel_residual": r.rel_residual, "solve_kernel_ms": r.kernel_ms,
                "mpix_iter_s": N * r.iters / 1e3 / r.kernel_ms,
                "solver_frac_of_hbm_peak": alg / (r.kernel_ms / 1000) / 1e9 / peaks["hbm_gbs"],
                "hbm_peak_gbs": peaks["hbm_gbs"], "peak_source": peaks.get("source")})
    for rep in range(2):
        alpha.fill_(0.5)
        rp = st.solve(alpha, "pcg", rtol=1e-6, max_iters=5000, stream=stream)
        torch.cuda.synchronize()
    out.update({"pcg_status": rp.status, "pcg_iters": rp.iters, "pcg_rel_residual": rp.rel_residual,
                "pcg_solve_kernel_ms": rp.kernel_ms})
    for rep in range(2):
        alpha.fill_(0.5)
        rm = st.solve(alpha, "mg", rtol=1e-6, max_iters=5000, stream=stream)
        torch.cuda.synchronize()
    out.update({"mg_status": rm.status, "mg_iters": rm.iters, "mg_rel_residual": rm.rel_residual,
                "mg_solve_ms": rm.kernel_ms})
    dalpha = 2.0 * (alpha - gt) / N
    for solver in ("cg", "pcg", "mg"):
        for rep in range(2):
            e0, e1 = ev()
            e0.record(stream)
            dimage, dgamma, lam, ra = st.adjoint(alpha, dalpha, solver=solver, rtol=1e-6, max_iters=5000,
                                                 stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
        key = "adjoint" if solver == "cg" else "adjoint_" + solver
        out.update({f"{key}_ms": e0.elapsed_time(e1), f"{key}_status": ra.status, f"{key}_iters": ra.iters,
                    f"{key}_rel_residual": ra.rel_residual, f"{key}_solve_kernel_ms": ra.kernel_ms,
                    f"{key}_backprop_ms": e0.elapsed_time(e1) - ra.kernel_ms,
                    f"{key}_dimage_finite": bool(torch.isfinite(dimage).all().item())})
    return out


def run_slab(args, prob, img_d, scr_d, stream) -> dict:
    """The row-slab split of the headline image (gpumatting_b200/slab.py) on
    this one GPU: the image cut into `n` slabs held by one process, halo rows
    copied on the device, the slab CG (one operator pass and one FP64
    reduction per iteration) to rel-res 1e-6 from alpha = 0.5.  On several
    GPUs each slab would sit on its own GPU and the halo rows travel by NCCL
    send/recv; here the figure is the data plane's cost per iteration (the
    scalars on the device, chunks of 10 iterations as one CUDA graph)."""
    import torch

    from gpumatting_b200 import slab as S

    W, H = prob.W, prob.H
    out = {"workload": f"{W}x{H} headline image, FP32 slab stores, slab CG to rel-res 1e-6 from alpha = 0.5, "
                       "all slabs on this GPU (halo rows copied on the device)"}
    for n in args.slabs:
        slabs = [S.LevinSlab(img_d, scr_d, prob.eps, 100.0, *S.slab_bounds(H, n, k)) for k in range(n)]
        bs = [sl.rhs() for sl in slabs]
        comm = S.SlabComm(n, 0, n)
        xs = [torch.full((sl.R, W), 0.5, device=img_d.device) for sl in slabs]
        S.slab_cg(slabs, comm, xs, bs, rtol=0.0, max_iters=60)  # warm-up (captures the chunk graph)
        xs = [torch.full((sl.R, W), 0.5, device=img_d.device) for sl in slabs]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = S.slab_cg(slabs, comm, xs, bs, rtol=1e-6, max_iters=5000)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[f"slabs_{n}"] = {"ms": ms, "iters": res.iters, "replacements": res.replacements,
                             "rel_residual": res.rel_residual, "status": res.status,
                             "ms_per_iter": ms / max(1, res.iters)}
    return out


def run_spmv(args, stream, peaks) -> dict:
    """Standalone SpMV passes at args.spmv_size^2 (inputs larger than L2, so
    no flush): gm_levin_apply on the FP16 store (iteration operator), on its
    FP32 true operator, and the reference-layout 25-band FP32 gm_bm_ax."""
    import torch

    from gpumatting_b200 import api
    from gpumatting_b200.synth import make_problem

    S = args.spmv_size
    N = S * S
    prob = cached_problem(S, S, 0)
    dev = torch.device("cuda", torch.cuda.current_device())
    img = torch.from_numpy(prob.image).to(dev)
    scr = torch.from_numpy(prob.scribbles).to(dev)
    out = {"size": f"{S}x{S}", "l2": "not flushed: every pass streams > 126 MB", "launches_timed": args.spmv_reps}

    def time_fn(fn, k):
        for _ in range(3):
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for a, b in ev:
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return statistics.mean(a.elapsed_time(b) for a, b in ev)

    st = api.LevinStore(S, S, "fp16").assemble(img, scr, eps=prob.eps, gamma_value=100.0)
    x = torch.rand((S, S), device=dev)
    y = torch.empty_like(x)
    for key, true_op in (("fp16", False), ("true_fp32", True)):
        ms = time_fn(lambda: st.apply(x, y, true_op=true_op, stream=stream), args.spmv_reps)
        gbs = SPMV_BYTES[key] * N / (ms / 1000) / 1e9
        out[key] = {"kernel": "gm::levin_apply_kernel", "ms": ms, "bytes_per_px": SPMV_BYTES[key],
                    "achieved_gbs": gbs, "frac_of_hbm_peak": gbs / peaks["hbm_gbs"]}
    del st
    a, b = api.levin_bands25(img, scr, eps=prob.eps, gamma_value=100.0, arithmetic="fp64")
    Lm = api.DeviceBandedMatrix(a, torch.tensor(api.levin_band_offsets(S), device=dev), N)
    xp = api.PaddedVector(N, api.levin_pad(S))
    xp.data.uniform_()
    yb = torch.empty(N, device=dev)
    ms = time_fn(lambda: api.bm_ax(yb, Lm, xp, stream=stream), args.spmv_reps)
    gbs = SPMV_BYTES["ref25"] * N / (ms / 1000) / 1e9
    out["ref25"] = {"kernel": "gm_bm_ax (reference 25-band FP32 layout)", "ms": ms,
                    "bytes_per_px": SPMV_BYTES["ref25"], "achieved_gbs": gbs,
                    "frac_of_hbm_peak": gbs / peaks["hbm_gbs"]}
    out["hbm_peak_gbs"] = peaks["hbm_gbs"]
    out["peak_source"] = peaks.get("source")
    return out


def run_batch(args, stream, world: int = 1, rank: int = 0) -> dict:
    """64 images, W and H uniform in [256, 1024] (seeded): all assembled into
    one FP16 batch store and solved to rel-res 1e-6 in ONE persistent launch
    replayed from a CUDA graph (launch shape from the batch autotuner), versus
    the same 64 images solved one after another with the plain FP32 method
    (25-band FP32 store, fused CG to 1e-6)."""
    import torch

    from gpumatting_b200 import api
    from gpumatting_b200.synth import batch_sizes, make_problem

    from gpumatting_b200.shard import shard_images

    all_sizes = batch_sizes(args.batch_count, 256, 1024, seed=0)
    mine = shard_images(all_sizes, world)[rank]  # whole images per rank, no exchange
    sizes = [all_sizes[k] for k in mine]
    dev = torch.device("cuda", torch.cuda.current_device())
    probs = [make_problem(W, H, 100 + k) for k, (W, H) in zip(mine, sizes)]
    imgs = [torch.from_numpy(p.image).to(dev) for p in probs]
    scrs = [torch.from_numpy(p.scribbles).to(dev) for p in probs]
    npx = sum(W * H for W, H in sizes)
    batch = api.LevinBatch(sizes, "fp16")
    for k, p in enumerate(probs):
        batch.assemble(k, imgs[k], scrs[k], eps=p.eps, gamma_value=100.0, stream=stream)
    alphas = [torch.empty((H, W), device=dev) for W, H in sizes]
    t_tune = time.time()
    shape = batch.tune(iters=20, stream=stream)
    t_tune = time.time() - t_tune
    ms, res = [], None
    for i in range(2 + args.batch_steps):
        for a in alphas:
            a.fill_(0.5)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = batch.solve(alphas, "cg", rtol=1e-6, max_iters=5000, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= 2:
            ms.append(e0.elapsed_time(e1))
    assert all(r.status == 0 and r.rel_residual <= 1e-6 for r in res), [r.status for r in res]
    ms_pcg = []
    for i in range(1 + args.batch_steps):
        for a in alphas:
            a.fill_(0.5)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res_p = batch.solve(alphas, "pcg", rtol=1e-6, max_iters=5000, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= 1:
            ms_pcg.append(e0.elapsed_time(e1))
    assert all(r.status == 0 and r.rel_residual <= 1e-6 for r in res_p), [r.status for r in res_p]
    # multigrid PCG on the same store views: one graph launch per image, the
    # images spread over up to 8 concurrent streams (gm_levin_solve_mg_many)
    views = [batch.store_view(k) for k in range(len(sizes))]
    ms_mg = []
    for i in range(2 + args.batch_steps):
        for a in alphas:
            a.fill_(0.5)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res_m = api.mg_solve_many(views, alphas, rtol=1e-6, max_iters=5000, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= 2:
            ms_mg.append(e0.elapsed_time(e1))
    assert all(r.status == 0 and r.rel_residual <= 1e-6 for r in res_m), [r.status for r in res_m]
    its = [r.iters for r in res]
    batch_ms = allreduce_max(statistics.mean(ms), world)
    work = allreduce_sum(sum(W * H * i for (W, H), i in zip(sizes, its)), world)
    npx = allreduce_sum(npx, world)
    out = {"images": len(all_sizes), "n_gpus": world, "mpix": npx / 1e6,
           "sizes": "W, H uniform in [256, 1024], seed 0; size-balanced bins of whole images per GPU",
           "batch_ms": batch_ms, "batch_mpix_iter_s": work / 1e3 / batch_ms,
           "iters_min_mean_max": [min(its), statistics.mean(its), max(its)],
           "launch": "1 cooperative launch per GPU from a CUDA graph", "tuned_shape": shape, "tune_s": t_tune,
           "batch_pcg_ms": allreduce_max(statistics.mean(ms_pcg), world),
           "pcg_iters_min_mean_max": [min(r.iters for r in res_p), statistics.mean(r.iters for r in res_p),
                                      max(r.iters for r in res_p)],
           "batch_mg_ms": allreduce_max(statistics.mean(ms_mg), world),
           "mg_iters_min_mean_max": [min(r.iters for r in res_m), statistics.mean(r.iters for r in res_m),
                                     max(r.iters for r in res_m)],
           "mg_launch": "1 graph launch per image on up to 8 concurrent streams, images dealt largest first"}
    if world > 1:
        return out
    # sequential plain FP32 solves of the same images
    seq_ms, seq_its = 0.0, []
    for k, p in enumerate(probs):
        W, H = sizes[k]
        a, b = api.levin_bands25(imgs[k], scrs[k], eps=p.eps, gamma_value=100.0, arithmetic="fp64")
        Lm = api.DeviceBandedMatrix(a, torch.tensor(api.levin_band_offsets(W), device=dev), W * H)
        x = api.PaddedVector(W * H, api.levin_pad(W))
        for rep in range(2):
            x.data.fill_(0.5)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = api.banded_solve(Lm, x, b, W=W, solver="cg", rtol=1e-6, max_iters=5000, replace_every=50)
            e1.record(stream)
            torch.cuda.synchronize()
        assert r.status == 0, r
        seq_ms += e0.elapsed_time(e1)
        seq_its.append(r.iters)
        del a, b, Lm, x
    out.update({"sequential_plain_fp32_ms": seq_ms, "sequential_iters_mean": statistics.mean(seq_its),
                "speedup_vs_sequential_plain": seq_ms / batch_ms,
                "pcg_speedup_vs_sequential_plain": seq_ms / out["batch_pcg_ms"],
                "mg_speedup_vs_sequential_plain": seq_ms / out["batch_mg_ms"]})
    return out


def run_solvers(args, prob, img_d, scr_d, store, flush, stream) -> dict:
    """The 1080p workload with every solver, mixed FP16 store against the plain
    FP32 25-band store: CG, steepest descent and damped Jacobi (omega 2/3) to
    true rel-res 1e-6, then CG and Jacobi PCG to 1e-10, the tolerance at which
    alpha comes within 1e-4 of the FP64 solution (rel-res 1e-6 leaves every
    solver, FP64 CG included, about 0.3 from it).  One solve per entry after
    the headline's warm-up; L2 flushed before each."""
    import torch

    from gpumatting_b200 import api

    W, H = prob.W, prob.H
    N = W * H
    alpha = torch.empty((H, W), dtype=torch.float32, device=img_d.device)
    a, b = api.levin_bands25(img_d, scr_d, eps=prob.eps, gamma_value=100.0, arithmetic="fp64")
    Lm = api.DeviceBandedMatrix(a, torch.tensor(api.levin_band_offsets(W), device=a.device), N)
    x = api.PaddedVector(N, api.levin_pad(W))

    def one(run, i):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = run()
        e1.record(stream)
        torch.cuda.synchronize()
        return {"ms": e0.elapsed_time(e1), "iters": r.iters, "replacements": r.replacements,
                "rel_residual": r.rel_residual, "status": r.status}

    def mixed(solver, rtol, max_iters):
        def run():
            alpha.fill_(0.5)
            return store.solve(alpha, solver, rtol=rtol, max_iters=max_iters, stream=stream)
        return run

    def plain(solver, rtol, max_iters):
        def run():
            x.data.fill_(0.5)
            return api.banded_solve(Lm, x, b, W=W, solver=solver, rtol=rtol, max_iters=max_iters, replace_every=50)
        return run

    out = {"workload": f"{W}x{H} headline problem, alpha0 = 0.5, max 400000 iterations (GD, Jacobi) / 50000 (CG)"}
    i = 0
    for solver in ("cg", "gd", "jacobi"):
        mi = 50000 if solver == "cg" else 400000
        out[f"{solver}_1e-6"] = {"mixed_fp16": one(mixed(solver, 1e-6, mi), i), "plain_fp32": one(plain(solver, 1e-6, mi), i + 1)}
        i += 2
    # plain FP32 CG stalls near rel-res 1e-5 below 1e-6 (FP32 iterate); 10000 iterations show it
    out["cg_1e-10"] = {"mixed_fp16": one(mixed("cg", 1e-10, 50000), i), "mixed_fp16_pcg": one(mixed("pcg", 1e-10, 50000), i + 1),
                       "mixed_fp16_mg": one(mixed("mg", 1e-10, 5000), i + 2),
                       "plain_fp32": one(plain("cg", 1e-10, 10000), i + 3)}
    return out


def run_plain(args, prob, img_d, scr_d, flush, stream, mixed_once) -> dict:
    """Plain FP32 method (25-band FP32 store + fused CG to 1e-6) timed
    interleaved with the mixed arm: each round solves with both (order
    alternating between rounds), L2 flushed before every solve, so clock or
    thermal drift hits both arms alike.  mixed_once(i) -> (ms, result)."""
    import numpy as np
    import torch

    from gpumatting_b200 import api

    W, H = prob.W, prob.H
    N = W * H
    a, b = api.levin_bands25(img_d, scr_d, eps=prob.eps, gamma_value=100.0, arithmetic="fp64")
    Lm = api.DeviceBandedMatrix(a, torch.tensor(api.levin_band_offsets(W), device=a.device), N)
    x = api.PaddedVector(N, api.levin_pad(W))

    def plain_once(i):
        x.data.fill_(0.5)
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = api.banded_solve(Lm, x, b, W=W, solver="cg", rtol=1e-6, max_iters=5000, replace_every=50)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    rounds = max(5, args.plain_steps)
    res_all, ms, mixed_ms, mixed_res = [], [], [], []
    for i in range(2 + rounds):
        order = (plain_once, mixed_once) if i % 2 == 0 else (mixed_once, plain_once)
        out = {f: f(2 * i + k) for k, f in enumerate(order)}
        if i >= 2:
            ms.append(out[plain_once][0])
            res_all.append(out[plain_once][1])
            mixed_ms.append(out[mixed_once][0])
            mixed_res.append(out[mixed_once][1])
    assert all(r.status == 0 and r.rel_residual <= 1e-6 for r in mixed_res), mixed_res
    it = statistics.mean(r.iters for r in res_all)
    kms = statistics.mean(r.kernel_ms for r in res_all)
    reps = statistics.mean(r.replacements for r in res_all)
    alg = N * (it * KRYLOV_BYTES["ref25"] + reps * REPLACE_BYTES["ref25"] + IMPORT_BYTES["ref25"])
    ratios = [p / m for p, m in zip(ms, mixed_ms)]
    return {"ms_per_solve": statistics.median(ms), "ms_min": min(ms), "ms_max": max(ms), "rounds": rounds,
            "iters": it, "rel_residual": res_all[-1].rel_residual,
            "mpix_iter_s": N * it / 1e6 / (statistics.median(ms) / 1000), "kernel_ms": kms,
            "achieved_gbs": alg / (kms / 1000) / 1e9, "status": res_all[-1].status,
            "mixed_ms_per_solve": statistics.median(mixed_ms), "mixed_ms_min": min(mixed_ms),
            "mixed_ms_max": max(mixed_ms), "mixed_iters": statistics.mean(r.iters for r in mixed_res),
            "speedup_median": statistics.median(ms) / statistics.median(mixed_ms),
            "speedup_per_round_min": min(ratios), "speedup_per_round_max": max(ratios)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--W", type=int, default=1920)
    ap.add_argument("--H", type=int, default=1080)
    ap.add_argument("--precision", choices=["fp16", "bf16", "fp32"], default="fp16")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-pcg", action="store_true", help="skip the Jacobi-preconditioned comparison")
    ap.add_argument("--no-mg", action="store_true", help="skip the multigrid-preconditioned comparison")
    ap.add_argument("--solver", choices=["cg", "pcg", "mg"], default="cg",
                    help="solver of the headline step (profiling; the reported metric uses cg)")
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--no-solvers", action="store_true", help="skip the GD / Jacobi / tight-tolerance section")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    ap.add_argument("--fixed-iters", type=int, default=0, help="profiling: run exactly this many CG iterations")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--spmv-size", type=int, default=4096, help="standalone SpMV measurement size (0 = skip)")
    ap.add_argument("--spmv-reps", type=int, default=20)
    ap.add_argument("--slabs", type=int, nargs="*", default=[2],
                    help="row-slab section: slab counts to run on this GPU (empty = skip)")
    ap.add_argument("--spmv-only", action="store_true", help="profiling: only the standalone SpMV passes")
    ap.add_argument("--batch-count", type=int, default=64, help="batched-solve measurement: images (0 = skip)")
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--batch-only", action="store_true", help="profiling: only the batched solve")
    ap.add_argument("--large-size", type=int, default=4096, help="large single solve + adjoint size (0 = skip)")
    ap.add_argument("--large-only", action="store_true", help="profiling: only the large solve + adjoint")
    ap.add_argument("--replace-every", type=int, default=50)
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="ring configuration: 0 auto, 3 shallow, 2 deep")
    ap.add_argument("--strip-width", type=int, default=0, help="fused solver strip width: 0 auto, 192, 128")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.large_only:
        import torch

        print(json.dumps({"large": run_large(args, torch.cuda.current_stream(), load_peaks())}), flush=True)
    elif args.batch_only:
        import torch

        print(json.dumps({"batch": run_batch(args, torch.cuda.current_stream())}), flush=True)
    elif args.spmv_only:
        import torch

        line = {"spmv": run_spmv(args, torch.cuda.current_stream(), load_peaks())}
        print(json.dumps(line), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
