"""Benchmark of the fixed-box carrier step on B200.

Workload (one "step" = one carrier step): 128^3 cells, f64 faces, unit
spacing, solid walls, random-Fourier initial velocity (8 modes, wavenumbers
1-8, amplitude 1, + 0.05 uniform noise), dt at CFL 0.5 of the reference's
Courant rate, semi-Lagrangian advection, RHS, Jacobi-PCG to relative residual
1e-8 (absolute 0, no divergence gate), gradient correction, actual-divergence
and Courant gates. Metric: cell-steps/s of accepted steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun), each rank advances its own replica
box (independent instances; no data-path collective), weak scaling. Timing is
per rank with CUDA events on the carrier's stream; the job time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

# 32 hardware work queues instead of the default 8, so that the batched and
# serving legs' per-instance streams run concurrently (read when the CUDA
# context is created; a value already in the environment wins).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOAD = ("fixed-box carrier step: {n}^3 cells, {storage} faces, random-Fourier init, CFL 0.5, "
            "{method} to rel residual 1e-8")
METRIC = "cell-steps/s at rel. residual 1e-8 (plain f64 GPU path)"
UNIT = "cell-steps/s"
MAXF = 1.7976931348623157e308


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--method", default="jacobi", choices=["jacobi", "rbsgs", "sgs", "mixed"])
    ap.add_argument("--storage", default="f64", choices=["f64", "f32"])
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=25.0, help="seconds of CPU work for the CPU baseline")
    ap.add_argument("--max-iters", type=int, default=0,
                    help="cap PCG iterations per step (profiling runs only; 0 = solve to 1e-8)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-instances", type=int, default=64)
    ap.add_argument("--batched-steps", type=int, default=20)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--solve-only", action="store_true",
                    help="profiling aid: time pressure solves of one step's RHS through the workspace")
    ap.add_argument("--serving-requests", type=int, default=200)
    ap.add_argument("--serving-plain-requests", type=int, default=12)
    ap.add_argument("--serving-budget-gb", type=float, default=150.0)
    ap.add_argument("--serving-projection-share", type=float, default=0.25,
                    help="share of serving requests that are projections of a supplied velocity")
    ap.add_argument("--no-profile", action="store_true")
    ap.add_argument("--no-dense3d", action="store_true")
    ap.add_argument("--dense3d", action="store_true",
                    help="dense3D frame stream alone (device encode, end to end to a file descriptor, CPU oracle)")
    ap.add_argument("--dense3d-frames", type=int, default=20)
    ap.add_argument("--no-liquid", action="store_true")
    ap.add_argument("--liquid", action="store_true",
                    help="liquid-volume transport alone (device interval, liquid step on the mixed carrier, CPU oracle)")
    ap.add_argument("--no-box-flux", action="store_true")
    ap.add_argument("--box-flux", action="store_true",
                    help="box-flux projection alone (device projection, passes, host-array call, CPU oracle)")
    ap.add_argument("--advect", action="store_true",
                    help="the advect_velocity primitive alone at --n (f64 faces, the reference's arithmetic)")
    ap.add_argument("--batch-profile", action="store_true",
                    help="per-kernel device times of one packed batched step (eager launches with events)")
    ap.add_argument("--oracle-steps", type=int, default=1,
                    help="buoyant-blob mode: steps also computed by the FP64 CPU oracle (all host threads)")
    ap.add_argument("--buoyant-blob", action="store_true",
                    help="mixed-precision buoyant-blob run (rel 1e-10) in lockstep with the f64 carrier, "
                         "per-step divergence and velocity/tracer error; --n cells per axis, --steps steps")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for i, name in enumerate(names):
                    if parts[5 + i].lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def run_e2e(args, g, cfg, faces, prm, flush, local, world):
    """Same metric through the public API with host buffers: per step, H2D of
    the step's input faces from pinned memory, the step, D2H of the result."""
    import torch

    import rheon_b200 as R

    pinned = [torch.from_numpy(f).pin_memory() for f in faces]
    sim = R.CarrierSimulation(g, cfg)
    sim.upload(faces)
    ptrs = [int(p.data_ptr()) for p in pinned]
    for _ in range(max(1, args.warmup)):
        sim.upload_ptrs(*ptrs)
        sim.step(prm)
        sim.download_ptrs(*ptrs)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    total = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.upload_ptrs(*ptrs)
        sim.step(prm)
        sim.download_ptrs(*ptrs)
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
    sim.close()
    if world > 1:
        import torch.distributed as dist

        tt = torch.tensor([total], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total = float(tt.item())
    return total


def run_batched(args, local, flush):
    """Batched uneven instances (the packed batch): boxes with edges drawn by
    seed from {32, 48, 64, 96, 128}, each with its own random-Fourier velocity,
    in the mixed-precision configuration at rel. residual 1e-8, all advanced
    together by one CUDA graph per batched step whose every stage is one launch
    over the packed instance table. The step is timed with CUDA events on the
    batch's stream. For comparison the same boxes also run as one resident
    carrier each, their step graphs launched together on separate streams."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import workloads as W

    edges = np.array([32, 48, 64, 96, 128])
    pick = ((W.uniform(args.seed, 40, args.batched_instances) + 1.0) * 0.5 * len(edges)).astype(int)
    sizes = [int(edges[min(i, len(edges) - 1)]) for i in pick]
    cfg = R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 1000), device=local)
    init = [W.fourier_faces((n, n, n), seed=args.seed + 1000 + i, dtype=np.float32) for i, n in enumerate(sizes)]
    batch = R.BatchedCarriers([R.GridGeometry((n, n, n)) for n in sizes], cfg)
    for i, f in enumerate(init):
        batch.upload(i, f)
    stream = torch.cuda.ExternalStream(batch.stream(), device=local)
    prm = R.StepParams(MAXF, cfl=0.5)
    for _ in range(max(3, args.warmup)):
        if any(st != 0 for st, _ in batch.step(prm)):
            raise RuntimeError("batched warm-up step rejected")
    cells = [n ** 3 for n in sizes]
    faces_total = [3 * n * n * (n + 1) for n in sizes]
    total_ms, cell_steps, iters, model_bytes, launches, solve_ms = 0.0, 0, [], 0.0, 0, 0.0
    for _ in range(args.batched_steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch.step_async(prm)
        b.record(stream)
        out = batch.step_wait()
        b.synchronize()
        if any(st != 0 for st, _ in out):
            raise RuntimeError("batched step rejected")
        total_ms += a.elapsed_time(b)
        cell_steps += sum(cells)
        its = [r.pressure.iterations for _, r in out]
        iters += its
        launches += out[0][1].kernel_launches
        solve_ms += out[0][1].pressure_ms
        # the algorithmic byte model of a mixed step, summed over instances:
        # 130N per outer iteration (FP32 V(2,2), levels summed, + FP64 defect
        # and accumulation) and 5 F s + 16N for advection, RHS and correction
        model_bytes += sum(it * 130 * c + 5 * f * 4 + 16 * c for it, c, f in zip(its, cells, faces_total))
    hbm, hbm_kind = peaks()
    achieved = model_bytes / (total_ms / 1e3) / 1e9
    ms_step = total_ms / args.batched_steps
    result = {
        "value": cell_steps / (total_ms / 1e3),
        "unit": UNIT,
        "instances": len(sizes),
        "edges": {str(e): sizes.count(int(e)) for e in edges},
        "cells": sum(cells),
        "steps": args.batched_steps,
        "ms_per_batched_step": ms_step,
        "solve_ms_per_batched_step": solve_ms / args.batched_steps,
        "iterations_per_step": statistics.mean(iters),
        "iterations_max": max(iters),
        "graph_launches_per_batched_step": 1,
        "kernels_per_batched_step": launches / args.batched_steps,
        "dtype": "mixed (f32 faces and V-cycles, f64 residual/accumulation/coarse solve)",
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "peak_kind": hbm_kind, "unit": "GB/s",
                     "frac": achieved / hbm, "bytes_per_batched_step": model_bytes / args.batched_steps,
                     "model": "sum over instances of 130N per outer iteration + 5Fs + 16N per step"},
    }
    batch.close()
    # the same boxes as separate resident carriers launched together
    sims = []
    for i, n in enumerate(sizes):
        sim = R.CarrierSimulation(R.GridGeometry((n, n, n)), cfg)
        sim.upload(init[i])
        sims.append(sim)
    streams = [torch.cuda.ExternalStream(sm.stream(), device=local) for sm in sims]
    join = torch.cuda.Stream(device=local)
    for _ in range(max(3, args.warmup)):
        R.step_all(sims, [prm] * len(sims))
    sep_ms = 0.0
    steps_sep = max(1, min(args.batched_steps, 5))
    for _ in range(steps_sep):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(join)
        for st in streams:
            st.wait_event(a)
        for sm in sims:
            sm.step_async(prm)
        for st in streams:
            e = torch.cuda.Event()
            e.record(st)
            join.wait_event(e)
        b.record(join)
        for sm in sims:
            sm.step_wait()
        b.synchronize()
        sep_ms += a.elapsed_time(b)
    for sm in sims:
        sm.close()
    result["separate_carriers"] = {"ms_per_batched_step": sep_ms / steps_sep,
                                   "value": sum(cells) * steps_sep / (sep_ms / 1e3),
                                   "note": "one step graph per box on its own stream, launched together"}
    return result


def run_advect(args, local):
    """advect_velocity (src/advection.rs:28-68) alone: f64 faces of the
    random-Fourier field at n^3, dt at CFL 0.5, the reference's f64
    arithmetic; device time per launch (CUDA events over 10 launches after 3)
    and the achieved bandwidth of its algorithmic bytes (read and write every
    face once: 2 F s)."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import workloads as W

    n = (args.n,) * 3
    g = R.GridGeometry(n)
    host = W.fourier_faces(n, seed=args.seed, dtype=np.float64)
    rate = sum(float(np.max(np.abs(host[d]))) for d in range(3))
    dt = 0.5 / rate
    f = [torch.from_numpy(a).to(f"cuda:{local}") for a in host]
    out = [torch.empty_like(a) for a in f]
    for _ in range(3):
        R.advect_velocity(g, f, dt, out)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(local)
    ms = 0.0
    for _ in range(10):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        R.advect_velocity(g, f, dt, out)
        b.record(stream)
        b.synchronize()
        ms += a.elapsed_time(b)
    ms /= 10
    faces = sum(g.face_len(d) for d in range(3))
    hbm, kind = peaks()
    ach = 2 * faces * 8 / (ms / 1e3) / 1e9
    return {"mode": "advect", "n": args.n, "faces": faces, "ms_per_launch_with_validation": ms,
            "note": "each call validates the faces (one pass) before advecting",
            "achieved_gbs": ach, "peak_gbs": hbm, "peak_kind": kind}


def run_batch_profile(args, local):
    """One packed batched step of the batched workload issued eagerly with an
    event after every launch: per kernel kind the device time and launches."""
    import rheon_b200 as R
    from rheon_b200 import workloads as W

    edges = np.array([32, 48, 64, 96, 128])
    pick = ((W.uniform(args.seed, 40, args.batched_instances) + 1.0) * 0.5 * len(edges)).astype(int)
    sizes = [int(edges[min(i, len(edges) - 1)]) for i in pick]
    cfg = R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 1000), device=local)
    batch = R.BatchedCarriers([R.GridGeometry((n, n, n)) for n in sizes], cfg)
    for i, n in enumerate(sizes):
        batch.upload(i, W.fourier_faces((n, n, n), seed=args.seed + 1000 + i, dtype=np.float32))
    prm = R.StepParams(MAXF, cfl=0.5)
    # warm-up steps issued eagerly too, so that every kernel of the process is
    # visible to a profiler (kernels inside the step graph's conditional nodes
    # are not)
    for _ in range(max(3, args.warmup)):
        batch.profile_step(prm)
    prof = batch.profile_step(prm)
    batch.close()
    total = sum(ms for ms, _ in prof["kernels"].values())
    return {"mode": "batch-profile", "instances": len(sizes), "cells": sum(n ** 3 for n in sizes),
            "iterations": sorted({r.pressure.iterations for r in prof["reports"]}), "total_ms": total,
            "kernels": {k: {"ms": ms, "launches": c, "share": ms / total}
                        for k, (ms, c) in sorted(prof["kernels"].items(), key=lambda kv: -kv[1][0])}}


def run_mixed_large(args, local, flush, n):
    """The mixed-precision carrier at n^3 (random-Fourier state generated on the
    device, CFL 0.5, rel. residual 1e-8): device-timed steps and the step's
    roofline under the algorithmic byte model (130N per outer iteration,
    5 F s + 16N per step, s = 4)."""
    import torch

    import rheon_b200 as R

    g = R.GridGeometry((n, n, n))
    sim = R.CarrierSimulation(g, R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 1000),
                                                       device=local))
    sim.init_fourier(args.seed)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    prm = R.StepParams(MAXF, cfl=0.5)
    for _ in range(args.warmup):
        sim.step(prm)
    ms, its, solve = 0.0, [], 0.0
    steps = max(1, args.steps)
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rep = sim.step(prm)
        b.record(stream)
        b.synchronize()
        ms += a.elapsed_time(b)
        its.append(rep.pressure.iterations)
        solve += rep.pressure_ms
    sim.close()
    cells = n ** 3
    faces = 3 * n * n * (n + 1)
    step_bytes = statistics.mean(its) * 130 * cells + 5 * faces * 4 + 16 * cells
    hbm, hbm_kind = peaks()
    ach = step_bytes / (ms / steps / 1e3) / 1e9
    return {"workload": f"mixed carrier step at {n}^3, random-Fourier init, CFL 0.5, rel 1e-8",
            "value": cells * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
            "pressure_ms_per_step": solve / steps, "iterations_per_step": statistics.mean(its),
            "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "peak_kind": hbm_kind, "unit": "GB/s",
                         "frac": ach / hbm, "bytes_per_step": step_bytes,
                         "model": "130N per outer iteration + 5Fs + 16N per step"}}


def run_serving(args, local):
    """Serving loop: step requests of k in [1, 20] steps and projection
    requests (one projection of a supplied velocity, dt 0.01) on boxes with
    edges log-uniform in [32, 256] (multiples of 8), random-Fourier velocity,
    mixed precision at rel. residual 1e-8, admitted while the pooled carriers
    fit the HBM budget. Capacity is measured first with every request arriving
    at once (this also warms the carrier pool); then a Poisson stream at 80 % of
    that capacity is served. The plain per-request f64 path (one request at a
    time, Jacobi-PCG f64 carriers) runs on the first requests of the same stream
    for comparison. Latency = finish - arrival (queueing included); every
    request's device interval is recorded with CUDA events on its carrier's
    stream, and the pairs of requests whose device intervals overlap are
    counted."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import serving as SV

    free, _total = torch.cuda.mem_get_info(local)
    budget = int(min(args.serving_budget_gb * 1e9, free - 8e9))
    cfg = R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 1000), device=local)
    share = args.serving_projection_share
    loop = SV.ServingLoop(cfg, budget, device_times=True)
    n_cap = max(8, min(args.serving_requests, 64))
    cap_reqs = SV.make_requests(n_cap, rate_hz=0.0, seed=args.seed + 5, projection_share=share)
    cap_done = loop.run(cap_reqs)
    capacity = len(cap_done) / loop.elapsed
    rate = 0.8 * capacity
    reqs = SV.make_requests(args.serving_requests, rate_hz=rate, seed=args.seed + 6, projection_share=share)
    done = loop.run(reqs)
    served = SV.summarize(done, loop.elapsed)
    served["overlapping_request_pairs"] = SV.overlapping_pairs(done)
    pool_gb = loop.pool.used / 1e9
    loop.close()
    plain_cfg = R.CarrierConfig(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 1000000), storage="f64",
                                implementation=R.PressureImplementation.JACOBI_PCG_V1, device=local)
    plain_reqs = reqs[: args.serving_plain_requests]
    plain = SV.ServingLoop(plain_cfg, budget, max_in_flight=1)
    plain_done = plain.run(plain_reqs)
    plain_summary = SV.summarize(plain_done, plain.elapsed)
    plain.close()
    return {
        "workload": f"step requests of k in [1,20] steps and projection requests ({share:.0%} of the stream, dt "
                    "0.01), edge log-uniform in [32,256] (multiple of 8), random-Fourier velocity, mixed precision "
                    "to rel residual 1e-8, Poisson arrivals at 0.8 x measured capacity",
        "requests": args.serving_requests,
        "capacity_requests_per_s": capacity,
        "arrival_rate_per_s": rate,
        "hbm_budget_gb": budget / 1e9,
        "pool_gb": pool_gb,
        "mixed": served,
        "plain_f64_per_request": dict(plain_summary, requests_run=len(plain_reqs)),
    }


def run_solve_only(args, local):
    """Profiling aid: pressure solves (method of --method) of the RHS of the
    workload's first step, through a PressureWorkspace, whose iteration chunks
    are plain CUDA graphs (listed kernel by kernel by ncu)."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import workloads as W

    torch.cuda.set_device(local)
    n = (args.n,) * 3
    g = R.GridGeometry(n)
    faces = [torch.from_numpy(f).cuda() for f in W.fourier_faces(n, seed=args.seed, dtype=np.float64)]
    op = R.PressureOperator(g, 1.0)
    rhs = torch.empty(g.cell_len(), dtype=torch.float64, device="cuda")
    op.build_rhs(faces, 0.05, rhs)
    method = {"jacobi": R.PressureImplementation.JACOBI_PCG_V1, "rbsgs": R.PressureImplementation.RBSGS_PCG,
              "sgs": R.PressureImplementation.SGS_PCG_V1, "mixed": R.PressureImplementation.MG_MIXED}[args.method]
    ws = R.PressureWorkspace(g, 1 << 40, method, device=local)
    settings = R.PressureSettings(1e-8, 0.0, MAXF, args.max_iters if args.max_iters > 0 else 1000000)
    stream = torch.cuda.ExternalStream(ws.stream(), device=local)
    for _ in range(args.warmup):
        ws.solve_rhs(op, rhs, 0.05, settings)
    total, its = 0.0, []
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rep = ws.solve_rhs(op, rhs, 0.05, settings)
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
        its.append(rep.iterations)
    return {"mode": "solve-only", "method": args.method, "n": args.n, "ms_per_solve": total / args.steps,
            "iterations": statistics.mean(its)}


def run_buoyant_blob(args, local):
    """Mixed precision on a buoyant Gaussian blob: the mixed carrier (FP32
    faces and advection, FP32 multigrid V(2,2) inside FP64 flexible CG, FP64
    residual, accumulation and coarsest solve) to relative residual 1e-10,
    stepped in lockstep with the f64 carrier (f64 faces and advection,
    Jacobi-PCG to 1e-10: the path that tracks the oracle per iteration). Both
    advect a passive density blob (sigma 20 cells, peak 1, centred at
    (n/2, n/4, n/2)) that drives buoyancy g_b = 1 on Y faces. Each step the
    mixed carrier takes the f64 carrier's dt (CFL 0.5). Per step: iterations,
    both actual divergences, velocity and tracer relative L2 errors. The first
    --oracle-steps steps are also computed by the FP64 CPU oracle on all host
    threads from the same state with the same dt, and both device paths are
    compared with it."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import workloads as W

    torch.cuda.set_device(local)
    n = (args.n,) * 3
    g = R.GridGeometry(n)
    rel = 1e-10
    faces = W.fourier_faces(n, seed=args.seed, dtype=np.float64)
    blob = W.gaussian_blob(n, sigma=20.0, peak=1.0)
    ref = R.CarrierSimulation(g, R.CarrierConfig(pressure=R.PressureSettings(rel, 0.0, MAXF, 1000000), storage="f64",
                                                 with_tracer=True, device=local))
    mix = R.CarrierSimulation(g, R.CarrierConfig.mixed(pressure=R.PressureSettings(rel, 0.0, MAXF, 1000),
                                                       with_tracer=True, device=local))
    ref.upload(faces, blob)
    mix.upload([f.astype(np.float32) for f in faces], blob)
    import oracle as O

    og = O.grid(n)
    o_faces, o_tracer = faces, blob
    threads = os.cpu_count() or 1
    cuda = torch.device(f"cuda:{local}")
    rb = [torch.empty(g.face_len(d), dtype=torch.float64, device=cuda) for d in range(3)]
    mb = [torch.empty(g.face_len(d), dtype=torch.float32, device=cuda) for d in range(3)]
    rt = torch.empty(g.cell_len(), dtype=torch.float32, device=cuda)
    mt = torch.empty(g.cell_len(), dtype=torch.float32, device=cuda)
    stream = torch.cuda.ExternalStream(mix.stream(), device=local)
    rows, mix_ms = [], 0.0
    for _ in range(args.steps):
        rr = ref.step(R.StepParams(MAXF, cfl=0.5, buoyancy=1.0))
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rm = mix.step(R.StepParams(rr.dt, cfl=0.0, buoyancy=1.0))
        b.record(stream)
        b.synchronize()
        mix_ms += a.elapsed_time(b)
        ref.download_ptrs(*[t.data_ptr() for t in rb], rt.data_ptr())
        mix.download_ptrs(*[t.data_ptr() for t in mb], mt.data_ptr())
        torch.cuda.synchronize()
        num = sum(float((mb[d].double() - rb[d]).pow(2).sum()) for d in range(3))
        den = sum(float(rb[d].pow(2).sum()) for d in range(3))
        terr = float((mt.double() - rt.double()).norm() / rt.double().norm())
        row = {"dt": rr.dt, "it_f64": rr.pressure.iterations, "it_mixed": rm.pressure.iterations,
               "div_f64": rr.actual_divergence_max, "div_mixed": rm.actual_divergence_max,
               "vel_rel_l2": math.sqrt(num / den), "tracer_rel_l2": terr}
        if len(rows) < args.oracle_steps:
            t0 = time.perf_counter()
            prm = O.StepParams(rr.dt, 1.0, O.JACOBI_PCG_V1, O.settings(rel, 0.0, MAXF, 1000000), 1.0, 0, threads)
            st, o_faces, o_tracer, orep = O.carrier_step(og, o_faces, prm, tracer=o_tracer)
            if st != O.OK:
                raise RuntimeError(f"oracle step failed: {st}")
            ot = torch.from_numpy(o_tracer.astype(np.float64))
            den_o = sum(float(np.dot(o_faces[d], o_faces[d])) for d in range(3))
            num_m = sum(float((mb[d].double().cpu() - torch.from_numpy(o_faces[d])).pow(2).sum()) for d in range(3))
            num_r = sum(float((rb[d].cpu() - torch.from_numpy(o_faces[d])).pow(2).sum()) for d in range(3))
            row["oracle"] = {"it": orep.pressure.iterations, "div": orep.actual_divergence_max,
                             "seconds": time.perf_counter() - t0, "threads": threads,
                             "mixed_vel_rel_l2": math.sqrt(num_m / den_o), "f64_vel_rel_l2": math.sqrt(num_r / den_o),
                             "mixed_tracer_rel_l2": float((mt.double().cpu() - ot).norm() / ot.norm()),
                             "f64_tracer_rel_l2": float((rt.double().cpu() - ot).norm() / ot.norm())}
        rows.append(row)
    cells = g.cell_len()
    out = {
        "mode": "buoyant-blob", "n": args.n, "steps": args.steps, "relative_residual": rel,
        "mixed_ms_per_step": mix_ms / args.steps,
        "mixed_cell_steps_per_s": cells * args.steps / (mix_ms / 1e3),
        "max_vel_rel_l2": max(r["vel_rel_l2"] for r in rows),
        "max_tracer_rel_l2": max(r["tracer_rel_l2"] for r in rows),
        "max_div_mixed": max(r["div_mixed"] for r in rows),
        "max_div_f64": max(r["div_f64"] for r in rows),
        "per_step": rows,
    }
    ref.close()
    mix.close()
    return out


# ------------------------------------------------------------------ our arm
def run_dense3d(args, local, with_cpu):
    """dense3D accepted-state frames (src/dense3d_sequence.rs:412-564) of the
    mixed carrier's state after one step at n^3 (f32 faces and tracer, a
    uniform [0, 1) f64 fraction, the step's f64 pressure): device encode time
    per frame (CUDA events on the encoding stream), the same frames end to end
    through the frame writer (encode, device-to-host copy into pinned memory,
    write(2) to /dev/null), and the oracle's text of one frame on one host
    core."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import dense3d as D

    torch.cuda.set_device(local)
    n = args.n
    g = R.GridGeometry((n, n, n))
    sim = R.CarrierSimulation(g, R.CarrierConfig.mixed(with_tracer=True, device=local))
    sim.init_fourier(seed=args.seed)
    rep = sim.step(R.StepParams(requested_dt=MAXF, cfl=0.5))
    gen = torch.Generator(device=f"cuda:{local}")
    gen.manual_seed(args.seed)
    fraction = torch.rand(g.cell_len(), dtype=torch.float64, device=f"cuda:{local}", generator=gen)
    fields = D.Dense3dFields.from_carrier(sim, fraction=fraction)
    diag = dict(pressure_iterations=rep.pressure.iterations, pressure_residual_m3_s2=rep.pressure.true_residual_max,
                carrier_divergence_s_inv=rep.actual_divergence_max)
    info = D.Dense3dFrameInfo(frame=1, time_s=rep.time, dt_s=rep.dt, carrier_stamp=(1, rep.generation),
                              liquid_stamp=(2, rep.generation), diagnostics=diag)
    enc = D.Dense3dEncoder(g, device=local)
    out = torch.empty(enc.bound(), dtype=torch.uint8, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()
    frames = max(1, args.dense3d_frames)
    for _ in range(3):
        length = enc.encode_into(info, fields, out.data_ptr(), out.numel(), stream.cuda_stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * frames)]
    for k in range(frames):
        ev[2 * k].record(stream)
        length = enc.encode_into(info, fields, out.data_ptr(), out.numel(), stream.cuda_stream)
        ev[2 * k + 1].record(stream)
    torch.cuda.synchronize()
    enc_ms = statistics.median(ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(frames))
    faces_n = sum(g.face_len(a) for a in range(3))
    in_bytes = 4 * (faces_n + g.cell_len()) + 16 * g.cell_len()
    hbm, kind = peaks()
    achieved = (in_bytes + length) / (enc_ms / 1e3) / 1e9
    cpu = {}
    if with_cpu:
        import oracle as O

        oracle_faces, tracer = sim.download(with_tracer=True)
        p = sim.pressure()
        fr = fraction.cpu().numpy()
        t0 = time.perf_counter()
        st, line = O.dense3d_frame_text(O.grid((n, n, n)), frame=1, time_s=rep.time, dt_s=rep.dt,
                                        carrier_stamp=(1, rep.generation), liquid_stamp=(2, rep.generation),
                                        diagnostics=diag, faces=oracle_faces, tracer=tracer, fraction=fr, pressure=p)
        cpu_s = time.perf_counter() - t0
        cpu["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": "frames/s", "cores": 1, "kind": "port",
                               "sample": f"one {n}^3 frame with the oracle's text routine (C library %.*e)"}
        out_host = out[:length].cpu().numpy().tobytes()
        cpu["matches_oracle"] = bool(st == 0 and line == out_host)
    # end to end: the frame writer on /dev/null (frame 0 is the constructor
    # frame); the copies and writes run behind write_frame, flush waits for all
    fd = os.open(os.devnull, os.O_WRONLY)
    w = D.Dense3dFrameWriter(g, fd, D.Dense3dLimits(g.cell_len(), 3 * frames + 2, 1 << 62), device=local)
    w.write_frame(D.Dense3dFrameInfo(carrier_stamp=(1, 0), liquid_stamp=(2, 0)), fields, stream.cuda_stream)
    w.flush()
    t0 = time.perf_counter()
    for k in range(1, frames + 1):
        w.write_frame(D.Dense3dFrameInfo(frame=k, time_s=rep.time, dt_s=rep.dt, carrier_stamp=(1, k),
                                         liquid_stamp=(2, k), diagnostics=diag), fields, stream.cuda_stream)
    w.flush()
    e2e_s = (time.perf_counter() - t0) / frames
    written = w.bytes_written()
    # dataset generation: one accepted mixed step, then its frame, repeatedly,
    # against the same steps without frames
    prm = R.StepParams(requested_dt=MAXF, cfl=0.5)
    sim_stream = sim.stream()
    t0 = time.perf_counter()
    for _ in range(frames):
        sim.step(prm)
    steps_s = (time.perf_counter() - t0) / frames
    t0 = time.perf_counter()
    for k in range(frames + 1, 2 * frames + 1):
        r = sim.step(prm)
        w.write_frame(D.Dense3dFrameInfo(frame=k, time_s=r.time, dt_s=r.dt, carrier_stamp=(1, r.generation),
                                         liquid_stamp=(2, r.generation),
                                         diagnostics=dict(diag, pressure_iterations=r.pressure.iterations)),
                      D.Dense3dFields.from_carrier(sim, fraction=fraction), sim_stream)
    w.flush()
    stream_s = (time.perf_counter() - t0) / frames
    w.close()
    os.close(fd)
    res = {
        "workload": f"dense3D frame of a {n}^3 carrier state: {faces_n + g.cell_len()} f32 values "
                    f"({{:.9e}}) and {2 * g.cell_len()} f64 values ({{:.17e}})",
        "frame_bytes": length,
        "ms_per_frame": enc_ms,
        "value": 1e3 / enc_ms,
        "unit": "frames/s",
        "text_gb_per_s": length / (enc_ms / 1e3) / 1e9,
        "values_per_s": (faces_n + 3 * g.cell_len()) / (enc_ms / 1e3),
        "roofline": {"kernel": "k_d3_measure + k_d3_scan + k_d3_write (one frame)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "peak_kind": kind, "unit": "GB/s", "frac": achieved / hbm,
                     "algorithmic_bytes_per_frame": in_bytes + length,
                     "note": "inputs read once and the text written once per frame; the inputs (L2-sized) are "
                             "read by two passes, the text (> L2) is written once"},
        "e2e": {"value": 1.0 / e2e_s, "unit": "frames/s", "ms_per_frame": e2e_s * 1e3,
                "d2h_bytes_per_frame": written // (frames + 1), "h2d_bytes_per_frame": 0,
                "sink": "write(2) to /dev/null after a device-to-host copy into pinned memory"},
        "step_and_frame": {"ms_per_step_with_frame": stream_s * 1e3, "ms_per_step_alone": steps_s * 1e3,
                           "steps": frames, "carrier": f"mixed, {n}^3, CFL 0.5"},
    }
    res.update(cpu)
    sim.close()
    return res


def run_liquid(args, local, with_cpu):
    """Liquid-volume transport (src/liquid_volume.rs:520-776) at n^3: a ball of
    represented liquid (0.875 occupancy, radius n/4) moved through the
    corrected faces of one mixed-carrier step. Device time of one interval
    (CUDA events on the launching stream), the liquid step against the plain
    mixed step, and the oracle's interval on one host core."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import liquid as L

    torch.cuda.set_device(local)
    n = args.n
    g = R.GridGeometry((n, n, n))
    sim = R.CarrierSimulation(g, R.CarrierConfig.mixed(device=local))
    sim.init_fourier(seed=args.seed)
    rep = sim.step(R.StepParams(requested_dt=MAXF, cfl=0.5))
    zz, yy, xx = np.meshgrid(*[np.arange(n) + 0.5] * 3, indexing="ij")
    r = np.sqrt((xx - n / 2) ** 2 + (yy - n / 2) ** 2 + (zz - n / 2) ** 2)
    fraction = (0.875 * np.clip(n / 4 + 0.5 - r, 0.0, 1.0)).reshape(-1)
    st = L.LiquidVolumeState(g, 800.0, (41, 0), fraction, device=local)
    u, v, w, _ = sim.state_device_ptrs()
    host_faces = sim.download() if with_cpu else None
    inlet = L.LiquidInlet((4, 0), [[0.0, 0.0]] * 3)
    settings = L.LiquidVolumeSettings(1.0, 1e-2)
    stream = torch.cuda.current_stream()
    for _ in range(3):
        st.advance([u, v, w], st.time, rep.dt, (43, 1), inlet, settings, stream=stream.cuda_stream)
    k = max(5, args.steps)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * k)]
    for i in range(k):
        ev[2 * i].record(stream)
        st.advance([u, v, w], st.time, rep.dt, (43, 1), inlet, settings, stream=stream.cuda_stream)
        ev[2 * i + 1].record(stream)
    torch.cuda.synchronize()
    ms = statistics.median(ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(k))
    cells = g.cell_len()
    faces = sum(g.face_len(a) for a in range(3))
    algo = 16 * cells + 4 * faces  # fraction read and written, f32 faces read
    hbm, kind = peaks()
    res = {
        "workload": f"liquid-volume interval at {n}^3 through a mixed-carrier step's corrected faces",
        "ms_per_interval": ms,
        "value": cells / (ms / 1e3),
        "unit": "cell-intervals/s",
        "roofline": {"kernel": "k_liquid_advance (one interval, with its decision)", "bound": "hbm",
                     "achieved": algo / (ms / 1e3) / 1e9, "peak": hbm, "peak_kind": kind, "unit": "GB/s",
                     "frac": algo / (ms / 1e3) / 1e9 / hbm, "algorithmic_bytes_per_interval": algo,
                     "note": "the interval's event time includes the input upload, the commit kernel and the "
                             "report read-back of the standalone call"},
    }
    # the liquid step: the transport inside the mixed carrier's step graph
    sim2 = R.CarrierSimulation(g, R.CarrierConfig.mixed(device=local))
    sim2.init_fourier(seed=args.seed)
    lts = L.LiquidTransportSimulation(sim2, 800.0, (41, 0), fraction, flow_id=43)
    prm = R.StepParams(requested_dt=MAXF, cfl=0.5)
    for _ in range(2):
        lts.step(prm, inlet, settings)
        sim.step(prm)
    steps = max(5, args.steps)
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step(prm)
    plain = (time.perf_counter() - t0) / steps
    t0 = time.perf_counter()
    for _ in range(steps):
        lr = lts.step(prm, inlet, settings)
    with_liquid = (time.perf_counter() - t0) / steps
    res["liquid_step"] = {"ms_per_step": with_liquid * 1e3, "ms_per_mixed_step_alone": plain * 1e3,
                          "liquid_volume_after": lr.liquid.liquid_volume_after,
                          "volume_balance_error": lr.liquid.volume_balance_error}
    if with_cpu:
        import oracle as O

        t0 = time.perf_counter()
        err, _, _ = O.liquid_advance(O.grid((n, n, n)), 800.0, fraction, host_faces, 0.0, rep.dt, inlet.fraction,
                                     actual_divergence_limit=1e-2)
        cpu_s = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": cells / cpu_s, "unit": "cell-intervals/s", "cores": 1, "kind": "port",
                               "sample": f"one {n}^3 interval of the oracle ({err})"}
    sim.close()
    sim2.close()
    return res


def run_box_flux(args, local, with_cpu):
    """Box-flux projection (src/box_flux.rs:213-397) at n^3 on the unit cube: a
    seeded random-Fourier provisional field with a 0.5 m/s through-flow along
    x imposed on the sides, projected with the reference's default pressure
    method (Jacobi-PCG) and with the mixed-precision multigrid. Device time of
    a whole projection (CUDA events on the workspace's stream, host polls of
    the solve included), the fused passes' own times inside it, the same call
    on pinned host arrays, and the oracle's projection on one host core."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import box_flux as B
    from rheon_b200 import workloads as W

    torch.cuda.set_device(local)
    n = args.n
    counts, spacing = (n, n, n), (1.0 / n,) * 3
    g = R.GridGeometry(counts, spacing)
    old_h = W.fourier_faces(counts, seed=args.seed, dtype=np.float32)
    old = [torch.from_numpy(f).cuda() for f in old_h]
    out = [torch.empty_like(f) for f in old]
    bc = B.PrescribedBoxFlux(B.BoxFluxStamp(1, 0), [[-0.5, 0.5], [0.0, 0.0], [0.0, 0.0]])
    settings = B.BoxFluxSettings(R.PressureSettings(1e-8, 0.0, MAXF, 1000000), 1.0)
    dt = 1e-3
    cells = g.cell_len()
    faces = sum(g.face_len(a) for a in range(3))
    hbm, kind = peaks()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > 126 MB L2
    res = {"workload": f"box-flux projection at {n}^3, x through-flow 0.5 m/s on a random-Fourier field, "
                       f"Jacobi-PCG (rel 1e-8)",
           "unit": "cell-projections/s"}
    k = max(3, args.steps)
    for name, method in (("jacobi_pcg_v1", R.PressureImplementation.JACOBI_PCG_V1),
                         ("mg_mixed", R.PressureImplementation.MG_MIXED)):
        w = B.BoxFluxWorkspace(g, 1.0, 1 << 40, method, device=local)
        stream = torch.cuda.ExternalStream(w.stream(), device=local)
        for _ in range(3):
            r = w.project(old, dt, bc, settings, out)
        times, rhs_ms, cor_ms = [], [], []
        for _ in range(k):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = w.project(old, dt, bc, settings, out)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            a, b = w.last_pass_ms()
            rhs_ms.append(a)
            cor_ms.append(b)
        ms = statistics.median(times)
        leg = {"ms_per_projection": ms, "value": cells / (ms / 1e3), "pcg_iterations": r.pressure.iterations,
               "actual_divergence_max": r.actual_divergence_max, "budget_error": r.work.budget_error,
               "kinetic_before": r.work.kinetic_before, "kinetic_after": r.work.kinetic_after,
               "rhs_pass_ms": statistics.median(rhs_ms), "correction_pass_ms": statistics.median(cor_ms)}
        if name == "jacobi_pcg_v1":
            res.update(value=leg["value"], ms_per_projection=ms)
            # k_bf_correct: f32 old faces read, f32 output written, f64 pressure read
            algo = 8 * faces + 8 * cells
            cm = leg["correction_pass_ms"]
            res["roofline"] = {"kernel": "k_bf_correct (correction, stored divergence, energy ledger)",
                               "bound": "hbm", "achieved": algo / (cm / 1e3) / 1e9, "peak": hbm, "peak_kind": kind,
                               "unit": "GB/s", "frac": algo / (cm / 1e3) / 1e9 / hbm,
                               "algorithmic_bytes_per_launch": algo, "avg_launch_ms": cm,
                               "rhs_pass": {"kernel": "k_bf_rhs", "algorithmic_bytes": 4 * faces + 8 * cells,
                                            "ms": leg["rhs_pass_ms"],
                                            "achieved": (4 * faces + 8 * cells) / (leg["rhs_pass_ms"] / 1e3) / 1e9},
                               "note": "both passes timed inside the projection (CUDA events on the workspace's "
                                       "stream); the pressure solve is the rest of the projection"}
        res[name] = leg
        if name == "jacobi_pcg_v1":
            # the same call on pinned host arrays: faces copied in and the output out
            hin = [torch.from_numpy(f).pin_memory() for f in old_h]
            hout = [torch.empty(f.size, dtype=torch.float32).pin_memory() for f in old_h]
            hin_np, hout_np = [t.numpy() for t in hin], [t.numpy() for t in hout]
            w.project(hin_np, dt, bc, settings, hout_np)
            t0 = time.perf_counter()
            for _ in range(k):
                w.project(hin_np, dt, bc, settings, hout_np)
            e2e = (time.perf_counter() - t0) / k
            same = all(np.array_equal(hout_np[a], out[a].cpu().numpy()) for a in range(3))
            res["e2e"] = {"value": cells / e2e, "unit": "cell-projections/s", "h2d_bytes_per_step": 4 * faces,
                          "d2h_bytes_per_step": 4 * faces, "ms_per_projection": e2e * 1e3,
                          "matches_device_path": same}
        w.close()
    res["box_flux_step"] = run_box_flux_step(args, local, with_cpu)
    if with_cpu:
        import oracle as O

        m = min(n, 64)
        og = O.grid((m, m, m), (1.0 / m,) * 3)
        ofaces = W.fourier_faces((m, m, m), seed=args.seed, dtype=np.float32)
        t0 = time.perf_counter()
        st, _, _, rep = O.box_flux_project(og, 1.0, O.JACOBI_PCG_V1, ofaces, dt, [[-0.5, 0.5], [0.0, 0.0],
                                                                                  [0.0, 0.0]],
                                           O.settings(1e-8, 0.0, MAXF, 1000000), 1.0)
        cpu_s = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": m ** 3 / cpu_s, "unit": "cell-projections/s", "cores": 1, "kind": "port",
                               "sample": f"one full {m}^3 projection of the same workload by the oracle "
                                         f"({rep['iterations']} PCG iterations, status {st}); the per-cell cost "
                                         f"grows with n (iterations), so this overstates the CPU at {n}^3"}
    return res


def run_box_flux_step(args, local, with_cpu):
    """Simulation::step_with_box_flux (src/simulation.rs:551-579) on the resident
    carrier at n^3 on the unit cube: the random-Fourier state, a smoke source in
    the box's centre, a uniform body force and a 0.5 m/s x through-flow, on the
    mixed carrier (FP32 multigrid) and the f32 Jacobi-PCG carrier (rel 1e-8).
    Wall time per step (the step is host-driven and synchronous), and the
    oracle's step on one host core."""
    import torch

    import rheon_b200 as R
    from rheon_b200 import simulation as SS
    from rheon_b200 import workloads as W
    from rheon_b200.box_flux import BoxFluxStamp, PrescribedBoxFlux

    torch.cuda.set_device(local)
    n = args.n
    g = R.GridGeometry((n, n, n), (1.0 / n,) * 3)
    faces = W.fourier_faces((n, n, n), seed=args.seed, dtype=np.float32)
    tracer = np.zeros(g.cell_len(), np.float32)
    src = SS.SmokeSource((0.375, 0.125, 0.375), (0.625, 0.375, 0.625), 0.5, 1.0)
    forces = [SS.BodyForce((0.0, -0.25, 0.0))]
    bnd = SS.BoxFluxStepBoundary(PrescribedBoxFlux(BoxFluxStamp(1, 0), [[-0.5, 0.5], [0.0, 0.0], [0.0, 0.0]]))
    pressure = R.PressureSettings(1e-8, 0.0, MAXF, 1000000)
    res = {"workload": f"box-flux step at {n}^3: random-Fourier state, smoke source, uniform body force, "
                       f"0.5 m/s x through-flow, rel 1e-8", "unit": "cell-steps/s"}
    k = max(3, min(args.steps, 5))
    for name, cfg in (("mg_mixed", R.CarrierConfig.mixed(device=local, with_tracer=True, pressure=pressure,
                                                         actual_divergence_limit=1.0)),
                      ("jacobi_pcg_v1_f32", R.CarrierConfig(storage="f32", device=local, with_tracer=True,
                                                            pressure=pressure, actual_divergence_limit=1.0))):
        sim = R.CarrierSimulation(g, cfg)
        sim.upload(faces, tracer)
        ws = SS.BoxFluxStepWorkspace(g, cfg.density, 1 << 40, cfg.implementation, device=local)
        for _ in range(2):
            SS.step_with_box_flux(sim, 1.0, src, forces, ws, bnd)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k):
            r = SS.step_with_box_flux(sim, 1.0, src, forces, ws, bnd)
        el = (time.perf_counter() - t0) / k
        res[name] = {"ms_per_step": el * 1e3, "value": g.cell_len() / el, "dt": r.step.dt,
                     "pcg_iterations": r.step.pressure.iterations, "budget_error": r.work.budget_error,
                     "kinetic_accepted": r.work.kinetic_accepted,
                     "actual_divergence_max": r.step.actual_divergence_max}
        ws.close()
        sim.close()
    res["value"] = res["mg_mixed"]["value"]
    if with_cpu:
        import oracle as O

        m = min(n, 32)
        og = O.grid((m, m, m), (1.0 / m,) * 3)
        sim = O.Simulation(og, 1.0, O.JACOBI_PCG_V1, O.settings(1e-8, 0.0, MAXF, 1000000), 1.0, 1.0,
                           W.fourier_faces((m, m, m), seed=args.seed, dtype=np.float32))
        t0 = time.perf_counter()
        st, rep = sim.step(1.0, dict(lower=src.lower, upper=src.upper, tracer_rate=src.tracer_rate,
                                     vertical_acceleration=src.vertical_acceleration),
                           [dict(value=forces[0].value, units=0, region=None)], [[-0.5, 0.5], [0.0, 0.0], [0.0, 0.0]])
        cpu_s = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": m ** 3 / cpu_s, "unit": "cell-steps/s", "cores": 1, "kind": "port",
                               "sample": f"one {m}^3 box-flux step of the same workload by the oracle (Jacobi-PCG, "
                                         f"{rep.pressure.iterations} iterations, status {st}); the per-cell cost "
                                         f"grows with n, so this overstates the CPU at {n}^3"}
    return res


def run_ours(args, world, rank, local):
    import torch

    import rheon_b200 as R
    from rheon_b200 import workloads as W

    torch.cuda.set_device(local)
    n = (args.n,) * 3
    g = R.GridGeometry(n)
    if args.method == "mixed":
        args.storage = "f32"
    dtype = np.float64 if args.storage == "f64" else np.float32
    faces = W.fourier_faces(n, seed=args.seed + rank, dtype=dtype)
    method = {"jacobi": R.PressureImplementation.JACOBI_PCG_V1, "rbsgs": R.PressureImplementation.RBSGS_PCG,
              "sgs": R.PressureImplementation.SGS_PCG_V1, "mixed": R.PressureImplementation.MG_MIXED}[args.method]
    settings = R.PressureSettings(1e-8, 0.0, MAXF, args.max_iters if args.max_iters > 0 else 1000000)
    if args.method == "mixed":
        cfg = R.CarrierConfig.mixed(pressure=settings, device=local)
    else:
        cfg = R.CarrierConfig(pressure=settings, storage=args.storage, implementation=method, device=local,
                              max_courant=1.0)
    sim = R.CarrierSimulation(g, cfg)
    sim.upload(faces)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    prm = R.StepParams(MAXF, cfl=0.5, iteration_limit_ok=args.max_iters > 0)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > 126 MB L2

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    for _ in range(args.warmup):
        sim.step(prm)
    torch.cuda.synchronize()
    barrier()
    clocks = Clocks(local)
    clocks.start()
    total_ms, iters, launches, pressure_ms = 0.0, [], 0, 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)  # L2 flush between timed steps (outside the timed interval)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rep = sim.step(prm)
        b.record(stream)
        b.synchronize()
        total_ms += a.elapsed_time(b)
        iters.append(rep.pressure.iterations)
        launches += rep.kernel_launches
        pressure_ms += rep.pressure_ms
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    # max over ranks
    t = total_ms
    if world > 1:
        import torch.distributed as dist

        tt = torch.tensor([t], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    cells = n[0] * n[1] * n[2]
    value = world * cells * args.steps / (t / 1e3)

    # roofline of the dominant kernel, timed on the carrier's stream on the
    # current vectors. With the persistent Jacobi-PCG kernel (one cooperative
    # launch per chunk of iterations) that kernel is the solve; otherwise the
    # larger of the two PCG passes.
    hbm, hbm_kind = peaks()
    launches_prof = 3 if args.no_profile else 50
    roof_kernel, roof_bytes, roof_ms, other_ms = None, None, None, None
    try:
        iter_ms = sim.profile(2, 4 * launches_prof)
        # algorithmic bytes per Jacobi-PCG iteration of the scope's minimal
        # kernel sequence: apply_A_dot 16N + update_dots 48N + direction 24N =
        # 88N (the persistent kernel's fused phases move 72N of it: phase 1
        # reads z, d_old and writes d_new, phase 2 reads d, p, r and writes
        # p, r, z)
        roof_kernel, roof_bytes, roof_ms = "k_jacobi_persistent (one PCG iteration)", 88 * cells, iter_ms
        other_ms = sim.profile(1, launches_prof) if method != R.PressureImplementation.MG_MIXED else 0.0
    except R.SimulationError:
        pass
    if roof_kernel is None:
        pass_ms = {0: sim.profile(0, launches_prof),
                   1: sim.profile(1, launches_prof) if method != R.PressureImplementation.MG_MIXED else 0.0}
        # algorithmic bytes: pass 1 reads z, d_old and writes d_new (24N); pass 2
        # reads p, d, r and writes p, r, z (48N)
        bytes_pass = {0: 24 * cells, 1: 48 * cells}
        dominant = 1 if pass_ms[1] >= pass_ms[0] else 0
        roof_kernel = ["k_pass1 (PCG pass 1)", "k_pass2 (PCG pass 2)"][dominant]
        roof_bytes, roof_ms, other_ms = bytes_pass[dominant], pass_ms[dominant], pass_ms[1 - dominant]
    achieved = roof_bytes / (roof_ms / 1e3) / 1e9

    # end to end through the public API with host buffers: per step, H2D of the
    # step's input faces from pinned memory, the step, D2H of the corrected faces.
    face_bytes = sum(f.nbytes for f in faces)
    e2e_ms = float("nan") if args.no_e2e else run_e2e(args, g, cfg, faces, prm, flush, local, world)

    variants = {}
    if not args.no_variants and rank == 0 and world == 1:
        mixed_pressure = R.PressureSettings(1e-8, 0.0, MAXF, 1000)
        cases = (
            ("rbsgs_pcg_f64", R.CarrierConfig(pressure=settings, storage=args.storage,
                                              implementation=R.PressureImplementation.RBSGS_PCG, device=local),
             faces),
            ("mixed_mg_f32", R.CarrierConfig.mixed(pressure=mixed_pressure, device=local),
             [f.astype(np.float32) for f in faces]),
            # the plain method with the AcceptedPreviousV1 initialization policy
            ("jacobi_warm_start_f64", R.CarrierConfig(pressure=settings, storage=args.storage,
                                                      implementation=R.PressureImplementation.JACOBI_PCG_V1,
                                                      device=local, warm_start=True), faces),
        )
        for name, vcfg, vfaces in cases:
            if vcfg.implementation == method and vcfg.storage == args.storage and not vcfg.warm_start:
                continue
            vs = R.CarrierSimulation(g, vcfg)
            vs.upload(vfaces)
            vstream = torch.cuda.ExternalStream(vs.stream(), device=local)
            for _ in range(args.warmup):
                vs.step(prm)
            vms, vit, vdiv = 0.0, [], 0.0
            for _ in range(args.steps):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(vstream)
                r = vs.step(prm)
                b.record(vstream)
                b.synchronize()
                vms += a.elapsed_time(b)
                vit.append(r.pressure.iterations)
                vdiv = max(vdiv, r.actual_divergence_max)
            vvalue = cells * args.steps / (vms / 1e3)
            variants[name] = {"value": vvalue, "unit": UNIT, "ms_per_step": vms / args.steps,
                              "iterations_per_step": statistics.mean(vit), "actual_divergence_max": vdiv,
                              "vs_plain_f64": vvalue / value}
            if vcfg.implementation == R.PressureImplementation.MG_MIXED:
                # whole-step roofline under the algorithmic byte model of a
                # mixed outer cycle: an FP32 V(2,2) with levels summed (about
                # 82N) plus the FP64 defect and accumulation (48N) = 130N per
                # outer iteration, and the step's non-iterative traffic
                # (advection, RHS, correction: 5 F s + 16N with s = 4 bytes)
                faces_total = sum(g.face_len(d) for d in range(3))
                step_bytes = statistics.mean(vit) * 130 * cells + 5 * faces_total * 4 + 16 * cells
                ach = step_bytes / (vms / args.steps / 1e3) / 1e9
                variants[name]["roofline"] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                                              "frac": ach / hbm, "bytes_per_step": step_bytes,
                                              "model": "130N per outer iteration + 5Fs + 16N per step"}
            vs.close()

    mixed256 = None
    if not args.no_variants and rank == 0 and world == 1:
        mixed256 = run_mixed_large(args, local, flush, 256)
    batched = None
    if not args.no_batched and rank == 0 and world == 1:
        batched = run_batched(args, local, flush)
    serving = None
    if not args.no_serving and rank == 0 and world == 1:
        serving = run_serving(args, local)

    result = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": args.storage,
        "data": "synthetic (seeded SplitMix64 random-Fourier velocity, host-generated)",
        "config": {
            "workload": WORKLOAD.format(n=args.n, storage=args.storage,
                                        method={"jacobi": "Jacobi-PCG", "rbsgs": "RB-SGS-PCG", "sgs": "SGS-PCG (v1)",
                                                "mixed": "FP32-multigrid FCG"}[args.method]),
            "cells": cells,
            "parallelism": f"replicas x{world} (independent boxes, no collective)",
            "l2": "256 MB buffer written between timed steps; per-step working set > 126 MB L2",
            "pcg_iterations_per_step": statistics.mean(iters),
            "pressure_ms_per_step": pressure_ms / args.steps,
        },
        "gpu_launches": launches,
        "roofline": {
            "kernel": roof_kernel,
            "bound": "hbm",
            "achieved": achieved,
            "peak": hbm,
            "peak_kind": hbm_kind,
            "unit": "GB/s",
            "frac": achieved / hbm,
            # DRAM bytes are not measured inside the bench (ncu replays kernels);
            # the ncu capture of this kernel is summarised under profiles/
            "traffic": None,
            "algorithmic_bytes_per_launch": roof_bytes,
            "avg_launch_ms": roof_ms,
            "other_pass_ms": other_ms,
            "note": "vectors of a 128^3 solve (6 x 16.8 MB) stay resident in the 126 MB L2 across passes",
        },
        "e2e": None if args.no_e2e else {
            "value": world * cells * args.steps / (e2e_ms / 1e3),
            "unit": UNIT,
            "h2d_bytes_per_step": face_bytes,
            "d2h_bytes_per_step": face_bytes,
        },
        "clocks": clk,
    }
    if variants:
        result["variants"] = variants
    # the target comparison in short keys: mixed against plain f64 at the
    # headline size, and the mixed path's HBM fractions (algorithmic bytes)
    target = {}
    if "mixed_mg_f32" in variants:
        target["mixed_vs_plain_f64"] = variants["mixed_mg_f32"]["vs_plain_f64"]
        target["mixed_128_frac"] = variants["mixed_mg_f32"]["roofline"]["frac"]
    if mixed256:
        result["mixed_256"] = mixed256
        target["mixed_256_frac"] = mixed256["roofline"]["frac"]
        target["mixed_256_value"] = mixed256["value"]
    if batched:
        target["batched_frac"] = batched["roofline"]["frac"]
        target["batched_value"] = batched["value"]
        target["batched_vs_plain_f64"] = batched["value"] / value
    if target:
        result["target"] = target
    if batched:
        result["batched"] = batched
    if serving:
        result["serving"] = serving
    sim.close()
    if not args.no_dense3d and world == 1:
        result["dense3d"] = run_dense3d(args, local, with_cpu=not args.no_cpu_baseline)
    if not args.no_liquid and world == 1:
        result["liquid"] = run_liquid(args, local, with_cpu=not args.no_cpu_baseline)
    if not args.no_box_flux and world == 1:
        result["box_flux"] = run_box_flux(args, local, with_cpu=not args.no_cpu_baseline)
    return result


# ------------------------------------------------------------------ CPU arms
def cpu_carrier(args, budget_s, threads, steps_cap, warmup=0, n=None):
    """The oracle carrier step of the bench's workload on host cores.

    Runs `warmup` untimed steps from the initial state, then timed steps until
    `steps_cap` steps or `budget_s` seconds. Returns a dict with the rate
    (cell-steps/s), the timed steps, seconds, PCG iterations per timed step and
    a description of the sample."""
    import oracle as O
    from rheon_b200 import workloads as W

    edge = args.n if n is None else n
    shape = (edge,) * 3
    g = O.grid(shape)
    dtype = np.float64 if args.storage == "f64" else np.float32
    faces = W.fourier_faces(shape, seed=args.seed, dtype=dtype)
    method = O.JACOBI_PCG_V1
    s = O.settings(1e-8, 0.0, MAXF, 1000000)

    def step(faces):
        _, rate = O.velocity_rate(g, faces)
        dt = min(MAXF, 0.5 / rate)
        prm = O.StepParams(dt, 1.0, method, s, 0.0, 0, threads)
        st, faces, _, rep = O.carrier_step(g, faces, prm)
        if st != O.OK:
            raise RuntimeError(f"oracle step failed: {st}")
        return faces, rep

    for _ in range(warmup):
        faces, _ = step(faces)
    done, iters, t0 = 0, [], time.perf_counter()
    while done < max(1, steps_cap):
        faces, rep = step(faces)
        iters.append(rep.pressure.iterations)
        done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    el = time.perf_counter() - t0
    cells = edge ** 3
    sample = (f"steps {warmup + 1}-{warmup + done} of the {edge}^3 workload's trajectory "
              f"({warmup} untimed warm-up step(s) first), {threads} thread(s)")
    return {"value": cells * done / el, "steps": done, "seconds": el, "warmup": warmup,
            "iterations_per_step": statistics.mean(iters), "sample": sample}


def run_reference(args, world, rank):
    """The CPU reference arm: the oracle port of the carrier step on all host
    cores, on the GPU arm's workload, metric and config keys. Each timed step is
    a full step of the same trajectory; the window is bounded (one untimed
    warm-up step, then up to --steps steps or about 150 s), so that the arm
    ends within a few minutes."""
    import oracle

    oracle.lib()
    threads = os.cpu_count() or 1
    r = cpu_carrier(args, budget_s=150.0, threads=threads, steps_cap=args.steps, warmup=min(args.warmup, 1))
    value = r["value"]
    cells = args.n ** 3
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": r["steps"],
        "warmup": r["warmup"],
        "ms_per_step": r["seconds"] * 1e3 / r["steps"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": args.storage,
        "data": "synthetic (seeded SplitMix64 random-Fourier velocity, host-generated)",
        "config": {
            "workload": WORKLOAD.format(n=args.n, storage=args.storage, method="Jacobi-PCG"),
            "cells": cells,
            "parallelism": f"rank 0 of {world} on host cores; replicas x{world} on the GPU arm",
            "l2": "host caches (CPU arm)",
            "pcg_iterations_per_step": r["iterations_per_step"],
            "pressure_ms_per_step": None,
            "step_window": r["sample"],
        },
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": r["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "Rheon is Rust and cannot be built here (no cargo/rustc); this arm times the oracle, a C++ "
                "restatement of its carrier arithmetic (serial Neumaier reductions, threaded stencil loops)",
    }


def relaunch(gpus):
    """`--gpus N` without a torchrun environment: start N ranks on this node
    under torch.distributed.run (rendezvous on 127.0.0.1) with the same
    arguments and return their exit status."""
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "--", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch(args.gpus))
    world, rank, local = dist_env()
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if args.impl == "ours":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device(f"cuda:{local}"))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        ranks = [rank]
        if world > 1:
            import torch.distributed as dist

            ranks = [None] * world
            dist.all_gather_object(ranks, rank)
        if rank == 0:
            line = run_reference(args, world, rank)
            line["ranks_started"] = sorted(ranks)
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.solve_only:
        print(json.dumps(run_solve_only(args, local)), flush=True)
        return
    if args.buoyant_blob:
        print(json.dumps(run_buoyant_blob(args, local)), flush=True)
        return
    if args.advect:
        print(json.dumps(run_advect(args, local)), flush=True)
        return
    if args.batch_profile:
        print(json.dumps(run_batch_profile(args, local)), flush=True)
        return
    if args.dense3d:
        print(json.dumps(run_dense3d(args, local, with_cpu=not args.no_cpu_baseline)), flush=True)
        return
    if args.liquid:
        print(json.dumps(run_liquid(args, local, with_cpu=not args.no_cpu_baseline)), flush=True)
        return
    if args.box_flux:
        print(json.dumps(run_box_flux(args, local, with_cpu=not args.no_cpu_baseline)), flush=True)
        return
    result = run_ours(args, world, rank, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        oracle.lib()
        threads = os.cpu_count() or 1
        r = cpu_carrier(args, budget_s=args.cpu_budget, threads=threads, steps_cap=1)
        result["cpu_baseline"] = {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "port",
                                  "sample": r["sample"], "iterations_per_step": r["iterations_per_step"]}
        # the serial figure: one thread, as the reference's bit-faithful serial
        # run; one step of the 64^3 box (a 128^3 step takes minutes on one core),
        # which understates the per-cell cost of 128^3 (more iterations per step)
        r1 = cpu_carrier(args, budget_s=args.cpu_budget, threads=1, steps_cap=1, n=min(args.n, 64))
        result["cpu_baseline"]["single_thread"] = {"value": r1["value"], "unit": UNIT, "cores": 1,
                                                   "sample": r1["sample"],
                                                   "iterations_per_step": r1["iterations_per_step"]}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
