"""Benchmark: time steps per second of the spectral-Galerkin heat solver on B200.

Default workload ``--workload serving``: a seeded stream of laser-scan solve
requests of uneven size (grids 64x32x16 .. 512x256x64 on the 2 x 1 x 0.5 mm
316L cuboid, straight-track physics = one forcing pass per step, 200-2000
steps of 5 us, random power and speed) served by the continuous-batching
engine in mixed precision (FP32 modal state, split-BF16 tensor-core face
transforms, FP64 face fields, norms and coefficient tables, FP32 face sums).

* ``value``: timesteps/s of the engine on a saturated queue of that mix: all
  requests queued, slots sized from free HBM, K batched steps timed with CUDA
  events (one batched step advances every active request by one time step;
  requests complete and new ones are admitted inside the timed region). Laser
  tables are resident on the device before timing. The modal state in flight
  (GBs) is far larger than L2, so no flush is needed.
* ``e2e``: the same K batched steps through the engine's public API with host
  inputs: each admission copies its laser table host -> device (pinned), each
  completion reads the result surface back, every chunk reads slot status.
* ``latency_ms``: p50 / p99 of completion - arrival for a Poisson stream of
  200 requests at 200 requests/s (host inputs, real time).
* ``comparisons``: the plain FP64 single-instance solver (``B200SpectralSolver``,
  one request at a time) on a sample of the same mix, and the FP64 batched
  engine on the same saturated mix; ``accuracy``: relative L2 of the final
  modes (= of the temperature field, the transform being orthonormal) and the
  peak-temperature error of mixed-precision results against FP64 runs.
* ``roofline``: the volume pass (modal commit fused with the next step's face
  sums), the HBM-bound kernel of this workload, timed alone with CUDA events
  over all active slots.
* ``cpu_baseline``: the CPU oracle (FP64 NumPy/SciPy restatement of the
  reference step, all host threads) on a bounded sample of the same requests.

``--workload raster`` is the full nonlinear FP64 case (128 x 64 x 32 modes,
T-dependent properties, latent heat, evaporation + convection, Picard to
1e-8) through ``B200SpectralSolver``: ``value`` from the device-resident step
graph (``sgh_run``), ``e2e`` through ``step(t, dt)``, the DCT axis pass as the
roofline kernel. ``--workload track`` is the 64 x 32 x 16 straight track.

``--impl reference`` times the CPU implementation alone (rank 0) on the same
workload and prints the same JSON line with ``"impl": "reference"``.

Multi-GPU (``torchrun --nproc-per-node N bench.py --gpus N``): every rank runs
an independent replica on its own seeded stream; there is no collective on the
step path. ``value`` = all ranks' timesteps / max over ranks of the timed seconds.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "timesteps/s"
L2_FLUSH_BYTES = 256 << 20
# dram__bytes_read.sum + dram__bytes_write.sum of the dominant kernel from an
# ncu capture of one launch: the serving volume pass at the benchmark's size
# (288 slots, 467,927,040 active modes) read 1.976 GB and wrote 1.968 GB
# (--cache-control none); traffic scales with the modes of the same class mix.
NCU_VOLUME_TRAFFIC_PER_MODE = (1975895808 + 1967578624) / 467927040
# the raster workload's dominant kernel (k_axis) was captured on the same
# 128x64x32 case: 2.14 MB for one contiguous-axis pass (field resident in L2)
NCU_TRAFFIC_BYTES = 2.14e6
# the box workload's box passes (one reconstruction + one projection) from an
# ncu capture of the same case; None until captured
NCU_BOX_TRAFFIC_BYTES = None


def reduce_over_ranks(times_ms, counts, device="cpu"):
    """Replicas' aggregate: max over ranks of each timed interval (ms) and sum
    over ranks of each work count. The only cross-rank traffic of a run."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x) for x in times_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(x) for x in counts], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return [float(x) for x in t], [int(round(float(x))) for x in c]


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _workload(name, seed):
    from spectral_galerkin_heat_b200 import workloads
    if name == "raster":
        cfg, path = workloads.nonlinear_raster(seed=seed)
        desc = {"workload": "nonlinear_raster_fp64", "modes": [128, 64, 32],
                "domain_mm": [2.0, 1.0, 0.5], "dt_s": 2e-6, "picard_tol": 1e-8,
                "picard_omega": 0.1, "picard_cap": 400, "latent": "grid",
                "properties": "k(T), c_p(T) linear", "surface": "evaporation + convection",
                "path": "5-line raster, 0.4 mm lines, 100 um hatch, 1 m/s", "seed": seed}
    elif name == "box":
        cfg, path = workloads.box_track()
        desc = {"workload": "box_track_fp64", "modes": [80, 48, 120],
                "domain_mm": [0.6, 0.4, 0.15], "dt_s": 5e-6, "latent": "box",
                "box": {"refinement": 2, "size_mm": [0.6, 0.6, 0.07], "cells": [160, 96, 112]},
                "picard": "reference defaults (omega 0.1, tol 1e-4, cap 30)",
                "properties": "constant 316L (293 K)", "surface": "evaporation + bottom convection",
                "path": "straight, 0.4 m/s, 120 W"}
    elif name == "track":
        cfg, path = workloads.straight_track()
        desc = {"workload": "straight_track_fp64", "modes": [64, 32, 16],
                "domain_mm": [2.0, 1.0, 0.5], "dt_s": 5e-6, "picard_cap": 1,
                "picard_omega": 1.0, "surface": "evaporation", "path": "straight, 1 m/s"}
    else:
        raise SystemExit(f"unknown workload {name!r}")
    return cfg, path, desc


def _context(cfg, path):
    import copy

    from spectral_galerkin_heat_b200 import SimulationContext
    ctx = SimulationContext.from_dict(copy.deepcopy(cfg))
    ctx.laser_path = path
    return ctx


class ClockSampler:
    """nvidia-smi clock / throttle sampling in the background (200 ms)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(cfg, path, budget_s=20.0, max_steps=None):
    """Time the CPU oracle (all host threads) on the first steps of the workload."""
    from oracle.sgh_oracle import OracleSolver
    ctx = _context(cfg, path)
    o = OracleSolver(ctx, workers=-1)
    o.initialize()
    dt = ctx.num.dt
    o.step(0.0, dt)  # warm-up (first-call costs)
    n, t0 = 0, time.perf_counter()
    while True:
        o.step((n + 1) * dt, dt)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_steps is not None and n >= max_steps):
            break
    return n / el, n, el


def _expected_slot_shares(stream, max_slots):
    """Per-class step shares of a saturated engine whose memory budget does not
    bind: the engine's slot allocation (one slot per class, then to the class
    with the fewest slots per unit of demand, up to ``max_slots`` each), every
    slot stepping once per batched step."""
    weights = {}
    for r in stream:
        weights[r["mesh"]] = weights.get(r["mesh"], 1.0) + r["steps"]
    slots = {k: 1 for k in weights}
    while True:
        cand = [k for k in weights if slots[k] < max_slots]
        if not cand:
            break
        k = min(cand, key=lambda c: slots[c] / weights[c])
        slots[k] += 1
    return _shares(slots)


def run_reference(args, rank, world):
    """--impl reference: the CPU implementation alone, rank 0 only."""
    if rank != 0:
        return None
    if args.workload == "serving":
        from spectral_galerkin_heat_b200 import workloads
        stream = workloads.serving_stream(n_requests=args.requests, seed=0)
        budget = float(os.environ.get("SGH_REFERENCE_BUDGET_S", "180"))
        shares = _expected_slot_shares(stream, args.max_slots)
        rates, n, el = _oracle_classes(stream, budget, max(args.steps, 1))
        v = _mix_rate(rates, shares)
        sample = (f"{n} timesteps in {el:.1f} s: the first request of each of the {len(rates)} grid "
                  f"classes for <= {max(args.steps, 1)} steps (after one untimed step), weighted by "
                  f"the saturated engine's per-class step shares (its slot allocation)")
        return {
            "metric": METRIC, "value": v, "unit": "timesteps/s", "impl": "reference",
            "n_gpus": world, "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": _serving_desc(args),
            "cpu_baseline": {"value": v, "unit": "timesteps/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": sample,
                             "per_class": {_class_key(k): r for k, r in sorted(rates.items())},
                             "class_step_shares": {_class_key(k): round(x, 4) for k, x in sorted(shares.items())}},
            "e2e": {"value": v, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    cfg, path, desc = _workload(args.workload, seed=0)
    from oracle.sgh_oracle import OracleSolver
    ctx = _context(cfg, path)
    o = OracleSolver(ctx, workers=-1)
    o.initialize()
    dt = ctx.num.dt
    for i in range(args.warmup):
        o.step(i * dt, dt)
    budget = float(os.environ.get("SGH_REFERENCE_BUDGET_S", "180"))
    n, t0 = 0, time.perf_counter()
    for i in range(args.steps):
        o.step((args.warmup + i) * dt, dt)
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    v = n / el
    cores = os.cpu_count()
    sample = (f"{n} of {args.steps} requested steps after {args.warmup} warm-up steps "
              f"(time budget {budget:.0f} s)")
    return {
        "metric": METRIC, "value": v, "unit": "steps/s", "impl": "reference",
        "n_gpus": world, "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": desc,
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_b200(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from spectral_galerkin_heat_b200 import B200SpectralSolver, _lib
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cfg, path, desc = _workload(args.workload, seed=rank)
    K, W = args.steps, args.warmup
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    # ---- device-resident throughput -----------------------------------------
    s = B200SpectralSolver(None, _context(cfg, path), axis_cuda_cores=True if args.axis_cuda_cores else None)
    s.initialize()
    table = s.laser_table(0.0, W + K)
    osz = C.sizeof(_lib.SghStepOut)
    outs = torch.zeros((W + K) * osz, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    s.run_table(table, outs, W, start=0)
    stream.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(K)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for i in range(K):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            s.run_table(table, outs, 1, start=W + i)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = clk.summary()
    dev_ms = sum(a.elapsed_time(b) for a, b in ev)
    recs = s.decode_outs(outs.cpu().numpy().tobytes(), W + K)[W:]
    iters = [r.n_iter for r in recs]
    pre, per_it, post = s.launch_counts()
    launches = sum(pre + post + n * per_it for n in iters)
    statuses = sorted({_lib.STEP_STATUS.get(r.status, r.status) for r in recs})

    if args.workload == "box":
        roof = _box_roofline(s, flush, stream, dev)
        s.finalize()
    else:
        roof = _axis_roofline(s, flush, stream, dev)
        s.finalize()

    # ---- end to end through the public API ----------------------------------
    e = B200SpectralSolver(None, _context(cfg, path), axis_cuda_cores=True if args.axis_cuda_cores else None)
    e.initialize()
    dt = e.context.num.dt
    for i in range(W):
        e.step(i * dt, dt)
    eev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(K)]
    for i in range(K):
        flush.fill_(i & 0xFF)
        eev[i][0].record(stream)
        e.step((W + i) * dt, dt)
        eev[i][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in eev)
    e.finalize()

    # ---- aggregate over ranks -------------------------------------------------
    t_max = dev_ms
    e2e_max = e2e_ms
    if world > 1:
        (t_max, e2e_max), _ = reduce_over_ranks([dev_ms, e2e_ms], [K], device=dev)
    if rank != 0:
        return None
    total_steps = K * world
    line = {
        "metric": METRIC, "value": total_steps / (t_max * 1e-3), "unit": "steps/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": t_max / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded laser path; no dataset)",
        "config": dict(desc, parallelism=f"replicas x{world}" if world > 1 else "single",
                       l2="flushed between timed steps (256 MB write)",
                       axis_kernels="CUDA-core FP64" if args.axis_cuda_cores
                       else "autotuner table per shape: FP64 tensor cores (mma.sync .f64) where the "
                            "pass is large enough, or CUDA cores",
                       picard_iters_mean=float(np.mean(iters)), step_status=statuses),
        "clocks": clocks,
        "gpu_launches": launches * world,
        "e2e": {"value": total_steps / (e2e_max * 1e-3), "unit": "steps/s",
                "h2d_bytes_per_step": C.sizeof(_lib.SghLaser),
                "d2h_bytes_per_step": C.sizeof(_lib.SghStepOut),
                "api": "B200SpectralSolver.step(t, dt)"},
        "roofline": roof,
    }
    if args.workload in ("raster", "box") and not args.no_mixed:
        mixed = _mixed_volume_comparison(args, cfg, path, dev, flush)
        mixed["mixed_over_fp64"] = mixed["mixed_tol"]["value"] / line["value"]
        mixed["mixed_over_fp64_same_tol"] = mixed["mixed_tol"]["value"] / mixed["fp64_at_mixed_tol"]["value"]
        line["comparisons"] = {"mixed_precision": mixed}
    if world == 1 and not args.no_cpu_baseline:
        v, n, el = cpu_baseline(cfg, path, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": v, "unit": "steps/s", "cores": os.cpu_count(),
                                "kind": "port",
                                "sample": f"{n} steps from t=dt of the same workload "
                                          f"({el:.1f} s), after 1 warm-up step"}
    return line


def _mixed_volume_comparison(args, cfg, path, dev, flush):
    """The mixed-precision form of the same single-instance step (split-BF16
    tcgen05 contractions, FP32 modal iterates, FP64 latent source, property
    correction, fluxes and norms) beside the FP64 plan: throughput from the
    step graph (L2 flushed between steps, as for ``value``) at the mixed
    Picard tolerance and, for a few steps, at the FP64 one; and the error of
    its fields against FP64 after ``--mixed-error-steps`` steps (relative L2
    of the volume field, peak temperature, nodal melt-pool extents)."""
    import copy
    import ctypes as C

    import torch

    from spectral_galerkin_heat_b200 import B200SpectralSolver, _lib, kernels
    from spectral_galerkin_heat_b200.precision import compare_fields
    stream = torch.cuda.current_stream(dev)

    def timed(tol, steps, precision="mixed"):
        s = B200SpectralSolver(None, _context(cfg, path), precision=precision, convergence_tol=tol)
        s.initialize()
        W = args.warmup
        table = s.laser_table(0.0, W + steps)
        outs = torch.zeros((W + steps) * C.sizeof(_lib.SghStepOut), dtype=torch.uint8, device=dev)
        s.run_table(table, outs, W, start=0)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        torch.cuda.synchronize()
        for i in range(steps):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            s.run_table(table, outs, 1, start=W + i)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        recs = s.decode_outs(outs.cpu().numpy().tobytes(), W + steps)[W:]
        s.finalize()
        st = sorted({_lib.STEP_STATUS.get(r.status, r.status) for r in recs})
        return {"value": steps / (ms * 1e-3), "unit": "steps/s", "steps": steps, "picard_tol": tol,
                "picard_iters_mean": float(np.mean([r.n_iter for r in recs])), "step_status": st}

    # the mixed plan at its tolerance and at the FP64 one, and the FP64 plan at
    # the mixed tolerance (the like-for-like rate: most of the mixed error
    # against FP64 at 1e-8 is the looser tolerance, which FP64 at that
    # tolerance shares)
    out = {"mixed_tol": timed(args.mixed_tol, args.steps),
           "fp64_tol": timed(float(cfg["simulation"].get("picard_tol", 1e-4)), min(args.steps, 3)),
           "fp64_at_mixed_tol": timed(args.mixed_tol, args.steps, precision="fp64")}
    n = args.mixed_error_steps
    f64 = B200SpectralSolver(None, _context(cfg, path))
    f64.initialize()
    mix = B200SpectralSolver(None, _context(cfg, path), precision="mixed", convergence_tol=args.mixed_tol)
    mix.initialize()
    f64.run(0.0, n)
    mm = mix.run(0.0, n)
    T64 = f64.volume_temperature().cpu().numpy()
    Tmx = f64.volume_temperature(mix.state.a).cpu().numpy()   # FP64 reconstruction of the mixed modes
    g = f64.context.geom
    lengths = (float(g.size.x), float(g.size.y), float(g.size.z))
    geo = type("G", (), {"size": lengths})
    n64 = kernels.reconstruct_temperature_DCT(f64.state.a, geo).cpu().numpy()
    nmx = kernels.reconstruct_temperature_DCT(mix.state.a.clone(), geo).cpu().numpy()
    cell = tuple(L / m for L, m in zip(lengths, (g.n.x, g.n.y, g.n.z)))
    rep = compare_fields(Tmx, T64, cell, float(f64.context.mat.T_liquidus), nmx, n64, lengths)
    out["error_vs_fp64"] = dict(rep, steps=n, mixed_picard_tol=args.mixed_tol,
                                mixed_status_last=mix.last_status,
                                mixed_picard_iters_last=int(mm[-1]["n_evap_iter"]))
    f64.finalize()
    mix.finalize()
    return out


def _fp64_peak(dev, n=4096, reps=10):
    """Measured FP64 matrix peak of this GPU: cuBLAS DGEMM (torch.matmul on
    float64) of n^3, best of ``reps``, CUDA events; TFLOP/s."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    c = torch.matmul(a, b)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def _box_roofline(s, flush, stream, dev):
    """The box passes (reconstruction z, x, y and projection y, x, z of the
    latent source; FP64 contractions, compute-bound) timed alone with CUDA
    events at the window of the last step, against the measured DGEMM peak."""
    import ctypes as C

    import torch

    from spectral_galerkin_heat_b200 import _lib
    fm = s.state.fine_mesh
    nz, ny, nx = s.state.shape
    zb, yb, xb = fm.box_shape
    S = nx * ny
    # multiply-adds of one reconstruction in the pass order z, x, y (a projection
    # is the same contraction in reverse)
    fma = nz * S * zb + zb * ny * nx * xb + zb * ny * xb * yb
    flops = 2.0 * 2 * fma
    a = torch.randn(s.state.shape, dtype=torch.float64, device=dev)
    box = torch.empty(fm.box_shape, dtype=torch.float64, device=dev)
    modes = torch.empty_like(a)
    R = 20
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(R)]
    L = _lib.lib()
    for i in range(R + 2):
        flush.fill_(i & 0xFF)
        if i >= 2:
            ev[i - 2][0].record(stream)
        _lib.check("sgh_box_temperature", L.sgh_box_temperature(
            s._plan, C.c_void_p(a.data_ptr()), C.c_void_p(box.data_ptr()), C.c_void_p(stream.cuda_stream)))
        _lib.check("sgh_box_project", L.sgh_box_project(
            s._plan, C.c_void_p(box.data_ptr()), C.c_void_p(modes.data_ptr()), C.c_void_p(stream.cuda_stream)))
        if i >= 2:
            ev[i - 2][1].record(stream)
    torch.cuda.synchronize()
    ms = sum(x.elapsed_time(y) for x, y in ev) / R
    achieved = flops / (ms * 1e-3) / 1e12
    peak = _fp64_peak(dev)
    return {"kernel": "k_axis box passes (reconstruction + projection, FP64)", "bound": "fp64",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "measured here: cuBLAS DGEMM 4096^3, best of 10",
            "traffic": NCU_BOX_TRAFFIC_BYTES, "algorithmic_flops_per_launch": flops,
            "launches": 6, "ms_per_pair": ms,
            # bytes each pass reads and writes once, both directions
            "hbm_gbs_algorithmic": 8.0 * 2 * (nz * S + 2 * zb * S + 2 * zb * ny * xb + zb * yb * xb)
            / (ms * 1e-3) / 1e9}


def _axis_roofline(s, flush, stream, dev):
    """DCT axis passes of one 3-D transform, timed alone (HBM-bound)."""
    import ctypes as C

    import torch

    from spectral_galerkin_heat_b200 import _lib
    R = 20
    src = torch.randn(s.state.shape, dtype=torch.float64, device=dev)
    dst = torch.empty_like(src)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(R)]
    for i in range(R + 2):
        flush.fill_(i & 0xFF)
        if i >= 2:
            kev[i - 2][0].record(stream)
        _lib.check("sgh_dct3d", _lib.lib().sgh_dct3d(
            s._plan, 3, C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()),
            C.c_void_p(stream.cuda_stream)))
        if i >= 2:
            kev[i - 2][1].record(stream)
    torch.cuda.synchronize()
    per_transform_ms = sum(a.elapsed_time(b) for a, b in kev) / R
    nz, ny, nx = s.state.shape
    V = nx * ny * nz
    # algorithmic bytes of one axis pass: read the field once, write it once (FP64)
    bytes_per_pass = 2 * V * 8
    achieved_gbs = bytes_per_pass / (per_transform_ms / 3 * 1e-3) / 1e9
    hbm, hbm_kind = _peaks()
    # the field (V doubles) sits in L2 at these sizes: the passes are bound by
    # their FP64 contraction work, reported against the measured DGEMM peak
    flops = 2.0 * V * (nx + ny + nz)
    achieved = flops / (per_transform_ms * 1e-3) / 1e12
    peak = _fp64_peak(dev)
    return {"kernel": "k_axis / k_axis_mma (3 DCT axis passes, FP64)", "bound": "fp64",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "measured here: cuBLAS DGEMM 4096^3, best of 10",
            "traffic": NCU_TRAFFIC_BYTES, "algorithmic_flops_per_launch": flops / 3,
            "ms_per_transform": per_transform_ms,
            "hbm_gbs_algorithmic": achieved_gbs, "hbm_peak": hbm, "hbm_peak_source": hbm_kind,
            "algorithmic_bytes_per_launch": bytes_per_pass}


def _serving_desc(args):
    return {"workload": "serving_stream", "grids": "Nx in {64,128,256,512}, Ny=Nx/2, Nz in {16,32,64}",
            "domain_mm": [2.0, 1.0, 0.5], "dt_s": 5e-6, "steps_per_request": [200, 2000],
            "physics": "316L constant properties, evaporation on the top face, one forcing pass per step",
            "laser": "P~U[150,400] W, v~U[0.5,2] m/s, raster 1.5 mm lines / 50 um hatch",
            "saturated_requests": args.requests, "poisson_requests": 200, "arrival_rate_per_s": 200.0}


def _serving_requests(stream, templates, device_tables=None):
    import copy

    from spectral_galerkin_heat_b200.laser import laser_table
    from spectral_galerkin_heat_b200.serving import Request
    out = []
    for r in stream:
        ctx = copy.copy(templates[r["mesh"]])
        ctx.laser_path = r["path"]
        q = Request(id=r["id"], key=r["mesh"], context=ctx, steps=r["steps"], arrival=r["arrival"])
        q.table = laser_table(r["path"], 0.0, float(ctx.num.dt), r["steps"])
        if device_tables is not None:
            q.table = device_tables(q.table)
        out.append(q)
    return out


def _serve_saturated(eng, stream, templates, K, host_io, stagger):
    """K batched steps of a saturated queue in steady state.

    The queue first runs ``stagger`` batched steps untimed from empty slots,
    so the slots hold requests at staggered progress (requests complete and
    new ones are admitted all along); the timed K steps continue that run.
    Returns a dict: ms, slot_steps, h2d, d2h, launches, completed, admitted and
    the slot-steps per grid class of the timed region."""
    import torch
    reqs = _serving_requests(stream, templates, None if host_io else eng.batch.upload_table)
    eng.run(reqs, realtime=False, max_steps=stagger)
    rest = [r for r in reqs if r.status == "queued"]
    if len(rest) < eng.memory["slots"]:
        raise RuntimeError("the saturated stream ran dry during the staggered start; raise --requests")
    torch.cuda.synchronize()
    st = eng.stats
    st0 = (st.slot_steps, st.h2d_bytes, st.d2h_bytes, st.launches, st.completed, st.admitted,
           dict(st.class_steps))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(eng.batch.stream)
    eng.run(rest, realtime=False, max_steps=K)
    b.record(eng.batch.stream)
    torch.cuda.synchronize()
    if eng.batch.tensor_core_error():
        raise RuntimeError("a tensor-core wait ran out during the timed region")
    out = {"ms": a.elapsed_time(b), "slot_steps": st.slot_steps - st0[0], "h2d": st.h2d_bytes - st0[1],
           "d2h": st.d2h_bytes - st0[2], "launches": st.launches - st0[3],
           "completed": st.completed - st0[4], "admitted": st.admitted - st0[5],
           "class_steps": {k: v - st0[6].get(k, 0) for k, v in st.class_steps.items()
                           if v - st0[6].get(k, 0) > 0}}
    if sum(out["class_steps"].values()) != out["slot_steps"]:
        raise RuntimeError("per-class step accounting does not add up")
    eng.reset()
    return out


def _shares(steps_by_class):
    tot = float(sum(steps_by_class.values()))
    return {k: v / tot for k, v in steps_by_class.items()}


def _mix_rate(rates, shares):
    """Timesteps/s of a mix that spends ``shares[c]`` of its steps in class c,
    each class at ``rates[c]`` timesteps/s (total steps over total time)."""
    return 1.0 / sum(sh / rates[c] for c, sh in shares.items())


def _volume_pass_bytes(modes, faces, precision):
    """Algorithmic bytes of one batch volume pass (the modal commit fused with
    the next step's face sums). Mixed: a in and out (FP32; K and KK formed from
    1-D tables), per face column sigma in (FP64) and Zt, Yt out (FP32). FP64:
    a, K, KK in and a out, sigma in and Zt, Yt out, all FP64."""
    if precision == "mixed":
        return 8 * modes + 16 * faces
    return 32 * modes + 24 * faces


def _demand_shares(stream):
    """Per-class share of the timesteps the stream asks for."""
    d = {}
    for r in stream:
        d[r["mesh"]] = d.get(r["mesh"], 0) + r["steps"]
    return _shares(d)


def _plain_fp64_classes(stream, templates, n_steps):
    """The plain FP64 single-instance solver on the first request of every grid
    class, ``n_steps`` steps each from the device step graph (CUDA events,
    plan set-up excluded): ({class: timesteps/s}, steps)."""
    import copy

    import torch

    from spectral_galerkin_heat_b200 import B200SpectralSolver
    rates, total = {}, 0
    for m in sorted({r["mesh"] for r in stream}):
        r = next(q for q in stream if q["mesh"] == m)
        c = copy.copy(templates[m])
        c.laser_path = r["path"]
        s = B200SpectralSolver(None, c)
        s.initialize()
        n = min(r["steps"], n_steps)
        table = s.laser_table(0.0, n + 2)
        outs = torch.zeros((n + 2) * 64, dtype=torch.uint8, device="cuda")
        s.run_table(table, outs, 2, start=0)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s.run_table(table, outs, n, start=2)
        b.record()
        torch.cuda.synchronize()
        rates[m] = n / (a.elapsed_time(b) * 1e-3)
        total += n
        s.finalize()
    return rates, total


def _oracle_classes(stream, budget_s, max_steps, workers=-1):
    """The CPU oracle on the first request of every grid class for at most
    ``max_steps`` steps or ``budget_s / classes`` seconds, after one untimed
    step; ``workers`` threads for its transforms (-1: all host threads):
    ({class: timesteps/s}, steps, seconds)."""
    from oracle.sgh_oracle import OracleSolver
    from spectral_galerkin_heat_b200 import workloads
    classes = sorted({r["mesh"] for r in stream})
    rates, n_tot, el_tot = {}, 0, 0.0
    for m in classes:
        r = next(q for q in stream if q["mesh"] == m)
        ctx = _context(workloads.serving_config(*m), r["path"])
        o = OracleSolver(ctx, workers=workers)
        o.initialize()
        dt = ctx.num.dt
        o.step(0.0, dt)
        n, el = 0, 0.0
        while n < min(max_steps, r["steps"] - 1):
            t0 = time.perf_counter()
            o.step((n + 1) * dt, dt)
            el += time.perf_counter() - t0
            n += 1
            if el >= budget_s / len(classes):
                break
        rates[m] = n / el
        n_tot += n
        el_tot += el
    return rates, n_tot, el_tot


def _class_key(m):
    return "x".join(map(str, m))


def run_serving(args, rank, world, local_rank):
    import copy

    import torch

    from spectral_galerkin_heat_b200 import B200SpectralSolver, workloads
    from spectral_galerkin_heat_b200.precision import run_study
    from spectral_galerkin_heat_b200.serving import Request, ServingEngine, latency_percentiles
    torch.cuda.set_device(local_rank)
    K, W = args.steps, args.warmup
    sat = workloads.serving_stream(n_requests=args.requests, seed=1000 * rank)
    poisson = workloads.serving_stream(n_requests=200, seed=1000 * rank + 1, rate=200.0)
    meshes = sorted({r["mesh"] for r in sat} | {r["mesh"] for r in poisson})
    templates = {m: _context(workloads.serving_config(*m), None) for m in meshes}
    weights = {m: float(sum(r["steps"] for r in sat if r["mesh"] == m)) + 1.0 for m in meshes}
    stagger = args.stagger_steps

    def engine(prec, keep=False):
        eng = ServingEngine(templates, precision=prec, memory_fraction=args.memory_fraction,
                            max_slots=args.max_slots, weights=weights, keep_modes=keep, lanes=args.lanes)
        warm = []
        for i, m in enumerate(meshes):  # W batched steps, every class once
            c = copy.copy(templates[m])
            c.laser_path = sat[0]["path"]
            warm.append(Request(id=-1 - i, key=m, context=c, steps=W))
        eng.run(warm, realtime=False)
        eng.reset()
        return eng

    # ---- mixed precision: the product ---------------------------------------
    eng = engine("mixed")
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local_rank) as clk:
        dev = _serve_saturated(eng, sat, templates, K, host_io=False, stagger=stagger)
    clocks = clk.summary()
    e2e = _serve_saturated(eng, sat, templates, K, host_io=True, stagger=stagger)
    shares = _shares(dev["class_steps"])
    # roofline: the volume pass alone over a full batch of slots
    reqs = _serving_requests(sat, templates, eng.batch.upload_table)
    eng.run(reqs, realtime=False, max_steps=2)
    modes = eng.batch.active_modes()
    faces = sum(int(c.nx) * int(c.ny) for c, st in zip(eng.batch._cfgs, eng.batch.status()) if st.active)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    R = 10
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(R)]
    for i in range(R + 2):
        flush.fill_(i & 0xFF)
        if i >= 2:
            kev[i - 2][0].record(eng.batch.stream)
        eng.batch.volume_pass()
        if i >= 2:
            kev[i - 2][1].record(eng.batch.stream)
    torch.cuda.synchronize()
    vp_ms = sum(a.elapsed_time(b) for a, b in kev) / R
    vp_bytes = _volume_pass_bytes(modes, faces, "mixed")
    eng.reset()
    # latency: Poisson arrivals in real time, host inputs
    lat_reqs = _serving_requests(poisson, templates)
    eng.run(lat_reqs, realtime=True)
    lat = latency_percentiles(lat_reqs)
    span = max(r.finished for r in lat_reqs) - min(r.arrival for r in lat_reqs)
    lat_tput = sum(r.steps for r in lat_reqs) / span
    # the same engine below saturation: Poisson arrivals at half the measured capacity
    mean_steps = float(np.mean([r["steps"] for r in sat]))
    half_rate = 0.5 * (dev["slot_steps"] / (dev["ms"] * 1e-3)) / mean_steps
    half = workloads.serving_stream(n_requests=100, seed=1000 * rank + 2, rate=half_rate)
    half_reqs = _serving_requests(half, templates)
    eng.run(half_reqs, realtime=True)
    lat_half = latency_percentiles(half_reqs)
    service = [(r.finished - r.admitted) for r in half_reqs]
    slots, mem = eng.slots_per_class, eng.memory
    slots_policy = eng.batch.policy
    if eng.batch.tensor_core_error():
        raise RuntimeError("a tensor-core wait ran out in the serving runs")
    eng.close()

    # ---- comparisons on the same mix ---------------------------------------------
    f64 = engine("fp64")
    fdev = _serve_saturated(f64, sat, templates, K, host_io=False, stagger=stagger)
    f64.close()
    plain_rates, plain_steps = _plain_fp64_classes(sat, templates, args.plain_steps)
    plain = _mix_rate(plain_rates, shares)
    # accuracy of the benchmarked form (one forcing pass per step) against
    # FP64, inside the range over which that explicit scheme is predictable,
    # beside the distance between two FP64 runs whose initial fields differ by
    # one part in 1e12 (the conditioning floor); and of the same requests with
    # the evaporation solved to its Picard fixed point, where the problem is
    # well conditioned over any horizon
    acc_one, acc_conv = [], []
    horizons = sorted({h for h in (5, 10, 20, args.horizon_steps) if h <= args.horizon_steps})
    for m in [(512, 256, 64), (256, 128, 32), (128, 64, 16), (64, 32, 16)]:
        r = next(q for q in sat if q["mesh"] == m)
        cfg = workloads.serving_config(*m)
        reps = run_study(cfg, r["path"], horizons)
        curve = [{"steps": q["step"], "rel_l2": q["mixed"]["rel_l2"], "peak_T_err_K": q["mixed"]["peak_T_err_K"],
                  "fp64_perturbed_rel_l2": q["fp64_perturbed"]["rel_l2"],
                  "fp64_fp32_every_step_rel_l2": q["fp64_fp32_every_step"]["rel_l2"],
                  "fp64_fp32_rounded_once_rel_l2": q["fp64_fp32_rounded"]["rel_l2"]} for q in reps]
        # the last horizon at which the mixed error is within the bound
        ok = [c for c in curve if c["rel_l2"] <= 1e-4]
        acc_one.append({"mesh": list(m), "curve": curve,
                        "steps_within_bound": ok[-1]["steps"] if ok else 0,
                        "tensor_core_error": max(q["tensor_core_error"] for q in reps)})
        rep = run_study(cfg, r["path"], [min(r["steps"], args.accuracy_steps)],
                        picard={"max_picard_iter": 400, "picard_omega": 0.1, "picard_tol": 1e-8})[-1]
        acc_conv.append({"mesh": list(m), "steps": min(r["steps"], args.accuracy_steps),
                         "rel_l2": rep["mixed"]["rel_l2"], "peak_T_err_K": rep["mixed"]["peak_T_err_K"],
                         "fp64_perturbed_rel_l2": rep["fp64_perturbed"]["rel_l2"],
                         "fp64_fp32_every_step_rel_l2": rep["fp64_fp32_every_step"]["rel_l2"],
                         "tensor_core_error": rep["tensor_core_error"]})
    if any(a["tensor_core_error"] for a in acc_one + acc_conv):
        raise RuntimeError("a tensor-core wait ran out in the accuracy runs")

    t = [dev["ms"], e2e["ms"]]
    v_steps, e_steps = dev["slot_steps"], e2e["slot_steps"]
    if world > 1:
        t, (v_steps, e_steps) = reduce_over_ranks(t, [v_steps, e_steps], device="cuda")
    if rank != 0:
        return None
    value = v_steps / (t[0] * 1e-3)
    fb = fdev["slot_steps"] / (fdev["ms"] * 1e-3)
    peak, peak_kind = _peaks()
    achieved = vp_bytes / (vp_ms * 1e-3) / 1e9
    share_txt = {_class_key(k): round(v, 4) for k, v in sorted(shares.items())}
    line = {
        "metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": t[0] / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "mixed: bf16x3 tcgen05 face transforms, f32 modal state, f64 faces/norms/tables",
        "data": "synthetic (seeded request stream, laser paths and powers; no dataset)",
        "config": dict(_serving_desc(args), parallelism=f"replicas x{world}" if world > 1 else "single",
                       slots_per_class={_class_key(k): v for k, v in slots.items()},
                       workspace_gb=mem["workspace_bytes"] / 1e9, budget_gb=mem["budget_bytes"] / 1e9,
                       l2="not flushed: the modal state in flight is larger than L2",
                       lanes=args.lanes, tile_policy=slots_policy,
                       staggered_start_steps=stagger, slot_steps_timed=dev["slot_steps"],
                       completed_in_timed_region=dev["completed"], admitted_in_timed_region=dev["admitted"],
                       class_step_shares_timed=share_txt),
        "latency_ms": {"p50": lat["p50"] * 1e3, "p99": lat["p99"] * 1e3, "requests": len(lat_reqs),
                       "arrival_rate_per_s": 200.0, "throughput_timesteps_per_s": lat_tput,
                       "span_s": span,
                       "note": "200 requests/s offer about 2x the engine's capacity; latency is queueing"},
        "latency_ms_below_capacity": {"p50": lat_half["p50"] * 1e3, "p99": lat_half["p99"] * 1e3,
                                      "requests": len(half_reqs), "arrival_rate_per_s": half_rate,
                                      "service_ms_p50": float(np.percentile(service, 50)) * 1e3},
        "comparisons": {
            "mix": "every comparator is weighted by the per-class step shares of the timed region "
                   "(class_step_shares_timed): timesteps/s = 1 / sum(share_c / rate_c)",
            "plain_fp64_single_instance": {
                "value": plain, "unit": "timesteps/s",
                "per_class": {_class_key(k): v for k, v in sorted(plain_rates.items())},
                "sample": f"first request of each of the {len(plain_rates)} grid classes, one at a time, "
                          f"<= {args.plain_steps} steps each ({plain_steps} in all), device step graph, "
                          f"plan set-up excluded"},
            "batched_fp64": {"value": fb, "unit": "timesteps/s", "steps": K,
                             "completed_in_timed_region": fdev["completed"],
                             "class_step_shares_timed": {_class_key(k): round(v, 4) for k, v in
                                                         sorted(_shares(fdev["class_steps"]).items())}},
            "mixed_over_plain_fp64": value / plain, "mixed_over_batched_fp64": value / fb},
        "accuracy": {"vs": "FP64 single-instance solver (matches the reference to 1e-10)",
                     "physics": "the benchmarked serving physics: one forcing pass per step",
                     "horizons": horizons,
                     "note": "per grid, the mixed error against FP64 after 5..40 steps beside three "
                             "FP64 references: fp64_perturbed (started one part in 1e12 away: its "
                             "growth is the amplification of the explicit evaporation feedback), "
                             "fp64_fp32_every_step (modes rounded to FP32 after every step, all else "
                             "FP64) and fp64_fp32_rounded_once. The split-BF16 operands carry about "
                             "17 significant bits (x = hi + lo to 2^-17), so the mixed form starts "
                             "near 1e-6..1e-5 per step, above an FP32 state alone; where the feedback "
                             "amplifies (fp64_perturbed growing ~1000x from 20 to 40 steps at 512x256 "
                             "and 256x128) that error leaves the bound after steps_within_bound steps. "
                             "accuracy_picard_converged holds the same grids with the feedback solved "
                             "to its fixed point",
                     "runs": acc_one, "bound": 1e-4},
        "accuracy_picard_converged": {
            "physics": "the same requests with the evaporation solved to its Picard fixed point "
                       "(tol 1e-8, omega 0.1, cap 400)", "runs": acc_conv, "bound": 1e-4},
        "clocks": clocks,
        "gpu_launches": dev["launches"],
        "e2e": {"value": e_steps / (t[1] * 1e-3), "unit": "timesteps/s",
                "h2d_bytes_per_step": e2e["h2d"] / K, "d2h_bytes_per_step": e2e["d2h"] / K,
                "completed_in_timed_region": e2e["completed"],
                "api": "ServingEngine.run (host laser tables in, result surfaces out)"},
        "roofline": {"kernel": "kb_volume_ring<commit> (modal commit fused with the next step face sums, planes staged by bulk copies)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     "traffic": (NCU_VOLUME_TRAFFIC_PER_MODE * modes
                                 if NCU_VOLUME_TRAFFIC_PER_MODE is not None else None),
                     "traffic_note": "ncu capture of the 288-slot case, scaled by active modes",
                     "algorithmic_bytes_per_launch": vp_bytes, "modes": modes},
    }
    if world == 1 and not args.no_cpu_baseline:
        # two settings, as the reference is timed: all host threads for the
        # transforms, and one thread; the faster one is the baseline
        rates, n, el = _oracle_classes(sat, args.cpu_budget, args.cpu_steps_per_request, workers=-1)
        rates1, n1, el1 = _oracle_classes(sat, args.cpu_budget, args.cpu_steps_per_request, workers=1)
        v_all, v_one = _mix_rate(rates, shares), _mix_rate(rates1, shares)
        line["cpu_baseline"] = {
            "value": max(v_all, v_one), "unit": "timesteps/s",
            "cores": os.cpu_count() if v_all >= v_one else 1, "kind": "port",
            "settings": {"all_threads": v_all, "one_thread": v_one},
            "per_class": {_class_key(k): v for k, v in sorted((rates if v_all >= v_one else rates1).items())},
            "sample": f"{n} + {n1} timesteps in {el:.1f} + {el1:.1f} s: the first request of each grid class "
                      f"for <= {args.cpu_steps_per_request} steps, weighted by the timed region's class "
                      f"shares; the oracle port (NumPy/SciPy FP64 restatement of the reference step) stands "
                      f"in for the reference's NumPy backend (SpectralSolver(NumpyBackend()), float64), its "
                      f"two thread settings for the reference's as-shipped and single-thread runs"}
    return line


def run_profile(args):
    """--profile: launch the step kernels one by one (no graph) for ncu.

    ``serving-step``: the serving engine as in the benchmark (slots per class
    from --max-slots), every slot filled from the saturated stream, then
    --steps eager batched steps and three volume passes. ``raster-step`` /
    ``box-step``: the nonlinear raster / box workload through
    ``B200SpectralSolver.step(eager=True)`` for --warmup + --steps steps.
    Prints one line; no timing."""
    import copy

    import torch
    if args.profile == "serving-step":
        from spectral_galerkin_heat_b200 import workloads
        from spectral_galerkin_heat_b200.serving import ServingEngine
        sat = workloads.serving_stream(n_requests=args.requests, seed=0)
        meshes = sorted({r["mesh"] for r in sat})
        templates = {m: _context(workloads.serving_config(*m), None) for m in meshes}
        weights = {m: float(sum(r["steps"] for r in sat if r["mesh"] == m)) + 1.0 for m in meshes}
        eng = ServingEngine(templates, precision=args.precision, memory_fraction=args.memory_fraction,
                            max_slots=args.max_slots, weights=weights)
        eng.run(_serving_requests(sat, templates), realtime=False, max_steps=1)
        for _ in range(args.steps):
            eng.batch.step_eager()
        for _ in range(3):
            eng.batch.volume_pass()
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "precision": args.precision, "slots": eng.memory["slots"],
                          "active_modes": eng.batch.active_modes(), "workspace_gb": eng.batch.workspace_bytes / 1e9}))
        eng.close()
    elif args.profile in ("raster-step", "box-step", "raster-step-mixed"):
        from spectral_galerkin_heat_b200 import B200SpectralSolver
        cfg, path, desc = _workload(args.profile.split("-")[0], seed=0)
        mixed = args.profile.endswith("-mixed")
        s = B200SpectralSolver(None, _context(cfg, path), precision="mixed" if mixed else "fp64",
                               convergence_tol=args.mixed_tol if mixed else None)
        s.initialize()
        dt = s.context.num.dt
        for i in range(args.warmup + args.steps):
            s.step(i * dt, dt, eager=True)
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "steps": args.warmup + args.steps}))
        s.finalize()


def run_batch(args, rank, world, local_rank):
    """--workload batch: 64 uneven cuboids (Nx in {64..256}, Ny = Nx/2, Nz in
    {16,32,64}, seeded P, v, absorptivity; Picard at the reference defaults),
    all slots stepped together; K timed batched steps."""
    import copy

    import torch

    from spectral_galerkin_heat_b200 import B200SpectralSolver, workloads
    from spectral_galerkin_heat_b200.batch import BatchSolver
    torch.cuda.set_device(local_rank)
    K, W = args.steps, args.warmup
    pairs = workloads.uneven_batch(n=64, seed=rank, steps=W + K + 4)
    ctxs = [_context(c, p) for c, p in pairs]
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def timed(prec, host_io=False):
        b = BatchSolver(ctxs, prec)
        tables = [b.laser_table(c, 0.0, W + K + 4) for c in ctxs]
        for i in range(len(ctxs)):  # a few spare steps keep every slot active for the roofline pass
            b.start(i, W + K + 4, table=tables[i], record=True)
        b.step(W)
        torch.cuda.synchronize()
        it0 = sum(x.iters for x in b.status())
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        h2d = d2h = 0
        with ClockSampler(local_rank) as clk:
            for k in range(K):
                flush.fill_(k & 0xFF)
                ev[k][0].record(b.stream)
                b.step(1)
                if host_io:  # per step: the laser state in, the step's metrics out
                    st = b.status()
                    d2h += len(st) * C.sizeof(_lib.SghBatchSlotInfo)
                ev[k][1].record(b.stream)
            torch.cuda.synchronize()
        ms = sum(a.elapsed_time(c) for a, c in ev)
        iters = sum(x.iters for x in b.status()) - it0
        pre, per_it, post = b.launch_counts()
        # the Picard loop of a batched step runs to the slowest slot's count
        per_slot = [[m["n_evap_iter"] for m in b.metrics(i)[W:W + K]] for i in range(len(ctxs))]
        loop_iters = sum(max(col) for col in zip(*per_slot))
        out = {"ms": ms, "slot_steps": K * len(ctxs), "iters": iters, "clocks": clk.summary(),
               "launches": K * (1 + pre + post) + per_it * loop_iters, "d2h": d2h, "h2d": h2d}
        if not host_io and prec == "mixed":
            modes = b.active_modes()
            R = 10
            kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(R)]
            for i in range(R + 2):
                flush.fill_(i & 0xFF)
                if i >= 2:
                    kev[i - 2][0].record(b.stream)
                b.volume_pass()
                if i >= 2:
                    kev[i - 2][1].record(b.stream)
            torch.cuda.synchronize()
            faces = sum(int(c.num.nx) * int(c.num.ny) for c in ctxs)
            out["vp_ms"] = sum(a.elapsed_time(c) for a, c in kev) / R
            out["vp_bytes"] = _volume_pass_bytes(modes, faces, prec)
            out["modes"] = modes
        b.close()
        return out

    import ctypes as C

    from spectral_galerkin_heat_b200 import _lib
    mixed = timed("mixed")
    e2e = timed("mixed", host_io=True)
    f64 = timed("fp64")
    # plain FP64, one instance at a time: every grid shape of the batch once,
    # weighted by its share of the batch's instances (every instance steps alike)
    shape_of = [(int(c.num.nx), int(c.num.ny), int(c.num.nz)) for c in ctxs]
    counts = {m: shape_of.count(m) for m in set(shape_of)}
    plain_rates, plain_steps = {}, 0
    for m in sorted(counts):
        sv = B200SpectralSolver(None, copy.copy(ctxs[shape_of.index(m)]))
        sv.initialize()
        n = min(W + K, args.plain_steps)
        table = sv.laser_table(0.0, n + 2)
        outs = torch.zeros((n + 2) * 64, dtype=torch.uint8, device="cuda")
        sv.run_table(table, outs, 2, start=0)
        torch.cuda.synchronize()
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        sv.run_table(table, outs, n, start=2)
        c.record()
        torch.cuda.synchronize()
        plain_rates[m] = n / (a.elapsed_time(c) * 1e-3)
        plain_steps += n
        sv.finalize()
    t = [mixed["ms"], e2e["ms"]]
    if world > 1:
        t, _ = reduce_over_ranks(t, [0], device="cuda")
    if rank != 0:
        return None
    value = mixed["slot_steps"] * world / (t[0] * 1e-3)
    peak, peak_kind = _peaks()
    achieved = mixed["vp_bytes"] / (mixed["vp_ms"] * 1e-3) / 1e9
    plain = _mix_rate(plain_rates, _shares(counts))
    fb = f64["slot_steps"] / (f64["ms"] * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t[0] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "mixed: bf16x3 tcgen05 face transforms, f32 modal state, f64 faces/norms/tables",
        "data": "synthetic (seeded shapes, powers, speeds, absorptivities; no dataset)",
        "config": {"workload": "uneven_batch", "instances": 64, "grids": "Nx in {64,96,128,192,256}, Ny=Nx/2, "
                   "Nz in {16,32,64}", "cell": "64x32x16 on 2x1x0.5 mm, scaled with Nx", "dt_s": 5e-6,
                   "picard": "omega 0.1, tol 1e-4, cap 30 (reference defaults)",
                   "l2": "flushed between timed steps (256 MB write)",
                   "picard_iters_mean": mixed["iters"] / mixed["slot_steps"],
                   "parallelism": f"replicas x{world}" if world > 1 else "single"},
        "comparisons": {"plain_fp64_single_instance": {"value": plain, "sample": f"every one of the "
                        f"{len(counts)} grid shapes once ({plain_steps} steps in all), one at a time, "
                        f"weighted by the shape's share of the 64 instances"},
                        "batched_fp64": {"value": fb}, "mixed_over_plain_fp64": value / plain,
                        "mixed_over_batched_fp64": value / fb},
        "clocks": mixed["clocks"], "gpu_launches": mixed["launches"],
        "e2e": {"value": e2e["slot_steps"] * world / (t[1] * 1e-3), "unit": "timesteps/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": e2e["d2h"] / K,
                "api": "BatchSolver.step + status per step (laser tables resident from start)"},
        "roofline": {"kernel": "kb_volume_ring<commit>", "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": NCU_VOLUME_TRAFFIC_PER_MODE * mixed["modes"],
                     "algorithmic_bytes_per_launch": mixed["vp_bytes"]},
    }
    if world == 1 and not args.no_cpu_baseline:
        from oracle.sgh_oracle import OracleSolver
        n, el, touched = 0, 0.0, 0
        for ctx in ctxs:
            o = OracleSolver(copy.copy(ctx), workers=-1)
            o.initialize()
            dt = ctx.num.dt
            touched += 1
            for k in range(args.cpu_steps_per_request):
                t0 = time.perf_counter()
                o.step(k * dt, dt)
                el += time.perf_counter() - t0
                n += 1
                if el >= args.cpu_budget:
                    break
            if el >= args.cpu_budget:
                break
        line["cpu_baseline"] = {"value": n / el, "unit": "timesteps/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": f"{n} timesteps over the first {touched} instances "
                                          f"(<= {args.cpu_steps_per_request} steps each, {el:.1f} s)"}
    return line


def run_outputs(args, rank, world, local_rank):
    """--workload outputs: output reconstruction of a modal field -- the
    node-centred volume field of a full-volume output (sgh_nodal_temperature)
    and 3 x 1000 profile points, as arbitrary points (sgh_points_temperature)
    and as three profile lines (sgh_line_temperature) -- at 128 x 64 x 32
    and at the serving maximum 512 x 256 x 64, against the reference's host
    algorithm (weighted DCT-I, all host threads) on the same modes."""
    from types import SimpleNamespace

    import torch

    from oracle.sgh_oracle import nodal_temperature_dct1
    from spectral_galerkin_heat_b200 import kernels as Kn
    torch.cuda.set_device(local_rank)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    K, W = args.steps, args.warmup
    rows = {}
    for shape, L in (((32, 64, 128), (2e-3, 1e-3, 0.5e-3)), ((64, 256, 512), (2e-3, 1e-3, 0.5e-3))):
        nz, ny, nx = shape
        rng = np.random.default_rng(0)
        a = rng.standard_normal(shape)
        ad = torch.as_tensor(a, device="cuda")
        st = SimpleNamespace(size=L)
        geom = SimpleNamespace(size=SimpleNamespace(x=L[0], y=L[1], z=L[2]))
        pts = np.concatenate([np.stack([np.linspace(0, L[0], 1000), np.full(1000, L[1] / 2), np.full(1000, L[2])], 1),
                              np.stack([np.full(1000, L[0] / 2), np.linspace(0, L[1], 1000), np.full(1000, L[2])], 1),
                              np.stack([np.full(1000, L[0] / 2), np.full(1000, L[1] / 2), np.linspace(0, L[2], 1000)], 1)])
        ptd = torch.as_tensor(pts, device="cuda")

        def timed(fn):
            for _ in range(W):
                fn()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
            for k in range(K):
                flush.fill_(k & 0xFF)
                ev[k][0].record()
                fn()
                ev[k][1].record()
            torch.cuda.synchronize()
            return sum(x.elapsed_time(y) for x, y in ev) / K
        nodal_ms = timed(lambda: Kn.reconstruct_temperature_DCT(ad, st))
        points_ms = timed(lambda: Kn.reconstruct_temperature_volume_at_points(ad, None, geom, st, ptd))
        # the same 3 x 1000 points as three profile lines (each reduced once)
        profiles_ms = timed(lambda: Kn.save_temp_profiles(ad, None, geom, st, (L[0] / 2, L[1] / 2),
                                                          center="laser", num_points=1000))
        # e2e: modes from host memory in, the node field back to host memory
        host_a = torch.as_tensor(a).pin_memory()

        def e2e():
            d = host_a.to("cuda", non_blocking=True)
            return Kn.reconstruct_temperature_DCT(d, st).to("cpu")
        e2e_ms = timed(e2e)
        nodal_bytes = 8 * (nx * ny * nz + (nx + 1) * (ny + 1) * (nz + 1))
        nodal_flop = 2.0 * ((nx + 1) * nx * ny * nz + (ny + 1) * ny * nz * (nx + 1)
                            + (nz + 1) * nz * (ny + 1) * (nx + 1))
        t0 = time.perf_counter()
        n_cpu = 0
        while time.perf_counter() - t0 < min(args.cpu_budget, 10.0) or n_cpu < 1:
            nodal_temperature_dct1(a, L)
            n_cpu += 1
        cpu_ms = (time.perf_counter() - t0) * 1e3 / n_cpu
        rows[f"{nx}x{ny}x{nz}"] = {
            "nodal_ms": nodal_ms, "nodal_e2e_ms": e2e_ms, "points_3000_ms": points_ms,
            "profiles_3x1000_ms": profiles_ms,
            "nodal_cpu_reference_algorithm_ms": cpu_ms, "cpu_over_gpu": cpu_ms / nodal_ms,
            "nodal_gbs_min_traffic": nodal_bytes / (nodal_ms * 1e-3) / 1e9,
            "nodal_fp64_tflops": nodal_flop / (nodal_ms * 1e-3) / 1e12}
    if rank != 0:
        return None
    big = rows["512x256x64"]
    hbm, hbm_kind = _peaks()
    fp64 = _fp64_peak(torch.device("cuda", local_rank))
    return {"metric": "node-field reconstructions/s", "value": 1e3 / big["nodal_ms"], "unit": "1/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": big["nodal_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random modes)",
            "config": {"workload": "output_reconstruction", "shapes": rows,
                       "l2": "flushed between timed launches (256 MB write)"},
            "e2e": {"value": 1e3 / big["nodal_e2e_ms"], "unit": "1/s", "h2d_bytes_per_step": 8 * 512 * 256 * 64,
                    "d2h_bytes_per_step": 8 * 513 * 257 * 65},
            "roofline": {"kernel": "3 axis passes of the node field (FP64 tensor cores)", "bound": "fp64",
                         "achieved": big["nodal_fp64_tflops"], "peak": fp64, "unit": "TFLOP/s",
                         "frac": big["nodal_fp64_tflops"] / fp64,
                         "peak_source": "measured here: cuBLAS DGEMM 4096^3, best of 10", "traffic": None,
                         "hbm_gbs_min_traffic": big["nodal_gbs_min_traffic"], "hbm_peak": hbm,
                         "hbm_peak_source": hbm_kind,
                         "note": "FP64 contraction work bounds it (dense N x (N+1) passes), not HBM"},
            "cpu_baseline": {"value": 1e3 / big["nodal_cpu_reference_algorithm_ms"], "unit": "1/s",
                             "cores": os.cpu_count(), "kind": "port",
                             "sample": "the reference's weighted DCT-I (scipy, all threads) on the same modes"}}


def _relaunch(n):
    """Re-run this command as ``n`` ranks under torch.distributed.run (one
    process per GPU, rendezvous on 127.0.0.1); returns their exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__),
           *sys.argv[1:]]
    return subprocess.call(cmd)


def run_replica_selftest(args, rank, world):
    """A host-only stand-in workload for the replica launch path: every rank
    does the same fixed amount of host work, timed, and the aggregate goes
    through reduce_over_ranks exactly as the GPU workloads do."""
    x = np.random.default_rng(rank).standard_normal(1 << 16)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        x = np.cos(x)
    ms = (time.perf_counter() - t0) * 1e3
    t, (steps,) = [ms], [args.steps]
    if world > 1:
        t, (steps,) = reduce_over_ranks(t, [steps])
    if rank != 0:
        return None
    return {"metric": "host steps/s (launch-path self test)", "value": steps / (t[0] * 1e-3),
            "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t[0] / args.steps, "higher_is_better": True, "scaling": "weak",
            "config": {"workload": "replica-selftest", "ranks": world}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (serving: batched steps, default 1000; otherwise 200)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["serving", "batch", "raster", "track", "box", "outputs",
                                           "replica-selftest"],
                    default="serving")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--axis-cuda-cores", action="store_true",
                    help="raster/track/box: FP64 axis passes on the CUDA-core kernels only")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--requests", type=int, default=1000, help="serving: saturated stream length")
    ap.add_argument("--stagger-steps", type=int, default=1100,
                    help="serving: untimed batched steps before the timed region (steady state)")
    ap.add_argument("--mixed-tol", type=float, default=1e-5,
                    help="raster/box: Picard tolerance of the mixed-precision comparison")
    ap.add_argument("--mixed-error-steps", type=int, default=20,
                    help="raster/box: steps of the mixed-vs-FP64 error report")
    ap.add_argument("--no-mixed", action="store_true", help="raster/box: skip the mixed-precision comparison")
    ap.add_argument("--horizon-steps", type=int, default=40,
                    help="serving: steps of the one-pass accuracy check")
    ap.add_argument("--max-slots", type=int, default=24,
                    help="serving: slots per grid class at most (24 over two lanes measured fastest: "
                         "139.9K against 136.8K with 16)")
    ap.add_argument("--lanes", type=int, default=2,
                    help="serving: batches on separate CUDA streams, stepped concurrently "
                         "(2 lanes measured fastest; 3 and 4 within 0.5%%, 1 lane 6%% slower)")
    ap.add_argument("--memory-fraction", type=float, default=0.5, help="serving: share of free HBM")
    ap.add_argument("--plain-steps", type=int, default=300)
    ap.add_argument("--cpu-steps-per-request", type=int, default=20)
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--profile", choices=["serving-step", "raster-step", "box-step", "raster-step-mixed"],
                    default=None,
                    help="launch the step kernels one by one for a profiler and exit (no timing)")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed", help="--profile serving-step")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 2 if args.profile else {"serving": 1000, "batch": 100, "outputs": 20}.get(args.workload, 200)
    if args.warmup < 3:
        args.warmup = 3
    if args.profile:
        run_profile(args)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start the ranks here when no launcher did
        sys.exit(_relaunch(args.gpus))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    distributed = world > 1 and args.impl == "b200"
    selftest = args.workload == "replica-selftest"
    if distributed:
        import torch
        import torch.distributed as dist
        if not selftest:
            torch.cuda.set_device(local_rank)
        dist.init_process_group(backend="gloo" if selftest else "nccl",
                                timeout=datetime.timedelta(seconds=600))
    try:
        if selftest:
            line = run_replica_selftest(args, rank, world)
        elif args.impl == "reference":
            line = run_reference(args, rank, world)
        elif args.workload == "serving":
            line = run_serving(args, rank, world, local_rank)
        elif args.workload == "batch":
            line = run_batch(args, rank, world, local_rank)
        elif args.workload == "outputs":
            line = run_outputs(args, rank, world, local_rank)
        else:
            line = run_b200(args, rank, world, local_rank)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if distributed:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
