"""Benchmark: time steps per second of the spectral-Galerkin heat solver on B200.

Workload (default ``--workload raster``): the full nonlinear FP64 case -- 316L
cuboid 2.0 x 1.0 x 0.5 mm at 128 x 64 x 32 modes, T-dependent k(T) and c_p(T),
latent heat over 1658-1723 K (grid mode), evaporation + top convection, Picard
to 1e-8 relative residual (omega 0.1, cap 400), dt = 2 us, seeded 5-line raster.
``--workload track`` is the 64 x 32 x 16 straight-track case (one forcing pass
per step).

One step = one ``SpectralSolver.step`` of that workload (laser/face forcing,
ETD1 update, the Picard loop to convergence, commit). W warm-up steps run from
t = 0, then K timed steps continue the same trajectory.

* ``value``: steps/s with everything resident on the device, each step one
  launch of the device-resident step graph (``sgh_run``), timed with CUDA events
  per step; L2 (126 MB, larger than the ~24 MB working set) is flushed between
  timed steps by writing a 256 MB buffer outside the timed intervals.
* ``e2e``: the same metric through the public API ``B200SpectralSolver.step(t, dt)``
  -- host laser state in, metrics copied back to the host and read every step.
* ``roofline``: the DCT axis-pass kernel (``k_axis``, the dominant kernel in the
  launch list), timed live here with CUDA events on a full-size 3-D transform.
* ``cpu_baseline``: the CPU oracle (NumPy/SciPy FP64 restatement of the
  reference step, all host threads) on a bounded sample of the same workload.

``--impl reference`` times that CPU implementation alone (rank 0) and prints
the same JSON line with ``"impl": "reference"``.

Multi-GPU (``torchrun --nproc-per-node N bench.py --gpus N``): every rank runs
an independent replica (its own seeded raster); there is no collective on the
step path. ``value`` = all ranks' steps / max over ranks of the timed seconds.
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
# dram__bytes_read.sum + dram__bytes_write.sum per launch of the dominant kernel
# (k_axis on the 128x64x32 transform) from an ncu capture of this workload;
# None until that capture exists.
NCU_TRAFFIC_BYTES = None


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


def run_reference(args, rank, world):
    """--impl reference: the CPU implementation alone, rank 0 only."""
    if rank != 0:
        return None
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
        "n_gpus": args.gpus, "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 / v,
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
    s = B200SpectralSolver(None, _context(cfg, path))
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

    # ---- dominant kernel, timed live: DCT axis passes of one 3-D transform ----
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
    peak, peak_kind = _peaks()
    s.finalize()

    # ---- end to end through the public API ----------------------------------
    e = B200SpectralSolver(None, _context(cfg, path))
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
        t = torch.tensor([dev_ms, e2e_ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_max, e2e_max = float(t[0]), float(t[1])
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
                       picard_iters_mean=float(np.mean(iters)), step_status=statuses),
        "clocks": clocks,
        "gpu_launches": launches * world,
        "e2e": {"value": total_steps / (e2e_max * 1e-3), "unit": "steps/s",
                "h2d_bytes_per_step": C.sizeof(_lib.SghLaser),
                "d2h_bytes_per_step": C.sizeof(_lib.SghStepOut),
                "api": "B200SpectralSolver.step(t, dt)"},
        "roofline": {"kernel": "k_axis (DCT axis pass, FP64)", "bound": "hbm",
                     "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak, "peak_source": peak_kind,
                     "traffic": NCU_TRAFFIC_BYTES,
                     "algorithmic_bytes_per_launch": bytes_per_pass,
                     "fp64_tflops": (2.0 * V * (nx + ny + nz) / 3)
                     / (per_transform_ms / 3 * 1e-3) / 1e12},
    }
    if world == 1 and not args.no_cpu_baseline:
        v, n, el = cpu_baseline(cfg, path, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": v, "unit": "steps/s", "cores": os.cpu_count(),
                                "kind": "port",
                                "sample": f"{n} steps from t=dt of the same workload "
                                          f"({el:.1f} s), after 1 warm-up step"}
    return line


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["raster", "track"], default="raster")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    distributed = world > 1 and args.impl == "b200"
    if distributed:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group(backend="nccl", timeout=datetime.timedelta(seconds=600))
    try:
        line = run_reference(args, rank, world) if args.impl == "reference" \
            else run_b200(args, rank, world, local_rank)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if distributed:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
