"""Autotuner of the FP64 axis-pass kernels and tiles, per grid shape.

Every axis pass of a plan (the x, y and z contractions of its 3-D and face
transforms) runs either on the FP64 tensor cores (``mma.sync`` .f64, when the
pass is large enough) or on the CUDA-core kernel with 2 x 4 or 1 x 1 register
tiles per thread; ``sgh_config.axis_cuda_cores = 1`` keeps every pass on the
CUDA cores. For the CUDA-core kernel, larger tiles
cut shared-memory operand traffic per flop; smaller ones give more CTAs, which
matters when a pass has few columns. The plan switches per pass on the number
of CTAs the 2 x 4 grid would have: 2 x 4 when it reaches
``sgh_config.axis_min_ctas`` (the built-in default is 132), so one threshold
selects a combination of tile shapes over the plan's passes. The best
threshold depends on (nx, ny, nz) and on the form of the step (face-space
Picard loop, or volume transforms when latent heat or the property correction
is on).

:func:`tune` times candidate (threshold, kernel) pairs on the real step of a
context -- the device-resident step graph, after warm-up, with CUDA events --
and keeps the fastest per Picard iteration (the tile shape changes the rounding of the
contractions, so iteration counts may differ by one). Results go into a JSON
table keyed by shape and form: the package ships ``tuned.json`` (made on B200
by ``python -m spectral_galerkin_heat_b200.autotune``), and a user table named
by the environment variable ``SGH_TUNE_TABLE`` takes precedence.
``B200SpectralSolver`` applies the table when it builds a plan.
"""
from __future__ import annotations

import argparse
import copy
import ctypes
import json
import os
import time
from typing import Dict, Iterable, Optional

__all__ = ["CANDIDATES", "KERNELS", "key_of", "lookup", "lookup_kernel", "tune", "tune_table"]

# always 2 x 4, three switch points, never 2 x 4
CANDIDATES = (1, 66, 132, 264, 1 << 30)
# axis_cuda_cores: 0 = tensor cores where the pass is large enough, 1 = CUDA cores only
KERNELS = (0, 1)
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json")
_cache: Dict[str, Dict] = {}


def _form(cfg) -> str:
    if int(getattr(cfg, "box", 0)):
        return "box"
    latent = float(cfg.L_f) > 0.0
    corr = bool(cfg.has_model) and not bool(cfg.model_constant)
    return "volume" if (latent or corr) else "face"


def key_of(cfg) -> str:
    """Table key of an ``sgh_config``: ``"<nx>x<ny>x<nz>:<form>"``."""
    return f"{int(cfg.nx)}x{int(cfg.ny)}x{int(cfg.nz)}:{_form(cfg)}"


def _load(path: str) -> Dict:
    if path not in _cache:
        try:
            with open(path) as f:
                _cache[path] = json.load(f).get("entries", {})
        except (OSError, ValueError):
            _cache[path] = {}
    return _cache[path]


def _entry(cfg) -> Optional[Dict]:
    k = key_of(cfg)
    for path in (os.environ.get("SGH_TUNE_TABLE"), SHIPPED):
        if path:
            e = _load(path).get(k)
            if e is not None:
                return e
    return None


def lookup(cfg) -> Optional[int]:
    """Tuned threshold for this plan's shape and form, or None (built-in default)."""
    e = _entry(cfg)
    return None if e is None else int(e["axis_min_ctas"])


def lookup_kernel(cfg) -> Optional[int]:
    """Tuned ``axis_cuda_cores`` (0 or 1) for this shape and form, or None (0)."""
    e = _entry(cfg)
    return None if e is None or "axis_cuda_cores" not in e else int(e["axis_cuda_cores"])


def tune(ctx, candidates: Iterable[int] = CANDIDATES, steps: int = 10, warmup: int = 3,
         kernels: Iterable[int] = KERNELS) -> Dict:
    """Time each (threshold, kernel) pair on ``ctx``'s step; returns the choice
    and the per-candidate ms per Picard iteration and per step (keys
    ``"<threshold>|<axis_cuda_cores>"``)."""
    res = {}
    for kern in kernels:
        for c in candidates:
            res[(int(c), int(kern))] = _time_one(ctx, int(c), int(kern), steps, warmup)
    best = min(res, key=lambda ck: res[ck]["ms_per_iter"])
    return {"axis_min_ctas": best[0], "axis_cuda_cores": best[1],
            "candidates": {f"{c}|{k}": v for (c, k), v in res.items()},
            "default_ms_per_iter": res.get((132, 0), {}).get("ms_per_iter")}


def _time_one(ctx, c: int, kern: int, steps: int, warmup: int) -> Dict:
    """One candidate on the device-resident step graph: ms per step and per Picard iteration."""
    import torch

    from . import _lib
    from .solver import B200SpectralSolver
    s = B200SpectralSolver(None, copy.copy(ctx), axis_min_ctas=c, axis_cuda_cores=bool(kern))
    s.initialize()
    table = s.laser_table(0.0, warmup + steps)
    osz = ctypes.sizeof(_lib.SghStepOut)
    outs = torch.zeros((warmup + steps) * osz, dtype=torch.uint8, device=s.state.workspace.device)
    s.run_table(table, outs, warmup, start=0)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s.state.stream)
    s.run_table(table, outs, steps, start=warmup)
    b.record(s.state.stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    recs = s.decode_outs(outs.cpu().numpy().tobytes(), warmup + steps)[warmup:]
    iters = max(1, sum(max(1, r.n_iter) for r in recs))
    s.finalize()
    return {"ms_per_step": ms / steps, "ms_per_iter": ms / iters, "iters": iters}


def tune_table(contexts: Dict[str, object], out: Optional[str] = None, **kw) -> Dict:
    """Tune every context (name -> SimulationContext) and write the table."""
    from .solver import make_config
    entries = {}
    for name, ctx in contexts.items():
        cfg = make_config(ctx, 0.1, 1e-4, 1)
        k = key_of(cfg)
        if k in entries:
            continue
        t0 = time.perf_counter()
        r = tune(ctx, **kw)
        r["workload"] = name
        r["tuning_s"] = time.perf_counter() - t0
        entries[k] = r
    table = {"note": "axis-pass kernel (tensor cores or CUDA cores) and CUDA-core tile threshold per grid "
                     "shape and step form, timed on the step graph",
             "entries": entries}
    if out:
        with open(out, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        _cache.pop(out, None)
    return table


def main(argv=None):
    from . import workloads
    from .config import SimulationContext
    ap = argparse.ArgumentParser(description="tune the axis-pass tiles for the benchmark shapes")
    ap.add_argument("--out", default=SHIPPED)
    ap.add_argument("--steps", type=int, default=10)
    args = ap.parse_args(argv)

    def ctx(cfg, path):
        c = SimulationContext.from_dict(copy.deepcopy(cfg))
        c.laser_path = path
        return c
    contexts = {}
    cfg, path = workloads.nonlinear_raster()
    contexts["nonlinear_raster"] = ctx(cfg, path)
    cfg, path = workloads.straight_track()
    contexts["straight_track"] = ctx(cfg, path)
    cfg, path = workloads.precision_track()
    contexts["precision_track"] = ctx(cfg, path)
    cfg, path = workloads.box_track()
    contexts["box_track"] = ctx(cfg, path)
    for r in workloads.serving_stream(n_requests=200, seed=0):
        name = "serving_" + "x".join(map(str, r["mesh"]))
        if name not in contexts:
            contexts[name] = ctx(r["cfg"], r["path"])
    table = tune_table(contexts, out=args.out, steps=args.steps)
    for k, e in sorted(table["entries"].items()):
        best = e["candidates"][f"{e['axis_min_ctas']}|{e['axis_cuda_cores']}"]
        print(f"{k:24s} -> {e['axis_min_ctas']:>10d} cuda_cores={e['axis_cuda_cores']}  "
              f"({best['ms_per_iter']:.4f} ms/iter; default {e['default_ms_per_iter']:.4f})")


if __name__ == "__main__":
    main()
