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

__all__ = ["CANDIDATES", "KERNELS", "key_of", "lookup", "lookup_kernel", "tune", "tune_table",
           "BATCH_CANDIDATES", "batch_key", "lookup_batch", "tune_batch"]

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


def _load(path: str, section: str = "entries") -> Dict:
    if (path, section) not in _cache:
        try:
            with open(path) as f:
                _cache[(path, section)] = json.load(f).get(section, {})
        except (OSError, ValueError):
            _cache[(path, section)] = {}
    return _cache[(path, section)]


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
        try:
            with open(out) as f:
                table["batch_entries"] = json.load(f).get("batch_entries", {})
        except (OSError, ValueError):
            pass
        with open(out, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        for k in list(_cache):
            if k[0] == out:
                _cache.pop(k)
    return table


# ---------------------------------------------------------------------------
# batched engine: the tile policy of its kernels per grid mix
# ---------------------------------------------------------------------------
# vol_unroll: z-planes whose loads one round of the volume pass (the
# bandwidth-bound modal commit) issues before their arithmetic; vol_vec:
# columns per thread (vector width of its loads). More planes and wider
# vectors keep more bytes in flight per thread; fewer keep registers, and so
# warps per SM, up. The best trade depends on nz and on the mix of slot shapes.
BATCH_CANDIDATES = tuple({"vol_unroll": u, "vol_vec": v} for v in (2, 4) for u in (2, 4, 8))


def batch_key(cfgs, precision: str) -> str:
    """Table key of a batch: its precision and grid mix (shape and form of
    every slot class, with the slot count)."""
    counts: Dict[str, int] = {}
    for c in cfgs:
        k = key_of(c)
        counts[k] = counts.get(k, 0) + 1
    return f"{precision}|" + "+".join(f"{n}*{k}" for k, n in sorted(counts.items()))


def _classes_of(key: str):
    """(precision, set of slot classes) of a batch key, slot counts dropped."""
    prec, _, mix = key.partition("|")
    return prec, frozenset(part.split("*", 1)[1] for part in mix.split("+") if "*" in part)


def lookup_batch(cfgs, precision: str) -> Optional[Dict]:
    """Tuned policy for this batch's precision and grid mix, or None. A mix
    tuned with other slot counts of the same classes (a serving batch dealt
    over lanes holds a share of every class) takes that entry's policy."""
    k = batch_key(cfgs, precision)
    tables = [_load(p, "batch_entries") for p in (os.environ.get("SGH_TUNE_TABLE"), SHIPPED) if p]
    for t in tables:
        if k in t:
            return dict(t[k]["policy"])
    want = _classes_of(k)
    for t in tables:
        for kk, e in sorted(t.items()):
            if _classes_of(kk) == want:
                return dict(e["policy"])
    return None


def tune_batch(contexts, precision: str = "mixed", steps: int = 20, warmup: int = 5,
               candidates=BATCH_CANDIDATES) -> Dict:
    """Time every candidate policy on a batch of ``contexts`` with all slots
    active: ms per batched step (step graph, CUDA events after warm-up) and
    ms of the volume pass alone; keeps the fastest step."""
    import torch

    from .batch import BatchSolver
    res = {}
    for pol in candidates:
        if precision != "mixed" and pol.get("vol_vec", 0) > 2:
            continue  # 4-wide vectors need FP32 modes
        b = BatchSolver(contexts, precision, policy=pol)
        for i in range(b.n):
            b.start(i, warmup + steps + 2, record=False)
        b.step(warmup)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(b.stream)
        b.step(steps)
        ev[1].record(b.stream)
        ev[2].record(b.stream)
        for _ in range(5):
            b.volume_pass()
        ev[3].record(b.stream)
        torch.cuda.synchronize()
        if b.tensor_core_error():
            raise RuntimeError("a tensor-core wait ran out while tuning")
        res[json.dumps(pol, sort_keys=True)] = {"ms_per_step": ev[0].elapsed_time(ev[1]) / steps,
                                                 "volume_pass_ms": ev[2].elapsed_time(ev[3]) / 5}
        b.close()
    best = min(res, key=lambda k: res[k]["ms_per_step"])
    return {"policy": json.loads(best), "candidates": res}


def tune_batch_table(mixes: Dict[str, tuple], out: Optional[str] = None, **kw) -> Dict:
    """Tune every named (contexts, precision) mix and merge the entries into
    the table's ``batch_entries``."""
    from .solver import make_config
    from .batch import _picard
    entries = {}
    for name, (ctxs, prec) in mixes.items():
        cfgs = [make_config(c, *_picard(c)) for c in ctxs]
        t0 = time.perf_counter()
        r = tune_batch(ctxs, prec, **kw)
        r["workload"] = name
        r["tuning_s"] = time.perf_counter() - t0
        entries[batch_key(cfgs, prec)] = r
    table = {"note": "", "entries": {}}
    if out:
        try:
            with open(out) as f:
                table = json.load(f)
        except (OSError, ValueError):
            pass
        table.setdefault("batch_entries", {}).update(entries)
        with open(out, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        for k in list(_cache):
            if k[0] == out:
                _cache.pop(k)
    return entries


def batch_mixes() -> Dict[str, tuple]:
    """The batched engine's benchmark mixes: the serving engine's slot classes
    (16 slots per class, mixed and FP64) and the 64 uneven instances."""
    from . import workloads
    from .config import SimulationContext

    def ctx(cfg, path=None):
        c = SimulationContext.from_dict(copy.deepcopy(cfg))
        c.laser_path = path
        return c
    stream = workloads.serving_stream(n_requests=1000, seed=0)
    serving = []
    for m in sorted({r["mesh"] for r in stream}):
        paths = [r["path"] for r in stream if r["mesh"] == m]
        serving += [ctx(workloads.serving_config(*m), paths[i % len(paths)]) for i in range(16)]
    uneven = [ctx(cfg, path) for cfg, path in workloads.uneven_batch()]
    return {"serving_mixed": (serving, "mixed"), "serving_fp64": (serving, "fp64"),
            "uneven_mixed": (uneven, "mixed"), "uneven_fp64": (uneven, "fp64")}


def main(argv=None):
    from . import workloads
    from .config import SimulationContext
    ap = argparse.ArgumentParser(description="tune the axis-pass tiles for the benchmark shapes")
    ap.add_argument("--out", default=SHIPPED)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--batch-only", action="store_true", help="tune only the batched engine's mixes")
    args = ap.parse_args(argv)

    def ctx(cfg, path):
        c = SimulationContext.from_dict(copy.deepcopy(cfg))
        c.laser_path = path
        return c
    mixes = batch_mixes()
    entries = tune_batch_table(mixes, out=args.out)
    for k, e in sorted(entries.items()):
        print(f"{e['workload']:24s} -> {e['policy']}  " + "  ".join(
            f"{pk}: {v['ms_per_step']:.3f} ms/step, volume {v['volume_pass_ms']:.3f} ms"
            for pk, v in e["candidates"].items()))
    if args.batch_only:
        return
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
