"""Precision study: the mixed-precision form of the step against FP64.

For one configuration and laser path this runs, side by side on the device:

* ``fp64``: the plain single-instance solver (:class:`B200SpectralSolver`),
  which matches the reference to 1e-10 relative L2;
* ``mixed``: the mixed-precision form (a batch of one slot: FP32 modal state,
  split-BF16 tensor-core face transforms with FP32 accumulation, FP64 faces,
  norms and coefficient tables);
* ``fp64_perturbed``: the FP64 solver again, from an initial field changed by
  one part in 1e12. Where this run already parts from ``fp64``, the problem
  is ill-conditioned and a difference between precisions there is not a
  precision error.

At each checkpoint step the report gives, against ``fp64``:

* ``rel_l2``: ||T - T_fp64|| / ||T_fp64|| over the cell-centred volume field
  (the transform is orthonormal, so this is also the relative L2 of the modes);
* ``peak_T``: the maximum of the volume field, and its difference in K;
* ``melt_pool``: length (x), width (y) and depth (from the top face z = Lz) of
  the cells at or above the liquidus, in metres (cell extents), and their
  differences.

Run it with ``python -m spectral_galerkin_heat_b200.precision`` (see --help);
the default is the 256 x 128 x 64 straight-track study with seeded power and
speed, once with one forcing pass per step and once with the evaporation
solved to its Picard fixed point.
"""
from __future__ import annotations

import argparse
import copy
import json
from typing import Dict, List, Optional, Sequence

import numpy as np

__all__ = ["melt_pool", "compare_fields", "run_study"]


def melt_pool(T: np.ndarray, dx: float, dy: float, dz: float, T_melt: float) -> Dict[str, float]:
    """Extents of the cells with ``T >= T_melt`` in a (nz, ny, nx) cell-centred
    field whose top face is z index nz - 1: length along x, width along y,
    depth below the top face (all in metres, whole cells; zero when none)."""
    m = T >= T_melt
    if not m.any():
        return {"length": 0.0, "width": 0.0, "depth": 0.0, "cells": 0}
    zs, ys, xs = np.nonzero(m)
    nz = T.shape[0]
    return {"length": float((xs.max() - xs.min() + 1) * dx), "width": float((ys.max() - ys.min() + 1) * dy),
            "depth": float((nz - zs.min()) * dz), "cells": int(m.sum())}


def compare_fields(T: np.ndarray, T_ref: np.ndarray, cell, T_melt: float) -> Dict[str, object]:
    """Error report of ``T`` against ``T_ref`` (both (nz, ny, nx), FP64)."""
    dx, dy, dz = cell
    mp, mp_ref = melt_pool(T, dx, dy, dz, T_melt), melt_pool(T_ref, dx, dy, dz, T_melt)
    return {
        "rel_l2": float(np.linalg.norm(T - T_ref) / np.linalg.norm(T_ref)),
        "peak_T": float(T.max()), "peak_T_ref": float(T_ref.max()),
        "peak_T_err_K": float(T.max() - T_ref.max()),
        "melt_pool": mp, "melt_pool_ref": mp_ref,
        "melt_pool_err_m": {k: mp[k] - mp_ref[k] for k in ("length", "width", "depth")},
    }


def run_study(cfg: dict, path, checkpoints: Sequence[int], picard: Optional[dict] = None,
              perturb: float = 1e-12, seed: int = 0) -> List[Dict[str, object]]:
    """Step the three runs to each checkpoint and compare (see the module doc)."""
    import torch

    from .batch import BatchSolver
    from .config import SimulationContext
    from .solver import B200SpectralSolver
    cfg = copy.deepcopy(cfg)
    if picard:
        cfg["simulation"].update(picard)
    ctx = SimulationContext.from_dict(cfg)
    ctx.laser_path = path
    num = ctx.num
    dt = float(num.dt)
    Lx, Ly, Lz = cfg["domain"]["size"]
    cell = (Lx / num.nx, Ly / num.ny, Lz / num.nz)
    T_melt = float(cfg["material"]["T_liquidus"])
    total = int(max(checkpoints))

    ref = B200SpectralSolver(None, copy.copy(ctx))
    ref.initialize()
    per = B200SpectralSolver(None, copy.copy(ctx))
    per.initialize()
    T0 = per.volume_temperature().cpu().numpy()
    rng = np.random.default_rng(seed)
    per.set_state(T0 * (1.0 + perturb * rng.standard_normal(T0.shape)))
    mix = BatchSolver([copy.copy(ctx)], "mixed")
    mix.start(0, total, record=True)

    out, done = [], 0
    for cp in sorted(set(int(c) for c in checkpoints)):
        n = cp - done
        ref_m = ref.run(done * dt, n)
        per.run(done * dt, n)
        mix.step(n)
        done = cp
        T_ref = ref.volume_temperature().cpu().numpy()
        T_per = per.volume_temperature().cpu().numpy()
        T_mix = ref.volume_temperature(mix.modes(0).to(torch.float64).contiguous()).cpu().numpy()
        mm = mix.metrics(0)[-1]
        out.append({
            "step": cp,
            "picard_iters_fp64_last": ref_m[-1]["n_evap_iter"], "picard_iters_mixed_last": mm["n_evap_iter"],
            "T_surface_max_fp64": ref_m[-1]["T_surface_max"], "T_surface_max_mixed": mm["T_surface_max"],
            "mixed": compare_fields(T_mix, T_ref, cell, T_melt),
            "fp64_perturbed": compare_fields(T_per, T_ref, cell, T_melt),
            "tensor_core_error": mix.tensor_core_error(),
        })
    ref.finalize()
    per.finalize()
    mix.close()
    return out


def main(argv=None):
    from . import workloads
    ap = argparse.ArgumentParser(description="mixed-precision vs FP64 error report")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--mesh", type=int, nargs=3, default=[256, 128, 64])
    ap.add_argument("--checkpoints", type=int, nargs="+", default=[20, 100, 500])
    ap.add_argument("--out", default=None, help="write the JSON report here")
    args = ap.parse_args(argv)
    nx, ny, nz = args.mesh
    cfg, path = workloads.precision_track(seed=args.seed, nx=nx, ny=ny, nz=nz)
    forms = {
        "one_pass": None,
        "picard_converged": {"max_picard_iter": 400, "picard_omega": 0.1, "picard_tol": 1e-8},
    }
    report = {"config": {"mesh": [nx, ny, nz], "domain_m": cfg["domain"]["size"], "seed": args.seed,
                         "power_W": path.power, "speed_m_s": path.vx,
                         "fp32_contraction_variant": "not built: the mixed form's contractions are "
                                                     "split-BF16 on the tensor cores"},
              "forms": {}}
    for name, picard in forms.items():
        report["forms"][name] = run_study(cfg, path, args.checkpoints, picard=picard, seed=args.seed)
    text = json.dumps(report, indent=1)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)
    print(text)


if __name__ == "__main__":
    main()
