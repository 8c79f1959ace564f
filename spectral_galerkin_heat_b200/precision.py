"""Precision study: the mixed-precision form of the step against FP64.

For one configuration and laser path this runs, side by side on the device:

* ``fp64``: the plain single-instance solver (:class:`B200SpectralSolver`),
  which matches the reference to 1e-10 relative L2;
* ``mixed``: the mixed-precision form (a batch of one slot: FP32 modal state,
  split-BF16 tensor-core face transforms with FP32 accumulation, FP64 face
  fields, norms and coefficient tables, FP32 face sums and weights);
* ``fp32``: the single-instance plan with every contraction in FP32
  arithmetic on the CUDA cores and the modal iterates in FP32 (FP64 faces,
  norms and tables), the plain FP32 arm against which the split-BF16
  contractions are judged;
* ``fp64_perturbed``: the FP64 solver again, from an initial field changed by
  one part in 1e12. Where this run already parts from ``fp64``, the problem
  is ill-conditioned and a difference between precisions there is not a
  precision error.
* ``fp64_fp32_rounded``: the FP64 solver again, with its modes rounded to
  FP32 once, after the first step. A random perturbation of the whole volume
  mostly lands in fast-decaying modes; this one has the structure of the
  rounding that an FP32 modal state undergoes every step, so it shows how far
  a single such rounding carries on this problem.
* ``fp64_fp32_every_step``: the FP64 solver with its modes rounded to FP32
  after every step -- the error of an FP32 modal state alone, with every
  contraction and all physics in FP64: the floor of any form that keeps the
  state in FP32, as the mixed form does.

At each checkpoint step the report gives, against ``fp64``:

* ``rel_l2``: ||T - T_fp64|| / ||T_fp64|| over the cell-centred volume field
  (the transform is orthonormal, so this is also the relative L2 of the modes);
* ``peak_T``: the maximum of the volume field, and its difference in K;
* ``melt_pool``: length (x) and width (y) of the region at or above the
  liquidus on the top face, and its depth below the top face (z = Lz), on the
  node-centred field (the reference's ``reconstruct_temperature_DCT``,
  evaluated on the device), each end located where the linear interpolation
  between neighbouring nodes crosses the liquidus; and their differences.
  ``melt_pool_cells`` gives the same extents in whole cells of the
  cell-centred field.

Run it with ``python -m spectral_galerkin_heat_b200.precision`` (see --help);
the default is the 256 x 128 x 64 straight-track study with seeded power and
speed, once with one forcing pass per step and once with the evaporation
solved to its Picard fixed point.
"""
from __future__ import annotations

import argparse
import copy
import json
from types import SimpleNamespace
from typing import Dict, List, Optional, Sequence

import numpy as np

__all__ = ["melt_pool", "melt_pool_nodal", "compare_fields", "run_study", "run_volume_study"]


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


def _crossings(T_line: np.ndarray, x: np.ndarray, T_melt: float):
    """Ends of the region T >= T_melt along one node line: (lo, hi) positions
    with the outer crossings interpolated linearly between nodes, or None."""
    hot = np.nonzero(T_line >= T_melt)[0]
    if hot.size == 0:
        return None
    i0, i1 = int(hot[0]), int(hot[-1])

    def cross(a, b):  # node a is hot, node b is not
        ta, tb = T_line[a], T_line[b]
        return x[a] + (x[b] - x[a]) * (ta - T_melt) / (ta - tb)
    lo = x[i0] if i0 == 0 else cross(i0, i0 - 1)
    hi = x[i1] if i1 == len(x) - 1 else cross(i1, i1 + 1)
    return lo, hi


def melt_pool_nodal(T_nodes: np.ndarray, lengths, T_melt: float) -> Dict[str, float]:
    """Melt-pool extents on a node-centred field ``T_nodes`` of shape
    (nx+1, ny+1, nz+1) at nodes (j Lx/nx, k Ly/ny, l Lz/nz), as
    ``reconstruct_temperature_DCT`` returns it: length along x and width along
    y of the region T >= T_melt on the top face z = Lz, and depth of that
    region below the top face; the ends are interpolated linearly to the
    isotherm (zero when no node melts)."""
    T = np.asarray(T_nodes, dtype=np.float64)
    nx, ny, nz = (n - 1 for n in T.shape)
    Lx, Ly, Lz = (float(v) for v in lengths)
    xs, ys, zs = (np.linspace(0.0, L, n + 1) for L, n in ((Lx, nx), (Ly, ny), (Lz, nz)))
    top = T[:, :, nz]
    out = {"length": 0.0, "width": 0.0, "depth": 0.0}
    spans = [c for c in (_crossings(top[:, k], xs, T_melt) for k in range(ny + 1)) if c]
    if not spans:
        return out
    out["length"] = float(max(h for _, h in spans) - min(lo for lo, _ in spans))
    spans = [c for c in (_crossings(top[j, :], ys, T_melt) for j in range(nx + 1)) if c]
    out["width"] = float(max(h for _, h in spans) - min(lo for lo, _ in spans))
    depth = 0.0
    for j, k in zip(*np.nonzero(top >= T_melt)):
        col = T[j, k, ::-1]                       # from the top face down
        c = _crossings(col, Lz - zs[::-1], T_melt)
        depth = max(depth, c[1])
    out["depth"] = float(depth)
    return out


def compare_fields(T: np.ndarray, T_ref: np.ndarray, cell, T_melt: float,
                   nodes=None, nodes_ref=None, lengths=None) -> Dict[str, object]:
    """Error report of ``T`` against ``T_ref`` (both (nz, ny, nx), FP64), with
    the nodal melt pool when the node-centred fields are given."""
    dx, dy, dz = cell
    mp, mp_ref = melt_pool(T, dx, dy, dz, T_melt), melt_pool(T_ref, dx, dy, dz, T_melt)
    rep = {
        "rel_l2": float(np.linalg.norm(T - T_ref) / np.linalg.norm(T_ref)),
        "peak_T": float(T.max()), "peak_T_ref": float(T_ref.max()),
        "peak_T_err_K": float(T.max() - T_ref.max()),
        "melt_pool_cells": mp, "melt_pool_cells_ref": mp_ref,
    }
    if nodes is not None:
        mn, mn_ref = melt_pool_nodal(nodes, lengths, T_melt), melt_pool_nodal(nodes_ref, lengths, T_melt)
        rep.update(melt_pool=mn, melt_pool_ref=mn_ref,
                   melt_pool_err_m={k: mn[k] - mn_ref[k] for k in ("length", "width", "depth")})
    return rep


def run_study(cfg: dict, path, checkpoints: Sequence[int], picard: Optional[dict] = None,
              perturb: float = 1e-12, seed: int = 0) -> List[Dict[str, object]]:
    """Step the runs to each checkpoint and compare (see the module doc)."""
    import torch

    from . import kernels
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
    lengths = (Lx, Ly, Lz)
    geo = SimpleNamespace(size=lengths)
    T_melt = float(cfg["material"]["T_liquidus"])
    total = int(max(checkpoints))

    ref = B200SpectralSolver(None, copy.copy(ctx))
    ref.initialize()
    per = B200SpectralSolver(None, copy.copy(ctx))
    per.initialize()
    T0 = per.volume_temperature().cpu().numpy()
    rng = np.random.default_rng(seed)
    per.set_state(T0 * (1.0 + perturb * rng.standard_normal(T0.shape)))
    f32 = B200SpectralSolver(None, copy.copy(ctx), precision="fp32")
    f32.initialize()
    rnd = B200SpectralSolver(None, copy.copy(ctx))
    rnd.initialize()
    rnd.run(0.0, 1)
    rnd.state.a.copy_(rnd.state.a.to(torch.float32).to(torch.float64))
    ev = B200SpectralSolver(None, copy.copy(ctx))
    ev.initialize()
    mix = BatchSolver([copy.copy(ctx)], "mixed")
    mix.start(0, total, record=True)

    out, done = [], 0
    for cp in sorted(set(int(c) for c in checkpoints)):
        n = cp - done
        ref_m = ref.run(done * dt, n)
        per.run(done * dt, n)
        rnd.run(max(done, 1) * dt, cp - max(done, 1))
        f32_m = f32.run(done * dt, n)
        for i in range(done, cp):
            ev.run(i * dt, 1)
            ev.state.a.copy_(ev.state.a.to(torch.float32).to(torch.float64))
        mix.step(n)
        done = cp
        T_ref = ref.volume_temperature().cpu().numpy()
        T_per = per.volume_temperature().cpu().numpy()
        T_rnd = rnd.volume_temperature().cpu().numpy()
        T_ev = ev.volume_temperature().cpu().numpy()
        a_mix = mix.modes(0).to(torch.float64).contiguous()
        T_mix = ref.volume_temperature(a_mix).cpu().numpy()
        T_f32 = ref.volume_temperature(f32.state.a).cpu().numpy()
        nodes = {name: kernels.reconstruct_temperature_DCT(a, geo).cpu().numpy()
                 for name, a in (("ref", ref.state.a), ("per", per.state.a), ("rnd", rnd.state.a),
                                 ("ev", ev.state.a),
                                 ("mix", a_mix), ("f32", f32.state.a.clone()))}
        mm = mix.metrics(0)[-1]
        out.append({
            "step": cp,
            "picard_iters_fp64_last": ref_m[-1]["n_evap_iter"], "picard_iters_mixed_last": mm["n_evap_iter"],
            "T_surface_max_fp64": ref_m[-1]["T_surface_max"], "T_surface_max_mixed": mm["T_surface_max"],
            "mixed": compare_fields(T_mix, T_ref, cell, T_melt, nodes["mix"], nodes["ref"], lengths),
            "fp32": compare_fields(T_f32, T_ref, cell, T_melt, nodes["f32"], nodes["ref"], lengths),
            "picard_iters_fp32_last": f32_m[-1]["n_evap_iter"],
            "fp64_perturbed": compare_fields(T_per, T_ref, cell, T_melt, nodes["per"], nodes["ref"],
                                             lengths),
            "fp64_fp32_rounded": compare_fields(T_rnd, T_ref, cell, T_melt, nodes["rnd"], nodes["ref"],
                                                lengths),
            "fp64_fp32_every_step": compare_fields(T_ev, T_ref, cell, T_melt, nodes["ev"], nodes["ref"],
                                                   lengths),
            "tensor_core_error": mix.tensor_core_error(),
        })
    ref.finalize()
    per.finalize()
    rnd.finalize()
    ev.finalize()
    f32.finalize()
    mix.close()
    return out


def run_volume_study(cfg: dict, path, checkpoints: Sequence[int], mixed_tol: float = 1e-5,
                     perturb: float = 1e-12, seed: int = 0) -> List[Dict[str, object]]:
    """The nonlinear volume step (latent heat, T-dependent properties,
    evaporation, convection) in its single-instance plans: ``fp64`` at the
    configuration's Picard tolerance, ``mixed`` (split-BF16 tensor-core
    contractions, FP32 modal iterates, FP64 latent source, correction, fluxes
    and norms) and ``fp32`` (FP32 CUDA-core contractions) at ``mixed_tol``,
    ``fp64_mixed_tol`` (the FP64 plan at ``mixed_tol``: the part of the error
    that the looser Picard tolerance alone causes) and ``fp64_perturbed``
    (the FP64 plan from an initial field changed by ``perturb`` relative),
    compared at each checkpoint step as in
    :func:`run_study`. Each form's device time (CUDA events around its
    table-driven runs), mean Picard iterations and step statuses are reported
    beside the errors."""
    import ctypes as C

    import torch

    from . import _lib, kernels
    from .config import SimulationContext
    from .solver import B200SpectralSolver
    ctx = SimulationContext.from_dict(copy.deepcopy(cfg))
    ctx.laser_path = path
    Lx, Ly, Lz = cfg["domain"]["size"]
    cell = (Lx / ctx.num.nx, Ly / ctx.num.ny, Lz / ctx.num.nz)
    lengths = (Lx, Ly, Lz)
    geo = SimpleNamespace(size=lengths)
    T_melt = float(cfg["material"]["T_liquidus"])
    forms = {
        "fp64": B200SpectralSolver(None, copy.copy(ctx)),
        "fp64_perturbed": B200SpectralSolver(None, copy.copy(ctx)),
        "mixed": B200SpectralSolver(None, copy.copy(ctx), precision="mixed", convergence_tol=mixed_tol),
        "fp32": B200SpectralSolver(None, copy.copy(ctx), precision="fp32", convergence_tol=mixed_tol),
        "fp64_mixed_tol": B200SpectralSolver(None, copy.copy(ctx), convergence_tol=mixed_tol),
    }
    for s in forms.values():
        s.initialize()
    per = forms["fp64_perturbed"]
    T0 = per.volume_temperature().cpu().numpy()
    per.set_state(T0 * (1.0 + perturb * np.random.default_rng(seed).standard_normal(T0.shape)))
    total = int(max(checkpoints))
    osz = C.sizeof(_lib.SghStepOut)
    tables = {k: s.laser_table(0.0, total) for k, s in forms.items()}
    outs = {k: torch.zeros(total * osz, dtype=torch.uint8, device=s.state.workspace.device)
            for k, s in forms.items()}
    ms = {k: 0.0 for k in forms}
    out, done = [], 0
    for cp in sorted(set(int(c) for c in checkpoints)):
        n = cp - done
        for name, s in forms.items():
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(s.state.stream)
            s.run_table(tables[name], outs[name], n, start=done)
            e1.record(s.state.stream)
            torch.cuda.synchronize()
            ms[name] += e0.elapsed_time(e1)
        done = cp
        ref = forms["fp64"]
        T_ref = ref.volume_temperature().cpu().numpy()
        n_ref = kernels.reconstruct_temperature_DCT(ref.state.a, geo).cpu().numpy()
        row = {"step": cp}
        for name in ("mixed", "fp32", "fp64_mixed_tol", "fp64_perturbed"):
            a = forms[name].state.a.clone()
            row[name] = compare_fields(ref.volume_temperature(a).cpu().numpy(), T_ref, cell, T_melt,
                                       kernels.reconstruct_temperature_DCT(a, geo).cpu().numpy(), n_ref,
                                       lengths)
        timing = {}
        for k, s in forms.items():
            recs = s.decode_outs(outs[k][:done * osz].cpu().numpy().tobytes(), done)
            st = {}
            for r in recs:
                key = _lib.STEP_STATUS.get(r.status, str(r.status))
                st[key] = st.get(key, 0) + 1
            timing[k] = {"steps_per_s": done / (ms[k] * 1e-3),
                         "picard_iters_mean": float(np.mean([r.n_iter for r in recs])), "step_status": st}
        row["timing"] = timing
        out.append(row)
    for s in forms.values():
        s.finalize()
    return out


def main(argv=None):
    from . import workloads
    ap = argparse.ArgumentParser(description="mixed-precision vs FP64 error report")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--mesh", type=int, nargs=3, default=None,
                    help="grid (default 256 128 64; with --volume 128 64 32)")
    ap.add_argument("--checkpoints", type=int, nargs="+", default=None,
                    help="steps to compare at (default 20 100 500; with --volume 20 100 250 500 1000)")
    ap.add_argument("--volume", action="store_true",
                    help="the nonlinear raster (latent heat, T-dependent k and c_p, evaporation, "
                         "convection; Picard to 1e-8 in FP64) in the single-instance plans")
    ap.add_argument("--mixed-tol", type=float, default=1e-5, help="--volume: Picard tolerance of mixed/fp32")
    ap.add_argument("--out", default=None, help="write the JSON report here")
    args = ap.parse_args(argv)
    if args.volume:
        nx, ny, nz = args.mesh or (128, 64, 32)
        cps = args.checkpoints or [20, 100, 250, 500, 1000]
        cfg, path = workloads.nonlinear_raster(seed=args.seed, nx=nx, ny=ny, nz=nz, steps=max(cps))
        report = {"config": {"workload": "nonlinear raster", "mesh": [nx, ny, nz],
                             "domain_m": cfg["domain"]["size"], "seed": args.seed,
                             "dt_s": cfg["simulation"]["dt"],
                             "fp64_picard_tol": cfg["simulation"]["picard_tol"],
                             "mixed_picard_tol": args.mixed_tol},
                  "checkpoints": run_volume_study(cfg, path, cps, mixed_tol=args.mixed_tol, seed=args.seed)}
        text = json.dumps(report, indent=1)
        if args.out:
            with open(args.out, "w") as f:
                f.write(text)
        print(text)
        return
    nx, ny, nz = args.mesh or (256, 128, 64)
    args.checkpoints = args.checkpoints or [20, 100, 500]
    cfg, path = workloads.precision_track(seed=args.seed, nx=nx, ny=ny, nz=nz)
    forms = {
        "one_pass": None,
        "picard_converged": {"max_picard_iter": 400, "picard_omega": 0.1, "picard_tol": 1e-8},
    }
    report = {"config": {"mesh": [nx, ny, nz], "domain_m": cfg["domain"]["size"], "seed": args.seed,
                         "power_W": path.power, "speed_m_s": path.vx},
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
