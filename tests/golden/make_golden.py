"""Generate the golden fixtures under ``tests/golden/`` from the reference itself.

Run where a checkout of the reference exists, naming its root (the directory
holding ``src/spectral_galerkin_heat``) with ``--reference`` or the
``SGH_REFERENCE`` environment variable::

    python tests/golden/make_golden.py --reference <checkout> [case ...]

The reference is the pure-Python package ``spectral_galerkin_heat``. Its module
imports pull in ``pint``, ``h5py``, ``matplotlib`` and ``pyfftw``, which are
absent from this image and unused on the time-step path, so empty stand-ins are
registered first (configs use plain SI numbers, so no unit conversion runs).
``NUMBA_CACHE_DIR`` is pointed at a temporary directory so nothing is written
into the reference tree.

For each case the reference ``SpectralSolver(NumpyBackend())`` is stepped
directly (no runner, so exactly ``steps`` calls of ``step(t, dt)`` with
``t = i * dt``), the CPU oracle (``oracle/sgh_oracle.py``) is stepped beside it
on the same context object, the two are required to agree, and the reference's
outputs are stored: modes at chosen steps (optionally a low-index block only),
the top-surface temperature, and per-step metrics. The ``outputs_*`` files hold
the reference's output reconstruction (node-centred field, point values,
profiles) of a case's modes. The versions of the libraries used are written
into every file.
"""
from __future__ import annotations

import copy
import os
import platform
import sys
import tempfile
import time
import types
import warnings
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
REF = None


def reference_root(argv=()):
    """The reference checkout named by ``--reference PATH`` or ``SGH_REFERENCE``."""
    argv = list(argv)
    if "--reference" in argv:
        i = argv.index("--reference")
        root = argv[i + 1]
        del argv[i:i + 2]
    else:
        root = os.environ.get("SGH_REFERENCE")
    if not root:
        raise SystemExit("name the reference checkout with --reference PATH or SGH_REFERENCE")
    root = Path(root)
    if not (root / "src" / "spectral_galerkin_heat").is_dir():
        raise SystemExit(f"{root} holds no src/spectral_galerkin_heat")
    return root, argv


def import_reference(root=None):
    global REF
    REF = Path(root) if root is not None else reference_root()[0]
    os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="sgh_numba_"))
    sys.dont_write_bytecode = True
    for name in ("pint", "h5py", "matplotlib", "matplotlib.pyplot", "pyfftw"):
        if name in sys.modules:
            continue
        mod = types.ModuleType(name)
        if name == "pint":
            class _Registry:
                def Quantity(self, *a, **k):
                    raise RuntimeError("unit conversion is not available (stand-in module)")
            mod.UnitRegistry = _Registry
        sys.modules[name] = mod
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    sys.path.insert(0, str(REF / "src"))
    sys.path.insert(0, str(REPO))
    import spectral_galerkin_heat as ref  # noqa: F401
    from spectral_galerkin_heat.backends import NumpyBackend
    from spectral_galerkin_heat.core.parameters import SimulationContext
    from spectral_galerkin_heat.solvers.spectral import SpectralSolver
    return SimulationContext, SpectralSolver, NumpyBackend


def cases():
    """Name -> (cfg, path, steps, snapshot steps, mode block or None)."""
    sys.path.insert(0, str(REPO))
    from spectral_galerkin_heat_b200 import workloads as W
    from spectral_galerkin_heat_b200.laser import FixedLaser, StraightTrack

    out = {}
    # straight track, full size: 300 steps of metrics; modes inside the
    # 60-step horizon over which this explicit (one-pass) scheme is not chaotic
    cfg, path = W.straight_track()
    out["track_64x32x16"] = (cfg, path, 300, [1, 30, 60], None)
    # nonlinear raster at reduced size on a reduced domain (melts in a few steps)
    cfg, path = W.nonlinear_raster(nx=32, ny=16, nz=8, size=(0.5e-3, 0.25e-3, 0.125e-3),
                                   line_length=0.1e-3, hatch=25e-6, steps=40)
    out["raster_32x16x8"] = (cfg, path, 40, [1, 10, 40], None)
    # nonlinear raster at the full mode count (the C2 grid), 20 steps, every mode stored
    cfg, path = W.nonlinear_raster(steps=20)
    out["raster_128x64x32"] = (cfg, path, 20, [20], None)
    # odd sizes, bottom + top convection, cell-integrated beam, T-dependent k only
    cfg, _ = W.nonlinear_raster(nx=13, ny=10, nz=6, size=(0.4e-3, 0.3e-3, 0.1e-3), steps=6,
                                tol=1e-9, omega=0.2, cap=200)
    cfg["material"]["h_conv_bottom"] = 5.0e3
    cfg["material"]["h_conv_top"] = 2.0e3
    cfg["material"]["Cp"] = 500.0
    cfg["laser"]["cell_integrated"] = True
    path = StraightTrack(0.1e-3, 0.14e-3, 0.7, 0.3, 180.0)
    out["odd_13x10x6_conv"] = (cfg, path, 6, [1, 6], None)
    # constant properties with latent heat (latent source without the property model)
    cfg, _ = W.straight_track(nx=24, ny=12, nz=8, steps=8, dt=2e-6,
                              size=(0.6e-3, 0.3e-3, 0.15e-3))
    cfg["material"]["L_f"] = 2.7e5
    cfg["simulation"].update({"max_picard_iter": 400, "picard_omega": 0.1, "picard_tol": 1e-8})
    path = StraightTrack(0.2e-3, 0.15e-3, 0.8, 0.0, 220.0)
    out["latent_const_24x12x8"] = (cfg, path, 8, [8], None)
    # super-Gaussian beam, elliptical, reference Picard defaults, laser moves in y
    cfg, _ = W.straight_track(nx=20, ny=18, nz=5, steps=5, dt=3e-6,
                              size=(0.5e-3, 0.45e-3, 0.1e-3))
    cfg["laser"].update({"profile": "super_gaussian", "super_gaussian_order": 4.0,
                         "r_x": 60e-6, "r_y": 40e-6})
    cfg["simulation"].pop("max_picard_iter")
    cfg["simulation"].pop("picard_omega")
    path = StraightTrack(0.25e-3, 0.1e-3, 0.0, 1.2, 250.0)
    out["supergauss_20x18x5"] = (cfg, path, 5, [5], None)
    # laser off: the field must stay at T0
    cfg, _ = W.straight_track(nx=8, ny=6, nz=4, steps=3)
    path = FixedLaser(1e-3, 0.5e-3, 200.0, is_on=False)
    out["laser_off_8x6x4"] = (cfg, path, 3, [3], None)
    # box mode, constant properties: a window narrower than the domain in x and
    # y, sliding diagonally (non-integer history shifts), partial depth
    cfg, _ = W.straight_track(nx=24, ny=12, nz=8, steps=8, dt=2e-6,
                              size=(0.6e-3, 0.3e-3, 0.15e-3))
    cfg["material"]["L_f"] = 2.7e5
    cfg["simulation"].update({"max_picard_iter": 400, "picard_omega": 0.1, "picard_tol": 1e-8})
    cfg["fine_mesh"] = {"refinement": 2, "box_size": [0.2e-3, 0.15e-3, 0.05e-3]}
    path = StraightTrack(0.2e-3, 0.13e-3, 2.0, 1.0, 220.0)
    out["box_const_24x12x8"] = (cfg, path, 8, [1, 8], None)
    # a box too shallow and narrow for the pool: the truncation warning fires
    cfg = copy.deepcopy(cfg)
    cfg["fine_mesh"] = {"refinement": 2, "box_size": [0.06e-3, 0.2e-3, 0.02e-3]}
    cfg["simulation"]["duration"] = 5 * 2e-6
    out["box_shallow_24x12x8"] = (cfg, path, 5, [5], None)
    # box mode with the T-dependent model (property correction) and convection
    cfg, path = W.nonlinear_raster(nx=16, ny=12, nz=8, size=(0.4e-3, 0.3e-3, 0.1e-3),
                                   line_length=0.1e-3, hatch=25e-6, steps=6)
    cfg["fine_mesh"] = {"refinement": 3, "box_size": [0.15e-3, 0.1e-3, 0.04e-3]}
    out["box_tdep_16x12x8"] = (cfg, path, 6, [6], None)
    # box mode at refinement 1 over the whole domain (the equivalence with grid
    # mode that the reference tests), bottom convection, laser at rest
    cfg, path = W.box_track(nx=20, ny=12, nz=30, steps=6, size=(0.6e-3, 0.4e-3, 0.15e-3),
                            refinement=1, box_size=(0.6e-3, 0.4e-3, 0.15e-3),
                            x0=0.3e-3, y0=0.2e-3, speed=0.0)
    cfg["simulation"]["max_picard_iter"] = 80
    out["box_full_r1_20x12x30"] = (cfg, path, 6, [6], None)
    # the material block of the reference's example 03 (distinct solid and
    # liquid polynomials, quadratic rho(T), a constant-string liquid Cp) on a
    # reduced grid of its 0.5 x 0.3 x 0.12 mm box, omega 0.31, in grid mode and
    # in box mode; the track melts from the fourth step on
    cfg, path = W.example03(nx=25, ny=15, nz=24, steps=10)
    out["tdep03_grid_25x15x24"] = (cfg, path, 10, [5, 10], None)
    cfg, path = W.example03(nx=25, ny=15, nz=24, steps=10, box=True)
    out["tdep03_box_25x15x24"] = (cfg, path, 10, [5, 10], None)
    # G-code laser paths (float32 positions and velocities): the path is read
    # from the config (path None here), so each side uses its own G-code
    # reader on the same file. One-pass track in grid mode, and box mode.
    gcode = {"type": "gcode", "file": str(HERE / "scan_two_segments.gcode"),
             "initial_position": [0.1, 0.2]}
    cfg, _ = W.straight_track(nx=30, ny=16, nz=8, steps=40, dt=2e-6,
                              size=(0.6e-3, 0.3e-3, 0.15e-3))
    cfg["laser"]["path"] = dict(gcode)
    out["gcode_track_30x16x8"] = (cfg, None, 40, [20, 40], None)
    cfg, _ = W.straight_track(nx=24, ny=12, nz=8, steps=12, dt=2e-6,
                              size=(0.6e-3, 0.3e-3, 0.15e-3))
    cfg["material"]["L_f"] = 2.7e5
    cfg["simulation"].update({"max_picard_iter": 400, "picard_omega": 0.1, "picard_tol": 1e-8})
    cfg["fine_mesh"] = {"refinement": 2, "box_size": [0.2e-3, 0.15e-3, 0.05e-3]}
    cfg["laser"]["path"] = dict(gcode)
    out["gcode_box_24x12x8"] = (cfg, None, 12, [6, 12], None)
    return out


def run_case(name, spec, Ctx, Solver, Numpy):
    sys.path.insert(0, str(REPO))
    from oracle.sgh_oracle import OracleSolver

    cfg, path, steps, snaps, block = spec
    ctx = Ctx.from_dict(copy.deepcopy(cfg))
    if path is not None:
        ctx.laser_path = path
    ref = Solver(Numpy(), ctx)
    ref.initialize()
    orc = OracleSolver(ctx)
    orc.initialize()
    dt = ctx.num.dt
    rec = {k: [] for k in ("T_surface_max", "P_laser", "n_evap_iter", "picard_converged",
                           "picard_rel_err")}
    files = {}
    worst = 0.0
    t0 = time.time()
    box_flags = []
    for i in range(steps):
        t = i * dt
        _, m = ref.step(t, dt)
        _, mo = orc.step(t, dt)
        box_flags.append(orc.box_flags)
        for k in rec:
            rec[k].append(float(m[k]))
        a = np.array(ref.state.a, dtype=np.float64, copy=True)
        if (i + 1) in snaps:
            rel = float(np.linalg.norm(orc.a - a) / np.linalg.norm(a))
            worst = max(worst, rel)
            assert rel < 1e-12, f"{name}: oracle differs from the reference at step {i+1}: {rel}"
            assert mo["n_evap_iter"] == int(m["n_evap_iter"]), f"{name}: Picard count differs"
            key = f"modes_step{i+1}"
            files[key] = a if block is None else a[:block[0], :block[1], :block[2]].copy()
            files[f"modes_norm_step{i+1}"] = np.array(np.linalg.norm(a))
            files[f"surface_step{i+1}"] = np.asarray(
                orc.surface_T(a, top=True), dtype=np.float64)
    for k, v in rec.items():
        files[f"metric_{k}"] = np.asarray(v)
    fm = getattr(ref.state, "fine_mesh", None)
    if fm is not None:
        # box history and window bases after the last step
        T_ref, Q_ref = np.asarray(fm.T_prev, np.float64), np.asarray(fm.Q_prev, np.float64)
        relT = float(np.linalg.norm(orc.box.T_prev - T_ref) / np.linalg.norm(T_ref))
        scaleQ = max(float(np.max(np.abs(Q_ref))), 1e-300)
        errQ = float(np.max(np.abs(orc.box.Q_prev - Q_ref))) / scaleQ
        for a in range(2):
            assert np.array_equal(np.asarray(fm.B_fine[a]), orc.box.B_fine[a]), f"{name}: window {a}"
        assert relT < 1e-12 and errQ < 1e-9, f"{name}: box history differs: {relT} {errQ}"
        worst = max(worst, relT)
        files["box_T_prev"] = T_ref
        files["box_Q_prev"] = Q_ref
        files["box_window"] = np.array(orc.box.window)
        warned = bool(ref._latent_truncation_warned)
        assert warned == any(box_flags), f"{name}: truncation check differs"
        files["box_truncation_warned"] = np.array(warned)
        files["box_flags"] = np.array(box_flags, dtype=np.int32)
        files["box_shape"] = np.array(orc.box.shape)
    import numba
    import scipy
    files["meta"] = np.array(str({
        "case": name, "steps": steps, "snapshots": snaps, "block": block, "dt": dt,
        "numpy": np.__version__, "scipy": scipy.__version__, "numba": numba.__version__,
        "python": platform.python_version(), "oracle_vs_reference_worst_relL2": worst,
    }))
    np.savez_compressed(HERE / f"{name}.npz", **files)
    print(f"{name}: {steps} steps in {time.time()-t0:.1f}s, oracle vs reference worst "
          f"rel L2 {worst:.2e}")


def output_cases():
    """Name -> (case of :func:`cases`, steps): the modes on which the reference's
    output reconstruction is evaluated."""
    return {"outputs_odd_13x10x6": ("odd_13x10x6_conv", 6),
            "outputs_raster_32x16x8": ("raster_32x16x8", 40)}


def run_outputs(name, case, steps, Ctx, Solver, Numpy):
    """Step the reference to ``steps`` and store its output reconstruction of
    the modes: the node-centred field (``reconstruct_temperature_DCT``), values
    at seeded points partly outside the domain
    (``reconstruct_temperature_volume_at_points``) and the three profiles for
    ``center="laser"`` and ``"hotspot"`` (``save_temp_profiles``); the oracle's
    restatement is required to agree."""
    sys.path.insert(0, str(REPO))
    from spectral_galerkin_heat.physics import spectral_helpers as H

    from oracle.sgh_oracle import nodal_temperature, points_temperature, temp_profiles
    cfg, path, *_ = cases()[case]
    ctx = Ctx.from_dict(copy.deepcopy(cfg))
    ctx.laser_path = path
    ref = Solver(Numpy(), ctx)
    ref.initialize()
    dt = ctx.num.dt
    for i in range(steps):
        ref.step(i * dt, dt)
    a = np.array(ref.state.a, dtype=np.float64, copy=True)
    st = ref.state
    lengths = (float(ctx.geom.size.x), float(ctx.geom.size.y), float(ctx.geom.size.z))
    files = {"modes": a, "lengths": np.array(lengths)}
    nodal = np.asarray(H.reconstruct_temperature_DCT(a, st), dtype=np.float64)
    rng = np.random.default_rng(7)
    coords = rng.uniform(-0.1, 1.1, size=(64, 3)) * np.array(lengths)
    pts = np.asarray(H.reconstruct_temperature_volume_at_points(a, ctx.num, ctx.geom, st, coords))
    lp = path.get_state(steps * dt, dt)
    files.update(nodal=nodal, coords=coords, points=pts, laser_position=np.array([lp.x, lp.y]))

    def rel(x, y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))
    worst = max(rel(nodal_temperature(a, lengths), nodal), rel(points_temperature(a, lengths, coords), pts))
    surface = np.asarray(ref.kernels.reconstruct_surface_temperature(a, st)) \
        if hasattr(ref, "kernels") else None
    for center, pos in (("laser", (lp.x, lp.y)), ("hotspot", None)):
        prof = H.save_temp_profiles(a, ctx.num, ctx.geom, st, pos, center=center, num_points=40)
        if surface is None:
            from oracle.sgh_oracle import OracleSolver
            o = OracleSolver(ctx)
            o.initialize()
            surface = o.surface_T(a, top=True)
        mine = temp_profiles(a, lengths, surface, pos, center=center, num_points=40)
        for key in "xyz":
            c, T = prof[key]
            files[f"profile_{center}_{key}_coords"] = np.asarray(c)
            files[f"profile_{center}_{key}_T"] = np.asarray(T)
            worst = max(worst, rel(mine[key][1], np.asarray(T)))
    assert worst < 1e-12, f"{name}: oracle differs from the reference output reconstruction: {worst}"
    import scipy
    files["meta"] = np.array(str({"case": case, "steps": steps, "numpy": np.__version__,
                                  "scipy": scipy.__version__, "oracle_vs_reference_worst_relL2": worst}))
    np.savez_compressed(HERE / f"{name}.npz", **files)
    print(f"{name}: outputs of {case} after {steps} steps, oracle vs reference worst rel L2 {worst:.2e}")


def run_gcode_states(name="gcode_states"):
    """The reference's own G-code reader (``io_utils/gcode_path.py``) on
    ``scan_two_segments.gcode``: laser states at ``t = i*dt`` over every
    segment, the jump with the beam off and the time after the last segment,
    for two step sizes and ``dt = 0``."""
    from spectral_galerkin_heat.io_utils.gcode_path import GCodeLaserPath as RefGCode
    path = RefGCode(str(HERE / "scan_two_segments.gcode"), initial_position=(0.1, 0.2))
    files = {}
    for tag, dt, n in (("dt2", 2e-6, 300), ("dt37", 3.7e-6, 170), ("dt0", 0.0, 50)):
        times = [i * (dt if dt else 1.3e-5) for i in range(n)]
        recs = [path.get_state(t, dt) for t in times]
        assert all(isinstance(r.x, np.float32) and isinstance(r.v[0], np.float32) for r in recs)
        files[f"{tag}_times"] = np.array(times)
        files[f"{tag}_xy"] = np.array([(r.x, r.y) for r in recs], dtype=np.float32)
        files[f"{tag}_v"] = np.array([r.v for r in recs], dtype=np.float32)
        files[f"{tag}_power"] = np.array([r.power for r in recs], dtype=np.float32)
        files[f"{tag}_on"] = np.array([r.is_on for r in recs])
        files[f"{tag}_dt"] = np.array(dt)
    files["meta"] = np.array(str({"gcode": "scan_two_segments.gcode", "initial_position": (0.1, 0.2),
                                  "numpy": np.__version__}))
    np.savez_compressed(HERE / f"{name}.npz", **files)
    print(f"{name}: reference G-code states stored")


def main(argv):
    warnings.simplefilter("ignore")
    root, argv = reference_root(argv)
    Ctx, Solver, Numpy = import_reference(root)
    sel = set(argv[1:])
    for name, spec in cases().items():
        if sel and name not in sel:
            continue
        run_case(name, spec, Ctx, Solver, Numpy)
    for name, (case, steps) in output_cases().items():
        if sel and name not in sel:
            continue
        run_outputs(name, case, steps, Ctx, Solver, Numpy)
    if not sel or "gcode_states" in sel:
        run_gcode_states()


if __name__ == "__main__":
    main(sys.argv)
