"""The drop-in against the reference's own objects (CPU only).

Imports the reference package from a checkout (``SGH_REFERENCE``, else a
directory ``reference`` beside this repository) with the stand-in modules of
``tests/golden/make_golden.py``, and checks that

* a ``SimulationContext`` built by the reference's own parser from a config
  gives the library exactly the ``sgh_config`` bytes that this package's
  parser gives for the same config (grid and box mode, constant and
  T-dependent materials, convection, super-Gaussian beams);
* a G-code path read by the reference's reader and by this package's reader
  give identical device laser tables;
* ``install_into_reference()`` makes the reference's ``get_backend("b200")``
  return the B200 backend and registers ``B200SpectralSolver`` as a
  ``HeatSolver`` of the reference, which resolves its Picard controls from a
  reference context as the reference solver does.

Skipped when no reference checkout is present (as on the GPU hosts).
"""
import copy
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_root():
    root = os.environ.get("SGH_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
    return root if os.path.isdir(os.path.join(root, "src", "spectral_galerkin_heat")) else None


pytestmark = pytest.mark.skipif(_reference_root() is None, reason="no reference checkout")


@pytest.fixture(scope="module")
def ref():
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden
    Ctx, Solver, Numpy = make_golden.import_reference(_reference_root())
    return Ctx


def _configs():
    from spectral_galerkin_heat_b200 import workloads
    out = {}
    out["track"], _ = workloads.straight_track()
    out["raster"], _ = workloads.nonlinear_raster()
    out["example03_grid"], _ = workloads.example03(nx=25, ny=15, nz=24)
    out["example03_box"], _ = workloads.example03(nx=25, ny=15, nz=24, box=True)
    out["box_track"], _ = workloads.box_track()
    cfg, _ = workloads.straight_track(nx=20, ny=18, nz=5)
    cfg["laser"].update({"profile": "super_gaussian", "super_gaussian_order": 4.0,
                         "r_x": 60e-6, "r_y": 40e-6, "cell_integrated": False})
    cfg["material"].update({"h_conv_top": 2.0e3, "h_conv_bottom": 5.0e3})
    cfg["simulation"].pop("max_picard_iter")
    out["supergauss_conv"] = cfg
    cfg = copy.deepcopy(out["track"])
    cfg["simulation"]["dtype"] = "float32"
    out["track_float32_parse"] = cfg
    return out


@pytest.mark.parametrize("name", sorted(_configs()))
def test_reference_context_gives_the_same_library_config(ref, name):
    from spectral_galerkin_heat_b200 import SimulationContext
    from spectral_galerkin_heat_b200.solver import B200SpectralSolver, make_config
    cfg = _configs()[name]
    ref_ctx = ref.from_dict(copy.deepcopy(cfg))
    ours = SimulationContext.from_dict(copy.deepcopy(cfg))
    picard = []
    for ctx in (ref_ctx, ours):
        s = B200SpectralSolver(None, ctx)
        s._resolve_picard_params(np.float64)
        picard.append((float(s.mixing_omega), float(s.convergence_tol), int(s.max_picard_iter)))
    assert picard[0] == picard[1]
    a = bytes(make_config(ref_ctx, *picard[0]))
    b = bytes(make_config(ours, *picard[1]))
    assert a == b
    assert (ref_ctx.num.n_steps, ref_ctx.num.dt) == (ours.num.n_steps, ours.num.dt)


def test_gcode_paths_of_both_readers_give_the_same_tables(ref):
    from spectral_galerkin_heat_b200 import SimulationContext, workloads
    from spectral_galerkin_heat_b200.laser import GCodeLaserPath, laser_table
    cfg, _ = workloads.straight_track(nx=24, ny=12, nz=8, dt=2e-6, size=(0.6e-3, 0.3e-3, 0.15e-3))
    cfg["laser"]["path"] = {"type": "gcode", "initial_position": [0.1, 0.2],
                            "file": os.path.join(ROOT, "tests", "golden", "scan_two_segments.gcode")}
    ref_ctx = ref.from_dict(copy.deepcopy(cfg))
    ours = SimulationContext.from_dict(copy.deepcopy(cfg))
    assert isinstance(ours.laser_path, GCodeLaserPath)
    assert type(ref_ctx.laser_path).__module__.startswith("spectral_galerkin_heat.")
    dt = ours.num.dt
    a = laser_table(ref_ctx.laser_path, 0.0, dt, 300)     # per-step get_state of the reference
    b = laser_table(ours.laser_path, 0.0, dt, 300)        # vectorised table
    assert a.tobytes() == b.tobytes()


def test_install_into_reference(ref):
    import spectral_galerkin_heat.backends as ref_backends
    from spectral_galerkin_heat.solvers.base import HeatSolver as RefHeatSolver

    from spectral_galerkin_heat_b200 import B200SpectralSolver, backends
    assert backends.install_into_reference() is True
    be = ref_backends.get_backend("b200")
    assert isinstance(be, backends.B200Backend) and be.name == "b200"
    assert issubclass(B200SpectralSolver, RefHeatSolver)
    assert isinstance(B200SpectralSolver(), RefHeatSolver)
    # the reference's own names are still its own
    assert ref_backends.get_backend("numpy").name == "numpy"
    # a reference context drives the B200 solver's set-up checks
    from spectral_galerkin_heat_b200 import workloads
    cfg, path = workloads.nonlinear_raster(nx=16, ny=8, nz=4)
    ref_ctx = ref.from_dict(cfg)
    ref_ctx.laser_path = path
    s = B200SpectralSolver(None, ref_ctx)
    s._resolve_picard_params(np.float64)
    assert (s.max_picard_iter, float(s.convergence_tol)) == (400, 1e-8)
