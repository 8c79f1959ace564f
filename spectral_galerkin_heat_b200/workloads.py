"""Synthetic workloads: configuration dicts and laser paths.

Each function returns a config dict in the reference's YAML schema (plain SI
scalars) plus the :class:`LaserPath` that drives it. All randomness comes from
``numpy.random.default_rng(seed)``.

* ``straight_track``: 316L cuboid 2.0 x 1.0 x 0.5 mm, 64 x 32 x 16 modes,
  constant properties (k = 20, rho = 7900, c_p = 500), T0 = 300 K, Gaussian
  beam 200 W / 50 um / A = 0.35 on a straight track along x at y = 0.5 mm,
  1 m/s from x = 0.25 mm; evaporation on the top face only; 300 ETD1 steps of
  5 us; one forcing pass per step (``max_picard_iter = 1``, ``omega = 1``).
* ``nonlinear_raster``: same cuboid at 128 x 64 x 32 modes; k(T) = 15 + 20
  (T - 300)/2700 and c_p(T) = 450 + 350 (T - 300)/2700 on both phase branches
  (reference constants 25 and 625), rho = 7900; latent heat 2.7e5 J/kg over
  1658-1723 K (grid mode); evaporation plus top convection h = 10 W/m^2K;
  Picard to 1e-8 with omega = 0.1 (cap 400); 1000 steps of 2 us; 5-line
  bidirectional raster, 0.4 mm lines, 100 um hatch, 1 m/s, start jittered by
  U[-50, 50] um from the seed.
* ``precision_track``: 256 x 128 x 64 modes on a 4 x 2 x 1 mm cuboid with the
  straight-track physics; P ~ U[150, 400] W and v ~ U[0.5, 2] m/s from the
  seed; 500 steps of 5 us from x = 0.5 mm.
* ``uneven_batch``: many cuboids of uneven grid size for batched stepping:
  Nx from {64, 96, 128, 192, 256}, Ny = Nx/2, Nz from {16, 32, 64}, the
  64 x 32 x 16 cell size kept (Lx = 2 mm * Nx/64, Ly = Lx/2, Lz = 0.5 mm);
  straight-track physics with P ~ U[150, 400] W, v ~ U[0.5, 2] m/s and
  absorptivity ~ U[0.3, 0.45] per instance; Picard with the reference defaults
  (omega 0.1, tol 1e-4, cap 30).
* ``serving_stream``: a seeded Poisson stream of laser-scan solve requests
  (mean rate 200 requests/s): grids Nx from {64, 128, 256, 512}, Ny = Nx/2,
  Nz from {16, 32, 64} on the fixed 2 x 1 x 0.5 mm cuboid; straight-track
  physics (one forcing pass per step); 200-2000 steps of 5 us; P ~ U[150, 400]
  W and v ~ U[0.5, 2] m/s per request on a bidirectional raster (1.5 mm lines,
  50 um hatch) that keeps the beam on the part.
"""
from __future__ import annotations

import copy

import numpy as np

from .laser import RasterPath, StraightTrack

__all__ = ["MATERIAL_316L", "straight_track", "nonlinear_raster", "precision_track",
           "uneven_batch", "serving_stream", "serving_config", "scaled", "box_track",
           "example03", "MATERIAL_316L_TDEP"]

MATERIAL_316L = {
    "name": "316L", "rho": 7900.0, "k": 20.0, "Cp": 500.0, "L_f": 0.0,
    "T_solidus": 1658.0, "T_liquidus": 1723.0, "T0": 300.0,
    "DeltaH_LV": 7.416e6, "R_v": 150.774, "Pa": 101325.0, "T_boil": 3090.0,
}


def straight_track(nx=64, ny=32, nz=16, steps=300, dt=5e-6, size=(2e-3, 1e-3, 0.5e-3),
                   x0=0.25e-3, y0=None, speed=1.0, power=200.0, absorptivity=0.35):
    """Constant-property straight track; returns ``(cfg, path)``."""
    cfg = {
        "simulation": {"backend": "b200", "dtype": "float64", "dt": dt,
                       "duration": steps * dt, "max_picard_iter": 1, "picard_omega": 1.0},
        "domain": {"size": list(size), "mesh": [nx, ny, nz]},
        "material": dict(MATERIAL_316L),
        "laser": {"radius": 50e-6, "absorptivity": absorptivity, "power_nominal": power},
    }
    y = size[1] / 2.0 if y0 is None else y0
    return cfg, StraightTrack(x0, y, speed, 0.0, power)


def nonlinear_raster(nx=128, ny=64, nz=32, steps=1000, dt=2e-6, seed=0,
                     size=(2e-3, 1e-3, 0.5e-3), line_length=0.4e-3, hatch=100e-6,
                     n_lines=5, speed=1.0, power=200.0, tol=1e-8, omega=0.1, cap=400):
    """T-dependent raster with latent heat, evaporation and convection; ``(cfg, path)``."""
    mat = dict(MATERIAL_316L)
    mat.update({
        "k": {"solid": "15 + 20*(T - 300)/2700", "liquid": "15 + 20*(T - 300)/2700",
              "reference": 25.0},
        "Cp": {"solid": "450 + 350*(T - 300)/2700", "liquid": "450 + 350*(T - 300)/2700",
               "reference": 625.0},
        "rho": 7900.0, "L_f": 2.7e5, "h_conv_top": 10.0,
    })
    cfg = {
        "simulation": {"backend": "b200", "dtype": "float64", "dt": dt,
                       "duration": steps * dt, "max_picard_iter": cap,
                       "picard_tol": tol, "picard_omega": omega},
        "domain": {"size": list(size), "mesh": [nx, ny, nz]},
        "material": mat,
        "laser": {"radius": 50e-6, "absorptivity": 0.35, "power_nominal": power},
    }
    rng = np.random.default_rng(seed)
    jx, jy = rng.uniform(-50e-6, 50e-6, size=2)
    x_start = 0.5 * size[0] - 0.5 * line_length + jx
    y_start = 0.5 * size[1] - 0.5 * (n_lines - 1) * hatch + jy
    return cfg, RasterPath(x_start, y_start, line_length, hatch, n_lines, speed, power)


def box_track(nx=80, ny=48, nz=120, steps=140, dt=5e-6, size=(0.6e-3, 0.4e-3, 0.15e-3),
              refinement=2, box_size=(0.6e-3, 0.6e-3, 0.07e-3), x0=0.15e-3, y0=None,
              speed=0.4, power=120.0):
    """Box-mode single track with latent heat and bottom convection (the layout of
    the reference's example 02, ``simulations/examples/02_single_track.yaml``):
    constant 316L properties at 293 K, Picard at the reference defaults, latent
    heat on a laser-following fine box; ``(cfg, path)``."""
    cfg = {
        "simulation": {"backend": "b200", "dtype": "float64", "dt": dt, "duration": steps * dt},
        "domain": {"size": list(size), "mesh": [nx, ny, nz]},
        "fine_mesh": {"refinement": refinement, "box_size": list(box_size)},
        "material": {"name": "316L", "rho": 7957.5, "k": 13.851, "Cp": 497.89, "L_f": 2.677e5,
                     "T_solidus": 1674.15, "T_liquidus": 1697.15, "T0": 293.0,
                     "h_conv_bottom": 3000.0, "DeltaH_LV": 7.416e6, "R_v": 150.774,
                     "Pa": 101325.0, "T_boil": 3090.0},
        "laser": {"radius": 60e-6, "absorptivity": 0.30, "power_nominal": power},
    }
    y = size[1] / 2.0 if y0 is None else y0
    return cfg, StraightTrack(x0, y, speed, 0.0, power)


# Temperature-dependent 316L of the reference's example 03
# (``simulations/examples/03_nonlinear_tdep.yaml:54-96``): distinct solid and
# liquid branches blended by the liquid fraction, a quadratic rho(T), a liquid
# Cp given as a constant string, and the reference constants of that file.
MATERIAL_316L_TDEP = {
    "name": "316L",
    "k": {"solid": "9.248 + 0.01571 * T", "liquid": "12.41 + 0.003279 * T",
          "reference": 24.5075},
    "rho": {"solid": "8084.2 - 0.42086 * T - 3.8942e-5 * T**2",
            "liquid": "7432.7 + 0.039338 * T - 1.8007e-4 * T**2", "reference": 6896.2365},
    "Cp": {"solid": "458.98 + 0.1328 * T", "liquid": "769.86", "reference": 633.8752},
    "L_f": 2.677e5, "T_solidus": 1674.15, "T_liquidus": 1697.15, "T0": 293.0,
    "h_conv_bottom": 3000.0, "DeltaH_LV": 7.416e6, "R_v": 150.774, "Pa": 101325.0,
    "T_boil": 3090.0,
}


def example03(nx=100, ny=60, nz=96, steps=50, dt=4e-6, box=False, power=24.0):
    """The reference's example-03 layout: 0.5 x 0.3 x 0.12 mm box, the T-dependent
    316L block above, Picard capped at 80 with omega 0.31 (tolerance at the
    default), a 30 um / A = 0.3 beam moving along +x at 0.15 m/s from
    (0.2, 0.15) mm; ``box`` adds the example's refinement-2 fine box
    (0.2 x 0.15 x 0.04 mm). ``(cfg, path)``."""
    cfg = {
        "simulation": {"backend": "b200", "dtype": "float64", "dt": dt, "duration": steps * dt,
                       "max_picard_iter": 80, "picard_omega": 0.31},
        "domain": {"size": [0.5e-3, 0.3e-3, 0.12e-3], "mesh": [nx, ny, nz]},
        "material": copy.deepcopy(MATERIAL_316L_TDEP),
        "laser": {"radius": 30e-6, "absorptivity": 0.30, "power_nominal": power},
    }
    if box:
        cfg["fine_mesh"] = {"refinement": 2, "box_size": [0.2e-3, 0.15e-3, 0.04e-3]}
    return cfg, StraightTrack(0.2e-3, 0.15e-3, 0.15, 0.0, power)


def precision_track(seed=0, nx=256, ny=128, nz=64, steps=500, dt=5e-6):
    """Large straight track with seeded power and speed; ``(cfg, path)``."""
    rng = np.random.default_rng(seed)
    power = float(rng.uniform(150.0, 400.0))
    speed = float(rng.uniform(0.5, 2.0))
    return straight_track(nx, ny, nz, steps=steps, dt=dt, size=(4e-3, 2e-3, 1e-3),
                          x0=0.5e-3, speed=speed, power=power)


def uneven_batch(n=64, seed=0, steps=300, dt=5e-6, nx_choices=(64, 96, 128, 192, 256),
                 nz_choices=(16, 32, 64)):
    """``n`` seeded ``(cfg, path)`` pairs of uneven grid size (see the module docstring)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.choice(nx_choices))
        nz = int(rng.choice(nz_choices))
        ny = nx // 2
        power = float(rng.uniform(150.0, 400.0))
        speed = float(rng.uniform(0.5, 2.0))
        absorptivity = float(rng.uniform(0.3, 0.45))
        size = (2e-3 * nx / 64, 1e-3 * ny / 32, 0.5e-3)
        cfg, _ = straight_track(nx, ny, nz, steps=steps, dt=dt, size=size, power=power,
                                absorptivity=absorptivity)
        cfg["simulation"].update({"max_picard_iter": 30, "picard_omega": 0.1, "picard_tol": 1e-4})
        out.append((cfg, StraightTrack(0.3e-3, size[1] / 2.0, speed, 0.0, power)))
    return out


def serving_config(nx, ny, nz, dt=5e-6):
    """Config of one serving request class: straight-track physics, fixed cuboid."""
    cfg, _ = straight_track(nx, ny, nz, steps=1, dt=dt)
    return cfg


def serving_stream(n_requests=200, seed=0, rate=200.0, dt=5e-6, nx_choices=(64, 128, 256, 512),
                   nz_choices=(16, 32, 64), steps_range=(200, 2000)):
    """Seeded Poisson request stream: a list of dicts with ``arrival`` (s from the
    stream start), ``mesh`` (nx, ny, nz), ``steps``, ``cfg`` and ``path``."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        nx = int(rng.choice(nx_choices))
        nz = int(rng.choice(nz_choices))
        ny = nx // 2
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        power = float(rng.uniform(150.0, 400.0))
        speed = float(rng.uniform(0.5, 2.0))
        length, hatch = 1.5e-3, 50e-6
        n_lines = max(1, min(14, int(np.ceil(steps * dt * speed / length))))
        path = RasterPath(0.25e-3, 0.2e-3, length, hatch, n_lines, speed, power)
        out.append({"id": i, "arrival": t, "mesh": (nx, ny, nz), "steps": steps,
                    "cfg": serving_config(nx, ny, nz, dt), "path": path})
    return out


def scaled(cfg, nx, ny, nz, size=None, steps=None):
    """Copy of ``cfg`` with another mesh (and optionally domain size / step count)."""
    out = copy.deepcopy(cfg)
    out["domain"]["mesh"] = [nx, ny, nz]
    if size is not None:
        out["domain"]["size"] = list(size)
    if steps is not None:
        out["simulation"]["duration"] = steps * out["simulation"]["dt"]
    return out
