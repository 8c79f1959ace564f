"""Simulation configuration for the B200 backend.

Mirrors the configuration objects that the reference solver consumes
(``core/parameters.py``: ``NumParams`` :125-184, ``MaterialParams`` :186-276,
``GeomParams`` :278-298, ``LaserParams`` :300-350, ``SimulationContext`` :482-682;
``core/vector.py``: ``Vec3``) with the same field names, the same YAML schema and
the same parse-time arithmetic, so that a config dict read by the reference
yields the same numbers here:

* ``dt`` is re-derived as ``t_end / round(t_end / dt_nominal)`` so that
  ``n_steps * dt == t_end`` (``core/parameters.py:545-549``);
* scalar material / laser values are cast to the configured precision;
* a temperature-dependent property needs an explicit ``reference:`` key, and
  the scalar ``k``/``rho``/``Cp`` fields then hold those reference constants
  (``core/parameters.py:593-630``).

Units: a value may be a plain SI number or a ``{value, unit}`` mapping whose
unit is the SI unit itself (no unit conversion library is used; any other unit
raises ``ValueError``).

The solver only reads these objects by attribute, so the reference's own
``SimulationContext`` instances are accepted as well.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Optional

import numpy as np

from .laser import LaserPath, LaserState  # noqa: F401  (re-exported)
from .properties import MaterialModel

__all__ = [
    "Vec3", "NumParams", "MaterialParams", "GeomParams", "LaserParams",
    "FineMeshParams", "SimulationContext", "resolve_dtype",
]


@dataclass(frozen=True, slots=True)
class Vec3:
    """Immutable ``(x, y, z)`` triple; iterates in x, y, z order."""

    x: Any
    y: Any
    z: Any

    def __iter__(self):
        return iter((self.x, self.y, self.z))

    def __getitem__(self, i):
        return (self.x, self.y, self.z)[i]

    def zyx(self) -> "Vec3":
        """The triple in array-index order ``(z, y, x)``."""
        return Vec3(self.z, self.y, self.x)

    def map(self, f) -> "Vec3":
        return Vec3(f(self.x), f(self.y), f(self.z))

    def __truediv__(self, other):
        if isinstance(other, Vec3):
            return Vec3(self.x / other.x, self.y / other.y, self.z / other.z)
        return Vec3(self.x / other, self.y / other, self.z / other)

    def __mul__(self, other):
        if isinstance(other, Vec3):
            return Vec3(self.x * other.x, self.y * other.y, self.z * other.z)
        return Vec3(self.x * other, self.y * other, self.z * other)


_DTYPES = {"float32": np.float32, "float64": np.float64}


def resolve_dtype(name) -> type:
    """``"float32"`` / ``"float64"`` -> numpy scalar type; ``ValueError`` otherwise."""
    key = str(name).lower()
    if key not in _DTYPES:
        raise ValueError(
            f"Unknown dtype: {name!r}. Choose one of: {', '.join(sorted(_DTYPES))}.")
    return _DTYPES[key]


@dataclass
class NumParams:
    """Time step, mode counts and Picard controls (``None`` = solver default)."""

    dt: float
    nx: int
    ny: int
    nz: int
    t_end: float = 0.0
    n_steps: int = 0
    dt_nominal: float = 0.0
    update_interval: float = 1e-3
    save_all: bool = False
    max_picard_iter: Optional[int] = None
    picard_tol: Optional[float] = None
    picard_omega: Optional[float] = None
    dtype: Any = np.float64


@dataclass
class MaterialParams:
    """Thermophysical constants (SI). With a T-dependent ``model`` the scalar
    ``rho``/``k``/``Cp`` are the reference constants of the ETD1 propagators."""

    name: str = "Material"
    rho: float = 1.0
    k: float = 1.0
    Cp: float = 1.0
    L_f: float = 0.0
    T_solidus: float = 0.0
    T_liquidus: float = 0.0
    Pa: float = 0.0
    R_v: float = 0.0
    T_boil: float = 0.0
    DeltaH_LV: float = 0.0
    T0: float = 0.0
    h_conv_top: float = 0.0
    h_conv_bottom: float = 0.0
    model: Optional[MaterialModel] = None

    @property
    def diff(self) -> float:
        return self.k / (self.rho * self.Cp)


@dataclass
class GeomParams:
    """Cuboid ``[0,Lx]x[0,Ly]x[0,Lz]`` with ``n`` cells per axis; ``d = size / n``."""

    size: Vec3
    n: Vec3
    d: Vec3 = field(init=False)

    def __post_init__(self):
        self.d = self.size / self.n


@dataclass
class LaserParams:
    """Beam parameters; ``r_x``/``r_y`` default to ``radius``."""

    radius: float
    absorptivity: float
    power: float = 0.0
    profile: str = "gaussian"
    r_x: float = 0.0
    r_y: float = 0.0
    super_gaussian_order: float = 2.0
    cell_integrated: bool = False

    def __post_init__(self):
        if not self.r_x:
            self.r_x = self.radius
        if not self.r_y:
            self.r_y = self.radius

    @property
    def ref_area(self) -> float:
        return self.r_x * self.r_y


@dataclass
class FineMeshParams:
    """Laser-following refined sub-box (box mode, ``core/parameters.py:391-410``):
    ``refinement`` fine cells per coarse cell on each axis, ``box_size`` the
    box extents in metres. ``None`` on the context selects grid mode."""

    refinement: int = 4
    box_size: Vec3 = Vec3(0.9e-3, 0.9e-3, 0.04e-3)


_SECTION_KEYS = {
    "simulation": {"name", "backend", "dtype", "dt", "duration", "update_interval",
                   "max_picard_iter", "picard_tol", "picard_omega"},
    "domain": {"size", "mesh"},
    "material": {"name", "rho", "k", "Cp", "L_f", "T_solidus", "T_liquidus", "T0",
                 "Pa", "R_v", "T_boil", "DeltaH_LV", "h_conv_top", "h_conv_bottom"},
    "laser": {"radius", "absorptivity", "power_nominal", "profile", "r_x", "r_y",
              "super_gaussian_order", "cell_integrated", "path"},
    "fine_mesh": {"refinement", "box_size"},
}
_PASSTHROUGH = {"io", "post_processing"}

# SI unit spellings accepted in a {value, unit} mapping, per target quantity.
_SI_SPELLINGS = {
    "m": {"m"}, "s": {"s"}, "K": {"K", "kelvin"}, "W": {"W"}, "Pa": {"Pa"},
    "kg/m3": {"kg/m3", "kg/m**3", "kg / m**3", "kg/m^3"},
    "W/mK": {"W/(m.K)", "W/(m*K)", "W / (m * K)", "W/m/K", "W/(m K)"},
    "J/kgK": {"J/(kg.K)", "J/(kg*K)", "J / (kg * K)", "J/kg/K", "J/(kg K)"},
    "J/kg": {"J/kg", "J / kg"},
    "W/m2K": {"W/(m2.K)", "W/(m**2*K)", "W / (m**2 * K)", "W/m2/K", "W/(m^2.K)"},
}


def _scalar(raw, si=None) -> float:
    if isinstance(raw, dict):
        unit = raw.get("unit")
        if unit and si is not None and unit.strip() not in _SI_SPELLINGS[si]:
            raise ValueError(
                f"Unit {unit!r} is not the SI unit {si!r}; this backend reads SI values only.")
        return float(raw["value"])
    if isinstance(raw, bool) or not isinstance(raw, (int, float, np.floating, np.integer)):
        raise TypeError(f"Cannot extract a value from type {type(raw)}")
    return float(raw)


def _vector(raw, si=None) -> list:
    if isinstance(raw, dict):
        unit = raw.get("unit")
        if unit and si is not None and unit.strip() not in _SI_SPELLINGS[si]:
            raise ValueError(
                f"Unit {unit!r} is not the SI unit {si!r}; this backend reads SI values only.")
        return [float(v) for v in raw["value"]]
    if isinstance(raw, (list, tuple)):
        return [_scalar(v, si) for v in raw]
    raise TypeError(f"Cannot extract a vector from type {type(raw)}")


def _validate(cfg: dict) -> None:
    known = set(_SECTION_KEYS) | _PASSTHROUGH
    for section in cfg:
        if section not in known:
            raise ValueError(f"Unknown config section {section!r}. "
                             f"Valid sections: {', '.join(sorted(known))}.")
    for section, allowed in _SECTION_KEYS.items():
        body = cfg.get(section)
        if isinstance(body, dict):
            for key in body:
                if key not in allowed:
                    raise ValueError(
                        f"Unknown key {key!r} in the {section!r} config section. "
                        f"Valid keys: {', '.join(sorted(allowed))}.")


@dataclass
class SimulationContext:
    """Numerics, material, geometry, laser and laser path of one solve."""

    num: NumParams
    mat: MaterialParams
    geom: GeomParams
    laser: LaserParams
    laser_path: Optional[LaserPath]
    io: dict = field(default_factory=dict)
    backend: str = "b200"
    fine: Optional[FineMeshParams] = None

    @classmethod
    def from_dict(cls, cfg: dict, config_dir: Optional[str] = None) -> "SimulationContext":
        """Parse a config dict with the reference's schema.

        The laser path is left ``None`` unless the config names a G-code file,
        which this backend does not parse: set ``ctx.laser_path`` to a
        :class:`LaserPath` instead.
        """
        _validate(cfg)
        sim = cfg.get("simulation", {})
        real_t = resolve_dtype(sim.get("dtype", "float32"))
        dom = cfg.get("domain", {})
        Lx, Ly, Lz = _vector(dom["size"], "m")
        nx, ny, nz = _vector(dom["mesh"])
        t_end = _scalar(sim.get("duration", 0.01), "s")
        dt_nominal = float(real_t(_scalar(sim["dt"], "s")))
        n_steps = round(t_end / dt_nominal)
        dt = t_end / n_steps
        num = NumParams(
            dt=dt, nx=int(nx), ny=int(ny), nz=int(nz), t_end=t_end, n_steps=n_steps,
            dt_nominal=dt_nominal,
            update_interval=_scalar(sim.get("update_interval", 1e-3), "s"),
            max_picard_iter=(int(sim["max_picard_iter"])
                             if sim.get("max_picard_iter") is not None else None),
            picard_tol=(float(sim["picard_tol"]) if sim.get("picard_tol") is not None else None),
            picard_omega=(float(sim["picard_omega"])
                          if sim.get("picard_omega") is not None else None),
            dtype=real_t,
        )
        geom = GeomParams(size=Vec3(Lx, Ly, Lz), n=Vec3(int(nx), int(ny), int(nz)))

        fine_cfg = cfg.get("fine_mesh")
        fine = None
        if fine_cfg is not None:
            box = fine_cfg.get("box_size", (0.9e-3, 0.9e-3, 0.04e-3))
            bx = [_scalar(v, "m") for v in box]
            fine = FineMeshParams(refinement=int(_scalar(fine_cfg.get("refinement", 4))),
                                  box_size=Vec3(*bx))

        m = cfg.get("material", {})
        T_sol = real_t(_scalar(m.get("T_solidus", 0.0), "K"))
        T_liq = real_t(_scalar(m.get("T_liquidus", 0.0), "K"))
        T0 = real_t(_scalar(m.get("T0", 0.0), "K"))
        T_boil = real_t(_scalar(m.get("T_boil", 0.0), "K"))
        model = MaterialModel.from_config(m, float(T_sol), float(T_liq))
        units = {"k": "W/mK", "rho": "kg/m3", "Cp": "J/kgK"}
        if model is None:
            rho = real_t(_scalar(m["rho"], "kg/m3"))
            k = real_t(_scalar(m["k"], "W/mK"))
            cp = real_t(_scalar(m["Cp"], "J/kgK"))
        else:
            refs, missing = {}, []
            for key, prop in (("k", model.k), ("rho", model.rho), ("Cp", model.c)):
                spec = m.get(key)
                branched = isinstance(spec, dict) and ("solid" in spec or "liquid" in spec)
                if branched and not prop.is_constant:
                    if "reference" not in spec:
                        missing.append(key)
                        continue
                    refs[key] = real_t(_scalar(spec["reference"], units[key]))
                else:
                    refs[key] = real_t(float(prop(float(T0))))
            if missing:
                rec = dict(zip(("k", "rho", "Cp"),
                               model.recommended_references(float(T0), float(T_boil))))
                hint = ", ".join(f"{k}.reference={rec[k]:g}" for k in missing)
                raise ValueError(
                    f"Temperature-dependent material property {missing} needs an explicit "
                    f"'reference:' key inside its block. Recommended values: {hint}.")
            k, rho, cp = refs["k"], refs["rho"], refs["Cp"]
        mat = MaterialParams(
            name=m.get("name", "Material"), rho=rho, k=k, Cp=cp,
            L_f=real_t(_scalar(m.get("L_f", 0.0), "J/kg")),
            T_solidus=T_sol, T_liquidus=T_liq,
            Pa=real_t(_scalar(m.get("Pa", 0.0), "Pa")),
            R_v=real_t(_scalar(m.get("R_v", 0.0), "J/kgK")),
            T_boil=T_boil,
            DeltaH_LV=real_t(_scalar(m.get("DeltaH_LV", 0.0), "J/kg")),
            T0=T0,
            h_conv_top=real_t(_scalar(m.get("h_conv_top", 0.0), "W/m2K")),
            h_conv_bottom=real_t(_scalar(m.get("h_conv_bottom", 0.0), "W/m2K")),
            model=model,
        )
        lc = cfg.get("laser", {})
        laser = LaserParams(
            radius=real_t(_scalar(lc["radius"], "m")),
            absorptivity=real_t(_scalar(lc["absorptivity"])),
            power=real_t(_scalar(lc["power_nominal"], "W")),
            profile=str(lc.get("profile", "gaussian")),
            r_x=real_t(_scalar(lc.get("r_x", 0.0), "m")),
            r_y=real_t(_scalar(lc.get("r_y", 0.0), "m")),
            super_gaussian_order=_scalar(lc.get("super_gaussian_order", 2.0)),
            cell_integrated=bool(lc.get("cell_integrated", False)),
        )
        path_cfg = lc.get("path", {}) or {}
        if str(path_cfg.get("type", "")).lower() == "gcode":
            raise ValueError("G-code laser paths are not parsed by this backend; "
                             "assign a LaserPath to context.laser_path instead.")
        return cls(num=num, mat=mat, geom=geom, laser=laser, laser_path=None,
                   io=cfg.get("io", {}), backend=str(sim.get("backend", "b200")).lower(),
                   fine=fine)

