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

import os
from dataclasses import dataclass, field
from typing import Any, Optional

import numpy as np

from .laser import GCodeLaserPath, LaserPath, LaserState  # noqa: F401  (re-exported)
from .properties import MaterialModel, TempProperty

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


# ---------------------------------------------------------------------------
# Schema. Each section maps its keys to a reader: how the raw value is turned
# into a number (``kind``), the SI unit a ``{value, unit}`` mapping must carry
# (``unit``) and the default of an absent key (``_NEED`` = the key is
# required). The keys and defaults are the reference's schema
# (``core/parameters.py:415-437, 514-682``); the reading machinery is this
# module's own. Readers of kind "real" round to the configured precision.
# ---------------------------------------------------------------------------

_NEED = object()


@dataclass(frozen=True)
class _Key:
    kind: str                 # real | float | int | opt_int | opt_float | vec | ivec | str | bool | raw
    unit: Optional[str] = None
    default: Any = _NEED


_SCHEMA: dict[str, dict[str, _Key]] = {
    "simulation": {
        "name": _Key("raw", default=None), "backend": _Key("str", default="b200"),
        "dtype": _Key("raw", default="float32"), "dt": _Key("float", "s"),
        "duration": _Key("float", "s", 0.01), "update_interval": _Key("float", "s", 1e-3),
        "max_picard_iter": _Key("opt_int", default=None),
        "picard_tol": _Key("opt_float", default=None),
        "picard_omega": _Key("opt_float", default=None),
    },
    "domain": {"size": _Key("vec", "m"), "mesh": _Key("ivec")},
    "material": {
        "name": _Key("raw", default="Material"),
        # k / rho / Cp may carry solid and liquid branches: _property_constants()
        "rho": _Key("raw"), "k": _Key("raw"), "Cp": _Key("raw"),
        "L_f": _Key("real", "J/kg", 0.0), "T_solidus": _Key("real", "K", 0.0),
        "T_liquidus": _Key("real", "K", 0.0), "T0": _Key("real", "K", 0.0),
        "Pa": _Key("real", "Pa", 0.0), "R_v": _Key("real", "J/kgK", 0.0),
        "T_boil": _Key("real", "K", 0.0), "DeltaH_LV": _Key("real", "J/kg", 0.0),
        "h_conv_top": _Key("real", "W/m2K", 0.0), "h_conv_bottom": _Key("real", "W/m2K", 0.0),
    },
    "laser": {
        "radius": _Key("real", "m"), "absorptivity": _Key("real"),
        "power_nominal": _Key("real", "W"), "profile": _Key("str", default="gaussian"),
        "r_x": _Key("real", "m", 0.0), "r_y": _Key("real", "m", 0.0),
        "super_gaussian_order": _Key("float", default=2.0),
        "cell_integrated": _Key("bool", default=False), "path": _Key("raw", default=None),
    },
    "fine_mesh": {"refinement": _Key("int", default=4),
                  "box_size": _Key("vec", "m", (0.9e-3, 0.9e-3, 0.04e-3))},
    "laser.path": {"type": _Key("str", default=""), "file": _Key("raw", default=None),
                   "initial_position": _Key("raw", default=(0.0, 0.0))},
}
# Sections carried through unread.
_UNREAD = ("io", "post_processing")

# SI spellings accepted in a {value, unit} mapping, per unit family.
_SI_SPELLINGS = {
    "m": {"m"}, "s": {"s"}, "K": {"K", "kelvin"}, "W": {"W"}, "Pa": {"Pa"},
    "kg/m3": {"kg/m3", "kg/m**3", "kg / m**3", "kg/m^3"},
    "W/mK": {"W/(m.K)", "W/(m*K)", "W / (m * K)", "W/m/K", "W/(m K)"},
    "J/kgK": {"J/(kg.K)", "J/(kg*K)", "J / (kg * K)", "J/kg/K", "J/(kg K)"},
    "J/kg": {"J/kg", "J / kg"},
    "W/m2K": {"W/(m2.K)", "W/(m**2*K)", "W / (m**2 * K)", "W/m2/K", "W/(m^2.K)"},
}
_PROPERTY_UNITS = {"k": "W/mK", "rho": "kg/m3", "Cp": "J/kgK"}


def _unwrap(raw, unit):
    """The payload of a ``{value, unit}`` mapping (checked to be SI), or ``raw``."""
    if not isinstance(raw, dict):
        return raw
    given = (raw.get("unit") or "").strip()
    if given and unit is not None and given not in _SI_SPELLINGS[unit]:
        raise ValueError(f"unit {given!r} given where {unit!r} is expected: this backend "
                         "reads SI values only (no unit conversion)")
    return raw["value"]


def _number(raw, unit=None) -> float:
    v = _unwrap(raw, unit)
    if isinstance(v, bool) or not isinstance(v, (int, float, np.floating, np.integer)):
        raise TypeError(f"expected a number, got {type(v).__name__}")
    return float(v)


_READERS = {
    "raw": lambda raw, unit, real: raw,
    "str": lambda raw, unit, real: str(raw),
    "bool": lambda raw, unit, real: bool(raw),
    "float": lambda raw, unit, real: _number(raw, unit),
    "real": lambda raw, unit, real: real(_number(raw, unit)),
    "int": lambda raw, unit, real: int(_number(raw, unit)),
    "opt_int": lambda raw, unit, real: None if raw is None else int(raw),
    "opt_float": lambda raw, unit, real: None if raw is None else float(raw),
    "vec": lambda raw, unit, real: [_number(v, unit) for v in _sequence(raw, unit)],
    "ivec": lambda raw, unit, real: [int(_number(v)) for v in _sequence(raw, unit)],
}


def _sequence(raw, unit):
    seq = _unwrap(raw, unit)
    if not isinstance(seq, (list, tuple)):
        raise TypeError(f"expected a sequence of numbers, got {type(seq).__name__}")
    return seq


def _check_keys(cfg: dict) -> None:
    """Refuse unknown sections and keys before anything is read."""
    for name in cfg:
        if name not in _SCHEMA and name not in _UNREAD:
            known = sorted(set(_SCHEMA) - {"laser.path"} | set(_UNREAD))
            raise ValueError(f"config section {name!r} is not part of the schema "
                             f"(sections: {', '.join(known)})")
    bodies = {name: cfg.get(name) for name in _SCHEMA}
    laser = cfg.get("laser")
    bodies["laser.path"] = laser.get("path") if isinstance(laser, dict) else None
    for name, body in bodies.items():
        if not isinstance(body, dict):
            continue
        extra = sorted(set(body) - set(_SCHEMA[name]))
        if extra:
            raise ValueError(f"key {extra[0]!r} is not part of config section {name!r} "
                             f"(keys: {', '.join(sorted(_SCHEMA[name]))})")


def _read(cfg: dict, section: str, real) -> dict:
    """Every key of ``section`` read through its schema entry."""
    body = cfg.get(section) or {}
    out = {}
    for key, spec in _SCHEMA[section].items():
        if key in body:
            out[key] = _READERS[spec.kind](body[key], spec.unit, real)
        elif spec.default is _NEED:
            raise KeyError(f"config section {section!r} needs the key {key!r}")
        else:
            out[key] = spec.default
    return out


def _gcode_path(cfg: dict, config_dir: Optional[str]):
    """The G-code laser path a ``laser.path`` section names, or None."""
    laser = cfg.get("laser") or {}
    if not isinstance(laser.get("path"), dict):
        return None
    path = _read({"laser.path": laser["path"]}, "laser.path", float)
    if path["type"].lower() != "gcode" or path["file"] is None:
        return None
    name = str(path["file"])
    if not os.path.isabs(name):
        base = (os.path.join(config_dir, "paths") if config_dir is not None
                else os.path.join(os.getcwd(), "simulations", "examples", "paths"))
        name = os.path.abspath(os.path.join(base, name))
        laser["path"]["file"] = name          # the reference writes the resolved name back
    return GCodeLaserPath(name, initial_position=tuple(path["initial_position"]))


def _property_constants(m: dict, raw: dict, model: Optional[MaterialModel], real) -> dict:
    """The constant ``k`` / ``rho`` / ``Cp`` of the ETD1 propagators.

    Without a model they are the section's numbers. With one, a property that
    varies with T takes its ``reference:`` value (required), and a constant
    one its value at T0 (``core/parameters.py:593-630``)."""
    if model is None:
        return {key: real(_number(raw[key], unit)) for key, unit in _PROPERTY_UNITS.items()}
    varying = [key for key in _PROPERTY_UNITS
               if TempProperty._branches(raw[key]) is not None
               and not model.by_config_key(key).is_constant]
    lacking = [key for key in varying if "reference" not in raw[key]]
    if lacking:
        rec = dict(zip(("k", "rho", "Cp"),
                       model.recommended_references(float(m["T0"]), float(m["T_boil"]))))
        hint = ", ".join(f"{key}.reference={rec[key]:g}" for key in lacking)
        raise ValueError(
            f"temperature-dependent {lacking} lack the 'reference:' constant that splits "
            f"each property into its implicit and explicit parts; a value in the middle of "
            f"the working range converges best (midpoints of the extrema over [T0, T_boil]: "
            f"{hint})")
    return {key: real(_number(raw[key]["reference"], unit)) if key in varying
            else real(float(model.by_config_key(key)(float(m["T0"]))))
            for key, unit in _PROPERTY_UNITS.items()}


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

        A ``laser.path`` of type ``gcode`` is read with :class:`GCodeLaserPath`;
        a relative file name is looked up in ``<config_dir>/paths`` (or
        ``./simulations/examples/paths`` without a ``config_dir``), as the
        reference does. Other paths leave ``laser_path`` ``None``: assign a
        :class:`LaserPath` to it.
        """
        _check_keys(cfg)
        real = resolve_dtype((cfg.get("simulation") or {}).get("dtype", "float32"))
        sim = _read(cfg, "simulation", real)
        dom = _read(cfg, "domain", real)
        m = _read(cfg, "material", real)
        las = _read(cfg, "laser", real)

        # the step is re-derived so that n_steps * dt == t_end exactly
        dt_nominal = float(real(sim["dt"]))
        n_steps = round(sim["duration"] / dt_nominal)
        mesh = [int(v) for v in dom["mesh"]]
        num = NumParams(
            dt=sim["duration"] / n_steps, nx=mesh[0], ny=mesh[1], nz=mesh[2],
            t_end=sim["duration"], n_steps=n_steps, dt_nominal=dt_nominal,
            update_interval=sim["update_interval"], max_picard_iter=sim["max_picard_iter"],
            picard_tol=sim["picard_tol"], picard_omega=sim["picard_omega"], dtype=real)
        geom = GeomParams(size=Vec3(*dom["size"]), n=Vec3(*mesh))

        fine = None
        if cfg.get("fine_mesh") is not None:
            fm = _read(cfg, "fine_mesh", real)
            fine = FineMeshParams(refinement=fm["refinement"], box_size=Vec3(*fm["box_size"]))

        raw_props = {key: m[key] for key in _PROPERTY_UNITS}
        model = MaterialModel.from_config(raw_props, float(m["T_solidus"]),
                                          float(m["T_liquidus"]))
        consts = _property_constants(m, raw_props, model, real)
        mat = MaterialParams(
            name=m["name"], rho=consts["rho"], k=consts["k"], Cp=consts["Cp"], model=model,
            **{key: m[key] for key in ("L_f", "T_solidus", "T_liquidus", "Pa", "R_v", "T_boil",
                                       "DeltaH_LV", "T0", "h_conv_top", "h_conv_bottom")})
        laser = LaserParams(
            radius=las["radius"], absorptivity=las["absorptivity"], power=las["power_nominal"],
            profile=las["profile"],
            r_x=las["r_x"], r_y=las["r_y"],
            super_gaussian_order=las["super_gaussian_order"],
            cell_integrated=las["cell_integrated"])
        return cls(num=num, mat=mat, geom=geom, laser=laser,
                   laser_path=_gcode_path(cfg, config_dir), io=cfg.get("io", {}),
                   backend=sim["backend"].lower(), fine=fine)
