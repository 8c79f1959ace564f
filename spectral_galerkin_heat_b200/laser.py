"""Laser state, laser paths and beam profiles.

Mirrors the reference's laser API (``core/laser.py``): ``LaserState`` :150-167,
the ``LaserPath`` ABC :169-217, the super-Gaussian area factor :34-39 and
``build_laser_profile`` :143-166, so user code written against the reference
(``get_state(t, dt) -> LaserState``) drives this backend unchanged.

The flux itself is evaluated on the device (``sgh_face_*`` kernels); the host
side here only resolves the profile and the energy-conserving peak intensity
``I0 = A*P / (f * r_x * r_y)`` (``core/laser.py:110-112``).

Two synthetic paths used by the benchmark workloads live here as well: a
constant-velocity straight track and a bidirectional raster.
"""
from __future__ import annotations

import math
from abc import ABC, abstractmethod
from dataclasses import dataclass

import numpy as np

__all__ = [
    "LaserState", "LaserPath", "LaserProfile", "build_laser_profile",
    "super_gaussian_area_factor", "StraightTrack", "RasterPath", "FixedLaser",
    "GCodeLaserPath", "LASER_DTYPE", "LASER_F32", "laser_table",
]


@dataclass
class LaserState:
    """Laser snapshot at one time: position (m), power (W), on/off, velocity (m/s)."""

    x: float
    y: float
    power: float
    is_on: bool
    v: tuple = (0.0, 0.0)


class LaserPath(ABC):
    """Laser trajectory; ``get_state`` is called once per time step."""

    @abstractmethod
    def get_state(self, time: float, dt: float) -> LaserState:
        """Return the laser state at ``time`` for a step of length ``dt``."""


def super_gaussian_area_factor(order: float) -> float:
    """``f`` with ``integral exp(-2 rho^n) dA = f r_x r_y``:
    ``f(n) = pi 2^(1-2/n) Gamma(2/n) / n`` (``f(2) = pi/2``)."""
    n = float(order)
    return math.pi * 2.0 ** (1.0 - 2.0 / n) * math.gamma(2.0 / n) / n


_PROFILE_ORDERS = {"gaussian": 2.0, "flat_top": 12.0, "super_gaussian": None}


@dataclass(frozen=True)
class LaserProfile:
    """Beam shape ``exp(-2 rho^order)`` and its normalisation."""

    name: str
    order: float
    cell_integrated: bool = False

    @property
    def area_factor(self) -> float:
        return super_gaussian_area_factor(self.order)

    def peak_intensity(self, power: float, absorptivity: float, ref_area: float) -> float:
        """``I0 = A*P / (f * ref_area)``."""
        return absorptivity * power / (self.area_factor * ref_area)


def build_laser_profile(name: str, order: float = 2.0,
                        cell_integrated: bool = False) -> LaserProfile:
    """Resolve ``"gaussian"`` / ``"flat_top"`` / ``"super_gaussian"``; ``ValueError`` otherwise."""
    key = str(name).lower()
    if key not in _PROFILE_ORDERS:
        raise ValueError(f"Unknown laser profile: {name!r}. Choose one of: "
                         f"{', '.join(sorted(_PROFILE_ORDERS))}.")
    canonical = _PROFILE_ORDERS[key]
    resolved = float(order) if canonical is None else canonical
    if cell_integrated and resolved != 2.0:
        raise ValueError("cell_integrated flux is only defined for the Gaussian "
                         f"(order 2), got order {resolved}.")
    return LaserProfile(name=key, order=resolved, cell_integrated=bool(cell_integrated))


class FixedLaser(LaserPath):
    """Stationary beam at ``(x, y)``."""

    def __init__(self, x, y, power, is_on=True):
        self.x, self.y, self.power, self.is_on = x, y, power, is_on

    def get_state(self, time, dt):
        return LaserState(x=self.x, y=self.y, power=self.power, is_on=self.is_on)


class StraightTrack(LaserPath):
    """Constant velocity ``(vx, vy)`` from ``(x0, y0)``: position ``x0 + vx*t``."""

    def __init__(self, x0, y0, vx, vy, power, is_on=True):
        self.x0, self.y0, self.vx, self.vy = x0, y0, vx, vy
        self.power, self.is_on = power, is_on

    def get_state(self, time, dt):
        return LaserState(x=self.x0 + self.vx * time, y=self.y0 + self.vy * time,
                          power=self.power, is_on=self.is_on, v=(self.vx, self.vy))


class RasterPath(LaserPath):
    """Bidirectional raster along x: ``n_lines`` tracks of ``length`` metres,
    ``hatch`` metres apart in y, scanned at ``speed`` m/s, alternating direction.

    Track ``j`` starts at ``(x0, y0 + j*hatch)`` when ``j`` is even and at
    ``(x0 + length, y0 + j*hatch)`` when odd. The turn between tracks is
    instantaneous. After the last track the beam switches off.
    """

    def __init__(self, x0, y0, length, hatch, n_lines, speed, power):
        self.x0, self.y0, self.length, self.hatch = x0, y0, length, hatch
        self.n_lines, self.speed, self.power = int(n_lines), speed, power

    def get_state(self, time, dt):
        t_line = self.length / self.speed
        j = int(math.floor(time / t_line)) if time >= 0.0 else 0
        if j >= self.n_lines:
            j = self.n_lines - 1
            s = self.length
            on = False
        else:
            s = (time - j * t_line) * self.speed
            on = True
        y = self.y0 + j * self.hatch
        if j % 2 == 0:
            x, vx = self.x0 + s, self.speed
        else:
            x, vx = self.x0 + self.length - s, -self.speed
        return LaserState(x=x, y=y, power=self.power if on else 0.0, is_on=on, v=(vx, 0.0))


_F32 = np.float32

# Segment table of a G-code path: start and end point, start and end time and
# power, all single precision (the reference quantises them so), and laser on.
_SEGMENT_DTYPE = np.dtype([("x0", "<f4"), ("y0", "<f4"), ("x1", "<f4"), ("y1", "<f4"),
                           ("t0", "<f4"), ("t1", "<f4"), ("power", "<f4"), ("on", "?")])


class GCodeLaserPath(LaserPath):
    """Laser path read from a G-code file (``io_utils/gcode_path.py:25-119``).

    Understood: ``G21`` (millimetres) and ``G20`` (inches) set the unit, metres
    otherwise; ``G0``/``G1`` move to ``X``/``Y`` at feed ``F`` (unit per
    minute); ``M3 S<W>`` switches the beam on at that power and ``M5`` off. A
    move made while the beam is on becomes a timed segment; moves with the beam
    off relocate it without taking time. Text after ``;`` is a comment.

    Positions, times and powers are kept in single precision, and ``get_state``
    interpolates them in single precision, because the reference does so: the
    states it returns (numpy float32 scalars) are the reference's bit for bit,
    and the solver forms the quantities it derives from them (warm-start shift,
    box window) in single precision too (``LASER_F32``).
    """

    def __init__(self, gcode_file, initial_position=(0.0, 0.0)):
        self.file = str(gcode_file)
        with open(self.file) as fh:
            self.segments, self.unit_scale = self.parse(fh.read().splitlines())
        self.initial_position = (_F32(initial_position[0]) * _F32(self.unit_scale),
                                 _F32(initial_position[1]) * _F32(self.unit_scale))

    @staticmethod
    def parse(lines):
        """``(segment table, unit scale)`` of G-code text lines."""
        scale, power, on, feed = 1.0, 0.0, False, 0.0
        pos = [0.0, 0.0]
        last = None
        clock = 0.0
        rows = []
        for raw in lines:
            line = raw.split(";", 1)[0].strip()
            if not line:
                continue
            if line.startswith("G21"):
                scale = 1.0 / 1000.0
            elif line.startswith("G20"):
                scale = 25.4 / 1000.0
            elif line.startswith(("G0", "G1")):
                for word in line.split()[1:]:
                    axis, val = word[0], word[1:]
                    if axis in "XY" and val:
                        pos["XY".index(axis)] = float(_F32(float(val) * scale))
                    elif axis == "F" and val:
                        feed = _F32(float(val) * scale)
                if last is not None and on:
                    length = float(np.sqrt((pos[0] - last[0]) ** 2 + (pos[1] - last[1]) ** 2))
                    speed = float(feed) / 60.0 if feed > 0 else 1.0
                    end = float(clock + (length / speed if speed > 0 else 0.0))
                    rows.append((last[0], last[1], pos[0], pos[1], clock, end, power, True))
                    clock = end
                last = list(pos)
            elif line.startswith("M3"):
                for word in line.split()[1:]:
                    if word.startswith("S"):
                        power = float(word[1:])
                on = True
            elif line.startswith("M5"):
                on, power = False, 0.0
        return np.array(rows, dtype=_SEGMENT_DTYPE), scale

    def get_state(self, time, dt):
        tab = self.table(np.array([float(time)]), float(dt))[0]
        return LaserState(x=_F32(tab["x"]), y=_F32(tab["y"]), power=_F32(tab["power"]),
                          is_on=bool(tab["is_on"]), v=(_F32(tab["vx"]), _F32(tab["vy"])))

    def table(self, times, dt: float) -> np.ndarray:
        """States at float64 ``times`` (each the value of a Python float time
        ``t``; the step ``dt`` a Python float) as ``sgh_laser`` records, with
        the reference's single-precision arithmetic: a Python float meets a
        float32 scalar in float32, and the velocity is a float64 difference
        quotient rounded to float32."""
        times = np.asarray(times, dtype=np.float64)
        out = np.zeros(times.shape, dtype=LASER_DTYPE)
        out["flags"] = LASER_F32
        t32 = times.astype(_F32)
        seg = self.segments
        hit = np.full(times.shape, -1, dtype=np.int64)
        for i in range(len(seg) - 1, -1, -1):            # first matching segment wins
            inside = (seg["t0"][i] <= t32) & (t32 <= seg["t1"][i])
            hit = np.where(inside, i, hit)
        found = hit >= 0
        if found.any():
            s = seg[hit[found]]
            tf = t32[found]
            span = s["t1"] - s["t0"]
            frac = np.where(s["t1"] > s["t0"], (tf - s["t0"]) / np.where(span > 0, span, _F32(1)),
                            _F32(0))
            x = (s["x0"] + frac * (s["x1"] - s["x0"])).astype(_F32)
            y = (s["y0"] + frac * (s["y1"] - s["y0"])).astype(_F32)
            moving = (tf > s["t0"]) & (dt > 0.0)
            tp = (times[found] - dt).astype(_F32)
            use = (tp >= s["t0"]) & (span > 0)
            pfrac = np.where(use, (tp - s["t0"]) / np.where(span > 0, span, _F32(1)), _F32(0))
            px = (s["x0"] + pfrac * (s["x1"] - s["x0"])).astype(_F32)
            py = (s["y0"] + pfrac * (s["y1"] - s["y0"])).astype(_F32)
            with np.errstate(all="ignore"):
                vx = ((x.astype(np.float64) - px.astype(np.float64)) / dt).astype(_F32)
                vy = ((y.astype(np.float64) - py.astype(np.float64)) / dt).astype(_F32)
            out["x"][found], out["y"][found] = x, y
            out["power"][found] = s["power"]
            out["is_on"][found] = s["on"].astype(np.int32)
            out["vx"][found] = np.where(moving, vx, _F32(0))
            out["vy"][found] = np.where(moving, vy, _F32(0))
        rest = ~found
        if rest.any():
            after = rest & (len(seg) > 0) & (t32 > (seg["t1"][-1] if len(seg) else _F32(0)))
            if after.any():
                out["x"][after], out["y"][after] = seg["x1"][-1], seg["y1"][-1]
            before = rest & ~after
            out["x"][before], out["y"][before] = self.initial_position
        return out


# Flag of an ``sgh_laser`` record whose position and velocity are float32
# values (G-code paths): the library then forms the warm-start shift and the
# box window from them in float32 arithmetic, as the reference does.
LASER_F32 = 1

# One ``sgh_laser`` record (include/sgh_b200.h): x, y, power, vx, vy, is_on, flags.
LASER_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("power", "<f8"), ("vx", "<f8"),
                        ("vy", "<f8"), ("is_on", "<i4"), ("flags", "<i4")])


def laser_table(path: LaserPath, t0: float, dt: float, n: int) -> np.ndarray:
    """``n`` laser states at ``t0 + i*dt`` as ``sgh_laser`` records.

    Same values as calling ``path.get_state(t0 + i*dt, dt)`` per step (the
    times and positions use the same float64 operations); straight tracks and
    rasters are evaluated in one vectorised pass, other paths step by step.
    """
    out = np.zeros(n, dtype=LASER_DTYPE)
    times = t0 + np.arange(n, dtype=np.float64) * dt
    if isinstance(path, StraightTrack):
        out["x"] = path.x0 + path.vx * times
        out["y"] = path.y0 + path.vy * times
        out["power"] = path.power
        out["vx"], out["vy"] = path.vx, path.vy
        out["is_on"] = 1 if path.is_on else 0
        return out
    if isinstance(path, RasterPath):
        t_line = path.length / path.speed
        j = np.where(times >= 0.0, np.floor(times / t_line), 0.0).astype(np.int64)
        off = j >= path.n_lines
        j = np.where(off, path.n_lines - 1, j)
        s = np.where(off, path.length, (times - j * t_line) * path.speed)
        even = (j % 2) == 0
        out["x"] = np.where(even, path.x0 + s, path.x0 + path.length - s)
        out["y"] = path.y0 + j * path.hatch
        out["power"] = np.where(off, 0.0, path.power)
        out["vx"] = np.where(even, path.speed, -path.speed)
        out["is_on"] = np.where(off, 0, 1)
        return out
    if isinstance(path, GCodeLaserPath):
        return path.table(times, float(dt))
    for i, t in enumerate(times):
        st = path.get_state(float(t), dt)
        single = isinstance(st.x, np.float32) and isinstance(st.v[0], np.float32)
        out[i] = (st.x, st.y, st.power, st.v[0], st.v[1], 1 if st.is_on else 0,
                  LASER_F32 if single else 0)
    return out
