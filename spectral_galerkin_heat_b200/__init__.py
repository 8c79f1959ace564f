"""B200 backend for the spectral-Galerkin laser heat solver.

The time step of the reference solver ``spectral_galerkin_heat`` (its
``SpectralSolver.step``) rebuilt for NVIDIA B200: hand-written sm_100a CUDA in
``libsgh_b200.so`` behind a C ABI (``include/sgh_b200.h``), driven from Python
through ctypes, with PyTorch tensors as device buffers.

Public API (mirrors the reference's names):

* :class:`B200SpectralSolver` -- ``initialize`` / ``step`` / ``set_state`` /
  ``finalize`` plus ``run`` for device-resident multi-step runs;
* :class:`SimulationContext` and the parameter dataclasses, :class:`LaserPath`,
  :class:`LaserState`;
* :func:`get_backend` / :func:`register_backend` / :class:`MathBackend`, with the
  ``"b200"`` backend registered; :func:`build_solver`.
"""
from .backends import (B200Backend, MathBackend, build_solver, get_backend,
                       install_into_reference, register_backend)
from .config import (FineMeshParams, GeomParams, LaserParams, MaterialParams, NumParams,
                     SimulationContext, Vec3)
from .laser import FixedLaser, LaserPath, LaserState, RasterPath, StraightTrack
from .properties import MaterialModel, PropertyExpr, TempProperty
from .solver import B200SpectralSolver, B200State, HeatSolver

__version__ = "0.1.0"

__all__ = [
    "B200SpectralSolver", "B200State", "HeatSolver", "B200Backend", "MathBackend",
    "build_solver", "get_backend", "register_backend", "install_into_reference",
    "SimulationContext", "NumParams", "MaterialParams", "GeomParams", "LaserParams",
    "FineMeshParams", "Vec3", "LaserPath", "LaserState", "FixedLaser", "StraightTrack",
    "RasterPath", "MaterialModel", "PropertyExpr", "TempProperty",
]
