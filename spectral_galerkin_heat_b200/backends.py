"""Backend plugin boundary: ``MathBackend`` + name registry, and the ``"b200"`` backend.

Mirrors ``backends/base.py:38-81`` (``MathBackend(name, xp, kernels)``) and
``backends/_registry.py:45-110`` (``register_backend`` refuses duplicates with
``ValueError``; ``get_backend`` raises ``ValueError`` for an unknown name).

``install_into_reference()`` registers the same ``"b200"`` factory in the
reference package's own registry when that package is importable, so
``spectral_galerkin_heat.backends.get_backend("b200")`` works there too.
"""
from __future__ import annotations

from typing import Callable, Dict

__all__ = ["MathBackend", "register_backend", "get_backend", "B200Backend",
           "install_into_reference", "build_solver"]


class MathBackend:
    """An array module plus the matching kernel module of one execution target."""

    def __init__(self, name: str, xp, kernels):
        self.name = name
        self.xp = xp
        self.kernels = kernels

    def to_numpy(self, arr):
        """Host ``numpy.ndarray`` copy of ``arr`` (torch tensors are copied off the device)."""
        import numpy as np
        if hasattr(arr, "detach"):
            return arr.detach().cpu().numpy()
        get = getattr(arr, "get", None)
        return get() if callable(get) else np.asarray(arr)

    def __repr__(self):
        return f"MathBackend(name={self.name!r})"


_FACTORIES: Dict[str, Callable[[], MathBackend]] = {}


def register_backend(name: str):
    """Decorator registering a zero-argument backend factory under ``name``."""

    def deco(factory):
        if name in _FACTORIES:
            raise ValueError(f"Backend {name!r} is already registered "
                             f"({_FACTORIES[name]!r}); cannot overwrite it.")
        _FACTORIES[name] = factory
        return factory

    return deco


def get_backend(name: str = "b200") -> MathBackend:
    """Fresh backend instance by name; ``ValueError`` if unknown."""
    factory = _FACTORIES.get(name)
    if factory is None:
        avail = ", ".join(sorted(_FACTORIES)) or "(none)"
        raise ValueError(f"Unknown backend: {name!r}. Registered backends: {avail}.")
    return factory()


@register_backend("b200")
class B200Backend(MathBackend):
    """torch device tensors + the libsgh_b200 kernel module."""

    def __init__(self):
        import torch

        from . import kernels
        super().__init__(name="b200", xp=torch, kernels=kernels)


def install_into_reference() -> bool:
    """Plug the B200 backend into the reference package when it is importable:
    ``"b200"`` goes into its backend registry (``backends/_registry.py:45-110``),
    so ``spectral_galerkin_heat.backends.get_backend("b200")`` builds a
    :class:`B200Backend`, and :class:`B200SpectralSolver` is registered as a
    virtual subclass of its ``HeatSolver`` ABC (``solvers/base.py:31-91``), so
    ``isinstance(solver, HeatSolver)`` holds in code written for the reference.
    Returns False when the reference is not importable."""
    try:
        from spectral_galerkin_heat.backends import _registry as ref_registry  # type: ignore
        from spectral_galerkin_heat.solvers.base import HeatSolver as RefHeatSolver  # type: ignore
    except Exception:
        return False
    if "b200" not in ref_registry._BACKEND_FACTORIES:
        ref_registry._BACKEND_FACTORIES["b200"] = B200Backend
    from .solver import B200SpectralSolver
    RefHeatSolver.register(B200SpectralSolver)
    return True


def build_solver(context):
    """``solvers/__init__.py:13-34`` with the extra case ``"b200"``.

    ``"b200"`` builds a :class:`~spectral_galerkin_heat_b200.solver.B200SpectralSolver`;
    the reference's own names are delegated to the reference when it is installed.
    """
    from .solver import B200SpectralSolver
    name = getattr(context, "backend", "b200")
    if name == "b200":
        return B200SpectralSolver(get_backend("b200"))
    if name in ("cpu", "gpu", "cpu_linear"):
        try:
            from spectral_galerkin_heat.solvers import build_solver as ref_build  # type: ignore
        except Exception as exc:
            raise ValueError(f"backend {name!r} belongs to the reference package, which is "
                             "not installed") from exc
        return ref_build(context)
    raise ValueError(f"Unknown backend: {name!r}. Choose 'b200', 'cpu', 'gpu', or 'cpu_linear'.")
