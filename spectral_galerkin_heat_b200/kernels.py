"""Kernel module of the ``"b200"`` backend (the ``MathBackend.kernels`` slot).

Functions with the reference kernel modules' names and meanings
(``physics/spectral_cpu_kernels.py``), on torch float64 CUDA tensors:

* ``DCT_II(q)`` / ``IDCT_II(a)``: orthonormal DCT-II / DCT-III over every axis of
  a 1-, 2- or 3-D array (``:374-389``) -> ``sgh_dctn``;
* ``reconstruct_surface_temperature(a, state)`` / ``reconstruct_bottom_temperature``
  (``physics/spectral_ops.py:210-231``) -> ``sgh_surface_temperature``;
* ``reconstruct_volume(a, state)`` / ``project_volume(f, state)``
  (``physics/spectral_ops.py:83-102``) -> ``sgh_reconstruct_volume`` /
  ``sgh_project_volume``.

``state`` is the :class:`~spectral_galerkin_heat_b200.solver.B200State` returned
by ``B200SpectralSolver.initialize``. The time step itself is not exposed
piecewise: it runs as one device graph inside the solver.
"""
from __future__ import annotations

import ctypes as C

from . import _lib

__all__ = ["DCT_II", "IDCT_II", "reconstruct_surface_temperature",
           "reconstruct_bottom_temperature", "reconstruct_volume", "project_volume"]

_scratch = {}


def _dctn(x, kind):
    import torch
    if not (isinstance(x, torch.Tensor) and x.is_cuda):
        raise TypeError("b200 kernels take CUDA tensors")
    x = x.to(torch.float64).contiguous()
    if x.dim() not in (1, 2, 3):
        raise ValueError("DCT_II/IDCT_II support 1-, 2- and 3-D arrays")
    shape = (C.c_int32 * x.dim())(*x.shape)
    nbytes = C.c_uint64()
    L = _lib.lib()
    _lib.check("sgh_dctn_workspace_bytes", L.sgh_dctn_workspace_bytes(x.dim(), shape, C.byref(nbytes)))
    key = (x.device, int(nbytes.value))
    ws = _scratch.get(key)
    if ws is None:
        ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=x.device)
        _scratch[key] = ws
    out = torch.empty_like(x)
    stream = torch.cuda.current_stream(x.device).cuda_stream
    _lib.check("sgh_dctn", L.sgh_dctn(kind, x.dim(), shape, C.c_void_p(x.data_ptr()),
                                      C.c_void_p(out.data_ptr()), C.c_void_p(ws.data_ptr()),
                                      nbytes.value, C.c_void_p(stream)))
    return out


def DCT_II(q):
    """Orthonormal DCT-II over all axes."""
    return _dctn(q, 2)


def IDCT_II(a):
    """Orthonormal DCT-III (inverse of :func:`DCT_II`) over all axes."""
    return _dctn(a, 3)


def _surface(a, state, top):
    import torch
    nz, ny, nx = state.shape
    a = a.to(torch.float64).contiguous()
    out = torch.empty((ny, nx), dtype=torch.float64, device=a.device)
    _lib.check("sgh_surface_temperature", _lib.lib().sgh_surface_temperature(
        state.plan, C.c_void_p(a.data_ptr()), 1 if top else 0, C.c_void_p(out.data_ptr()),
        C.c_void_p(state.stream.cuda_stream)))
    return out


def reconstruct_surface_temperature(a, state):
    """Temperature on the top face z = Lz."""
    return _surface(a, state, True)


def reconstruct_bottom_temperature(a, state):
    """Temperature on the bottom face z = 0."""
    return _surface(a, state, False)


def reconstruct_volume(a, state):
    """``IDCT_II(a) / sqrt(dV)`` on the cell centres."""
    import torch
    a = a.to(torch.float64).contiguous()
    out = torch.empty_like(a)
    _lib.check("sgh_reconstruct_volume", _lib.lib().sgh_reconstruct_volume(
        state.plan, C.c_void_p(a.data_ptr()), C.c_void_p(out.data_ptr()),
        C.c_void_p(state.stream.cuda_stream)))
    return out


def project_volume(f, state):
    """``sqrt(dV) DCT_II(f)``."""
    import torch
    f = f.to(torch.float64).contiguous()
    out = torch.empty_like(f)
    _lib.check("sgh_project_volume", _lib.lib().sgh_project_volume(
        state.plan, C.c_void_p(f.data_ptr()), C.c_void_p(out.data_ptr()),
        C.c_void_p(state.stream.cuda_stream)))
    return out
