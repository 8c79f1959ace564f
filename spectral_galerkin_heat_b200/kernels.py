"""Kernel module of the ``"b200"`` backend (the ``MathBackend.kernels`` slot).

Functions with the reference kernel modules' names and meanings
(``physics/spectral_cpu_kernels.py``), on torch float64 CUDA tensors:

* ``DCT_II(q)`` / ``IDCT_II(a)``: orthonormal DCT-II / DCT-III over every axis of
  a 1-, 2- or 3-D array (``:374-389``) -> ``sgh_dctn``;
* ``reconstruct_surface_temperature(a, state)`` / ``reconstruct_bottom_temperature``
  (``physics/spectral_ops.py:210-231``) -> ``sgh_surface_temperature``;
* ``reconstruct_volume(a, state)`` / ``project_volume(f, state)``
  (``physics/spectral_ops.py:83-102``) -> ``sgh_reconstruct_volume`` /
  ``sgh_project_volume``;
* output reconstruction with the reference's names and arguments
  (``physics/spectral_helpers.py``): ``reconstruct_temperature_DCT(a, state)``
  (node-centred field, :146-204) -> ``sgh_nodal_temperature``;
  ``reconstruct_temperature_volume_at_points(a, num, geom, state, coords)``
  (:206-248) -> ``sgh_points_temperature``; ``save_temp_profiles(a, num, geom,
  state, laser_position, center, num_points)`` (:251-333), each line reduced
  once (``sgh_line_temperature``) and evaluated at its points. The
  results stay on the device (torch tensors); the reference returns NumPy;
* box mode (``physics/spectral_ops.py``): ``reconstruct_temperature_box(a, state)``
  (:173-179) -> ``sgh_box_temperature`` and ``project_box_to_modes(field_box,
  state)`` (:53-74) -> ``sgh_box_project``, on the window of the last step;
  both raise ``RuntimeError`` for a grid-mode state, as the reference does.

``state`` is the :class:`~spectral_galerkin_heat_b200.solver.B200State` returned
by ``B200SpectralSolver.initialize``. The time step itself is not exposed
piecewise: it runs as one device graph inside the solver.
"""
from __future__ import annotations

import ctypes as C

from . import _lib

__all__ = ["DCT_II", "IDCT_II", "reconstruct_surface_temperature",
           "reconstruct_bottom_temperature", "reconstruct_volume", "project_volume",
           "reconstruct_temperature_DCT", "reconstruct_temperature_volume_at_points",
           "save_temp_profiles", "reconstruct_temperature_box", "project_box_to_modes"]

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


def _fine_mesh(state):
    fm = getattr(state, "fine_mesh", None)
    if fm is None:
        raise RuntimeError("Fine mesh not initialized.")
    return fm


def reconstruct_temperature_box(a, state):
    """Temperature on the fine box at the current window, (nz_box, ny_box, nx_box)."""
    import torch
    fm = _fine_mesh(state)
    a = a.to(torch.float64).contiguous()
    if tuple(a.shape) != tuple(state.shape):
        raise ValueError(f"modes shape {tuple(a.shape)} != {tuple(state.shape)}")
    out = torch.empty(fm.box_shape, dtype=torch.float64, device=a.device)
    _lib.check("sgh_box_temperature", _lib.lib().sgh_box_temperature(
        state.plan, C.c_void_p(a.data_ptr()), C.c_void_p(out.data_ptr()),
        C.c_void_p(state.stream.cuda_stream)))
    return out


def project_box_to_modes(field_box, state):
    """Modes of a fine-box field: ``dV_fine`` times its contraction with the window bases."""
    import torch
    fm = _fine_mesh(state)
    f = field_box.to(torch.float64).contiguous()
    if tuple(f.shape) != fm.box_shape:
        raise ValueError(f"box field shape {tuple(f.shape)} != {fm.box_shape}")
    out = torch.empty(state.shape, dtype=torch.float64, device=f.device)
    _lib.check("sgh_box_project", _lib.lib().sgh_box_project(
        state.plan, C.c_void_p(f.data_ptr()), C.c_void_p(out.data_ptr()),
        C.c_void_p(state.stream.cuda_stream)))
    return out


# ---- output reconstruction -----------------------------------------------------


def _workspace(key, nbytes, device):
    import torch
    ws = _scratch.get((device, key))
    if ws is None or ws.numel() < nbytes:
        ws = torch.empty(max(int(nbytes), 8), dtype=torch.uint8, device=device)
        _scratch[(device, key)] = ws
    return ws


def _lengths(state, geom=None):
    if geom is not None:
        return float(geom.size.x), float(geom.size.y), float(geom.size.z)
    return tuple(float(v) for v in state.size)


def reconstruct_temperature_DCT(a, state):
    """Node-centred temperature ``T(x_j, y_k, z_l)`` at ``x_j = j Lx / nx``
    (``j = 0..nx``, likewise y, z) of modes ``a`` (nz, ny, nx), returned as
    (nx+1, ny+1, nz+1) like the reference (``spectral_helpers.py:146-204``)."""
    import torch
    if not (isinstance(a, torch.Tensor) and a.is_cuda):
        raise TypeError("b200 kernels take CUDA tensors")
    a = a.to(torch.float64).contiguous()
    nz, ny, nx = a.shape
    Lx, Ly, Lz = _lengths(state)
    L = _lib.lib()
    nbytes = C.c_uint64()
    _lib.check("sgh_nodal_workspace_bytes", L.sgh_nodal_workspace_bytes(nx, ny, nz, C.byref(nbytes)))
    ws = _workspace("nodal", nbytes.value, a.device)
    out = torch.empty((nz + 1, ny + 1, nx + 1), dtype=torch.float64, device=a.device)
    _lib.check("sgh_nodal_temperature", L.sgh_nodal_temperature(
        nx, ny, nz, Lx, Ly, Lz, C.c_void_p(a.data_ptr()), C.c_void_p(out.data_ptr()),
        C.c_void_p(ws.data_ptr()), ws.numel(), C.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)))
    return out.permute(2, 1, 0).contiguous()


def reconstruct_temperature_volume_at_points(a, num, geom, state, coords):
    """Temperature of modes ``a`` at points ``coords`` (N, 3), each clipped to
    the domain (``spectral_helpers.py:206-248``); returns (N,) on the device.
    ``ValueError`` unless ``coords`` has shape (N, 3)."""
    import numpy as np
    import torch
    c = coords if isinstance(coords, torch.Tensor) else np.asarray(coords)
    if c.ndim != 2 or c.shape[1] != 3:
        raise ValueError("coords must be of shape (N, 3)")
    if not (isinstance(a, torch.Tensor) and a.is_cuda):
        raise TypeError("b200 kernels take CUDA tensors")
    a = a.to(torch.float64).contiguous()
    pts = torch.as_tensor(c, dtype=torch.float64, device=a.device).contiguous()
    nz, ny, nx = a.shape
    Lx, Ly, Lz = _lengths(state, geom)
    n = int(pts.shape[0])
    out = torch.empty(n, dtype=torch.float64, device=a.device)
    if n == 0:
        return out
    L = _lib.lib()
    nbytes = C.c_uint64()
    _lib.check("sgh_points_workspace_bytes", L.sgh_points_workspace_bytes(nx, ny, nz, n, C.byref(nbytes)))
    ws = _workspace("points", nbytes.value, a.device)
    _lib.check("sgh_points_temperature", L.sgh_points_temperature(
        nx, ny, nz, Lx, Ly, Lz, C.c_void_p(a.data_ptr()), n, C.c_void_p(pts.data_ptr()),
        C.c_void_p(out.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel(),
        C.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)))
    return out


def save_temp_profiles(a, num, geom, state, laser_position, center="laser", num_points=1000):
    """Temperature along three lines through a centre on the top face z = Lz
    (``spectral_helpers.py:251-333``): along x at (y_c, Lz), along y at
    (x_c, Lz), along z at (x_c, y_c), ``num_points`` points each from 0 to the
    domain length. ``center="laser"`` uses ``laser_position``; ``"hotspot"`` the
    cell centre of the hottest top-face cell. Returns ``{"x": (coords, T), ...}``
    with host coordinates and device temperatures."""
    import numpy as np
    import torch
    Lx, Ly, Lz = _lengths(state, geom)
    nz, ny, nx = a.shape
    z_top = float(Lz)
    if center == "hotspot":
        T_surf = reconstruct_surface_temperature(a, state)
        iy, ix = np.unravel_index(int(torch.argmax(T_surf).item()), tuple(T_surf.shape))
        x_center = (ix + 0.5) * (Lx / nx)
        y_center = (iy + 0.5) * (Ly / ny)
    elif center == "laser":
        if laser_position is None:
            raise ValueError("Laser position required for center='laser'")
        x_center, y_center = float(laser_position[0]), float(laser_position[1])
    else:
        raise ValueError(f"Unknown center method: {center}")
    x_center = float(np.clip(x_center, 0.0, Lx))
    y_center = float(np.clip(y_center, 0.0, Ly))
    axes_cfg = [("x", Lx, (0.0, y_center, z_top)), ("y", Ly, (x_center, 0.0, z_top)),
                ("z", Lz, (x_center, y_center, 0.0))]
    if not (isinstance(a, torch.Tensor) and a.is_cuda):
        raise TypeError("b200 kernels take CUDA tensors")
    a = a.to(torch.float64).contiguous()
    L = _lib.lib()
    nbytes = C.c_uint64()
    _lib.check("sgh_line_workspace_bytes", L.sgh_line_workspace_bytes(nx, ny, nz, C.byref(nbytes)))
    ws = _workspace("line", nbytes.value, a.device)
    stream = C.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)
    profiles = {}
    for axis, (key, L_axis, fixed) in enumerate(axes_cfg):
        coords = np.linspace(0.0, L_axis, num_points, dtype=np.float64)
        out = torch.empty(num_points, dtype=torch.float64, device=a.device)
        if num_points > 0:
            xs = torch.as_tensor(coords, device=a.device)
            # the modes reduced once along the line, then its cosine series at the points
            _lib.check("sgh_line_temperature", L.sgh_line_temperature(
                nx, ny, nz, Lx, Ly, Lz, C.c_void_p(a.data_ptr()), axis, float(fixed[0]), float(fixed[1]),
                float(fixed[2]), num_points, C.c_void_p(xs.data_ptr()), C.c_void_p(out.data_ptr()),
                C.c_void_p(ws.data_ptr()), ws.numel(), stream))
            torch.cuda.current_stream(a.device).synchronize()
        profiles[key] = (coords, out)
    return profiles
