"""``B200SpectralSolver``: the reference's ``HeatSolver`` contract on one B200.

Drop-in for ``SpectralSolver`` (``solvers/spectral.py:38-628``) behind the same
lifecycle (``solvers/base.py:31-91``):

* ``initialize(context) -> state``; ``RuntimeError`` without a context;
* ``step(t, dt) -> (state, metrics)`` with the metric keys ``T_surface_max``,
  ``P_laser``, ``n_evap_iter``, ``picard_converged``, ``picard_rel_err``;
* ``set_state(T)``; ``RuntimeError`` before ``initialize``;
* ``finalize()``;
* Picard controls resolved as constructor argument > config > default
  (0.1 / 1e-4 / 30) (``solvers/spectral.py:107-123``); a one-time warning when
  a step hits the iteration cap (``:486-499``) and a one-time warning for the
  grid-mode T-dependent configuration (``:210-216``);
* grid mode (no ``fine_mesh``) and box mode (``fine_mesh``: latent heat on a
  laser-following refined sub-box, ``state.fine_mesh`` mirroring
  ``FineMeshState``), with the one-time box-truncation warning (``:545-586``).

The whole step runs on the device (``libsgh_b200.so``): the host calls
``LaserPath.get_state(t, dt)``, hands the laser state to ``sgh_step`` and reads
back the metrics once per step. ``run()`` advances many steps with the laser
states precomputed into a device table and no host round trip per step.

PyTorch provides the device buffer (one workspace tensor per instance) and the
stream; all arithmetic is in the library. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import logging
import math
from abc import ABC, abstractmethod
from typing import Any, Optional

import numpy as np

from . import _lib
from .laser import LASER_F32, build_laser_profile
from .properties import PropertyExpr

logger = logging.getLogger(__name__)

__all__ = ["HeatSolver", "B200SpectralSolver", "B200State", "B200FineMesh", "make_config",
           "laser_struct"]


class HeatSolver(ABC):
    """Lifecycle of a heat solver: ``initialize`` once, ``step`` repeatedly, ``finalize``."""

    @abstractmethod
    def initialize(self, context) -> Any:
        """Allocate and set the initial condition; return the state."""

    @abstractmethod
    def step(self, t: float, dt: float):
        """Advance by ``dt``; return ``(state, metrics)``."""

    @abstractmethod
    def finalize(self) -> None:
        """Release resources."""


def _torch():
    import torch
    return torch


def _program(source) -> _lib.SghProgram:
    ops, consts = PropertyExpr(source).program()
    p = _lib.SghProgram()
    p.n_ops = len(ops)
    p.n_consts = len(consts)
    for i, v in enumerate(ops):
        p.ops[i] = int(v)
    if len(consts) > _lib.MAX_CONSTS:
        raise ValueError(f"property expression {source!r} has more than "
                         f"{_lib.MAX_CONSTS} constants")
    for i, v in enumerate(consts):
        p.consts[i] = float(v)
    return p


def make_config(ctx, omega: float, tol: float, max_iter: int) -> _lib.SghConfig:
    """Translate a ``SimulationContext`` into the library's ``sgh_config``."""
    g, mat, lp, num = ctx.geom, ctx.mat, ctx.laser, ctx.num
    c = _lib.SghConfig()
    c.nx, c.ny, c.nz = int(num.nx), int(num.ny), int(num.nz)
    if (c.nx, c.ny, c.nz) != (int(g.n.x), int(g.n.y), int(g.n.z)):
        raise ValueError("num.(nx, ny, nz) and geom.n disagree")
    c.precision = 0
    c.Lx, c.Ly, c.Lz = float(g.size.x), float(g.size.y), float(g.size.z)
    c.dt = float(num.dt)
    c.k, c.rho, c.cp = float(mat.k), float(mat.rho), float(mat.Cp)
    c.L_f = float(getattr(mat, "L_f", 0.0))
    c.T_solidus, c.T_liquidus = float(mat.T_solidus), float(mat.T_liquidus)
    c.Pa, c.R_v, c.T_boil = float(mat.Pa), float(mat.R_v), float(mat.T_boil)
    c.dH_LV, c.T0 = float(mat.DeltaH_LV), float(mat.T0)
    c.h_top = float(getattr(mat, "h_conv_top", 0.0))
    c.h_bottom = float(getattr(mat, "h_conv_bottom", 0.0))
    model = getattr(mat, "model", None)
    if model is not None:
        c.has_model = 1
        c.model_constant = int(bool(model.is_constant))
        c.k_constant = int(bool(model.k.is_constant))
        for name, prop in (("k", model.k), ("rho", model.rho), ("c", model.c)):
            setattr(c, f"{name}_solid", _program(prop.solid.source))
            setattr(c, f"{name}_liquid", _program(prop.liquid.source))
    prof = build_laser_profile(getattr(lp, "profile", "gaussian"),
                               getattr(lp, "super_gaussian_order", 2.0),
                               cell_integrated=bool(getattr(lp, "cell_integrated", False)))
    c.r_x, c.r_y = float(lp.r_x), float(lp.r_y)
    c.absorptivity = float(lp.absorptivity)
    c.order = float(prof.order)
    c.area_factor = float(prof.area_factor)
    c.cell_integrated = int(prof.cell_integrated)
    c.max_iter = int(max_iter)
    c.omega, c.tol = float(omega), float(tol)
    fine = getattr(ctx, "fine", None)
    if fine is not None:
        c.box = 1
        c.box_refinement = int(fine.refinement)
        bs = fine.box_size
        c.box_size[0], c.box_size[1], c.box_size[2] = float(bs[0]), float(bs[1]), float(bs[2])
    return c


def laser_struct(state, dt: float, plan_dt: float) -> _lib.SghLaser:
    """``LaserState`` -> ``sgh_laser``. The library shifts the warm-start flux by
    ``v * plan_dt``; a call with another ``dt`` rescales ``v`` to keep ``v * dt``."""
    L = _lib.SghLaser()
    L.x, L.y, L.power = float(state.x), float(state.y), float(state.power)
    vx, vy = state.v
    if dt != plan_dt:
        vx, vy = vx * dt / plan_dt, vy * dt / plan_dt
    L.vx, L.vy = float(vx), float(vy)
    L.is_on = 1 if state.is_on else 0
    # float32 states (G-code paths): shifts and the box window in float32
    single = isinstance(state.x, np.float32) and isinstance(state.v[0], np.float32)
    L.flags = LASER_F32 if single and dt == plan_dt else 0
    return L


class B200State:
    """Device-resident state of one instance; arrays are views into the workspace."""

    def __init__(self, plan, workspace, shape, stream, sqrt_dV, dtype=np.float64):
        self.plan = plan
        self.workspace = workspace
        self.shape = shape
        self.stream = stream
        self.dtype = dtype
        self.sqrt_dV = sqrt_dV
        self.a = self.buffer("modes")
        self.K = self.buffer("K")
        self.KK = self.buffer("KK")
        self.T_prev = self.buffer("T_prev")
        self.q_evap_old = self.buffer("q_evap_old")
        self.fine_mesh = None

    def raw_buffer(self, name):
        """torch float64 1-D view of a named workspace buffer."""
        torch = _torch()
        ptr = C.c_void_p()
        nbytes = C.c_uint64()
        _lib.check("sgh_plan_buffer",
                   _lib.lib().sgh_plan_buffer(self.plan, _lib.BUF[name], C.byref(ptr), C.byref(nbytes)))
        off = ptr.value - self.workspace.data_ptr()
        return self.workspace[off:off + nbytes.value].view(torch.float64)

    def buffer(self, name):
        """torch float64 view of a named workspace buffer."""
        torch = _torch()
        ptr = C.c_void_p()
        nbytes = C.c_uint64()
        _lib.check("sgh_plan_buffer",
                   _lib.lib().sgh_plan_buffer(self.plan, _lib.BUF[name], C.byref(ptr), C.byref(nbytes)))
        off = ptr.value - self.workspace.data_ptr()
        view = self.workspace[off:off + nbytes.value].view(torch.float64)
        nz, ny, nx = self.shape
        return view.view(nz, ny, nx) if view.numel() == nz * ny * nx else view.view(ny, nx)


class B200FineMesh:
    """Fine box of a box-mode instance (``FineMeshState``, ``physics/spectral_state.py:166-239``).

    Geometry attributes carry the reference's names and values; ``B_fine_full``
    (cosine bases, modes x fine cells), ``T_prev`` and ``Q_prev`` are views of
    the device workspace. The window follows the laser inside the step on the
    device (``FineMeshState.update``); :meth:`window` reads its start indices.
    ``T_prev`` and ``Q_prev`` are ``None`` until the first step, as in the
    reference.
    """

    def __init__(self, state, fine):
        g = _lib.SghBoxGeom()
        _lib.check("sgh_box_geometry", _lib.lib().sgh_box_geometry(state.plan, C.byref(g)))
        self._state = state
        self.refinement = int(fine.refinement)
        self.nx_box, self.ny_box, self.nz_box = (int(v) for v in g.n_box)
        self.n_fine_totals = [int(v) for v in g.n_fine_total]
        self.dx_fine, self.dy_fine, self.dz_fine = (float(v) for v in g.d_fine)
        self.dV_fine = float(g.dV_fine)
        self.z0 = float(g.z0)
        self.box_shape = (self.nz_box, self.ny_box, self.nx_box)
        self.coords_fine = [(np.arange(n) + 0.5) * d for n, d in
                            zip(self.n_fine_totals, (self.dx_fine, self.dy_fine, self.dz_fine))]
        nz, ny, nx = state.shape
        fx, fy, _ = self.n_fine_totals
        bx = state.raw_buffer("box_Bx").view(fx, nx)
        by = state.raw_buffer("box_By").view(fy, ny)
        bz = state.raw_buffer("box_Bz").view(self.nz_box + 1, nz)
        self.B_fine_full = [bx.t(), by.t(), bz[:self.nz_box].t()]
        self._T_prev = state.raw_buffer("box_T_prev").view(*self.box_shape)
        self._Q_prev = state.raw_buffer("box_Q_prev").view(*self.box_shape)
        self.primed = False

    @property
    def T_prev(self):
        return self._T_prev if self.primed else None

    @property
    def Q_prev(self):
        return self._Q_prev if self.primed else None

    def window(self):
        """``(i_start_x, i_start_y)`` of the last step's window; ``(-1, -1)`` before the first."""
        w = (C.c_int32 * 2)()
        _lib.check("sgh_box_window", _lib.lib().sgh_box_window(
            self._state.plan, w, C.c_void_p(self._state.stream.cuda_stream)))
        return int(w[0]), int(w[1])


class B200SpectralSolver(HeatSolver):
    """Spectral-Galerkin heat step on one B200 (grid or box mode).

    ``precision="fp64"`` (default) is the plain form, FP64 throughout.
    ``precision="mixed"`` runs every DCT contraction of the step as split-BF16
    products on the tensor cores (tcgen05, FP32 accumulation) and keeps the
    modal iterates rounded to FP32; the latent source across the
    solidus-liquidus band, the property correction, the face fluxes, the
    Picard norms and the coefficient tables stay FP64. ``precision="fp32"``
    is the same with FP32 contractions on the CUDA cores (the FP32 arm of the
    precision study)."""

    def __init__(self, backend=None, context=None, *, mixing_omega=None,
                 convergence_tol=None, max_picard_iter=None, device=None, axis_min_ctas=None,
                 axis_cuda_cores=None, precision: str = "fp64"):
        if precision not in _lib.PLAN_PRECISION:
            raise ValueError(f"precision must be one of {sorted(_lib.PLAN_PRECISION)}")
        self.precision = precision
        self.backend = backend
        self.context = context
        # tile policy of the axis passes: explicit, else the autotuner's table, else default
        self.axis_min_ctas = axis_min_ctas
        # True: every FP64 axis pass on the CUDA-core kernels (no FP64 tensor cores);
        # None: the autotuner's table, else False
        self.axis_cuda_cores = axis_cuda_cores
        self.state: Optional[B200State] = None
        self.device = device
        self._req = (mixing_omega, convergence_tol, max_picard_iter)
        self._resolve_picard_params(np.float32)
        self.track_picard_history = False
        self.picard_history = []
        self._plan = None
        self._picard_cap_warned = False
        self._property_correction = False
        self._grid_latent = False
        self._latent_truncation_warned = False
        self.last_flags = 0  # sgh_step_out.flags of the last step (box truncation bits)
        self.last_status = None  # Picard outcome of the last step

    # ---- configuration -------------------------------------------------
    def _resolve_picard_params(self, dtype) -> None:
        num = self.context.num if self.context is not None else None

        def pick(explicit, attr, default):
            if explicit is not None:
                return explicit
            if num is not None and getattr(num, attr, None) is not None:
                return getattr(num, attr)
            return default

        om, tol, mx = self._req
        self.mixing_omega = dtype(pick(om, "picard_omega", 0.1))
        self.convergence_tol = dtype(pick(tol, "picard_tol", 1e-4))
        self.max_picard_iter = int(pick(mx, "max_picard_iter", 30))

    def initialize(self, context=None) -> B200State:
        if context is not None:
            self.context = context
        if self.context is None:
            raise RuntimeError("SimulationContext must be provided either at construction "
                               "or in initialize().")
        ctx = self.context
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("the b200 backend needs a CUDA device (no CPU fallback)")
        L = _lib.lib()
        self.finalize()
        self._resolve_picard_params(np.float64)
        cfg = make_config(ctx, float(self.mixing_omega), float(self.convergence_tol),
                          self.max_picard_iter)
        cfg.precision = _lib.PLAN_PRECISION[self.precision]
        policy = self.axis_min_ctas
        if policy is None:
            from .autotune import lookup
            policy = lookup(cfg)
        cfg.axis_min_ctas = int(policy or 0)
        cores = self.axis_cuda_cores
        if cores is None:
            from .autotune import lookup_kernel
            cores = lookup_kernel(cfg)
        cfg.axis_cuda_cores = 1 if cores else 0
        self.kernel_policy = int(cfg.axis_cuda_cores)
        self.tile_policy = int(cfg.axis_min_ctas)
        plan = C.c_void_p()
        _lib.check("sgh_plan_create", L.sgh_plan_create(C.byref(cfg), C.byref(plan)))
        self._plan = plan
        nbytes = C.c_uint64()
        _lib.check("sgh_plan_workspace_bytes", L.sgh_plan_workspace_bytes(plan, C.byref(nbytes)))
        dev = torch.device("cuda", torch.cuda.current_device()) if self.device is None \
            else torch.device(self.device)
        ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=dev)
        if ws.data_ptr() % 256:
            raise RuntimeError("workspace allocation is not 256-byte aligned")
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream(dev)
        _lib.check("sgh_plan_bind",
                   L.sgh_plan_bind(plan, C.c_void_p(ws.data_ptr()), nbytes.value,
                                   C.c_void_p(stream.cuda_stream)))
        g = ctx.geom
        sqrt_dV = math.sqrt(float(g.d.x * g.d.y * g.d.z))
        self.state = B200State(plan, ws, (cfg.nz, cfg.ny, cfg.nx), stream, sqrt_dV)
        self.state.size = (float(g.size.x), float(g.size.y), float(g.size.z))
        self._cfg = cfg
        model = getattr(ctx.mat, "model", None)
        self._property_correction = model is not None and not model.is_constant
        fine = getattr(ctx, "fine", None)
        self._grid_latent = fine is None and float(getattr(ctx.mat, "L_f", 0.0)) > 0.0
        if fine is not None:
            self.state.fine_mesh = B200FineMesh(self.state, fine)
        self._latent_truncation_warned = False
        if self._property_correction and self._grid_latent:
            logger.warning(
                "Temperature-dependent run in grid mode (no fine_mesh): the sharp latent-heat "
                "source is projected on the coarse grid and can ring.")
        self._picard_cap_warned = False
        return self.state

    # ---- stepping --------------------------------------------------------
    def _require(self):
        if self.state is None or self._plan is None:
            raise RuntimeError("Solver must be initialized before stepping.")

    def step(self, t: float, dt: float, eager: bool = False):
        """One time step. ``eager=True`` launches the same kernels one by one with
        the Picard loop driven from the host (for profilers and debugging)."""
        self._require()
        self._check_box_dt(dt)
        st = self.context.laser_path.get_state(t, dt)
        laser = laser_struct(st, dt, self._cfg.dt)
        out = _lib.SghStepOut()
        fn = "sgh_step_eager" if eager else "sgh_step"
        _lib.check(fn, getattr(_lib.lib(), fn)(self._plan, C.byref(laser), C.byref(out),
                                               C.c_void_p(self.state.stream.cuda_stream)))
        if self.state.fine_mesh is not None:
            self.state.fine_mesh.primed = True
        metrics = self._metrics(out, t)
        if self.track_picard_history:
            self.picard_history = self.read_picard_history()
        return self.state, metrics

    def read_picard_history(self):
        """Per-iteration record of the last step, as the reference keeps it with
        ``track_picard_history`` (``solvers/spectral.py:470-481``): ``iter``,
        ``rms_diff`` (rms of the residual), ``rho`` (its ratio to the previous
        iteration's) and ``true_rel_err``; written on the device by the
        convergence test, read in one copy (the first SGH_PICARD_HISTORY_MAX
        iterations)."""
        self._require()
        cap = _lib.PICARD_HISTORY_MAX
        buf = (C.c_double * (2 * cap))()
        n = C.c_int32()
        _lib.check("sgh_picard_history", _lib.lib().sgh_picard_history(
            self._plan, buf, cap, C.byref(n), C.c_void_p(self.state.stream.cuda_stream)))
        hist = []
        for k in range(min(n.value, cap)):
            rms, rel = buf[2 * k], buf[2 * k + 1]
            prev = hist[-1]["rms_diff"] if hist else 0.0
            hist.append({"iter": k, "rms_diff": rms, "rho": rms / prev if k > 0 and prev > 0 else None,
                         "true_rel_err": rel})
        return hist

    def _check_box_dt(self, dt) -> None:
        # The box history moves by v * num.dt (physics/spectral_ops.py:300-302)
        # while the face warm start moves by v * dt; the library shifts both by
        # v * dt of the plan, so box mode steps at the configured dt only.
        if self.state.fine_mesh is not None and float(dt) != float(self._cfg.dt):
            raise ValueError(f"box mode steps at the configured dt={self._cfg.dt!r} only "
                             f"(got dt={dt!r})")

    def _box_warning(self, flags) -> None:
        """One-time truncation warning (``solvers/spectral.py:545-586``)."""
        if not flags or self._latent_truncation_warned:
            return
        fm = self.state.fine_mesh
        hit = [name for bit, name in sorted(_lib.STEP_FLAGS.items()) if flags & bit]
        box_mm = (fm.nx_box * fm.dx_fine * 1e3, fm.ny_box * fm.dy_fine * 1e3,
                  fm.nz_box * fm.dz_fine * 1e3)
        logger.warning(
            "Latent-heat source reaches the fine-mesh box boundary (%s): the melt pool extends "
            "beyond the refined sub-box, so its latent heat is truncated. Enlarge "
            "fine_mesh.box_size (currently %.3g x %.3g x %.3g mm) to enclose the pool.",
            ", ".join(hit), *box_mm)
        self._latent_truncation_warned = True

    def _metrics(self, out, t):
        self.last_flags = int(out.flags)
        # "converged" | "capped" | "nonfinite" (the Picard loop stops on a
        # non-finite residual, as the reference's comparison with the
        # tolerance would never succeed on one)
        self.last_status = _lib.STEP_STATUS.get(int(out.status), int(out.status))
        self._box_warning(self.last_flags)
        conv = bool(out.converged)
        if not conv and out.n_iter > 0 and not self._picard_cap_warned:
            self._picard_cap_warned = True
            logger.warning(
                "Picard iteration hit max_picard_iter=%d at t=%.6g s without reaching "
                "picard_tol=%g (last relative residual %.3g, status %s). The returned field "
                "is not converged. Warned once per run.", self.max_picard_iter, t,
                float(self.convergence_tol), out.picard_rel_err,
                _lib.STEP_STATUS.get(out.status, out.status))
        return {"T_surface_max": float(out.T_surface_max), "P_laser": float(out.P_laser),
                "n_evap_iter": int(out.n_iter), "picard_converged": conv,
                "picard_rel_err": float(out.picard_rel_err)}

    def run(self, t0: float, n_steps: int, dt: Optional[float] = None):
        """Advance ``n_steps`` steps from time ``t0`` in one asynchronous launch.

        Laser states for ``t0 + i*dt`` are evaluated on the host up front and
        uploaded as a device table; the metrics of every step come back in one
        copy at the end. Returns the list of per-step metric dicts.
        """
        self._require()
        torch = _torch()
        dt = self._cfg.dt if dt is None else dt
        self._check_box_dt(dt)
        n = int(n_steps)
        if n <= 0:
            return []
        table = self.laser_table(t0, n, dt)
        outs = torch.empty(n * C.sizeof(_lib.SghStepOut), dtype=torch.uint8,
                           device=self.state.workspace.device)
        self.run_table(table, outs, n)
        host = outs.cpu().numpy()
        res = []
        for i in range(n):
            o = _lib.SghStepOut.from_buffer_copy(host[i * C.sizeof(_lib.SghStepOut):
                                                      (i + 1) * C.sizeof(_lib.SghStepOut)])
            res.append(self._metrics(o, t0 + i * dt))
        return res

    def laser_table(self, t0: float, n: int, dt: Optional[float] = None):
        """Device table (uint8 tensor) of ``sgh_laser`` for steps ``t0 + i*dt``."""
        torch = _torch()
        dt = self._cfg.dt if dt is None else dt
        arr = (_lib.SghLaser * n)()
        for i in range(n):
            arr[i] = laser_struct(self.context.laser_path.get_state(t0 + i * dt, dt), dt,
                                  self._cfg.dt)
        host = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8)
        return host.to(self.state.workspace.device)

    def run_table(self, table, outs, n: int, start: int = 0) -> None:
        """Enqueue ``n`` steps reading laser states ``start..start+n-1`` from ``table``
        (device) and writing ``sgh_step_out`` records into the same slots of ``outs``
        (device); returns without waiting."""
        lsz, osz = C.sizeof(_lib.SghLaser), C.sizeof(_lib.SghStepOut)
        if table.numel() < (start + n) * lsz or outs.numel() < (start + n) * osz:
            raise ValueError("laser or metrics table too short")
        if self.state.fine_mesh is not None and n > 0:
            self.state.fine_mesh.primed = True
        _lib.check("sgh_run", _lib.lib().sgh_run(
            self._plan, C.c_void_p(table.data_ptr() + start * lsz), int(n),
            C.c_void_p(outs.data_ptr() + start * osz), C.c_void_p(self.state.stream.cuda_stream)))

    def launch_counts(self):
        """``(pre, per_iteration, post)`` kernel launches of one step."""
        self._require()
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        _lib.check("sgh_plan_launch_counts", _lib.lib().sgh_plan_launch_counts(
            self._plan, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    @staticmethod
    def decode_outs(host_bytes, n):
        """Decode ``n`` ``sgh_step_out`` records from a host byte buffer."""
        sz = C.sizeof(_lib.SghStepOut)
        return [_lib.SghStepOut.from_buffer_copy(host_bytes[i * sz:(i + 1) * sz]) for i in range(n)]

    # ---- state access ------------------------------------------------------
    def set_state(self, temperature_field) -> None:
        """Modes from a cell-centred field: ``a = sqrt(dV) DCT_II(T)`` (``solvers/spectral.py:588-619``)."""
        if self.state is None or self._plan is None:
            raise RuntimeError("Solver must be initialized before calling set_state().")
        torch = _torch()
        T = torch.as_tensor(temperature_field, dtype=torch.float64,
                            device=self.state.workspace.device).contiguous()
        if tuple(T.shape) != self.state.shape:
            raise ValueError(f"field shape {tuple(T.shape)} != modes shape {self.state.shape}")
        _lib.check("sgh_project_volume", _lib.lib().sgh_project_volume(
            self._plan, C.c_void_p(T.data_ptr()), C.c_void_p(self.state.a.data_ptr()),
            C.c_void_p(self.state.stream.cuda_stream)))
        self.state.stream.synchronize()

    def surface_temperature(self, top: bool = True, modes=None):
        """Top (or bottom) face temperature of ``modes`` (default: the state), (ny, nx)."""
        self._require()
        torch = _torch()
        a = self.state.a if modes is None else modes
        nz, ny, nx = self.state.shape
        out = torch.empty((ny, nx), dtype=torch.float64, device=self.state.workspace.device)
        _lib.check("sgh_surface_temperature", _lib.lib().sgh_surface_temperature(
            self._plan, C.c_void_p(a.data_ptr()), 1 if top else 0, C.c_void_p(out.data_ptr()),
            C.c_void_p(self.state.stream.cuda_stream)))
        return out

    def volume_temperature(self, modes=None):
        """Cell-centred temperature ``IDCT_II(a)/sqrt(dV)``, (nz, ny, nx)."""
        self._require()
        torch = _torch()
        a = self.state.a if modes is None else modes
        out = torch.empty(self.state.shape, dtype=torch.float64, device=self.state.workspace.device)
        _lib.check("sgh_reconstruct_volume", _lib.lib().sgh_reconstruct_volume(
            self._plan, C.c_void_p(a.data_ptr()), C.c_void_p(out.data_ptr()),
            C.c_void_p(self.state.stream.cuda_stream)))
        return out

    def dct3d(self, x, kind: int = 2):
        """Orthonormal 3-D DCT-II (``kind=2``) or DCT-III (``kind=3``) of a
        field of the plan's shape with the plan's own contractions (FP64, or
        split-BF16 on the tensor cores in a mixed plan); a new tensor."""
        self._require()
        torch = _torch()
        x = torch.as_tensor(x, dtype=torch.float64, device=self.state.workspace.device).contiguous()
        if tuple(x.shape) != self.state.shape:
            raise ValueError(f"field shape {tuple(x.shape)} != plan shape {self.state.shape}")
        out = torch.empty_like(x)
        _lib.check("sgh_dct3d", _lib.lib().sgh_dct3d(
            self._plan, int(kind), C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
            C.c_void_p(self.state.stream.cuda_stream)))
        return out

    # ---- checkpoints ------------------------------------------------------
    CHECKPOINT_FORMAT = "sgh_b200 modal checkpoint 1"

    def _config_digest(self) -> str:
        import hashlib
        c = _lib.SghConfig.from_buffer_copy(bytes(self._cfg))
        c.axis_min_ctas = 0
        c.axis_cuda_cores = 0
        return hashlib.sha256(bytes(c)).hexdigest()

    def checkpoint(self, t: float = 0.0, step: int = 0) -> dict:
        """Host copy of everything a later step reads, for an exact resume.

        ``modes`` / ``time`` / ``step`` follow the datasets of the reference's
        ``modes.h5`` (``io_utils/spectral_fs_io.py:207-241``): modes as
        ``(1, nz, ny, nx)``. The rest is the warm start the reference keeps in
        memory between steps: the previous evaporation flux
        (``buffers.q_evap_old``), the previous converged field
        (``_T_prev_full``), the previous latent modes (``_Q_latent_modes_prev``,
        grid mode) and the box history (``fine_mesh.T_prev`` / ``Q_prev``).
        """
        self._require()
        st = self.state
        flags = C.c_int32()
        _lib.check("sgh_state_flags", _lib.lib().sgh_state_flags(
            self._plan, C.byref(flags), C.c_void_p(st.stream.cuda_stream)))
        ck = {
            "format": np.array(self.CHECKPOINT_FORMAT),
            "config_digest": np.array(self._config_digest()),
            "modes": st.a.cpu().numpy()[None].copy(),
            "time": np.array([float(t)], dtype=np.float64),
            "step": np.array([int(step)], dtype=np.int64),
            "q_evap_old": st.q_evap_old.cpu().numpy().copy(),
            "T_prev_full": st.T_prev.cpu().numpy().copy(),
            "Q_latent_modes_prev": st.buffer("Q_modes").cpu().numpy().copy(),
            "flags": np.array(int(flags.value), dtype=np.int32),
        }
        fm = st.fine_mesh
        if fm is not None:
            ck["fine_T_prev"] = fm._T_prev.cpu().numpy().copy()
            ck["fine_Q_prev"] = fm._Q_prev.cpu().numpy().copy()
        return ck

    def restore(self, ck: dict) -> tuple:
        """Load a :meth:`checkpoint` into this instance (same configuration);
        returns ``(time, step)`` of the checkpoint."""
        self._require()
        torch = _torch()
        if str(ck["format"]) != self.CHECKPOINT_FORMAT:
            raise ValueError(f"not a {self.CHECKPOINT_FORMAT!r} checkpoint")
        if str(ck["config_digest"]) != self._config_digest():
            raise ValueError("checkpoint was written by an instance with another configuration")
        st = self.state
        modes = np.asarray(ck["modes"])
        if modes.shape != (1, *st.shape):
            raise ValueError(f"checkpoint modes {modes.shape} do not match {(1, *st.shape)}")
        flags = int(ck["flags"])
        fm = st.fine_mesh
        if (fm is not None) != ("fine_T_prev" in ck):
            raise ValueError("checkpoint and instance disagree on box mode")

        def put(dst, arr):
            dst.copy_(torch.as_tensor(np.ascontiguousarray(arr, dtype=np.float64)).reshape(dst.shape))

        with torch.cuda.stream(st.stream):
            put(st.a, modes[0])
            put(st.q_evap_old, ck["q_evap_old"])
            put(st.T_prev, ck["T_prev_full"])
            put(st.buffer("Q_modes"), ck["Q_latent_modes_prev"])
            if fm is not None:
                put(fm._T_prev, ck["fine_T_prev"])
                put(fm._Q_prev, ck["fine_Q_prev"])
        _lib.check("sgh_state_set_flags", _lib.lib().sgh_state_set_flags(
            self._plan, flags, C.c_void_p(st.stream.cuda_stream)))
        st.stream.synchronize()
        if fm is not None:
            fm.primed = bool(flags & 2)
        return float(ck["time"][0]), int(ck["step"][0])

    def save_checkpoint(self, path: str, t: float = 0.0, step: int = 0) -> str:
        """:meth:`checkpoint` written as ``.npz`` (dataset names as above)."""
        ck = self.checkpoint(t, step)
        path = str(path)
        if not path.endswith(".npz"):
            path += ".npz"
        np.savez(path, **ck)
        return path

    def load_checkpoint(self, path: str) -> tuple:
        """:meth:`restore` from a file written by :meth:`save_checkpoint`."""
        with np.load(str(path)) as f:
            return self.restore({k: f[k] for k in f.files})

    def reset(self) -> None:
        """Back to the initial condition (keeps the plan and its graph)."""
        self._require()
        _lib.check("sgh_state_reset", _lib.lib().sgh_state_reset(
            self._plan, C.c_void_p(self.state.stream.cuda_stream)))
        if self.state.fine_mesh is not None:
            self.state.fine_mesh.primed = False
        self._latent_truncation_warned = False

    def finalize(self) -> None:
        if self._plan is not None:
            if self.state is not None:
                self.state.stream.synchronize()
            _lib.lib().sgh_plan_destroy(self._plan)
            self._plan = None
        self.state = None

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass
