"""CPU oracle for the spectral-Galerkin heat time step (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
The B200 backend (``spectral_galerkin_heat_b200``) never calls into it and has
no CPU fallback.

It restates, in plain NumPy/SciPy and in FP64, the grid-mode time step of the
reference solver ``SpectralSolver.step`` (``solvers/spectral.py:219-543``) and
the pieces it calls:

* grid tables ``SpectralGrid`` (``physics/spectral_state.py:98-143``) and the
  normalisation ``_C_coef`` (``physics/spectral_helpers.py:26-46``);
* propagators ``precompute_K_KK`` (``physics/spectral_state.py:374-421``);
* laser flux ``super_gaussian_flux`` / ``gaussian_cell_integrated_flux``
  (``core/laser.py:42-91``);
* warm-start shift ``_ndshift`` / ``shift_flux``
  (``physics/spectral_cpu_kernels.py:328-371, 392-396``);
* ``update_modes_etd1`` / ``add_source_term_modes`` /
  ``add_bottom_surface_source`` (``spectral_cpu_kernels.py:83-113``);
* latent source, constant and blended-rho forms
  (``spectral_cpu_kernels.py:115-140``, ``core/properties.py:197-239``);
* evaporation flux (``spectral_cpu_kernels.py:144-162``);
* property fluctuations and the divergence-form correction stencil
  (``core/properties.py:154-194``, ``spectral_cpu_kernels.py:165-252``,
  ``physics/spectral_ops.py:105-170``);
* surface / volume reconstructions and projections
  (``physics/spectral_ops.py:83-102, 210-231``);
* output reconstruction: the node-centred field, point values and the three
  temperature profiles (``physics/spectral_helpers.py:146-333``), written as
  explicit cosine-series contractions (the reference evaluates the node
  field as a weighted DCT-I; both give the same series).

The orthonormal DCT-II/III pair is ``scipy.fft.dctn(type=2|3, norm='ortho')``,
the same third-party routine the reference calls
(``spectral_cpu_kernels.py:374-389``; reference pins scipy 1.17.1 in
``uv.lock``; this image has 1.18.1). ``dct_matrix`` restates the published
definition ``C[k, n] = w_k cos(pi k (2n+1) / (2N))`` so tests can check SciPy
against it.

Pinning: ``tests/golden/make_golden.py`` runs the reference itself on the same
inputs and stores its outputs under ``tests/golden/``; ``tests/test_oracle.py``
checks this module against those fixtures.

Box mode (``fine_mesh``): the laser-following fine box ``FineMeshState``
(``physics/spectral_state.py:166-239``) with its window
``_calculate_subgrid_indices`` (``physics/spectral_helpers.py:49-85``), the box
reconstruction and projection (``physics/spectral_ops.py:53-74, 173-207``), the
3-D history shift (``physics/spectral_ops.py:292-306`` with the tables of
``_ndshift``, ``spectral_cpu_kernels.py:302-371``) and the truncation check
(``solvers/spectral.py:545-586``) are restated in :class:`FineBox`.
"""
from __future__ import annotations

import ast
import math
import warnings

import numpy as np
import scipy.fft
import scipy.special

__all__ = ["OracleSolver", "FineBox", "dct2", "dct3", "dct_matrix", "evaluate_expression"]


# --------------------------------------------------------------------------
# transforms
# --------------------------------------------------------------------------

def dct2(x, workers=None):
    """Orthonormal DCT-II over every axis (``spectral_cpu_kernels.py:374-381``)."""
    x = np.ascontiguousarray(x)
    return scipy.fft.dctn(x, type=2, norm="ortho", axes=tuple(range(x.ndim)),
                          workers=workers)


def dct3(x, workers=None):
    """Orthonormal DCT-III (inverse of :func:`dct2`) over every axis (``:383-389``)."""
    x = np.ascontiguousarray(x)
    return scipy.fft.dctn(x, type=3, norm="ortho", axes=tuple(range(x.ndim)),
                          workers=workers)


def dct_matrix(n: int) -> np.ndarray:
    """Orthonormal DCT-II matrix: ``X = M @ x``; ``M.T`` is the DCT-III."""
    k = np.arange(n, dtype=np.float64)[:, None]
    j = np.arange(n, dtype=np.float64)[None, :]
    w = np.full((n, 1), math.sqrt(2.0 / n))
    w[0, 0] = math.sqrt(1.0 / n)
    return w * np.cos(np.pi * k * (2.0 * j + 1.0) / (2.0 * n))


# --------------------------------------------------------------------------
# property expressions (``core/property_expr.py`` grammar, evaluated with numpy)
# --------------------------------------------------------------------------

_FUNCS = {
    "sqrt": np.sqrt, "exp": np.exp, "log": np.log, "log2": np.log2, "log10": np.log10,
    "sin": np.sin, "cos": np.cos, "tan": np.tan, "asin": np.arcsin, "acos": np.arccos,
    "atan": np.arctan, "atan2": np.arctan2, "sinh": np.sinh, "cosh": np.cosh,
    "tanh": np.tanh, "asinh": np.arcsinh, "acosh": np.arccosh, "atanh": np.arctanh,
    "fabs": np.abs, "ceil": np.ceil, "floor": np.floor, "trunc": np.trunc,
    "log1p": np.log1p, "expm1": np.expm1,
}


def evaluate_expression(source: str, T):
    """Evaluate a property expression of ``T`` (a number or the whitelisted grammar)."""
    try:
        return T * 0.0 + float(source)
    except ValueError:
        pass

    def ev(node):
        if isinstance(node, ast.Constant):
            return node.value
        if isinstance(node, ast.Name):
            return T if node.id == "T" else {"pi": math.pi, "e": math.e}[node.id]
        if isinstance(node, ast.BinOp):
            a, b = ev(node.left), ev(node.right)
            return {ast.Add: lambda: a + b, ast.Sub: lambda: a - b,
                    ast.Mult: lambda: a * b, ast.Div: lambda: a / b,
                    ast.Pow: lambda: a ** b}[type(node.op)]()
        if isinstance(node, ast.UnaryOp):
            v = ev(node.operand)
            return -v if isinstance(node.op, ast.USub) else v
        if isinstance(node, ast.Call):
            return _FUNCS[node.func.id](*(ev(a) for a in node.args))
        raise ValueError(f"unsupported node {type(node).__name__}")

    return ev(ast.parse(str(source).strip(), mode="eval").body)


class _Prop:
    """Solid/liquid branches of one property (``TempProperty``, ``core/properties.py:80-150``)."""

    def __init__(self, tprop, T_s, T_l):
        self.solid = tprop.solid.source
        self.liquid = tprop.liquid.source
        self.const = bool(tprop.is_constant)
        self.T_s, self.T_l = float(T_s), float(T_l)

    def blended(self, T):
        """``TempProperty.__call__``: ``(1-f_l) p_s + f_l p_l`` with ``f_l`` by division."""
        if self.const:
            return evaluate_expression(self.solid, T)
        ps = evaluate_expression(self.solid, T)
        pl = evaluate_expression(self.liquid, T)
        if self.T_l <= self.T_s:
            fl = np.where(np.asarray(T) >= self.T_s, 1.0, 0.0)
        else:
            fl = np.clip((T - self.T_s) / (self.T_l - self.T_s), 0.0, 1.0)
        return (1.0 - fl) * ps + fl * pl


def _fl_kernel(T, t_sol, inv_band, degenerate):
    """Liquid fraction as the fused kernels compute it (multiply by ``1/band``)."""
    if degenerate:
        return np.where(T >= t_sol, 1.0, 0.0)
    return np.clip((T - t_sol) * inv_band, 0.0, 1.0)


# --------------------------------------------------------------------------
# box mode
# --------------------------------------------------------------------------

def _ccoef(n, L):
    c = math.sqrt(2.0 / L) * np.ones(n)
    c[0] = math.sqrt(1.0 / L)
    return c


def _shift_table(n, shift):
    """Clamped neighbours, linear weights and in-range mask of an order-1 shift
    (``_shift_axis_tables``, ``spectral_cpu_kernels.py:328-350``)."""
    p = np.arange(n, dtype=np.float64) - float(shift)
    i0 = np.floor(p).astype(np.int64)
    t = p - i0
    inside = (p >= 0.0) & (p <= n - 1)
    return np.clip(i0, 0, n - 1), np.clip(i0 + 1, 0, n - 1), 1.0 - t, t, inside


def shift_xy(f, sy, sx, nearest):
    """Order-1 translation of a 2-D field or of every z-layer of a 3-D field by
    ``(sy, sx)`` pixels, ``mode='nearest'`` or ``'constant'`` with 0 outside
    (``_ndshift``, ``spectral_cpu_kernels.py:353-371``)."""
    ny, nx = f.shape[-2:]
    a, b, wy0, wy1, iny = _shift_table(ny, sy)
    c, d, wx0, wx1, inx = _shift_table(nx, sx)
    wy0, wy1 = wy0[:, None], wy1[:, None]
    fa, fb = f[..., a, :], f[..., b, :]
    out = (wy0 * (wx0 * fa[..., c] + wx1 * fa[..., d])
           + wy1 * (wx0 * fb[..., c] + wx1 * fb[..., d]))
    if not nearest:
        out[..., ~(iny[:, None] & inx[None, :])] = 0.0
    return out


def subgrid_start(pos, d, n_total, n_box):
    """Window start (``_calculate_subgrid_indices``, ``physics/spectral_helpers.py:49-85``)."""
    idx_global = round(max(0.0, min(pos / d, n_total - 1)))
    start = idx_global - n_box // 2
    max_start = max(0, n_total - n_box)
    return max(0, min(start, max_start))


class FineBox:
    """Laser-following fine box (``FineMeshState``, ``physics/spectral_state.py:166-239``)."""

    def __init__(self, fine, d, size, n):
        dx, dy, dz = d
        Lx, Ly, Lz = size
        self.refinement = int(fine.refinement)
        Lxb, Lyb, Lzb = (float(v) for v in fine.box_size)
        r = self.refinement
        self.dx_fine, self.dy_fine, self.dz_fine = dx / r, dy / r, dz / r
        dfine = (self.dx_fine, self.dy_fine, self.dz_fine)
        self.n_fine_totals = [int(np.ceil(L / q)) for L, q in zip((Lx, Ly, Lzb), dfine)]
        coords = [(np.arange(m) + 0.5) * q for m, q in zip(self.n_fine_totals, dfine)]
        coords[2] = (Lz - Lzb) + coords[2]
        self.B_fine_full = [_ccoef(nm, L)[:, None] * np.cos(np.pi * np.arange(nm)[:, None] * c[None, :] / L)
                            for nm, c, L in zip(n, coords, (Lx, Ly, Lz))]
        self.nx_box = min(int(np.ceil(Lxb / self.dx_fine)), self.n_fine_totals[0])
        self.ny_box = min(int(np.ceil(Lyb / self.dy_fine)), self.n_fine_totals[1])
        self.nz_box = min(int(np.ceil(Lzb / self.dz_fine)), self.n_fine_totals[2])
        self.B_fine = [np.zeros((n[0], self.nx_box)), np.zeros((n[1], self.ny_box)),
                       self.B_fine_full[2][:, :self.nz_box]]
        self.dV_fine = self.dx_fine * self.dy_fine * self.dz_fine
        self.window = (-1, -1)
        self.T_prev = None
        self.Q_prev = None

    @property
    def shape(self):
        return (self.nz_box, self.ny_box, self.nx_box)

    def update(self, x, y):
        """Slide the x and y windows to the laser (``FineMeshState.update``)."""
        ix = subgrid_start(x, self.dx_fine, self.n_fine_totals[0], self.nx_box)
        iy = subgrid_start(y, self.dy_fine, self.n_fine_totals[1], self.ny_box)
        self.B_fine[0][:, :] = self.B_fine_full[0][:, ix:ix + self.nx_box]
        self.B_fine[1][:, :] = self.B_fine_full[1][:, iy:iy + self.ny_box]
        self.window = (ix, iy)

    def reconstruct(self, a):
        """``reconstruct_temperature_box`` (``physics/spectral_ops.py:173-179``)."""
        return np.einsum("ZYX,Zz,Yy,Xx->zyx", a, self.B_fine[2], self.B_fine[1], self.B_fine[0],
                         optimize=True)

    def project(self, f):
        """``project_box_to_modes`` (``physics/spectral_ops.py:53-74``)."""
        return np.einsum("zyx,Zz,Yy,Xx->ZYX", f, self.B_fine[2], self.B_fine[1], self.B_fine[0],
                         optimize=True) * self.dV_fine

    def shift_history(self, vx, vy, dt):
        """``shift_latent_heat_history`` (``physics/spectral_ops.py:292-306``)."""
        if self.T_prev is None:
            return
        sy, sx = -(vy * dt) / self.dy_fine, -(vx * dt) / self.dx_fine
        self.T_prev = shift_xy(self.T_prev, sy, sx, nearest=True)
        if self.Q_prev is not None:
            self.Q_prev = shift_xy(self.Q_prev, sy, sx, nearest=False)

    def truncation(self, Q):
        """Faces of the box reached by the source (``solvers/spectral.py:545-586``):
        flag bits 1 (floor), 2 (x window edge), 4 (y window edge)."""
        peak = float(np.max(np.abs(Q)))
        if peak <= 0.0:
            return 0
        thr = 1e-2 * peak
        flags = 0
        if float(np.max(np.abs(Q[0, :, :]))) > thr:
            flags |= 1
        if self.nx_box < self.n_fine_totals[0] and float(np.max(np.abs(Q[:, :, (0, -1)]))) > thr:
            flags |= 2
        if self.ny_box < self.n_fine_totals[1] and float(np.max(np.abs(Q[:, (0, -1), :]))) > thr:
            flags |= 4
        return flags


# --------------------------------------------------------------------------
# the solver
# --------------------------------------------------------------------------

class OracleSolver:
    """FP64 grid-mode restatement of ``SpectralSolver`` (``solvers/spectral.py:38-628``).

    ``initialize`` / ``step`` / ``set_state`` follow the reference contract;
    ``step`` returns ``(self, metrics)`` with host floats.
    """

    def __init__(self, context=None, *, mixing_omega=None, convergence_tol=None,
                 max_picard_iter=None, workers=None):
        self.context = context
        self._req = (mixing_omega, convergence_tol, max_picard_iter)
        self.workers = workers
        self.a = None
        self.picard_history = []
        self.track_picard_history = False
        self._cap_warned = False

    # ---- setup -----------------------------------------------------------
    def _picard_params(self):
        num = self.context.num

        def pick(explicit, attr, default):
            if explicit is not None:
                return explicit
            v = getattr(num, attr, None)
            return default if v is None else v

        om, tol, mx = self._req
        self.omega = float(pick(om, "picard_omega", 0.1))
        self.tol = float(pick(tol, "picard_tol", 1e-4))
        self.max_iter = int(pick(mx, "max_picard_iter", 30))

    def initialize(self, context=None):
        if context is not None:
            self.context = context
        if self.context is None:
            raise RuntimeError("SimulationContext must be provided either at construction "
                               "or in initialize().")
        ctx = self.context
        g, mat, num = ctx.geom, ctx.mat, ctx.num
        nx, ny, nz = int(g.n.x), int(g.n.y), int(g.n.z)
        Lx, Ly, Lz = float(g.size.x), float(g.size.y), float(g.size.z)
        dx, dy, dz = float(g.d.x), float(g.d.y), float(g.d.z)
        self.shape = (nz, ny, nx)
        self.dx, self.dy, self.dz = dx, dy, dz
        self.x = (np.arange(nx) + 0.5) * dx
        self.y = (np.arange(ny) + 0.5) * dy

        def ccoef(n, L):
            c = math.sqrt(2.0 / L) * np.ones(n)
            c[0] = math.sqrt(1.0 / L)
            return c

        Cz = ccoef(nz, Lz)
        sign = np.power(-1.0, np.arange(nz, dtype=np.float64))
        self.Cp_top = Cz * sign
        self.Cp_bot = Cz.copy()
        self.dct_scale = (dx * dy) * np.sqrt((nx * ny) / (Lx * Ly))
        self.recon_scale = np.sqrt(nx * ny) / np.sqrt(Lx * Ly)
        self.sqrt_dV = np.sqrt(float(dx * dy * dz))

        self._picard_params()
        self.K, self.KK = self.propagators(mat, num.dt, (nz, ny, nx), (Lz, Ly, Lx))

        self.a = np.zeros(self.shape)
        self.a[0, 0, 0] = float(mat.T0) * math.sqrt(Lx * Ly * Lz)
        self.q_evap_old = np.zeros((ny, nx))
        self.q_evap = np.zeros((ny, nx))
        self.a_temp = np.zeros(self.shape)

        model = getattr(mat, "model", None)
        fine = getattr(ctx, "fine", None)
        self.box = None if fine is None else FineBox(fine, (dx, dy, dz), (Lx, Ly, Lz), (nx, ny, nz))
        self.box_flags = 0
        self.grid_latent = fine is None and float(getattr(mat, "L_f", 0.0)) > 0.0
        self.prop_corr = model is not None and not model.is_constant
        Ts, Tl = float(mat.T_solidus), float(mat.T_liquidus)
        self.T_s, self.T_l = Ts, Tl
        if model is not None:
            self.k_prop = _Prop(model.k, Ts, Tl)
            self.rho_prop = _Prop(model.rho, Ts, Tl)
            self.c_prop = _Prop(model.c, Ts, Tl)
        self.model = model
        if self.prop_corr:
            self.kbar = float(mat.k)
            self.abar = float(mat.rho) * float(mat.Cp)
        self.T_prev_full = (np.full(self.shape, float(mat.T0))
                            if (self.prop_corr or self.grid_latent) else None)
        self.Q_modes_prev = None

        lp = ctx.laser
        prof = getattr(lp, "profile", "gaussian")
        order = {"gaussian": 2.0, "flat_top": 12.0}.get(
            str(prof).lower(), float(getattr(lp, "super_gaussian_order", 2.0)))
        self.order = order
        self.cell_integrated = bool(getattr(lp, "cell_integrated", False))
        n = order
        self.area_factor = math.pi * 2.0 ** (1.0 - 2.0 / n) * math.gamma(2.0 / n) / n
        return self

    @staticmethod
    def propagators(mat, dt, shape, lengths):
        """``K = exp(-alpha lam dt)``, ``KK = phi_1 / (rho c)`` (``spectral_state.py:374-421``)."""
        nz, ny, nx = shape
        Lz, Ly, Lx = lengths
        kz, ky, kx = [np.pi * np.arange(n) / L for n, L in zip(shape, lengths)]
        alpha = mat.k / (mat.rho * mat.Cp)
        rc = mat.rho * mat.Cp
        lam = alpha * (kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2)
        K = np.exp(-lam * dt)
        lam[0, 0, 0] = 1.0
        phi = (K - 1.0) / (-lam)
        phi[0, 0, 0] = dt
        return K, phi / rc

    # ---- face pieces -----------------------------------------------------
    def laser_flux(self, x0, y0, I0):
        lp = self.context.laser
        rx, ry = float(lp.r_x), float(lp.r_y)
        if self.cell_integrated:
            s2 = math.sqrt(2.0)
            hx, hy = self.dx, self.dy
            nxm = rx * math.sqrt(math.pi / 8.0)
            nym = ry * math.sqrt(math.pi / 8.0)
            erf = scipy.special.erf
            mx = nxm * (erf((self.x - x0 + hx / 2.0) * s2 / rx)
                        - erf((self.x - x0 - hx / 2.0) * s2 / rx)) / hx
            my = nym * (erf((self.y - y0 + hy / 2.0) * s2 / ry)
                        - erf((self.y - y0 - hy / 2.0) * s2 / ry)) / hy
            return I0 * (my[:, None] * mx[None, :])
        ux = (self.x[None, :] - x0) / rx
        uy = (self.y[:, None] - y0) / ry
        r2 = ux * ux + uy * uy
        if self.order == 2.0:
            shape = np.exp(-2.0 * r2)
        else:
            shape = np.exp(-2.0 * r2 ** (self.order / 2.0))
        return I0 * shape

    @staticmethod
    def _axis_table(n, shift):
        p = np.arange(n, dtype=np.float64) - float(shift)
        i0 = np.floor(p).astype(np.int64)
        t = p - i0
        inside = (p >= 0.0) & (p <= n - 1)
        return np.clip(i0, 0, n - 1), np.clip(i0 + 1, 0, n - 1), 1.0 - t, t, inside

    def shift(self, f, sx_m, sy_m):
        """Order-1 shift, zero outside (``_ndshift`` ``mode='constant'``)."""
        ny, nx = f.shape
        a, b, wy0, wy1, iny = self._axis_table(ny, sy_m / self.dy)
        c, d, wx0, wx1, inx = self._axis_table(nx, sx_m / self.dx)
        out = (wy0[:, None] * (wx0[None, :] * f[np.ix_(a, c)] + wx1[None, :] * f[np.ix_(a, d)])
               + wy1[:, None] * (wx0[None, :] * f[np.ix_(b, c)] + wx1[None, :] * f[np.ix_(b, d)]))
        out[~(iny[:, None] & inx[None, :])] = 0.0
        return out

    def evaporation(self, Ts):
        mat = self.context.mat
        P0, Tb, dH, Rv, Tliq = (float(mat.Pa), float(mat.T_boil), float(mat.DeltaH_LV),
                                float(mat.R_v), float(mat.T_liquidus))
        f1 = 0.82 * dH * P0 / np.sqrt(2 * np.pi * Rv)
        f2 = dH / (Rv * Tb)
        with np.errstate(all="ignore"):
            q = f1 * ((1.0 / np.sqrt(Ts)) * np.exp(f2 * (1.0 - Tb / Ts)))
        return np.where(Ts < Tliq, 0.0, q)

    def surface_T(self, a, top=True):
        w = self.Cp_top if top else self.Cp_bot
        A = np.einsum("p,pij->ij", w, a, optimize=True)
        return self.recon_scale * dct3(A, self.workers)

    def face_dct(self, q):
        return self.dct_scale * dct2(q, self.workers)

    # ---- volume pieces ---------------------------------------------------
    def reconstruct_volume(self, a):
        return dct3(a, self.workers) / self.sqrt_dV

    def project_volume(self, f):
        return dct2(f, self.workers) * self.sqrt_dV

    def _band(self):
        degenerate = self.T_l <= self.T_s
        inv = 0.0 if degenerate else 1.0 / (self.T_l - self.T_s)
        return self.T_s, inv, degenerate

    def latent_source(self, T, T_prev):
        """Grid-mode latent sink (``spectral_ops.py:270-289``)."""
        mat, dt = self.context.mat, self.context.num.dt
        Lf = float(mat.L_f)
        if self.model is not None and not self.model.is_constant:
            ts, inv, deg = self._band()
            flc = _fl_kernel(T, ts, inv, deg)
            flp = _fl_kernel(T_prev, ts, inv, deg)
            rho = ((1.0 - flc) * evaluate_expression(self.rho_prop.solid, T)
                   + flc * evaluate_expression(self.rho_prop.liquid, T))
            return -rho * Lf * (flc - flp) * (1.0 / dt)
        inv = 1.0 / (self.T_l - self.T_s)
        fc = np.clip((T - self.T_s) * inv, 0.0, 1.0)
        fp = np.clip((T_prev - self.T_s) * inv, 0.0, 1.0)
        return (-float(mat.rho) * Lf / dt) * (fc - fp)

    def correction_modes(self, a_trial):
        """``sqrt(dV) DCT(div(k' grad T) - a' (T - T_prev)/dt)`` (``spectral_ops.py:105-170``)."""
        dt = self.context.num.dt
        T = self.reconstruct_volume(a_trial)
        ts, inv, deg = self._band()
        fl = _fl_kernel(T, ts, inv, deg)
        om = 1.0 - fl
        kv = (om * evaluate_expression(self.k_prop.solid, T)
              + fl * evaluate_expression(self.k_prop.liquid, T))
        rv = (om * evaluate_expression(self.rho_prop.solid, T)
              + fl * evaluate_expression(self.rho_prop.liquid, T))
        cv = (om * evaluate_expression(self.c_prop.solid, T)
              + fl * evaluate_expression(self.c_prop.liquid, T))
        kp = kv - self.kbar
        ap = rv * cv - self.abar
        idx, idy, idz = 1.0 / self.dx, 1.0 / self.dy, 1.0 / self.dz

        def grad(F, axis, inv_h):
            G = np.empty_like(F)
            sl = [slice(None)] * 3

            def s(i):
                q = list(sl)
                q[axis] = i
                return tuple(q)
            n = F.shape[axis]
            G[s(slice(1, n - 1))] = (F[s(slice(2, n))] - F[s(slice(0, n - 2))]) * (0.5 * inv_h)
            G[s(0)] = (F[s(1)] - F[s(0)]) * inv_h
            G[s(n - 1)] = (F[s(n - 1)] - F[s(n - 2)]) * inv_h
            return G

        gx = kp * grad(T, 2, idx)
        gy = kp * grad(T, 1, idy)
        gz = kp * grad(T, 0, idz)
        f = (grad(gx, 2, idx) + grad(gy, 1, idy) + grad(gz, 0, idz)
             - ap * ((T - self.T_prev_full) * (1.0 / dt)))
        return self.project_volume(f)

    # ---- the step --------------------------------------------------------
    def step(self, t, dt):
        if self.a is None:
            raise RuntimeError("Solver must be initialized before step().")
        ctx = self.context
        mat, lp = ctx.mat, ctx.laser
        st = ctx.laser_path.get_state(t, dt)
        vx, vy = st.v
        # the absorptivity is a float64 scalar in the reference, so a float32
        # power (G-code paths) is widened before the product (core/laser.py:110-112)
        I0 = (float(lp.absorptivity) * float(st.power) / (self.area_factor * float(lp.ref_area))
              if st.is_on else 0.0)
        q_las = self.laser_flux(st.x, st.y, I0)
        P_laser = float(np.sum(q_las) * self.dx * self.dy)

        self.a *= self.K
        aK = self.a
        KK = self.KK
        T0 = float(mat.T0)
        htop, hbot = float(mat.h_conv_top), float(mat.h_conv_bottom)
        Ct, Cb = self.Cp_top[:, None, None], self.Cp_bot[:, None, None]
        box = self.box
        if box is not None:
            # reposition, seed the history on the first step, shift it (solvers/spectral.py:288-294)
            box.update(st.x, st.y)
            if box.T_prev is None:
                box.T_prev = box.reconstruct(aK).copy()
                if box.Q_prev is None:
                    box.Q_prev = np.zeros(box.shape)
            box.shift_history(vx, vy, ctx.num.dt)

        q_shift = self.shift(self.q_evap_old, vx * dt, vy * dt)
        S_top = self.face_dct(q_las - q_shift)
        a_temp = aK + KK * Ct * S_top
        if box is not None and box.T_prev is not None and box.Q_prev is not None:
            a_temp += KK * box.project(box.Q_prev)
        elif self.grid_latent and self.Q_modes_prev is not None:
            a_temp += KK * self.Q_modes_prev
        if htop > 0:
            Ts0 = self.surface_T(a_temp, top=True)
            a_temp += KK * Ct * self.face_dct(-htop * (Ts0 - T0))
        if hbot > 0:
            Tb0 = self.surface_T(a_temp, top=False)
            a_temp += KK * Cb * self.face_dct(-hbot * (Tb0 - T0))
        S_las = self.face_dct(q_las)
        S_bot = None
        if hbot > 0:
            Tb = self.surface_T(a_temp, top=False)
            qc = -hbot * (Tb - T0)
            if self.prop_corr:
                qc = qc * (self.kbar / self.k_prop.blended(Tb))
            S_bot = self.face_dct(qc)

        n_el = float(a_temp.size)
        it, rel, converged = -1, float("nan"), False
        Qm = None
        Q_raw = None
        if self.track_picard_history:
            self.picard_history = []
        for it in range(self.max_iter):
            a_old = a_temp
            Ts = self.surface_T(a_old, top=True)
            q_ev = self.evaporation(Ts)
            q_cv = htop * (Ts - T0) if htop > 0 else 0.0
            if self.prop_corr:
                S_raw = self.face_dct((q_las - q_ev - q_cv) * (self.kbar / self.k_prop.blended(Ts)))
            else:
                S_raw = S_las - self.face_dct(q_ev)
                if htop > 0:
                    S_raw = S_raw - self.face_dct(q_cv)
            Qm = None
            if box is not None and box.T_prev is not None:
                Q_raw = self.latent_source(box.reconstruct(a_old), box.T_prev)
                Qm = box.project(Q_raw)
            elif self.grid_latent:
                Tf = self.reconstruct_volume(a_old)
                Qm = self.project_volume(self.latent_source(Tf, self.T_prev_full))
            a_new = aK + KK * Ct * S_raw
            if Qm is not None:
                a_new += KK * Qm
            if S_bot is not None:
                a_new += KK * Cb * S_bot
            if self.prop_corr:
                a_new += KK * self.correction_modes(a_new)
            res = a_new - a_old
            a_temp = res * self.omega
            a_temp += a_old
            rms_d = math.sqrt(float(np.vdot(res, res)) / n_el)
            rms_o = math.sqrt(float(np.vdot(a_old, a_old)) / n_el)
            rel = rms_d / max(rms_o, 1e-9)
            if self.track_picard_history:
                # contraction ratio to the previous iteration (solvers/spectral.py:470-481)
                prev = self.picard_history[-1]["rms_diff"] if self.picard_history else 0.0
                rho = rms_d / prev if it > 0 and prev > 0 else None
                self.picard_history.append({"iter": it, "rms_diff": rms_d, "rho": rho,
                                            "true_rel_err": rel})
            self.q_evap = q_ev
            if rel < self.tol:
                converged = True
                break
        if not converged and not self._cap_warned:
            self._cap_warned = True
            warnings.warn(f"Picard iteration hit max_picard_iter={self.max_iter} at t={t:.6g}",
                          RuntimeWarning, stacklevel=2)
        T_temp = self.surface_T(a_temp, top=True)
        if self.grid_latent:
            self.Q_modes_prev = Qm
        self.q_evap_old = self.q_evap.copy()
        self.a = a_temp.copy()
        self.a_temp = a_temp
        if self.prop_corr or self.grid_latent:
            self.T_prev_full = self.reconstruct_volume(self.a)
        self.box_flags = 0
        if box is not None:
            # history of the converged step (solvers/spectral.py:525-533)
            box.T_prev = box.reconstruct(a_temp)
            if box.Q_prev is None:
                box.Q_prev = np.zeros(box.shape)
            if Q_raw is not None:
                box.Q_prev = Q_raw.copy()
                self.box_flags = box.truncation(Q_raw)
        metrics = {"T_surface_max": float(np.max(T_temp)), "P_laser": P_laser,
                   "n_evap_iter": it + 1, "picard_converged": converged,
                   "picard_rel_err": rel}
        return self, metrics

    def set_state(self, T):
        if self.a is None:
            raise RuntimeError("Solver must be initialized before calling set_state().")
        self.a = dct2(np.asarray(T, dtype=np.float64), self.workers) * self.sqrt_dV

    def surface_temperature(self):
        return self.surface_T(self.a, top=True)

    def volume_temperature(self):
        return self.reconstruct_volume(self.a)


# ---- output reconstruction (physics/spectral_helpers.py:146-333) -----------------


def _coef(n, length):
    """C_0 = sqrt(1/L), C_m = sqrt(2/L) (physics/spectral_helpers.py:26-46)."""
    c = np.full(n, np.sqrt(2.0 / length))
    c[0] = np.sqrt(1.0 / length)
    return c


def nodal_temperature(a, lengths):
    """Node-centred field of modes ``a`` (nz, ny, nx) at x_j = j Lx / nx,
    j = 0..nx (likewise y, z), shape (nx+1, ny+1, nz+1)
    (``reconstruct_temperature_DCT``, physics/spectral_helpers.py:146-204)."""
    nz, ny, nx = a.shape
    Lx, Ly, Lz = lengths
    B = []
    for n, L in ((nx, Lx), (ny, Ly), (nz, Lz)):
        j = np.arange(n + 1)[:, None]
        m = np.arange(n)[None, :]
        B.append(_coef(n, L)[None, :] * np.cos(np.pi * ((m * j) % (2 * n)) / n))
    Bx, By, Bz = B
    return np.einsum("jm,kn,lp,pnm->jkl", Bx, By, Bz, a, optimize=True)


def nodal_temperature_dct1(a, lengths, workers=-1):
    """The node-centred field as the reference computes it on the host: the
    modes weighted by C (halved beyond index 0), zero-padded by one plane per
    axis, and an unnormalised 3-D DCT-I (physics/spectral_helpers.py:146-204).
    Same result as :func:`nodal_temperature`; used as the CPU baseline."""
    nz, ny, nx = a.shape
    Lx, Ly, Lz = lengths
    w = []
    for n, L in ((nz, Lz), (ny, Ly), (nx, Lx)):
        c = _coef(n, L)
        c[1:] *= 0.5
        w.append(c)
    padded = np.zeros((nz + 1, ny + 1, nx + 1))
    padded[:nz, :ny, :nx] = a * w[0][:, None, None] * w[1][None, :, None] * w[2][None, None, :]
    T = scipy.fft.dctn(padded, type=1, norm=None, workers=workers)
    return np.ascontiguousarray(T.transpose(2, 1, 0))


def points_temperature(a, lengths, coords):
    """Temperature at points ``coords`` (N, 3), clipped to the domain
    (``reconstruct_temperature_volume_at_points``, physics/spectral_helpers.py:206-248)."""
    coords = np.asarray(coords, dtype=np.float64)
    if coords.ndim != 2 or coords.shape[1] != 3:
        raise ValueError("coords must be of shape (N, 3)")
    nz, ny, nx = a.shape
    B = []
    for col, (n, L) in enumerate(((nx, lengths[0]), (ny, lengths[1]), (nz, lengths[2]))):
        x = np.clip(coords[:, col], 0.0, L)
        B.append(_coef(n, L)[:, None] * np.cos(np.pi * np.arange(n)[:, None] * x[None, :] / L))
    Bx, By, Bz = B
    return np.einsum("pnm,pi,ni,mi->i", a, Bz, By, Bx, optimize=True)


def temp_profiles(a, lengths, surface, laser_position=None, center="laser", num_points=1000):
    """Profiles along x, y and z through a centre on the top face
    (``save_temp_profiles``, physics/spectral_helpers.py:251-333); ``surface``
    is the top-face field used by ``center="hotspot"``."""
    Lx, Ly, Lz = lengths
    nz, ny, nx = a.shape
    if center == "hotspot":
        iy, ix = np.unravel_index(int(np.argmax(surface)), surface.shape)
        xc, yc = (ix + 0.5) * (Lx / nx), (iy + 0.5) * (Ly / ny)
    elif center == "laser":
        if laser_position is None:
            raise ValueError("Laser position required for center='laser'")
        xc, yc = float(laser_position[0]), float(laser_position[1])
    else:
        raise ValueError(f"Unknown center method: {center}")
    xc, yc = float(np.clip(xc, 0.0, Lx)), float(np.clip(yc, 0.0, Ly))
    out = {}
    for key, L_axis, fixed in (("x", Lx, (None, yc, Lz)), ("y", Ly, (xc, None, Lz)), ("z", Lz, (xc, yc, None))):
        c = np.linspace(0.0, L_axis, num_points)
        pts = np.stack([c if v is None else np.full(num_points, v) for v in fixed], axis=1)
        out[key] = (c, points_temperature(a, lengths, pts))
    return out
