"""ctypes binding of ``libsgh_b200.so`` (declared in ``include/sgh_b200.h``).

The library is built in-tree by ``spectral_galerkin_heat_b200.build`` and is
loaded from this package directory only. There is no fallback: if the library
is missing or fails to load, :func:`lib` raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

__all__ = ["lib", "LIB_PATH", "SghProgram", "SghConfig", "SghLaser", "SghStepOut", "check",
           "EXPORTED", "SghError", "BUF", "STEP_STATUS", "SghBatchSlotInfo", "PRECISION",
           "SghBoxGeom", "STEP_FLAGS", "ABI_VERSION"]

ABI_VERSION = 3

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsgh_b200.so")

MAX_PROGRAM = 64
MAX_CONSTS = 32
PICARD_HISTORY_MAX = 4096  # SGH_PICARD_HISTORY_MAX

ERRORS = {-1: "SGH_ERR_INVALID", -2: "SGH_ERR_CUDA", -3: "SGH_ERR_STATE",
          -4: "SGH_ERR_UNSUPPORTED", -5: "SGH_ERR_WORKSPACE"}
STEP_STATUS = {0: "converged", 1: "capped", 2: "nonfinite", 3: "tensor_core_timeout"}
PRECISION = {"fp64": 0, "mixed": 1}          # batches and plans
PLAN_PRECISION = {"fp64": 0, "mixed": 1, "fp32": 2}   # single-instance plans
BUF = {"modes": 0, "K": 1, "KK": 2, "T_prev": 3, "q_evap_old": 4, "Q_modes": 5,
       "surface": 6, "scratch": 7, "box_T_prev": 8, "box_Q_prev": 9, "box_Bx": 10,
       "box_By": 11, "box_Bz": 12}
# sgh_step_out.flags: faces of the fine box reached by the latent source
STEP_FLAGS = {1: "floor (depth)", 2: "x window edge", 4: "y window edge"}

# Every function declared in include/sgh_b200.h (checked by the tests).
EXPORTED = (
    "sgh_abi_version", "sgh_last_error", "sgh_plan_create", "sgh_plan_destroy",
    "sgh_plan_workspace_bytes", "sgh_plan_bind", "sgh_plan_buffer", "sgh_plan_launch_counts", "sgh_state_reset",
    "sgh_step", "sgh_step_eager", "sgh_run", "sgh_dct3d", "sgh_surface_temperature", "sgh_project_volume",
    "sgh_reconstruct_volume", "sgh_dctn_workspace_bytes", "sgh_dctn", "sgh_dctn_noalloc",
    "sgh_nodal_workspace_bytes", "sgh_nodal_temperature", "sgh_points_workspace_bytes",
    "sgh_points_temperature", "sgh_box_geometry", "sgh_box_window", "sgh_box_temperature",
    "sgh_box_project", "sgh_state_flags", "sgh_state_set_flags", "sgh_line_workspace_bytes",
    "sgh_line_temperature", "sgh_picard_history",
    "sgh_batch_create", "sgh_batch_destroy", "sgh_batch_workspace_bytes", "sgh_batch_bind",
    "sgh_batch_slot_start", "sgh_batch_slot_stop", "sgh_batch_slot_resume", "sgh_batch_step", "sgh_batch_step_eager",
    "sgh_batch_status",
    "sgh_batch_buffer", "sgh_batch_launch_counts", "sgh_batch_volume_pass", "sgh_batch_error",
    "sgh_batch_set_wait_limit", "sgh_batch_set_policy", "sgh_dct2_bf16x3_workspace_bytes",
    "sgh_dct2_bf16x3",
)


class SghProgram(C.Structure):
    _fields_ = [("n_ops", C.c_int32), ("n_consts", C.c_int32),
                ("ops", C.c_int32 * MAX_PROGRAM), ("consts", C.c_double * MAX_CONSTS)]


class SghConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("precision", C.c_int32),
        ("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double), ("dt", C.c_double),
        ("k", C.c_double), ("rho", C.c_double), ("cp", C.c_double),
        ("L_f", C.c_double), ("T_solidus", C.c_double), ("T_liquidus", C.c_double),
        ("Pa", C.c_double), ("R_v", C.c_double), ("T_boil", C.c_double), ("dH_LV", C.c_double),
        ("T0", C.c_double), ("h_top", C.c_double), ("h_bottom", C.c_double),
        ("has_model", C.c_int32), ("model_constant", C.c_int32), ("k_constant", C.c_int32),
        ("pad0", C.c_int32),
        ("k_solid", SghProgram), ("k_liquid", SghProgram), ("rho_solid", SghProgram),
        ("rho_liquid", SghProgram), ("c_solid", SghProgram), ("c_liquid", SghProgram),
        ("r_x", C.c_double), ("r_y", C.c_double), ("absorptivity", C.c_double),
        ("order", C.c_double), ("area_factor", C.c_double),
        ("cell_integrated", C.c_int32), ("max_iter", C.c_int32),
        ("omega", C.c_double), ("tol", C.c_double),
        ("axis_min_ctas", C.c_int32), ("axis_cuda_cores", C.c_int32),
        ("box", C.c_int32), ("box_refinement", C.c_int32), ("box_size", C.c_double * 3),
    ]


class SghLaser(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("power", C.c_double),
                ("vx", C.c_double), ("vy", C.c_double), ("is_on", C.c_int32), ("flags", C.c_int32)]


class SghBatchPolicy(C.Structure):
    _fields_ = [("vol_unroll", C.c_int32), ("vol_vec", C.c_int32), ("reserved", C.c_int32 * 6)]


class SghStepOut(C.Structure):
    _fields_ = [("T_surface_max", C.c_double), ("P_laser", C.c_double),
                ("picard_rel_err", C.c_double), ("n_iter", C.c_int32),
                ("converged", C.c_int32), ("status", C.c_int32), ("flags", C.c_int32)]


class SghBoxGeom(C.Structure):
    _fields_ = [("n_box", C.c_int32 * 3), ("n_fine_total", C.c_int32 * 3),
                ("d_fine", C.c_double * 3), ("dV_fine", C.c_double), ("z0", C.c_double)]


class SghBatchSlotInfo(C.Structure):
    _fields_ = [("active", C.c_int32), ("step", C.c_int32), ("n_steps", C.c_int32),
                ("iters", C.c_int32), ("last", SghStepOut)]


class SghError(RuntimeError):
    """A libsgh_b200 call returned a negative status."""

    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed with {ERRORS.get(code, code)}: {msg}")
        self.code = code


_lock = threading.Lock()
_lib = None


def lib() -> C.CDLL:
    """Load (once) and return the library; raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libsgh_b200.so not found at {LIB_PATH}; build it with "
                "`python -m spectral_galerkin_heat_b200.build` (the B200 backend has no "
                "CPU fallback).")
        L = C.CDLL(LIB_PATH)
        vp, u64p, i32 = C.c_void_p, C.POINTER(C.c_uint64), C.c_int32
        sig = {
            "sgh_abi_version": ([], C.c_int),
            "sgh_last_error": ([], C.c_char_p),
            "sgh_plan_create": ([C.POINTER(SghConfig), C.POINTER(vp)], C.c_int),
            "sgh_plan_destroy": ([vp], C.c_int),
            "sgh_plan_workspace_bytes": ([vp, u64p], C.c_int),
            "sgh_plan_bind": ([vp, vp, C.c_uint64, vp], C.c_int),
            "sgh_plan_buffer": ([vp, i32, C.POINTER(vp), u64p], C.c_int),
            "sgh_plan_launch_counts": ([vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)], C.c_int),
            "sgh_state_reset": ([vp, vp], C.c_int),
            "sgh_step": ([vp, C.POINTER(SghLaser), C.POINTER(SghStepOut), vp], C.c_int),
            "sgh_step_eager": ([vp, C.POINTER(SghLaser), C.POINTER(SghStepOut), vp], C.c_int),
            "sgh_run": ([vp, vp, i32, vp, vp], C.c_int),
            "sgh_dct3d": ([vp, i32, vp, vp, vp], C.c_int),
            "sgh_surface_temperature": ([vp, vp, i32, vp, vp], C.c_int),
            "sgh_project_volume": ([vp, vp, vp, vp], C.c_int),
            "sgh_reconstruct_volume": ([vp, vp, vp, vp], C.c_int),
            "sgh_dctn_workspace_bytes": ([i32, C.POINTER(i32), u64p], C.c_int),
            "sgh_dctn": ([i32, i32, C.POINTER(i32), vp, vp, vp, C.c_uint64, vp], C.c_int),
            "sgh_dctn_noalloc": ([i32, i32, C.POINTER(i32), vp, vp, vp], C.c_int),
            "sgh_nodal_workspace_bytes": ([i32, i32, i32, u64p], C.c_int),
            "sgh_nodal_temperature": ([i32, i32, i32, C.c_double, C.c_double, C.c_double, vp, vp, vp,
                                       C.c_uint64, vp], C.c_int),
            "sgh_points_workspace_bytes": ([i32, i32, i32, i32, u64p], C.c_int),
            "sgh_points_temperature": ([i32, i32, i32, C.c_double, C.c_double, C.c_double, vp, i32, vp, vp,
                                        vp, C.c_uint64, vp], C.c_int),
            "sgh_dct2_bf16x3_workspace_bytes": ([i32, i32, u64p], C.c_int),
            "sgh_dct2_bf16x3": ([i32, i32, i32, vp, vp, vp, C.c_uint64, vp], C.c_int),
            "sgh_batch_create": ([C.POINTER(SghConfig), i32, i32, C.POINTER(vp)], C.c_int),
            "sgh_batch_destroy": ([vp], C.c_int),
            "sgh_batch_workspace_bytes": ([vp, u64p], C.c_int),
            "sgh_batch_bind": ([vp, vp, C.c_uint64, vp], C.c_int),
            "sgh_batch_slot_start": ([vp, i32, vp, i32, vp, vp], C.c_int),
            "sgh_batch_slot_stop": ([vp, i32, vp], C.c_int),
            "sgh_batch_slot_resume": ([vp, i32, vp, i32, i32, vp, vp], C.c_int),
            "sgh_batch_step": ([vp, i32, vp], C.c_int),
            "sgh_batch_step_eager": ([vp, vp], C.c_int),
            "sgh_batch_status": ([vp, C.POINTER(SghBatchSlotInfo), vp], C.c_int),
            "sgh_batch_buffer": ([vp, i32, i32, C.POINTER(vp), u64p], C.c_int),
            "sgh_batch_error": ([vp, C.POINTER(i32), vp], C.c_int),
            "sgh_batch_set_wait_limit": ([vp, C.c_uint32, i32, vp], C.c_int),
            "sgh_batch_set_policy": ([vp, C.POINTER(SghBatchPolicy)], C.c_int),
            "sgh_batch_launch_counts": ([vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)], C.c_int),
            "sgh_batch_volume_pass": ([vp, vp], C.c_int),
            "sgh_box_geometry": ([vp, C.POINTER(SghBoxGeom)], C.c_int),
            "sgh_box_window": ([vp, C.POINTER(i32), vp], C.c_int),
            "sgh_box_temperature": ([vp, vp, vp, vp], C.c_int),
            "sgh_box_project": ([vp, vp, vp, vp], C.c_int),
            "sgh_state_flags": ([vp, C.POINTER(i32), vp], C.c_int),
            "sgh_line_workspace_bytes": ([i32, i32, i32, u64p], C.c_int),
            "sgh_line_temperature": ([i32, i32, i32, C.c_double, C.c_double, C.c_double, vp, i32,
                                      C.c_double, C.c_double, C.c_double, i32, vp, vp, vp, C.c_uint64, vp],
                                     C.c_int),
            "sgh_state_set_flags": ([vp, i32, vp], C.c_int),
            "sgh_picard_history": ([vp, C.POINTER(C.c_double), i32, C.POINTER(i32), vp], C.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        if L.sgh_abi_version() != ABI_VERSION:
            raise RuntimeError("libsgh_b200.so ABI version mismatch; rebuild it")
        _lib = L
        return L


def check(fn_name: str, code: int) -> None:
    """Raise :class:`SghError` for a negative status."""
    if code != 0:
        msg = lib().sgh_last_error()
        raise SghError(fn_name, code, msg.decode() if msg else "")
