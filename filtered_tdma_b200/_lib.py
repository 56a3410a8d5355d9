"""ctypes binding of the C ABI in include/btdma.h (libbtdma.so, built in-tree).

Importing this module loads the CUDA library; it raises if the library is
missing, because there is no other implementation of the solve.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libbtdma.so")

# enums of include/btdma.h
PASCAL, FILTERED_V1, FILTERED_V2 = 0, 1, 2
FP64, FP32_REFINE, FP32_STORE = 0, 1, 2
FLAG_J_HOST = 1
FLAG_REFERENCE_ORDER = 2
OK, ERR_ARG, ERR_SEGMENT, ERR_CUDA, ERR_SIZE, ERR_UNSUPPORTED, ERR_DEVICE = 0, -1, -2, -3, -4, -5, -6
STATUS_TIMEOUT, STATUS_NONFINITE = 1, 2
TILE_AUTO, TILE_NARROW, TILE_WIDE = 0, 1, 2

# every exported symbol of include/btdma.h
EXPORTS = (
    "btdma_create", "btdma_destroy", "btdma_solve", "btdma_solve_cyclic", "btdma_solve_out",
    "btdma_solve_host",
    "btdma_set_eps_constant", "btdma_set_rho", "btdma_set_rho_all", "btdma_last_J",
    "btdma_status", "btdma_set_method", "btdma_segments", "btdma_last_error",
    "btdma_solve_noalloc", "btdma_solve_f32", "btdma_set_refine", "btdma_last_stats",
    "btdma_solve_ragged", "btdma_solve_ragged_f32", "btdma_ragged_autotune",
    "btdma_ragged_plan_info", "btdma_heat_create", "btdma_heat_destroy", "btdma_heat_init",
    "btdma_heat_step", "btdma_heat_l2_error", "btdma_heat_step_profile", "btdma_poisson_create", "btdma_poisson_destroy",
    "btdma_poisson_solve", "btdma_poisson_status", "btdma_momentum_create",
    "btdma_momentum_destroy", "btdma_momentum_sweep", "btdma_momentum_adi", "btdma_momentum_status",
    "btdma_selftest_wait_timeout", "btdma_set_tile_shape", "btdma_ragged_set_plan",
    "btdma_momentum_set_backend",
)
NOALLOC_MAX_ELEMS = 1 << 20
REFINE_MAX_SWEEPS = 4


class Stats(ctypes.Structure):
    """btdma_stats of include/btdma.h."""
    _fields_ = [("n_systems", ctypes.c_int), ("sweeps", ctypes.c_int),
                ("converged_after", ctypes.c_int * (REFINE_MAX_SWEEPS + 1)),
                ("n_fallback", ctypes.c_int), ("filtered_exact", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {"n_systems": self.n_systems, "sweeps": self.sweeps,
                "converged_after": list(self.converged_after), "n_fallback": self.n_fallback,
                "filtered_exact": self.filtered_exact}


class RaggedBucket(ctypes.Structure):
    """btdma_ragged_bucket of include/btdma.h."""
    _fields_ = [("periodic", ctypes.c_int), ("n_systems", ctypes.c_int),
                ("n_row_min", ctypes.c_int), ("n_row_max", ctypes.c_int),
                ("lanes_per_system", ctypes.c_int), ("warps_per_cta", ctypes.c_int),
                ("cta_per_system", ctypes.c_int), ("tuned_ms", ctypes.c_float),
                ("persistent", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class BtdmaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"btdma error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded CUDA library (raises FileNotFoundError when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m filtered_tdma_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.btdma_create.argtypes = [i, i, i, i, i, i, ctypes.POINTER(vp)]
        L.btdma_destroy.argtypes = [vp]
        L.btdma_solve.argtypes = [vp, vp, vp, vp, vp, i, i, vp]
        L.btdma_solve_cyclic.argtypes = [vp, vp, vp, vp, vp, i, i, vp]
        L.btdma_solve_out.argtypes = [vp, vp, vp, vp, vp, vp, i, i, i, vp]
        L.btdma_solve_host.argtypes = [vp, vp, vp, vp, vp, vp, i, i, i, vp]
        L.btdma_set_eps_constant.argtypes = [vp, d]
        L.btdma_set_rho.argtypes = [vp, vp, vp, vp, i, i, vp]
        L.btdma_set_rho_all.argtypes = [vp, vp, vp, vp, i, i, vp]
        L.btdma_last_J.argtypes = [vp, ctypes.POINTER(i), i, ctypes.POINTER(i)]
        L.btdma_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint)]
        L.btdma_set_method.argtypes = [vp, i]
        L.btdma_segments.argtypes = [vp, ctypes.POINTER(i)]
        L.btdma_set_tile_shape.argtypes = [vp, i]
        L.btdma_ragged_set_plan.argtypes = [vp, ctypes.POINTER(RaggedBucket), i]
        L.btdma_solve_noalloc.argtypes = [vp, vp, vp, vp, i, i, vp]
        L.btdma_solve_f32.argtypes = [vp, vp, vp, vp, vp, vp, i, i, i, vp]
        L.btdma_set_refine.argtypes = [vp, i, d]
        L.btdma_last_stats.argtypes = [vp, ctypes.POINTER(Stats)]
        L.btdma_solve_ragged.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i, vp]
        L.btdma_solve_ragged_f32.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i, vp]
        L.btdma_ragged_autotune.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i, vp]
        L.btdma_ragged_plan_info.argtypes = [vp, ctypes.POINTER(RaggedBucket), i,
                                             ctypes.POINTER(i)]
        L.btdma_heat_create.argtypes = [i, i, i, d, ctypes.POINTER(vp)]
        L.btdma_heat_destroy.argtypes = [vp]
        L.btdma_heat_init.argtypes = [vp, vp, vp]
        L.btdma_heat_step.argtypes = [vp, vp, i, i, vp]
        L.btdma_heat_l2_error.argtypes = [vp, vp, d, ctypes.POINTER(d)]
        L.btdma_heat_step_profile.argtypes = [vp, vp, ctypes.POINTER(d), vp]
        L.btdma_poisson_create.argtypes = [i, vp, vp, i, vp, i, ctypes.POINTER(vp)]
        L.btdma_poisson_destroy.argtypes = [vp]
        L.btdma_poisson_solve.argtypes = [vp, vp, vp]
        L.btdma_poisson_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint), vp]
        L.btdma_momentum_create.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp, i, i,
                                            ctypes.POINTER(vp)]
        L.btdma_momentum_destroy.argtypes = [vp]
        L.btdma_momentum_sweep.argtypes = [vp, i, i, vp, vp, d, vp]
        L.btdma_momentum_adi.argtypes = [vp, i, vp, vp, d, vp]
        L.btdma_momentum_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint), vp]
        L.btdma_momentum_set_backend.argtypes = [vp, i, i, i, d]
        L.btdma_selftest_wait_timeout.argtypes = [i, ctypes.POINTER(ctypes.c_uint), vp]
        L.btdma_last_error.restype = ctypes.c_char_p
        for name in EXPORTS:
            if name != "btdma_last_error":
                getattr(L, name).restype = i
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != OK:
        msg = lib().btdma_last_error()
        raise BtdmaError(rc, msg.decode() if msg else "")
