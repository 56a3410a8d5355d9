"""CPU oracle for the batched tridiagonal solve — TEST INFRASTRUCTURE ONLY.

numpy/ctypes front end to two shared libraries built by ``oracle/Makefile``:

* ``_build/liboracle.so``: the C restatement in ``tdma_oracle.c`` (serial
  Thomas, periodic Thomas, PaScaL with P segments, Filtered v1/v2 with P
  segments, J estimators), each function citing the reference file:line it
  restates.
* ``_ref/libref.so``: the reference's own CPU library compiled from its
  unmodified sources with a thread-rank MPI stand-in; present only where it was
  built.  It pins the restatement (``tests/test_oracle.py``) and is the CPU
  baseline of ``bench.py --impl reference``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use this module, and only as the checker.  Arrays are ``[n_row, n_sys]``
C-contiguous float64 (row j of system i at ``j*n_sys + i``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "_build", "liboracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libref.so")

J_DEVICE = 0  # J estimator of the reference's CUDA library
J_HOST = 1    # J estimator of the reference's CPU library

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def reference_dir() -> str | None:
    """Root of the reference sources, from the environment variable
    BTDMA_REFERENCE_DIR (no default: the build recipe sets it where the sources
    exist)."""
    d = os.environ.get("BTDMA_REFERENCE_DIR")
    return d if d and os.path.isdir(os.path.join(d, "libs")) else None


def build(with_ref: bool | None = None) -> None:
    """Compile the restatement (and the reference build when its sources exist)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    ref_dir = reference_dir()
    if with_ref is None:
        with_ref = ref_dir is not None
    if with_ref:
        if ref_dir is None:
            raise RuntimeError("BTDMA_REFERENCE_DIR does not name the reference sources")
        subprocess.run(["make", "-s", "-C", _HERE, "ref", "ref_gpu", "ref_channel",
                        f"REF={ref_dir}"], check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_ORACLE_SO):
            build(with_ref=False)
        L = ctypes.CDLL(_ORACLE_SO)
        for name in ("orc_thomas", "orc_thomas_cyclic"):
            getattr(L, name).argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
            getattr(L, name).restype = None
        L.orc_pascal.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int]
        L.orc_pascal.restype = ctypes.c_int
        L.orc_filtered.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int,
                                   _ip]
        L.orc_filtered.restype = ctypes.c_int
        L.orc_rho_rows.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_rho_rows_all.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_split.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip]
        L.orc_rhs_bound_factor.argtypes = [ctypes.c_double]
        L.orc_rhs_bound_factor.restype = ctypes.c_double
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def ref():
    """The reference's own CPU library (raises if it was not built here)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(_REF_SO + " not built (make -C oracle ref)")
        L = ctypes.CDLL(_REF_SO)
        for name in ("ref_tdma_many", "ref_ftdma_many", "ref_tdma_cyclic_many",
                     "ref_ftdma_cyclic_many"):
            getattr(L, name).argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
            getattr(L, name).restype = None
        L.ref_pascal.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int]
        L.ref_filtered.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp]
        L.ref_time_solve.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]
        L.ref_para_range.argtypes = [ctypes.c_int] * 4 + [_ip, _ip]
        _ref = L
    return _ref


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _copies(*arrs):
    return [np.ascontiguousarray(a, dtype=np.float64).copy() for a in arrs]


def split(n: int, nparts: int):
    """Segment (first_row, count) list of the reference's block split."""
    out = []
    for p in range(nparts):
        f, c = ctypes.c_int(), ctypes.c_int()
        lib().orc_split(n, nparts, p, ctypes.byref(f), ctypes.byref(c))
        out.append((f.value, c.value))
    return out


# ---------------------------------------------------------------- restatement
def thomas(A, B, C, D):
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    lib().orc_thomas(_p(A), _p(B), _p(C), _p(D), n_sys, n_row)
    return D


def thomas_cyclic(A, B, C, D):
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    lib().orc_thomas_cyclic(_p(A), _p(B), _p(C), _p(D), n_sys, n_row)
    return D


def pascal(A, B, C, D, P, cyclic=False):
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    rc = lib().orc_pascal(_p(A), _p(B), _p(C), _p(D), n_sys, n_row, P, int(cyclic))
    if rc != 0:
        raise ValueError("every segment needs at least 3 rows")
    return D


def filtered(A, B, C, D, P, version=2, cyclic=False, eps_constant=1e-3, rho_row=None,
             jmode=J_DEVICE):
    """Returns (x, J per segment)."""
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    if rho_row is None:
        rho_row = rho_rows(A, B, C, sys=0)
    rho_row = np.ascontiguousarray(rho_row, dtype=np.float64)
    J = np.zeros(P, dtype=np.int32)
    rc = lib().orc_filtered(_p(A), _p(B), _p(C), _p(D), n_sys, n_row, P, version, int(cyclic),
                            float(eps_constant), _p(rho_row), jmode,
                            J.ctypes.data_as(_ip))
    if rc != 0:
        raise ValueError("every segment needs at least 3 rows")
    return D, J


def rho_rows(A, B, C, sys=0):
    A, B, C = _copies(A, B, C)
    n_row, n_sys = A.shape
    out = np.zeros(n_row)
    lib().orc_rho_rows(_p(A), _p(B), _p(C), n_sys, n_row, sys, _p(out))
    return out


def rho_rows_all(A, B, C):
    A, B, C = _copies(A, B, C)
    n_row, n_sys = A.shape
    out = np.zeros(n_row)
    lib().orc_rho_rows_all(_p(A), _p(B), _p(C), n_sys, n_row, _p(out))
    return out


# ------------------------------------------------------- the reference itself
def ref_thomas(A, B, C, D, filtered_copy=False):
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    f = ref().ref_ftdma_many if filtered_copy else ref().ref_tdma_many
    f(_p(A), _p(B), _p(C), _p(D), n_sys, n_row)
    return D


def ref_thomas_cyclic(A, B, C, D, filtered_copy=False):
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    f = ref().ref_ftdma_cyclic_many if filtered_copy else ref().ref_tdma_cyclic_many
    f(_p(A), _p(B), _p(C), _p(D), n_sys, n_row)
    return D


def ref_pascal(A, B, C, D, nprocs, cyclic=False):
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    ref().ref_pascal(_p(A), _p(B), _p(C), _p(D), n_sys, n_row, nprocs, int(cyclic))
    return D


def ref_filtered(A, B, C, D, nprocs, version=2, cyclic=False, eps_constant=1e-3, rho_row=None):
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    rr = None
    if rho_row is not None:
        rr = np.ascontiguousarray(rho_row, dtype=np.float64)
    ref().ref_filtered(_p(A), _p(B), _p(C), _p(D), n_sys, n_row, nprocs, version, int(cyclic),
                       float(eps_constant), _p(rr) if rr is not None else None)
    return D


def ref_time_solve(A, B, C, D, nprocs, method="pascal", eps_constant=1e-3, reps=3):
    """Seconds per solve (max over thread ranks) of the reference CPU library."""
    A, B, C, D = _copies(A, B, C, D)
    n_row, n_sys = D.shape
    out = np.zeros(reps)
    ref().ref_time_solve(_p(A), _p(B), _p(C), _p(D), n_sys, n_row, nprocs,
                         0 if method == "pascal" else 2, float(eps_constant), reps, _p(out))
    return out
