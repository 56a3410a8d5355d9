"""The reference's own GPU kernels on one GPU — TEST INFRASTRUCTURE ONLY.

ctypes front end to ``_ref/libref_gpu.so`` (built by ``make -C oracle ref_gpu``
from the reference's unmodified libs/pascal_tdma/gpu/tdma_local_cuda.cu and
libs/filtered_tdma/gpu/filtered_tdma_kernels.cuh, driven by
``ref_gpu_driver.cu``: P ranks' slabs on one GPU, the MPI transport replaced by
pointers).  Used by tests/test_reference_gpu.py and by bench.py's
reference-GPU baseline leg, only as a baseline and a checker; the library
never calls it.  Every solve is in place on torch CUDA tensors [n_row, n_sys]
float64 and overwrites A and C as the reference does.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_ref", "libref_gpu.so")
_lib = None


def available() -> bool:
    return os.path.exists(_SO)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(_SO)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.refgpu_tdma_many.argtypes = [vp, vp, vp, vp, i, i, vp]
        L.refgpu_pascal.argtypes = [vp, vp, vp, vp, i, i, i, vp]
        L.refgpu_filtered_set_rho.argtypes = [vp, vp, vp, i, i, i, vp]
        L.refgpu_filtered_v2.argtypes = [vp, vp, vp, vp, i, i, i, d,
                                         ctypes.POINTER(ctypes.c_int), vp]
        L.refgpu_launches.argtypes = [i, i]
        for f in (L.refgpu_tdma_many, L.refgpu_pascal, L.refgpu_filtered_set_rho,
                  L.refgpu_filtered_v2, L.refgpu_launches):
            f.restype = i
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: reference GPU driver returned {rc}")


def _stream(stream):
    return ctypes.c_void_p(stream or 0)


def tdma_many(A, B, C, D, stream=0):
    n_row, n_sys = D.shape
    _check(lib().refgpu_tdma_many(A.data_ptr(), B.data_ptr(), C.data_ptr(), D.data_ptr(),
                                  n_sys, n_row, _stream(stream)), "tdma_many")


def pascal(A, B, C, D, P, stream=0):
    n_row, n_sys = D.shape
    _check(lib().refgpu_pascal(A.data_ptr(), B.data_ptr(), C.data_ptr(), D.data_ptr(), n_sys,
                               n_row, P, _stream(stream)), "pascal")


def filtered_set_rho(A, B, C, P, stream=0):
    n_row, n_sys = A.shape
    _check(lib().refgpu_filtered_set_rho(A.data_ptr(), B.data_ptr(), C.data_ptr(), n_sys,
                                         n_row, P, _stream(stream)), "filtered set_rho")


def filtered_v2(A, B, C, D, P, eps_constant, stream=0, want_J=False):
    n_row, n_sys = D.shape
    J = (ctypes.c_int * P)()
    _check(lib().refgpu_filtered_v2(A.data_ptr(), B.data_ptr(), C.data_ptr(), D.data_ptr(),
                                    n_sys, n_row, P, float(eps_constant),
                                    J if want_J else None, _stream(stream)), "filtered_v2")
    return list(J) if want_J else None


def launches(method: str, P: int) -> int:
    return lib().refgpu_launches({"tdma_many": 0, "pascal": 1, "filtered_v2": 2}[method], P)
