"""The reference's channel-flow coefficient-build kernels on one GPU — TEST
INFRASTRUCTURE ONLY.

ctypes front end to ``_ref/libref_channel.so`` (``make -C oracle ref_channel``:
the reference's apps/channel_gpu/MomentumSolverGPU.cu and PressureSolverGPU.cu
compiled unmodified, driven by ``ref_channel_driver.cu``).  It runs the
reference's k_build_{x,y,z} / k_scatter_{x,y,z} (MomentumSolverGPU.cu:135-220)
and k_build_poisson_tdma / k_zero_mode / k_write_poisson_solution
(PressureSolverGPU.cu:183-234) so that tests/ can check
oracle/momentum_oracle.py and oracle/poisson_oracle.py against what the
reference computes.  The library's solver classes are never constructed; it is
loaded lazily because their other symbols (MPI transposes, cuFFT, the TDMA
objects) stay unbound.  Arguments are torch CUDA tensors.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_ref", "libref_channel.so")
_lib = None


def available() -> bool:
    return os.path.exists(_SO)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(_SO, mode=os.RTLD_LAZY | os.RTLD_LOCAL)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.refch_build.argtypes = [i, i, vp, vp, vp, vp, vp, vp, vp, i, i, i, d, i, i]
        L.refch_scatter.argtypes = [i, vp, vp, i, i, i]
        L.refch_poisson_build.argtypes = [vp] * 13 + [i, i, i, i, i]
        L.refch_poisson_write.argtypes = [vp, vp, vp, i, i, i, i]
        for f in (L.refch_build, L.refch_scatter, L.refch_poisson_build, L.refch_poisson_write):
            f.restype = i
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: reference channel driver returned CUDA error {rc}")


def momentum_build(direction, comp, q, A, B, C, D, d, dm, nx, ny, nz, c, low=1, high=1):
    """k_build_{x,y,z} of one sweep: q the ghosted field, A..D flat n_row x
    n_sys arrays in the reference's sweep layout, (d, dm) the axis metrics."""
    _check(lib().refch_build(direction, comp, q.data_ptr(), A.data_ptr(), B.data_ptr(),
                             C.data_ptr(), D.data_ptr(), d.data_ptr(), dm.data_ptr(), nx, ny, nz,
                             float(c), low, high), "k_build")


def momentum_scatter(direction, D, q, nx, ny, nz):
    _check(lib().refch_scatter(direction, D.data_ptr(), q.data_ptr(), nx, ny, nz), "k_scatter")


def poisson_build(hat, Am, Ac, Ap, Am2, Ac2, Ap2, Br, Bi, dzg, dmzg, kx2, ky2, n3, nsys, hme,
                  n2m, pin=True):
    """k_build_poisson_tdma (+ k_zero_mode) on one rank; hat complex128 [n3, nsys]."""
    _check(lib().refch_poisson_build(hat.data_ptr(), Am.data_ptr(), Ac.data_ptr(), Ap.data_ptr(),
                                     Am2.data_ptr(), Ac2.data_ptr(), Ap2.data_ptr(),
                                     Br.data_ptr(), Bi.data_ptr(), dzg.data_ptr(),
                                     dmzg.data_ptr(), kx2.data_ptr(), ky2.data_ptr(), n3, nsys,
                                     hme, n2m, 1 if pin else 0), "k_build_poisson_tdma")


def poisson_write(hat, Br, Bi, n3, nsys, hme, n2m):
    _check(lib().refch_poisson_write(hat.data_ptr(), Br.data_ptr(), Bi.data_ptr(), n3, nsys, hme,
                                     n2m), "k_write_poisson_solution")
