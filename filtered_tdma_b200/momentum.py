"""Channel momentum ADI sweeps on one GPU (C ABI btdma_momentum_*), the implicit
viscous half-step of apps/channel_gpu/MomentumSolverGPU.cu (adi_z_, adi_y_,
adi_x_ with k_build_* / k_scatter_*).

    m = ChannelMomentum(256, 256, 256)            # x, y periodic; z stretched walls
    m.adi(comp, rhs, q, nu_dt_half)               # z, y, x sweeps of rhs into q
                                                  # (a Filtered backend: z, y in place on rhs)
"""
from __future__ import annotations

import ctypes
import math

from . import _lib as L
from .channel_grid import axis_metrics


class ChannelMomentum:
    def __init__(self, nx, ny, nz, H=2.0, aspect1=2 * math.pi, aspect2=math.pi, gamma3=1.5,
                 pbc_x=True, pbc_y=True):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.metrics = [axis_metrics(nx, H * aspect1, periodic=pbc_x),
                        axis_metrics(ny, H * aspect2, periodic=pbc_y),
                        axis_metrics(nz, H, gamma3, uniform=abs(gamma3) < 1e-14)]
        self.pbc = (bool(pbc_x), bool(pbc_y))
        (dx0, dm0), (dx1, dm1), (dx2, dm2) = self.metrics
        h = ctypes.c_void_p()
        L.check(L.lib().btdma_momentum_create(
            nx, ny, nz, dx0.ctypes.data, dm0.ctypes.data, dx1.ctypes.data, dm1.ctypes.data,
            dx2.ctypes.data, dm2.ctypes.data, int(pbc_x), int(pbc_y), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            L.lib().btdma_momentum_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2)

    def sweep(self, direction, comp, q, dst, c, stream=0):
        L.check(L.lib().btdma_momentum_sweep(self._h, int(direction), int(comp), q.data_ptr(),
                                             dst.data_ptr(), float(c), stream))
        return dst

    def adi(self, comp, rhs, q_out, c, stream=0):
        L.check(L.lib().btdma_momentum_adi(self._h, int(comp), rhs.data_ptr(), q_out.data_ptr(),
                                           float(c), stream))
        return q_out

    def set_backend(self, method="pascal", P=1, flags=0, eps_constant=1.0e-12):
        """Solver of the sweeps: "pascal" (default, tiled exact solve with
        generated coefficients), or a Filtered method ("filtered", "filtered_v2"
        or the integer method) with P segments: the reference channel's
        build / set_rho / solve / scatter sequence on explicit arrays."""
        if isinstance(method, str):
            t = method.lower()
            method = (L.PASCAL if t in ("pascal", "pascal_tdma") else
                      L.FILTERED_V1 if t in ("filtered_v1",) else L.FILTERED_V2)
        L.check(L.lib().btdma_momentum_set_backend(self._h, int(method), int(P), int(flags),
                                                   float(eps_constant)))

    def status(self, stream=0) -> int:
        st = ctypes.c_uint()
        L.check(L.lib().btdma_momentum_status(self._h, ctypes.byref(st), stream))
        return st.value
