"""Fused 3-D heat ADI step on one GPU (C ABI btdma_heat_*), the B200 form of the
reference's heat application step (apps/heat_gpu/solve_theta.cu,
SolveTheta::profile).

    h = HeatADI(n, n, n, rho=0.25)          # dt from rho as the reference's "order" option
    theta = h.field()                        # device array with ghosts, initial condition
    h.step(theta, h.steps)                   # CUDA-graph replay per step
    h.l2_error(theta, h.steps * h.dt)        # the reference's L2 against the exact solution
"""
from __future__ import annotations

import ctypes

from . import _lib as L


def dt_from_rho(rho: float, n_ref: int, option: str = "order") -> float:
    """dt = rho / (1 - 2 rho) * 2 dd^2 with dd = 2 / n_ref (apps/heat_cpu/global.cpp:82-96:
    dd = dx for "order", dz for "strong")."""
    dd = 2.0 / n_ref
    return rho / (1.0 - 2.0 * rho) * (2.0 * dd * dd)


def order_steps(rho: float, n: int) -> int:
    """Nt of the reference's "order" option: 128 steps of the 512 grid's dt."""
    q = (rho / (1.0 - 2.0 * rho) * 2.0 * (2.0 / 512.0) ** 2 * 128.0) / dt_from_rho(rho, n)
    return int(q + 0.5)


class HeatADI:
    def __init__(self, ix, iy, iz, dt=None, rho=None, option="order"):
        if dt is None:
            if rho is None:
                raise ValueError("give dt or rho")
            dt = dt_from_rho(rho, ix if option == "order" else iz)
        self.ix, self.iy, self.iz, self.dt = int(ix), int(iy), int(iz), float(dt)
        self.steps = order_steps(rho, ix) if (rho is not None and option == "order") else None
        h = ctypes.c_void_p()
        L.check(L.lib().btdma_heat_create(self.ix, self.iy, self.iz, self.dt, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            L.lib().btdma_heat_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return (self.iz + 2, self.iy + 2, self.ix + 2)

    def field(self, device="cuda"):
        """A new device field [iz + 2, iy + 2, ix + 2] holding the initial condition."""
        import torch
        th = torch.empty(self.shape, dtype=torch.float64, device=device)
        self.init(th)
        return th

    def init(self, theta, stream=0):
        L.check(L.lib().btdma_heat_init(self._h, theta.data_ptr(), stream))

    def step(self, theta, n_steps=1, graph=True, stream=0):
        L.check(L.lib().btdma_heat_step(self._h, theta.data_ptr(), int(n_steps), int(graph),
                                        stream))

    def step_profile(self, theta, stream=0):
        """One step timed phase by phase: the reference's 12 timing events (seconds)."""
        t = (ctypes.c_double * 12)()
        L.check(L.lib().btdma_heat_step_profile(self._h, theta.data_ptr(), t, stream))
        return list(t)

    def l2_error(self, theta, t_phys):
        out = ctypes.c_double()
        L.check(L.lib().btdma_heat_l2_error(self._h, theta.data_ptr(), float(t_phys),
                                            ctypes.byref(out)))
        return out.value
