"""Wall-normal solve of the channel flow's FFT Poisson equation (C ABI
btdma_poisson_*), with the reference's stretched grid and modified wavenumbers.

    p = ChannelPoisson(n1m=128, n2m=128, n3m=192, gamma=2.0)
    p.solve(hat)     # hat: complex128 device tensor [n3m, n2m, n1m // 2 + 1], in place

Grid (apps/channel_gpu/Grid.cpp:16-96): faces xf_i = L/2 (1 - tanh(gamma (1 - 2 i/n))
/ tanh(gamma)), centres between faces, mirror ghosts at the walls; dz = face
spacing, dmz = centre spacing.  Wavenumbers (PressureSolverGPU.cu:362-368):
kx2_i = 2 (1 - cos(2 pi i / n1m)) / dx^2, ky2_j likewise with j folded to
[-n2m/2, n2m/2]; mode m = j * (n1m/2 + 1) + i has lambda_m = kx2_i + ky2_j.
"""
from __future__ import annotations

import ctypes
import math

from . import _lib as L
from .channel_grid import axis_metrics, mode_lambdas  # noqa: F401  (re-exported)


def wall_normal_grid(n: int, gamma: float, length: float):
    """(dz, dmz), nz + 2 entries each, ghosts included (non-periodic axis)."""
    return axis_metrics(n, length, gamma, uniform=abs(gamma) < 1e-14, periodic=False)


class ChannelPoisson:
    """Wall-normal Poisson solves of an n1m x n2m x n3m channel (H = 2, x and y
    periodic with lengths H * aspect1 and H * aspect2, z stretched by gamma)."""

    def __init__(self, n1m=128, n2m=128, n3m=192, gamma=2.0, H=2.0,
                 aspect1=2 * math.pi, aspect2=math.pi, pin_mode0=True):
        self.n1m, self.n2m, self.n3m = n1m, n2m, n3m
        self.nxh = n1m // 2 + 1
        self.dz, self.dmz = wall_normal_grid(n3m, gamma, H)
        self.lam = mode_lambdas(n1m, n2m, H * aspect1, H * aspect2)
        self.n_modes = self.lam.size
        h = ctypes.c_void_p()
        L.check(L.lib().btdma_poisson_create(
            n3m, self.dz.ctypes.data, self.dmz.ctypes.data, self.n_modes, self.lam.ctypes.data,
            int(pin_mode0), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            L.lib().btdma_poisson_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, hat, stream=0):
        """hat: complex128 device tensor [n3m, n2m, nxh] (or [n3m, n_modes]), in place."""
        import torch
        if hat.dtype != torch.complex128 or not hat.is_contiguous():
            raise TypeError("expected a contiguous complex128 tensor")
        if hat.numel() != self.n3m * self.n_modes:
            raise ValueError("hat must hold n3m x n_modes values")
        L.check(L.lib().btdma_poisson_solve(self._h, hat.data_ptr(), stream))
        return hat

    def status(self, stream=0) -> int:
        st = ctypes.c_uint()
        L.check(L.lib().btdma_poisson_status(self._h, ctypes.byref(st), stream))
        return st.value
