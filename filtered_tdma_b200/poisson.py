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

import numpy as np

from . import _lib as L


def wall_normal_grid(n: int, gamma: float, length: float):
    """(dz, dmz), nz + 2 entries each, ghosts included (Grid::build_axis, one rank,
    non-periodic axis)."""
    if abs(gamma) < 1e-14:
        xf = [length * i / n for i in range(n + 1)]
    else:
        th = math.tanh(gamma)
        xf = [0.5 * length * (1.0 - math.tanh(gamma * (1.0 - 2.0 * (i / n))) / th)
              for i in range(n + 1)]
    xc = [0.0] * (n + 2)
    for i in range(1, n + 1):
        xc[i] = 0.5 * (xf[i - 1] + xf[i])
    xc[0] = xf[0] - (xc[1] - xf[0])
    xc[n + 1] = xf[n] + (xf[n] - xc[n])
    dz = [0.0] * (n + 2)
    for i in range(1, n + 1):
        dz[i] = xf[i] - xf[i - 1]
    dz[0], dz[n + 1] = dz[1], dz[n]
    dmz = [0.0] * (n + 2)
    for i in range(1, n + 2):
        dmz[i] = xc[i] - xc[i - 1]
    dmz[0] = dmz[1]
    return np.array(dz), np.array(dmz)


def mode_lambdas(n1m: int, n2m: int, lx: float, ly: float) -> np.ndarray:
    """lambda per mode m = j * (n1m // 2 + 1) + i."""
    nxh = n1m // 2 + 1
    dx, dy = lx / n1m, ly / n2m
    kx2 = np.array([2.0 * (1.0 - math.cos(2.0 * math.pi * i / n1m)) / (dx * dx)
                    for i in range(nxh)])
    ky2 = np.array([2.0 * (1.0 - math.cos(2.0 * math.pi * (j if j <= n2m // 2 else j - n2m)
                                          / n2m)) / (dy * dy) for j in range(n2m)])
    return (ky2[:, None] + kx2[None, :]).reshape(-1)


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
