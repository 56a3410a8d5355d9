"""Grid metrics of the reference's channel flow (apps/channel_gpu/Grid.cpp:16-96,
one rank holding the whole axis).

For an axis of n cells: face positions xf_0..xf_n (uniform, or tanh-stretched
xf_i = L/2 (1 - tanh(gamma (1 - 2 i/n)) / tanh(gamma))), cell centres between
faces, ghost centres mirrored through the walls (or wrapped when periodic);
dx_i = xf_i - xf_{i-1} (cell size) and dmx_i = xc_i - xc_{i-1} (centre
spacing), n + 2 entries each with the ghosts.
"""
from __future__ import annotations

import math

import numpy as np


def face_positions(n: int, gamma: float, length: float, uniform: bool):
    if uniform or abs(gamma) < 1e-14:
        return [length * i / n for i in range(n + 1)]
    th = math.tanh(gamma)
    return [0.5 * length * (1.0 - math.tanh(gamma * (1.0 - 2.0 * (i / n))) / th)
            for i in range(n + 1)]


def axis_metrics(n: int, length: float, gamma: float = 0.0, uniform: bool = True,
                 periodic: bool = False):
    """(dx, dmx) arrays of n + 2 entries (Grid::build_axis)."""
    xf = face_positions(n, gamma, length, uniform)
    xc = [0.0] * (n + 2)
    for i in range(1, n + 1):
        xc[i] = 0.5 * (xf[i - 1] + xf[i])
    if periodic:
        xc[0] = xc[n] - length
        xc[n + 1] = xc[1] + length
    else:
        xc[0] = xf[0] - (xc[1] - xf[0])
        xc[n + 1] = xf[n] + (xf[n] - xc[n])
    dx = [0.0] * (n + 2)
    for i in range(1, n + 1):
        dx[i] = xf[i] - xf[i - 1]
    dx[0] = dx[n] if periodic else dx[1]
    dx[n + 1] = dx[1] if periodic else dx[n]
    dmx = [0.0] * (n + 2)
    for i in range(1, n + 2):
        dmx[i] = xc[i] - xc[i - 1]
    dmx[0] = dmx[n] if periodic else dmx[1]
    return np.array(dx), np.array(dmx)


def mode_lambdas(n1m: int, n2m: int, lx: float, ly: float) -> np.ndarray:
    """kx^2 + ky^2 of every Fourier mode m = j * (n1m // 2 + 1) + i
    (PressureSolverGPU.cu:362-368)."""
    nxh = n1m // 2 + 1
    dx, dy = lx / n1m, ly / n2m
    kx2 = np.array([2.0 * (1.0 - math.cos(2.0 * math.pi * i / n1m)) / (dx * dx)
                    for i in range(nxh)])
    ky2 = np.array([2.0 * (1.0 - math.cos(2.0 * math.pi * (j if j <= n2m // 2 else j - n2m)
                                          / n2m)) / (dy * dy) for j in range(n2m)])
    return (ky2[:, None] + kx2[None, :]).reshape(-1)
