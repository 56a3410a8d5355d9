"""CPU restatement of the channel momentum ADI sweeps — TEST INFRASTRUCTURE ONLY.

Builds A, B, C, D of one sweep exactly as k_build_{x,y,z}
(apps/channel_gpu/MomentumSolverGPU.cu:135-210; walls for one rank holding
all of z), solves with the oracle's serial Thomas or periodic Thomas
(tdma_many / tdma_cyclic_many restated), and scatters back (k_scatter_*).
Fields are numpy arrays q[k, j, i] with one ghost layer.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def _coeffs(dx, dm, n, comp, d, c):
    """A, B, C for rows r = 1..n (one column; every system of the sweep shares it)."""
    a = np.empty(n)
    b = np.empty(n)
    cc = np.empty(n)
    for r in range(1, n + 1):
        if comp == d:
            ar, cr = 1.0 / (dm[r] * dx[r - 1]), 1.0 / (dm[r] * dx[r])
        else:
            ar, cr = 1.0 / (dx[r] * dm[r]), 1.0 / (dx[r] * dm[r + 1])
        av, cv = -c * ar, -c * cr
        bv = 1.0 - av - cv
        if d == 2:
            is_w = comp == 2
            if r == 1:
                av = 0.0
                if not is_w:
                    bv += c * ar
            if r == n:
                cv = 0.0
                if not is_w:
                    bv += c * cr
            if is_w and r == 1:
                av, bv, cv = 0.0, 1.0, 0.0
        a[r - 1], b[r - 1], cc[r - 1] = av, bv, cv
    return a, b, cc


def sweep(q, metrics, direction, comp, c, periodic, solver=None):
    """The solution of one sweep, scattered into a copy of q's interior.
    solver(A, B, C, D, periodic) -> x replaces the serial (periodic) Thomas."""
    nz, ny, nx = q.shape[0] - 2, q.shape[1] - 2, q.shape[2] - 2
    n = (nx, ny, nz)[direction]
    dx, dm = metrics[direction]
    a, b, cc = _coeffs(dx, dm, n, comp, direction, c)
    inner = q[1:-1, 1:-1, 1:-1]
    axis = {0: 2, 1: 1, 2: 0}[direction]
    D = np.moveaxis(inner, axis, 0).reshape(n, -1).copy()   # rows along the sweep
    if direction == 2 and comp == 2:
        D[0] = 0.0
    n_sys = D.shape[1]
    A = np.repeat(a[:, None], n_sys, axis=1)
    B = np.repeat(b[:, None], n_sys, axis=1)
    C = np.repeat(cc[:, None], n_sys, axis=1)
    if solver is not None:
        x = solver(A, B, C, D, periodic)
    else:
        x = O.thomas_cyclic(A, B, C, D) if periodic else O.thomas(A, B, C, D)
    out = q.copy()
    shape = list(np.moveaxis(inner, axis, 0).shape)
    out[1:-1, 1:-1, 1:-1] = np.moveaxis(x.reshape(shape), 0, axis)
    return out


def adi(rhs, metrics, comp, c, pbc):
    """z, y, x sweeps (MomentumSolverGPU::advance's diffuse step after k_lap)."""
    r = sweep(rhs, metrics, 2, comp, c, False)
    r = sweep(r, metrics, 1, comp, c, pbc[1])
    return sweep(r, metrics, 0, comp, c, pbc[0])
