"""CPU restatement of the channel Poisson wall-normal solve — TEST INFRASTRUCTURE ONLY.

Builds, per Fourier mode, the tridiagonal system of k_build_poisson_tdma
(apps/channel_gpu/PressureSolverGPU.cu:183-210) with the mode-(0,0) pin of
k_zero_mode (:212-220), and solves the real and imaginary right-hand sides
with the oracle's serial Thomas (tdma_many restated), as solve_tdma_z_
(:514-537) does with two TDMA calls.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def matrices(dz, dmz, lam, nz, pin_mode0=True):
    """A, B, C as [nz, n_modes] arrays."""
    n_modes = lam.size
    a = np.array([0.0 if k == 0 else 1.0 / (dz[k + 1] * dmz[k + 1]) for k in range(nz)])
    c = np.array([0.0 if k == nz - 1 else 1.0 / (dz[k + 1] * dmz[k + 2]) for k in range(nz)])
    A = np.repeat(a[:, None], n_modes, axis=1)
    C = np.repeat(c[:, None], n_modes, axis=1)
    B = -(A + C) - lam[None, :]
    if pin_mode0:
        A[0, 0], B[0, 0], C[0, 0] = 0.0, 1.0, 0.0
    return A, B, C


def solve(dz, dmz, lam, rhs, pin_mode0=True):
    """rhs: complex [nz, n_modes]; returns the complex solution."""
    nz = rhs.shape[0]
    A, B, C = matrices(dz, dmz, lam, nz, pin_mode0)
    re = np.ascontiguousarray(rhs.real)
    im = np.ascontiguousarray(rhs.imag)
    if pin_mode0:
        re[0, 0] = 0.0
        im[0, 0] = 0.0
    return O.thomas(A, B, C, re) + 1j * O.thomas(A, B, C, im)
