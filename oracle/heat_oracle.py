"""CPU restatement of the reference's 3-D heat ADI step — TEST INFRASTRUCTURE ONLY.

numpy for the stencil, ghost and layout work; the tridiagonal sweeps go through
the oracle's serial Thomas (tdma_many restated in tdma_oracle.c), which is what
the reference's heat application runs with the pascal backend on one rank.

Follows, for one MPI rank (every face a physical Dirichlet wall):
  * parameters and dt policy        apps/heat_cpu/global.cpp:60-104
  * mesh (cell centres + ghosts)    apps/heat_cpu/mpi_subdomain.cpp mesh()
  * initial field                   mpi_subdomain.cpp initialization()
  * ghost fill u_g = 2 u_BC - u_adj mpi_subdomain.cpp boundary()
  * right-hand side                 apps/heat_gpu/solve_theta.cu:121-160
  * Z / Y / X sweeps with fully implicit walls   solve_theta.cu:168-332
                                                 (heat_cpu/solve_theta.cpp:142-327)
  * L2 error                        apps/heat_cpu/main.cpp:59-79

Pinned by the reference's own published numbers: the order-accuracy run at 32^3
(apps/heat_cpu/results/order_accuracy/order_cpu_20260628_201654.txt, pascal,
np=1) reports L2 = 0.00153948 at rho = 0.25 and 0.0134171 at rho = 0.40.
Arrays are theta[k, j, i] on the full grid (n + 2 points per axis).
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

PI = 3.14159265358979323846


def params(n: int, rho: float, option: str = "order", nt: int | None = None):
    """(dx, dt, Nt) of a cubic n^3 run (global.cpp: nx is the input plus one,
    dx = 2 / (nx - 1); "order": dt = rho / (1 - 2 rho) * 2 dx^2 and Nt =
    round(Tmax / dt) with Tmax = 128 steps of the 512 grid; "strong": the given
    Nt)."""
    dx = 2.0 / n
    dt = rho / (1.0 - 2.0 * rho) * (2.0 * dx * dx)
    if option == "order":
        dt_n = rho / (1.0 - 2.0 * rho) * (2.0 * (2.0 / 512.0) * (2.0 / 512.0))
        t_max = dt_n * 128.0
        q = t_max / dt
        steps = int(math.floor(q + 0.5))  # std::round: halves away from zero
    else:
        steps = int(nt)
    return dx, dt, steps


def coords(n: int) -> np.ndarray:
    dd = 2.0 / n
    return np.array([-1.0 + dd / 2.0 + (i - 1) * dd for i in range(n + 2)])


def initial(ix: int, iy: int, iz: int) -> np.ndarray:
    """sin(pi x) sin(pi y) sin(pi z) + cos(pi x) cos(pi y) cos(pi z) on the full
    grid (products of the 1-D factors, evaluated left to right per cell)."""
    x, y, z = coords(ix), coords(iy), coords(iz)
    sx, sy, sz = np.sin(PI * x), np.sin(PI * y), np.sin(PI * z)
    cx, cy, cz = np.cos(PI * x), np.cos(PI * y), np.cos(PI * z)
    return ((sx[None, None, :] * sy[None, :, None]) * sz[:, None, None]
            + (cx[None, None, :] * cy[None, :, None]) * cz[:, None, None])


def _ghosts(th, x, y, z):
    """u_ghost = 2 u_BC - u_adjacent on the six faces (interior face points)."""
    ix, iy, iz = th.shape[2] - 2, th.shape[1] - 2, th.shape[0] - 2
    cy, cz = np.cos(PI * y[1:iy + 1]), np.cos(PI * z[1:iz + 1])
    cx = np.cos(PI * x[1:ix + 1])
    ubc = -(cz[:, None] * cy[None, :])                          # x walls, [k, j]
    th[1:-1, 1:-1, 0] = 2.0 * ubc - th[1:-1, 1:-1, 1]
    th[1:-1, 1:-1, -1] = 2.0 * ubc - th[1:-1, 1:-1, -2]
    ubc = -(cz[:, None] * cx[None, :])                          # y walls, [k, i]
    th[1:-1, 0, 1:-1] = 2.0 * ubc - th[1:-1, 1, 1:-1]
    th[1:-1, -1, 1:-1] = 2.0 * ubc - th[1:-1, -2, 1:-1]
    ubc = -(cy[:, None] * cx[None, :])                          # z walls, [j, i]
    th[0, 1:-1, 1:-1] = 2.0 * ubc - th[1, 1:-1, 1:-1]
    th[-1, 1:-1, 1:-1] = 2.0 * ubc - th[-2, 1:-1, 1:-1]


def _sweep(D, base, n_row):
    """Solve the constant-coefficient sweep: rows -base, 1 + 2 base (+ base on
    the wall rows), -base; D is [n_row, n_sys]."""
    n_sys = D.shape[1]
    A = np.full((n_row, n_sys), -base)
    C = np.full((n_row, n_sys), -base)
    B = np.full((n_row, n_sys), 1.0 - (-2.0 * base))
    B[0] += base
    B[-1] += base
    return O.thomas(A, B, C, D)


def step(th: np.ndarray, dt: float) -> np.ndarray:
    """One ADI step; returns the new field (ghosts refreshed from the old one)."""
    th = th.copy()
    iz, iy, ix = th.shape[0] - 2, th.shape[1] - 2, th.shape[2] - 2
    x, y, z = coords(ix), coords(iy), coords(iz)
    _ghosts(th, x, y, z)
    bx, by, bz = (dt / (2.0 * (2.0 / m) * (2.0 / m)) for m in (ix, iy, iz))
    t = th[1:-1, 1:-1, 1:-1]
    cx = np.cos(PI * x[1:-1])[None, None, :]
    cy = np.cos(PI * y[1:-1])[None, :, None]
    cz = np.cos(PI * z[1:-1])[:, None, None]
    src = dt * 3.0 * PI * PI * cx * cy * cz
    rhs = ((bx * th[1:-1, 1:-1, 2:] + bx * th[1:-1, 1:-1, :-2])
           + (by * th[1:-1, 2:, 1:-1] + by * th[1:-1, :-2, 1:-1])
           + (bz * th[2:, 1:-1, 1:-1] + bz * th[:-2, 1:-1, 1:-1])
           + (1.0 + (-2.0 * bx) + (-2.0 * by) + (-2.0 * bz)) * t + src)
    # Z sweep: [kk][jj][ii] = [n_row = iz, n_sys = iy * ix]
    rhs[0] += bz * (th[0, 1:-1, 1:-1] + th[1, 1:-1, 1:-1])
    rhs[-1] += bz * (th[-1, 1:-1, 1:-1] + th[-2, 1:-1, 1:-1])
    xz = _sweep(rhs.reshape(iz, iy * ix), bz, iz).reshape(iz, iy, ix)
    # Y sweep: [jj][kk][ii]
    dy = np.ascontiguousarray(xz.transpose(1, 0, 2))
    dy[0] += by * (th[1:-1, 0, 1:-1] + th[1:-1, 1, 1:-1])
    dy[-1] += by * (th[1:-1, -1, 1:-1] + th[1:-1, -2, 1:-1])
    xy = _sweep(dy.reshape(iy, iz * ix), by, iy).reshape(iy, iz, ix)
    # X sweep: [ii][kk][jj]
    dx = np.ascontiguousarray(xy.transpose(2, 1, 0))
    dx[0] += bx * (th[1:-1, 1:-1, 0] + th[1:-1, 1:-1, 1])
    dx[-1] += bx * (th[1:-1, 1:-1, -1] + th[1:-1, 1:-1, -2])
    xx = _sweep(dx.reshape(ix, iz * iy), bx, ix).reshape(ix, iz, iy)
    th[1:-1, 1:-1, 1:-1] = xx.transpose(1, 2, 0)
    return th


def l2_error(th: np.ndarray, t_phys: float) -> float:
    """Global L2 error against the manufactured solution, divided by
    (ix + 1)(iy + 1)(iz + 1) as the reference does (main.cpp:59-79)."""
    iz, iy, ix = th.shape[0] - 2, th.shape[1] - 2, th.shape[2] - 2
    x, y, z = coords(ix)[1:-1], coords(iy)[1:-1], coords(iz)[1:-1]
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    exact = (np.sin(PI * X) * np.sin(PI * Y) * np.sin(PI * Z) * np.exp(-3.0 * PI * PI * t_phys)
             + np.cos(PI * X) * np.cos(PI * Y) * np.cos(PI * Z))
    err = th[1:-1, 1:-1, 1:-1] - exact
    return float(np.sqrt(np.sum(err * err) / ((ix + 1) * (iy + 1) * (iz + 1))))


def run(n: int, rho: float, option: str = "order", nt: int | None = None):
    """(theta, L2, steps) of the reference's heat run on an n^3 grid."""
    _, dt, steps = params(n, rho, option, nt)
    th = initial(n, n, n)
    for _ in range(steps):
        th = step(th, dt)
    return th, l2_error(th, steps * dt), steps
