"""Seeded synthetic batches with the shapes and value distributions of the
reference's workloads.

The reference has no public dataset; its benchmarks solve the tridiagonal
systems of a 3-D heat ADI step and of a channel-flow Poisson/momentum solve.
These generators stand in for them:

* ``heat_sweep``      constant-coefficient heat sweep, A = C = -r, B = 1+2r with
                      one r for the whole batch (r = 1 gives rho = 1/3, as in the
                      reference's 64^3 heat case; apps/heat_cpu/solve_theta.cpp:
                      142-327 builds the same stencil).
* ``diag_dominant``   per-system r drawn log-uniform in [r_lo, r_hi]
                      (A = C = -r, B = 1+2r), D uniform in [-1, 1].
* ``weak_dominance``  per-system rho uniform in [rho_lo, rho_hi], r = rho/(1-2rho).
* ``rho_band``        per-system rho = max(|A/B|, |C/B|) uniform in
                      [rho_lo, rho_hi], reaching past 0.5 while the rows stay
                      strictly dominant: B = 1, A = -rho, C = -(0.9 - rho)
                      (|A| + |C| = 0.9), D uniform in [-1, 1].  The Filtered
                      J bound does not hold at rho >= 0.5 (the reference then
                      sets J = m - 1).
* ``row_varying``     every coefficient drawn on its own (|A|, |C| log-uniform in
                      [0.05, 5] with random signs, B = (|A| + |C|) / rho with rho
                      uniform in [0.3, 0.9] per row), so a kernel that takes a
                      coefficient from the wrong row or system is caught.
* ``ragged_batch``    systems of different lengths (n log-uniform in
                      [n_lo, n_hi]) stored back to back with CSR row offsets,
                      a fraction of them periodic, per-system r log-uniform.

All arrays are [n_row, n_sys] row-interleaved (row j of system i at
j*n_sys + i), as the reference lays them out.  numpy generation (``device=None``)
is bit-reproducible across machines; torch generation on a CUDA device is
reproducible for a given seed on that device type and is used for the large
benchmark batches.
"""
from __future__ import annotations

import numpy as np

try:
    import torch
except ImportError:  # numpy-only use
    torch = None


def _np_batch(r_sys: np.ndarray, n_row: int, D: np.ndarray, dtype):
    n_sys = r_sys.shape[0]
    r = np.broadcast_to(r_sys[None, :], (n_row, n_sys))
    A = np.ascontiguousarray(-r, dtype=dtype)
    C = np.ascontiguousarray(-r, dtype=dtype)
    B = np.ascontiguousarray(1.0 + 2.0 * r, dtype=dtype)
    return A, B, C, np.ascontiguousarray(D, dtype=dtype)


def heat_sweep(n_sys: int, n_row: int, r: float = 1.0, seed: int = 1, dtype=np.float64,
               device=None):
    if device is not None:
        return _torch_batch(np.full(1, r), n_sys, n_row, seed, dtype, device, const_r=r)
    rng = np.random.default_rng(seed)
    D = rng.uniform(-1.0, 1.0, size=(n_row, n_sys))
    return _np_batch(np.full(n_sys, r), n_row, D, dtype)


def diag_dominant(n_sys: int, n_row: int, r_lo: float = 0.1, r_hi: float = 10.0, seed: int = 2,
                  dtype=np.float64, device=None):
    if device is not None:
        return _torch_batch(None, n_sys, n_row, seed, dtype, device,
                            log_r=(np.log10(r_lo), np.log10(r_hi)))
    rng = np.random.default_rng(seed)
    r = 10.0 ** rng.uniform(np.log10(r_lo), np.log10(r_hi), size=n_sys)
    D = rng.uniform(-1.0, 1.0, size=(n_row, n_sys))
    return _np_batch(r, n_row, D, dtype)


def weak_dominance(n_sys: int, n_row: int, rho_lo: float = 0.45, rho_hi: float = 0.499,
                   seed: int = 3, dtype=np.float64, device=None):
    if device is not None:
        return _torch_batch(None, n_sys, n_row, seed, dtype, device, rho=(rho_lo, rho_hi))
    rng = np.random.default_rng(seed)
    rho = rng.uniform(rho_lo, rho_hi, size=n_sys)
    r = rho / (1.0 - 2.0 * rho)
    D = rng.uniform(-1.0, 1.0, size=(n_row, n_sys))
    return _np_batch(r, n_row, D, dtype)


def rho_band(n_sys: int, n_row: int, rho_lo: float = 0.45, rho_hi: float = 0.55,
             seed: int = 8, dtype=np.float64):
    rng = np.random.default_rng(seed)
    rho = rng.uniform(rho_lo, rho_hi, size=n_sys)
    A = np.broadcast_to(-rho[None, :], (n_row, n_sys))
    C = np.broadcast_to(-(0.9 - rho)[None, :], (n_row, n_sys))
    B = np.ones((n_row, n_sys))
    D = rng.uniform(-1.0, 1.0, size=(n_row, n_sys))
    return tuple(np.ascontiguousarray(v, dtype=dtype) for v in (A, B, C, D))


def row_varying(n_sys: int, n_row: int, seed: int = 7, dtype=np.float64):
    rng = np.random.default_rng(seed)
    shape = (n_row, n_sys)
    a = 10.0 ** rng.uniform(np.log10(0.05), np.log10(5.0), size=shape)
    c = 10.0 ** rng.uniform(np.log10(0.05), np.log10(5.0), size=shape)
    a *= rng.choice([-1.0, 1.0], size=shape)
    c *= rng.choice([-1.0, 1.0], size=shape)
    b = (np.abs(a) + np.abs(c)) / rng.uniform(0.3, 0.9, size=shape)
    D = rng.uniform(-1.0, 1.0, size=shape)
    return tuple(np.ascontiguousarray(v, dtype=dtype) for v in (a, b, c, D))


def _torch_batch(_unused, n_sys, n_row, seed, dtype, device, const_r=None, log_r=None, rho=None):
    if torch is None:
        raise RuntimeError("torch is required for device-side generation")
    tdt = {np.float64: torch.float64, np.float32: torch.float32}.get(dtype, dtype)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if const_r is not None:
        r = torch.full((n_sys,), float(const_r), dtype=torch.float64, device=device)
    elif log_r is not None:
        u = torch.rand(n_sys, generator=g, dtype=torch.float64, device=device)
        r = 10.0 ** (log_r[0] + (log_r[1] - log_r[0]) * u)
    else:
        u = torch.rand(n_sys, generator=g, dtype=torch.float64, device=device)
        rh = rho[0] + (rho[1] - rho[0]) * u
        r = rh / (1.0 - 2.0 * rh)
    D = torch.rand((n_row, n_sys), generator=g, dtype=torch.float64, device=device) * 2.0 - 1.0
    A = (-r).expand(n_row, n_sys).contiguous().to(tdt)
    C = A.clone()
    B = (1.0 + 2.0 * r).expand(n_row, n_sys).contiguous().to(tdt)
    return A, B, C, D.to(tdt)


def ragged_batch(n_sys: int, n_lo: int = 16, n_hi: int = 4096, periodic_frac: float = 0.25,
                 r_lo: float = 0.05, r_hi: float = 20.0, seed: int = 5, dtype=np.float64):
    """Ragged batch in the CSR layout: system i occupies rows
    [off[i], off[i+1]) of the 1-D arrays A, B, C, D (contiguous).  n_i is
    floor(exp(U[ln n_lo, ln n_hi])), a fraction periodic_frac of the systems is
    periodic, r_i is log-uniform in [r_lo, r_hi] (A = C = -r_i, B = 1 + 2 r_i) and
    D is uniform in [-1, 1].  Returns (A, B, C, D, off int64, periodic uint8)."""
    rng = np.random.default_rng(seed)
    n = np.floor(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=n_sys))).astype(np.int64)
    n = np.clip(n, n_lo, n_hi)
    periodic = (rng.uniform(size=n_sys) < periodic_frac).astype(np.uint8)
    r = 10.0 ** rng.uniform(np.log10(r_lo), np.log10(r_hi), size=n_sys)
    off = np.zeros(n_sys + 1, dtype=np.int64)
    np.cumsum(n, out=off[1:])
    rr = np.repeat(r, n)
    A = np.ascontiguousarray(-rr, dtype=dtype)
    C = np.ascontiguousarray(-rr, dtype=dtype)
    B = np.ascontiguousarray(1.0 + 2.0 * rr, dtype=dtype)
    D = np.ascontiguousarray(rng.uniform(-1.0, 1.0, size=int(off[-1])), dtype=dtype)
    return A, B, C, D, off, periodic
