"""The reference's channel-flow coefficient builds (oracle/_ref/libref_channel.so:
k_build_{x,y,z} / k_scatter_{x,y,z} of apps/channel_gpu/MomentumSolverGPU.cu and
k_build_poisson_tdma / k_zero_mode / k_write_poisson_solution of
PressureSolverGPU.cu, compiled unmodified) pin the CPU restatements in
oracle/momentum_oracle.py and oracle/poisson_oracle.py.

Each test runs the reference's own pipeline for one solve on the GPU -- its
build kernel, the serial Thomas (the oracle's, bit-identical to the
reference's tdma_many / tdma_cyclic_many), its scatter / write-back kernel --
and requires the restatement's result bit for bit.  The library's own paths
are compared with the restatements in tests/test_momentum.py and
tests/test_poisson.py, so these tests carry the reference's numbers through to
them.
"""
import numpy as np
import pytest

from oracle import momentum_oracle as MO
from oracle import poisson_oracle as PO
from oracle import ref_channel as RC

needs_ref = pytest.mark.skipif(not RC.available(), reason="reference channel build absent")


@needs_ref
def test_reference_channel_library_exports():
    L = RC.lib()
    for name in ("refch_build", "refch_scatter", "refch_poisson_build", "refch_poisson_write"):
        assert hasattr(L, name)


def _ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return int(np.max(np.abs(ia - ib))) if a.size else 0


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("comp", [0, 1, 2])
def test_momentum_sweep_pinned_by_reference_build(cuda, orc, direction, comp):
    import torch
    from filtered_tdma_b200.channel_grid import axis_metrics
    nx, ny, nz = 32, 24, 40
    metrics = (axis_metrics(nx, 4.0, periodic=True), axis_metrics(ny, 2.0, periodic=True),
               axis_metrics(nz, 2.0, gamma=1.5, uniform=False))
    rng = np.random.default_rng(90 + 3 * direction + comp)
    q = rng.uniform(-1, 1, (nz + 2, ny + 2, nx + 2))
    c = 0.5 * (1.0 / 180.0) * 2e-3 * 50
    periodic = direction < 2
    n_row = (nx, ny, nz)[direction]
    n_sys = nx * ny * nz // n_row
    dq = torch.from_numpy(q).to(cuda)
    A, B, C, D = (torch.empty(n_row * n_sys, dtype=torch.float64, device=cuda) for _ in range(4))
    d, dm = (torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for v in metrics[direction])
    RC.momentum_build(direction, comp, dq, A, B, C, D, d, dm, nx, ny, nz, c)
    torch.cuda.synchronize()
    Ah, Bh, Ch, Dh = (t.cpu().numpy().reshape(n_row, n_sys) for t in (A, B, C, D))
    # every system of a sweep has the same coefficient column
    a, b, cc = MO._coeffs(metrics[direction][0], metrics[direction][1], n_row, comp, direction, c)
    for got, want, name in ((Ah, a, "A"), (Bh, b, "B"), (Ch, cc, "C")):
        col = np.repeat(want[:, None], n_sys, axis=1)
        assert np.array_equal(got, col), (name, _ulps(got, col),
                                          np.nonzero((got != col).any(axis=1))[0].tolist())
    x = orc.thomas_cyclic(Ah, Bh, Ch, Dh) if periodic else orc.thomas(Ah, Bh, Ch, Dh)
    D.copy_(torch.from_numpy(np.ascontiguousarray(x).reshape(-1)))
    out = dq.clone()
    RC.momentum_scatter(direction, D, out, nx, ny, nz)
    torch.cuda.synchronize()
    ref = MO.sweep(q, metrics, direction, comp, c, periodic)
    assert np.array_equal(out.cpu().numpy(), ref)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("n1m,n2m,n3m,gamma", [(32, 16, 64, 2.0), (16, 8, 48, 0.0)])
def test_poisson_solve_pinned_by_reference_build(cuda, orc, n1m, n2m, n3m, gamma):
    import torch
    from filtered_tdma_b200.poisson import wall_normal_grid
    dz, dmz = wall_normal_grid(n3m, gamma, 2.0)
    hme = n1m // 2 + 1
    nsys = hme * n2m
    rng = np.random.default_rng(7 + n1m + n3m)
    kx2 = rng.uniform(0.0, 40.0, hme)
    ky2 = rng.uniform(0.0, 40.0, n2m)
    kx2[0] = ky2[0] = 0.0
    lam = (kx2[None, :] + ky2[:, None]).reshape(-1)   # mode m = j * hme + ix
    rhs = rng.uniform(-1, 1, (n3m, nsys)) + 1j * rng.uniform(-1, 1, (n3m, nsys))
    hat = torch.from_numpy(rhs.copy()).to(cuda)
    bufs = [torch.empty(n3m * nsys, dtype=torch.float64, device=cuda) for _ in range(8)]
    Am, Ac, Ap, Am2, Ac2, Ap2, Br, Bi = bufs
    dev = [torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for v in (dz, dmz, kx2, ky2)]
    RC.poisson_build(hat, Am, Ac, Ap, Am2, Ac2, Ap2, Br, Bi, *dev, n3m, nsys, hme, n2m)
    torch.cuda.synchronize()
    h = [t.cpu().numpy().reshape(n3m, nsys) for t in bufs]
    A, B, C = PO.matrices(dz, dmz, lam, n3m)
    for got, want, name in ((h[0], A, "Am"), (h[1], B, "Ac"), (h[2], C, "Ap"),
                            (h[3], A, "Am2"), (h[4], B, "Ac2"), (h[5], C, "Ap2")):
        assert np.array_equal(got, want), (name, _ulps(got, want))
    xr = orc.thomas(h[0], h[1], h[2], h[6])
    xi = orc.thomas(h[3], h[4], h[5], h[7])
    Br.copy_(torch.from_numpy(np.ascontiguousarray(xr).reshape(-1)))
    Bi.copy_(torch.from_numpy(np.ascontiguousarray(xi).reshape(-1)))
    out = torch.zeros_like(hat)
    RC.poisson_write(out, Br, Bi, n3m, nsys, hme, n2m)
    torch.cuda.synchronize()
    ref = PO.solve(dz, dmz, lam, rhs)
    assert np.array_equal(out.cpu().numpy(), ref)
