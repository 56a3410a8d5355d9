"""Channel Poisson wall-normal solve (btdma_poisson_*) against the CPU
restatement of the reference's build + two TDMA solves.

The matrices are diagonally dominant for every mode but (0, 0), whose row sums
vanish except at the pinned row; that mode is the worst conditioned, so the
bar is stated on the residual of every mode (backward error, 1e-13) plus the
1e-12 relative forward error on all modes but (0, 0).
"""
import numpy as np
import pytest

from oracle import poisson_oracle as PO


def _residual(A, B, C, x, rhs):
    r = B * x - rhs
    r[1:] += A[1:] * x[:-1]
    r[:-1] += C[:-1] * x[1:]
    return r


@pytest.mark.gpu
@pytest.mark.parametrize("n1m,n2m,n3m,gamma", [(32, 16, 64, 2.0), (128, 128, 192, 2.0),
                                              (16, 8, 48, 0.0)])
def test_poisson_matches_oracle(cuda, orc, n1m, n2m, n3m, gamma):
    import torch
    from filtered_tdma_b200.poisson import ChannelPoisson
    p = ChannelPoisson(n1m, n2m, n3m, gamma=gamma)
    rng = np.random.default_rng(4)
    rhs = rng.uniform(-1, 1, (n3m, p.n_modes)) + 1j * rng.uniform(-1, 1, (n3m, p.n_modes))
    hat = torch.from_numpy(rhs.copy()).to(cuda)
    p.solve(hat)
    torch.cuda.synchronize()
    assert p.status() == 0
    x = hat.cpu().numpy()
    ref = PO.solve(p.dz, p.dmz, p.lam, rhs)
    err = np.abs(x - ref).max(axis=0) / np.abs(ref).max(axis=0)
    assert err[1:].max() <= 1e-12
    A, B, C = PO.matrices(p.dz, p.dmz, p.lam, n3m)
    b = rhs.copy()
    b[0, 0] = 0.0
    for part in (np.real, np.imag):
        res = _residual(A, B, C, part(x), part(b))
        scale = (np.abs(A) + np.abs(B) + np.abs(C)) * np.abs(part(x)).max(axis=0) + np.abs(part(b))
        assert (np.abs(res) / scale.max(axis=0)).max() <= 1e-13


def test_poisson_grid_matches_reference_formulas():
    from filtered_tdma_b200.poisson import mode_lambdas, wall_normal_grid
    dz, dmz = wall_normal_grid(8, 2.0, 2.0)
    assert abs(dz[1:-1].sum() - 2.0) < 1e-14       # faces span the channel height
    assert dz[0] == dz[1] and dz[-1] == dz[-2]      # mirror ghosts
    assert dmz[1] == dz[1]                           # mirror convention at the wall
    lam = mode_lambdas(8, 4, 4.0, 2.0)
    assert lam.shape == (4 * 5,) and lam[0] == 0.0 and (lam[1:] > 0).all()


def test_poisson_argument_checks():
    import ctypes
    from filtered_tdma_b200 import _lib as L
    h = ctypes.c_void_p()
    z = np.zeros(40)
    assert L.lib().btdma_poisson_create(30, z.ctypes.data, z.ctypes.data, 4, z.ctypes.data, 1,
                                        ctypes.byref(h)) == L.ERR_UNSUPPORTED
    assert L.lib().btdma_poisson_create(32, None, None, 4, None, 1, ctypes.byref(h)) == L.ERR_ARG
    assert L.lib().btdma_poisson_solve(None, None, None) == L.ERR_ARG
