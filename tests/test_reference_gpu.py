"""The reference's own GPU kernels (oracle/_ref/libref_gpu.so: tdma_many_cuda,
PaScaL's modified Thomas / update, Filtered v2's passes, compiled for sm_100a
from the reference's unmodified sources) on one GPU, against the oracle.

These kernels are the GPU baseline bench.py times beside the library's own, so
they must be shown to solve the same systems: the P ranks of the reference run
as row blocks of one array with the MPI transport replaced by pointers
(oracle/ref_gpu_driver.cu).  The reference's GPU kernels divide where its CPU
code multiplies by a reciprocal, and nvcc contracts multiply-adds, so the bar is
1e-12 relative, not bit identity (the library's P = 1 kernel is the bit-exact
one).
"""
import numpy as np
import pytest

from filtered_tdma_b200 import workloads as W
from oracle import ref_gpu as R

needs_ref = pytest.mark.skipif(not R.available(), reason="reference GPU build absent")


def rel_err(x, ref):
    return float(np.max(np.abs(x - ref)) / np.max(np.abs(ref)))


@needs_ref
def test_reference_gpu_library_exports():
    L = R.lib()
    for name in ("refgpu_tdma_many", "refgpu_pascal", "refgpu_filtered_set_rho",
                 "refgpu_filtered_v2", "refgpu_launches"):
        assert hasattr(L, name)
    assert R.launches("pascal", 8) == 17


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("n_sys,n_row", [(4096, 64), (8192, 512)])
def test_reference_tdma_many(cuda, orc, n_sys, n_row):
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=31)
    dA, dB, dC, dD = _dev(cuda, A, B, C, D)
    R.tdma_many(dA, dB, dC, dD)
    assert rel_err(dD.cpu().numpy(), orc.thomas(A, B, C, D)) <= 1e-12


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("n_sys,n_row,P", [(4096, 64, 4), (8192, 512, 8), (1000, 200, 5)])
def test_reference_pascal(cuda, orc, n_sys, n_row, P):
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=32)
    dA, dB, dC, dD = _dev(cuda, A, B, C, D)
    R.pascal(dA, dB, dC, dD, P)
    assert rel_err(dD.cpu().numpy(), orc.pascal(A, B, C, D, P)) <= 1e-12


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("r_hi", [1.0, 10.0])
def test_reference_filtered_v2(cuda, orc, r_hi):
    # r_hi = 1: J < m - 2 (the truncation active); r_hi = 10: J = m - 1
    n_sys, n_row, P = 8192, 512, 8
    A, B, C, D = W.diag_dominant(n_sys, n_row, 0.1, r_hi, seed=33)
    dA, dB, dC, dD = _dev(cuda, A, B, C, D)
    R.filtered_set_rho(dA, dB, dC, P)
    J = R.filtered_v2(dA, dB, dC, dD, P, 1e-3, want_J=True)
    xo, Jo = orc.filtered(A, B, C, D, P, 2, False, 1e-3, orc.rho_rows(A, B, C, 0),
                          orc.J_DEVICE)
    assert J == list(Jo)
    assert rel_err(dD.cpu().numpy(), xo) <= 1e-12
