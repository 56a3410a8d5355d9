"""The allocation-free entry point, btdma_solve_noalloc, through the C ABI.

It serves callers that may not allocate device memory (a framework that owns
the memory pool, latency-critical loops, contexts where allocation calls are
forbidden): its scratch is a fixed array inside the library.  Here it must give
exactly what the oracle's serial Thomas (the reference's tdma_many restated)
gives — bit-identical, the bar of every P = 1 test — and exactly what the
handle-based entry point (btdma_solve with P = 1) gives, on two calls in a row
(the array keeps the first call's contents), and refuse batches above its
limit.

This file is collected last so that a failure here cannot hide another test;
it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

from filtered_tdma_b200 import Solver
from filtered_tdma_b200 import _lib as L
from filtered_tdma_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _solve_noalloc(cuda, A, B, C, D):
    import torch
    dA, dB, dC, dD = [torch.from_numpy(np.ascontiguousarray(x)).to(cuda) for x in (A, B, C, D)]
    n_row, n_sys = D.shape
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.lib().btdma_solve_noalloc(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), dD.data_ptr(),
                                     n_sys, n_row, stream)
    L.check(rc)
    torch.cuda.synchronize()
    assert np.array_equal(dA.cpu().numpy(), A) and np.array_equal(dC.cpu().numpy(), C)
    return dD.cpu().numpy()


def _solve_handle(cuda, A, B, C, D):
    import torch
    dA, dB, dC, dD = [torch.from_numpy(np.ascontiguousarray(x)).to(cuda) for x in (A, B, C, D)]
    n_row, n_sys = D.shape
    Solver("pascal", n_sys, n_row, 1).solve(dA, dB, dC, dD)
    return dD.cpu().numpy()


def test_noalloc_matches_oracle_and_handle_solve_twice(cuda, orc):
    # Two different batches back to back: the second call reuses the scratch
    # array the first one left behind.
    batches = [W.diag_dominant(4096, 64, seed=21), W.heat_sweep(2048, 512, r=1.0, seed=22)]
    for A, B, C, D in batches:
        x_na = _solve_noalloc(cuda, A, B, C, D)
        assert np.array_equal(x_na, orc.thomas(A, B, C, D))
        x_h = _solve_handle(cuda, A, B, C, D)
        assert np.array_equal(x_na, x_h)


def test_noalloc_rejects_oversize(cuda):
    import torch
    n_sys, n_row = 2049, 512  # one system past the 1 << 20 element limit
    assert n_sys * n_row > L.NOALLOC_MAX_ELEMS
    x = torch.zeros((n_row, n_sys), dtype=torch.float64, device=cuda)
    rc = L.lib().btdma_solve_noalloc(x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(),
                                     n_sys, n_row, torch.cuda.current_stream().cuda_stream)
    assert rc == L.ERR_SIZE
    assert b"allocation-free limit" in L.lib().btdma_last_error()
