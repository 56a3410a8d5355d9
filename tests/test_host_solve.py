"""btdma_solve_host: batches in host memory, copied in, solved and copied out in
overlapping chunks of systems.

A PaScaL chunk is solved by the same kernels as the whole batch, so the result
equals btdma_solve_out on device copies of the arrays bit for bit when every
chunk takes the tiled path (even chunk sizes); a batch with an odd last chunk
is held to the tiled path's 1e-12 relative bound against the serial Thomas.
Filtered batches go through as one chunk and equal the device solve exactly.
"""
import numpy as np
import pytest

from filtered_tdma_b200 import Solver
from filtered_tdma_b200 import _lib as L
from filtered_tdma_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel_err(x, ref):
    return float(np.max(np.abs(x - ref)) / np.max(np.abs(ref)))


def host_arrays(arrays, pinned=True):
    import torch
    out = [torch.from_numpy(np.ascontiguousarray(v)) for v in arrays]
    return [t.pin_memory() for t in out] if pinned else out


def device_solve(s, arrays, cuda, cyclic=False):
    import torch
    dA, dB, dC, dD = [torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for v in arrays]
    X = torch.empty_like(dD)
    s.solve_out(dA, dB, dC, dD, X, cyclic=cyclic)
    torch.cuda.synchronize()
    return X.cpu().numpy()


def host_solve(s, arrays, pinned=True, cyclic=False):
    import torch
    hA, hB, hC, hD = host_arrays(arrays, pinned)
    hX = torch.full_like(hD, 7.0)
    hX = hX.pin_memory() if pinned else hX
    s.solve_host(hA, hB, hC, hD, hX, cyclic=cyclic)
    torch.cuda.synchronize()
    assert np.array_equal(hD.numpy(), arrays[3])  # D unchanged
    assert s.status() == 0
    return hX.numpy().copy()


@pytest.mark.parametrize("cyclic", [False, True])
def test_chunks_equal_device_solve(cuda, orc, cyclic):
    # 40000 systems: 8 chunks of 5024 (the last 4832), each on the tiled path
    n_sys, n_row = 40000, 256
    arrays = W.row_varying(n_sys, n_row, seed=3 + int(cyclic))
    s = Solver("pascal", n_sys, n_row, 8)
    xh = host_solve(s, arrays, cyclic=cyclic)
    xd = device_solve(s, arrays, cuda, cyclic=cyclic)
    assert np.array_equal(xh, xd)
    ref = orc.thomas_cyclic(*arrays) if cyclic else orc.thomas(*arrays)
    assert rel_err(xh, ref) <= 1e-12


def test_two_calls_in_a_row_and_pageable_memory(cuda, orc):
    n_sys, n_row = 20000, 512
    s = Solver("pascal", n_sys, n_row, 8)
    for seed, pinned in ((11, True), (12, False)):
        arrays = W.row_varying(n_sys, n_row, seed=seed)
        xh = host_solve(s, arrays, pinned=pinned)
        assert np.array_equal(xh, device_solve(s, arrays, cuda))


def test_odd_last_chunk(cuda, orc):
    n_sys, n_row = 30001, 128  # chunks of 4096, the last 1329 systems
    arrays = W.row_varying(n_sys, n_row, seed=5)
    s = Solver("pascal", n_sys, n_row, 4)
    assert rel_err(host_solve(s, arrays), orc.thomas(*arrays)) <= 1e-12


@pytest.mark.parametrize("method,P,flags", [("filtered_v2", 8, 0), ("pascal", 1, 0),
                                            ("pascal", 4, L.FLAG_REFERENCE_ORDER)])
def test_exact_paths_equal_device_solve(cuda, method, P, flags):
    n_sys, n_row = 9000, 256
    arrays = W.row_varying(n_sys, n_row, seed=P)
    s = Solver(method, n_sys, n_row, P, flags=flags)
    assert np.array_equal(host_solve(s, arrays), device_solve(s, arrays, cuda))


def test_rejects(cuda):
    import torch
    s = Solver("pascal", 1024, 64, 4, precision=L.FP32_STORE)
    h = [torch.zeros((64, 1024), dtype=torch.float64) for _ in range(5)]
    with pytest.raises(L.BtdmaError):
        s.solve_host(*h)
    s = Solver("pascal", 1024, 64, 4)
    with pytest.raises(L.BtdmaError):
        s.solve_host(*[torch.zeros((64, 2048), dtype=torch.float64) for _ in range(5)])
    with pytest.raises(ValueError):
        s.solve_host(*[x.to(cuda) for x in h])


def test_failed_chunk_leaves_the_handle_usable(cuda):
    # periodic systems need 3 rows: the solve of the first chunk fails after its
    # copy-in was queued; the call reports it and the handle keeps working
    import torch
    n_sys, n_row = 8192, 2
    arrays = W.row_varying(n_sys, n_row, seed=9)
    s = Solver("pascal", n_sys, n_row, 1)
    hA, hB, hC, hD = host_arrays(arrays)
    hX = torch.zeros_like(hD).pin_memory()
    with pytest.raises(L.BtdmaError):
        s.solve_host(hA, hB, hC, hD, hX, cyclic=True)
    torch.cuda.synchronize()
    assert np.array_equal(host_solve(s, arrays), device_solve(s, arrays, cuda))
