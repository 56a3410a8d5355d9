"""Stream-ordered solves inside CUDA graphs, and the failure path of the
bounded pipeline waits (a wait that runs out sets a status bit; the context
stays usable)."""
import ctypes

import numpy as np
import pytest

from filtered_tdma_b200 import Solver
from filtered_tdma_b200 import _lib as L
from filtered_tdma_b200 import workloads as W


@pytest.mark.gpu
def test_tiled_and_refined_solves_replay_in_a_graph(cuda, orc):
    import torch
    A, B, C, D = W.diag_dominant(4096, 512, seed=61)
    dA, dB, dC, dD = [torch.from_numpy(x).to(cuda) for x in (A, B, C, D)]
    X = torch.zeros_like(dD)
    s = Solver("pascal", 4096, 512, 8)
    s.solve_out(dA, dB, dC, dD, X)  # first use outside the capture
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        s.solve_out(dA, dB, dC, dD, X, stream=stream.cuda_stream)
    X.zero_()
    g.replay()
    torch.cuda.synchronize()
    ref = orc.thomas(A, B, C, D)
    assert np.max(np.abs(X.cpu().numpy() - ref)) / np.max(np.abs(ref)) <= 1e-12
    # FP32 refinement: the gated sweeps are part of the graph
    A32, B32, C32, D32 = [np.ascontiguousarray(x, dtype=np.float32) for x in (A, B, C, D)]
    fA, fB, fC, fD = [torch.from_numpy(x).to(cuda) for x in (A32, B32, C32, D32)]
    r = Solver("pascal", 4096, 512, 8, precision=L.FP32_REFINE)
    r.solve_f32(fA, fB, fC, fD, X)
    torch.cuda.synchronize()
    g2 = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g2, stream=stream):
        r.solve_f32(fA, fB, fC, fD, X, stream=stream.cuda_stream)
    X.zero_()
    g2.replay()
    torch.cuda.synchronize()
    wid = [x.astype(np.float64) for x in (A32, B32, C32, D32)]
    ref2 = orc.thomas(*wid)
    assert np.max(np.abs(X.cpu().numpy() - ref2)) / np.max(np.abs(ref2)) <= 1e-12
    assert r.last_stats()["n_fallback"] == 0


@pytest.mark.gpu
def test_ragged_solve_replays_in_a_graph(cuda, orc):
    import torch
    from ragged_ref import ragged_reference
    A, B, C, D, off, per = W.ragged_batch(200, seed=62)
    dA, dB, dC, dD = [torch.from_numpy(x).to(cuda) for x in (A, B, C, D)]
    X = torch.zeros(int(off[-1]), dtype=torch.float64, device=cuda)
    s = Solver("pascal", 200, 64, 2)
    s.solve_ragged(dA, dB, dC, dD, X, off, per)  # builds the plan outside the capture
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        s.solve_ragged(dA, dB, dC, dD, X, off, per, stream=stream.cuda_stream)
    X.zero_()
    g.replay()
    torch.cuda.synchronize()
    ref = ragged_reference(orc, A, B, C, D, off, per)
    assert np.max(np.abs(X.cpu().numpy() - ref)) / np.max(np.abs(ref)) <= 1e-12


@pytest.mark.gpu
def test_bounded_wait_times_out_and_context_survives(cuda, orc):
    import torch
    st = ctypes.c_uint()
    L.check(L.lib().btdma_selftest_wait_timeout(64, ctypes.byref(st), None))
    assert st.value & 1  # BTDMA_STATUS_TIMEOUT
    # the context still solves correctly afterwards
    A, B, C, D = W.heat_sweep(1024, 64, r=1.0, seed=63)
    dA, dB, dC, dD = [torch.from_numpy(x).to(cuda) for x in (A, B, C, D)]
    Solver("pascal", 1024, 64, 1).solve(dA, dB, dC, dD)
    assert np.array_equal(dD.cpu().numpy(), orc.thomas(A, B, C, D))


def test_selftest_argument_check():
    st = ctypes.c_uint()
    assert L.lib().btdma_selftest_wait_timeout(0, ctypes.byref(st), None) == L.ERR_ARG
