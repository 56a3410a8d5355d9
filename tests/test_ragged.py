"""Ragged batches (CSR row offsets, systems of different lengths, some periodic)
through the C ABI, against the oracle's serial Thomas / periodic Thomas solved
system by system (tdma_many / tdma_cyclic_many with n_sys = 1).

PaScaL's segmented elimination is not the serial order, so the bar is the
1e-12 relative bound of the segmented FP64 paths; FP32-stored batches are
compared with the oracle on the widened values.
"""
import numpy as np
import pytest

from filtered_tdma_b200 import Solver
from filtered_tdma_b200 import _lib as L
from filtered_tdma_b200 import workloads as W


def ragged_oracle(orc, A, B, C, D, off, per):
    x = np.empty_like(np.asarray(D, dtype=np.float64))
    for i in range(len(off) - 1):
        s = slice(int(off[i]), int(off[i + 1]))
        cols = [np.asarray(v[s], dtype=np.float64)[:, None] for v in (A, B, C, D)]
        f = orc.thomas_cyclic if per[i] else orc.thomas
        x[s] = f(*cols)[:, 0]
    return x


def per_system_err(x, ref, off):
    worst = 0.0
    for i in range(len(off) - 1):
        s = slice(int(off[i]), int(off[i + 1]))
        worst = max(worst, float(np.max(np.abs(x[s] - ref[s])) / np.max(np.abs(ref[s]))))
    return worst


def solve_on_device(cuda, arrays, off, per, precision=L.FP64, tune=False, inplace=False):
    import torch
    dA, dB, dC, dD = [torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for v in arrays]
    n_rows = int(off[-1])
    s = Solver("pascal", len(off) - 1, 64, 2, precision=precision)
    X = dD if inplace else torch.zeros(n_rows, dtype=torch.float64, device=cuda)
    if tune:
        plan = s.ragged_autotune(dA, dB, dC, dD, X, off, per)
        assert all(b["tuned_ms"] > 0 for b in plan)
        dD = torch.from_numpy(np.ascontiguousarray(arrays[3])).to(cuda)
        if inplace:
            X = dD
        else:
            X.zero_()  # the tuner's solves wrote X: the tuned plan's solve alone counts
    s.solve_ragged(dA, dB, dC, dD, X, off, per)
    torch.cuda.synchronize()
    assert s.status() == 0
    return X.cpu().numpy(), s.ragged_plan()


@pytest.mark.gpu
def test_ragged_config_shape_fp64(cuda, orc):
    # the ragged workload's distributions (n log-uniform in [16, 4096], 25 %
    # periodic, r log-uniform in [0.05, 20]) at 400 systems
    A, B, C, D, off, per = W.ragged_batch(400, seed=5)
    ref = ragged_oracle(orc, A, B, C, D, off, per)
    x, plan = solve_on_device(cuda, (A, B, C, D), off, per)
    assert per_system_err(x, ref, off) <= 1e-12
    assert sum(b["n_systems"] for b in plan) == 400
    assert {b["periodic"] for b in plan} == {0, 1}


@pytest.mark.gpu
def test_ragged_full_config_10000(cuda, orc):
    # the whole ragged configuration: 10000 systems, n log-uniform in
    # [16, 4096] (7.3 M rows), 25 % periodic, r log-uniform in [0.05, 20],
    # autotuned; FP64 and FP32 storage (on the widened values), every system
    # within 1e-12 of the oracle's serial (periodic) Thomas
    A, B, C, D, off, per = W.ragged_batch(10000, seed=5)
    assert int(off[-1]) > 7_000_000 and per.sum() > 2000
    ref = ragged_oracle(orc, A, B, C, D, off, per)
    x, plan = solve_on_device(cuda, (A, B, C, D), off, per, tune=True)
    assert per_system_err(x, ref, off) <= 1e-12
    assert sum(b["n_systems"] for b in plan) == 10000
    A32, B32, C32, D32 = (v.astype(np.float32) for v in (A, B, C, D))
    ref32 = ragged_oracle(orc, *(v.astype(np.float64) for v in (A32, B32, C32, D32)), off, per)
    x32, _ = solve_on_device(cuda, (A32, B32, C32, D32), off, per, precision=L.FP32_STORE,
                             tune=True)
    assert per_system_err(x32, ref32, off) <= 1e-12


@pytest.mark.gpu
def test_ragged_autotuned_and_inplace(cuda, orc):
    A, B, C, D, off, per = W.ragged_batch(300, seed=51)
    ref = ragged_oracle(orc, A, B, C, D, off, per)
    x, plan = solve_on_device(cuda, (A, B, C, D), off, per, tune=True, inplace=True)
    assert per_system_err(x, ref, off) <= 1e-12
    for b in plan:
        assert b["lanes_per_system"] & (b["lanes_per_system"] - 1) == 0
        assert b["n_row_min"] // b["lanes_per_system"] >= 3


@pytest.mark.gpu
def test_ragged_fp32_storage(cuda, orc):
    A, B, C, D, off, per = W.ragged_batch(300, seed=52, dtype=np.float32)
    wid = [v.astype(np.float64) for v in (A, B, C, D)]
    ref = ragged_oracle(orc, *wid, off, per)
    x, _ = solve_on_device(cuda, (A, B, C, D), off, per, precision=L.FP32_STORE)
    assert per_system_err(x, ref, off) <= 1e-12


@pytest.mark.gpu
def test_ragged_short_and_uniform_systems(cuda, orc):
    # 3..40 rows (one lane per system below 6 rows), every length present, both
    # kinds; then a uniform batch that fills one bucket
    rng = np.random.default_rng(53)
    n = np.repeat(np.arange(3, 41), 3)
    per = (np.arange(n.size) % 2).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
    r = np.repeat(10.0 ** rng.uniform(-1, 1, n.size), n)
    A, C, B = -r, -r, 1 + 2 * r
    D = rng.uniform(-1, 1, int(off[-1]))
    ref = ragged_oracle(orc, A, B, C, D, off, per)
    x, _ = solve_on_device(cuda, (A, B, C, D), off, per)
    assert per_system_err(x, ref, off) <= 1e-12
    off2 = np.arange(0, 257 * 128, 128, dtype=np.int64)
    A2, B2, C2, D2 = [v[:, 0].copy() for v in W.diag_dominant(1, 256 * 128, seed=54)]
    x2, plan = solve_on_device(cuda, (A2, B2, C2, D2), off2, None)
    ref2 = ragged_oracle(orc, A2, B2, C2, D2, off2, np.zeros(256, np.uint8))
    assert per_system_err(x2, ref2, off2) <= 1e-12
    assert len(plan) == 1


def test_ragged_argument_checks():
    import ctypes
    lib = L.lib()
    vp = ctypes.c_void_p(1)
    off = np.array([0, 2, 10], dtype=np.int64)  # a 2-row system
    assert lib.btdma_solve_ragged(None, vp, vp, vp, vp, vp, off.ctypes.data, None, 2,
                                  None) == L.ERR_ARG
    assert lib.btdma_ragged_autotune(None, vp, vp, vp, vp, vp, off.ctypes.data, None, 2,
                                     None) == L.ERR_ARG
    n = ctypes.c_int()
    assert lib.btdma_ragged_plan_info(None, None, 0, ctypes.byref(n)) == L.ERR_ARG
    assert lib.btdma_ragged_set_plan(None, None, 0) == L.ERR_ARG


@pytest.mark.gpu
def test_ragged_long_systems_cta_path(cuda, orc):
    # one CTA per system above 512 rows, up to 8192 rows (512 threads x 16 rows)
    rng = np.random.default_rng(55)
    n = np.array([513, 600, 1000, 1024, 1025, 2047, 4096, 5000, 8192, 8192, 700, 3000])
    per = np.array([0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 1, 0], dtype=np.uint8)
    off = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
    r = np.repeat(10.0 ** rng.uniform(-1.3, 1.3, n.size), n)
    A, C, B = -r, -r, 1 + 2 * r
    D = rng.uniform(-1, 1, int(off[-1]))
    ref = ragged_oracle(orc, A, B, C, D, off, per)
    x, plan = solve_on_device(cuda, (A, B, C, D), off, per)
    assert per_system_err(x, ref, off) <= 1e-12
    assert any(b["cta_per_system"] == 1 and b["lanes_per_system"] == 512 for b in plan)
    x, plan = solve_on_device(cuda, (A, B, C, D), off, per, tune=True)
    assert per_system_err(x, ref, off) <= 1e-12


@pytest.mark.gpu
def test_ragged_row_varying_coefficients(cuda, orc):
    # coefficients drawn per row (the other ragged batches hold one triple per
    # system), lengths across the warp and CTA kinds, both kinds of system
    n = np.array([3, 5, 17, 40, 64, 100, 255, 256, 511, 600, 1024, 3000, 5000] * 3)
    per = (np.arange(n.size) % 3 == 1).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
    A, B, C, D = [v[:, 0].copy() for v in W.row_varying(1, int(off[-1]), seed=57)]
    ref = ragged_oracle(orc, A, B, C, D, off, per)
    x, _ = solve_on_device(cuda, (A, B, C, D), off, per)
    assert per_system_err(x, ref, off) <= 1e-12
    x, _ = solve_on_device(cuda, (A, B, C, D), off, per, tune=True)
    assert per_system_err(x, ref, off) <= 1e-12


def _shapes(b):
    """Every launch shape the library accepts for bucket b: (P, cta_per_system)."""
    out = []
    for P in (1, 2, 4, 8, 16, 32):
        if b["n_row_min"] // P >= 3 and -(-b["n_row_max"] // P) <= 32:
            out.append((P, 0))
    for P in (64, 128, 256, 512):
        mcap = -(-b["n_row_max"] // P)  # rows per thread
        if b["n_row_min"] // P >= 3 and mcap <= 16:
            out.append((P, 1))
            if 4 * P * (mcap | 1) * 8 + 6 * (P + 2) * 8 <= 227 * 1024:  # staged tile fits
                out.append((P, 2))
    if not b["periodic"]:
        out.append((1, 3))  # interleaved: padded row-interleaved batch, tiled kernel
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ragged_every_launch_shape(cuda, orc, precision):
    """Every shape of every bucket (warp lanes, CTA, CTA staged through shared
    memory, interleaved copy for the tiled kernel), applied with
    btdma_ragged_set_plan, against the oracle."""
    import torch
    dtype = np.float64 if precision == "fp64" else np.float32
    A, B, C, D, off, per = W.ragged_batch(600, seed=58, dtype=dtype)
    ref = ragged_oracle(orc, *[v.astype(np.float64) for v in (A, B, C, D)], off, per)
    dA, dB, dC, dD = [torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for v in (A, B, C, D)]
    s = Solver("pascal", 600, 64, 2, precision=L.FP64 if precision == "fp64" else L.FP32_STORE)
    X = torch.zeros(int(off[-1]), dtype=torch.float64, device=cuda)
    s.solve_ragged(dA, dB, dC, dD, X, off, per)
    plan = s.ragged_plan()
    for bad in (dict(plan[0], lanes_per_system=3), dict(plan[-1], cta_per_system=1,
                                                          lanes_per_system=32),
                dict(plan[0], n_row_max=plan[0]["n_row_max"] + 1)):
        with pytest.raises(L.BtdmaError):
            s.ragged_set_plan([bad] + plan[1:] if bad["n_row_min"] == plan[0]["n_row_min"]
                              else plan[:-1] + [bad])
    cyc = [i for i, b in enumerate(plan) if b["periodic"]]
    assert cyc
    with pytest.raises(L.BtdmaError):  # padding would break the wrap-around coupling
        s.ragged_set_plan([dict(b, cta_per_system=3, lanes_per_system=1) if i == cyc[0] else b
                           for i, b in enumerate(plan)])
    assert s.ragged_plan() == plan  # a rejected plan leaves the current one
    opts = [_shapes(b) for b in plan]
    assert all(opts)
    assert any((P, 2) in o for o in opts for P in (64, 128, 256))
    assert any((512, 2) in o for o in opts)  # staged 512-thread CTAs (<= 8 rows a thread)
    # each shape as a launch of its own, then in the persistent launch (CTA
    # kinds of at most 256 threads, split into groups of their thread counts;
    # warp kinds of at most 16 rows a lane, one warp per task)
    for pers in (0, 1):
        for j in range(max(len(o) for o in opts)):
            want = [o[j % len(o)] for o in opts]
            s.ragged_set_plan([dict(b, lanes_per_system=P, cta_per_system=k, persistent=pers)
                               for b, (P, k) in zip(plan, want)])
            got = s.ragged_plan()
            assert [(b["lanes_per_system"], b["cta_per_system"]) for b in got] == want
            # in the persistent launch: CTA kinds of at most 256 threads, and the
            # warp kind of at most 16 rows a lane as its warp class
            assert [b["persistent"] for b in got] == [
                int(pers and ((k in (1, 2) and P <= 256) or
                              (k == 0 and -(-b["n_row_max"] // P) <= 16)))
                for b, (P, k) in zip(plan, want)]
            X.zero_()
            s.solve_ragged(dA, dB, dC, dD, X, off, per)
            torch.cuda.synchronize()
            assert s.status() == 0
            assert per_system_err(X.cpu().numpy(), ref, off) <= 1e-12, (pers, want)


@pytest.mark.gpu
def test_ragged_persistent_plan_bit_identical_over_repeats(cuda, orc):
    # the persistent launch (groups pulling systems from counters, then warps
    # pulling short systems) with the in-place shapes of the plan: which CTA
    # takes which system changes from run to run, the results must not
    import torch
    A, B, C, D, off, per = W.ragged_batch(2000, seed=59)
    dA, dB, dC, dD = [torch.from_numpy(v).to(cuda) for v in (A, B, C, D)]
    s = Solver("pascal", 2000, 64, 2)
    X = torch.zeros(int(off[-1]), dtype=torch.float64, device=cuda)
    s.solve_ragged(dA, dB, dC, dD, X, off, per)
    plan = [dict(b, persistent=1) for b in s.ragged_plan()]
    s.ragged_set_plan(plan)
    assert any(b["persistent"] for b in s.ragged_plan())
    outs = []
    for _ in range(4):
        X = torch.zeros(int(off[-1]), dtype=torch.float64, device=cuda)
        s.solve_ragged(dA, dB, dC, dD, X, off, per)
        torch.cuda.synchronize()
        assert s.status() == 0
        outs.append(X)
    assert all(torch.equal(o, outs[0]) for o in outs[1:])
    ref = ragged_oracle(orc, A, B, C, D, off, per)
    assert per_system_err(outs[0].cpu().numpy(), ref, off) <= 1e-12
