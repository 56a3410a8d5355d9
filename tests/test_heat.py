"""Fused heat ADI step (btdma_heat_*) against the CPU restatement of the
reference's heat step, and both against the reference's published numbers.

The order-accuracy run of the reference at 32^3 (one step; pascal backend,
np = 1, apps/heat_cpu/results/order_accuracy/order_cpu_20260628_201654.txt)
reports L2 = 0.00153948 (rho = 0.25) and 0.0134171 (rho = 0.40); both the oracle
and the GPU step must reproduce those printed digits.  Field parity: the GPU
step's PaScaL sweeps differ from the oracle's serial Thomas only in operation
order, so the bar is 1e-12 relative.
"""
import numpy as np
import pytest

from oracle import heat_oracle as H

PUBLISHED = {0.25: 0.00153948, 0.40: 0.0134171}


@pytest.mark.parametrize("rho", [0.25, 0.40])
def test_oracle_reproduces_published_l2(orc, rho):
    _, l2, steps = H.run(32, rho)
    assert steps == 1
    assert float(f"{l2:.6g}") == PUBLISHED[rho]


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("rho", [0.25, 0.40])
def test_gpu_step_matches_oracle_and_published(cuda, orc, rho):
    from filtered_tdma_b200.heat import HeatADI
    h = HeatADI(32, 32, 32, rho=rho)
    th = h.field(cuda)
    assert _rel(th.cpu().numpy(), H.initial(32, 32, 32)) <= 1e-15  # device sin/cos: last bit
    h.step(th, h.steps)
    ref, l2_ref, _ = H.run(32, rho)
    assert _rel(th.cpu().numpy()[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]) <= 1e-12
    l2 = h.l2_error(th, h.steps * h.dt)
    assert abs(l2 - l2_ref) <= 1e-12 * l2_ref
    assert float(f"{l2:.6g}") == PUBLISHED[rho]


@pytest.mark.gpu
def test_gpu_steps_graph_and_eager_agree_non_cubic(cuda, orc):
    # 48 x 32 x 64 (three different sweep lengths), 3 steps
    from filtered_tdma_b200.heat import HeatADI
    dt = 0.3 / (1 - 0.6) * 2 * (2.0 / 64) ** 2
    h = HeatADI(48, 32, 64, dt=dt)
    a = h.field(cuda)
    b = a.clone()
    h.step(a, 3, graph=True)
    h.step(b, 3, graph=False)
    assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())
    ref = H.initial(48, 32, 64)
    for _ in range(3):
        ref = H.step(ref, dt)
    assert _rel(a.cpu().numpy()[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("grid", [(16, 384, 16), (16, 16, 512), (256, 16, 16), (16, 16, 256),
                                  (128, 16, 16), (32, 48, 48), (16, 16, 80)])
def test_gpu_step_long_sweeps_match_oracle(cuda, orc, grid):
    # the shared-matrix sweeps at the sub-segment counts of the 256 x 384 x 512
    # step: Y 384 rows (24 sub-segments, two per thread), Z 512 rows (32, the
    # fused right-hand side), X 256 rows (16, two 256-thread CTAs per SM); also
    # 16 and 8 sub-segments along Z and X, and odd sub-segment counts (3, 5)
    # along Z, whose theta boxes need the ring's 128-byte stage padding
    from filtered_tdma_b200.heat import HeatADI, dt_from_rho
    ix, iy, iz = grid
    dt = dt_from_rho(1.0 / 3.0, iz, option="strong")
    h = HeatADI(ix, iy, iz, dt=dt)
    th = h.field(cuda)
    h.step(th, 2)
    ref = H.initial(ix, iy, iz)
    for _ in range(2):
        ref = H.step(ref, dt)
    assert _rel(th.cpu().numpy()[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]) <= 1e-12


@pytest.mark.gpu
def test_gpu_step_benched_grid_matches_oracle(cuda, orc):
    # one step of the benched 256 x 384 x 512 grid (Z 512, Y 384, X 256 rows)
    from filtered_tdma_b200.heat import HeatADI, dt_from_rho
    ix, iy, iz = 256, 384, 512
    dt = dt_from_rho(1.0 / 3.0, iz, option="strong")
    h = HeatADI(ix, iy, iz, dt=dt)
    th = h.field(cuda)
    h.step(th, 1)
    got = th.cpu().numpy()[1:-1, 1:-1, 1:-1]
    del th
    h.close()
    ref = H.step(H.initial(ix, iy, iz), dt)[1:-1, 1:-1, 1:-1]
    assert _rel(got, ref) <= 1e-12


def test_heat_argument_checks():
    import ctypes
    from filtered_tdma_b200 import _lib as L
    h = ctypes.c_void_p()
    assert L.lib().btdma_heat_create(30, 32, 32, 1e-3, ctypes.byref(h)) == L.ERR_UNSUPPORTED
    assert L.lib().btdma_heat_create(32, 32, 32, -1.0, ctypes.byref(h)) == L.ERR_ARG
    assert L.lib().btdma_heat_step(None, None, 1, 1, None) == L.ERR_ARG


def test_timing_csv_format(tmp_path):
    from filtered_tdma_b200 import timing_csv as T
    p = str(tmp_path / "timing_513_111_pascal.csv")
    rows = [[1e-4 * (e + 1) + s for e in range(12)] for s in range(3)]
    T.write_csv(p, rows, T.meta_line(513, 513, 513, 1.25e-5, 13))
    lines = open(p).read().splitlines()
    assert lines[0] == "# grid=513x513x513, np=1 (1,1,1), dt= 1.250E-05, Nt=13, solver_kind=pascal"
    assert lines[1] == "rank,t_step,event,time_sec"
    assert lines[2] == "0,1,rhs, 1.000000000E-04"  # %16.9E, as timing_csv.hpp writes
    assert len(lines) == 2 + 3 * 12
    meta, vals = T.read_csv(p)
    assert vals[(0, 3, "tdma_x_gpu")] == rows[2][11]


@pytest.mark.gpu
def test_timing_csv_from_profiled_steps(cuda, tmp_path):
    from filtered_tdma_b200 import timing_csv as T
    p = T.profile_run(64, 48, 32, steps=3, warmup=1, path=str(tmp_path / "t.csv"))
    meta, vals = T.read_csv(p)
    assert meta.startswith("grid=65x49x33, np=1 (1,1,1)")
    assert len(vals) == 3 * 12
    for t in (1, 2, 3):
        assert vals[(0, t, "solve_z")] >= vals[(0, t, "tdma_z_gpu")] > 0
        assert vals[(0, t, "comm")] == 0.0


@pytest.mark.gpu
def test_step_bit_identical_over_repeats_and_handles(cuda):
    # the step's sweeps share shared memory between groups and warps run ahead
    # of one another: a race between them would show as runs that differ.  One
    # step on the benched sweep lengths (Z 512, Y 384 two sub-segments a
    # thread, X 256), repeated on one handle's graph and on fresh handles, must
    # come out bit for bit the same.
    import torch
    from filtered_tdma_b200.heat import HeatADI, dt_from_rho
    ix, iy, iz = 256, 384, 512
    dt = dt_from_rho(1.0 / 3.0, iz, option="strong")
    outs = []
    for handle in range(3):
        h = HeatADI(ix, iy, iz, dt=dt)
        for _ in range(2 if handle == 0 else 1):
            th = h.field(cuda)
            h.step(th, 1)
            torch.cuda.synchronize()
            outs.append(th.clone())
            del th
        h.close()
    assert all(torch.equal(o, outs[0]) for o in outs[1:])
