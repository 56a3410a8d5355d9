"""The wide-box tiled kernel (btdma_set_tile_shape(BTDMA_TILE_WIDE)) against the
narrow one and the oracle.

Both kernels run the same expressions (measured: bit-identical for FP64
storage, 1-ulp differences for FP32 storage where ptxas fuses a multiply and
an add differently); the bar between them is 1e-13 relative.
The oracle bar is the tiled path's 1e-12 relative bound to the serial Thomas
(FP32 storage: of the widened values).  Shapes cover every wide instantiation
(32, 64 and 128 systems per CTA), ragged last groups (n_sys not a multiple of
the group), non-power-of-two sub-segment counts and periodic systems, on
batches whose coefficients differ in every row and system.
"""
import numpy as np
import pytest

from filtered_tdma_b200 import Solver
from filtered_tdma_b200 import _lib as L
from filtered_tdma_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel_err(x, ref):
    return float(np.max(np.abs(x - ref)) / np.max(np.abs(ref)))


def solve_shape(cuda, arrays, precision, shape, cyclic):
    import torch
    n_row, n_sys = arrays[3].shape
    s = Solver("pascal", n_sys, n_row, 8, precision=precision)
    s.set_tile_shape(shape)
    dA, dB, dC, dD = [torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for v in arrays]
    X = torch.full((n_row, n_sys), 7.0, dtype=torch.float64, device=cuda)
    st = torch.cuda.current_stream().cuda_stream
    if precision == L.FP64:
        L.check(L.lib().btdma_solve_out(s._h, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(),
                                        dD.data_ptr(), X.data_ptr(), n_sys, n_row, int(cyclic),
                                        st))
    else:
        L.check(L.lib().btdma_solve_f32(s._h, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(),
                                        dD.data_ptr(), X.data_ptr(), n_sys, n_row, int(cyclic),
                                        st))
    torch.cuda.synchronize()
    assert s.status() == 0
    return X.cpu().numpy()


# (n_sys, n_row, cyclic): nseg = n_row / 16 in [8, 32], even
SHAPES = [
    (4096, 512, False),   # 32 systems per CTA, 128 groups
    (1000, 512, False),   # last group partly outside the batch
    (2048, 512, True),
    (1036, 384, False),   # nseg 24: W = 32 lanes for 24 sub-segments
    (4096, 256, False),   # 64 systems per CTA
    (520, 256, True),
    (1000, 160, False),   # nseg 10, 64 systems per CTA, 320 threads
    (4096, 128, False),   # 128 systems per CTA
    (1028, 128, True),
]


@pytest.mark.parametrize("n_sys,n_row,cyclic", SHAPES)
@pytest.mark.parametrize("precision", [L.FP64, L.FP32_STORE])
def test_wide_equals_narrow_and_oracle(cuda, orc, n_sys, n_row, cyclic, precision):
    A, B, C, D = W.row_varying(n_sys, n_row, seed=n_sys + n_row + int(cyclic))
    if precision == L.FP32_STORE:
        arrays = [np.ascontiguousarray(v, dtype=np.float32) for v in (A, B, C, D)]
    else:
        arrays = [A, B, C, D]
    xw = solve_shape(cuda, arrays, precision, L.TILE_WIDE, cyclic)
    xn = solve_shape(cuda, arrays, precision, L.TILE_NARROW, cyclic)
    assert rel_err(xw, xn) <= 1e-13
    wid = [v.astype(np.float64) for v in arrays]
    ref = orc.thomas_cyclic(*wid) if cyclic else orc.thomas(*wid)
    assert rel_err(xw, ref) <= 1e-12


def test_wide_weak_dominance_fp32(cuda, orc):
    # rho up to 0.499: the reduced systems are barely dominant
    A, B, C, D = W.weak_dominance(2048, 512, seed=11)
    arrays = [np.ascontiguousarray(v, dtype=np.float32) for v in (A, B, C, D)]
    xw = solve_shape(cuda, arrays, L.FP32_STORE, L.TILE_WIDE, False)
    xn = solve_shape(cuda, arrays, L.FP32_STORE, L.TILE_NARROW, False)
    assert rel_err(xw, xn) <= 1e-13
    assert rel_err(xw, orc.thomas(*[v.astype(np.float64) for v in arrays])) <= 1e-12


def test_wide_shape_outside_its_range_uses_narrow(cuda, orc):
    # nseg = 4 and nseg = 64 are not wide shapes: the request falls back to the
    # narrow / cluster kernels with the same results
    for n_sys, n_row in [(512, 64), (64, 1024)]:
        A, B, C, D = W.row_varying(n_sys, n_row, seed=n_row)
        xw = solve_shape(cuda, [A, B, C, D], L.FP64, L.TILE_WIDE, False)
        xn = solve_shape(cuda, [A, B, C, D], L.FP64, L.TILE_NARROW, False)
        assert np.array_equal(xw, xn)  # the same kernel ran
        assert rel_err(xw, orc.thomas(A, B, C, D)) <= 1e-12
