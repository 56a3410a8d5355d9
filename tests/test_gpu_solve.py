"""GPU parity: the CUDA kernels, called through the C ABI, against the oracle.

Bars:
  * P = 1 (serial Thomas, periodic Thomas): bit-identical to the oracle, which
    is bit-identical to the reference's tdma_many / tdma_cyclic_many.
  * PaScaL, P > 1: bit-identical to the oracle's PaScaL (itself bit-identical to
    the reference's PaScaLTDMA with nprocs = P) and within 1e-12 (relative to
    max|x|) of the serial Thomas.
  * Filtered v1/v2: bit-identical to the oracle's Filtered with the same rho
    and the device J estimator, the same J per segment, and within eps of PaScaL.
  * A, B, C are not modified; in-place and out-of-place solves agree.
"""
import numpy as np
import pytest

from filtered_tdma_b200 import FilteredTDMACUDA, PaScaLTDMACUDA, Solver, TdmaBackendGPU
from filtered_tdma_b200 import workloads as W

pytestmark = pytest.mark.gpu


def dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


def host(t):
    return t.cpu().numpy()


def run(cuda, method, A, B, C, D, P, cyclic=False, out=False, rho=None, eps_c=1e-3, flags=0):
    n_row, n_sys = D.shape
    s = Solver(method, n_sys, n_row, P, flags=flags)
    s.set_eps_constant(eps_c)
    dA, dB, dC, dD = dev(cuda, A, B, C, D)
    if rho is not None:
        import torch
        # the per-row bound goes in through set_rho on a system-0 column
        # holding exactly rho (A = -rho, B = 1, C = -rho).
        col = torch.zeros((n_row, 1), dtype=torch.float64, device=cuda)
        r = torch.from_numpy(np.ascontiguousarray(rho)).to(cuda)[:, None]
        s.set_rho(-r.contiguous(), (col + 1).contiguous(), -r.contiguous(), 1, n_row)
    if out:
        X = dD.clone().zero_()
        s.solve_out(dA, dB, dC, dD, X, cyclic=cyclic)
        import torch
        torch.cuda.synchronize()
        assert np.array_equal(host(dD), D), "out-of-place solve modified D"
        res = host(X)
    else:
        s.solve(dA, dB, dC, dD, cyclic=cyclic)
        res = host(dD)
    assert np.array_equal(host(dA), A) and np.array_equal(host(dB), B) and \
        np.array_equal(host(dC), C), "A, B or C modified"
    assert s.status() == 0
    return res, s


SHAPES_P1 = [(1, 1), (3, 2), (5, 3), (31, 17), (64, 64), (4096, 64), (1000, 129), (257, 512)]
# even n_sys and at most 128 rows: the staged kernel (c', d' in shared memory),
# including ragged last chunks and a last CTA of fewer than 32 systems
SHAPES_P1_STAGED = [(2, 1), (2, 2), (34, 3), (100, 16), (66, 17), (4096, 64), (1000, 100),
                    (262, 128), (16384, 128), (65536, 64)]


@pytest.mark.parametrize("n_sys,n_row", SHAPES_P1)
def test_thomas_bit_exact(cuda, orc, n_sys, n_row):
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=n_sys + n_row)
    x, _ = run(cuda, "pascal", A, B, C, D, 1)
    assert np.array_equal(x, orc.thomas(A, B, C, D))
    x2, _ = run(cuda, "pascal", A, B, C, D, 1, out=True)
    assert np.array_equal(x2, x)


@pytest.mark.parametrize("n_sys,n_row", SHAPES_P1_STAGED)
def test_thomas_staged_bit_exact(cuda, orc, n_sys, n_row):
    A, B, C, D = W.row_varying(n_sys, n_row, seed=n_sys + 3 * n_row)
    x, _ = run(cuda, "pascal", A, B, C, D, 1)
    assert np.array_equal(x, orc.thomas(A, B, C, D))
    x2, _ = run(cuda, "pascal", A, B, C, D, 1, out=True)
    assert np.array_equal(x2, x)


@pytest.mark.parametrize("n_sys,n_row", [(5, 3), (31, 17), (4096, 64), (257, 300)])
def test_thomas_cyclic_bit_exact(cuda, orc, n_sys, n_row):
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=7 * n_sys + n_row)
    x, _ = run(cuda, "pascal", A, B, C, D, 1, cyclic=True)
    assert np.array_equal(x, orc.thomas_cyclic(A, B, C, D))


def rel_err(x, ref):
    return np.max(np.abs(x - ref)) / np.max(np.abs(ref))


@pytest.mark.parametrize("n_sys,n_row,P", [
    (32, 64, 2), (64, 64, 4), (4096, 64, 4), (100, 96, 8), (33, 100, 7), (7, 48, 16),
    (2048, 512, 8), (96, 515, 16), (130, 37, 3), (64, 1000, 16)])
def test_pascal_reference_order_bit_exact(cuda, orc, n_sys, n_row, P):
    """Cluster kernel, reference operation order: bit-identical to PaScaLTDMA
    with nprocs = P (through the oracle, itself pinned to the reference)."""
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=P * 1000 + n_row)
    x, _ = run(cuda, "pascal", A, B, C, D, P, flags=L.FLAG_REFERENCE_ORDER)
    assert np.array_equal(x, orc.pascal(A, B, C, D, P))
    assert rel_err(x, orc.thomas(A, B, C, D)) <= 1e-12
    x2, _ = run(cuda, "pascal", A, B, C, D, P, out=True, flags=L.FLAG_REFERENCE_ORDER)
    assert np.array_equal(x2, x)


@pytest.mark.parametrize("n_sys,n_row,P", [(32, 64, 2), (100, 96, 8), (33, 100, 7),
                                           (64, 512, 16)])
def test_pascal_cyclic_reference_order_bit_exact(cuda, orc, n_sys, n_row, P):
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=P + n_row)
    x, _ = run(cuda, "pascal", A, B, C, D, P, cyclic=True, flags=L.FLAG_REFERENCE_ORDER)
    assert np.array_equal(x, orc.pascal(A, B, C, D, P, cyclic=True))
    assert rel_err(x, orc.thomas_cyclic(A, B, C, D)) <= 1e-12


# Default PaScaL: the register-tiled kernel where the shape allows it
# (n_row = 16 * nseg, nseg <= 32, even n_sys), else the cluster kernel.  Exact to
# rounding: within 1e-12 (relative to max|x|) of the serial Thomas.
@pytest.mark.parametrize("n_sys,n_row", [
    (16, 16), (32, 32), (100, 48), (4096, 64), (1000, 128), (2048, 192), (130, 256),
    (4094, 384), (2048, 512), (98, 512), (33, 64), (64, 100), (64, 1024)])
def test_pascal_default_within_1e12(cuda, orc, n_sys, n_row):
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=n_sys + 3 * n_row)
    P = 2 if n_row < 64 else 8
    x, _ = run(cuda, "pascal", A, B, C, D, P)
    assert rel_err(x, orc.thomas(A, B, C, D)) <= 1e-12
    x2, _ = run(cuda, "pascal", A, B, C, D, P, out=True)
    assert np.array_equal(x2, x)


@pytest.mark.parametrize("n_sys,n_row", [(96, 768), (64, 1024), (34, 2048), (32, 4096),
                                         (1000, 384)])
def test_pascal_default_long_systems(cuda, orc, n_sys, n_row):
    """Sub-segments split over 2-16 CTAs of a cluster (distributed shared memory)."""
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=n_row + 7)
    x, _ = run(cuda, "pascal", A, B, C, D, 8)
    assert rel_err(x, orc.thomas(A, B, C, D)) <= 1e-12


@pytest.mark.parametrize("n_sys,n_row", [(16, 16), (64, 32), (1000, 64), (256, 128),
                                         (2048, 512), (64, 1024), (40, 4096)])
def test_pascal_default_cyclic_within_1e12(cuda, orc, n_sys, n_row):
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=n_sys + n_row + 1)
    x, _ = run(cuda, "pascal", A, B, C, D, 4, cyclic=True)
    assert rel_err(x, orc.thomas_cyclic(A, B, C, D)) <= 1e-12


def test_pascal_default_weak_dominance(cuda, orc):
    # rho up to 0.499: the reduced system is barely dominant
    A, B, C, D = W.weak_dominance(512, 512, seed=3)
    x, _ = run(cuda, "pascal", A, B, C, D, 8)
    assert rel_err(x, orc.thomas(A, B, C, D)) <= 1e-12


FILTERED_SHAPES = [(64, 128, 2), (100, 96, 8), (33, 200, 5), (2048, 512, 8)]


@pytest.mark.parametrize("version", [1, 2])
@pytest.mark.parametrize("cyclic", [False, True])
@pytest.mark.parametrize("n_sys,n_row,P", FILTERED_SHAPES)
def test_filtered_bit_exact(cuda, orc, version, cyclic, n_sys, n_row, P):
    # BTDMA_FLAG_REFERENCE_ORDER: the reference's Filtered everywhere, also
    # where J reaches m - 2 (no exact fallback)
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.diag_dominant(n_sys, n_row, 0.1, 1.0, seed=version + n_row)
    rho = orc.rho_rows_all(A, B, C)
    x, s = run(cuda, f"filtered_v{version}", A, B, C, D, P, cyclic=cyclic, rho=rho,
               flags=L.FLAG_REFERENCE_ORDER)
    xo, Jo = orc.filtered(A, B, C, D, P, version, cyclic, 1e-3, rho, orc.J_DEVICE)
    assert s.last_J() == list(Jo)
    assert np.array_equal(x, xo)
    assert s.last_stats()["filtered_exact"] == 0
    # The eps bound holds when the truncation is active in every segment
    # (J < m-2); the dropped interface couplings then decay below it too.
    segs = orc.split(n_row, P)
    if max(Jo) < min(c for _, c in segs) - 2:
        xp = orc.pascal(A, B, C, D, P, cyclic)
        eps = 1e-3 / float(min(c for _, c in segs) * P) ** 2
        assert np.max(np.abs(x - xp)) <= eps


def filtered_tiled(version, n_sys, n_row, P, cyclic):
    # the default Filtered v2 solve runs on the tiled kernels when the segments
    # are whole power-of-two groups of 16-row sub-segments (at most 32) and
    # the arrays suit TMA (n_sys even here)
    if version != 2 or n_row % 16 or n_sys % 2:
        return False
    nseg = n_row // 16
    if nseg > 32 or nseg % P:
        return False
    R = nseg // P
    return R & (R - 1) == 0 and (not cyclic or nseg & (nseg - 1) == 0)


@pytest.mark.parametrize("version", [1, 2])
@pytest.mark.parametrize("cyclic", [False, True])
@pytest.mark.parametrize("n_sys,n_row,P", FILTERED_SHAPES)
def test_filtered_default_exact_fallback(cuda, orc, version, cyclic, n_sys, n_row, P):
    # default Filtered: while every segment truncates (J < m - 2), the
    # reference's scheme -- bit for bit on the segment kernels, within eps of
    # it (and of PaScaL) on the tiled kernels; the exact reduced solve (within
    # 1e-12 of the serial Thomas) as soon as one segment does not, reported by
    # last_stats
    A, B, C, D = W.diag_dominant(n_sys, n_row, 0.1, 1.0, seed=version + n_row)
    rho = orc.rho_rows_all(A, B, C)
    x, s = run(cuda, f"filtered_v{version}", A, B, C, D, P, cyclic=cyclic, rho=rho)
    xo, Jo = orc.filtered(A, B, C, D, P, version, cyclic, 1e-3, rho, orc.J_DEVICE)
    assert s.last_J() == list(Jo)
    segs = orc.split(n_row, P)
    exact = any(J >= c - 2 for J, (_, c) in zip(Jo, segs))
    assert s.last_stats()["filtered_exact"] == int(exact)
    if exact:
        xt = orc.thomas_cyclic(A, B, C, D) if cyclic else orc.thomas(A, B, C, D)
        assert rel_err(x, xt) <= 1e-12
    elif filtered_tiled(version, n_sys, n_row, P, cyclic):
        eps = 1e-3 / float(n_row) ** 2
        xp = orc.pascal(A, B, C, D, P, cyclic)
        assert np.max(np.abs(x - xp)) <= eps
        assert np.max(np.abs(x - xo)) <= 2 * eps
    else:
        assert np.array_equal(x, xo)


@pytest.mark.parametrize("cyclic", [False, True])
@pytest.mark.parametrize("n_sys,n_row,P", [(4096, 512, 8), (2048, 256, 4), (1024, 128, 2),
                                           (2048, 512, 4), (2050, 384, 6), (512, 512, 16)])
def test_filtered_v2_tiled_within_eps(cuda, orc, cyclic, n_sys, n_row, P):
    # Filtered v2 on the tiled kernels (the default where the shape allows):
    # each segment solved exactly, Filtered's 2 x 2 interfaces between them,
    # the full correction; J and the fallback decision from the reference's
    # device estimator.  Bar: within the reference's eps = eps_c / n_row^2 of
    # PaScaL, and of the reference's own Filtered result.
    if cyclic and (n_row // 16) & (n_row // 16 - 1):
        pytest.skip("periodic tiled solves need 2^k sub-segments")
    A, B, C, D = W.diag_dominant(n_sys, n_row, 0.1, 1.0, seed=40 + P + n_row)
    rho = orc.rho_rows_all(A, B, C)
    x, s = run(cuda, "filtered_v2", A, B, C, D, P, cyclic=cyclic, rho=rho)
    xo, Jo = orc.filtered(A, B, C, D, P, 2, cyclic, 1e-3, rho, orc.J_DEVICE)
    assert s.last_J() == list(Jo)
    m = n_row // P
    assert max(Jo) < m - 2  # the truncation regime: no fallback
    assert s.last_stats()["filtered_exact"] == 0
    eps = 1e-3 / float(n_row) ** 2
    xp = orc.pascal(A, B, C, D, P, cyclic)
    assert np.max(np.abs(x - xp)) <= eps
    assert np.max(np.abs(x - xo)) <= 2 * eps
    assert not np.array_equal(x, xo) or P == 1  # not the segment kernels' result


@pytest.mark.parametrize("version", [1, 2])
def test_filtered_config2_coefficients(cuda, orc, version):
    # the Filtered-vs-PaScaL shape's coefficients, r log-uniform in [0.1, 10]
    # (rho up to 0.476), 32768 x 512, P = 8 (m = 64): J clamps to m - 1 = 63 in
    # every segment.  Reference order: bit-identical to the oracle, J = 63.
    # Default: the exact fallback, within 1e-12 of the serial Thomas; the
    # reference's result is within its eps of it.
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.diag_dominant(32768, 512, seed=2)
    rho = orc.rho_rows_all(A, B, C)
    xo, Jo = orc.filtered(A, B, C, D, 8, version, False, 1e-3, rho, orc.J_DEVICE)
    assert list(Jo) == [63] * 8
    x, s = run(cuda, f"filtered_v{version}", A, B, C, D, 8, rho=rho,
               flags=L.FLAG_REFERENCE_ORDER)
    assert s.last_J() == list(Jo)
    assert np.array_equal(x, xo)
    x, s = run(cuda, f"filtered_v{version}", A, B, C, D, 8, rho=rho)
    assert s.last_stats()["filtered_exact"] == 1
    xt = orc.thomas(A, B, C, D)
    assert rel_err(x, xt) <= 1e-12
    assert np.max(np.abs(xo - xt)) <= 1e-3 / 512.0 ** 2


@pytest.mark.parametrize("cyclic", [False, True])
def test_filtered_rho_at_one_half(cuda, orc, cyclic):
    # rho = max(|A/B|, |C/B|) uniform in [0.45, 0.55] (rows still dominant): the
    # bound does not hold past 0.5; the default Filtered solve takes the exact
    # reduced system and says so, the reference order keeps the 2x2 interface
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.rho_band(4096, 512, 0.45, 0.55, seed=8)
    rho = orc.rho_rows_all(A, B, C)
    assert rho.max() >= 0.5
    xt = orc.thomas_cyclic(A, B, C, D) if cyclic else orc.thomas(A, B, C, D)
    for version in (1, 2):
        x, s = run(cuda, f"filtered_v{version}", A, B, C, D, 8, cyclic=cyclic, rho=rho)
        assert s.last_stats()["filtered_exact"] == 1
        assert rel_err(x, xt) <= 1e-12
        x, s = run(cuda, f"filtered_v{version}", A, B, C, D, 8, cyclic=cyclic, rho=rho,
                   flags=L.FLAG_REFERENCE_ORDER)
        xo, Jo = orc.filtered(A, B, C, D, 8, version, cyclic, 1e-3, rho, orc.J_DEVICE)
        assert list(Jo) == [63] * 8
        assert np.array_equal(x, xo)


def test_filtered_untileable_shape_falls_back_to_reference_order_pascal(cuda, orc):
    # odd n_sys (no TMA) and 100 rows (not a multiple of 16): the exact fallback
    # runs the reference-order PaScaL kernel, bit-identical to the oracle's
    A, B, C, D = W.diag_dominant(101, 100, 1.0, 10.0, seed=12)
    rho = orc.rho_rows_all(A, B, C)
    x, s = run(cuda, "filtered_v2", A, B, C, D, 4, rho=rho)
    assert s.last_stats()["filtered_exact"] == 1
    assert np.array_equal(x, orc.pascal(A, B, C, D, 4))


@pytest.mark.parametrize("version", [1, 2])
def test_filtered_host_j_semantics(cuda, orc, version):
    A, B, C, D = W.diag_dominant(80, 160, 0.1, 1.0, seed=42)
    rho = orc.rho_rows_all(A, B, C)
    from filtered_tdma_b200 import _lib as L
    x, s = run(cuda, f"filtered_v{version}", A, B, C, D, 4, rho=rho,
               flags=L.FLAG_J_HOST | L.FLAG_REFERENCE_ORDER)
    xo, Jo = orc.filtered(A, B, C, D, 4, version, False, 1e-3, rho, orc.J_HOST)
    assert np.array_equal(x, xo)


def test_filtered_set_rho_system0(cuda, orc):
    # set_rho reads system 0's column, like the reference's k_set_rho.
    A, B, C, D = W.diag_dominant(64, 96, seed=3)
    n_row, n_sys = D.shape
    from filtered_tdma_b200 import _lib as L
    s = Solver("filtered_v2", n_sys, n_row, 4, flags=L.FLAG_REFERENCE_ORDER)
    s.set_eps_constant(1e-3)
    dA, dB, dC, dD = dev(cuda, A, B, C, D)
    s.set_rho(dA, dB, dC)
    s.solve(dA, dB, dC, dD)
    xo, Jo = orc.filtered(A, B, C, D, 4, 2, False, 1e-3, orc.rho_rows(A, B, C, 0), orc.J_DEVICE)
    assert np.array_equal(host(dD), xo)
    assert s.last_J() == list(Jo)


def test_no_tma_path_odd_systems(cuda, orc):
    # odd n_sys: the row stride is not a multiple of 16 bytes, plain loads are used
    A, B, C, D = W.diag_dominant(101, 128, seed=9)
    from filtered_tdma_b200 import _lib as L
    x, _ = run(cuda, "pascal", A, B, C, D, 4, flags=L.FLAG_REFERENCE_ORDER)
    assert np.array_equal(x, orc.pascal(A, B, C, D, 4))
    x, _ = run(cuda, "pascal", A, B, C, D, 4)
    assert rel_err(x, orc.thomas(A, B, C, D)) <= 1e-12


def test_dropin_classes(cuda, orc):
    A, B, C, D = W.heat_sweep(4096, 64, r=1.0, seed=1)
    n_row, n_sys = D.shape
    xt = orc.thomas(A, B, C, D)
    # PaScaL with nprocs = 4 segments (config: heat 64^3, P = 4)
    dA, dB, dC, dD = dev(cuda, A, B, C, D)
    p = PaScaLTDMACUDA(n_sys, 0, 4, None)
    p.solve(dA, dB, dC, dD, n_sys, n_row)
    assert rel_err(host(dD), xt) <= 1e-12
    # TdmaBackendGPU strings
    for kind in ("pascal", "filtered", "filtered_v2"):
        dA, dB, dC, dD = dev(cuda, A, B, C, D)
        b = TdmaBackendGPU(kind, n_sys, n_row, 0, 1, None, -2, -2, 1e-3)
        b.set_rho_device(dA, dB, dC)
        b.set_eps_constant(1e-3)
        b.solve(dA, dB, dC, dD)
        assert np.array_equal(host(dD), xt)  # nprocs = 1: serial Thomas
        assert b.last_comm_ms() == 0.0 and b.last_gpu_ms() > 0.0
    # m = 16 rows per segment, J = 22 >= m - 2: the exact fallback by default,
    # the reference's Filtered bit for bit with the reference-order flag
    from filtered_tdma_b200 import _lib as L
    xo, Jo = orc.filtered(A, B, C, D, 4, 2, False, 1e-3, orc.rho_rows(A, B, C, 0), orc.J_DEVICE)
    assert min(Jo) >= 16 - 2
    for flags, want, exact in ((0, None, True), (L.FLAG_REFERENCE_ORDER, xo, False)):
        f = FilteredTDMACUDA(n_sys, n_row, 0, 4, None, -2, -2, 1e-3, flags=flags)
        dA, dB, dC, dD = dev(cuda, A, B, C, D)
        f.set_rho_device(dA, dB, dC)
        f.solve_filtered_v2(dA, dB, dC, dD)
        if exact:
            assert rel_err(host(dD), xt) <= 1e-12
        else:
            assert np.array_equal(host(dD), want)
        assert f.last_J() == Jo[0]


def test_full_size_properties(cuda):
    """262144 x 512 (the benchmark batch): PaScaL P=8 residual and agreement
    with the serial Thomas, both on the device."""
    import torch
    A, B, C, D = W.diag_dominant(262144, 512, seed=2, device=cuda)
    n_row, n_sys = D.shape
    X8 = torch.empty_like(D)
    X1 = torch.empty_like(D)
    Solver("pascal", n_sys, n_row, 8).solve_out(A, B, C, D, X8)
    Solver("pascal", n_sys, n_row, 1).solve_out(A, B, C, D, X1)
    rel = (X8 - X1).abs().max() / X1.abs().max()
    assert rel.item() <= 1e-12
    r = B * X8 - D
    r[1:] += A[1:] * X8[:-1]
    r[:-1] += C[:-1] * X8[1:]
    assert (r.abs().max() / D.abs().max()).item() <= 1e-12


# ----------------------------------------------------------------- FP32 storage
def run_f32(cuda, A, B, C, D, precision, cyclic=False, refine=None, stats=None):
    """FP32-stored inputs, FP64 solution; returns (x, widened inputs).  refine:
    (max_sweeps, eta_tol) for FP32_REFINE; stats: a dict filled with the
    refinement statistics."""
    import torch
    from filtered_tdma_b200 import _lib as L
    A32, B32, C32, D32 = [np.ascontiguousarray(x, dtype=np.float32) for x in (A, B, C, D)]
    n_row, n_sys = D.shape
    s = Solver("pascal", n_sys, n_row, 8 if n_row >= 48 else 2, precision=precision)
    if refine is not None:
        s.set_refine(*refine)
    dA, dB, dC, dD = [torch.from_numpy(x).to(cuda) for x in (A32, B32, C32, D32)]
    X = torch.zeros((n_row, n_sys), dtype=torch.float64, device=cuda)
    L.check(L.lib().btdma_solve_f32(s._h, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(),
                                    dD.data_ptr(), X.data_ptr(), n_sys, n_row, int(cyclic),
                                    torch.cuda.current_stream().cuda_stream))
    assert s.status() == 0
    if stats is not None:
        stats.update(s.last_stats())
    wid = [x.astype(np.float64) for x in (A32, B32, C32, D32)]
    return host(X), wid


@pytest.mark.parametrize("n_sys,n_row", [(64, 64), (1000, 128), (512, 256), (2048, 512),
                                         (96, 1024)])
def test_fp32_store_within_1e12(cuda, orc, n_sys, n_row):
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=n_row + 5)
    x, wid = run_f32(cuda, A, B, C, D, L.FP32_STORE)
    assert rel_err(x, orc.thomas(*wid)) <= 1e-12


def test_fp32_store_cyclic_and_weak(cuda, orc):
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.weak_dominance(1024, 512, seed=3)
    x, wid = run_f32(cuda, A, B, C, D, L.FP32_STORE)
    assert rel_err(x, orc.thomas(*wid)) <= 1e-12
    A, B, C, D = W.diag_dominant(256, 256, seed=4)
    x, wid = run_f32(cuda, A, B, C, D, L.FP32_STORE, cyclic=True)
    assert rel_err(x, orc.thomas_cyclic(*wid)) <= 1e-12


# ---------------------------------------------- FP32 storage + iterative refinement
@pytest.mark.parametrize("n_sys,n_row", [(1000, 128), (2048, 512), (96, 1024)])
def test_fp32_refine_within_1e12(cuda, orc, n_sys, n_row):
    """FP32 sweeps + FP64 residual refinement reach the FP64 solve of the widened
    values; every system converges without the fallback, in at most 3 sweeps."""
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=n_row + 6)
    st = {}
    x, wid = run_f32(cuda, A, B, C, D, L.FP32_REFINE, stats=st)
    assert rel_err(x, orc.thomas(*wid)) <= 1e-12
    assert st["n_systems"] == n_sys
    assert st["n_fallback"] == 0
    assert sum(st["converged_after"]) == n_sys
    assert st["converged_after"][0] == 0  # the FP32 solve alone is not FP64-accurate
    assert 1 <= st["sweeps"] <= 3


def test_fp32_refine_weak_dominance_needs_more_sweeps(cuda, orc):
    """rho in [0.45, 0.499] (cond(T) up to ~1e3): refinement still converges,
    with at least as many sweeps as the strongly dominant batch."""
    from filtered_tdma_b200 import _lib as L
    strong, weak = {}, {}
    A, B, C, D = W.diag_dominant(2048, 512, seed=31)
    run_f32(cuda, A, B, C, D, L.FP32_REFINE, stats=strong)
    A, B, C, D = W.weak_dominance(2048, 512, seed=32)
    x, wid = run_f32(cuda, A, B, C, D, L.FP32_REFINE, stats=weak)
    assert rel_err(x, orc.thomas(*wid)) <= 1e-12
    assert weak["n_fallback"] == 0
    assert weak["sweeps"] >= strong["sweeps"]


def test_fp32_refine_fallback(cuda, orc):
    """No sweep allowed, or an unreachable bound: every system falls back to the
    FP64-arithmetic solve, which still meets 1e-12."""
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.diag_dominant(512, 256, seed=33)
    for refine in ((0, 8 * 2.0**-53), (2, 1e-30)):
        st = {}
        x, wid = run_f32(cuda, A, B, C, D, L.FP32_REFINE, refine=refine, stats=st)
        assert rel_err(x, orc.thomas(*wid)) <= 1e-12
        assert st["n_fallback"] == 512
        assert st["sweeps"] == refine[0]


def test_fp32_refine_cyclic(cuda, orc):
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.diag_dominant(256, 256, seed=34)
    st = {}
    x, wid = run_f32(cuda, A, B, C, D, L.FP32_REFINE, cyclic=True, stats=st)
    assert rel_err(x, orc.thomas_cyclic(*wid)) <= 1e-12
    assert st["n_fallback"] == 0


# ------------------------------------------- coefficients that differ in every row
# The generators above give each system one coefficient triple; these batches
# draw A, B, C per row and system, so a kernel that takes a coefficient from the
# wrong row, sub-segment or system fails by far more than rounding.
@pytest.mark.parametrize("n_sys,n_row", [(96, 64), (1000, 129), (258, 512)])
def test_row_varying_thomas_bit_exact(cuda, orc, n_sys, n_row):
    A, B, C, D = W.row_varying(n_sys, n_row, seed=n_row)
    x, _ = run(cuda, "pascal", A, B, C, D, 1)
    assert np.array_equal(x, orc.thomas(A, B, C, D))
    x, _ = run(cuda, "pascal", A, B, C, D, 1, cyclic=True)
    assert np.array_equal(x, orc.thomas_cyclic(A, B, C, D))


@pytest.mark.parametrize("n_sys,n_row,P", [(64, 64, 4), (100, 96, 8), (64, 1000, 16)])
def test_row_varying_reference_order_bit_exact(cuda, orc, n_sys, n_row, P):
    from filtered_tdma_b200 import _lib as L
    A, B, C, D = W.row_varying(n_sys, n_row, seed=P + n_row)
    x, _ = run(cuda, "pascal", A, B, C, D, P, flags=L.FLAG_REFERENCE_ORDER)
    assert np.array_equal(x, orc.pascal(A, B, C, D, P))
    x, _ = run(cuda, "pascal", A, B, C, D, P, cyclic=True, flags=L.FLAG_REFERENCE_ORDER)
    assert np.array_equal(x, orc.pascal(A, B, C, D, P, cyclic=True))


@pytest.mark.parametrize("n_sys,n_row", [(4096, 64), (1000, 128), (130, 256), (4094, 384),
                                         (2048, 512), (96, 768), (64, 1024), (34, 2048)])
def test_row_varying_tiled_within_1e12(cuda, orc, n_sys, n_row):
    """Every tiled shape: one CTA (16 to 128 systems a CTA) and clusters."""
    A, B, C, D = W.row_varying(n_sys, n_row, seed=n_sys + n_row)
    x, _ = run(cuda, "pascal", A, B, C, D, 8)
    assert rel_err(x, orc.thomas(A, B, C, D)) <= 1e-12
    if (n_row // 16) & (n_row // 16 - 1) == 0:
        x, _ = run(cuda, "pascal", A, B, C, D, 8, cyclic=True)
        assert rel_err(x, orc.thomas_cyclic(A, B, C, D)) <= 1e-12


@pytest.mark.parametrize("precision", ["store", "refine"])
def test_row_varying_fp32(cuda, orc, precision):
    from filtered_tdma_b200 import _lib as L
    prec = L.FP32_STORE if precision == "store" else L.FP32_REFINE
    for n_sys, n_row, cyc in ((2048, 512, False), (520, 256, True), (96, 1024, False)):
        A, B, C, D = W.row_varying(n_sys, n_row, seed=n_row + 1)
        x, wid = run_f32(cuda, A, B, C, D, prec, cyclic=cyc)
        ref = orc.thomas_cyclic(*wid) if cyc else orc.thomas(*wid)
        assert rel_err(x, ref) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_tiled_solve_bit_identical_over_repeats(cuda, storage):
    # the headline kernels (the wide tiled kernel re-reads half of each group
    # through its TMA ring while warps run ahead of one another): repeated
    # solves and a fresh handle must agree bit for bit
    import torch
    from filtered_tdma_b200 import _lib as L
    n_sys, n_row = 65536, 512
    A, B, C, D = W.diag_dominant(n_sys, n_row, 0.1, 10.0, seed=2, device=cuda)
    if storage == "f32":
        A, B, C, D = [t.float() for t in (A, B, C, D)]
    outs = []
    for handle in range(2):
        s = Solver("pascal", n_sys, n_row, 8,
                   precision=L.FP32_STORE if storage == "f32" else L.FP64)
        for _ in range(3 if handle == 0 else 1):
            X = torch.empty((n_row, n_sys), dtype=torch.float64, device=cuda)
            if storage == "f32":
                s.solve_f32(A, B, C, D, X)
            else:
                s.solve_out(A, B, C, D, X)
            torch.cuda.synchronize()
            assert s.status() == 0
            outs.append(X)
    assert all(torch.equal(o, outs[0]) for o in outs[1:])
