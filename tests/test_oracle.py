"""The oracle is pinned before it is trusted.

1. Against the golden vectors produced by the reference's own CPU library
   (tests/golden/ref_vectors.npz, made by tests/golden/make_golden.py): the
   restatement must reproduce them bit for bit.
2. Against the reference build itself (oracle/_ref/libref.so) on fresh seeded
   shapes, when that build is present.
3. Self-consistency: PaScaL at P > 1 within 1e-12 of the serial Thomas; Filtered
   within its eps bound of PaScaL when rho is estimated conservatively.
"""
import os

import numpy as np
import pytest

from filtered_tdma_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_vectors.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _inputs(gold, name):
    return [gold[f"{name}/{k}"] for k in "ABCD"]


@pytest.mark.parametrize("name", ["dd", "heat", "odd"])
def test_golden_thomas(orc, gold, name):
    A, B, C, D = _inputs(gold, name)
    assert np.array_equal(orc.thomas(A, B, C, D), gold[f"{name}/thomas"])
    assert np.array_equal(orc.thomas_cyclic(A, B, C, D), gold[f"{name}/thomas_cyclic"])


@pytest.mark.parametrize("name", ["dd", "heat", "odd"])
def test_golden_pascal_and_filtered(orc, gold, name):
    A, B, C, D = _inputs(gold, name)
    checked = 0
    for P in (2, 3, 4, 8):
        key = f"{name}/pascal_P{P}"
        if key not in gold:
            continue
        assert np.array_equal(orc.pascal(A, B, C, D, P), gold[key])
        assert np.array_equal(orc.pascal(A, B, C, D, P, cyclic=True),
                              gold[f"{name}/pascal_cyclic_P{P}"])
        rho = orc.rho_rows(A, B, C, sys=0)
        for v in (1, 2):
            for cyc in (False, True):
                x, _ = orc.filtered(A, B, C, D, P, version=v, cyclic=cyc, eps_constant=1e-3,
                                    rho_row=rho, jmode=orc.J_HOST)
                tag = f"{name}/filtered_v{v}{'_cyclic' if cyc else ''}_P{P}"
                assert np.array_equal(x, gold[tag]), tag
        checked += 1
    assert checked > 0


needs_ref = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                                    "libref.so")),
    reason="reference build oracle/_ref not present")


@needs_ref
@pytest.mark.parametrize("n_sys,n_row,seed", [(1, 3, 1), (7, 17, 2), (64, 100, 3), (33, 513, 4)])
def test_ref_serial(orc, n_sys, n_row, seed):
    A, B, C, D = W.diag_dominant(n_sys, n_row, seed=seed)
    assert np.array_equal(orc.thomas(A, B, C, D), orc.ref_thomas(A, B, C, D))
    assert np.array_equal(orc.thomas(A, B, C, D), orc.ref_thomas(A, B, C, D, filtered_copy=True))
    assert np.array_equal(orc.thomas_cyclic(A, B, C, D), orc.ref_thomas_cyclic(A, B, C, D))


@needs_ref
@pytest.mark.parametrize("P", [2, 3, 5, 8, 16])
def test_ref_pascal(orc, P):
    A, B, C, D = W.diag_dominant(29, 16 * P + 5, seed=P)
    for cyc in (False, True):
        assert np.array_equal(orc.pascal(A, B, C, D, P, cyc), orc.ref_pascal(A, B, C, D, P, cyc))


@needs_ref
@pytest.mark.parametrize("P", [2, 3, 4, 8])
@pytest.mark.parametrize("version", [1, 2])
def test_ref_filtered(orc, P, version):
    A, B, C, D = W.diag_dominant(21, 24 * P + 3, seed=10 + P)
    rho = orc.rho_rows(A, B, C, sys=0)
    for cyc in (False, True):
        x, J = orc.filtered(A, B, C, D, P, version, cyc, 1e-3, rho, orc.J_HOST)
        xr = orc.ref_filtered(A, B, C, D, P, version, cyc, 1e-3)
        assert np.array_equal(x, xr)


def test_pascal_close_to_thomas(orc):
    A, B, C, D = W.diag_dominant(50, 256, seed=5)
    xt = orc.thomas(A, B, C, D)
    for P in (2, 4, 8, 16):
        xp = orc.pascal(A, B, C, D, P)
        assert np.max(np.abs(xp - xt)) <= 1e-12 * np.max(np.abs(xt))


def test_filtered_within_eps_of_pascal(orc):
    # Conservative rho (max over all systems): the truncation and the dropped
    # interface couplings stay below eps = eps_c/(m P)^2 per segment.
    A, B, C, D = W.diag_dominant(40, 512, 0.1, 2.0, seed=6)
    rho = orc.rho_rows_all(A, B, C)
    P, eps_c = 8, 1e-3
    xp = orc.pascal(A, B, C, D, P)
    for v in (1, 2):
        x, J = orc.filtered(A, B, C, D, P, v, False, eps_c, rho, orc.J_DEVICE)
        eps = eps_c / (512.0 ** 2)
        assert np.max(np.abs(x - xp)) <= eps, (v, J)


def test_pascal_two_row_segments_rejected(orc):
    A, B, C, D = W.diag_dominant(4, 8, seed=1)
    with pytest.raises(ValueError):
        orc.pascal(A, B, C, D, 4)


@needs_ref
def test_reference_pascal_two_row_segments_is_wrong(orc):
    # Documents why segments need >= 3 rows: the reference's row-0 reduction
    # treats row 1 as interior, so with 2-row segments its PaScaL is not exact.
    A, B, C, D = W.diag_dominant(8, 8, seed=5)
    err = np.max(np.abs(orc.ref_pascal(A, B, C, D, 4) - orc.thomas(A, B, C, D)))
    assert err > 1e-3
