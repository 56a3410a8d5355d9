"""The C-ABI library loads and exports every symbol include/btdma.h declares,
and its host-side argument checks work without a GPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "btdma.h")).read()
    return sorted(set(re.findall(r"\b(btdma_[a-z_A-Z0-9]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from filtered_tdma_b200 import _lib
    from filtered_tdma_b200.build import build
    build()
    return _lib.lib()


def test_exports_every_declared_symbol(lib):
    from filtered_tdma_b200 import _lib
    syms = header_symbols()
    assert set(syms) == set(_lib.EXPORTS)
    for s in syms:
        assert hasattr(lib, s), s


def _create(lib, method, n_sys, n_row, P, precision=0, flags=0):
    h = ctypes.c_void_p()
    rc = lib.btdma_create(method, n_sys, n_row, P, precision, flags, ctypes.byref(h))
    return rc, h


def test_argument_checks(lib):
    from filtered_tdma_b200 import _lib as L
    assert _create(lib, 7, 10, 10, 1)[0] == L.ERR_ARG
    assert _create(lib, 0, 0, 10, 1)[0] == L.ERR_ARG
    assert _create(lib, 0, 10, 10, -1)[0] == L.ERR_ARG
    assert _create(lib, 0, 10, 8, 4)[0] == L.ERR_SEGMENT      # 2-row segments
    assert _create(lib, 0, 10, 4096, 17)[0] == L.ERR_UNSUPPORTED  # above the cluster limit
    assert lib.btdma_solve(None, None, None, None, None, 1, 1, None) == L.ERR_ARG
    assert b"null" in lib.btdma_last_error()
    assert lib.btdma_set_refine(None, 3, 1e-15) == L.ERR_ARG
    assert lib.btdma_last_stats(None, None) == L.ERR_ARG
    assert lib.btdma_set_tile_shape(None, L.TILE_WIDE) == L.ERR_ARG


def test_stats_struct_layout():
    # btdma_stats: n_systems, sweeps, converged_after[BTDMA_REFINE_MAX_SWEEPS + 1],
    # n_fallback, filtered_exact
    import os
    import re
    from filtered_tdma_b200 import _lib as L
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "btdma.h")).read()
    m = re.search(r"#define BTDMA_REFINE_MAX_SWEEPS (\d+)", hdr)
    assert m and int(m.group(1)) == L.REFINE_MAX_SWEEPS
    assert ctypes.sizeof(L.Stats) == 4 * (4 + L.REFINE_MAX_SWEEPS + 1)
    fields = re.search(r"typedef struct btdma_stats \{(.*?)\} btdma_stats;", hdr, re.S).group(1)
    names = re.findall(r"int (\w+)", re.sub(r"/\*.*?\*/", "", fields, flags=re.S))
    assert names == [f[0] for f in L.Stats._fields_]


def test_backend_strings():
    from filtered_tdma_b200 import TdmaBackendGPU
    K = TdmaBackendGPU.Kind
    assert TdmaBackendGPU.parse("pascal") == K.PASCAL
    assert TdmaBackendGPU.parse("PaScaL_TDMA") == K.PASCAL
    assert TdmaBackendGPU.parse("filtered_v2") == K.FILTERED_V2
    assert TdmaBackendGPU.parse("Filtered_V2") == K.FILTERED_V2
    for s in ("filtered", "filtered_v1", "filtered_tdma", "anything"):
        assert TdmaBackendGPU.parse(s) == K.FILTERED


def test_segment_split_matches_para_range(orc):
    # The kernels' seg_range and the oracle's split are the reference's
    # para_range over [0, n_row).
    for n, P in [(512, 8), (100, 7), (37, 3), (4096, 16)]:
        segs = orc.split(n, P)
        assert sum(c for _, c in segs) == n
        assert segs[0][0] == 0
        for (f0, c0), (f1, _) in zip(segs, segs[1:]):
            assert f1 == f0 + c0
        assert max(c for _, c in segs) - min(c for _, c in segs) <= 1
