"""The C++ drop-in layer (include/btdma.hpp) used the way a reference caller
would: tests/cpp/dropin_main.cpp is compiled with g++ against the header and
linked with libbtdma.so (CPU test), then run on a GPU and its solutions
compared with the oracle (GPU test)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(out_dir):
    exe = os.path.join(out_dir, "dropin_main")
    lib_dir = os.path.join(ROOT, "filtered_tdma_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp"),
           "-o", exe, "-L" + lib_dir, "-lbtdma", "-Wl,-rpath," + lib_dir,
           "-L" + os.path.join(CUDA, "lib64"), "-lcudart"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_dropin_compiles(tmp_path):
    assert os.path.exists(_build(str(tmp_path)))


@pytest.mark.gpu
def test_cpp_dropin_runs_and_matches_oracle(cuda, orc, tmp_path):
    exe = _build(str(tmp_path))
    d_path = str(tmp_path / "d.bin")
    prefix = str(tmp_path / "x")
    out = subprocess.run([exe, d_path, prefix], check=True, capture_output=True, text=True).stdout
    lines = dict(line.split(None, 1) for line in out.strip().splitlines())
    n_sys, n_row = 4096, 64
    D = np.fromfile(d_path, dtype=np.float64).reshape(n_row, n_sys)
    A = np.full_like(D, -1.0)
    C = np.full_like(D, -1.0)
    B = np.full_like(D, 3.0)

    def got(name):
        return np.fromfile(f"{prefix}_{name}.bin", dtype=np.float64).reshape(n_row, n_sys)

    xt = orc.thomas(A, B, C, D)
    assert np.array_equal(got("pascal_p1"), xt)  # serial Thomas: bit-identical
    assert np.max(np.abs(got("pascal") - xt)) / np.max(np.abs(xt)) <= 1e-12
    rho = orc.rho_rows(A, B, C, sys=0)
    # m = 16 rows per segment and J = 22 >= m - 2: the default Filtered solves
    # take the exact reduced system; with the reference-order flag the
    # reference's Filtered runs, bit for bit
    for name, version, cyc in (("filtered", 1, False), ("filtered_v2", 2, False),
                               ("filtered_v2_cyclic", 2, True)):
        x, J = orc.filtered(A, B, C, D, 4, version=version, cyclic=cyc, eps_constant=1e-3,
                            rho_row=rho)
        assert min(J) >= 16 - 2
        want = orc.thomas_cyclic(A, B, C, D) if cyc else xt
        assert np.max(np.abs(got(name) - want)) / np.max(np.abs(want)) <= 1e-12, name
    x, _ = orc.filtered(A, B, C, D, 4, version=2, cyclic=False, eps_constant=1e-3, rho_row=rho)
    assert np.array_equal(got("filtered_v2_reference"), x)
    assert float(lines["heat_l2"]) == pytest.approx(0.00153948, abs=5e-9)
    assert float(lines["ragged_periodic_x"]) == pytest.approx(0.5, rel=1e-13)
    # the same values as 512 systems x 512 rows through both tiled kernel shapes
    D5 = D.reshape(512, 512)
    A5, B5, C5 = (np.full_like(D5, v) for v in (-1.0, 3.0, -1.0))
    x5 = orc.thomas(A5, B5, C5, D5)
    w = np.fromfile(f"{prefix}_pascal512_wide.bin", dtype=np.float64).reshape(512, 512)
    nw = np.fromfile(f"{prefix}_pascal512_narrow.bin", dtype=np.float64).reshape(512, 512)
    for x in (w, nw):
        assert np.max(np.abs(x - x5)) / np.max(np.abs(x5)) <= 1e-12
    assert np.max(np.abs(w - nw)) / np.max(np.abs(x5)) <= 1e-13
