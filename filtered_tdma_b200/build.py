"""Build the CUDA library in-tree: filtered_tdma_b200/libbtdma.so (sm_100a only).

    python -m filtered_tdma_b200.build

nvcc cross-compiles for sm_100a without a GPU.  The CUDA runtime is linked
statically, so the library does not depend on which libcudart the host process
(e.g. PyTorch) has loaded; the driver entry point for tensor-map encoding is
resolved at run time through cudaGetDriverEntryPoint.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libbtdma.so")
SOURCES = [os.path.join(PKG, "csrc", f) for f in ("btdma_api.cu", "btdma_ragged.cu", "btdma_apps.cu")]
DEPS = SOURCES + [os.path.join(PKG, "csrc", f) for f in os.listdir(os.path.join(PKG, "csrc"))] + [
    os.path.join(ROOT, "include", "btdma.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-Wall",
    "-shared", "-cudart", "static",
    "-Xlinker", "--exclude-libs=ALL",  # keep the static runtime's symbols private
    "-I" + os.path.join(ROOT, "include"),
]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in DEPS if os.path.exists(f))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit to an object in parallel, then link."""
    if force or stale():
        from concurrent.futures import ThreadPoolExecutor
        obj_dir = os.path.join(PKG, "_build")
        os.makedirs(obj_dir, exist_ok=True)
        compile_flags = [f for f in NVCC_FLAGS if f not in ("-shared",)]
        compile_flags = [f for f in compile_flags if f not in ("-cudart", "static")]
        compile_flags = [f for f in compile_flags
                         if f not in ("-Xlinker", "--exclude-libs=ALL")]

        def one(src):
            obj = os.path.join(obj_dir, os.path.basename(src).replace(".cu", ".o"))
            cmd = ["nvcc", *compile_flags, "-c", "-o", obj, src]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            return obj

        with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
            objs = list(ex.map(one, SOURCES))
        link = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart",
                "static", "-Xlinker", "--exclude-libs=ALL", "-o", LIB, *objs]
        subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
