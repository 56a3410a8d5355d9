"""Generate tests/golden/ref_vectors.npz from the reference's own CPU library.

Run where the reference sources exist, with BTDMA_REFERENCE_DIR naming their
root (``make -C oracle ref REF=<dir>`` builds oracle/_ref/libref.so from them):

    BTDMA_REFERENCE_DIR=<reference root> python tests/golden/make_golden.py

Every output in the file was produced by the reference's code (tdma_many,
tdma_cyclic_many, PaScaLTDMA::solve[_cyclic], FilteredTDMA::solve_[cycl_]
filtered_v{1,2} with thread ranks); the inputs are seeded synthetic batches.
The tests pin the oracle to these vectors so it stays checked on machines
without the reference.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from filtered_tdma_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    O.build(with_ref=True)
    out = {}
    cases = {
        "dd": W.diag_dominant(37, 48, seed=11),       # per-system r in [0.1, 10]
        "heat": W.heat_sweep(16, 64, r=1.0, seed=1),  # heat 64-row sweep, rho = 1/3
        "odd": W.diag_dominant(5, 37, 0.05, 0.5, seed=12),
    }
    for name, (A, B, C, D) in cases.items():
        for k, v in zip("ABCD", (A, B, C, D)):
            out[f"{name}/{k}"] = v
        out[f"{name}/thomas"] = O.ref_thomas(A, B, C, D)
        out[f"{name}/thomas_cyclic"] = O.ref_thomas_cyclic(A, B, C, D)
        n_row = D.shape[0]
        for P in (2, 3, 4, 8):
            if n_row // P < 3:
                continue
            out[f"{name}/pascal_P{P}"] = O.ref_pascal(A, B, C, D, P)
            out[f"{name}/pascal_cyclic_P{P}"] = O.ref_pascal(A, B, C, D, P, cyclic=True)
            for v in (1, 2):
                for cyc in (False, True):
                    tag = f"{name}/filtered_v{v}{'_cyclic' if cyc else ''}_P{P}"
                    out[tag] = O.ref_filtered(A, B, C, D, P, version=v, cyclic=cyc,
                                              eps_constant=1e-3)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_vectors.npz")
    np.savez_compressed(path, **out)
    print(path, len(out), "arrays")


if __name__ == "__main__":
    main()
