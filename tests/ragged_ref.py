"""Shared helper of the ragged tests: the oracle solution of a CSR batch."""
import numpy as np


def ragged_reference(orc, A, B, C, D, off, per):
    x = np.empty(int(off[-1]))
    for i in range(len(off) - 1):
        s = slice(int(off[i]), int(off[i + 1]))
        cols = [np.asarray(v[s], dtype=np.float64)[:, None] for v in (A, B, C, D)]
        x[s] = (orc.thomas_cyclic if per[i] else orc.thomas)(*cols)[:, 0]
    return x
