"""HBM bandwidth of the row-interleaved layout versus contiguous piece width.

    python -m filtered_tdma_b200.width_probe [n_sys] [n_row]

Runs the probe built from csrc/width_probe.cu (filtered_tdma_b200/_width_probe,
compiled by build.py): streams four [n_row x n_sys] input arrays (FP32 and FP64)
and one FP64 output in row pieces of 64, 128, 256 and 512 bytes and prints one
JSON object per case.  The tiled solver reads rows in pieces of
(systems per CTA) x (element size) bytes, so the line with its piece width is
the bandwidth ceiling of that access pattern.
"""
from __future__ import annotations

import subprocess
import sys

from .build import PROBE, build_probe


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    build_probe()
    return subprocess.run([PROBE, *argv]).returncode


if __name__ == "__main__":
    raise SystemExit(main())
