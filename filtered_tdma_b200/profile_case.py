"""Run one solve configuration a few times (the command the ncu summaries in
profiles/ were captured from).

    python -m filtered_tdma_b200.profile_case --method pascal --P 8 \
        --n-sys 32768 --n-row 512 --reps 3

Inputs: per-system r log-uniform in [0.1, 10] (A = C = -r, B = 1 + 2r), D
uniform in [-1, 1], generated on the device.  Prints the CUDA-event time of
each solve and the algorithmic HBM rate (40 B/row for FP64 storage).
"""
from __future__ import annotations

import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--method", default="pascal")
    ap.add_argument("--P", type=int, default=8)
    ap.add_argument("--n-sys", type=int, default=32768)
    ap.add_argument("--n-row", type=int, default=512)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--cyclic", action="store_true")
    args = ap.parse_args()

    import torch

    from filtered_tdma_b200 import Solver
    from filtered_tdma_b200 import workloads as W

    dev = torch.device("cuda:0")
    A, B, C, D = W.diag_dominant(args.n_sys, args.n_row, seed=2, device=dev)
    X = torch.empty_like(D)
    s = Solver(args.method, args.n_sys, args.n_row, args.P)
    if args.method != "pascal":
        s.set_eps_constant(1e-3)
        s.set_rho(A, B, C, all_systems=True)
    rows = args.n_sys * args.n_row
    for r in range(args.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s.solve_out(A, B, C, D, X, cyclic=args.cyclic)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        print(f"rep {r}: {ms:.4f} ms  {rows / ms / 1e6:.3e} rows/s  "
              f"{40 * rows / ms / 1e6:.1f} GB/s (40 B/row)")
    if s.status() != 0:
        raise SystemExit("device status word set")


if __name__ == "__main__":
    main()
