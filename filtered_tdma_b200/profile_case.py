"""Run one solve configuration a few times (the command the ncu summaries in
profiles/ were captured from).

    python -m filtered_tdma_b200.profile_case --method pascal --P 8 \
        --n-sys 32768 --n-row 512 --reps 3

Inputs: per-system r log-uniform in [0.1, 10] (A = C = -r, B = 1 + 2r), D
uniform in [-1, 1], generated on the device.  Prints the CUDA-event time of
each solve and the algorithmic HBM rate (40 B/row for FP64 storage, 24 B/row for
FP32 storage).
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
    ap.add_argument("--storage", choices=["f64", "f32"], default="f64",
                    help="f32: A, B, C, D stored in FP32 (FP32_STORE handle)")
    args = ap.parse_args()

    import torch

    from filtered_tdma_b200 import Solver
    from filtered_tdma_b200 import _lib as L
    from filtered_tdma_b200 import workloads as W

    dev = torch.device("cuda:0")
    A, B, C, D = W.diag_dominant(args.n_sys, args.n_row, seed=2, device=dev)
    X = torch.empty_like(D)
    f32 = args.storage == "f32"
    if f32:
        A, B, C, D = [t.float() for t in (A, B, C, D)]
    s = Solver(args.method, args.n_sys, args.n_row, args.P,
               precision=L.FP32_STORE if f32 else L.FP64)
    if args.method != "pascal":
        s.set_eps_constant(1e-3)
        s.set_rho(A, B, C, all_systems=True)
    rows = args.n_sys * args.n_row
    bpr = 24 if f32 else 40
    for r in range(args.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if f32:
            s.solve_f32(A, B, C, D, X, cyclic=args.cyclic)
        else:
            s.solve_out(A, B, C, D, X, cyclic=args.cyclic)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        print(f"rep {r}: {ms:.4f} ms  {rows / ms / 1e6:.3e} rows/s  "
              f"{bpr * rows / ms / 1e6:.1f} GB/s ({bpr} B/row)")
    if s.status() != 0:
        raise SystemExit("device status word set")


if __name__ == "__main__":
    main()
