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
    ap.add_argument("--case", choices=["batch", "ragged", "heat", "poisson", "momentum"],
                    default="batch",
                    help="batch: uniform [n_row x n_sys] solve; ragged: 10000 CSR systems "
                         "(n log-uniform 16..4096, autotuned); heat: fused ADI steps on "
                         "--heat-grid; poisson: channel wall-normal solve 128 x 65 x 192; "
                         "momentum: channel momentum ADI (z, y, x sweeps) of one velocity "
                         "component on 256^3")
    ap.add_argument("--heat-grid", default="256,384,512")
    ap.add_argument("--no-tune", action="store_true", help="ragged: keep the default plan")
    ap.add_argument("--tile-shape", choices=["auto", "narrow", "wide"], default="auto",
                    help="batch: kernel shape of the tiled PaScaL solve")
    args = ap.parse_args()
    if args.case != "batch":
        return other_case(args)

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
    s.set_tile_shape({"auto": L.TILE_AUTO, "narrow": L.TILE_NARROW,
                      "wide": L.TILE_WIDE}[args.tile_shape])
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
        print(f"rep {r}: {ms:.4f} ms  {rows / ms / 1e6:.2f} G rows/s  "
              f"{bpr * rows / ms / 1e6:.1f} GB/s ({bpr} B/row)")
    if s.status() != 0:
        raise SystemExit("device status word set")


def other_case(args):
    import numpy as np
    import torch

    from filtered_tdma_b200 import Solver
    from filtered_tdma_b200 import _lib as L
    from filtered_tdma_b200 import workloads as W

    dev = torch.device("cuda:0")

    def timed(fn, reps):
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return out

    if args.case == "ragged":
        f32 = args.storage == "f32"
        A, B, C, D, off, per = W.ragged_batch(10000, seed=5,
                                              dtype=np.float32 if f32 else np.float64)
        dA, dB, dC, dD = [torch.from_numpy(v).to(dev) for v in (A, B, C, D)]
        X = torch.empty(int(off[-1]), dtype=torch.float64, device=dev)
        s = Solver("pascal", 10000, 64, 2, precision=L.FP32_STORE if f32 else L.FP64)
        if not args.no_tune:
            s.ragged_autotune(dA, dB, dC, dD, X, off, per)
        ms = timed(lambda: s.solve_ragged(dA, dB, dC, dD, X, off, per), args.reps)
        print("ragged", ["%.4f ms" % t for t in ms], int(off[-1]), "rows")
    elif args.case == "heat":
        from filtered_tdma_b200.heat import HeatADI, dt_from_rho
        ix, iy, iz = (int(v) for v in args.heat_grid.split(","))
        h = HeatADI(ix, iy, iz, dt=dt_from_rho(1.0 / 3.0, iz, option="strong"))
        th = h.field(dev)
        ms = timed(lambda: h.step(th, 1), args.reps)
        print("heat step", ["%.4f ms" % t for t in ms], ix * iy * iz, "cells")
    elif args.case == "momentum":
        from filtered_tdma_b200.momentum import ChannelMomentum
        mm = ChannelMomentum(256, 256, 256, gamma3=1.5)
        rhs = torch.rand(mm.shape, dtype=torch.float64, device=dev)
        q = torch.zeros_like(rhs)
        c_visc = 0.5 * (1.0 / 180.0) * 1e-3  # as bench.py
        ms = timed(lambda: mm.adi(0, rhs, q, c_visc), args.reps)
        print("momentum component", ["%.4f ms" % t for t in ms], "status", mm.status())
    else:
        from filtered_tdma_b200.poisson import ChannelPoisson
        cp = ChannelPoisson(128, 128, 192, gamma=2.0)
        hat = torch.complex(torch.rand((192, cp.n_modes), dtype=torch.float64, device=dev),
                            torch.rand((192, cp.n_modes), dtype=torch.float64, device=dev))
        ms = timed(lambda: cp.solve(hat), args.reps)
        print("poisson", ["%.4f ms" % t for t in ms], cp.n_modes, "modes")


if __name__ == "__main__":
    main()
