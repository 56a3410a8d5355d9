"""Benchmark of the batched tridiagonal solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step = one solve of one batch, inputs resident in HBM):
  262144 systems x 512 rows, FP64, A = C = -r, B = 1 + 2r with per-system r
  log-uniform in [0.1, 10], D uniform in [-1, 1] (the reference's Filtered-vs-
  PaScaL comparison shape), solved by PaScaL with P = 8 segments per system.
  A, B, C, D are 4.3 GB, far above the 126 MB L2, so no flush is needed between
  steps.  Under torchrun every rank solves its own batch (systems are
  independent: weak scaling, no collective on the data path).

Printed by rank 0: one JSON line with value = rows/s over all ranks (device
time, max over ranks), the roofline of the dominant kernel, the CPU baseline
(the reference's own CPU library on this host's cores), an end-to-end figure
through the public API with host buffers, the SM clocks seen during the timed
region and the other solve variants on the same batch.

``--impl reference`` times the reference's CPU implementation (PaScaLTDMA with
one thread rank per host core, built from its sources into oracle/_ref) on a
bounded sample of the same workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "rows/s & HBM GB/s: FP32+refine vs plain FP64 at ≤1e-12 rel err, 1 B200"
N_SYS, N_ROW, P = 262144, 512, 8
BYTES_PER_ROW_F64 = 40  # read A, B, C, D + write x, FP64
WORKLOAD = ("262144 systems x 512 rows FP64, per-system r log-uniform [0.1,10] "
            "(A=C=-r, B=1+2r), D uniform [-1,1]; PaScaL, 8 segments per system")


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (no MEASURED_PEAKS.json)"


def ncu_traffic(kernel_tag):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"{kernel_tag}.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """SM clock and throttle-reason samples taken DURING a timed region.

    NVML is polled from a thread every millisecond between start() and stop()
    (a solve step lasts about a millisecond, so nvidia-smi's 200 ms loop would
    miss short regions); nvidia-smi one-shot queries are the fallback when NVML
    cannot be loaded.  Reason names follow nvidia-smi's clocks_event_reasons."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4),
               ("hw_power_brake_slowdown", 0x80))

    def __init__(self, torch_device):
        self.dev = torch_device
        self.sm, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._ready = threading.Event()
        self._t = None
        self._nvml = None
        self._h = None

    def _open(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            try:
                self._h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
            except Exception:
                self._h = pynvml.nvmlDeviceGetHandleByIndex(self.dev.index or 0)
            self._nvml = pynvml
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self._nvml = None

    def _sample(self):
        if self._nvml is not None:
            n = self._nvml
            self.sm.append(float(n.nvmlDeviceGetClockInfo(self._h, n.NVML_CLOCK_SM)))
            mask = int(n.nvmlDeviceGetCurrentClocksEventReasons(self._h))
            for name, bit in self.REASONS:
                if mask & bit:
                    self.reasons.add(name)
            return
        out = subprocess.run(
            ["nvidia-smi", "-i", str(self.dev.index or 0),
             "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits"],
            capture_output=True, text=True, timeout=10).stdout.strip().split(",")
        if len(out) >= 6:
            self.sm.append(float(out[0]))
            self.max_mhz = float(out[1])
            for (name, _), v in zip(self.REASONS, out[2:6]):
                if v.strip().lower() == "active":
                    self.reasons.add(name)

    def _run(self):
        while True:
            try:
                self._sample()
            except Exception:
                pass
            self._ready.set()
            if self._stop.wait(0.001):
                break

    def start(self):
        self._open()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        self._ready.wait(timeout=10)  # first sample taken before the region starts

    def stop(self):
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=10)
        try:
            self._sample()  # at least one sample at the end of the region
        except Exception:
            pass

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.sm),
                "source": "nvml" if self._nvml is not None else "nvidia-smi"}


def cpu_reference_rate(sample_sys, reps, warm=1):
    """rows/s of the reference's CPU PaScaL on this host (thread ranks = cores),
    or of the oracle's single-thread restatement when the reference build is absent."""
    import numpy as np
    from filtered_tdma_b200 import workloads as W
    from oracle import oracle as O
    A, B, C, D = W.diag_dominant(sample_sys, N_ROW, seed=2)
    rows = sample_sys * N_ROW
    cores = len(os.sched_getaffinity(0))
    if O.ref_available():
        nprocs = max(1, min(cores, N_ROW // 3))
        t = O.ref_time_solve(A, B, C, D, nprocs, "pascal", reps=warm + reps)[warm:]
        kind, used = "reference", nprocs
        desc = (f"reference PaScaLTDMA::solve (libs/pascal_tdma/cpu/pascal_tdma.cpp) with "
                f"{nprocs} thread ranks, {sample_sys} systems x {N_ROW} rows, median of {reps}")
    else:
        ts = []
        for _ in range(warm + reps):
            t0 = time.perf_counter()
            O.pascal(A, B, C, D, P)
            ts.append(time.perf_counter() - t0)
        t = ts[warm:]
        kind, used = "port", 1
        desc = f"oracle PaScaL restatement, 1 thread, {sample_sys} x {N_ROW}, median of {reps}"
    med = float(np.median(t))
    return rows / med, kind, used, desc, t


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps_rate = []
    rate0 = None
    kind = used = desc = None
    sample = 16384
    for i in range(args.warmup + args.steps):
        rate, kind, used, desc, _ = cpu_reference_rate(sample, reps=1, warm=0)
        if i >= args.warmup:
            steps_rate.append(rate)
        rate0 = rate
    value = statistics.median(steps_rate) if steps_rate else rate0
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sample * N_ROW / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_sys": N_SYS, "n_row": N_ROW, "P": P,
                   "method": "pascal", "sample_systems": sample},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": used, "kind": kind,
                         "sample": desc},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def reference_gpu_leg(torch, A, B, C, D, rows, peak, reps, ours):
    """Time the reference's GPU kernels (tdma_many_cuda at P = 1, PaScaL and
    Filtered v2 with 8 ranks) on the headline batch: CUDA events around each
    solve, inputs restored from pristine copies between solves."""
    from oracle import ref_gpu as R
    if not R.available():
        return {"unavailable": "oracle/_ref/libref_gpu.so was not built"}
    out = {"source": "reference libs/pascal_tdma/gpu/tdma_local_cuda.cu and "
                     "libs/filtered_tdma/gpu/filtered_tdma_kernels.cuh, unmodified, nvcc "
                     "-O3 sm_100a; P ranks as row blocks of one array on this GPU",
           "reps": reps}
    wA, wC, wD = A.clone(), C.clone(), D.clone()

    def restore():
        wA.copy_(A)
        wC.copy_(C)
        wD.copy_(D)

    def timed(fn):
        restore()
        fn()  # warm-up (first call allocates the driver's scratch)
        ts = []
        for _ in range(reps):
            restore()
            torch.cuda.synchronize()
            e0, e1 = _events(torch)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return sum(ts) / len(ts)

    def entry(key, ms, method, P):
        o = ours[key]
        return {"ms_per_solve": ms, "rows_per_s": rows / (ms * 1e-3),
                "hbm_gbs_algorithmic": BYTES_PER_ROW_F64 * rows / (ms * 1e-3) / 1e9,
                "frac_of_peak": BYTES_PER_ROW_F64 * rows / (ms * 1e-3) / 1e9 / peak,
                "launches": R.launches(method, P), "ours_ms": o, "speedup_ours": ms / o}

    ms = timed(lambda: R.tdma_many(wA, B, wC, wD))
    out["tdma_many_P1"] = entry("tdma_many_P1", ms, "tdma_many", 1)
    ms = timed(lambda: R.pascal(wA, B, wC, wD, P))
    out["pascal_P8"] = entry("pascal_P8", ms, "pascal", P)
    restore()
    R.filtered_set_rho(wA, B, wC, P)
    ms = timed(lambda: R.filtered_v2(wA, B, wC, wD, P, 1e-3))
    e = entry("filtered_v2_P8", ms, "filtered_v2", P)
    e["ours_reference_order_ms"] = ours["filtered_v2_P8_reference_order"]
    e["speedup_ours_reference_order"] = ms / ours["filtered_v2_P8_reference_order"]
    restore()
    e["J"] = R.filtered_v2(wA, B, wC, wD, P, 1e-3, want_J=True)
    out["filtered_v2_P8"] = e
    del wA, wC, wD
    return out


def small_sweep_leg(torch, dev, peak, reps):
    """4096 x 64 heat sweep: library P = 1 and P = 4 against the reference's
    tdma_many_cuda and PaScaL kernels, L2 flushed before each repetition."""
    from filtered_tdma_b200 import Solver
    from filtered_tdma_b200 import workloads as W
    n_sys, n_row = 4096, 64
    rows = n_sys * n_row
    A, B, C, D = W.heat_sweep(n_sys, n_row, r=1.0, seed=1, device=dev)
    X = torch.empty_like(D)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 2x the 126 MB L2

    def timed(fn, prep=None):
        fn()
        ts = []
        for _ in range(reps):
            if prep is not None:
                prep()
            flush.fill_(1)
            torch.cuda.synchronize()
            e0, e1 = _events(torch)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return sum(ts) / len(ts)

    out = {"workload": "heat sweep of the 64^3 grid: 4096 systems x 64 rows, A = C = -1, "
                       "B = 3, D uniform [-1, 1]", "l2": "flushed (256 MB write) before "
                                                        "every timed solve", "reps": reps}
    for name, P in (("thomas_P1", 1), ("pascal_P4", 4)):
        s = Solver("pascal", n_sys, n_row, P)
        ms = timed(lambda: s.solve_out(A, B, C, D, X))
        out[name] = {"ms_per_solve": ms, "rows_per_s": rows / (ms * 1e-3),
                     "hbm_gbs_algorithmic": 40 * rows / (ms * 1e-3) / 1e9}
        s.close()
    from oracle import ref_gpu as R
    if R.available():
        wA, wC, wD = A.clone(), C.clone(), D.clone()

        def restore():
            wA.copy_(A)
            wC.copy_(C)
            wD.copy_(D)
        for name, fn in (("reference_tdma_many_P1", lambda: R.tdma_many(wA, B, wC, wD)),
                         ("reference_pascal_P4", lambda: R.pascal(wA, B, wC, wD, 4))):
            ms = timed(fn, restore)
            out[name] = {"ms_per_solve": ms, "rows_per_s": rows / (ms * 1e-3)}
        out["speedup_P1"] = out["reference_tdma_many_P1"]["ms_per_solve"] / \
            out["thomas_P1"]["ms_per_solve"]
        out["speedup_P4"] = out["reference_pascal_P4"]["ms_per_solve"] / \
            out["pascal_P4"]["ms_per_solve"]
    return out


def time_variant(torch, solver, A, B, C, D, X, steps, warmup, launches_per_step, sampler=None):
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        solver.solve_out(A, B, C, D, X)
    torch.cuda.synchronize()
    if sampler is not None:
        sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for e0, e1 in ev:
        e0.record(stream)
        solver.solve_out(A, B, C, D, X)
        e1.record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    if sampler is not None:
        sampler.stop()
    per = [e0.elapsed_time(e1) for e0, e1 in ev]
    return t0.elapsed_time(t1), per, steps * launches_per_step


def run_case(args):
    """One configuration solved a few times (``--case``), for ncu captures.

    batch: a uniform [n_row x n_sys] batch (per-system r log-uniform in
    [0.1, 10], A = C = -r, B = 1 + 2r, D uniform in [-1, 1], generated on the
    device); ragged: the 10000-system CSR batch (n log-uniform 16..4096,
    autotuned); heat: fused ADI steps on --heat-grid; poisson: the channel
    wall-normal solve 128 x 65 x 192; momentum: the channel momentum ADI (z, y, x
    sweeps) of one velocity component on 256^3.  Prints the CUDA-event time of
    each repetition and, for batches, the algorithmic HBM rate."""
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

    if args.case == "batch":
        r_lo, r_hi = (float(v) for v in args.r_range.split(","))
        A, B, C, D = W.diag_dominant(args.n_sys, args.n_row, r_lo, r_hi, seed=2, device=dev)
        X = torch.empty_like(D)
        f32 = args.storage == "f32"
        if f32:
            A, B, C, D = [t.float() for t in (A, B, C, D)]
        s = Solver(args.method, args.n_sys, args.n_row, args.P,
                   precision=L.FP32_STORE if f32 else L.FP64, flags=args.flags)
        s.set_tile_shape({"auto": L.TILE_AUTO, "narrow": L.TILE_NARROW,
                          "wide": L.TILE_WIDE}[args.tile_shape])
        if args.method != "pascal":
            s.set_eps_constant(1e-3)
            s.set_rho(A, B, C, all_systems=True)
        rows = args.n_sys * args.n_row
        bpr = 24 if f32 else 40
        if f32:
            ms = timed(lambda: s.solve_f32(A, B, C, D, X, cyclic=args.cyclic), args.reps)
        else:
            ms = timed(lambda: s.solve_out(A, B, C, D, X, cyclic=args.cyclic), args.reps)
        for r, t in enumerate(ms):
            print(f"rep {r}: {t:.4f} ms  {rows / t / 1e6:.2f} G rows/s  "
                  f"{bpr * rows / t / 1e6:.1f} GB/s ({bpr} B/row)")
        if s.status() != 0:
            raise SystemExit("device status word set")
    elif args.case == "ragged":
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
        c_visc = 0.5 * (1.0 / 180.0) * 1e-3
        ms = timed(lambda: mm.adi(0, rhs, q, c_visc), args.reps)
        print("momentum component", ["%.4f ms" % t for t in ms], "status", mm.status())
    else:
        from filtered_tdma_b200.poisson import ChannelPoisson
        cp = ChannelPoisson(128, 128, 192, gamma=2.0)
        hat = torch.complex(torch.rand((192, cp.n_modes), dtype=torch.float64, device=dev),
                            torch.rand((192, cp.n_modes), dtype=torch.float64, device=dev))
        ms = timed(lambda: cp.solve(hat), args.reps)
        print("poisson", ["%.4f ms" % t for t in ms], cp.n_modes, "modes")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg")
    # single-configuration runs for ncu captures (no JSON line)
    ap.add_argument("--case", choices=["batch", "ragged", "heat", "poisson", "momentum"],
                    help="run one configuration --reps times and print its times")
    ap.add_argument("--method", default="pascal")
    ap.add_argument("--P", type=int, default=8)
    ap.add_argument("--flags", type=int, default=0, help="batch: btdma_create flags")
    ap.add_argument("--n-sys", type=int, default=32768)
    ap.add_argument("--n-row", type=int, default=512)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--cyclic", action="store_true")
    ap.add_argument("--storage", choices=["f64", "f32"], default="f64",
                    help="f32: A, B, C, D stored in FP32 (FP32_STORE handle)")
    ap.add_argument("--heat-grid", default="256,384,512")
    ap.add_argument("--no-tune", action="store_true", help="ragged: keep the default plan")
    ap.add_argument("--tile-shape", choices=["auto", "narrow", "wide"], default="auto",
                    help="batch: kernel shape of the tiled PaScaL solve")
    ap.add_argument("--r-range", default="0.1,10",
                    help="batch: per-system r log-uniform in [lo, hi] (A = C = -r, B = 1 + 2r)")
    args = ap.parse_args()
    if args.case:
        return run_case(args)
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    from filtered_tdma_b200 import Solver
    from filtered_tdma_b200 import workloads as W
    from filtered_tdma_b200.replicas import max_over_ranks, whole_job_rate

    A, B, C, D = W.diag_dominant(N_SYS, N_ROW, seed=2 + rank, device=dev)
    X = torch.empty_like(D)
    rows = N_SYS * N_ROW

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---------------------------------------------------------- headline
    pas = Solver("pascal", N_SYS, N_ROW, P)
    barrier()
    clk = ClockSampler(dev)
    total_ms, per, launches = time_variant(torch, pas, A, B, C, D, X, args.steps, args.warmup, 1,
                                           sampler=clk)
    barrier()
    total_ms = max_over_ranks(total_ms, device=dev)
    ms_step = total_ms / args.steps
    value = whole_job_rate(rows, world, ms_step)

    peak, peak_src = measured_peak()
    k_ms = sum(per) / len(per)  # one kernel launch per PaScaL step
    achieved = BYTES_PER_ROW_F64 * rows / (k_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": ncu_traffic("tile_wide_f64_262144x512"),
                "kernel": "btdma::tile_wide_kernel<32, false, double>", "peak_source": peak_src,
                "algorithmic_bytes_per_launch": BYTES_PER_ROW_F64 * rows}

    # ---------------------------------------------------------- variants (rank 0 reports)
    variants = {}
    if rank == 0:
        def gbps(ms, bpr):
            return bpr * rows / (ms * 1e-3) / 1e9

        from filtered_tdma_b200 import _lib as L
        # Filtered v2 (eps_c = 1e-3, rho over all systems): by default the exact
        # reduced solve where J reaches m - 2 (here J = 63 = m - 1 in every
        # segment), bit-identical to the reference's Filtered with
        # FLAG_REFERENCE_ORDER; PaScaL in the reference's operation order; the
        # serial Thomas (P = 1, bit-identical to tdma_many)
        for name, method, Pv, lps, fl in (
                ("filtered_v2_P8", "filtered_v2", 8, 4, 0),
                ("filtered_v2_reference_order_P8", "filtered_v2", 8, 3, L.FLAG_REFERENCE_ORDER),
                ("pascal_reference_order_P8", "pascal", 8, 1, L.FLAG_REFERENCE_ORDER),
                ("thomas_P1", "pascal", 1, 1, 0)):
            s = Solver(method, N_SYS, N_ROW, Pv, flags=fl)
            if method != "pascal":
                s.set_eps_constant(1e-3)
                s.set_rho(A, B, C, all_systems=True)
            tot, pv, _ = time_variant(torch, s, A, B, C, D, X, max(3, args.steps // 2), 3, lps)
            ms = tot / max(3, args.steps // 2)
            variants[name] = {"rows_per_s": rows / (ms * 1e-3), "ms_per_step": ms,
                              "hbm_gbs_algorithmic": gbps(ms, BYTES_PER_ROW_F64),
                              "frac_of_peak": gbps(ms, BYTES_PER_ROW_F64) / peak,
                              "launches_per_step": lps}
            if method != "pascal":
                variants[name]["J"] = s.last_J()
                variants[name]["filtered_exact"] = s.last_stats()["filtered_exact"]
            s.close()

        # Filtered v2 where the truncation holds: the same shape with r
        # log-uniform in [0.1, 1] (rho <= 1/3, J = 9 < m - 2).  By default the
        # tiled kernels with Filtered's 2 x 2 interfaces (4 launches: J, the
        # Filtered solve, the gated exact one); with FLAG_REFERENCE_ORDER the
        # reference's scheme bit for bit (3 launches).  Their distance to the
        # tiled PaScaL solve of the same batch is reported beside eps.
        tA, tB, tC, tD = W.diag_dominant(N_SYS, N_ROW, 0.1, 1.0, seed=3, device=dev)
        tX = torch.empty_like(tD)
        sp_ = Solver("pascal", N_SYS, N_ROW, 8)
        sp_.solve_out(tA, tB, tC, tD, tX)
        torch.cuda.synchronize()
        xpas = tX.clone()
        sp_.close()
        trunc = {"workload": "262144 x 512, r log-uniform [0.1, 1] (rho <= 1/3), eps_c = 1e-3, "
                             "rho over all systems", "eps": 1e-3 / N_ROW ** 2}
        for key, fl, lps in (("tiled", 0, 4), ("reference_order", L.FLAG_REFERENCE_ORDER, 3)):
            s = Solver("filtered_v2", N_SYS, N_ROW, 8, flags=fl)
            s.set_eps_constant(1e-3)
            s.set_rho(tA, tB, tC, all_systems=True)
            tot, _, _ = time_variant(torch, s, tA, tB, tC, tD, tX, max(3, args.steps // 2), 3,
                                     lps)
            ms = tot / max(3, args.steps // 2)
            torch.cuda.synchronize()
            trunc[key] = {"ms_per_step": ms, "rows_per_s": rows / (ms * 1e-3),
                          "frac_of_peak": gbps(ms, BYTES_PER_ROW_F64) / peak,
                          "launches_per_step": lps, "J": s.last_J(),
                          "filtered_exact": s.last_stats()["filtered_exact"],
                          "max_abs_diff_vs_pascal": float((tX - xpas).abs().max().item())}
            s.close()
        trunc["speedup_tiled_vs_reference_order"] = (trunc["reference_order"]["ms_per_step"] /
                                                     trunc["tiled"]["ms_per_step"])
        variants["filtered_v2_truncating_P8"] = trunc
        del tA, tB, tC, tD, tX, xpas

        # The reference's own GPU kernels on this GPU (oracle/_ref/libref_gpu.so:
        # the reference's sources compiled for sm_100a, its P ranks run as row
        # blocks of one array with the MPI transport replaced by pointers), on
        # the same batch; they overwrite A, C, D, so pristine copies are put
        # back before every repetition, outside the timed events.
        variants["reference_gpu_kernels"] = reference_gpu_leg(
            torch, A, B, C, D, rows, peak, max(3, args.steps // 2),
            ours={"tdma_many_P1": variants["thomas_P1"]["ms_per_step"],
                  "pascal_P8": ms_step,
                  "filtered_v2_P8": variants["filtered_v2_P8"]["ms_per_step"],
                  "filtered_v2_P8_reference_order":
                      variants["filtered_v2_reference_order_P8"]["ms_per_step"]})

        # The 64^3 heat sweep of the reference's small configuration: 4096
        # systems x 64 rows, A = C = -1, B = 3 (rho = 1/3), D uniform in [-1, 1];
        # serial Thomas (P = 1, bit-identical to tdma_many) and PaScaL with 4
        # segments, against the reference's GPU kernels.  The batch (8 MB)
        # fits in L2, so L2 is flushed before every timed repetition.
        variants["heat_sweep_4096x64"] = small_sweep_leg(torch, dev, peak,
                                                         max(5, args.steps))

        # FP32 storage (A, B, C, D as float, x as double): 24 B/row.
        #   fp32_store: FP64 arithmetic on the exactly widened values (one pass);
        #   fp32_refine: FP32 sweeps + FP64 residual refinement (config batch A),
        #   and the same on a weakly dominant batch (rho in [0.45, 0.499], batch B).
        stream = torch.cuda.current_stream().cuda_stream
        nrep = max(3, args.steps // 2)

        def f32_variant(name, prec, arrs):
            A32, B32, C32, D32 = arrs
            s = Solver("pascal", N_SYS, N_ROW, P, precision=prec)

            def run_f32():
                L.check(L.lib().btdma_solve_f32(s._h, A32.data_ptr(), B32.data_ptr(),
                                                C32.data_ptr(), D32.data_ptr(), X.data_ptr(),
                                                N_SYS, N_ROW, 0, stream))
            for _ in range(3):
                run_f32()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(nrep):
                run_f32()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / nrep
            # accuracy against the FP64 solve of the widened values (device, P=1 Thomas)
            Xr = torch.empty_like(X)
            ref = Solver("pascal", N_SYS, N_ROW, 1)
            ref.solve_out(A32.double(), B32.double(), C32.double(), D32.double(), Xr)
            run_f32()
            err = ((X - Xr).abs().max() / Xr.abs().max()).item()
            ref.close()
            del Xr
            v = {"rows_per_s": rows / (ms * 1e-3), "ms_per_step": ms,
                 "hbm_gbs_algorithmic": gbps(ms, 24),
                 "frac_of_peak": gbps(ms, 24) / peak,
                 "speedup_vs_fp64_value": (rows / (ms * 1e-3)) / (rows / (ms_step * 1e-3)),
                 "max_rel_err_vs_fp64_thomas": err}
            if prec == L.FP32_REFINE:
                v["refinement"] = s.last_stats()
            else:
                v["refinement_sweeps"] = 0
                v["kernel"] = "btdma::tile_wide_kernel<32, false, float>"
                v["traffic"] = ncu_traffic("tile_wide_f32_262144x512")
            variants[name] = v
            s.close()

        arrs = [t.to(torch.float32) for t in (A, B, C, D)]
        f32_variant("fp32_store_P8", L.FP32_STORE, arrs)
        f32_variant("fp32_refine_P8", L.FP32_REFINE, arrs)
        del arrs
        Aw, Bw, Cw, Dw = W.weak_dominance(N_SYS, N_ROW, seed=3, device=dev)
        arrs = [t.to(torch.float32) for t in (Aw, Bw, Cw, Dw)]
        del Aw, Bw, Cw, Dw
        f32_variant("fp32_refine_weak_P8", L.FP32_REFINE, arrs)
        f32_variant("fp32_store_weak_P8", L.FP32_STORE, arrs)
        del arrs

        # Ragged batch: 10000 systems, n log-uniform in [16, 4096] (CSR offsets),
        # 25 % periodic, r log-uniform in [0.05, 20]; autotuned per length bucket.
        # (FP32-stored values, widened for the FP64 solve, so both solve one system)
        rA, rB, rC, rD, roff, rper = W.ragged_batch(10000, seed=5, dtype=np.float32)
        rrows = int(roff[-1])
        rX = torch.empty(rrows, dtype=torch.float64, device=dev)
        ref_x = None
        for name, prec, dt, bpr in (("ragged_fp64", L.FP64, torch.float64, 40),
                                    ("ragged_fp32_store", L.FP32_STORE, torch.float32, 24)):
            dA, dB, dC, dD = [torch.from_numpy(v).to(dev).to(dt) for v in (rA, rB, rC, rD)]
            s = Solver("pascal", 10000, 64, 2, precision=prec)
            plan = s.ragged_autotune(dA, dB, dC, dD, rX, roff, rper)
            for _ in range(3):
                s.solve_ragged(dA, dB, dC, dD, rX, roff, rper)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(nrep):
                s.solve_ragged(dA, dB, dC, dD, rX, roff, rper)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / nrep
            v = {"rows_per_s": rrows / (ms * 1e-3), "ms_per_step": ms, "rows": rrows,
                 "hbm_gbs_algorithmic": bpr * rrows / (ms * 1e-3) / 1e9,
                 "frac_of_peak": bpr * rrows / (ms * 1e-3) / 1e9 / peak,
                 "length_buckets": len(plan),
                 "plan": [{k: b[k] for k in ("periodic", "n_systems", "n_row_min", "n_row_max",
                                             "lanes_per_system", "warps_per_cta")} for b in plan]}
            if ref_x is None:
                ref_x = rX.clone()
            else:
                v["max_rel_err_vs_ragged_fp64"] = ((rX - ref_x).abs().max()
                                                    / ref_x.abs().max()).item()
            variants[name] = v
            s.close()
            del dA, dB, dC, dD
        del rX, ref_x

        # Fused heat ADI step, 256 x 384 x 512 interior cells (Z, Y, X sweeps of
        # n_row 512 / 384 / 256 over 98304 / 131072 / 196608 systems), rho_z = 1/3,
        # one CUDA graph per step.  Algorithmic traffic per cell and step: the
        # three sweeps each read and write one field, 48 B (the right-hand side
        # and the update fused into them); the design's own passes are reported
        # beside it.  Parity of this grid with the oracle: tests/test_heat.py.
        from filtered_tdma_b200.heat import HeatADI, dt_from_rho
        hx, hy, hz = 256, 384, 512
        heat = HeatADI(hx, hy, hz, dt=dt_from_rho(1.0 / 3.0, hz, option="strong"))
        th = heat.field(dev)
        heat.step(th, 3)
        torch.cuda.synchronize()
        hsteps = max(5, args.steps)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        heat.step(th, hsteps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / hsteps
        cells = hx * hy * hz
        variants["heat_adi_step_256x384x512"] = {
            "ms_per_step": ms, "cells_per_s": cells / (ms * 1e-3),
            "sweep_rows_per_s": 3 * cells / (ms * 1e-3),
            "algorithmic_bytes_per_cell": 48,
            "hbm_gbs_algorithmic": 48 * cells / (ms * 1e-3) / 1e9,
            "frac_of_peak": 48 * cells / (ms * 1e-3) / 1e9 / peak,
            # the design's field passes of 16 B: Z sweep reading theta (its
            # right-hand side computed inside the solve) into the Y layout, Y
            # sweep into the X layout, X sweep into theta (plus the wall planes)
            "design_bytes_per_cell": 48,
            "parity": "tests/test_heat.py::test_gpu_step_benched_grid_matches_oracle",
            # 5 kernels a step (the sweeps' factor tables are built at
            # create): Z sweep with the right-hand side, Y wall folds, Y sweep,
            # X wall folds, X sweep
            "launches_per_step": 5, "graph": True,
            "finite": bool(torch.isfinite(th).all().item())}
        heat.close()
        del th

        # Channel Poisson wall-normal solve: 128 x 65 complex modes x 192 rows,
        # tanh-stretched (gamma = 2), real and imaginary parts with one set of
        # generated coefficients; 16 B per real row (read rhs, write p).
        from filtered_tdma_b200.poisson import ChannelPoisson
        cp = ChannelPoisson(128, 128, 192, gamma=2.0)
        g = torch.Generator(device=dev)
        g.manual_seed(4)
        hat0 = torch.complex(torch.rand((192, cp.n_modes), generator=g, dtype=torch.float64,
                                        device=dev),
                             torch.rand((192, cp.n_modes), generator=g, dtype=torch.float64,
                                        device=dev))
        hat = hat0.clone()
        for _ in range(3):
            cp.solve(hat)
        torch.cuda.synchronize()
        preps = max(20, args.steps)
        e0.record()
        for _ in range(preps):
            cp.solve(hat)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / preps
        prow = 2 * 192 * cp.n_modes
        variants["channel_poisson_128x65x192"] = {
            "ms_per_solve": ms, "real_rows_per_s": prow / (ms * 1e-3),
            "hbm_gbs_algorithmic": 16 * prow / (ms * 1e-3) / 1e9,
            "frac_of_peak": 16 * prow / (ms * 1e-3) / 1e9 / peak,
            "modes": cp.n_modes, "note": "working set 26 MB (< L2): L2-resident, not HBM-bound"}
        cp.close()
        del hat, hat0

        # Channel momentum ADI (implicit viscous half-step of one velocity
        # component: z, y, x sweeps) on the reference's 256^3 channel grid (x, y
        # periodic, z tanh-stretched walls): three generated-coefficient
        # sweeps, the z sweep reading the field, each storing into the next
        # sweep's layout, the x sweep into the field: 3 passes of 16 B per cell.
        from filtered_tdma_b200.momentum import ChannelMomentum
        mm = ChannelMomentum(256, 256, 256, gamma3=1.5)
        mrhs = torch.rand(mm.shape, dtype=torch.float64, device=dev)
        mq = torch.zeros_like(mrhs)
        c_visc = 0.5 * (1.0 / 180.0) * 1e-3
        for _ in range(3):
            mm.adi(0, mrhs, mq, c_visc)
        torch.cuda.synchronize()
        mreps = max(5, args.steps)
        e0.record()
        for _ in range(mreps):
            mm.adi(0, mrhs, mq, c_visc)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / mreps
        mcells = 256 ** 3
        variants["channel_momentum_adi_256cubed"] = {
            "ms_per_component": ms, "cells_per_s": mcells / (ms * 1e-3),
            "sweep_rows_per_s": 3 * mcells / (ms * 1e-3),
            # three sweeps reading and writing one field: 48 B per cell
            "algorithmic_bytes_per_cell": 48,
            "hbm_gbs_algorithmic": 48 * mcells / (ms * 1e-3) / 1e9,
            "frac_of_peak": 48 * mcells / (ms * 1e-3) / 1e9 / peak,
            # 3 kernels a component once the factor tables exist (the first
            # call for a coefficient builds them: 3 more)
            "design_bytes_per_cell": 48, "launches": 3,
            "status": mm.status()}
        mm.close()
        del mrhs, mq

    # ---------------------------------------------------------- end to end
    e2e = None
    if not args.no_e2e:
        hA, hB, hC, hD = [x.cpu().pin_memory() for x in (A, B, C, D)]
        hX = torch.empty_like(hD).pin_memory()
        e2e_steps = max(2, min(args.steps, 5))
        barrier()

        def e2e_step():
            # host arrays in, host solution out: copy-in, solve and copy-out
            # overlap chunk by chunk inside the library
            pas.solve_host(hA, hB, hC, hD, hX)

        e2e_step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record()
        for _ in range(e2e_steps):
            e2e_step()
        e1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, device=dev)
        pas.solve_out(A, B, C, D, X)  # the device path on the same arrays
        same = bool(torch.equal(X.cpu(), hX))
        e2e = {"value": whole_job_rate(rows, world, ms), "unit": "rows/s",
               "equals_device_solve": same,
               "h2d_bytes_per_step": 4 * 8 * rows, "d2h_bytes_per_step": 8 * rows,
               "ms_per_step": ms, "path": "Solver.solve_host (C ABI btdma_solve_host): pinned "
                                         "host A, B, C, D in, host x out every step, copies "
                                         "and solves overlapped in chunks of systems"}
        del hA, hB, hC, hD, hX

    # ---------------------------------------------------------- CPU baseline
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, kind, used, desc, _ = cpu_reference_rate(16384, reps=3)
        cpu = {"value": rate, "unit": "rows/s", "cores": used, "kind": kind, "sample": desc}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_sys": N_SYS, "n_row": N_ROW, "P": P,
                       "method": "pascal", "per_rank_batch": True,
                       "kernel_sub_segments": N_ROW // 16,
                       "kernel_note": "P = 8 is the reference's rank count; the tiled "
                                      "kernel splits every system into n_row / 16 = 32 "
                                      "sub-segments of 16 rows and solves the 64-unknown "
                                      "reduced system exactly, so the result does not "
                                      "depend on P",
                       "cpu_baseline_sample": "16384 systems x 512 rows (1/16 of the "
                                              "batch), median of 3 solves",
                       "l2": "inputs 4.3 GB per rank > 126 MB L2; no flush needed"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk.summary(), "variants": variants,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
