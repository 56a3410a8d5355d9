"""Per-step timing of the fused heat ADI step in the reference's long CSV format
(apps/heat_gpu/timing_csv.hpp:13-18 and timing_save_csv :85-106; file name and
meta line as SolveTheta::profile writes them, solve_theta.cu:604-625), so the
reference's plot scripts read B200 runs unchanged:

    # grid=513x513x513, np=1 (1,1,1), dt= 1.234E-05, Nt=40, solver_kind=pascal
    rank,t_step,event,time_sec
    0,1,rhs, 1.234567890E-04
    ...

    python -m filtered_tdma_b200.timing_csv --grid 512 512 512 --steps 40 --warmup 10
"""
from __future__ import annotations

import argparse
import os

EVENTS = ("rhs", "solve_z", "solve_y", "solve_x", "etc", "comm",
          "tdma_z_comm", "tdma_y_comm", "tdma_x_comm",
          "tdma_z_gpu", "tdma_y_gpu", "tdma_x_gpu")


def meta_line(nx, ny, nz, dt, nt, backend="pascal", np_dim=(1, 1, 1)) -> str:
    """nx, ny, nz are the reference's parameters (the input size plus one)."""
    npt = np_dim[0] * np_dim[1] * np_dim[2]
    return (f"grid={nx}x{ny}x{nz}, np={npt} ({np_dim[0]},{np_dim[1]},{np_dim[2]}), "
            f"dt={dt:10.3E}, Nt={nt}, solver_kind={backend}")


def default_path(nx, backend="pascal", np_dim=(1, 1, 1)) -> str:
    env = os.environ.get("TIMING_CSV", "")
    if env:
        return env
    return f"results/timing_{nx}_{np_dim[0]}{np_dim[1]}{np_dim[2]}_{backend}.csv"


def write_csv(path, per_step_times, meta) -> None:
    """per_step_times: list over timed steps of the 12 event times (one rank)."""
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w") as f:
        f.write(f"# {meta}\n")
        f.write("rank,t_step,event,time_sec\n")
        for t, row in enumerate(per_step_times, start=1):
            for name, v in zip(EVENTS, row):
                f.write(f"0,{t},{name},{v:16.9E}\n")


def read_csv(path):
    """(meta, {(rank, t_step, event): seconds})."""
    out = {}
    with open(path) as f:
        meta = f.readline()[2:].rstrip("\n")
        assert f.readline().strip() == "rank,t_step,event,time_sec"
        for line in f:
            r, t, e, v = line.rstrip("\n").split(",")
            out[(int(r), int(t), e)] = float(v)
    return meta, out


def profile_run(ix, iy, iz, steps, warmup, rho=1.0 / 3.0, path=None):
    """Run warmup + steps fused heat steps (dt from rho and dz, the reference's
    "strong" option) timing each phase, and write the CSV; returns the path."""
    import torch

    from .heat import HeatADI, dt_from_rho
    dt = dt_from_rho(rho, iz, option="strong")
    h = HeatADI(ix, iy, iz, dt=dt)
    th = h.field(torch.device("cuda:0"))
    rows = []
    for s in range(warmup + steps):
        t = h.step_profile(th)
        if s >= warmup:
            rows.append(t)
    nx, ny, nz = ix + 1, iy + 1, iz + 1
    path = path or default_path(nx)
    write_csv(path, rows, meta_line(nx, ny, nz, dt, warmup + steps))
    h.close()
    return path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[256, 256, 256])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--rho", type=float, default=1.0 / 3.0)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    print(profile_run(*a.grid, a.steps, a.warmup, a.rho, a.out))


if __name__ == "__main__":
    main()
