"""Runs RK4 steps of the plate workload for profiling.

    python -m pdmtel_b200.profile_run [--dims 200,200,4] [--steps 2] [--warmup 1] [--prec fp32c|fp64]

Builds the pre-cracked plate deck at the requested lattice size, runs the
drop-in's InitialProblem (device bond search, host MLS setup), then
`warmup` + `steps` device-resident RK4 steps in the chosen arithmetic, and
prints the device time per step.  Meant to be run under ncu on a size that
keeps a capture short.
"""
import argparse
import os
import sys
import tempfile
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="200,200,4")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--prec", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--spacing", type=float, default=5e-4)
    a = ap.parse_args()
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import pdmtel_b200 as P
    from pdmtel_b200 import decks as D

    dims = tuple(int(v) for v in a.dims.split(","))
    wd = tempfile.mkdtemp(prefix="pdprof_")
    # slit of 20% of the plate width, centred, as in the 400-wide plate
    D.config_plate(dims=dims, spacing=a.spacing, slit_half_length=0.1 * dims[0] * a.spacing, dt=5e-9).write(wd)
    t0 = time.time()
    dm = P.pdDataManager(wd)
    P.pdSolve.InitialProblem(dm)
    ctx = dm.context()
    ctx.set_energy(False)
    ctx.set_precision(P.PREC_FP32C if a.prec == "fp32c" else P.PREC_FP64)
    setup = time.time() - t0
    dt = 5e-9
    ctx.rk4_steps(dt, 0.0, a.warmup)
    ctx.sync()
    t1 = time.time()
    ctx.rk4_steps(dt, a.warmup * dt, a.steps)
    ctx.sync()
    el = time.time() - t1
    ev = 4 * ctx.evals_per_stage()
    print(f"nodes {ctx.n} setup {setup:.1f}s  {1e3 * el / max(a.steps, 1):.3f} ms/step (wall)  "
          f"{ev * a.steps / el / 1e9:.1f} G evals/s")


if __name__ == "__main__":
    main()
