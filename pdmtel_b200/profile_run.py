"""Small, self-contained runs of each hot kernel, for profiling.

    python -m pdmtel_b200.profile_run [--mode plate|static|adjoint|batch] ...

plate:   the pre-cracked plate deck at --dims (default 200,200,4), `warmup`
         + `steps` device-resident RK4 steps in --prec (fp32c|fp64);
static:  the clamped cube of --cube nodes per side (stencil operator), one
         FP64 and one FP32 static solve capped at --iters CG iterations;
adjoint: the 64x64x8 identification specimen (or --dims), pd_adjoint_forward
         of --steps steps and the reverse sweep;
batch:   --count specimens of 1k..--nmax nodes, --steps RK4 steps in one
         persistent launch and in the graph of a step.

Each prints the device-independent facts of its run and its wall time.
Meant to be run under ncu on a size that keeps a capture short.
"""
import argparse
import os
import sys
import tempfile
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default="plate", choices=["plate", "static", "adjoint", "batch"])
    ap.add_argument("--dims", default=None)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--prec", default="fp32c", choices=["fp32c", "fp64", "fp64a"])
    ap.add_argument("--spacing", type=float, default=5e-4)
    ap.add_argument("--cube", type=int, default=96)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--count", type=int, default=16)
    ap.add_argument("--nmax", type=int, default=20000)
    ap.add_argument("--sell", action="store_true", help="plate: FP32 gather from the SELL copy")
    ap.add_argument("--quad", action="store_true", help="plate: FP32 force with four nodes per thread")
    ap.add_argument("--order-tile", default=None, help="plate: node-order tile exponents bx,by,bz")
    ap.add_argument("--stencil", type=int, default=0, help="plate: lattice-stencil force, block shape 1..4")
    ap.add_argument("--patterns", action="store_true", help="plate: FP32 gather from contributor patterns")
    a = ap.parse_args()
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import pdmtel_b200 as P
    from pdmtel_b200 import decks as D

    prec = {"fp32c": P.PREC_FP32C, "fp64": P.PREC_FP64, "fp64a": P.PREC_FP64A}[a.prec]
    wd = tempfile.mkdtemp(prefix="pdprof_")
    t0 = time.time()
    if a.mode == "plate":
        dims = tuple(int(v) for v in (a.dims or "200,200,4").split(","))
        # slit of 20% of the plate width, centred, as in the 400-wide plate
        D.config_plate(dims=dims, spacing=a.spacing, slit_half_length=0.1 * dims[0] * a.spacing, dt=5e-9).write(wd)
        dm = P.pdDataManager(wd)
        P.pdSolve.InitialProblem(dm)
        ctx = dm.context()
        ctx.set_energy(False)
        ctx.set_precision(prec)
        if a.order_tile:
            bx, by, bz = (int(v) for v in a.order_tile.split(","))
            ctx.set_option(P.OPT_TILE, bx | (by << 8) | (bz << 16))
        if a.sell:
            ctx.set_option(P.OPT_GATHER_SELL, 1)
        if a.quad:
            ctx.set_option(P.OPT_FORCE_QUAD, 1)
        if a.stencil:
            ctx.set_option(P.OPT_FORCE_STENCIL, a.stencil)
        if a.patterns:
            ctx.set_option(P.OPT_GATHER_STENCIL, 1)
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
    elif a.mode == "static":
        D.config_cube(n=a.cube, intg_point=1).write(wd)
        dm = P.pdDataManager(wd)
        dm.InitNode()
        dm.InitBond()
        dm.InitMaterial()
        ctx = dm.context()
        st = ctx.static_prepare()
        for p in (P.PREC_FP64, P.PREC_FP32C):
            t1 = time.time()
            try:
                ctx.static_solve(1.0, precision=p, rtol=1e-10, maxit=a.iters)
            except P.PdError:
                pass  # capped on purpose
            print(f"nodes {ctx.n} stencil {st} prec {p}: {a.iters} CG iterations {time.time() - t1:.3f}s (wall)")
    elif a.mode == "adjoint":
        dims = tuple(int(v) for v in (a.dims or "64,64,8").split(","))
        D.config_identify(dims=dims, dt=1e-8, steps=a.steps).write(wd)
        dm = P.pdDataManager(wd)
        P.pdSolve.InitialProblem(dm)
        ctx = dm.context()
        ctx.set_precision(prec)
        import numpy as np
        ctx.set_spring_factor(np.ones(ctx.n))
        t1 = time.time()
        ctx.adjoint_forward(1e-8, 0.0, a.steps, max(1, a.steps // 2))
        U, _ = ctx.get_state()
        ctx.adjoint_backward(U)
        print(f"nodes {ctx.n} adjoint of {a.steps} steps {time.time() - t1:.3f}s (wall)")
    else:
        from pdmtel_b200 import batch as B
        spec = B.BatchSpec(dims=B.draw_dims(a.count, 7, 1000, a.nmax), seed=7)
        bt = B.Batch(wd, spec, precision=P.PREC_FP32C)
        for persistent in (True, False):
            bt.ctx.reset_state()
            t1 = time.time()
            bt.run(a.steps, persistent=persistent)
            print(f"nodes {bt.offsets[-1]} persistent {persistent}: {a.steps} steps {time.time() - t1:.3f}s (wall)")


if __name__ == "__main__":
    main()
