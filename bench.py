#!/usr/bin/env python
"""Bond-force evaluations per second of the pdMTEL hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form precision|batch|static]

Workload: the pre-cracked plate, 400x400x4 nodes on a cubic lattice (spacing
0.5 mm, horizon 3.015 spacings, E = 72 GPa, rho = 2440 kg/m^3, 2x2x2 Gauss
points with MLS), a central 40 mm slit along x through the thickness, +-0.05
m/s on the top and bottom node layers, dt = 5e-9 s, from rest.  Synthetic
input (a generated lattice); one step is one RK4 step (4 stages, each one
Gauss-point force evaluation per unbroken family entry and point).

ours: the FP32-compensated form is the headline `value`; the FP64 drop-in is
timed beside it (`fp64`) and the relative displacement/velocity error of the
FP32 form against it after W+K steps is reported.  `e2e` is the same metric
through the C ABI with host buffers (pd_rk4_steps_host, one step per call:
state uploaded from pinned memory and downloaded every step).

reference: the reference CPU solver (oracle/_ref, built from the reference
sources) on a 40x40x4 sub-plate of the same workload, one process per host
core, each step one RK4 step of every process.

The headline line also carries `adjoint`: seconds per RK4 step of the
differentiation form (forward with checkpoints + reverse sweep; FP64, FP64A,
FP32C with FP64 point terms, FP32C with FP32 point terms) on the
64x64x8 identification specimen (spacing 1 mm, fixed face and 0.02 m/s pulled
face, log-micromodulus a Gaussian random field, sigma 0.2, correlation 5 mm).

--form batch: the batching form, 256 specimens with node counts log-uniform
in [1k, 60k] (aspect factors uniform in [1, 4]), lognormal micromodulus
factors (sigma 0.15, correlation 4 spacings), K RK4 steps of all specimens
batched (launch shape from the autotuner: one persistent launch or the
graph of a step) against the same specimens stepped one context at a time.

--form identify: the differentiation config end to end: a hidden
log-micromodulus field (Gaussian random field, sigma 0.2, correlation 5 mm)
on the 64x64x8 specimen generates displacements from 1000 RK4 steps with
1e-3 RMS noise; the adjoint gradient of the misfit at m = 0 is checked by
central finite differences (h = 1e-6) along 32 random directions; L-BFGS
runs 50 iterations (FP64A arithmetic, checkpoints every 50 steps).

--form accuracy: the precision form's error over the plate run: 2000 RK4
steps in FP32C and in the FP64 drop-in, relative displacement and velocity
errors at steps 100, 500 and 2000.

--form static: the 128^3 cube (bottom clamped, 1 MPa shear traction on top),
CG to relative residual 1e-10: FP32 matvec inside FP64 iterative refinement
against plain FP64 CG; time to solution and the difference of the solutions.
(--cube N changes the cube, --maxit caps the CG iterations.)  The headline
line carries the same comparison under "static" (--no-static leaves it out).

--form steps: W + K device-resident RK4 steps of the plate (--plate-dims,
--prec, launch shapes from --shape or the tuner) and nothing else: the run
profiler captures are taken on.  --form adjoint: the adjoint pair alone on the
identification specimen (--adjoint-steps).

--form ai: the adaptive-trapezoid (ai_on) form on the 20x10x10 bar (FP64
drop-in, trapezoid index 3, MLS): RK4 steps on the device, in trapezoid-point
force evaluations per second, against one stage of the oracle port on the
host (the reference's own AI setup on this bar runs for tens of minutes).

Multi-GPU: replicas (one full plate per rank, no data-path collective);
weak scaling; time = max over ranks of the device-timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bond-force evals/s on 1 B200: FP32-comp vs FP64 at ≤1e-6 rel err; adjoint s/step"
UNIT = "bond-force evals/s"
PLATE = dict(dims=(400, 400, 4), spacing=5e-4, slit_half_length=0.02, vel=0.05, dt=5e-9)
SUBPLATE = dict(dims=(40, 40, 4), spacing=5e-4, slit_half_length=0.004, vel=0.05, dt=5e-9)
FP32_LANES_PER_SM = 128  # sm_100: 4 SM sub-partitions x 32 FP32 lanes
FLOP_PER_EVAL = 22


def fp32_peak(sm_max_mhz):
    """Nominal FP32 rate of the device: SMs (from the device) x FP32 lanes x
    2 (FMA) x the maximum SM clock nvidia-smi reports (1965 MHz on B200 when
    nvidia-smi is unavailable)."""
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = sm_max_mhz or 1965.0
    return sms * FP32_LANES_PER_SM * 2 * mhz * 1e6, sms, mhz


def plate_cfg(dims_text):
    """The plate workload at other dimensions (for profiler captures): the
    slit keeps a tenth of the plate width on each side of the centre."""
    dims = tuple(int(v) for v in dims_text.split("x"))
    cfg = dict(PLATE, dims=dims)
    cfg["slit_half_length"] = 0.1 * dims[0] * PLATE["spacing"]
    return cfg


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_barrier(ws):
    """all ranks meet (after their device work is done)"""
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    """the max of a per-rank scalar over all ranks (NCCL on the GPU, or
    whatever backend the process group has)"""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(ws, work_per_rank, seconds_max):
    """whole-job rate of `ws` replicas: every rank's work over the slowest
    rank's time"""
    return ws * work_per_rank / seconds_max


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region.

    Samples carry nvidia-smi's own timestamp; start() returns once the first
    sample has arrived, begin()/end() mark the timed region on the same wall
    clock, and stop() keeps the samples inside it (or, for a region shorter
    than the sampling interval, the nearest sample before and after it)."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, interval_ms=20):
        self.gpu = gpu_index
        self.interval = interval_ms
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", str(self.interval)],
                                     stdout=self.f, stderr=subprocess.DEVNULL)
        deadline = time.time() + 5.0
        while time.time() < deadline and os.path.getsize(self.path) == 0:
            time.sleep(0.01)

    def begin(self):
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    @staticmethod
    def _when(stamp):
        import datetime
        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(stamp, fmt).timestamp()
            except ValueError:
                pass
        return None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(2.5 * self.interval / 1000.0)  # one sample after the region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 10:
                continue
            try:
                rows.append((self._when(p[0]), float(p[2]), float(p[3]), p[6:10]))
            except ValueError:
                continue
        os.unlink(self.path)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        inside = [r for r in rows if r[0] is not None and self.t0 is not None and self.t0 <= r[0] <= self.t1]
        note = "samples inside the timed region"
        if not inside and rows and self.t0 is not None:
            before = [r for r in rows if r[0] is not None and r[0] < self.t0]
            after = [r for r in rows if r[0] is not None and r[0] > self.t1]
            inside = before[-1:] + after[:1]
            note = "timed region shorter than the sampling interval: nearest samples before and after"
        reasons = set()
        for r in inside:
            for k, n in enumerate(names):
                if r[3][k].lower().startswith("active"):
                    reasons.add(n)
        sm = [r[1] for r in inside]
        smax = [r[2] for r in inside]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "interval_ms": self.interval, "note": note}


def setup_plate(workdir, cfg):
    import pdmtel_b200 as P
    from pdmtel_b200 import decks as D
    deck = D.config_plate(dims=cfg["dims"], spacing=cfg["spacing"], slit_half_length=cfg["slit_half_length"],
                          vel=cfg["vel"], dt=cfg["dt"], steps=100000)
    deck.write(workdir)
    t0 = time.time()
    dm = P.pdDataManager(workdir)
    P.pdSolve.InitialProblem(dm)
    ctx = dm.context()
    ctx.set_energy(False)
    return dm, ctx, time.time() - t0


def cpu_baseline_reference(workers, steps, tmp):
    """Times the reference solver on the 40x40x4 sub-plate with `workers`
    concurrent processes; returns (evals/s aggregate, details)."""
    from pdmtel_b200 import decks as D
    harness = os.path.join(ROOT, "oracle", "_ref", "pdref_harness")
    if not os.path.exists(harness):
        return None
    cfg = SUBPLATE
    procs = []
    for w in range(workers):
        wd = os.path.join(tmp, f"ref{w}")
        D.config_plate(dims=cfg["dims"], spacing=cfg["spacing"], slit_half_length=cfg["slit_half_length"],
                       vel=cfg["vel"], dt=cfg["dt"], steps=100000).write(wd)
        procs.append(subprocess.Popen([harness, "time", wd, str(steps)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True))
    outs = [json.loads(p.communicate()[0]) for p in procs]
    return outs


def plate_evals_per_step_oracle(cfg):
    """Bond-force evals per RK4 step of a plate config (4 stages x unbroken
    bond halves x 8 Gauss points), counted with the CPU oracle's bond search
    and slit rule on the deck's lattice (node coordinates (l - (n + 1) / 2)
    spacing per axis, as InitNode places them).  Labels the sub-plate
    extrapolation of the reference arm; nothing here is timed."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    dims, sp = cfg["dims"], cfg["spacing"]
    ax = [(np.arange(1, d + 1) - (d + 1) * 0.5) * sp for d in dims]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    pts = np.ascontiguousarray(np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).ravel())
    rp, col, _ = O.bond_search(pts, sp, 3.015 * sp)
    h = cfg["slit_half_length"]
    br = O.slit_mark(pts, rp, col, [(-h, h, 0.0, 0.0, -1.0, 1.0)])
    return 4 * 8 * int(len(col) - int(br.sum()))


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    workers = max(1, min(os.cpu_count() or 1, 32))
    tmp = tempfile.mkdtemp(prefix="pdref_")
    outs = cpu_baseline_reference(workers, args.warmup + args.steps, tmp)
    if outs is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pdref_harness is not built "
                          "(run make -C oracle where the reference sources exist)"}))
        return 0
    ev = sum(o["evals_per_step"] for o in outs)
    t_steps = max(sum(o["step_s"][args.warmup:]) for o in outs)
    value = ev * args.steps / t_steps
    ms = 1e3 * t_steps / args.steps
    try:
        full_ev = plate_evals_per_step_oracle(PLATE)
    except Exception:  # the oracle library is not built: no extrapolation
        full_ev = None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "plate 400x400x4 (sample: 40x40x4 sub-plate per process)",
                       "sample_nodes": outs[0]["nodes"], "processes": workers},
            "same_config": False,
            "proxy": ("evals/s of the reference solver on 40x40x4 sub-plates (same spacing, horizon, material, "
                      "2x2x2 Gauss + MLS, slit rule and velocity load; 6,400 nodes each) stand in for the "
                      "640k-node plate, whose reference setup (O(N^2) bond search, ~5 GB of MLS objects) does "
                      "not fit a bench run"),
            "extrapolation": None if not full_ev else {
                "full_plate_evals_per_step": full_ev,
                "ms_per_step_one_core": 1e3 * full_ev / (value / workers),
                "ms_per_step_all_processes": 1e3 * full_ev / value,
                "basis": "full-plate evals per step (oracle bond search and slit rule) / sample evals/s"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "reference",
                             "sample": f"{workers} processes x 40x40x4 sub-plate, {args.steps} timed RK4 steps each"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


IDENT = dict(dims=(64, 64, 8), spacing=1e-3, vel=0.02, dt=1e-8, sigma=0.2, corr=5e-3, every=50)


def accuracy_leg(ctx, dt, marks=(100, 500)):
    """The precision form's error over a longer window than the timed steps:
    the plate from rest in FP32C and in FP64 (untimed, same context and
    launch shapes), relative L2 error of U and V at each step count."""
    import numpy as np
    import pdmtel_b200 as P
    try:
        states = {}
        for name, prec in (("fp32c", P.PREC_FP32C), ("fp64", P.PREC_FP64)):
            ctx.set_precision(prec)
            ctx.reset_state()
            done = 0
            for m in marks:
                ctx.rk4_steps(dt, done * dt, m - done)
                ctx.sync()
                done = m
                states[(name, m)] = ctx.get_state()
        out = {}
        for m in marks:
            U32, V32 = states[("fp32c", m)]
            U64, V64 = states[("fp64", m)]
            out[str(m)] = {"U": float(np.linalg.norm(U32 - U64) / max(np.linalg.norm(U64), 1e-300)),
                           "V": float(np.linalg.norm(V32 - V64) / max(np.linalg.norm(V64), 1e-300))}
        out["note"] = "plate from rest, FP32C against FP64, untimed; keys are RK4 step counts"
        return out
    except Exception as e:  # the headline line is printed whatever happens here
        return {"error": repr(e)}


def adjoint_leg(tmp, steps):
    """Seconds per RK4 step of the adjoint pair on the identification
    specimen: pd_adjoint_forward (checkpoints) + pd_adjoint_backward."""
    import numpy as np
    import torch
    import pdmtel_b200 as P
    from pdmtel_b200 import adjoint as AD
    from pdmtel_b200 import decks as D
    wd = os.path.join(tmp, "ident")
    c = IDENT
    D.config_identify(dims=c["dims"], spacing=c["spacing"], vel=c["vel"], dt=c["dt"], steps=steps).write(wd)
    dm = P.pdDataManager(wd)
    P.pdSolve.InitialProblem(dm)
    ctx = dm.context()
    x, _, _ = dm.nodes()
    ctx.set_spring_factor(np.exp(AD.gaussian_random_field(x, c["spacing"], c["corr"], c["sigma"], seed=1)))
    stream = torch.cuda.ExternalStream(ctx.stream)
    # untimed: the first pair builds the transposed gather and the work pool
    ctx.reset_state()
    ctx.adjoint_forward(c["dt"], 0.0, 2, c["every"])
    U, _ = ctx.get_state()
    ctx.adjoint_backward(U)
    out = {}
    grads = {}
    for name, prec, vjp32 in (("fp64", P.PREC_FP64, 0), ("fp64a", P.PREC_FP64A, 0), ("fp32c", P.PREC_FP32C, 0),
                              ("fp32c_vjp32", P.PREC_FP32C, 1)):
        ctx.set_precision(prec)
        ctx.set_option(P.OPT_ADJOINT_VJP32, vjp32)
        if name == "fp32c":
            ctx.autotune(c["dt"], 2)  # untimed: the FP32 form's launch shapes for this specimen
        # untimed: a short pair in this precision (graphs, launch-shape setup)
        ctx.reset_state()
        ctx.adjoint_forward(c["dt"], 0.0, 2, c["every"])
        U, _ = ctx.get_state()
        ctx.adjoint_backward(U)
        ctx.reset_state()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(stream)
        ctx.adjoint_forward(c["dt"], 0.0, steps, c["every"])
        ev[1].record(stream)
        U, _ = ctx.get_state()
        g = ctx.adjoint_backward(U)
        ev[2].record(stream)
        ev[2].synchronize()
        fw = ev[0].elapsed_time(ev[1]) / 1e3
        bw = ev[1].elapsed_time(ev[2]) / 1e3
        out[name] = {"s_per_step": (fw + bw) / steps, "forward_s_per_step": fw / steps,
                     "backward_s_per_step": bw / steps, "grad_norm": float(np.linalg.norm(g))}
        grads[name] = g
    ev_step = 4 * ctx.evals_per_stage()
    dm.close()
    for name in ("fp64a", "fp32c", "fp32c_vjp32"):
        out[name]["grad_rel_diff_vs_fp64"] = float(np.linalg.norm(grads[name] - grads["fp64"]) /
                                                   np.linalg.norm(grads["fp64"]))
    res = dict(out["fp64"])
    res.update({"unit": "s/step", "steps": steps, "checkpoint_every": c["every"], "nodes": int(x.size // 3),
                "evals_per_step": ev_step, "fp64a": out["fp64a"], "fp32c": out["fp32c"],
                "fp32c_vjp32": out["fp32c_vjp32"],
                "config": "64x64x8 identification specimen, J = 0.5|U|^2, forward + reverse sweep; the main "
                          "figures FP64; fp32c = FP32-compensated forward and recompute, FP64 point terms in "
                          "the reverse sweep; fp32c_vjp32 = FP32 point terms too"})
    return res


def run_batch(args):
    """--form batch"""
    import torch
    import pdmtel_b200 as P
    from pdmtel_b200 import batch as B
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    tmp = tempfile.mkdtemp(prefix=f"pdbatch{rank}_")
    t0 = time.time()
    spec = B.BatchSpec(dims=B.draw_dims(256, 2026 + rank), seed=2026 + rank)
    bt = B.Batch(tmp, spec, precision=P.PREC_FP32C, device_setup=True)  # MLS solved on the device
    setup_s = time.time() - t0
    stream = torch.cuda.ExternalStream(bt.ctx.stream)
    ev_step = bt.evals_per_step()
    tune = bt.tune(steps=2)

    def timed(fn, sampler=None):
        bt.ctx.reset_state()
        fn(args.warmup)
        bt.ctx.reset_state()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if sampler:
            sampler.begin()
        e0.record(stream)
        fn(args.steps)
        e1.record(stream)
        e1.synchronize()
        if sampler:
            sampler.end()
        return e0.elapsed_time(e1) / 1e3

    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    t_b = timed(lambda k: bt.run(k), sampler)
    clocks = sampler.stop()
    t_other = timed(lambda k: bt.run(k, persistent=not bt.persistent))
    # one context per specimen, stepped one after the other
    ctxs = bt.specimen_contexts(P.PREC_FP32C)
    t_seq = 0.0
    for c in ctxs:
        c.rk4_steps(spec.dt, 0.0, args.warmup)
        c.sync()
        c.reset_state()
        s = torch.cuda.ExternalStream(c.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        c.rk4_steps(spec.dt, 0.0, args.steps)
        e1.record(s)
        e1.synchronize()
        t_seq += e0.elapsed_time(e1) / 1e3
    value = ev_step * args.steps / t_b
    n = int(bt.offsets[-1])
    line = {"metric": "bond-force evals/s, 256 specimens in one batch (FP32-comp)", "value": value,
            "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_b / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "256 box specimens, nodes log-uniform [1k, 60k], aspect [1, 4], "
                                   "lognormal micromodulus (sigma 0.15, corr 4 spacings), fixed + pulled faces",
                       "nodes": n, "evals_per_step": ev_step, "form": "batched, one context"},
            "autotune": tune,
            "launch": "persistent" if bt.persistent else "graph of one step",
            "other_launch": {"launch": "graph of one step" if bt.persistent else "persistent",
                             "value": ev_step * args.steps / t_other},
            "sequential": {"value": ev_step * args.steps / t_seq, "ms_per_step": 1e3 * t_seq / args.steps,
                           "speedup_batched_over_sequential": t_seq / t_b},
            "gpu_launches": 1 if bt.persistent else (13 + (4 if (tune or {}).get("force_stencil") else 0)) * args.steps,
            "clocks": clocks, "setup_s": setup_s}
    print(json.dumps(line))
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


def run_accuracy(args):
    """--form accuracy"""
    import numpy as np
    import torch
    import pdmtel_b200 as P
    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp(prefix="pdacc_")
    dm, ctx, setup_s = setup_plate(tmp, PLATE)
    dt = PLATE["dt"]
    marks = [100, 500, 2000]
    states = {}
    seconds = {}
    for name, prec in (("fp32c", P.PREC_FP32C), ("fp64", P.PREC_FP64)):
        ctx.set_precision(prec)
        ctx.reset_state()
        done, t = 0, 0.0
        t0 = time.time()
        for m in marks:
            ctx.rk4_steps(dt, done * dt, m - done)
            ctx.sync()
            done = m
            states[(name, m)] = ctx.get_state()
        seconds[name] = time.time() - t0
    err = {}
    for m in marks:
        U32, V32 = states[("fp32c", m)]
        U64, V64 = states[("fp64", m)]
        err[str(m)] = {"U": float(np.linalg.norm(U32 - U64) / np.linalg.norm(U64)),
                       "V": float(np.linalg.norm(V32 - V64) / np.linalg.norm(V64)),
                       "U_max_abs_fp64": float(np.abs(U64).max())}
    line = {"metric": "relative displacement/velocity error of FP32C against the FP64 drop-in, plate",
            "value": err["2000"]["U"], "unit": "relative L2", "n_gpus": 1, "steps": 2000, "warmup": 0,
            "ms_per_step": None, "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "plate 400x400x4, 2x2x2 Gauss+MLS, 40 mm slit, +-0.05 m/s, dt 5e-9"},
            "errors": err, "wall_s": seconds, "setup_s": setup_s}
    print(json.dumps(line))
    dm.close()
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


def run_identify(args):
    """--form identify"""
    import numpy as np
    import torch
    import pdmtel_b200 as P
    from pdmtel_b200 import adjoint as AD
    from pdmtel_b200 import decks as D
    torch.cuda.set_device(0)
    c = IDENT
    dims = tuple(int(v) for v in args.ident_dims.split("x"))
    nsteps, every = args.ident_steps, c["every"]
    tmp = tempfile.mkdtemp(prefix="pdident_")
    D.config_identify(dims=dims, spacing=c["spacing"], vel=c["vel"], dt=c["dt"], steps=nsteps).write(tmp)
    t0 = time.time()
    dm = P.pdDataManager(tmp)
    P.pdSolve.InitialProblem(dm)
    ctx = dm.context()
    ctx.set_precision(P.PREC_FP64A)
    setup_s = time.time() - t0
    x, _, _ = dm.nodes()
    n = ctx.n
    dt = c["dt"]
    m_true = AD.gaussian_random_field(x, c["spacing"], c["corr"], c["sigma"], seed=2026)

    def final_U(m):
        ctx.set_spring_factor(np.exp(m))
        ctx.reset_state()
        ctx.rk4_steps(dt, 0.0, nsteps)
        ctx.sync()
        return ctx.get_state()[0]

    U_true = final_U(m_true)
    rng = np.random.default_rng(7)
    U_obs = U_true + 1e-3 * np.sqrt(np.mean(U_true ** 2)) * rng.standard_normal(U_true.shape)
    Uo = torch.from_numpy(U_obs.reshape(n, 3))
    stream = torch.cuda.ExternalStream(ctx.stream)
    # gradient at m = 0, timed
    m0 = torch.zeros(n, dtype=torch.float64, requires_grad=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    U, _ = AD.trajectory(m0, ctx, dt, nsteps, every)
    loss = AD.misfit(U, Uo)
    loss.backward()
    e1.record(stream)
    e1.synchronize()
    grad_s = e0.elapsed_time(e1) / 1e3
    g = m0.grad.numpy().copy()
    J0 = float(loss.detach())

    def J(m):
        Uf = final_U(m)
        return 0.5 * np.sum((Uf - U_obs) ** 2) / np.sum(U_obs ** 2)

    h = 1e-6
    errs = []
    drng = np.random.default_rng(11)
    for _ in range(args.fd_dirs):
        v = drng.standard_normal(n)
        fd = (J(h * v) - J(-h * v)) / (2 * h)
        errs.append(abs(fd - g @ v) / abs(g @ v))
    res = AD.identify(ctx, U_obs, dt, nsteps, iters=args.lbfgs_iters, every=every)
    rms = lambda a: float(np.sqrt(np.mean(np.asarray(a) ** 2)))
    line = {"metric": "adjoint s/step, 64x64x8 identification (forward + reverse, FP64A)",
            "value": grad_s / nsteps, "unit": "s/step", "n_gpus": 1, "steps": nsteps, "warmup": 0,
            "ms_per_step": 1e3 * grad_s / nsteps, "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{dims[0]}x{dims[1]}x{dims[2]} identification, fixed face + "
                                   f"{c['vel']} m/s pulled face, dt {dt}, hidden GRF sigma {c['sigma']} "
                                   f"corr {c['corr']} m, noise 1e-3 RMS", "nodes": n,
                       "checkpoint_every": every},
            "gradient_check": {"h": h, "directions": args.fd_dirs, "max_rel_err": max(errs) if errs else None,
                               "median_rel_err": float(np.median(errs)) if errs else None},
            "lbfgs": {"iterations": args.lbfgs_iters, "evaluations": res.evaluations, "seconds": res.seconds,
                      "misfit_first": res.loss[0], "misfit_last": res.loss[-1],
                      "m_rms_error_start": rms(m_true), "m_rms_error_end": rms(res.m - m_true)},
            "misfit_at_zero": J0, "setup_s": setup_s}
    print(json.dumps(line))
    dm.close()
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


def static_solves(tmp, n, maxit=100000, precond=True, split=4):
    """The static config on an n^3 cube (bottom clamped, 1 MPa shear traction
    on top), block-Jacobi preconditioned CG to relative residual 1e-10 in
    three forms: FP64 with the split-form stencil operator (the default
    solve), FP64 with the difference-form operator, and FP32 matvecs with
    FP64 reliable updates (FP64 until the residual is below 0.1); device time
    of each solve, iterations and the difference of the solutions."""
    import numpy as np
    import torch
    import pdmtel_b200 as P
    from pdmtel_b200 import decks as D
    wd = os.path.join(tmp, f"cube{n}")
    D.config_cube(n=n, intg_point=1).write(wd)
    t0 = time.time()
    dm = P.pdDataManager(wd)
    dm.InitNode()
    dm.InitBond()
    dm.InitMaterial()
    ctx = dm.context()
    ctx.set_option(P.OPT_STATIC_PRECOND, int(bool(precond)))
    stencil = ctx.static_prepare()
    setup_s = time.time() - t0
    stream = torch.cuda.ExternalStream(ctx.stream)
    I = dm.info()
    res = {}
    for name, prec, sp in (("fp64_cg", P.PREC_FP64, split), ("fp64_cg_difference_form", P.PREC_FP64, 0),
                           ("fp32_ir", P.PREC_FP32C, split)):
        ctx.set_option(P.OPT_STATIC_SPLIT, sp)
        ctx.static_solve(1.0, precision=prec, rtol=1e-2, maxit=maxit)  # untimed: preconditioner, first launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        try:
            x, it, rr = ctx.static_solve(1.0, precision=prec, rtol=1e-10, maxit=maxit)
        except P.PdError:
            if maxit >= 100000:
                raise
            x, it, rr = np.zeros(3 * ctx.n), maxit, float("nan")  # capped on purpose
        e1.record(stream)
        e1.synchronize()
        res[name] = {"s": e0.elapsed_time(e1) / 1e3, "iterations": it, "rel_residual": rr, "x": x}
    ref = res["fp64_cg"]["x"]
    nref = max(np.linalg.norm(ref), 1e-300)
    for r in res.values():
        r["rel_diff_vs_fp64_cg"] = float(np.linalg.norm(r.pop("x") - ref) / nref)
        r["ms_per_iteration"] = 1e3 * r["s"] / max(r["iterations"], 1)
    out = {"workload": f"cube {n}^3, bottom clamped, 1 MPa shear traction on top", "nodes": I.num_nodes,
           "bond_halves": I.num_halves,
           "operator": (f"lattice stencil, split form, {split} nodes per thread" if split else
                        "lattice stencil, difference form") if stencil else "family lists",
           "preconditioner": "block Jacobi (3x3 diagonal blocks)" if precond else "none",
           **res, "setup_s": setup_s}
    dm.close()
    return out


def run_static(args):
    """--form static"""
    import torch
    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp(prefix="pdstatic_")
    r = static_solves(tmp, args.cube, args.maxit, precond=not args.no_precond, split=args.split)
    line = {"metric": f"static solve time to relative residual 1e-10, {args.cube}^3 cube",
            "value": r["fp64_cg"]["s"], "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": 1e3 * r["fp64_cg"]["s"], "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": r["workload"], "nodes": r["nodes"], "bond_halves": r["bond_halves"],
                       "operator": r["operator"], "preconditioner": r["preconditioner"]},
            **{k: r[k] for k in ("fp64_cg", "fp64_cg_difference_form", "fp32_ir", "setup_s")}}
    print(json.dumps(line))
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


def run_steps(args):
    """--form steps: device-resident RK4 steps of the plate and nothing else
    (the command profiler captures are taken on)."""
    import torch
    import pdmtel_b200 as P
    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp(prefix="pdsteps_")
    cfg = plate_cfg(args.plate_dims)
    dm, ctx, setup_s = setup_plate(tmp, cfg)
    prec = {"fp32c": P.PREC_FP32C, "fp64": P.PREC_FP64}[args.prec]
    ctx.set_precision(prec)
    tune = apply_shape(ctx, json.loads(args.shape)) if args.shape else (
        ctx.autotune(cfg["dt"], 5) if prec == P.PREC_FP32C else {})
    dt = cfg["dt"]
    ctx.reset_state()
    ctx.rk4_steps(dt, 0.0, args.warmup)
    ctx.sync()
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.rk4_steps(dt, args.warmup * dt, args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ev = 4 * ctx.evals_per_stage()
    print(json.dumps({"form": "steps", "workload": "plate {}x{}x{}".format(*cfg["dims"]), "prec": args.prec,
                      "nodes": ctx.n, "ms_per_step": ms / args.steps, "value": ev * args.steps / (ms / 1e3),
                      "unit": UNIT, "shape": tune, "setup_s": setup_s}))
    dm.close()
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


def ai_deck(dims):
    """The 20x10x10 bar of the plain-FP64 config with adaptive-trapezoid
    integration (ai_on, trapezoid index 3, MLS): left face held, right face
    pulled by a ramped displacement."""
    from pdmtel_b200 import decks as D
    h = 1e-3
    return D.Deck(dims=dims, spacing=h, horizon=3.015 * h, total_time=1.0, total_step=100, fixed_dt=1e-8,
                  bdry_eff=1, ai_mls=1, intg_point=3,
                  bcs=[D.BC(D.DISPL, (1, 1, 1), (0, 0, 0), 1.0, 2.0), D.BC(D.DISPL, (1, 1, 1), (2e-6, 0, 0), 2e-7, 1.0)],
                  bc_spaces=[D.Space(1, D.face_box(dims, h, 0, -1)), D.Space(2, D.face_box(dims, h, 0, +1))])


def ai_oracle_stage_seconds(dm, dims, trap=3):
    """One AI force stage of the oracle port (single thread) on the same deck:
    the CPU baseline of the AI form."""
    import ctypes as C
    import numpy as np
    import pdmtel_b200 as P
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as OL
    x, mat, bc = dm.nodes()
    rp, col, br = dm.family()
    cp, ci, _ = dm.mls()
    mats, bcs, _, _ = dm.tables()
    h = 1e-3
    ptr, regs = P.ai_plan(x, rp, col, h, 3.015 * h)
    tp, tc = P.ai_mls_table(x, rp, col, ptr, regs, h, 3.015 * h, trap, cp, ci, 3.0 * h)
    n = x.size // 3
    rng = np.random.default_rng(1)
    u = 1e-7 * rng.standard_normal(3 * n)
    m = OL.Model(n=n, x=x, dx=h, delta=3.015 * h, mls=1, npt=1, fam_ptr=rp, fam_col=col, broken=br,
                 cb_ptr=cp, cb_idx=ci, bdry_eff=dm.bdry_eff(), mat=mat, mat_spring=[q["spring"] for q in mats],
                 mat_ecrit=[q["ecrit"] for q in mats], mat_density=[q["density"] for q in mats],
                 mat_ymod=[72e9] * len(mats), bc=bc, bc_type=[b["type"] for b in bcs],
                 bc_dir=[d for b in bcs for d in b["dir"]], bc_val=[v for b in bcs for v in b["value"]],
                 bc_end=[b["end_time"] for b in bcs], bc_load=[b["load_type"] for b in bcs], U=u)
    L = OL.lib()
    L.or_ai_force_stage.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 6 + [C.c_double, C.c_double,
                                                                              C.c_void_p, C.c_void_p]
    brk = np.ascontiguousarray(br, np.uint8).copy()
    dmg = np.zeros(n, np.int32)
    k = np.zeros(3 * n)
    tp = np.ascontiguousarray(tp, np.int64)
    tc = np.ascontiguousarray(tc, np.float64)
    t0 = time.perf_counter()
    L.or_ai_force_stage(C.addressof(m.m), trap, ptr.ctypes.data, C.addressof(regs), tp.ctypes.data, tc.ctypes.data,
                        brk.ctypes.data, dmg.ctypes.data, 1e-8, 1e-8, u.ctypes.data, k.ctypes.data)
    return time.perf_counter() - t0


def run_ai(args):
    """--form ai: the adaptive-trapezoid (ai_on) form, FP64 drop-in, on the
    20x10x10 bar: W + K device RK4 steps (graph of one step), trapezoid-point
    force evaluations per second, against one stage of the oracle port."""
    import torch
    import pdmtel_b200 as P
    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp(prefix="pdai_")
    dims = (20, 10, 10)
    ai_deck(dims).write(tmp)
    t0 = time.perf_counter()
    dm = P.pdDataManager(tmp)
    P.pdSolve.InitialProblem(dm)
    ctx = dm.context()
    setup_s = time.perf_counter() - t0
    dt = 1e-8
    ctx.rk4_steps(dt, 0.0, args.warmup)
    ctx.sync()
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.rk4_steps(dt, args.warmup * dt, args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    pts = 4 * ctx.evals_per_stage()
    cpu_stage = None if args.no_cpu_baseline else ai_oracle_stage_seconds(dm, dims)
    line = {"form": "ai", "metric": "AI trapezoid-point force evaluations per second (FP64 drop-in)",
            "value": pts / (ms / 1e3), "unit": "point evals/s", "ms_per_step": ms, "steps": args.steps,
            "warmup": args.warmup, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "bar 20x10x10, spacing 1 mm, horizon 3.015 spacings, ai_on with MLS, "
                                   "trapezoid index 3", "nodes": ctx.n, "points_per_step": pts},
            "setup_s": setup_s}
    if cpu_stage is not None:
        line["cpu_baseline"] = {"value": pts / 4 / cpu_stage, "unit": "point evals/s", "cores": 1, "kind": "port",
                                "sample": "one force stage of the oracle port on the same deck",
                                "s_per_step": 4 * cpu_stage}
    print(json.dumps(line))
    dm.close()
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


def run_adjoint(args):
    """--form adjoint: the adjoint pair alone (profiler captures)."""
    import torch
    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp(prefix="pdadj_")
    res = adjoint_leg(tmp, args.adjoint_steps)
    print(json.dumps({"form": "adjoint", **res}))
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


def apply_shape(ctx, shape):
    """Sets the launch-shape options a pd_autotune result names (for runs
    whose timing must not depend on a tuner, e.g. under a profiler)."""
    import pdmtel_b200 as P
    opts = [("tile", P.OPT_TILE), ("gather_per_point", P.OPT_GATHER_PER_POINT), ("gather_sell", P.OPT_GATHER_SELL),
            ("gather_stencil", P.OPT_GATHER_STENCIL),
            ("force_stencil", P.OPT_FORCE_STENCIL),
            ("force_quad", P.OPT_FORCE_QUAD), ("force_tile", P.OPT_FORCE_TILE)]
    for key, opt in opts:
        if key in shape:
            ctx.set_option(opt, int(shape[key]))
    return dict(shape, applied=True)


def run_ours(args):
    import numpy as np
    import torch
    import pdmtel_b200 as P

    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    tmp = tempfile.mkdtemp(prefix=f"pdbench{rank}_")
    cfg = plate_cfg(args.plate_dims)
    dm, ctx, setup_s = setup_plate(tmp, cfg)
    dt = cfg["dt"]
    stream = torch.cuda.ExternalStream(ctx.stream)
    evals_stage = ctx.evals_per_stage()
    evals_step = 4 * evals_stage
    n = ctx.n

    def barrier():
        rank_barrier(ws)

    def timed(prec, sampler=None):
        ctx.set_precision(prec)
        ctx.reset_state()
        ctx.rk4_steps(dt, 0.0, args.warmup)
        ctx.sync()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.start()
            sampler.begin()
        e0.record(stream)
        ctx.rk4_steps(dt, args.warmup * dt, args.steps)
        e1.record(stream)
        e1.synchronize()
        if sampler:
            sampler.end()
        clocks = sampler.stop() if sampler else None
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), ws)
        U, V = ctx.get_state()
        return ms, U, V, clocks

    # launch shapes for this plate (pd_autotune: node order, gather and force
    # variants, persistent launch; state restored), or the shapes given
    ctx.set_precision(P.PREC_FP32C)
    if args.shape:
        tune = apply_shape(ctx, json.loads(args.shape))
    else:
        tune = ctx.autotune(dt, 5)
    sampler = ClockSampler(dev)
    ms32, U32, V32, clocks = timed(P.PREC_FP32C, sampler)
    ms64, U64, V64, _ = timed(P.PREC_FP64)
    err_u = float(np.linalg.norm(U32 - U64) / max(np.linalg.norm(U64), 1e-300))
    err_v = float(np.linalg.norm(V32 - V64) / max(np.linalg.norm(V64), 1e-300))

    # per-kernel device times of one step, FP32 form (events on the context stream)
    ctx.set_precision(P.PREC_FP32C)
    prof = np.zeros(4)
    reps = 3
    t = (args.warmup + args.steps) * dt
    for _ in range(reps):
        t += dt
        prof += ctx.profile_step(dt, t)
    prof /= reps
    ctx.set_precision(P.PREC_FP64)
    prof64 = ctx.profile_step(dt, t + dt)

    # end to end through the C ABI with host buffers
    ctx.set_precision(P.PREC_FP32C)
    ctx.reset_state()
    hU = torch.zeros(3 * n, dtype=torch.float64).pin_memory()
    hV = torch.zeros(3 * n, dtype=torch.float64).pin_memory()
    import ctypes as C
    pU = C.cast(hU.data_ptr(), C.POINTER(C.c_double))
    pV = C.cast(hV.data_ptr(), C.POINTER(C.c_double))
    L = P.lib()
    for k in range(args.warmup):
        L.pd_rk4_steps_host(ctx.h, dt, k * dt, 1, pU, pV, pU, pV)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        rc = L.pd_rk4_steps_host(ctx.h, dt, (args.warmup + k) * dt, 1, pU, pV, pU, pV)
        if rc != 0:
            raise P.PdError(rc, "pd_rk4_steps_host")
    e1.record(stream)
    e1.synchronize()
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), ws)

    I = dm.info()
    hbm_peak, peak_kind = load_peaks()
    peak32, sms, mhz = fp32_peak((clocks or {}).get("sm_max_mhz"))
    force_ms = prof[0] / 4.0  # one launch per stage
    gather_ms = prof[1] / 4.0
    npt = I.num_gauss
    ncb = I.num_contrib
    # the kernels the tuner kept
    sten = bool(tune.get("force_stencil"))
    force_kernel = ("k_force_f32c_sten" if sten else "k_force_f32c_quad" if tune.get("force_quad")
                    else "k_force_f32c_tiled" if tune.get("force_tile") else "k_force_f32c_pair")
    pat, sell = bool(tune.get("gather_stencil")), bool(tune.get("gather_sell"))
    gather_kernel = "k_gather_f32c_ring" if (pat and sell) else "k_gather_f32c"
    # coefficients, contributor ids (pattern ids instead with patterns), trial
    # displacement, output blocks, partition-of-unity sums, row pointers
    gather_bytes = (ncb * npt * 4 + (n * 4 if pat else ncb * 4 + (n + 1) * 8) + n * 8 * 4 + n * npt * 12
                    + n * npt * 4)
    force_flops = FLOP_PER_EVAL * evals_stage
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get("force_f32c_sten_bytes_per_launch" if sten else "force_f32c_bytes_per_launch")
    value = replica_throughput(ws, evals_step * args.steps, ms32 / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "plate {}x{}x{}, 2x2x2 Gauss+MLS, {:g} mm slit, +-0.05 m/s, dt 5e-9".format(
                       *cfg["dims"], 2e3 * cfg["slit_half_length"]),
                   "nodes": n, "bond_halves": I.num_halves, "broken_halves": I.num_broken,
                   "evals_per_step": evals_step, "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (MLS coefficients and family lists are GBs per step)",
                   "form": "FP32 forces + Kahan family sums, FP64 state"},
        "fp64": {"value": ws * evals_step * args.steps / (ms64 / 1e3), "ms_per_step": ms64 / args.steps,
                 "speedup_fp32c_over_fp64": ms64 / ms32},
        "rel_err_vs_fp64": {"U": err_u, "V": err_v, "after_steps": args.warmup + args.steps},
        "e2e": {"value": ws * evals_step * args.steps / (ms_e2e / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 2 * 3 * n * 8, "d2h_bytes_per_step": 2 * 3 * n * 8},
        # per step: 4 stages x (gather, force, epilogue) + the time advance;
        # the stencil force is two launches (series pass, exact pass)
        "gpu_launches": (13 + (4 if sten else 0)) * args.steps,
        "roofline": {"bound": "fp32", "kernel": force_kernel, "achieved": force_flops / (force_ms / 1e3) / 1e12,
                     "peak": peak32 / 1e12, "unit": "TFLOP/s",
                     "frac": force_flops / (force_ms / 1e3) / peak32, "traffic": traffic,
                     "peak_kind": f"nominal FP32 ({sms} SMs x {FP32_LANES_PER_SM} lanes x FMA x {mhz:.0f} MHz, "
                                  "the maximum SM clock); no measured FP32 peak",
                     "launch_ms": force_ms, "flop_per_launch": force_flops},
        "roofline_gather": {"bound": "hbm", "kernel": gather_kernel,
                            "achieved": gather_bytes / (gather_ms / 1e3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                            "frac": gather_bytes / (gather_ms / 1e3) / 1e9 / hbm_peak,
                            "peak_kind": peak_kind, "launch_ms": gather_ms, "bytes_per_launch": gather_bytes},
        "kernel_ms_per_step": {"fp32c": {"force": prof[0], "gather": prof[1], "epilogue": prof[2], "other": prof[3]},
                               "fp64": {"force": prof64[0], "gather": prof64[1], "epilogue": prof64[2],
                                        "other": prof64[3]}},
        "clocks": clocks, "setup_s": setup_s, "autotune": tune,
    }
    if rank == 0 and not args.no_accuracy_leg:
        line["rel_err_vs_fp64_long"] = accuracy_leg(ctx, dt)
    if rank == 0 and not args.no_adjoint:
        line["adjoint"] = adjoint_leg(tmp, args.adjoint_steps)
    if rank == 0 and not args.no_static:
        line["static"] = static_solves(tmp, args.cube)
    if rank == 0 and not args.no_cpu_baseline:
        outs = cpu_baseline_reference(1, 2, tmp)
        if outs:
            o = outs[0]
            line["cpu_baseline"] = {"value": o["evals_per_step"] / o["step_s"][-1], "unit": UNIT, "cores": 1,
                                    "kind": "reference", "same_config": False,
                                    "sample": "40x40x4 sub-plate of the workload (6,400 nodes, same spacing, "
                                              "horizon, material, Gauss + MLS and slit rule; a proxy for the "
                                              "640k-node plate), reference solver, 2nd RK4 step"}
        else:
            line["cpu_baseline"] = None
    if rank == 0:
        print(json.dumps(line))
    shutil.rmtree(tmp, ignore_errors=True)
    del ctx
    dm.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-accuracy-leg", action="store_true",
                    help="leave out the untimed 100/500-step FP32C-vs-FP64 error check of the headline line")
    ap.add_argument("--no-static", action="store_true", help="leave the static solve out of the headline line")
    ap.add_argument("--shape", default=None,
                    help="skip pd_autotune and apply these launch shapes, a JSON object with keys of its result "
                         "(tile, gather_per_point, gather_sell, gather_stencil, force_stencil, force_quad, "
                         "force_tile)")
    ap.add_argument("--adjoint-steps", type=int, default=100)
    ap.add_argument("--form", default="precision",
                    choices=["precision", "batch", "static", "identify", "accuracy", "steps", "adjoint", "ai"])
    ap.add_argument("--plate-dims", default="400x400x4", help="plate lattice of the precision/steps forms")
    ap.add_argument("--prec", default="fp32c", choices=["fp32c", "fp64"], help="arithmetic of --form steps")
    ap.add_argument("--cube", type=int, default=128, help="cube side of --form static")
    ap.add_argument("--split", type=int, default=4, choices=[0, 2, 4, 8],
                    help="nodes per thread of the split-form static operator (0: difference form)")
    ap.add_argument("--maxit", type=int, default=100000, help="CG iteration cap of --form static")
    ap.add_argument("--no-precond", action="store_true", help="--form static: plain CG, no block Jacobi")
    ap.add_argument("--ident-dims", default="64x64x8")
    ap.add_argument("--ident-steps", type=int, default=1000)
    ap.add_argument("--fd-dirs", type=int, default=32)
    ap.add_argument("--lbfgs-iters", type=int, default=50)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.form == "batch":
        return run_batch(args)
    if args.form == "static":
        return run_static(args)
    if args.form == "identify":
        return run_identify(args)
    if args.form == "accuracy":
        return run_accuracy(args)
    if args.form == "steps":
        return run_steps(args)
    if args.form == "adjoint":
        return run_adjoint(args)
    if args.form == "ai":
        return run_ai(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
