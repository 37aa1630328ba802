"""Batching form: many independent specimens of uneven size stepped together.

No counterpart in the reference, which runs one deck per process.  Each
specimen is an ordinary deck (a box lattice with one face fixed and the
opposite face pulled, 2x2x2 Gauss points with MLS) and carries a per-node
micromodulus factor f = exp(sigma z), z a unit Gaussian random field seeded
per specimen.  ``pdDataManager.batch`` places the specimens side by side on
one lattice, far enough apart that no bond joins two of them, so one device
context holds all of them: every kernel launch (or the one persistent launch
of ``pd_rk4_steps_persistent``) advances every specimen, whatever its size.
``pd_autotune`` picks the launch shapes on the batch itself.

``specimen_contexts`` cuts per-specimen contexts out of the batch with the
same coordinates, tables, family and MLS data: stepping them one after the
other is the "one launch per specimen" comparison, and gives the same numbers
bit for bit.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import DeviceContext, PREC_FP32C, pdDataManager
from .adjoint import gaussian_random_field
from .decks import config_identify


def draw_dims(count: int, seed: int, nmin: int = 1000, nmax: int = 60000, amin: float = 1.0,
              amax: float = 4.0) -> List[Tuple[int, int, int]]:
    """Box lattices whose node counts are log-uniform in [nmin, nmax] and
    whose axis aspect factors are uniform in [amin, amax]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        a = rng.uniform(amin, amax, size=3)
        s = (n / float(np.prod(a))) ** (1.0 / 3.0)
        out.append(tuple(int(max(2, round(s * v))) for v in a))
    return out


@dataclass
class BatchSpec:
    dims: Sequence[Tuple[int, int, int]]
    spacing: float = 1e-3
    vel: float = 0.05
    dt: float = 1e-8
    sigma: float = 0.15
    corr_cells: float = 4.0
    seed: int = 0


class Batch:
    """Writes one deck per specimen under ``workdir``, opens them, draws
    their micromodulus fields and assembles the batch model (device bond
    search, per-specimen MLS)."""

    def __init__(self, workdir: str, spec: BatchSpec, precision: int = PREC_FP32C, device_setup: bool = False):
        self.spec = spec
        self.specimens: List[pdDataManager] = []
        self.factors: List[np.ndarray] = []
        h = spec.spacing
        for k, dims in enumerate(spec.dims):
            d = os.path.join(workdir, f"specimen_{k:04d}")
            config_identify(dims=tuple(dims), spacing=h, vel=spec.vel, dt=spec.dt, steps=1).write(d)
            m = pdDataManager(d)
            m.InitNode()
            x, _, _ = m.nodes()
            z = gaussian_random_field(x, h, spec.corr_cells * h, 1.0, seed=spec.seed * 100003 + k)
            f = np.exp(spec.sigma * z)
            m.SetSpringFactor(f)
            self.specimens.append(m)
            self.factors.append(f)
        self.model = pdDataManager.batch(os.path.join(workdir, "batch"), self.specimens)
        self.model.InitBond()
        # device_setup: every specimen's MLS solved on the device (pd_mls_setup,
        # each in its own frame) instead of on the host
        self.model.SetDeviceSetup(device_setup)
        self.model.InitIntegrationPoint()
        self.model.SetPrecision(precision)
        self.ctx = self.model.context()
        self.ctx.set_energy(False)
        self.offsets = self.model.batch_offsets()
        self.persistent = False

    @property
    def num_specimens(self) -> int:
        return len(self.offsets) - 1

    def evals_per_step(self) -> int:
        return 4 * self.ctx.evals_per_stage()

    def tune(self, steps: int = 3) -> dict:
        r = self.ctx.autotune(self.spec.dt, steps)
        self.persistent = bool(r["persistent"])
        return r

    def run(self, nsteps: int, t0: float = 0.0, persistent: Optional[bool] = None):
        """nsteps RK4 steps of every specimen: one persistent launch, or the
        graph of one step replayed (the tuner's choice unless given)."""
        use = self.persistent if persistent is None else persistent
        if use:
            self.ctx.rk4_steps_persistent(self.spec.dt, t0, nsteps)
        else:
            self.ctx.rk4_steps(self.spec.dt, t0, nsteps)
            self.ctx.sync()

    def specimen_state(self, U, k: int):
        o = self.offsets
        return np.asarray(U).reshape(-1, 3)[o[k]:o[k + 1]]

    def specimen_contexts(self, precision: int = PREC_FP32C) -> List[DeviceContext]:
        """One device context per specimen, cut out of the batch: same
        coordinates, material and BC tables, family, MLS data and factors."""
        m = self.model
        I = m.info()
        x, mat, bc = m.nodes()
        x = x.reshape(-1, 3)
        rp, col, br = m.family()
        cp, ci, co = m.mls()
        mats, bcs, ab, wt = m.tables()
        sf = np.concatenate(self.factors)
        out = []
        npt = I.num_gauss
        for k in range(self.num_specimens):
            a, b = int(self.offsets[k]), int(self.offsets[k + 1])
            ctx = DeviceContext.create(x[a:b].reshape(-1), mat[a:b], mats, bcs, bc[a:b], I.grid_spacing, I.horizon,
                                       integration=1, cci_modified=0, intg_point=I.intg_point, abscissae=ab,
                                       weights=wt, damping=I.damping, spring_factor=sf[a:b])
            ctx.set_family(rp[a:b + 1] - rp[a], col[rp[a]:rp[b]] - a, br[rp[a]:rp[b]])
            ctx.set_bdry_eff(np.ones(b - a))
            ctx.set_mls(cp[a:b + 1] - cp[a], ci[cp[a]:cp[b]] - a, co[cp[a] * npt:cp[b] * npt])
            ctx.set_precision(precision)
            ctx.set_energy(False)
            out.append(ctx)
        return out
