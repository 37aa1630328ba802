"""Differentiation form: identifying a per-node micromodulus field from
displacements.

No counterpart in the reference, whose spring constant is per material with
the min(c_i, c_j) pair rule (pdDataManager.cpp:1926).  Here each node carries
a log-micromodulus m_i; the pair constant of a bond is
min(c_i, c_j) * (exp(m_i) + exp(m_j)) / 2, smooth in m.

The trajectory is the reference's RK4 scheme in FP64 on the device
(pd_adjoint_forward, checkpoints every `every` steps); its vector-Jacobian
product is pd_adjoint_backward (a reverse sweep over the checkpointed
segments, each recomputed once).  `Trajectory` wraps the pair as a
torch.autograd.Function so that any torch-expressed loss of the final state
differentiates back to m.  torch is used here only for the autograd
bookkeeping and the L-BFGS loop; every step and every gradient runs in the
library's CUDA kernels.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import DeviceContext


def lattice_index(coords, spacing):
    """Integer lattice positions [N, 3] of nodes on a cubic lattice."""
    x = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
    return np.rint((x - x.min(axis=0)) / spacing).astype(np.int64)


def gaussian_random_field(coords, spacing, corr_len, sigma, seed):
    """A stationary Gaussian random field on the nodes of a cubic lattice:
    white noise smoothed by a Gaussian kernel (covariance
    exp(-d^2 / (2 corr_len^2)), corr_len in length units) by FFT over a
    padded box, scaled to standard deviation sigma."""
    ijk = lattice_index(coords, spacing)
    dims = ijk.max(axis=0) + 1
    ell = corr_len / spacing
    pad = int(np.ceil(3 * ell))
    shape = tuple(int(d) + 2 * pad for d in dims)
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    # the kernel whose self-convolution is the covariance: width ell/sqrt(2)
    freqs = np.meshgrid(*[np.fft.fftfreq(s) for s in shape], indexing="ij")
    k2 = sum(f * f for f in freqs) * (2 * np.pi) ** 2
    kern = np.exp(-0.25 * ell * ell * k2)
    z = np.real(np.fft.ifftn(np.fft.fftn(w) * kern))
    z = z[pad:pad + dims[0], pad:pad + dims[1], pad:pad + dims[2]]
    z = (z - z.mean()) / z.std()
    return sigma * z[ijk[:, 0], ijk[:, 1], ijk[:, 2]]


class Trajectory(torch.autograd.Function):
    """(m) -> (U, V) after nsteps RK4 steps from rest; backward through
    pd_adjoint_backward.  One pending forward per context: the backward must
    follow its own forward before the next forward on that context."""

    @staticmethod
    def forward(ctx, m, dev: DeviceContext, dt: float, nsteps: int, every: int):
        f = np.exp(m.detach().cpu().numpy().astype(np.float64))
        dev.set_spring_factor(f)
        dev.reset_state()
        dev.adjoint_forward(dt, 0.0, nsteps, every)
        U, V = dev.get_state()
        dev._adjoint_token = getattr(dev, "_adjoint_token", 0) + 1
        ctx.dev = dev
        ctx.token = dev._adjoint_token
        ctx.f = f
        n = dev.n
        return (torch.from_numpy(U.reshape(n, 3)).to(m.device),
                torch.from_numpy(V.reshape(n, 3)).to(m.device))

    @staticmethod
    def backward(ctx, gU, gV):
        dev = ctx.dev
        if dev._adjoint_token != ctx.token:
            raise RuntimeError("Trajectory.backward: another forward ran on this context since")
        lu = gU.detach().cpu().numpy().astype(np.float64).reshape(-1)
        lv = None if gV is None else gV.detach().cpu().numpy().astype(np.float64).reshape(-1)
        g = dev.adjoint_backward(lu, lv)
        gm = torch.from_numpy(g * ctx.f).to(gU.device)
        return gm, None, None, None, None


def trajectory(m: torch.Tensor, dev: DeviceContext, dt: float, nsteps: int, every: int = 50):
    return Trajectory.apply(m, dev, dt, nsteps, every)


def misfit(U: torch.Tensor, U_obs: torch.Tensor) -> torch.Tensor:
    """0.5 * ||U - U_obs||^2 / ||U_obs||^2"""
    return 0.5 * ((U - U_obs) ** 2).sum() / (U_obs ** 2).sum()


@dataclass
class FitResult:
    m: np.ndarray
    loss: List[float] = field(default_factory=list)
    evaluations: int = 0
    seconds: float = 0.0


def identify(dev: DeviceContext, U_obs, dt: float, nsteps: int, m0=None, iters: int = 50, every: int = 50,
             reg: float = 0.0, history_size: int = 10, callback=None) -> FitResult:
    """L-BFGS (strong-Wolfe line search) on the misfit of the final
    displacements, plus reg * 0.5 * ||m||^2 / N, over the log-micromodulus."""
    n = dev.n
    U_obs = torch.as_tensor(np.asarray(U_obs, dtype=np.float64).reshape(n, 3))
    m = torch.zeros(n, dtype=torch.float64) if m0 is None else torch.tensor(np.asarray(m0, np.float64))
    m.requires_grad_(True)
    opt = torch.optim.LBFGS([m], lr=1.0, max_iter=iters, history_size=history_size,
                            line_search_fn="strong_wolfe", tolerance_grad=0.0, tolerance_change=0.0)
    res = FitResult(m=None)
    t0 = time.perf_counter()

    def closure():
        opt.zero_grad()
        U, _ = trajectory(m, dev, dt, nsteps, every)
        loss = misfit(U, U_obs)
        if reg:
            loss = loss + reg * 0.5 * (m ** 2).sum() / n
        loss.backward()
        res.evaluations += 1
        res.loss.append(float(loss.detach()))
        if callback is not None:
            callback(res)
        return loss

    opt.step(closure)
    res.seconds = time.perf_counter() - t0
    res.m = m.detach().numpy().copy()
    return res
