"""Differentiation form: the gradient of a functional of the final RK4 state
with respect to the per-node spring factors.

CPU: the oracle's reverse sweep (or_adjoint_grad) against central finite
differences of the oracle's own forward steps.  GPU: pd_adjoint_forward /
pd_adjoint_backward against that oracle gradient (forward bit for bit, the
gradient to 1e-10) and against central finite differences (h = 1e-6 in the
log-factor, 32 random directions, 1e-4 relative) of the device's steps.

The finite differences run in PD_PREC_FP64A: the reference's own extension
p - r cancels at the strains of these specimens (1e-5), which leaves a
rounding noise of about eps/strain in every force; at h = 1e-6 that noise
alone reaches 1e-4 of the difference quotient."""
import numpy as np
import pytest

import pdmtel_b200 as P
from conftest import deck_dir, load_golden, CASES
from golden_model import model_from_golden

FGI_CASES = ["fgi_velo", "fgi3_ramp", "fgi1_hole", "fgi_slit"]
# a step five times the decks' own, so that within a few dozen steps the
# waves cross the specimen and the state depends strongly on the stiffness
DT = 5e-8


def _factors(n, seed, sigma=0.2):
    rng = np.random.default_rng(seed)
    return np.exp(sigma * rng.standard_normal(n))


def _functional(n, seed):
    """J = a.U + b.V with random weights; dJ/dU = a, dJ/dV = b."""
    rng = np.random.default_rng(seed + 1000)
    return rng.standard_normal(3 * n), rng.standard_normal(3 * n)


def _oracle_final(g, f, nsteps, dt=DT):
    m = model_from_golden(g, spring_factor=f)
    t = 0.0
    for _ in range(nsteps):
        t += dt
        m.rk4_step(dt, t)
    return m.U.copy(), m.V.copy()


@pytest.mark.parametrize("name", ["fgi_velo", "fgi3_ramp", "fgi1_hole"])
def test_oracle_adjoint_matches_finite_differences(name):
    g = load_golden(name)
    n = int(g["n"][0])
    dt = DT
    nsteps = 24
    f = _factors(n, 1)
    a, b = _functional(n, 1)
    m = model_from_golden(g, spring_factor=f)
    grad = m.adjoint_grad(dt, 0.0, nsteps, a, b)
    # the forward inside the adjoint is the plain oracle step
    U, V = _oracle_final(g, f, nsteps)
    assert np.array_equal(m.U, U) and np.array_equal(m.V, V)
    assert np.abs(grad).max() > 0
    rng = np.random.default_rng(7)
    # h = 1e-4: truncation O(h^2) and rounding O(eps/h) both near 1e-8
    h = 1e-4
    for _ in range(3):
        v = rng.standard_normal(n)
        Up, Vp = _oracle_final(g, f * np.exp(h * v), nsteps)
        Um, Vm = _oracle_final(g, f * np.exp(-h * v), nsteps)
        fd = (a @ (Up - Um) + b @ (Vp - Vm)) / (2 * h)
        an = (grad * f) @ v
        assert abs(fd - an) <= 1e-5 * abs(an), (fd, an)


# ------------------------------------------------------------------ GPU


def _gpu_ctx(name):
    dm = P.pdDataManager(deck_dir(name) if name in CASES else name)
    P.pdSolve.InitialProblem(dm)
    return dm, dm.context()


def _gpu_final(ctx, f, dt, nsteps):
    ctx.set_spring_factor(f)
    ctx.reset_state()
    ctx.rk4_steps(dt, 0.0, nsteps)
    ctx.sync()
    return ctx.get_state()


@pytest.mark.gpu
@pytest.mark.parametrize("name", FGI_CASES)
def test_device_adjoint_matches_oracle_gradient(name):
    g = load_golden(name)
    n = int(g["n"][0])
    dt = DT
    nsteps, every = 10, 3  # segments of 3, 3, 3 and 1 steps
    f = _factors(n, 2)
    a, b = _functional(n, 2)
    grad_or = model_from_golden(g, spring_factor=f).adjoint_grad(dt, 0.0, nsteps, a, b)
    dm, ctx = _gpu_ctx(name)
    ctx.set_spring_factor(f)
    ctx.reset_state()
    ctx.adjoint_forward(dt, 0.0, nsteps, every)
    U, V = ctx.get_state()
    Uo, Vo = _oracle_final(g, f, nsteps)
    assert np.array_equal(U, Uo) and np.array_equal(V, Vo)
    grad = ctx.adjoint_backward(a, b)
    err = np.linalg.norm(grad - grad_or) / np.linalg.norm(grad_or)
    assert err <= 1e-10, err
    # the state is back at the start of the forward run
    U0, V0 = ctx.get_state()
    assert not U0.any() and not V0.any()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fgi_velo", "fgi3_ramp", "fgi_slit"])
def test_fp32c_adjoint_matches_fp64_gradient(name):
    """The adjoint of the FP32-compensated form: FP32C forward steps (the
    FP32C trajectory bit for bit) and segment recompute, reverse sweep with
    FP64 point terms on that tape (default) or FP32 ones
    (PD_OPT_ADJOINT_VJP32).  Its gradient agrees with the FP64 adjoint's to
    1e-5 (1e-3 with FP32 point terms), and it leaves the state and the node
    blocks the next FP32C step reads at the start of the forward run."""
    g = load_golden(name)
    n = int(g["n"][0])
    dt = DT
    nsteps, every = 10, 3
    f = _factors(n, 3)
    a, b = _functional(n, 3)
    dm, ctx = _gpu_ctx(name)
    ctx.set_energy(False)
    ctx.set_spring_factor(f)
    ctx.set_precision(P.PREC_FP64)
    ctx.reset_state()
    ctx.adjoint_forward(dt, 0.0, nsteps, every)
    g64 = ctx.adjoint_backward(a, b)
    ctx.set_precision(P.PREC_FP32C)
    U32, V32 = _gpu_final(ctx, f, dt, nsteps)
    for vjp32, bar in ((0, 1e-5), (1, 1e-3)):
        ctx.set_option(P.OPT_ADJOINT_VJP32, vjp32)
        ctx.reset_state()
        ctx.adjoint_forward(dt, 0.0, nsteps, every)
        U, V = ctx.get_state()
        assert np.array_equal(U, U32) and np.array_equal(V, V32)
        g32 = ctx.adjoint_backward(a, b)
        err = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
        assert err <= bar, (vjp32, err)
        U0, V0 = ctx.get_state()
        assert not U0.any() and not V0.any()
        # a forward run after the reverse sweep repeats the first one
        ctx.adjoint_forward(dt, 0.0, nsteps, every)
        U2, V2 = ctx.get_state()
        assert np.array_equal(U2, U32) and np.array_equal(V2, V32)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fgi_velo", "fgi3_ramp"])
def test_device_adjoint_matches_finite_differences(name):
    g = load_golden(name)
    n = int(g["n"][0])
    dt = DT
    nsteps, every = 40, 7
    f = _factors(n, 3)
    a, b = _functional(n, 3)
    dm, ctx = _gpu_ctx(name)
    ctx.set_precision(P.PREC_FP64A)
    ctx.set_spring_factor(f)
    ctx.reset_state()
    ctx.adjoint_forward(dt, 0.0, nsteps, every)
    grad = ctx.adjoint_backward(a, b)
    rng = np.random.default_rng(11)
    h = 1e-6
    worst = 0.0
    for _ in range(32):
        v = rng.standard_normal(n)
        Up, Vp = _gpu_final(ctx, f * np.exp(h * v), dt, nsteps)
        Um, Vm = _gpu_final(ctx, f * np.exp(-h * v), dt, nsteps)
        fd = (a @ (Up - Um) + b @ (Vp - Vm)) / (2 * h)
        an = (grad * f) @ v
        worst = max(worst, abs(fd - an) / abs(an))
    assert worst <= 1e-4, worst


@pytest.mark.gpu
def test_identification_gradient_and_fit(tmp_path):
    """A small identification specimen (fixed face, pulled face): the
    misfit gradient against finite differences along smooth random
    directions, then a few L-BFGS iterations lower the misfit."""
    import torch
    from pdmtel_b200 import adjoint as AD
    from pdmtel_b200 import decks as D
    dt, nsteps = 1e-8, 200
    D.config_identify(dims=(16, 8, 4), dt=dt, steps=nsteps).write(str(tmp_path))
    dm, ctx = _gpu_ctx(str(tmp_path))
    ctx.set_precision(P.PREC_FP64A)
    x, _, _ = dm.nodes()
    n = ctx.n
    m_true = AD.gaussian_random_field(x, 1e-3, 2e-3, 0.2, seed=1)
    U_true, _ = _gpu_final(ctx, np.exp(m_true), dt, nsteps)
    rng = np.random.default_rng(2)
    U_obs = U_true + 1e-3 * np.sqrt(np.mean(U_true ** 2)) * rng.standard_normal(U_true.shape)
    m0 = torch.zeros(n, dtype=torch.float64, requires_grad=True)
    U, _ = AD.trajectory(m0, ctx, dt, nsteps, every=50)
    loss = AD.misfit(U, torch.from_numpy(U_obs.reshape(n, 3)))
    loss.backward()
    g = m0.grad.numpy()
    Uo = U_obs.reshape(-1)

    def J(m):
        Uf, _ = _gpu_final(ctx, np.exp(m), dt, nsteps)
        return 0.5 * np.sum((Uf - Uo) ** 2) / np.sum(Uo ** 2)

    h = 1e-6
    for k in range(8):
        v = AD.gaussian_random_field(x, 1e-3, 2e-3, 1.0, seed=100 + k)
        fd = (J(h * v) - J(-h * v)) / (2 * h)
        assert abs(fd - g @ v) <= 1e-4 * abs(g @ v), (k, fd, g @ v)
    res = AD.identify(ctx, U_obs, dt, nsteps, iters=5, every=50)
    assert res.loss[-1] < 0.5 * res.loss[0], res.loss


@pytest.mark.gpu
def test_adjoint_rejects_misuse():
    dm, ctx = _gpu_ctx("fgi_velo")
    n = ctx.n
    with pytest.raises(P.PdError):
        ctx.adjoint_backward(np.zeros(3 * n))  # no forward run yet
    with pytest.raises(P.PdError):
        ctx.set_spring_factor(-np.ones(n))
    dmc, cctx = _gpu_ctx("cci_grad")
    with pytest.raises(P.PdError):
        cctx.adjoint_forward(1e-8, 0.0, 2, 1)  # CCI is not covered


# ------------------------------------------------- host-side plumbing (CPU)


class _LinearDevice:
    """Stands in for a DeviceContext: U = A f, V = B f (f the spring
    factors), so the autograd wrapper and the L-BFGS loop run without a GPU."""

    def __init__(self, n, seed=0):
        rng = np.random.default_rng(seed)
        self.n = n
        self.A = rng.standard_normal((3 * n, n)) / n
        self.B = rng.standard_normal((3 * n, n)) / n
        self.f = np.ones(n)
        self.forwards = 0

    def set_spring_factor(self, f):
        self.f = np.asarray(f, dtype=np.float64).copy()

    def reset_state(self):
        pass

    def adjoint_forward(self, dt, t0, nsteps, every):
        self.forwards += 1

    def get_state(self):
        return self.A @ self.f, self.B @ self.f

    def adjoint_backward(self, lu, lv=None):
        g = self.A.T @ lu
        if lv is not None:
            g = g + self.B.T @ lv
        return g


def test_trajectory_autograd_chain_rule():
    import torch
    from pdmtel_b200 import adjoint as AD
    dev = _LinearDevice(20)
    m = torch.tensor(np.random.default_rng(1).standard_normal(20) * 0.1, requires_grad=True)
    U, V = AD.trajectory(m, dev, 1e-8, 5)
    w = torch.tensor(np.random.default_rng(2).standard_normal((20, 3)))
    loss = (w * U).sum() + (V ** 2).sum()
    loss.backward()
    f = np.exp(m.detach().numpy())
    Vn = dev.B @ f
    expect = (dev.A.T @ w.numpy().reshape(-1) + dev.B.T @ (2 * Vn)) * f
    assert np.allclose(m.grad.numpy(), expect, rtol=1e-12, atol=0)


def test_trajectory_backward_refuses_a_stale_forward():
    import torch
    from pdmtel_b200 import adjoint as AD
    dev = _LinearDevice(8)
    m = torch.zeros(8, dtype=torch.float64, requires_grad=True)
    U1, _ = AD.trajectory(m, dev, 1e-8, 2)
    AD.trajectory(m, dev, 1e-8, 2)
    with pytest.raises(RuntimeError):
        U1.sum().backward()


def test_identify_recovers_a_linear_model():
    from pdmtel_b200 import adjoint as AD
    dev = _LinearDevice(12, seed=3)
    m_true = np.random.default_rng(4).standard_normal(12) * 0.2
    U_obs = dev.A @ np.exp(m_true)
    res = AD.identify(dev, U_obs, 1e-8, 3, iters=50)
    assert res.loss[-1] < 1e-12 * max(res.loss[0], 1e-300) or res.loss[-1] < 1e-20
    assert res.evaluations == dev.forwards


def test_gaussian_random_field_statistics():
    from pdmtel_b200 import adjoint as AD
    dims = (48, 48, 8)
    ijk = np.stack(np.meshgrid(*[np.arange(d) for d in dims], indexing="ij"), -1).reshape(-1, 3)
    x = ijk * 1e-3
    z = AD.gaussian_random_field(x, 1e-3, 5e-3, 0.2, seed=0)
    assert z.shape == (len(x),)
    assert abs(z.std() - 0.2) < 1e-12 and abs(z.mean()) < 1e-12
    grid = z.reshape(dims)
    # neighbours one spacing apart are strongly correlated, 15 apart barely
    c1 = np.corrcoef(grid[:-1].ravel(), grid[1:].ravel())[0, 1]
    c15 = np.corrcoef(grid[:-15].ravel(), grid[15:].ravel())[0, 1]
    assert c1 > 0.9 and abs(c15) < 0.3
    # the same seed gives the same field
    assert np.array_equal(z, AD.gaussian_random_field(x, 1e-3, 5e-3, 0.2, seed=0))
