"""The plain-FP64 config on the device against the reference: the 20x10x10
bar (spacing 1 mm, horizon 3.015 mm, 2x2x2 Gauss points with MLS, fixed left
face, pulled right face, dt 1e-8 s) with the boundary-effect factor off and
on, 100 RK4 steps from rest.  Family lists, boundary-effect factors, MLS
coefficients, the stage-1 force at a non-trivial displacement and the state
every 10 steps are compared bit for bit with the reference's (energies, which
the device sums as a tree, to 1e-12), with both FP64 force kernels.  The
decks hold full 250-node families and nodes of all three branches of the
boundary-effect factor."""
import numpy as np
import pytest

import pdmtel_b200 as P
from long_golden import LONG_CASES, load_long, long_deck, same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lanes", [True, False], ids=["8-lane", "thread-per-node"])
@pytest.mark.parametrize("name", LONG_CASES)
def test_bar_100_steps_bit_exact(name, lanes):
    g = load_long(name)
    dm = P.pdDataManager(long_deck(name))
    P.pdSolve.InitialProblem(dm)
    rp, col, br = dm.family()
    assert np.array_equal(rp, g["fam_ptr"]) and same(col, g["sha_fam_col"])
    assert same(br.astype(np.int32), g["sha_broken"])
    assert dm.info().min_bond_length == g["min_bond"][0]
    assert np.array_equal(dm.bdry_eff(), g["bdry_eff"])
    cp, ci, co = dm.mls()
    assert np.array_equal(cp, g["cb_ptr"]) and same(ci, g["sha_cb_idx"]) and same(co, g["sha_coeff"])
    ctx = dm.context()
    # 8 lanes per node is the default below 131,072 nodes; 0 forces one thread per node
    ctx.set_option(P.OPT_F64_LANES_BELOW, 1 << 30 if lanes else 0)
    t, dts = g["force_args"]
    ctx.set_state(g["u_test"], g["v_test"])
    ctx.init_dynamic()
    ctx.gather(t, g["u_test"])
    assert same(ctx.get_gauss_displ(), g["sha_ug_force"])
    k = ctx.force_stage(dts, t, g["u_test"])
    assert np.array_equal(k, g["k"])
    assert np.array_equal(ctx.get_vbuf(), g["vbuf"])
    assert np.array_equal(ctx.get_energy_density(), g["eed"])
    ctx.reset_state()
    dt = g["dt"][0]
    for it in range(1, 101):
        ke, ee = ctx.rk4_step(dt, g["times"][it - 1])
        assert ke == pytest.approx(g["ke"][it - 1], rel=1e-12, abs=1e-300)
        assert ee == pytest.approx(g["ee"][it - 1], rel=1e-12, abs=1e-300)
        if it % 10 == 0:
            U, V = ctx.get_state()
            if f"U_{it}" in g:
                assert np.array_equal(U, g[f"U_{it}"]) and np.array_equal(V, g[f"V_{it}"])
            assert same(U, g[f"sha_U_{it}"]) and same(V, g[f"sha_V_{it}"]), it
            assert same(ctx.get_gauss_displ(), g[f"sha_ug_{it}"]), it
    assert np.abs(g["U_100"]).max() > 0


@pytest.mark.parametrize("name", LONG_CASES)
def test_bar_fp32c_within_1e6_after_100_steps(name):
    """The precision form on the same decks: relative displacement error
    against the reference's FP64 trajectory after 100 steps."""
    g = load_long(name)
    dm = P.pdDataManager(long_deck(name))
    dm.SetPrecision(P.PREC_FP32C)
    P.pdSolve.InitialProblem(dm)
    ctx = dm.context()
    ctx.rk4_steps(g["dt"][0], 0.0, 100)
    ctx.sync()
    U, V = ctx.get_state()
    eu = np.linalg.norm(U - g["U_100"]) / np.linalg.norm(g["U_100"])
    ev = np.linalg.norm(V - g["V_100"]) / np.linalg.norm(g["V_100"])
    assert eu <= 1e-6, eu
    assert ev <= 1e-5, ev
