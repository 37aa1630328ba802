"""Adaptive-trapezoid (AI, ai_on) integration, pdIntgManager types 1-3.

Golden fixtures tests/golden/ai/*.npz come from the reference itself
(tests/golden/make_golden.py --ai): one force stage from the harness's test
fields and a few RK4 steps, with the bonds the stage broke.

CPU: the planner (pd_ai_plan, pd_ai_mls_table, host only) feeding the
oracle's restatement of the nested trapezoid rule reproduces the reference's
stage bit for bit.  GPU: the device path, through the deck and the C ABI,
reproduces the same stage and the trajectory bit for bit.
"""
import ctypes as C
import glob
import os

import numpy as np
import pytest

import pdmtel_b200 as P
import oracle_lib as OL
from conftest import GOLDEN
from golden_model import model_from_golden, params

AI_DIR = os.path.join(GOLDEN, "ai")
AI_CASES = sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(AI_DIR, "*.npz")))


def load_ai(name):
    with np.load(os.path.join(AI_DIR, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def plan(g):
    Pm = params(g)
    ptr, regs = P.ai_plan(g["coords"], g["fam_ptr"], g["fam_col"], Pm["dx"], Pm["delta"])
    tab = (None, None)
    if Pm["mls"]:
        tab = P.ai_mls_table(g["coords"], g["fam_ptr"], g["fam_col"], ptr, regs, Pm["dx"], Pm["delta"],
                             Pm["intg_point"], g["cb_ptr"], g["cb_idx"], Pm["rw"])
    return ptr, regs, tab


def oracle_stage(g, m, trap, ptr, regs, tab, dts, t, us, broken):
    L = OL.lib()
    L.or_ai_force_stage.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 6 + [C.c_double, C.c_double,
                                                                              C.c_void_p, C.c_void_p]
    n = int(g["n"][0])
    brk = np.ascontiguousarray(broken, np.uint8).copy()
    dmg = np.zeros(n, np.int32)
    us = np.ascontiguousarray(us, np.float64)
    k = np.zeros(3 * n)
    tp = np.zeros(n + 1, np.int64) if tab[0] is None else np.ascontiguousarray(tab[0], np.int64)
    tc = np.zeros(1) if tab[1] is None else np.ascontiguousarray(tab[1], np.float64)
    L.or_ai_force_stage(C.addressof(m.m), trap, ptr.ctypes.data, C.addressof(regs), tp.ctypes.data, tc.ctypes.data,
                        brk.ctypes.data, dmg.ctypes.data, dts, t, us.ctypes.data, k.ctypes.data)
    return k, brk, dmg


def oracle_model(g, **kw):
    n = int(g["n"][0])
    return model_from_golden(g, coeff=None, xg=np.zeros(3 * n), npt=1, **kw)


@pytest.mark.parametrize("name", AI_CASES)
def test_plan_and_oracle_stage_match_reference(name):
    g = load_ai(name)
    t, dts = g["force_args"]
    ptr, regs, tab = plan(g)
    assert len(ptr) == len(g["fam_col"]) + 1 and ptr[-1] > 0
    m = oracle_model(g, U=g["u_test"], V=g["v_test"])
    m.vbuf[:] = g["v_test"]
    k, brk, dmg = oracle_stage(g, m, params(g)["intg_point"], ptr, regs, tab, dts, t, g["u_test"], g["broken"])
    assert np.array_equal(k, g["k"])
    assert np.array_equal(m.vbuf, g["vbuf"])
    assert np.array_equal(m.eed, g["eed"])
    assert np.array_equal(brk.astype(np.int32), g["broken_after"])
    assert np.array_equal(dmg, g["dmg"])


def test_break_case_breaks_bonds():
    """the critical-stretch fixture exercises the break path in the stage"""
    if "ai_break" not in AI_CASES:
        pytest.skip("no ai_break fixture")
    g = load_ai("ai_break")
    assert g["broken_after"].sum() > g["broken"].sum() and g["dmg"].sum() > 0


def test_plan_regions_are_valid():
    g = load_ai(AI_CASES[0])
    ptr, regs, _ = plan(g)
    n = ptr[-1]
    for r in range(n):
        R = regs[r]
        assert sorted(R.axis) == [0, 1, 2]
        for q in range(2):
            assert R.lim[q] < 6 or 8 <= R.lim[q] < 44
        for q in range(2, 4):
            assert R.lim[q] < 6 or 8 <= R.lim[q] < 14


def gpu_model(name):
    dm = P.pdDataManager(os.path.join(GOLDEN, "decks", name))
    P.pdSolve.InitialProblem(dm)
    return dm


@pytest.mark.gpu
@pytest.mark.parametrize("name", AI_CASES)
def test_device_stage_bit_exact(name):
    g = load_ai(name)
    t, dts = g["force_args"]
    dm = gpu_model(name)
    rp, col, br = dm.family()
    assert np.array_equal(rp, g["fam_ptr"]) and np.array_equal(col, g["fam_col"])
    assert np.array_equal(dm.bdry_eff(), g["bdry_eff"])
    ctx = dm.context()
    ctx.set_state(g["u_test"], g["v_test"])
    ctx.init_dynamic()
    ctx.gather(t, g["u_test"])
    k = ctx.force_stage(dts, t, g["u_test"])
    assert np.array_equal(k, g["k"])
    assert np.array_equal(ctx.get_vbuf(), g["vbuf"])
    assert np.array_equal(ctx.get_energy_density(), g["eed"])
    brk, cnt = ctx.get_damage(len(col))
    assert np.array_equal(brk.astype(np.int32), g["broken_after"])
    assert np.array_equal(cnt, g["dmg"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", [c for c in AI_CASES])
def test_device_trajectory_bit_exact(name):
    g = load_ai(name)
    if "traj_times" not in g:
        pytest.skip("no trajectory in this fixture")
    dm = gpu_model(name)
    ctx = dm.context()
    dt = g["dt"][0]
    H = len(g["fam_col"])
    for it, t in enumerate(g["traj_times"], start=1):
        ke, ee = ctx.rk4_step(dt, t)
        assert ke == pytest.approx(g["traj_ke"][it - 1], rel=1e-12, abs=1e-300)
        assert ee == pytest.approx(g["traj_ee"][it - 1], rel=1e-12, abs=1e-300)
        if f"traj_U_{it}" in g:
            U, V = ctx.get_state()
            assert np.array_equal(U, g[f"traj_U_{it}"])
            assert np.array_equal(V, g[f"traj_V_{it}"])
            brk, _ = ctx.get_damage(H)
            assert np.array_equal(brk.astype(np.int32), g[f"traj_broken_{it}"])


@pytest.mark.gpu
def test_device_without_mls_matches_oracle(tmp_path):
    """ai_on 1 0: every node carries a displacement gradient and eta = G xi
    (pdIntgManager2.cpp:211-235).  The reference's RK4 crashes on this form
    (a zero-length contributor array deleted through its element 0), so the
    oracle is the pin."""
    from pdmtel_b200 import decks as D
    h = 1e-3
    g0 = D.BC(D.DISPLGRAD, (0, 0, 0), (1e-4, 2e-5, 0, 0, -3e-5, 0, 1e-5, 0, 5e-5), 1.0, 2.0)
    d = D.Deck(dims=(6, 5, 5), spacing=h, horizon=3.015 * h, fixed_dt=1e-8, bdry_eff=0, ai_mls=0, intg_point=3,
               bcs=[g0], bc_spaces=[D.Space(1, (-1, 1, -1, 1, -1, 1))])
    d.write(str(tmp_path))
    dm = P.pdDataManager(str(tmp_path))
    P.pdSolve.InitialProblem(dm)
    ctx = dm.context()
    n = dm.info().num_nodes
    rng = np.random.default_rng(7)
    u = 1e-7 * rng.standard_normal(3 * n)
    v = 1e-3 * rng.standard_normal(3 * n)
    ctx.set_state(u, v)
    ctx.init_dynamic()
    k = ctx.force_stage(1e-8, 1e-8, u)
    x, mat, bc = dm.nodes()
    rp, col, br = dm.family()
    mats, bcs, _, _ = dm.tables()
    ptr, regs = P.ai_plan(x, rp, col, h, 3.015 * h)
    g = dict(n=np.array([n]))
    b = bcs[0]
    m = OL.Model(n=n, x=x, dx=h, delta=3.015 * h, mls=0, npt=1, fam_ptr=rp, fam_col=col, broken=br,
                 bdry_eff=dm.bdry_eff(), mat=mat, mat_spring=[mt["spring"] for mt in mats],
                 mat_ecrit=[mt["ecrit"] for mt in mats], mat_density=[mt["density"] for mt in mats],
                 mat_ymod=[72e9] * len(mats), bc=bc, bc_type=[b["type"]], bc_dir=list(b["dir"]),
                 bc_val=list(b["value"]), bc_end=[b["end_time"]], bc_load=[b["load_type"]], U=u, V=v)
    m.vbuf[:] = v
    ko, _, _ = oracle_stage(g, m, 3, ptr, regs, (None, None), 1e-8, 1e-8, u, br)
    assert np.array_equal(k, ko)
    assert np.array_equal(ctx.get_vbuf(), m.vbuf)
