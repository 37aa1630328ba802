"""The plain-FP64 config, the 20x10x10 bar (spacing 1 mm, horizon 3.015 mm,
2x2x2 Gauss points with MLS, boundary-effect factor off and on), pinned to
the reference: the host layer's setup and the oracle's restatement agree
with the reference's family lists, boundary-effect factors and MLS
coefficients bit for bit, and the oracle's force stage and first ten RK4 steps
with the reference's.  These decks hold interior nodes with full 250-node
families and, with the factor on, nodes of all three branches of
InitBdryEffectFactor.  (The device runs all 100 steps in test_long_gpu.py.)"""
import numpy as np
import pytest

import oracle_lib as O
import pdmtel_b200 as P
from golden_model import params
from long_golden import LONG_CASES, bdry_classes, digest, load_long, long_deck, same


def host_setup(name):
    """The host layer's setup on the CPU, with the oracle's bond search in
    place of the device search."""
    g = load_long(name)
    dm = P.pdDataManager(long_deck(name))
    dm.InitNode()
    x, mat, bc = dm.nodes()
    p = params(g)
    rp, col, mb = O.bond_search(x, p["dx"], p["delta"])
    dm.SetFamily(rp, col, np.zeros(len(col), np.int32), mb)
    dm.InitMaterial()
    dm.InitBdryEffectFactor()
    dm.InitGridBoundary()
    dm.InitIntegrationPoint()
    return g, dm, x, mat, bc, rp, col, mb


@pytest.mark.parametrize("name", LONG_CASES)
def test_bar_setup_matches_reference(name):
    g, dm, x, mat, bc, rp, col, mb = host_setup(name)
    p = params(g)
    assert np.array_equal(rp, g["fam_ptr"]) and same(col, g["sha_fam_col"]) and mb == g["min_bond"][0]
    assert int(np.diff(rp).max()) == 250
    assert len(col) == 2 * int(g["num_bonds"][0]) == 2 * 168392
    assert np.array_equal(dm.bdry_eff(), g["bdry_eff"])
    assert dm.info().stable_dt == g["dt"][0]
    cp, ci, co = dm.mls()
    assert np.array_equal(cp, g["cb_ptr"]) and same(ci, g["sha_cb_idx"]) and same(co, g["sha_coeff"])
    npt = 8
    # the coefficients of the sampled nodes, in full
    got = np.concatenate([co[cp[i] * npt:cp[i + 1] * npt] for i in g["coeff_nodes"]])
    assert np.array_equal(got, g["coeff_samples"])
    if p["bdry"]:
        cls = bdry_classes(x, rp, p["dims"], p["dx"], p["delta"], p["center"])
        counts = np.bincount(cls, minlength=3)
        assert counts.min() > 0, counts  # every branch is exercised
        bE = g["bdry_eff"]
        assert np.all(bE[cls == 0] == 1.0) and np.all(bE[cls != 0] != 1.0)
    else:
        assert np.all(g["bdry_eff"] == 1.0)


def oracle_model(name):
    """The oracle's own restatement of the setup (search, Gauss points, MLS,
    boundary-effect factors) on the reference's coordinates and tables."""
    g = load_long(name)
    p = params(g)
    dm = P.pdDataManager(long_deck(name))
    dm.InitNode()
    x, mat, bc = dm.nodes()
    assert np.array_equal(mat, g["mat"]) and np.array_equal(bc, g["bc"])
    rp, col, mb = O.bond_search(x, p["dx"], p["delta"])
    xg, gw = O.gauss_points(x, p["dx"], p["intg_point"])
    assert same(xg, g["sha_gauss_x"]) and np.array_equal(gw, g["gw"])
    cp, ci = O.mls_contributors(x, rp, col, p["rw"])
    co = O.mls_coeff(x, xg, 8, cp, ci, p["rw"])
    kw = dict(n=len(mat), x=x, dx=p["dx"], delta=p["delta"], cci=0, mls=1, npt=8, xg=xg, gw=gw, fam_ptr=rp,
              fam_col=col, cb_ptr=cp, cb_idx=ci, coeff=co, mat=mat, bc=bc, damping=p["damping"],
              mat_spring=g["spring"], mat_ecrit=g["mat_ecrit"], mat_density=g["mat_density"],
              mat_ymod=g["mat_ymod"], mat_grav=g["mat_grav"], bc_type=g["bc_type"], bc_dir=g["bc_dir"],
              bc_val=g["bc_val"], bc_end=g["bc_end"], bc_load=g["bc_load"])
    m = O.Model(**kw)
    if p["bdry"]:
        bE, full = m.bdry_eff(p["dims"], p["center"])
        assert full == 250
        m = O.Model(**dict(kw, bdry_eff=bE))
    return g, m, co


@pytest.mark.parametrize("name", LONG_CASES)
def test_oracle_force_and_ten_steps_match_reference(name):
    g, m, co = oracle_model(name)
    assert same(co, g["sha_coeff"])
    assert np.array_equal(m.keep["bdry_eff"], g["bdry_eff"])
    t, dts = g["force_args"]
    m.U[:] = g["u_test"]
    m.V[:] = g["v_test"]
    m.vbuf[:] = g["v_test"]
    m.gather(t, g["u_test"])
    assert same(m.ug, g["sha_ug_force"])
    k = m.force_stage(dts, t, g["u_test"])
    assert np.array_equal(k, g["k"])
    assert np.array_equal(m.vbuf, g["vbuf"])
    assert np.array_equal(m.eed, g["eed"])
    # ten steps from rest
    m.U[:] = 0.0
    m.V[:] = 0.0
    m.vbuf[:] = 0.0
    m.ug[:] = 0.0
    dt = g["dt"][0]
    for it in range(1, 11):
        ke, ee = m.rk4_step(dt, g["times"][it - 1])
        assert ke == pytest.approx(g["ke"][it - 1], rel=1e-12, abs=1e-300)
        assert ee == pytest.approx(g["ee"][it - 1], rel=1e-12, abs=1e-300)
    assert np.array_equal(m.U, g["U_10"]) and np.array_equal(m.V, g["V_10"])
    assert same(m.ug, g["sha_ug_10"])
