"""The CPU oracle is pinned bit for bit against the reference's own outputs
(tests/golden/*.npz, generated by tests/golden/make_golden.py from the
reference harness)."""
import numpy as np
import pytest

import oracle_lib as O
from conftest import kat
from golden_model import model_from_golden, params


def test_bond_search_matches_reference(golden_case):
    name, g = golden_case
    P = params(g)
    rp, col, mb = O.bond_search(g["coords"], P["dx"], P["delta"])
    assert np.array_equal(rp, g["fam_ptr"])
    assert np.array_equal(col, g["fam_col"])
    assert mb == g["min_bond"][0]


def test_slit_marks_match_harness(golden_case):
    name, g = golden_case
    slits = {"fgi_slit": [(-2.0e-3, 2.0e-3, 0.0, 0.0, -1.0, 1.0)]}.get(name, [])
    br = O.slit_mark(g["coords"], g["fam_ptr"], g["fam_col"], slits) if slits else np.zeros_like(g["broken"])
    assert np.array_equal(br.astype(np.int32), g["broken"])
    if slits:
        assert br.sum() > 0


def test_gauss_points_and_mls(golden_case):
    name, g = golden_case
    P = params(g)
    if P["cci"]:
        pytest.skip("CCI has no Gauss points")
    xg, gw = O.gauss_points(g["coords"], P["dx"], P["intg_point"])
    assert np.array_equal(xg, g["gauss_x"])
    assert np.array_equal(gw, g["gw"])
    if not P["mls"]:
        return
    cp, ci = O.mls_contributors(g["coords"], g["fam_ptr"], g["fam_col"], P["rw"])
    assert np.array_equal(cp, g["cb_ptr"]) and np.array_equal(ci, g["cb_idx"])
    co = O.mls_coeff(g["coords"], xg, int(g["num_gauss"][0]), cp, ci, P["rw"])
    assert np.array_equal(co, g["coeff"])


def test_bdry_eff(golden_case):
    name, g = golden_case
    P = params(g)
    if not P["bdry"]:
        assert np.all(g["bdry_eff"] == 1.0)
        return
    m = model_from_golden(g)
    bE, full = m.bdry_eff(P["dims"], P["center"])
    assert full == int(g["num_max_family"][0])
    assert np.array_equal(bE, g["bdry_eff"])


def test_force_stage(golden_case):
    name, g = golden_case
    t, dts = g["force_args"]
    m = model_from_golden(g, U=g["u_test"], V=g["v_test"])
    m.vbuf[:] = g["v_test"]
    m.gather(t, g["u_test"])
    if len(g["ug"]):
        assert np.array_equal(m.ug, g["ug"])
    k = m.force_stage(dts, t, g["u_test"])
    assert np.array_equal(k, g["k"])
    assert np.array_equal(m.vbuf, g["vbuf"])
    assert np.array_equal(m.U, g["U_after"])
    assert np.array_equal(m.eed, g["eed"])


def test_rk4_trajectory(golden_case):
    name, g = golden_case
    m = model_from_golden(g)
    times = g["traj_times"]
    for it, t in enumerate(times, start=1):
        ke, ee = m.rk4_step(g["dt"][0], t)
        assert ke == g["traj_ke"][it - 1] and ee == g["traj_ee"][it - 1]
        if f"traj_U_{it}" in g:
            assert np.array_equal(m.U, g[f"traj_U_{it}"])
            assert np.array_equal(m.V, g[f"traj_V_{it}"])
            if len(g[f"traj_ug_{it}"]):
                assert np.array_equal(m.ug, g[f"traj_ug_{it}"])


@pytest.mark.slow
def test_bond_count_bar_20x10x10():
    """Known answer: the 20x10x10 lattice (spacing 1 mm, horizon 3.015 mm)
    has 168,392 bonds and full-sphere families of 250."""
    x = []
    h = 1e-3
    for n in range(1, 11):
        for mm in range(1, 11):
            for l in range(1, 21):
                x += [(l - 21 * 0.5) * h, (mm - 11 * 0.5) * h, (n - 11 * 0.5) * h]
    rp, col, mb = O.bond_search(np.array(x), h, 3.015 * h)
    K = kat()["bar_20x10x10"]
    assert len(col) == 2 * K["bonds"] == 336784
    assert np.diff(rp).max() == K["max_family"] == 250
    assert mb == pytest.approx(h)
