"""The C++ host layer (pdDataManager mirror) on the CPU: deck reading, the
lattice, and the one-time setup that stays on the host (boundary-effect
factors, MLS coefficients) reproduce the reference bit for bit."""
import ctypes as C
import os
import shutil

import numpy as np
import pytest

import pdmtel_b200 as P
from conftest import deck_dir, load_golden, CASES
from pdmtel_b200 import decks as D


def setup_from_golden(name, workdir=None):
    g = load_golden(name)
    dm = P.pdDataManager(workdir or deck_dir(name))
    dm.InitNode()
    dm.SetFamily(g["fam_ptr"], g["fam_col"], g["broken"], g["min_bond"][0])
    dm.InitMaterial()
    dm.InitBdryEffectFactor()
    dm.InitGridBoundary()
    dm.InitIntegrationPoint()
    return dm, g


@pytest.mark.parametrize("name", CASES)
def test_host_setup_matches_reference(name):
    dm, g = setup_from_golden(name)
    x, mat, bc = dm.nodes()
    assert np.array_equal(x, g["coords"]) and np.array_equal(mat, g["mat"]) and np.array_equal(bc, g["bc"])
    assert np.array_equal(dm.bdry_eff(), g["bdry_eff"])
    I = dm.info()
    assert I.stable_dt == g["dt"][0]
    if I.mls:
        cp, ci, co = dm.mls()
        assert np.array_equal(cp, g["cb_ptr"]) and np.array_equal(ci, g["cb_idx"]) and np.array_equal(co, g["coeff"])


def test_crlf_deck_reads_like_lf(tmp_path):
    src = os.path.join(deck_dir("fgi_velo"), "pds_input.txt")
    with open(src) as f:
        text = f.read()
    (tmp_path / "pds_input.txt").write_bytes(text.replace("\n", "\r\n").encode())
    dm, g = setup_from_golden("fgi_velo", str(tmp_path))
    assert np.array_equal(dm.bdry_eff(), g["bdry_eff"])
    cp, ci, co = dm.mls()
    assert np.array_equal(co, g["coeff"])


def test_trailing_spaces_and_blank_lines(tmp_path):
    src = os.path.join(deck_dir("cci_grad"), "pds_input.txt")
    lines = open(src).read().split("\n")
    out = [""]
    for k in range(0, len(lines) - 1, 2):
        out += ["   " + lines[k] + "   ", lines[k + 1] + "  ", ""]
    (tmp_path / "pds_input.txt").write_text("\n".join(out))
    dm = P.pdDataManager(str(tmp_path))
    dm.InitNode()
    assert dm.info().num_nodes == 160


def write_deck(tmp_path, deck):
    deck.write(str(tmp_path))
    return str(tmp_path)


def test_missing_required_keyword_is_an_error(tmp_path):
    d = D.config_bar(dims=(5, 4, 4))
    text = d.text().replace("damping_coeff\n", "damping_coefficient\n")
    (tmp_path / "pds_input.txt").write_text(text)
    with pytest.raises(P.PdError) as e:
        P.pdDataManager(str(tmp_path))
    assert e.value.code == -1 and "damping_coeff" in str(e.value)


def test_missing_value_is_an_error(tmp_path):
    d = D.config_bar(dims=(5, 4, 4))
    text = d.text().replace("grid_dimension\n 5 4 4\n", "grid_dimension\n 5 4\n")
    (tmp_path / "pds_input.txt").write_text(text)
    with pytest.raises(P.PdError) as e:
        P.pdDataManager(str(tmp_path))
    assert "value missing" in str(e.value)


def test_missing_deck_is_an_error(tmp_path):
    with pytest.raises(P.PdError):
        P.pdDataManager(str(tmp_path / "nowhere"))


def test_node_outside_last_material_space(tmp_path):
    """Every material space overwrites the material of every node, so a node
    outside the LAST space has none (pdDataManager.cpp:937-970): fatal."""
    d = D.config_bar(dims=(6, 4, 4))
    d.material_spaces = [D.Space(1, (-1, 1, -1, 1, -1, 1)), D.Space(1, (-1, 0.0, -1, 1, -1, 1))]
    dm = P.pdDataManager(write_deck(tmp_path, d))
    with pytest.raises(P.PdError) as e:
        dm.InitNode()
    assert "not in any material space" in str(e.value)


def test_deletion_space_renumbers_nodes(tmp_path):
    d = D.config_bar(dims=(6, 4, 4))
    d.deletion_spaces = [D.Space(0, (-1e-3, 1e-3, -1, 1, -1, 1))]
    dm = P.pdDataManager(write_deck(tmp_path, d))
    dm.InitNode()
    x, _, _ = dm.nodes()
    assert dm.info().num_nodes == 6 * 4 * 4 - 2 * 4 * 4
    assert np.all(np.abs(x.reshape(-1, 3)[:, 0]) > 1e-3)


def _ai_deck(tmp_path, extra=""):
    d = D.config_bar(dims=(5, 4, 4))
    text = d.text().replace("fgi_on\n 1\n", "fgi_on\n 0\nai_on\n 1 1\n" + extra)
    (tmp_path / "pds_input.txt").write_text(text)
    return str(tmp_path)


def test_adaptive_integration_deck(tmp_path):
    """ai_on decks are read (pdDataManager.cpp:656-717) and echoed with the
    reference's AI lines (:747-753)."""
    path = _ai_deck(tmp_path, "intg_point\n 2\n")
    P.pdDataManager(path)
    log = (tmp_path / "pds_output.dat").read_text()
    assert "Adaptive integration method flag = 1" in log
    assert "Starting trapezoidal index = 2" in log
    assert "Error control method flag = 0" in log


@pytest.mark.parametrize("extra,word", [("error_control_on\n 1\n", "error_control_on"),
                                        ("intg_point\n 4\n", "trapezoid index")])
def test_adaptive_integration_refusals(tmp_path, extra, word):
    """The refinement with error control reads MLS list entries the setup pass
    never stored, and an index above 3 refines a stale sum: both refused."""
    with pytest.raises(P.PdError) as e:
        P.pdDataManager(_ai_deck(tmp_path, extra))
    assert word in str(e.value)


def test_no_gpu_fails_loudly(tmp_path):
    if P.device_count() > 0:
        pytest.skip("a CUDA device is present")
    dm = P.pdDataManager(write_deck(tmp_path, D.config_bar(dims=(5, 4, 4))))
    dm.InitNode()
    with pytest.raises(P.PdError) as e:
        dm.InitBond()
    assert e.value.code == -8
