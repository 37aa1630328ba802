"""The static operator pinned to the reference.

The reference's matrix-free pass pdDataManager::CalcDampingCoeff
(pdDataManager2.cpp:1616-1907) uses the coefficients of pdSolve::
AssembleEquation (pdSolve.cpp:195-527): per family pair c V_j xi xi^T / r^3.
It returns the per-dof sum of |K_ij| (absKVector; dt = 2 makes its dt^2/4
scale exactly 1) and 2 sqrt(u.Ku / sum_i absK_i u_i^2) at a displacement u.
tests/golden/static/*.npz hold those values from the reference on three
decks without boundary conditions (so K is the unconstrained operator):
the oracle's operator (CPU) and the device operator (both kernels, through
the C ABI) are assembled column by column and must give the same row sums to
1e-13 and the same coefficients at three fields to 1e-12 (the reference sums
in another order)."""
import glob
import os

import numpy as np
import pytest

import oracle_lib as O
import pdmtel_b200 as P
from golden_model import params

HERE = os.path.dirname(os.path.abspath(__file__))
SDIR = os.path.join(HERE, "golden", "static")
SCASES = sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(SDIR, "*.npz")))


def load(name):
    with np.load(os.path.join(SDIR, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def assemble(apply, n3):
    """Columns K e_j of a linear operator, as a dense matrix."""
    K = np.zeros((n3, n3))
    e = np.zeros(n3)
    for j in range(n3):
        e[j] = 1.0
        K[:, j] = apply(e)
        e[j] = 0.0
    return K


def check(g, K):
    absK = np.abs(K).sum(axis=1)
    np.testing.assert_allclose(absK, g["absK"], rtol=1e-13, atol=0)
    for f in range(3):
        u = g[f"u_field_{f}"]
        nom = u @ (K @ u)
        dem = np.sum(absK * u * u)
        damp = 2.0 * np.sqrt(nom / dem)
        assert damp == pytest.approx(g["damp_coeff"][f], rel=1e-12)


def test_static_cases_present():
    assert len(SCASES) == 3


@pytest.mark.parametrize("name", SCASES)
def test_oracle_static_operator_matches_reference(name):
    g = load(name)
    p = params(g)
    n = int(g["n"][0])
    m = O.Model(n=n, x=g["coords"], dx=p["dx"], delta=p["delta"], cci=p["cci"], mls=0, npt=1,
                fam_ptr=g["fam_ptr"], fam_col=g["fam_col"], broken=g["broken"].astype(np.uint8), mat=g["mat"],
                mat_spring=g["spring"], mat_ecrit=np.full(len(g["spring"]), 1e20), mat_density=g["mat_density"],
                mat_ymod=np.ones(len(g["spring"])))
    assert not g["broken"].any()
    check(g, assemble(lambda x: m.static_apply(1.0, x), 3 * n))


def _deck(name):
    return os.path.join(SDIR, "decks", name)


@pytest.mark.gpu
@pytest.mark.parametrize("stencil", [1, 0], ids=["stencil-if-eligible", "family-lists"])
@pytest.mark.parametrize("name", SCASES)
def test_device_static_operator_matches_reference(name, stencil):
    g = load(name)
    dm = P.pdDataManager(_deck(name))
    dm.InitNode()
    dm.InitBond()
    dm.InitMaterial()
    rp, col, _ = dm.family()
    assert np.array_equal(rp, g["fam_ptr"]) and np.array_equal(col, g["fam_col"])
    ctx = dm.context()
    ctx.set_option(P.OPT_STATIC_STENCIL, stencil)
    used = ctx.static_prepare()
    if stencil == 0:
        assert not used
    if name in ("static_bar", "static_cci") and stencil:
        assert used  # complete boxes run the stencil kernel
    n3 = 3 * int(g["n"][0])
    check(g, assemble(lambda x: ctx.static_matvec(1.0, x), n3))
