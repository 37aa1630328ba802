"""InitIntegrationPoint on the device (pd_mls_setup) against the host setup,
which reproduces the reference bit for bit.  The contributor lists must be
identical.  The coefficients follow the reference's operation order, except
that the spline weight's d^3 and d^4 are rounded once where the reference
takes glibc's pow (off the correctly rounded value for ~4e-4 of the
arguments): most coefficients are identical, the rest differ by the moment
matrix's round-off, bounded here by 1e-6 of the largest coefficient of the
same point.  The FP32 form run from device coefficients stays within its
1e-6 bar of the FP64 drop-in run from the reference's."""
import os

import numpy as np
import pytest

import pdmtel_b200 as P
from conftest import deck_dir, load_golden
from pdmtel_b200 import decks as D

pytestmark = pytest.mark.gpu


def _compare(cp_h, ci_h, co_h, cp_d, ci_d, co_d, npt=8):
    assert np.array_equal(cp_h, cp_d) and np.array_equal(ci_h, ci_d)
    same = co_h == co_d
    worst = 0.0
    n = len(cp_h) - 1
    for i in range(n):
        b, e = cp_h[i], cp_h[i + 1]
        h = co_h[b * npt:e * npt].reshape(npt, -1)
        d = co_d[b * npt:e * npt].reshape(npt, -1)
        worst = max(worst, float((np.abs(h - d).max(axis=1) / np.abs(h).max(axis=1)).max()))
    return same.mean(), worst


@pytest.mark.parametrize("name", ["fgi_velo", "fgi_slit", "fgi3_ramp"])
def test_device_mls_matches_reference_goldens(name):
    g = load_golden(name)
    dm = P.pdDataManager(deck_dir(name))
    dm.SetDeviceSetup(True)
    P.pdSolve.InitialProblem(dm)
    cp, ci, co = dm.mls()
    npt = int(g["num_gauss"][0])
    frac, worst = _compare(g["cb_ptr"], g["cb_idx"], g["coeff"], cp, ci, co, npt)
    assert frac > 0.9, frac
    assert worst <= 1e-6, worst


def test_device_mls_on_a_plate(tmp_path):
    """A 60x60x4 slit plate: device against host coefficients, and 100 FP32C
    steps from the device setup against 100 FP64 steps from the host's."""
    D.config_plate(dims=(60, 60, 4), spacing=5e-4, slit_half_length=6e-3, dt=5e-9, vel=0.05).write(str(tmp_path))
    host = P.pdDataManager(str(tmp_path))
    P.pdSolve.InitialProblem(host)
    dev = P.pdDataManager(str(tmp_path))
    dev.SetDeviceSetup(True)
    dev.SetPrecision(P.PREC_FP32C)
    P.pdSolve.InitialProblem(dev)
    frac, worst = _compare(*host.mls(), *dev.mls())
    assert frac > 0.9, frac
    assert worst <= 1e-6, worst
    a = host.context()
    b = dev.context()
    a.rk4_steps(5e-9, 0.0, 100)
    b.rk4_steps(5e-9, 0.0, 100)
    a.sync()
    b.sync()
    Ua, _ = a.get_state()
    Ub, _ = b.get_state()
    assert np.abs(Ua).max() > 0
    assert np.linalg.norm(Ub - Ua) <= 1e-6 * np.linalg.norm(Ua)


def test_device_mls_of_a_batch_equals_its_specimens(tmp_path):
    """A batch solves every specimen's MLS in the specimen's own frame: the
    device setup of the merged problem equals each specimen's own device
    setup, entry for entry."""
    from pdmtel_b200 import batch as B
    spec = B.BatchSpec(dims=[(12, 10, 8), (9, 14, 7), (16, 8, 6)], seed=5)
    bt = B.Batch(str(tmp_path), spec, precision=P.PREC_FP32C, device_setup=True)
    cp, ci, co = bt.model.mls()
    off = bt.offsets
    for k in range(len(off) - 1):
        sdir = os.path.join(str(tmp_path), f"specimen_{k:04d}")
        dm = P.pdDataManager(sdir)
        dm.SetDeviceSetup(True)
        P.pdSolve.InitialProblem(dm)
        scp, sci, sco = dm.mls()
        o, n = off[k], off[k + 1] - off[k]
        b0, b1 = cp[o], cp[o + n]
        assert np.array_equal(cp[o:o + n + 1] - b0, scp)
        assert np.array_equal(ci[b0:b1] - o, sci)
        assert np.array_equal(co[b0 * 8:b1 * 8], sco)
