"""The output files of pdSolve::SolveDynamic against the reference's own
(tests/golden/outputs/<case>/ref_*, written by the reference's SolveDynamic
through the harness): the pds_output.dat log (deck echo, setup messages and
one line per step), the pds_steps.dat probe of the node at (dx/2, dx/2,
dx/2) and every pds_tecplot_<step>.dat, line by line and character by
character (pdSolve.cpp:24-130,708-774, pdNode.cpp:418-433).  One deck with
2x2x2 Gauss points, MLS, boundary factors and a shortened last step; one
CCI deck with a ramped displacement gradient."""
import glob
import os
import shutil

import pytest

import pdmtel_b200 as P

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ODIR = os.path.join(HERE, "golden", "outputs")
OCASES = sorted(os.path.basename(p) for p in glob.glob(os.path.join(ODIR, "out_*")))


def _lines(path):
    with open(path) as f:
        return f.read().splitlines()


@pytest.mark.parametrize("case", OCASES)
def test_output_files_match_reference(case, tmp_path):
    src = os.path.join(ODIR, case)
    shutil.copy(os.path.join(src, "pds_input.txt"), str(tmp_path))
    dm = P.pdDataManager(str(tmp_path))
    P.pdSolve.InitialProblem(dm)
    P.pdSolve.SolveDynamic(dm, write_files=True)
    refs = sorted(glob.glob(os.path.join(src, "ref_pds_*.dat")))
    assert len(refs) >= 4
    for ref in refs:
        name = os.path.basename(ref)[len("ref_"):]
        mine = os.path.join(str(tmp_path), name)
        assert os.path.exists(mine), name
        a, b = _lines(ref), _lines(mine)
        for k, (la, lb) in enumerate(zip(a, b)):
            assert la == lb, f"{name} line {k + 1}:\nreference: {la!r}\nhere:      {lb!r}"
        assert len(a) == len(b), (name, len(a), len(b))
    produced = sorted(os.path.basename(p) for p in glob.glob(os.path.join(str(tmp_path), "pds_*.dat")))
    assert produced == sorted(os.path.basename(r)[len("ref_"):] for r in refs)
