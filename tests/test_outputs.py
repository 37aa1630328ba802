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
    refs = sorted(glob.glob(os.path.join(src, "ref_pds_*.dat")))  # the run's files (ref_afd_*: PostAFD below)
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


def _afd_requests(case):
    """The requests the reference's PostAFD read from its console when the
    fixture was made (tests/golden/make_golden.py, AFD_SCRIPTS)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    step, runs = mg.AFD_SCRIPTS[case]
    req = [("plane", int(r[1]), float(r[2])) if r[0] == "1" else ("node", int(r[1])) for r in runs]
    return int(step), req


@pytest.mark.parametrize("case", OCASES)
def test_post_afd_matches_reference(case, tmp_path):
    """PostAFD (areal force density stress from a Tecplot dump, pdSolve.cpp:
    810-834, pdDataManager3.cpp:442-635,1101-1223) on the last dump of the
    run above, for planes normal to each axis and single nodes: the file
    matches the reference's character by character."""
    src = os.path.join(ODIR, case)
    shutil.copy(os.path.join(src, "pds_input.txt"), str(tmp_path))
    dm = P.pdDataManager(str(tmp_path))
    P.pdSolve.InitialProblem(dm)
    P.pdSolve.SolveDynamic(dm, write_files=True)
    step, req = _afd_requests(case)
    P.pdSolve.PostAFD(dm, step, req)
    a = _lines(os.path.join(src, f"ref_afd_pds_AFD_{step}.dat"))
    b = _lines(os.path.join(str(tmp_path), f"pds_AFD_{step}.dat"))
    assert len(a) > 10
    for k, (la, lb) in enumerate(zip(a, b)):
        assert la == lb, f"line {k + 1}:\nreference: {la!r}\nhere:      {lb!r}"
    assert len(a) == len(b)
