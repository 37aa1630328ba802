"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute call here: this runs without a GPU)."""
import ctypes as C
import glob
import os
import re

import numpy as np

import pdmtel_b200 as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(pd[h]?_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) > 40
    L = C.CDLL(P.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version_and_device_count():
    assert P.lib().pd_abi_version() == 1
    assert P.device_count() >= 0


def test_argument_validation_precedes_device_use():
    L = P.lib()
    prob = P.pd_problem()
    prob.num_nodes = -5
    h = C.c_void_p()
    assert L.pd_ctx_create(C.byref(prob), C.byref(h)) == -1
    assert L.pd_ctx_create(None, C.byref(h)) == -1
    assert b"null" in L.pd_last_error()


def test_null_context_is_rejected():
    L = P.lib()
    assert L.pd_sync(None) == -1
    assert L.pd_rk4_steps(None, 1e-8, 0.0, 1) == -1
    assert L.pd_static_solve(None, 0.0, 0, 1e-10, 10, None, None, None) == -1


def _header_text():
    return re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "pdmtel_b200.h")).read(), flags=re.S)


def test_option_constants_match_the_header():
    """Every PD_OPT_* of the header has the same value in the Python layer."""
    opts = {m.group(1): int(m.group(2)) for m in re.finditer(r"\bPD_OPT_(\w+)\s*=\s*(\d+)", _header_text())}
    assert len(opts) >= 14
    for name, v in opts.items():
        assert getattr(P, "OPT_" + name) == v, name


def test_tune_result_layout_matches_the_header():
    """pd_tune_result: same fields, order and sizes in the header and ctypes."""
    body = re.search(r"typedef struct pd_tune_result \{(.*?)\} pd_tune_result;", _header_text(), flags=re.S).group(1)
    fields = []
    for m in re.finditer(r"\b(int64_t|int32_t|double)\s+([\w\s,]+);", body):
        for n in m.group(2).split(","):
            fields.append((n.strip(), {"int64_t": 8, "int32_t": 4, "double": 8}[m.group(1)]))
    py = [(n, C.sizeof(t)) for n, t in P.pd_tune_result._fields_]
    assert fields == py
