"""pd_bond_search_noalloc: the bond search for callers that cannot allocate
device memory (a host that owns every device byte through its own pool, a
plugin inside such a host, a loop that must not stall on cudaMalloc).  It
writes into buffers the caller allocated and works in the library's fixed
device array, so it is checked here against the ordinary entry point,
pd_bond_search, on the same decks: the family lists are integers, so they
must agree exactly, and they must still agree on a second call in a row,
when the shared array holds the first call's data.

This file is named to run last: the array it uses lives as long as the
process, and every other test must already have run if it fails."""
import ctypes as C

import numpy as np
import pytest

import pdmtel_b200 as P
from pdmtel_b200 import decks as D

pytestmark = pytest.mark.gpu


def _entry():
    f = P.lib().pd_bond_search_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_int32, C.POINTER(C.c_double), C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    f.restype = C.c_int
    return f


def _decks():
    return {
        "plate_slit_60x60x4": D.config_plate(dims=(60, 60, 4), spacing=5e-4, slit_half_length=6e-3),
        "bar_20x10x10": D.config_bar(dims=(20, 10, 10), traction_as_veloc=0.05),
        "plate_slit_12x10x3": D.config_plate(dims=(12, 10, 3), spacing=1e-3, slit_half_length=2e-3),
    }


@pytest.mark.parametrize("name", list(_decks()))
def test_noalloc_search_matches_device_search(name, tmp_path):
    import torch

    deck = _decks()[name]
    deck.write(str(tmp_path))
    dm = P.pdDataManager(str(tmp_path))
    dm.InitNode()
    dm.InitBond()  # the ordinary entry point, pd_bond_search
    rp_ref, col_ref, br_ref = dm.family()
    info = dm.info()
    x, _, _ = dm.nodes()
    n = info.num_nodes
    slits = np.ascontiguousarray(np.asarray(deck.slits, dtype=np.float64).reshape(-1))
    ns = slits.size // 6
    f = _entry()
    d_x = torch.tensor(x, dtype=torch.float64, device="cuda")
    d_rp = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda")
    cap = len(col_ref)
    d_col = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
    d_br = torch.full((cap,), 7, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    for call in range(2):
        nh = C.c_int64(0)
        mb = C.c_double(0.0)
        rc = f(d_x.data_ptr(), n, info.grid_spacing, info.horizon, ns,
               slits.ctypes.data_as(C.POINTER(C.c_double)) if ns else None,
               d_rp.data_ptr(), d_col.data_ptr(), d_br.data_ptr(), cap, None, C.byref(nh), C.byref(mb))
        assert rc == 0, P.lib().pd_last_error()
        assert nh.value == len(col_ref)
        assert mb.value == info.min_bond_length
        assert np.array_equal(d_rp.cpu().numpy(), rp_ref)
        assert np.array_equal(d_col.cpu().numpy(), col_ref)
        assert np.array_equal(d_br.cpu().numpy(), br_ref)
        if ns:
            assert br_ref.sum() > 0
        # scribble over the outputs before the second call
        d_rp.fill_(-1)
        d_col.fill_(-1)
        d_br.fill_(7)


def test_noalloc_reports_capacity_and_size(tmp_path):
    import torch

    D.config_bar(dims=(8, 5, 4), traction_as_veloc=0.05).write(str(tmp_path))
    dm = P.pdDataManager(str(tmp_path))
    dm.InitNode()
    dm.InitBond()
    info = dm.info()
    x, _, _ = dm.nodes()
    f = _entry()
    d_x = torch.tensor(x, dtype=torch.float64, device="cuda")
    d_rp = torch.zeros(info.num_nodes + 1, dtype=torch.int64, device="cuda")
    d_col = torch.zeros(10, dtype=torch.int32, device="cuda")
    nh = C.c_int64(0)
    mb = C.c_double(0.0)
    rc = f(d_x.data_ptr(), info.num_nodes, info.grid_spacing, info.horizon, 0, None, d_rp.data_ptr(),
           d_col.data_ptr(), None, 10, None, C.byref(nh), C.byref(mb))
    assert rc == -6  # PD_ERR_CAPACITY
    assert nh.value == info.num_halves
    assert np.array_equal(d_rp.cpu().numpy(), dm.family()[0])
    too_many = 65536 + 1
    rc = f(d_x.data_ptr(), too_many, info.grid_spacing, info.horizon, 0, None, d_rp.data_ptr(),
           d_col.data_ptr(), None, 10, None, C.byref(nh), C.byref(mb))
    assert rc == -6


def _search(f, x, spacing, horizon, slits=None, cap=0):
    """Runs the entry point on coordinates x [n][3]; returns (status, halves)."""
    import torch
    n = len(x)
    d_x = torch.tensor(np.ascontiguousarray(x, dtype=np.float64), device="cuda")
    d_rp = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    d_col = torch.zeros(max(cap, 1), dtype=torch.int32, device="cuda")
    sl = None if slits is None else np.ascontiguousarray(slits, dtype=np.float64).reshape(-1)
    ns = 0 if sl is None else sl.size // 6
    nh = C.c_int64(0)
    mb = C.c_double(0.0)
    rc = f(d_x.data_ptr(), n, spacing, horizon, ns, sl.ctypes.data_as(C.POINTER(C.c_double)) if ns else None,
           d_rp.data_ptr(), d_col.data_ptr(), None, cap, None, C.byref(nh), C.byref(mb))
    torch.cuda.synchronize()
    return rc, nh.value


def _still_usable(f):
    """After a refused call the library still searches a small bar correctly."""
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        D.config_bar(dims=(8, 5, 4), traction_as_veloc=0.05).write(td)
        dm = P.pdDataManager(td)
        dm.InitNode()
        dm.InitBond()
        info = dm.info()
        x, _, _ = dm.nodes()
        rc, nh = _search(f, x.reshape(-1, 3), info.grid_spacing, info.horizon, cap=info.num_halves)
        assert rc == 0 and nh == info.num_halves


def test_noalloc_refuses_too_many_cells():
    f = _entry()
    # two nodes 1 m apart with a 1 nm horizon: 5e8 cells along x
    x = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    assert _search(f, x, 1e-9, 1e-9)[0] == -6
    # three axes of 1e9 cells each: the product would overflow a 64-bit integer
    x = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]])
    assert _search(f, x, 1e-10, 1e-9)[0] == -6
    # 301 cells per axis: each axis is within the limit, their product is not
    assert _search(f, x, 1e-3, 1.0 / 300.0 - 1e-3)[0] == -6
    # a non-finite coordinate is an argument error, not a cell count
    x = np.array([[0.0, 0.0, 0.0], [np.nan, 0.0, 0.0]])
    assert _search(f, x, 1e-3, 3e-3)[0] == -1
    _still_usable(f)


def test_noalloc_refuses_too_many_slits():
    f = _entry()
    x = np.array([[0.0, 0.0, 0.0], [1e-3, 0.0, 0.0]])
    slits = np.tile([-1.0, 1.0, 0.0, 0.0, -1.0, 1.0], 17)
    assert _search(f, x, 1e-3, 3e-3, slits=slits)[0] == -1  # above PD_NOALLOC_MAX_SLITS
    _still_usable(f)


def test_noalloc_refuses_family_beyond_shared_buffer():
    f = _entry()
    # 14^3 nodes all within one horizon: families of 2743 exceed the 48 KB
    # shared buffer of four warps
    g = np.arange(14, dtype=np.float64) * 1e-3
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    n = len(x)
    rc, nh = _search(f, x, 1e-3, 0.05, cap=n * (n - 1))
    assert nh == n * (n - 1)
    assert rc == -6
    _still_usable(f)
