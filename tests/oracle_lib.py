"""ctypes binding of the CPU oracle (oracle/liboracle.so).

Test infrastructure: the oracle is the checker the CUDA path is compared
against.  ``Model`` builds an ``or_model`` from plain numpy arrays, for example
those a reference dump (tests/pdb_io.py) or the product's own setup export.
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "liboracle.so")

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)
_u8 = C.POINTER(C.c_uint8)


class OrModel(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("x", _d), ("dx", C.c_double), ("delta", C.c_double),
        ("cci", C.c_int), ("cci_mdf", C.c_int), ("mls", C.c_int), ("npt", C.c_int),
        ("xg", _d), ("gw", _d), ("fam_ptr", _i64), ("fam_col", _i32), ("broken", _u8),
        ("cb_ptr", _i64), ("cb_idx", _i32), ("coeff", _d), ("bdry_eff", _d), ("mat", _i32),
        ("mat_spring", _d), ("mat_ecrit", _d), ("mat_density", _d), ("mat_grav", _d), ("mat_ymod", _d),
        ("bc", _i32), ("bc_type", _i32), ("bc_dir", _i32), ("bc_val", _d), ("bc_end", _d), ("bc_load", _d),
        ("spring_factor", _d), ("damping", C.c_double),
        ("U", _d), ("V", _d), ("vbuf", _d), ("ug", _d), ("eed", _d), ("ke", C.c_double), ("ee", C.c_double),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        L.or_gauss_1d.argtypes = [C.c_int, _d, _d]
        L.or_gauss_points.argtypes = [C.c_int64, _d, C.c_double, C.c_int, _d, _d]
        L.or_bond_search.argtypes = [C.c_int64, _d, C.c_double, C.c_double, _i64, _i32, C.c_int64, _d]
        L.or_bond_search.restype = C.c_int64
        L.or_slit_mark.argtypes = [C.c_int64, _d, _i64, _i32, C.c_int, _d, _u8]
        L.or_mls_contributors.argtypes = [C.c_int64, _d, _i64, _i32, C.c_double, _i64, _i32]
        L.or_mls_contributors.restype = C.c_int64
        L.or_mls_coeff.argtypes = [C.c_int64, _d, _d, C.c_int, _i64, _i32, C.c_double, _d]
        L.or_mls_coeff.restype = C.c_int64
        L.or_bdry_eff.argtypes = [C.POINTER(OrModel), C.POINTER(C.c_int), _d, _d]
        L.or_gather.argtypes = [C.POINTER(OrModel), C.c_double, _d]
        L.or_force_stage.argtypes = [C.POINTER(OrModel), C.c_double, C.c_double, _d, _d]
        L.or_rk4_step.argtypes = [C.POINTER(OrModel), C.c_double, C.c_double]
        L.or_static_apply.argtypes = [C.POINTER(OrModel), C.c_double, _d, _d]
        L.or_static_rhs.argtypes = [C.POINTER(OrModel), C.c_double, _d]
        L.or_static_cg.argtypes = [C.POINTER(OrModel), C.c_double, _d, _d, C.c_double, C.c_int, _d]
        L.or_static_cg.restype = C.c_int
        L.or_adjoint_grad.argtypes = [C.POINTER(OrModel), C.c_double, C.c_double, C.c_int, _d, _d, _d]
        L.or_adjoint_grad.restype = C.c_int
        _lib = L
    return _lib


def ptr(a, t):
    if a is None:
        return C.cast(None, t)
    return a.ctypes.data_as(t)


def gauss_1d(n):
    a = np.zeros(8)
    w = np.zeros(8)
    m = lib().or_gauss_1d(n, ptr(a, _d), ptr(w, _d))
    return a[:m].copy(), w[:m].copy()


def gauss_points(x, dx, n1):
    m = len(gauss_1d(n1)[0])
    npt = m ** 3
    n = x.shape[0] // 3
    xg = np.zeros(n * npt * 3)
    gw = np.zeros(npt * 3)
    lib().or_gauss_points(n, ptr(x, _d), dx, n1, ptr(xg, _d), ptr(gw, _d))
    return xg, gw


def bond_search(x, dx, delta):
    n = x.shape[0] // 3
    rp = np.zeros(n + 1, dtype=np.int64)
    mb = C.c_double(0)
    tot = lib().or_bond_search(n, ptr(x, _d), dx, delta, ptr(rp, _i64), ptr(None, _i32), 0, C.byref(mb))
    col = np.zeros(max(tot, 1), dtype=np.int32)
    lib().or_bond_search(n, ptr(x, _d), dx, delta, ptr(rp, _i64), ptr(col, _i32), tot, C.byref(mb))
    return rp, col[:tot], mb.value


def slit_mark(x, rp, col, slits):
    s = np.ascontiguousarray(np.asarray(slits, dtype=np.float64).reshape(-1))
    br = np.zeros(max(len(col), 1), dtype=np.uint8)
    lib().or_slit_mark(len(rp) - 1, ptr(x, _d), ptr(rp, _i64), ptr(col, _i32), len(s) // 6, ptr(s, _d), ptr(br, _u8))
    return br[:len(col)]


def mls_contributors(x, rp, col, rw):
    n = len(rp) - 1
    cp = np.zeros(n + 1, dtype=np.int64)
    tot = lib().or_mls_contributors(n, ptr(x, _d), ptr(rp, _i64), ptr(col, _i32), rw, ptr(cp, _i64), ptr(None, _i32))
    ci = np.zeros(max(tot, 1), dtype=np.int32)
    lib().or_mls_contributors(n, ptr(x, _d), ptr(rp, _i64), ptr(col, _i32), rw, ptr(cp, _i64), ptr(ci, _i32))
    return cp, ci[:tot]


def mls_coeff(x, xg, npt, cp, ci, rw):
    n = len(cp) - 1
    co = np.zeros(max(int(cp[-1]) * npt, 1))
    rc = lib().or_mls_coeff(n, ptr(x, _d), ptr(xg, _d), npt, ptr(cp, _i64), ptr(ci, _i32), rw, ptr(co, _d))
    if rc != 0:
        raise RuntimeError(f"singular moment matrix at node {-rc - 1}")
    return co[: int(cp[-1]) * npt]


class Model:
    """Holds numpy arrays alive and exposes an ``or_model``."""

    def __init__(self, **kw):
        self.keep = {}
        self.m = OrModel()
        n = int(kw["n"])
        self.m.n = n
        self.m.dx = kw["dx"]
        self.m.delta = kw["delta"]
        self.m.cci = int(kw.get("cci", 0))
        self.m.cci_mdf = int(kw.get("cci_mdf", 0))
        self.m.mls = int(kw.get("mls", 1))
        self.m.npt = int(kw.get("npt", 8))
        self.m.damping = float(kw.get("damping", 0.0))

        def put(name, arr, dtype, t):
            if arr is None:
                setattr(self.m, name, C.cast(None, t))
                return None
            a = np.ascontiguousarray(np.asarray(arr, dtype=dtype))
            self.keep[name] = a
            setattr(self.m, name, a.ctypes.data_as(t))
            return a

        put("x", kw["x"], np.float64, _d)
        put("xg", kw.get("xg"), np.float64, _d)
        put("gw", kw.get("gw"), np.float64, _d)
        put("fam_ptr", kw["fam_ptr"], np.int64, _i64)
        put("fam_col", kw["fam_col"], np.int32, _i32)
        br = kw.get("broken")
        put("broken", br if br is not None else np.zeros(len(kw["fam_col"]), np.uint8), np.uint8, _u8)
        put("cb_ptr", kw.get("cb_ptr"), np.int64, _i64)
        put("cb_idx", kw.get("cb_idx"), np.int32, _i32)
        put("coeff", kw.get("coeff"), np.float64, _d)
        put("bdry_eff", kw.get("bdry_eff", np.ones(n)), np.float64, _d)
        put("mat", kw.get("mat", np.zeros(n)), np.int32, _i32)
        for k in ("mat_spring", "mat_ecrit", "mat_density", "mat_ymod"):
            put(k, kw[k], np.float64, _d)
        put("mat_grav", kw.get("mat_grav", np.zeros(3 * len(kw["mat_spring"]))), np.float64, _d)
        put("bc", kw.get("bc", -np.ones(n)), np.int32, _i32)
        nbc = max(len(kw.get("bc_type", [])), 1)
        put("bc_type", kw.get("bc_type", np.zeros(nbc)), np.int32, _i32)
        put("bc_dir", kw.get("bc_dir", np.zeros(3 * nbc)), np.int32, _i32)
        put("bc_val", kw.get("bc_val", np.zeros(9 * nbc)), np.float64, _d)
        put("bc_end", kw.get("bc_end", np.ones(nbc)), np.float64, _d)
        put("bc_load", kw.get("bc_load", 2 * np.ones(nbc)), np.float64, _d)
        put("spring_factor", kw.get("spring_factor"), np.float64, _d)
        self.U = put("U", kw.get("U", np.zeros(3 * n)), np.float64, _d)
        self.V = put("V", kw.get("V", np.zeros(3 * n)), np.float64, _d)
        self.vbuf = put("vbuf", np.zeros(3 * n), np.float64, _d)
        self.ug = put("ug", kw.get("ug", np.zeros(n * self.m.npt * 3)), np.float64, _d)
        self.eed = put("eed", np.zeros(n), np.float64, _d)

    @property
    def ref(self):
        return C.byref(self.m)

    def bdry_eff(self, dims, center):
        n = self.m.n
        out = np.zeros(n)
        d = (C.c_int * 3)(*dims)
        c = np.asarray(center, dtype=np.float64)
        full = lib().or_bdry_eff(self.ref, d, ptr(c, _d), ptr(out, _d))
        return out, full

    def gather(self, t, us):
        us = np.ascontiguousarray(us, dtype=np.float64)
        lib().or_gather(self.ref, t, ptr(us, _d))

    def force_stage(self, dts, t, us):
        us = np.ascontiguousarray(us, dtype=np.float64)
        k = np.zeros(3 * self.m.n)
        lib().or_force_stage(self.ref, dts, t, ptr(us, _d), ptr(k, _d))
        return k

    def rk4_step(self, dt, t):
        lib().or_rk4_step(self.ref, dt, t)
        return self.m.ke, self.m.ee

    def static_apply(self, t, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        lib().or_static_apply(self.ref, t, ptr(x, _d), ptr(y, _d))
        return y

    def static_rhs(self, t):
        b = np.zeros(3 * self.m.n)
        lib().or_static_rhs(self.ref, t, ptr(b, _d))
        return b

    def adjoint_grad(self, dt, t0, nsteps, lam_U, lam_V=None):
        lu = np.ascontiguousarray(lam_U, dtype=np.float64)
        lv = None if lam_V is None else np.ascontiguousarray(lam_V, dtype=np.float64)
        g = np.zeros(self.m.n)
        rc = lib().or_adjoint_grad(self.ref, dt, t0, int(nsteps), ptr(lu, _d), ptr(lv, _d), ptr(g, _d))
        if rc != 0:
            raise MemoryError("or_adjoint_grad")
        return g

    def static_cg(self, t, b, rtol=1e-10, maxit=100000):
        x = np.zeros(3 * self.m.n)
        rr = C.c_double(0)
        it = lib().or_static_cg(self.ref, t, ptr(b, _d), ptr(x, _d), rtol, maxit, C.byref(rr))
        return x, it, rr.value
