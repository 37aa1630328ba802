"""B200-native pdMTEL hot path: Python face of libpdmtel_b200.so.

The product is the shared library (CUDA kernels for sm_100a behind the C ABI
of include/pdmtel_b200.h, and the C++ pdDataManager/pdSolve host layer of
include/pdmtel_host.h).  This module only binds it with ctypes:

* ``pdDataManager`` / ``pdSolve`` mirror the reference's classes
  (pdDataManager.h:39-268, pdSolve.h:18-47) for a working folder holding a
  ``pds_input.txt`` deck;
* ``DeviceContext`` wraps a ``pd_ctx`` for direct array-level use.

There is no CPU fallback: loading fails loudly if the library is missing,
and every GPU entry point raises ``PdError`` when no CUDA device exists.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

__all__ = ["PdError", "lib", "pdDataManager", "pdSolve", "DeviceContext", "PREC_FP64", "PREC_FP32C", "PREC_FP64A",
           "LIB_PATH"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpdmtel_b200.so")

PD_OK = 0
PREC_FP64, PREC_FP32C, PREC_FP64A = 0, 1, 2
OPT_F64_LANES_BELOW, OPT_TILE, OPT_PERSIST_BLOCKS_PER_SM = 1, 2, 3
OPT_PERSIST_FORCE_CHUNK, OPT_PERSIST_GATHER_CHUNK, OPT_STATIC_STENCIL, OPT_GATHER_PER_POINT = 4, 5, 6, 7
OPT_FORCE_TILE, OPT_FORCE_QUAD, OPT_PERSIST_WAIT_US, OPT_PERSIST_TEST_STALL = 8, 9, 10, 11
OPT_GATHER_SELL, OPT_FORCE_STENCIL, OPT_GATHER_STENCIL, OPT_STATIC_PRECOND = 12, 13, 14, 15
OPT_STATIC_SPLIT, OPT_STATIC_F32_BELOW, OPT_ADJOINT_VJP32 = 16, 17, 18
BC_DISPL, BC_VELOC, BC_DISPLGRAD, BC_TRACTION = 1, 2, 3, 4
INTG_CCI, INTG_FGI, INTG_AI = 0, 1, 2
_ERRS = {-1: "PD_ERR_ARG", -2: "PD_ERR_OOM", -3: "PD_ERR_CUDA", -4: "PD_ERR_TIMEOUT", -5: "PD_ERR_SINGULAR",
         -6: "PD_ERR_CAPACITY", -7: "PD_ERR_NOCONV", -8: "PD_ERR_NODEV"}


class PdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRS.get(code, code)}: {msg}")
        self.code = code


_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)
_u8 = C.POINTER(C.c_uint8)
_vp = C.c_void_p


class pd_material(C.Structure):
    _fields_ = [("spring", C.c_double), ("density", C.c_double), ("ecrit", C.c_double), ("grav", C.c_double * 3)]


class pd_ai_region(C.Structure):
    _fields_ = [("a", C.c_double), ("b", C.c_double), ("axis", C.c_uint8 * 3), ("lim", C.c_uint8 * 4),
                ("flags", C.c_uint8)]


class pd_bc(C.Structure):
    _fields_ = [("type", C.c_int32), ("dir", C.c_int32 * 3), ("value", C.c_double * 9), ("end_time", C.c_double),
                ("load_type", C.c_double)]


class pd_problem(C.Structure):
    _fields_ = [("num_nodes", C.c_int64), ("coords", _d), ("mat_id", _i32), ("bc_id", _i32),
                ("num_materials", C.c_int32), ("materials", C.POINTER(pd_material)), ("num_bcs", C.c_int32),
                ("bcs", C.POINTER(pd_bc)), ("grid_spacing", C.c_double), ("horizon", C.c_double),
                ("integration", C.c_int32), ("cci_modified", C.c_int32), ("intg_point", C.c_int32),
                ("abscissae", _d), ("weights", _d), ("damping", C.c_double), ("num_slits", C.c_int32),
                ("slits", _d), ("spring_factor", _d), ("stream", _vp)]


class pdh_info(C.Structure):
    _fields_ = [("num_nodes", C.c_int64), ("num_halves", C.c_int64), ("num_broken", C.c_int64),
                ("num_contrib", C.c_int64), ("num_gauss", C.c_int32), ("cci", C.c_int32), ("mls", C.c_int32),
                ("bdry_eff_on", C.c_int32), ("dims", C.c_int32 * 3), ("total_step", C.c_int32),
                ("dump_frequency", C.c_int32), ("num_max_family", C.c_int32), ("grid_spacing", C.c_double),
                ("horizon", C.c_double), ("total_time", C.c_double), ("stable_dt", C.c_double),
                ("min_bond_length", C.c_double), ("ke", C.c_double), ("ee", C.c_double),
                ("num_materials", C.c_int32), ("num_bcs", C.c_int32), ("intg_point", C.c_int32),
                ("pad", C.c_int32), ("damping", C.c_double)]


class pd_tune_result(C.Structure):
    _fields_ = [("tile", C.c_int64), ("persistent", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("force_chunk", C.c_int32), ("gather_chunk", C.c_int32), ("trials", C.c_int32),
                ("ms_per_step", C.c_double), ("gather_per_point", C.c_int32), ("pad", C.c_int32),
                ("force_tile", C.c_int64), ("force_quad", C.c_int32), ("gather_sell", C.c_int32),
                ("force_stencil", C.c_int32), ("gather_stencil", C.c_int32)]


# name -> argtypes; every entry point returns int
_SIGS = {
    "pd_device_count": [C.POINTER(C.c_int)],
    "pd_ctx_create": [C.POINTER(pd_problem), C.POINTER(_vp)],
    "pd_ctx_destroy": [_vp],
    "pd_ctx_stream": [_vp, C.POINTER(_vp)],
    "pd_sync": [_vp],
    "pd_bond_search": [_vp, _i64, _i64, _d],
    "pd_get_family": [_vp, _i64, _i32, _u8],
    "pd_set_family": [_vp, _i64, _i32, _u8],
    "pd_set_bdry_eff": [_vp, _d],
    "pd_set_mls": [_vp, _i64, _i32, _d],
    "pd_mls_setup": [_vp, C.c_double, _d, _i64],
    "pd_get_mls": [_vp, _i64, _i32, _d],
    "pd_mls_size": [_vp, _i64],
    "pd_set_precision": [_vp, C.c_int],
    "pd_set_energy": [_vp, C.c_int],
    "pd_set_state": [_vp, _d, _d],
    "pd_get_state": [_vp, _d, _d],
    "pd_get_vbuf": [_vp, _d],
    "pd_set_gauss_displ": [_vp, _d],
    "pd_get_gauss_displ": [_vp, _d],
    "pd_get_energy_density": [_vp, _d],
    "pd_init_dynamic": [_vp],
    "pd_gather": [_vp, C.c_double, _d],
    "pd_force_stage": [_vp, C.c_double, C.c_double, _d, _d],
    "pd_rk4_step": [_vp, C.c_double, C.c_double, _d, _d],
    "pd_rk4_steps": [_vp, C.c_double, C.c_double, C.c_int],
    "pd_rk4_steps_host": [_vp, C.c_double, C.c_double, C.c_int, _d, _d, _d, _d],
    "pd_evals_per_stage": [_vp, _i64],
    "pd_reset_state": [_vp],
    "pd_profile_step": [_vp, C.c_double, C.c_double, _d],
    "pd_static_prepare": [_vp, C.POINTER(C.c_int)],
    "pd_static_matvec": [_vp, C.c_double, _d, _d],
    "pd_static_rhs": [_vp, C.c_double, _d],
    "pd_static_solve": [_vp, C.c_double, C.c_int, C.c_double, C.c_int, _d, C.POINTER(C.c_int), _d],
    "pd_set_spring_factor": [_vp, _d],
    "pd_set_option": [_vp, C.c_int, C.c_int64],
    "pd_get_option": [_vp, C.c_int, _i64],
    "pd_adjoint_forward": [_vp, C.c_double, C.c_double, C.c_int, C.c_int],
    "pd_adjoint_backward": [_vp, _d, _d, _d],
    "pdh_open": [C.c_char_p, C.POINTER(_vp)],
    "pdh_close": [_vp],
    "pdh_get_info": [_vp, C.POINTER(pdh_info)],
    "pdh_init_node": [_vp],
    "pdh_init_bond": [_vp],
    "pdh_init_material": [_vp],
    "pdh_init_bdry_effect_factor": [_vp],
    "pdh_init_grid_boundary": [_vp],
    "pdh_init_integration_point": [_vp],
    "pdh_initial_problem": [_vp],
    "pdh_set_family": [_vp, _i64, _i32, _u8, C.c_double],
    "pdh_set_spring_factor": [_vp, _d],
    "pdh_get_nodes": [_vp, _d, _i32, _i32],
    "pdh_get_family": [_vp, _i64, _i32, _u8],
    "pdh_get_bdry_eff": [_vp, _d],
    "pdh_get_mls": [_vp, _i64, _i32, _d],
    "pdh_context": [_vp, C.POINTER(_vp)],
    "pdh_set_precision": [_vp, C.c_int],
    "pdh_set_device_setup": [_vp, C.c_int],
    "pdh_post_afd": [_vp, C.c_int, C.c_int, _i32, _i32, _d, _i64],
    "pd_afd": [_vp, _d, _d, C.c_int64, _i64, _i64, _i32, _d],
    "pdh_solve_dynamic": [_vp, C.c_int],
    "pdh_solve_static": [_vp, C.c_int, C.c_double, C.POINTER(C.c_int), _d],
    "pdh_batch_create": [C.c_char_p, C.POINTER(_vp), C.c_int, C.POINTER(_vp)],
    "pdh_batch_offsets": [_vp, _i64],
    "pdh_batch_count": [_vp, C.POINTER(C.c_int)],
    "pdh_get_tables": [_vp, C.POINTER(pd_material), C.POINTER(pd_bc), _d, _d],
    "pd_rk4_steps_persistent": [_vp, C.c_double, C.c_double, C.c_int],
    "pd_set_boxes": [_vp, C.c_int, _i64],
    "pd_ai_plan": [C.c_int64, _d, _i64, _i32, C.c_double, C.c_double, _i64, C.POINTER(pd_ai_region), C.c_int64,
                   _i64],
    "pd_ai_mls_table": [C.c_int64, _d, _i64, _i32, _i64, C.POINTER(pd_ai_region), C.c_double, C.c_double, C.c_int,
                        _i64, _i32, C.c_double, _i64, _d, C.c_int64, _i64, _i64],
    "pd_set_ai": [_vp, C.c_int, _i64, C.POINTER(pd_ai_region), _i64, _i32, _i64, _d],
    "pd_get_damage": [_vp, _u8, _i32],
    "pd_autotune": [_vp, C.c_double, C.c_int, C.POINTER(pd_tune_result)],
}

_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Loads libpdmtel_b200.so (building it first if only the sources exist)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _b
            _b.build()
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.pd_last_error.restype = C.c_char_p
        L.pd_last_error.argtypes = []
        L.pdh_last_error.restype = C.c_char_p
        L.pdh_last_error.argtypes = [_vp]
        L.pd_abi_version.restype = C.c_int
        _lib = L
    return _lib


def _p(a, t):
    return C.cast(None, t) if a is None else a.ctypes.data_as(t)


def _check(rc: int, where: str, model=None):
    if rc != PD_OK:
        if model is not None:
            msg = lib().pdh_last_error(model).decode(errors="replace")
        else:
            msg = lib().pd_last_error().decode(errors="replace")
        raise PdError(rc, f"{where}: {msg}")


def device_count() -> int:
    n = C.c_int(0)
    lib().pd_device_count(C.byref(n))
    return n.value


def ai_plan(coords, row_ptr, col, grid_spacing, horizon):
    """Regions of every family entry of the adaptive-trapezoid form
    (pd_ai_plan; host only): (reg_ptr [entries + 1], regions array)."""
    x = _f64(coords)
    n = x.size // 3
    rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    ptr = np.zeros(int(rp[-1]) + 1, np.int64)
    cnt = C.c_int64(0)
    args = (n, _p(x, _d), _p(rp, _i64), _p(cl, _i32), float(grid_spacing), float(horizon), _p(ptr, _i64))
    _check(lib().pd_ai_plan(*args, None, 0, C.byref(cnt)), "pd_ai_plan")
    regs = (pd_ai_region * max(cnt.value, 1))()
    _check(lib().pd_ai_plan(*args, regs, cnt.value, C.byref(cnt)), "pd_ai_plan")
    return ptr, regs


def ai_mls_table(coords, row_ptr, col, reg_ptr, regions, grid_spacing, horizon, trap_index, cb_ptr, cb_idx, rw):
    """The per-node MLS coefficient lists of the adaptive-trapezoid form
    (pd_ai_mls_table; host only): (tab_ptr [n + 1], tab_coeff)."""
    x = _f64(coords)
    n = x.size // 3
    rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    gp = np.ascontiguousarray(reg_ptr, dtype=np.int64)
    cp = np.ascontiguousarray(cb_ptr, dtype=np.int64)
    ci = np.ascontiguousarray(cb_idx, dtype=np.int32)
    tp = np.zeros(n + 1, np.int64)
    cnt, bad = C.c_int64(0), C.c_int64(-1)
    head = (n, _p(x, _d), _p(rp, _i64), _p(cl, _i32), _p(gp, _i64), regions, float(grid_spacing), float(horizon),
            int(trap_index), _p(cp, _i64), _p(ci, _i32), float(rw), _p(tp, _i64))
    _check(lib().pd_ai_mls_table(*head, None, 0, C.byref(cnt), C.byref(bad)), "pd_ai_mls_table")
    co = np.zeros(max(cnt.value, 1))
    _check(lib().pd_ai_mls_table(*head, _p(co, _d), cnt.value, C.byref(cnt), C.byref(bad)), "pd_ai_mls_table")
    return tp, co[:cnt.value]


def _f64(a, n=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


class DeviceContext:
    """A ``pd_ctx``: device arrays of one problem (include/pdmtel_b200.h)."""

    def __init__(self, handle, owner=None, n=None, npt=None):
        self.h = handle
        self._owner = owner  # a pdDataManager owns the context when set
        self.n = n
        self.npt = npt

    @classmethod
    def create(cls, coords, mat_id, materials, bcs=(), bc_id=None, grid_spacing=1.0, horizon=3.015,
               integration=1, cci_modified=0, intg_point=2, abscissae=None, weights=None, damping=0.0,
               slits=(), spring_factor=None, stream=None):
        coords = _f64(coords)
        n = coords.size // 3
        keep = [coords]
        P = pd_problem()
        P.num_nodes = n
        P.coords = _p(coords, _d)
        mid = np.ascontiguousarray(np.asarray(mat_id, dtype=np.int32))
        keep.append(mid)
        P.mat_id = _p(mid, _i32)
        if bc_id is not None:
            bid = np.ascontiguousarray(np.asarray(bc_id, dtype=np.int32))
            keep.append(bid)
            P.bc_id = _p(bid, _i32)
        mats = (pd_material * len(materials))()
        for k, m in enumerate(materials):
            mats[k].spring, mats[k].density, mats[k].ecrit = m["spring"], m["density"], m["ecrit"]
            for a in range(3):
                mats[k].grav[a] = m.get("grav", (0.0, 0.0, 0.0))[a]
        P.num_materials = len(materials)
        P.materials = mats
        bct = (pd_bc * max(len(bcs), 1))()
        for k, b in enumerate(bcs):
            bct[k].type = b["type"]
            for a in range(3):
                bct[k].dir[a] = b["dir"][a]
            for a, v in enumerate(b["value"]):
                bct[k].value[a] = v
            bct[k].end_time = b.get("end_time", 1.0)
            bct[k].load_type = b.get("load_type", 2.0)
        P.num_bcs = len(bcs)
        P.bcs = bct
        P.grid_spacing, P.horizon = grid_spacing, horizon
        P.integration, P.cci_modified, P.intg_point = integration, cci_modified, intg_point
        if abscissae is not None:
            ab, wt = _f64(abscissae), _f64(weights)
            keep += [ab, wt]
            P.abscissae, P.weights = _p(ab, _d), _p(wt, _d)
        P.damping = damping
        if len(slits):
            sl = _f64(slits)
            keep.append(sl)
            P.num_slits = sl.size // 6
            P.slits = _p(sl, _d)
        if spring_factor is not None:
            sf = _f64(spring_factor, n)
            keep.append(sf)
            P.spring_factor = _p(sf, _d)
        P.stream = stream
        h = _vp()
        _check(lib().pd_ctx_create(C.byref(P), C.byref(h)), "pd_ctx_create")
        npt = intg_point ** 3 if integration == 1 else 1
        return cls(h, None, n, npt)

    def close(self):
        if self.h and self._owner is None:
            lib().pd_ctx_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        s = _vp()
        _check(lib().pd_ctx_stream(self.h, C.byref(s)), "pd_ctx_stream")
        return s.value or 0

    def sync(self):
        _check(lib().pd_sync(self.h), "pd_sync")

    def bond_search(self):
        nh, nb, mb = C.c_int64(0), C.c_int64(0), C.c_double(0)
        _check(lib().pd_bond_search(self.h, C.byref(nh), C.byref(nb), C.byref(mb)), "pd_bond_search")
        return nh.value, nb.value, mb.value

    def get_family(self, num_halves):
        rp = np.zeros(self.n + 1, np.int64)
        col = np.zeros(max(num_halves, 1), np.int32)
        br = np.zeros(max(num_halves, 1), np.uint8)
        _check(lib().pd_get_family(self.h, _p(rp, _i64), _p(col, _i32), _p(br, _u8)), "pd_get_family")
        return rp, col[:num_halves], br[:num_halves]

    def set_family(self, row_ptr, col, broken=None):
        rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
        cl = np.ascontiguousarray(col, dtype=np.int32)
        br = None if broken is None else np.ascontiguousarray(broken, dtype=np.uint8)
        _check(lib().pd_set_family(self.h, _p(rp, _i64), _p(cl, _i32), _p(br, _u8)), "pd_set_family")

    def set_bdry_eff(self, bE):
        b = _f64(bE, self.n)
        _check(lib().pd_set_bdry_eff(self.h, _p(b, _d)), "pd_set_bdry_eff")

    def set_ai(self, reg_ptr, regions, cb_ptr=None, cb_idx=None, tab_ptr=None, tab_coeff=None):
        """pd_set_ai: MLS on when the contributors and tables are given"""
        gp = np.ascontiguousarray(reg_ptr, dtype=np.int64)
        mls = cb_ptr is not None
        cp = np.ascontiguousarray(cb_ptr, dtype=np.int64) if mls else None
        ci = np.ascontiguousarray(cb_idx, dtype=np.int32) if mls else None
        tp = np.ascontiguousarray(tab_ptr, dtype=np.int64) if mls else None
        tc = _f64(tab_coeff) if mls else None
        _check(lib().pd_set_ai(self.h, int(mls), _p(gp, _i64), regions, _p(cp, _i64), _p(ci, _i32), _p(tp, _i64),
                               _p(tc, _d)), "pd_set_ai")

    def get_damage(self, num_halves):
        """(broken flags per family entry, failed points per node of the last step)"""
        br = np.zeros(max(num_halves, 1), np.uint8)
        cnt = np.zeros(self.n, np.int32)
        _check(lib().pd_get_damage(self.h, _p(br, _u8), _p(cnt, _i32)), "pd_get_damage")
        return br[:num_halves], cnt

    def set_mls(self, cb_ptr, cb_idx, coeff):
        cp = np.ascontiguousarray(cb_ptr, dtype=np.int64)
        ci = np.ascontiguousarray(cb_idx, dtype=np.int32)
        co = _f64(coeff)
        _check(lib().pd_set_mls(self.h, _p(cp, _i64), _p(ci, _i32), _p(co, _d)), "pd_set_mls")

    def mls_setup(self, rw, mls_coords=None):
        """InitIntegrationPoint on the device (pd_mls_setup); returns the
        number of contributor entries."""
        x = None if mls_coords is None else _f64(mls_coords, 3 * self.n)
        T = C.c_int64(0)
        _check(lib().pd_mls_setup(self.h, float(rw), _p(x, _d), C.byref(T)), "pd_mls_setup")
        return T.value

    def get_mls(self):
        """(cb_ptr, cb_idx, coeff) held by the context, in pd_set_mls's layout"""
        T = C.c_int64(0)
        _check(lib().pd_mls_size(self.h, C.byref(T)), "pd_mls_size")
        cp = np.zeros(self.n + 1, np.int64)
        ci = np.zeros(max(T.value, 1), np.int32)
        co = np.zeros(max(T.value * self.npt, 1))
        _check(lib().pd_get_mls(self.h, _p(cp, _i64), _p(ci, _i32), _p(co, _d)), "pd_get_mls")
        return cp, ci[:T.value], co[:T.value * self.npt]

    def set_precision(self, p):
        _check(lib().pd_set_precision(self.h, int(p)), "pd_set_precision")

    def set_energy(self, on):
        _check(lib().pd_set_energy(self.h, int(bool(on))), "pd_set_energy")

    def set_state(self, U=None, V=None):
        u = None if U is None else _f64(U, 3 * self.n)
        v = None if V is None else _f64(V, 3 * self.n)
        _check(lib().pd_set_state(self.h, _p(u, _d), _p(v, _d)), "pd_set_state")

    def get_state(self):
        U = np.zeros(3 * self.n)
        V = np.zeros(3 * self.n)
        _check(lib().pd_get_state(self.h, _p(U, _d), _p(V, _d)), "pd_get_state")
        return U, V

    def get_vbuf(self):
        v = np.zeros(3 * self.n)
        _check(lib().pd_get_vbuf(self.h, _p(v, _d)), "pd_get_vbuf")
        return v

    def get_gauss_displ(self):
        ug = np.zeros(3 * self.n * self.npt)
        _check(lib().pd_get_gauss_displ(self.h, _p(ug, _d)), "pd_get_gauss_displ")
        return ug

    def set_gauss_displ(self, ug):
        u = _f64(ug, 3 * self.n * self.npt)
        _check(lib().pd_set_gauss_displ(self.h, _p(u, _d)), "pd_set_gauss_displ")

    def get_energy_density(self):
        e = np.zeros(self.n)
        _check(lib().pd_get_energy_density(self.h, _p(e, _d)), "pd_get_energy_density")
        return e

    def init_dynamic(self):
        _check(lib().pd_init_dynamic(self.h), "pd_init_dynamic")

    def gather(self, t, us=None):
        u = None if us is None else _f64(us, 3 * self.n)
        _check(lib().pd_gather(self.h, float(t), _p(u, _d)), "pd_gather")

    def force_stage(self, dts, t, us):
        u = _f64(us, 3 * self.n)
        k = np.zeros(3 * self.n)
        _check(lib().pd_force_stage(self.h, float(dts), float(t), _p(u, _d), _p(k, _d)), "pd_force_stage")
        return k

    def rk4_step(self, dt, t):
        ke, ee = C.c_double(0), C.c_double(0)
        _check(lib().pd_rk4_step(self.h, float(dt), float(t), C.byref(ke), C.byref(ee)), "pd_rk4_step")
        return ke.value, ee.value

    def rk4_steps(self, dt, t0, nsteps):
        _check(lib().pd_rk4_steps(self.h, float(dt), float(t0), int(nsteps)), "pd_rk4_steps")

    def rk4_steps_host(self, dt, t0, nsteps, U_in, V_in, U_out, V_out):
        _check(lib().pd_rk4_steps_host(self.h, float(dt), float(t0), int(nsteps), _p(U_in, _d), _p(V_in, _d),
                                       _p(U_out, _d), _p(V_out, _d)), "pd_rk4_steps_host")

    def evals_per_stage(self):
        e = C.c_int64(0)
        _check(lib().pd_evals_per_stage(self.h, C.byref(e)), "pd_evals_per_stage")
        return e.value

    def reset_state(self):
        _check(lib().pd_reset_state(self.h), "pd_reset_state")

    def profile_step(self, dt, t):
        """Device ms of the force, gather, epilogue and other kernels of one step."""
        ms = np.zeros(4)
        _check(lib().pd_profile_step(self.h, float(dt), float(t), _p(ms, _d)), "pd_profile_step")
        return ms

    def static_matvec(self, t, x):
        xv = _f64(x, 3 * self.n)
        y = np.zeros_like(xv)
        _check(lib().pd_static_matvec(self.h, float(t), _p(xv, _d), _p(y, _d)), "pd_static_matvec")
        return y

    def static_rhs(self, t):
        b = np.zeros(3 * self.n)
        _check(lib().pd_static_rhs(self.h, float(t), _p(b, _d)), "pd_static_rhs")
        return b

    def static_prepare(self):
        st = C.c_int(0)
        _check(lib().pd_static_prepare(self.h, C.byref(st)), "pd_static_prepare")
        return bool(st.value)

    def static_solve(self, t, precision=PREC_FP64, rtol=1e-10, maxit=200000, x0=None):
        x = np.zeros(3 * self.n) if x0 is None else _f64(x0, 3 * self.n).copy()
        it, rr = C.c_int(0), C.c_double(0)
        _check(lib().pd_static_solve(self.h, float(t), int(precision), float(rtol), int(maxit), _p(x, _d),
                                     C.byref(it), C.byref(rr)), "pd_static_solve")
        return x, it.value, rr.value


    def set_option(self, option, value):
        _check(lib().pd_set_option(self.h, int(option), int(value)), "pd_set_option")

    def set_boxes(self, offsets):
        """pd_set_boxes: node ranges offsets[b] .. offsets[b + 1] - 1 that are
        complete box lattices (an empty list returns to one box)."""
        o = np.ascontiguousarray(offsets, dtype=np.int64)
        nb = max(len(o) - 1, 0)
        _check(lib().pd_set_boxes(self.h, nb, _p(o, _i64) if nb else None), "pd_set_boxes")

    def get_option(self, option):
        v = C.c_int64(0)
        _check(lib().pd_get_option(self.h, int(option), C.byref(v)), "pd_get_option")
        return v.value

    def rk4_steps_persistent(self, dt, t0, nsteps):
        _check(lib().pd_rk4_steps_persistent(self.h, float(dt), float(t0), int(nsteps)), "pd_rk4_steps_persistent")

    def autotune(self, dt, steps=3):
        R = pd_tune_result()
        _check(lib().pd_autotune(self.h, float(dt), int(steps), C.byref(R)), "pd_autotune")
        return {k: getattr(R, k) for k, _ in R._fields_}

    def set_spring_factor(self, f):
        fa = _f64(f, self.n)
        _check(lib().pd_set_spring_factor(self.h, _p(fa, _d)), "pd_set_spring_factor")

    def adjoint_forward(self, dt, t0, nsteps, checkpoint_every=50):
        _check(lib().pd_adjoint_forward(self.h, float(dt), float(t0), int(nsteps), int(checkpoint_every)),
               "pd_adjoint_forward")

    def adjoint_backward(self, lam_U, lam_V=None):
        """dJ/df for the adjoints lam_U, lam_V ([N, 3]) of the final state of
        the last adjoint_forward; the state returns to that run's start."""
        lu = _f64(lam_U, 3 * self.n)
        lv = None if lam_V is None else _f64(lam_V, 3 * self.n)
        g = np.zeros(self.n)
        _check(lib().pd_adjoint_backward(self.h, _p(lu, _d), _p(lv, _d), _p(g, _d)), "pd_adjoint_backward")
        return g


class pdDataManager:
    """The reference's pdDataManager for the working folder ``workdir``
    (SetWkDir + ReadInputFile happen on construction)."""

    def __init__(self, workdir: str):
        h = _vp()
        rc = lib().pdh_open(os.fsencode(os.path.abspath(workdir)), C.byref(h))
        self.h = h
        _check(rc, "pdh_open", self.h)

    @classmethod
    def batch(cls, out_dir: str, specimens):
        """One model over the specimen models (pdh_batch_create); the
        specimens must stay open while the batch lives."""
        os.makedirs(out_dir, exist_ok=True)
        arr = (_vp * len(specimens))(*[s.h for s in specimens])
        obj = cls.__new__(cls)
        obj._specimens = list(specimens)
        h = _vp()
        rc = lib().pdh_batch_create(os.fsencode(os.path.abspath(out_dir)), arr, len(specimens), C.byref(h))
        obj.h = h
        _check(rc, "pdh_batch_create", obj.h)
        return obj

    def batch_offsets(self):
        k = C.c_int(0)
        self._call("pdh_batch_count", C.byref(k))
        o = np.zeros(k.value + 1, np.int64)
        self._call("pdh_batch_offsets", _p(o, _i64))
        return o

    def tables(self):
        """(materials, bcs, abscissae, weights) as the device context gets them"""
        I = self.info()
        mats = (pd_material * max(I.num_materials, 1))()
        bcs = (pd_bc * max(I.num_bcs, 1))()
        n1 = max(I.intg_point, 1)
        ab, wt = np.zeros(n1), np.zeros(n1)
        self._call("pdh_get_tables", mats, bcs, _p(ab, _d), _p(wt, _d))
        ml = [{"spring": m.spring, "density": m.density, "ecrit": m.ecrit, "grav": tuple(m.grav)}
              for m in list(mats)[:I.num_materials]]
        bl = [{"type": b.type, "dir": tuple(b.dir), "value": tuple(b.value), "end_time": b.end_time,
               "load_type": b.load_type} for b in list(bcs)[:I.num_bcs]]
        return ml, bl, ab, wt

    def close(self):
        if self.h:
            lib().pdh_close(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args):
        _check(getattr(lib(), name)(self.h, *args), name, self.h)

    def info(self) -> pdh_info:
        I = pdh_info()
        self._call("pdh_get_info", C.byref(I))
        return I

    # pdSolve::InitialProblem steps
    def InitNode(self):
        self._call("pdh_init_node")

    def InitBond(self):
        self._call("pdh_init_bond")

    def InitMaterial(self):
        self._call("pdh_init_material")

    def InitBdryEffectFactor(self):
        self._call("pdh_init_bdry_effect_factor")

    def InitGridBoundary(self):
        self._call("pdh_init_grid_boundary")

    def InitIntegrationPoint(self):
        self._call("pdh_init_integration_point")

    def SetFamily(self, row_ptr, col, broken=None, min_bond=0.0):
        rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
        cl = np.ascontiguousarray(col, dtype=np.int32)
        br = None if broken is None else np.ascontiguousarray(broken, dtype=np.uint8)
        self._call("pdh_set_family", _p(rp, _i64), _p(cl, _i32), _p(br, _u8), float(min_bond))

    def SetSpringFactor(self, f):
        fa = _f64(f, self.info().num_nodes)
        self._call("pdh_set_spring_factor", _p(fa, _d))

    def SetPrecision(self, p):
        self._call("pdh_set_precision", int(p))

    def SetDeviceSetup(self, on=True):
        """InitIntegrationPoint on the device (pd_mls_setup); set it before
        InitIntegrationPoint.  The host setup (default) is the reference's
        arithmetic bit for bit; the device one differs only where glibc's pow
        is not correctly rounded."""
        self._call("pdh_set_device_setup", int(bool(on)))

    def CalcStableTimeStep(self) -> float:
        return self.info().stable_dt

    def nodes(self):
        n = self.info().num_nodes
        x = np.zeros(3 * n)
        m = np.zeros(n, np.int32)
        b = np.zeros(n, np.int32)
        self._call("pdh_get_nodes", _p(x, _d), _p(m, _i32), _p(b, _i32))
        return x, m, b

    def family(self):
        I = self.info()
        rp = np.zeros(I.num_nodes + 1, np.int64)
        col = np.zeros(max(I.num_halves, 1), np.int32)
        br = np.zeros(max(I.num_halves, 1), np.uint8)
        self._call("pdh_get_family", _p(rp, _i64), _p(col, _i32), _p(br, _u8))
        return rp, col[:I.num_halves], br[:I.num_halves]

    def bdry_eff(self):
        b = np.zeros(self.info().num_nodes)
        self._call("pdh_get_bdry_eff", _p(b, _d))
        return b

    def mls(self):
        I = self.info()
        cp = np.zeros(I.num_nodes + 1, np.int64)
        ci = np.zeros(max(I.num_contrib, 1), np.int32)
        co = np.zeros(max(I.num_contrib * I.num_gauss, 1))
        self._call("pdh_get_mls", _p(cp, _i64), _p(ci, _i32), _p(co, _d))
        return cp, ci[:I.num_contrib], co[:I.num_contrib * I.num_gauss]

    def context(self) -> DeviceContext:
        h = _vp()
        self._call("pdh_context", C.byref(h))
        I = self.info()
        return DeviceContext(h, owner=self, n=I.num_nodes, npt=I.num_gauss)


class pdSolve:
    """Static façade of the reference (pdSolve.h:18-47)."""

    @staticmethod
    def InitialProblem(dat: pdDataManager):
        dat._call("pdh_initial_problem")

    @staticmethod
    def SolveDynamic(dat: pdDataManager, write_files: bool = True):
        dat._call("pdh_solve_dynamic", int(bool(write_files)))

    @staticmethod
    def PostAFD(dat: pdDataManager, step: int, requests):
        """pdSolve::PostAFD without the console: the areal force density of
        pds_tecplot_<step>.dat on planes ("plane", normal 1..3, location)
        and nodes ("node", id), written to pds_AFD_<step>.dat."""
        n = len(requests)
        kind = np.zeros(max(n, 1), np.int32)
        norm = np.zeros(max(n, 1), np.int32)
        coord = np.zeros(max(n, 1))
        node = np.zeros(max(n, 1), np.int64)
        for k, r in enumerate(requests):
            if r[0] == "plane":
                kind[k], norm[k], coord[k] = 1, int(r[1]), float(r[2])
            elif r[0] == "node":
                kind[k], node[k] = 2, int(r[1])
            else:
                raise ValueError(f"unknown PostAFD request {r!r}")
        dat._call("pdh_post_afd", int(step), n, _p(kind, _i32), _p(norm, _i32), _p(coord, _d), _p(node, _i64))

    @staticmethod
    def SolveStatic(dat: pdDataManager, precision=PREC_FP64, rtol=1e-10):
        it, rr = C.c_int(0), C.c_double(0)
        dat._call("pdh_solve_static", int(precision), float(rtol), C.byref(it), C.byref(rr))
        return it.value, rr.value
