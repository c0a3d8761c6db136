"""ctypes bindings of the B200 force-engine libraries, mirroring the reference C APIs.

The libraries are the product; this module only binds them for Python callers (tests,
benchmark).  Every class exposes the reference's own function names and argument meaning:

* ``G5``       -> lib/libpg5.so      (PG5/newton/libpg5/gp5util.h:10-39, quad_util.h:8-15)
* ``G5Sym``    -> lib/libpg5sym.so   (same API built with symmetric softening)
* ``G5Table``  -> lib/libpg5table.so (PG5/table/libpg5/gp5util.h:9-35, pg5_table.h:38-40)
* ``G6``       -> lib/libpg6.so      (PG6/libpg6/gp6util.h:1-101)

Loading fails loudly (``OSError``) if a library has not been built: there is no fallback.
Each library is opened privately (RTLD_LOCAL) because the GRAPE-5 libraries share names.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")

dp = C.POINTER(C.c_double)
fp = C.POINTER(C.c_float)
ip = C.POINTER(C.c_int)
vp = C.c_void_p


def lib_path(name: str) -> str:
    return os.path.join(LIBDIR, name)


def _load(name: str) -> C.CDLL:
    path = lib_path(name)
    if not os.path.exists(path):
        raise OSError(f"{path} is not built (run __graft_entry__.build() or make -C phantom-grape_b200)")
    return C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)


def _sig(L, name, args, res=None):
    f = getattr(L, name)
    f.argtypes = args
    f.restype = res
    return f


def ptr(a, t=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


class _ErrMixin:
    prefix = "pgb5"

    def last_error(self):
        buf = C.create_string_buffer(512)
        code = getattr(self.L, f"{self.prefix}_last_error")(buf, 512)
        return code, buf.value.decode()

    def clear_error(self):
        getattr(self.L, f"{self.prefix}_clear_error")()

    def set_abort(self, on: bool):
        getattr(self.L, f"{self.prefix}_set_abort")(1 if on else 0)


class G5(_ErrMixin):
    """GRAPE-5 newton + newton_quad API (libpg5.so) or its symmetric build (libpg5sym.so)."""

    LIBNAME = "libpg5.so"
    SYMMETRIC = False
    # kinds of the batched path (include/pgb_g5.h)
    NEWTON, SYMMETRIC_KIND, QUAD = 0, 1, 2

    def __init__(self):
        L = self.L = _load(self.LIBNAME)
        _sig(L, "g5_open", [])
        _sig(L, "g5_close", [])
        _sig(L, "g5_get_number_of_pipelines", [], C.c_int)
        _sig(L, "g5_get_jmemsize", [], C.c_int)
        _sig(L, "g5_set_eps_to_all", [C.c_double])
        _sig(L, "g5_set_eps", [C.c_int, dp])
        _sig(L, "g5_set_epsMC", [C.c_int, C.c_int, dp])
        _sig(L, "g5_set_n", [C.c_int])
        _sig(L, "g5_set_nMC", [C.c_int, C.c_int])
        _sig(L, "g5_set_xi", [C.c_int, dp])
        _sig(L, "g5_set_xiMC", [C.c_int, C.c_int, dp])
        _sig(L, "g5_set_xei", [C.c_int, dp, dp])
        _sig(L, "g5_set_xeiMC", [C.c_int, C.c_int, dp, dp])
        if self.SYMMETRIC:
            _sig(L, "g5_set_xmj", [C.c_int, C.c_int, dp, dp, dp])
            _sig(L, "g5_set_xmjMC", [C.c_int, C.c_int, C.c_int, dp, dp, dp])
        else:
            _sig(L, "g5_set_xmj", [C.c_int, C.c_int, dp, dp])
            _sig(L, "g5_set_xmjMC", [C.c_int, C.c_int, C.c_int, dp, dp])
        _sig(L, "g5_run", [])
        _sig(L, "g5_runMC", [C.c_int])
        _sig(L, "g5_get_force", [C.c_int, dp, dp])
        _sig(L, "g5_get_forceMC", [C.c_int, C.c_int, dp, dp])
        _sig(L, "g5_calculate_force_on_x", [dp, dp, dp, C.c_int])
        _sig(L, "g5_calculate_force_on_xMC", [C.c_int, dp, dp, dp, C.c_int])
        _sig(L, "g5_calculate_force_on_xe", [dp, dp, dp, dp, C.c_int])
        _sig(L, "g5_calculate_force_on_xeMC", [C.c_int, dp, dp, dp, dp, C.c_int])
        _sig(L, "g5c_set_nMC", [C.c_int, C.c_int])
        _sig(L, "g5c_set_xmjMC", [C.c_int, C.c_int, C.c_int, dp, dp, dp])
        _sig(L, "g5c_set_xmjMC0", [C.c_int, C.c_int, C.c_int, dp, dp, dp])
        _sig(L, "g5c_runMC", [C.c_int])
        _sig(L, "g5c_runMC0", [C.c_int])
        _sig(L, "g5c_calculate_force_on_xMC", [C.c_int, dp, dp, dp, C.c_int])
        _sig(L, "g5c_calculate_force_on_xMC0", [C.c_int, dp, dp, dp, C.c_int])
        _sig(L, "pgb5_last_error", [C.c_char_p, C.c_int], C.c_int)
        _sig(L, "pgb5_clear_error", [])
        _sig(L, "pgb5_set_abort", [C.c_int])
        _sig(L, "pgb5_plan_create", [C.POINTER(vp), C.c_int, C.c_int, ip], C.c_int)
        _sig(L, "pgb5_plan_launch", [vp, vp, vp, vp, vp, vp], C.c_int)
        _sig(L, "pgb5_plan_destroy", [vp])
        _sig(L, "pgb5_plan_interactions", [vp], C.c_longlong)
        _sig(L, "pgb5_plan_tasks", [vp], C.c_int)

    # convenience wrappers with numpy arrays -------------------------------------------------
    def set_xmj(self, adr, xj, mj, epsj2=None, devid=None):
        xj, mj = f64(xj, (-1, 3)), f64(mj)
        nj = len(xj) - adr if adr else len(xj)
        if self.SYMMETRIC:
            e = f64(np.broadcast_to(epsj2, (len(mj),)))
            if devid is None:
                self.L.g5_set_xmj(adr, nj, ptr(xj), ptr(mj), ptr(e))
            else:
                self.L.g5_set_xmjMC(devid, adr, nj, ptr(xj), ptr(mj), ptr(e))
        elif devid is None:
            self.L.g5_set_xmj(adr, nj, ptr(xj), ptr(mj))
        else:
            self.L.g5_set_xmjMC(devid, adr, nj, ptr(xj), ptr(mj))

    def calculate_force_on_x(self, x, eps2=None, devid=None):
        x = f64(x, (-1, 3))
        ni = len(x)
        a = np.zeros((ni, 3))
        p = np.zeros(ni)
        if eps2 is not None:
            e = f64(np.broadcast_to(eps2, (ni,)))
            if devid is None:
                self.L.g5_calculate_force_on_xe(ptr(x), ptr(e), ptr(a), ptr(p), ni)
            else:
                self.L.g5_calculate_force_on_xeMC(devid, ptr(x), ptr(e), ptr(a), ptr(p), ni)
        elif devid is None:
            self.L.g5_calculate_force_on_x(ptr(x), ptr(a), ptr(p), ni)
        else:
            self.L.g5_calculate_force_on_xMC(devid, ptr(x), ptr(a), ptr(p), ni)
        return a, p

    def force(self, xj, mj, eps, xi, epsj2=None):
        """One direct-sum evaluation the way PG5/newton/direct/direct.c:133-176 drives it."""
        self.L.g5_open()
        self.set_xmj(0, xj, mj, epsj2)
        self.L.g5_set_eps_to_all(eps)
        self.L.g5_set_n(len(mj))
        return self.calculate_force_on_x(xi)

    def quad_force(self, eps, xi, xc, mc, qc, devid=0):
        xi, xc, mc, qc = f64(xi, (-1, 3)), f64(xc, (-1, 3)), f64(mc), f64(qc, (-1, 6))
        self.L.g5_set_eps_to_all(eps)
        self.L.g5c_set_xmjMC(devid, 0, len(xc), ptr(xc), ptr(mc), ptr(qc))
        self.L.g5c_set_nMC(devid, len(xc))
        a = np.zeros((len(xi), 3))
        p = np.zeros(len(xi))
        self.L.g5c_calculate_force_on_xMC(devid, ptr(xi), ptr(a), ptr(p), len(xi))
        return a, p

    # batched path --------------------------------------------------------------------------
    def plan_create(self, kind, items):
        items = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
        h = vp()
        rc = self.L.pgb5_plan_create(C.byref(h), kind, len(items), ptr(items, C.c_int))
        if rc:
            raise RuntimeError(f"pgb5_plan_create failed: {self.last_error()}")
        return h

    def plan_launch(self, plan, ipos, jpos, jaux, out, stream=0):
        rc = self.L.pgb5_plan_launch(plan, ipos, jpos, jaux, out, stream)
        if rc:
            raise RuntimeError(f"pgb5_plan_launch failed: {self.last_error()}")

    def plan_destroy(self, plan):
        self.L.pgb5_plan_destroy(plan)


class G5Sym(G5):
    LIBNAME = "libpg5sym.so"
    SYMMETRIC = True
