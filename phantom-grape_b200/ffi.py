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
    """GRAPE-5 newton + newton_quad API (libpg5.so) or its symmetric build (libpg5sym.so).

    ``lib`` picks another build of the same API, e.g. "libpg5_newton.so" (the reference's
    Newton-refined rsqrt)."""

    LIBNAME = "libpg5.so"
    SYMMETRIC = False
    # kinds of the batched path (include/pgb_g5.h)
    NEWTON, SYMMETRIC_KIND, QUAD = 0, 1, 2

    def __init__(self, lib: str = None):
        L = self.L = _load(lib or self.LIBNAME)
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
        _sig(L, "pgb5_plan_tune", [vp, vp, vp, vp, vp, vp, C.POINTER(C.c_float)], C.c_int)
        _sig(L, "pgb5_plan_config", [vp], C.c_int)
        _sig(L, "pgb5_plan_set_config", [vp, C.c_int], C.c_int)
        _sig(L, "pgb5_plan_update", [vp, C.c_int, ip], C.c_int)
        _sig(L, "pgb5_plan_launch_indexed", [vp, vp, vp, vp, vp, vp, vp], C.c_int)
        _sig(L, "pgb5_plan_tune_indexed", [vp, vp, vp, vp, vp, vp, vp, C.POINTER(C.c_float)], C.c_int)

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

    def plan_update(self, plan, items):
        """pgb5_plan_update: new items for an existing plan (configuration and buffers kept)."""
        items = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
        rc = self.L.pgb5_plan_update(plan, len(items), ptr(items, C.c_int))
        if rc:
            raise RuntimeError(f"pgb5_plan_update failed: {self.last_error()}")

    def plan_launch(self, plan, ipos, jpos, jaux, out, stream=0):
        rc = self.L.pgb5_plan_launch(plan, ipos, jpos, jaux, out, stream)
        if rc:
            raise RuntimeError(f"pgb5_plan_launch failed: {self.last_error()}")

    def plan_launch_indexed(self, plan, ipos, jpos, jaux, jidx, out, stream=0):
        rc = self.L.pgb5_plan_launch_indexed(plan, ipos, jpos, jaux, jidx, out, stream)
        if rc:
            raise RuntimeError(f"pgb5_plan_launch_indexed failed: {self.last_error()}")

    def plan_tune_indexed(self, plan, ipos, jpos, jaux, jidx, out, stream=0):
        """Autotune a plan launched with an index list; (cfg, ms)."""
        ms = C.c_float(0)
        cfg = self.L.pgb5_plan_tune_indexed(plan, ipos, jpos, jaux, jidx, out, stream, C.byref(ms))
        if cfg < 0:
            raise RuntimeError(f"pgb5_plan_tune_indexed failed: {self.last_error()}")
        return cfg, ms.value

    def plan_tune(self, plan, ipos, jpos, jaux, out, stream=0):
        """Autotune the plan's kernel configuration on these device arrays; (cfg, ms)."""
        ms = C.c_float(0)
        cfg = self.L.pgb5_plan_tune(plan, ipos, jpos, jaux, out, stream, C.byref(ms))
        if cfg < 0:
            raise RuntimeError(f"pgb5_plan_tune failed: {self.last_error()}")
        return cfg, ms.value

    def plan_destroy(self, plan):
        self.L.pgb5_plan_destroy(plan)


class G5Sym(G5):
    LIBNAME = "libpg5sym.so"
    SYMMETRIC = True


class G6(_ErrMixin):
    """GRAPE-6 API (libpg6.so): g6_open ... g6calc_lasthalf2np, plus the batched pgb6_* path.

    ``lib`` picks another build of the same API, e.g. "libpg6_newton.so" (the reference's
    Newton-refined rsqrt)."""

    prefix = "pgb6"
    NN = 1
    POS_F64 = 2

    def __init__(self, lib: str = "libpg6.so"):
        L = self.L = _load(lib)
        for n in ("g6_open", "g6_close", "g6_set_tunit", "g6_set_xunit", "g6_reset", "g6_reset_fofpga"):
            _sig(L, n, [C.c_int])
        _sig(L, "g6_npipes", [], C.c_int)
        _sig(L, "g6_setup_njdata", [C.c_int, C.c_int])
        _sig(L, "g6_set_j_particle", [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                      dp, dp, dp, dp, dp])
        _sig(L, "g6_set_ti", [C.c_int, C.c_double])
        _sig(L, "g6calc_firsthalf", [C.c_int, C.c_int, C.c_int, ip, dp, dp, dp, dp, dp, C.c_double, dp])
        base = [C.c_int, C.c_int, C.c_int, ip, dp, dp, C.c_double, dp, dp, dp, dp]
        _sig(L, "g6calc_lasthalf", base, C.c_int)
        _sig(L, "g6calc_lasthalf2", base + [ip], C.c_int)
        _sig(L, "g6calc_lasthalf2p", base + [ip, fp], C.c_int)
        _sig(L, "g6calc_lasthalfn", base, C.c_int)
        _sig(L, "g6calc_lasthalf2n", base + [ip], C.c_int)
        _sig(L, "g6calc_lasthalf2np", base + [ip, fp], C.c_int)
        _sig(L, "g6_read_neighbour_list", [C.c_int], C.c_int)
        _sig(L, "g6_get_neighbour_list", [C.c_int, C.c_int, C.c_int, ip, ip], C.c_int)
        _sig(L, "pgb6_last_error", [C.c_char_p, C.c_int], C.c_int)
        _sig(L, "pgb6_clear_error", [])
        _sig(L, "pgb6_set_abort", [C.c_int])
        _sig(L, "pgb6_set_call_timing", [C.c_int])
        _sig(L, "pgb6_call_device_ms", [C.c_int], C.c_double)
        _sig(L, "pgb6_record_sizes", [ip, ip, ip, ip])
        _sig(L, "pgb6_plan_create", [C.POINTER(vp), C.c_int, ip, C.c_int], C.c_int)
        _sig(L, "pgb6_plan_launch", [vp, vp, vp, C.c_double, vp, vp], C.c_int)
        _sig(L, "pgb6_plan_destroy", [vp])
        _sig(L, "pgb6_plan_interactions", [vp], C.c_longlong)
        _sig(L, "pgb6_plan_tasks", [vp], C.c_int)
        _sig(L, "pgb6_plan_config", [vp], C.c_int)
        _sig(L, "pgb6_plan_kernels", [vp], C.c_int)
        _sig(L, "pgb6_plan_chunks", [vp], C.c_int)
        _sig(L, "pgb6_plan_update", [vp, C.c_int, ip], C.c_int)
        _sig(L, "pgb6_plan_set_config", [vp, C.c_int], C.c_int)
        _sig(L, "pgb6_plan_tune", [vp, vp, vp, C.c_double, vp, vp, C.POINTER(C.c_float)], C.c_int)
        _sig(L, "pgb6_predict", [vp, C.c_int, C.c_double, vp, C.c_int, vp], C.c_int)
        _sig(L, "pgb6_batch_host", [C.c_int, ip, C.c_int, dp, dp, ip, C.c_int, dp, dp, dp, ip, C.c_double,
                                    dp, dp, dp, ip, fp], C.c_int)
        _sig(L, "pgb6_hermite_create", [C.POINTER(vp), C.c_int, dp, dp, dp, C.c_double, C.c_double, C.c_double,
                                        C.c_double], C.c_int)
        _sig(L, "pgb6_hermite_step", [vp, dp, ip], C.c_int)
        _sig(L, "pgb6_hermite_advance", [vp, C.c_double, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], C.c_int)
        _sig(L, "pgb6_hermite_time", [vp], C.c_double)
        _sig(L, "pgb6_hermite_set_wait_limit", [vp, C.c_longlong], C.c_int)
        _sig(L, "pgb6_hermite_wait_status", [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int)
        _sig(L, "pgb6_hermite_get", [vp, dp, dp, dp, dp, dp, dp, dp], C.c_int)
        _sig(L, "pgb6_hermite_last_step", [vp, ip, dp, dp, dp], C.c_int)
        _sig(L, "pgb6_hermite_energy", [vp, dp, dp], C.c_int)
        _sig(L, "pgb6_hermite_counts", [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)])
        _sig(L, "pgb6_hermite_stream", [vp], vp)
        _sig(L, "pgb6_hermite_stats", [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)])
        _sig(L, "pgb6_hermite_destroy", [vp])
        sz = [C.c_int() for _ in range(4)]
        L.pgb6_record_sizes(*[C.byref(s) for s in sz])
        self.sizes = dict(ptcl=sz[0].value, predj=sz[1].value, irec=sz[2].value, out=sz[3].value)

    # numpy helpers --------------------------------------------------------------------------
    def set_j(self, pos, vel, acc2, jrk6, mass, tj, idx=None, addr=None):
        """g6_set_j_particle for every particle (acc2 = acc/2, jrk6 = jerk/6)."""
        pos, vel, acc2, jrk6 = (f64(a, (-1, 3)) for a in (pos, vel, acc2, jrk6))
        snp = np.zeros(3)
        n = len(pos)
        for j in range(n):
            a = int(addr[j]) if addr is not None else j
            self.L.g6_set_j_particle(0, a, int(idx[j]) if idx is not None else j, float(tj[j]), 0.0,
                                     float(mass[j]), ptr(snp), ptr(jrk6[j]), ptr(acc2[j]), ptr(vel[j]),
                                     ptr(pos[j]))

    def calc(self, ti, nj, xi, vi, idi, eps2, h2=None, variant="2p", set_ti=True, maxlen=1024):
        """g6_set_ti + chunked g6calc_firsthalf / g6calc_lasthalf<variant> over all i."""
        xi, vi = f64(xi, (-1, 3)), f64(vi, (-1, 3))
        idi = np.ascontiguousarray(idi, np.int32)
        ni = len(xi)
        h2 = f64(np.zeros(ni) if h2 is None else np.broadcast_to(h2, (ni,)))
        acc = np.zeros((ni, 3))
        jrk = np.zeros((ni, 3))
        pot = np.zeros(ni)
        nnb = np.zeros(ni, np.int32)
        rnnb = np.zeros(ni, np.float32)
        nbl = {}
        if set_ti:
            self.L.g6_set_ti(0, ti)
        npipe = self.L.g6_npipes()
        fn = getattr(self.L, "g6calc_lasthalf" + ("" if variant == "plain" else variant))
        for i0 in range(0, ni, npipe):
            n = min(npipe, ni - i0)
            sl = slice(i0, i0 + n)
            args = [0, nj, n, ptr(idi[sl], C.c_int), ptr(xi[sl]), ptr(vi[sl])]
            self.L.g6calc_firsthalf(*args, ptr(acc[sl]), ptr(jrk[sl]), ptr(pot[sl]), eps2, ptr(h2[sl]))
            rest = [eps2, ptr(h2[sl]), ptr(acc[sl]), ptr(jrk[sl]), ptr(pot[sl])]
            if variant in ("2", "2n"):
                rest.append(ptr(nnb[sl], C.c_int))
            if variant in ("2p", "2np"):
                rest += [ptr(nnb[sl], C.c_int), ptr(rnnb[sl], C.c_float)]
            fn(*args, *rest)
            if variant in ("n", "2n", "2np"):
                err = self.L.g6_read_neighbour_list(0)
                for ii in range(n):
                    cnt = C.c_int()
                    buf = np.zeros(maxlen, np.int32)
                    rc = self.L.g6_get_neighbour_list(0, ii, maxlen, C.byref(cnt), ptr(buf, C.c_int))
                    nbl[i0 + ii] = (rc, err, buf[:cnt.value].copy() if rc == 0 else None)
        return dict(acc=acc, jrk=jrk, pot=pot, nnb=nnb, rnnb=rnnb, nbl=nbl)

    def batch_host(self, items, xi, vi, idi, xj, vj, mj, idj, eps2, nn=True):
        items = np.ascontiguousarray(items, np.int32).reshape(-1, 4)
        xi, vi, xj, vj, mj = f64(xi, (-1, 3)), f64(vi, (-1, 3)), f64(xj, (-1, 3)), f64(vj, (-1, 3)), f64(mj)
        idi = np.ascontiguousarray(idi, np.int32)
        idj = np.ascontiguousarray(idj, np.int32)
        ni = len(xi)
        acc = np.zeros((ni, 3))
        jrk = np.zeros((ni, 3))
        pot = np.zeros(ni)
        nnb = np.zeros(ni, np.int32) if nn else None
        rnnb = np.zeros(ni, np.float32) if nn else None
        rc = self.L.pgb6_batch_host(len(items), ptr(items, C.c_int), ni, ptr(xi), ptr(vi), ptr(idi, C.c_int),
                                    len(xj), ptr(xj), ptr(vj), ptr(mj), ptr(idj, C.c_int), eps2, ptr(acc),
                                    ptr(jrk), ptr(pot), ptr(nnb, C.c_int), ptr(rnnb, C.c_float))
        if rc:
            raise RuntimeError(f"pgb6_batch_host failed: {self.last_error()}")
        return dict(acc=acc, jrk=jrk, pot=pot, nnb=nnb, rnnb=rnnb)

    def plan_create(self, items, nn=True, f64=False):
        """f64: the device records hold FP64 positions (else the double-float layout)."""
        items = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
        h = vp()
        flags = (self.NN if nn else 0) | (self.POS_F64 if f64 else 0)
        rc = self.L.pgb6_plan_create(C.byref(h), len(items), ptr(items, C.c_int), flags)
        if rc:
            raise RuntimeError(f"pgb6_plan_create failed: {self.last_error()}")
        return h

    def plan_update(self, plan, items):
        """pgb6_plan_update: new items for an existing plan (configuration and buffers kept)."""
        items = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
        rc = self.L.pgb6_plan_update(plan, len(items), ptr(items, C.c_int))
        if rc:
            raise RuntimeError(f"pgb6_plan_update failed: {self.last_error()}")

    def plan_launch(self, plan, ipart, jpred, eps2, out, stream=0):
        rc = self.L.pgb6_plan_launch(plan, ipart, jpred, eps2, out, stream)
        if rc:
            raise RuntimeError(f"pgb6_plan_launch failed: {self.last_error()}")

    def plan_tune(self, plan, ipart, jpred, eps2, out, stream=0):
        ms = C.c_float()
        cfg = self.L.pgb6_plan_tune(plan, ipart, jpred, eps2, out, stream, C.byref(ms))
        if cfg < 0:
            raise RuntimeError(f"pgb6_plan_tune failed: {self.last_error()}")
        return cfg, ms.value

    def plan_destroy(self, plan):
        self.L.pgb6_plan_destroy(plan)


# Device record layouts (must match csrc/pgb_g6_kernels.cuh), as numpy structured dtypes.
G6PTCL = np.dtype([("pos", "<f8", 3), ("vel", "<f8", 3), ("acc2", "<f8", 3), ("jrk6", "<f8", 3),
                   ("mass", "<f8"), ("tim", "<f8"), ("idx", "<i4"), ("pad", "<i4", 3)])
# Positions: FP64 layout (x, y, z doubles) or the double-float layout (xh, yh, zh, xl, yl, zl
# floats, x = xh + xl) selected by the plan's PGB6_POS_F64 flag.
G6PREDJ = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("m", "<f4"), ("id", "<i4"),
                    ("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4"), ("pad", "<f4")])
G6IREC = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("vx", "<f4"), ("vy", "<f4"),
                   ("vz", "<f4"), ("id", "<i4"), ("h2", "<f4"), ("pad", "<f4")])
_FF = [("xh", "<f4"), ("yh", "<f4"), ("zh", "<f4"), ("xl", "<f4"), ("yl", "<f4"), ("zl", "<f4")]
G6PREDJ_FF = np.dtype(_FF + [("m", "<f4"), ("id", "<i4"), ("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4"),
                             ("pad", "<f4")])
G6IREC_FF = np.dtype(_FF + [("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4"), ("id", "<i4"), ("h2", "<f4"),
                            ("pad", "<f4")])


def _set_pos(rec, pos, ff):
    pos = np.asarray(pos, np.float64)
    for k, c in enumerate("xyz"):
        if ff:
            hi = pos[:, k].astype(np.float32)
            rec[c + "h"] = hi
            rec[c + "l"] = (pos[:, k] - hi.astype(np.float64)).astype(np.float32)
        else:
            rec[c] = pos[:, k]


def g6_irecords(pos, vel, ids, h2=None, ff=True):
    """i-particle records (G6I) as a numpy structured array."""
    rec = np.zeros(len(pos), G6IREC_FF if ff else G6IREC)
    _set_pos(rec, pos, ff)
    for k, c in enumerate("xyz"):
        rec["v" + c] = np.asarray(vel)[:, k]
    rec["id"] = ids
    if h2 is not None:
        rec["h2"] = h2
    return rec


def g6_jrecords(pos, vel, mass, ids, ff=True):
    """predicted j records (G6PredJ) as a numpy structured array."""
    rec = np.zeros(len(pos), G6PREDJ_FF if ff else G6PREDJ)
    _set_pos(rec, pos, ff)
    for k, c in enumerate("xyz"):
        rec["v" + c] = np.asarray(vel)[:, k]
    rec["m"] = mass
    rec["id"] = ids
    return rec
G6OUT = np.dtype([("ax", "<f8"), ("ay", "<f8"), ("az", "<f8"), ("jx", "<f8"), ("jy", "<f8"),
                  ("jz", "<f8"), ("pot", "<f8"), ("key", "<f4"), ("jadr", "<i4")])


FORCE_FN = C.CFUNCTYPE(C.c_double, C.c_double)


class G5Table(_ErrMixin):
    """GRAPE-5 table (cutoff force) API, libpg5table.so."""

    TABLE = 3   # kind of the batched path

    def __init__(self):
        L = self.L = _load("libpg5table.so")
        _sig(L, "g5_open", [])
        _sig(L, "g5_close", [])
        _sig(L, "g5_get_number_of_pipelines", [], C.c_int)
        _sig(L, "g5_set_range", [C.c_double, C.c_double, C.c_double])
        _sig(L, "g5_set_eta", [C.c_double])
        _sig(L, "g5_set_eps_to_all", [C.c_double])
        _sig(L, "g5_set_n", [C.c_int])
        _sig(L, "g5_set_nMC", [C.c_int, C.c_int])
        _sig(L, "g5_set_xmj", [C.c_int, C.c_int, dp, dp])
        _sig(L, "g5_set_xmjMC", [C.c_int, C.c_int, C.c_int, dp, dp])
        _sig(L, "g5_set_xi", [C.c_int, dp])
        _sig(L, "g5_set_xiMC", [C.c_int, C.c_int, dp])
        _sig(L, "g5_run", [])
        _sig(L, "g5_runMC", [C.c_int])
        _sig(L, "g5_get_force", [C.c_int, dp, dp])
        _sig(L, "g5_get_forceMC", [C.c_int, C.c_int, dp, dp])
        _sig(L, "g5_calculate_force_on_x", [dp, dp, dp, C.c_int])
        _sig(L, "g5_calculate_force_on_xMC", [C.c_int, dp, dp, dp, C.c_int])
        _sig(L, "g5_set_cutoff_table", [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_double, C.c_double])
        _sig(L, "pg5_gen_force_table", [C.c_void_p, C.c_double])
        _sig(L, "pg5_gen_s2_force_table", [C.c_double, C.c_double])
        _sig(L, "pg5_set_xscale", [C.c_double])
        _sig(L, "pg5_set_table_bits", [C.c_int, C.c_int], C.c_int)
        _sig(L, "pg5_get_table", [fp, C.c_int, dp], C.c_int)
        _sig(L, "pgb5_last_error", [C.c_char_p, C.c_int], C.c_int)
        _sig(L, "pgb5_clear_error", [])
        _sig(L, "pgb5_set_abort", [C.c_int])
        _sig(L, "pgb5_plan_create", [C.POINTER(vp), C.c_int, C.c_int, ip], C.c_int)
        _sig(L, "pgb5_plan_launch", [vp, vp, vp, vp, vp, vp], C.c_int)
        _sig(L, "pgb5_plan_destroy", [vp])
        _sig(L, "pgb5_plan_interactions", [vp], C.c_longlong)
        _sig(L, "pgb5_plan_tasks", [vp], C.c_int)
        _sig(L, "pgb5_plan_tune", [vp, vp, vp, vp, vp, vp, C.POINTER(C.c_float)], C.c_int)
        _sig(L, "pgb5_plan_config", [vp], C.c_int)
        _sig(L, "pgb5_plan_set_config", [vp, C.c_int], C.c_int)
        _sig(L, "pgb5_plan_update", [vp, C.c_int, ip], C.c_int)
        _sig(L, "pgb5_plan_launch_indexed", [vp, vp, vp, vp, vp, vp, vp], C.c_int)
        _sig(L, "pgb5_plan_tune_indexed", [vp, vp, vp, vp, vp, vp, vp, C.POINTER(C.c_float)], C.c_int)
        self._cb = None

    def set_table(self, func, rcut, frc_bit=None):
        if frc_bit is not None:
            self.L.pg5_set_table_bits(4, frc_bit)
        self._cb = FORCE_FN(func)  # keep the callback alive
        self.L.pg5_gen_force_table(C.cast(self._cb, C.c_void_p), rcut)

    def table(self):
        xs = C.c_double()
        n = self.L.pg5_get_table(None, 0, C.byref(xs))
        t = np.zeros((n, 2), np.float32)
        self.L.pg5_get_table(ptr(t, C.c_float), n, C.byref(xs))
        return t, xs.value

    def force(self, xj, mj, xi, devid=None):
        xj, mj, xi = f64(xj, (-1, 3)), f64(mj), f64(xi, (-1, 3))
        if devid is None:
            self.L.g5_set_xmj(0, len(xj), ptr(xj), ptr(mj))
            self.L.g5_set_n(len(xj))
        else:
            self.L.g5_set_xmjMC(devid, 0, len(xj), ptr(xj), ptr(mj))
            self.L.g5_set_nMC(devid, len(xj))
        a = np.zeros((len(xi), 3))
        p = np.zeros(len(xi))
        if devid is None:
            self.L.g5_calculate_force_on_x(ptr(xi), ptr(a), ptr(p), len(xi))
        else:
            self.L.g5_calculate_force_on_xMC(devid, ptr(xi), ptr(a), ptr(p), len(xi))
        return a, p

    def plan_create(self, items):
        items = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
        h = vp()
        rc = self.L.pgb5_plan_create(C.byref(h), self.TABLE, len(items), ptr(items, C.c_int))
        if rc:
            raise RuntimeError(f"pgb5_plan_create failed: {self.last_error()}")
        return h

    def plan_launch(self, plan, ipos, jpos, out, stream=0):
        rc = self.L.pgb5_plan_launch(plan, ipos, jpos, None, out, stream)
        if rc:
            raise RuntimeError(f"pgb5_plan_launch failed: {self.last_error()}")

    def plan_tune(self, plan, ipos, jpos, out, stream=0):
        """Autotune the plan's kernel configuration on these device arrays; (cfg, ms)."""
        ms = C.c_float(0)
        cfg = self.L.pgb5_plan_tune(plan, ipos, jpos, None, out, stream, C.byref(ms))
        if cfg < 0:
            raise RuntimeError(f"pgb5_plan_tune failed: {self.last_error()}")
        return cfg, ms.value

    def plan_destroy(self, plan):
        self.L.pgb5_plan_destroy(plan)


class Hermite:
    """The device Hermite block-time-step integrator (pgb6_hermite_*) over numpy arrays."""

    def __init__(self, g6: "G6", mass, pos, vel, eps2, eta, eta_s, dtmax):
        self.g6, self.L = g6, g6.L
        mass, pos, vel = f64(mass), f64(pos, (-1, 3)), f64(vel, (-1, 3))
        self.n = len(mass)
        h = vp()
        rc = self.L.pgb6_hermite_create(C.byref(h), self.n, ptr(mass), ptr(pos), ptr(vel), eps2, eta, eta_s, dtmax)
        if rc:
            raise RuntimeError(f"pgb6_hermite_create failed ({rc}): {g6.last_error()}")
        self.h = h

    def _check(self, rc, what):
        if rc:
            raise RuntimeError(f"pgb6_hermite_{what} failed ({rc}): {self.g6.last_error()}")

    def step(self):
        """One block step; (global time after it, particles advanced)."""
        t, ni = C.c_double(), C.c_int()
        self._check(self.L.pgb6_hermite_step(self.h, C.byref(t), C.byref(ni)), "step")
        return t.value, ni.value

    def advance(self, tend):
        """Block steps while the time is below tend; (particle steps, block steps) taken."""
        p, b = C.c_longlong(), C.c_longlong()
        self._check(self.L.pgb6_hermite_advance(self.h, tend, C.byref(p), C.byref(b)), "advance")
        return p.value, b.value

    @property
    def time(self):
        return self.L.pgb6_hermite_time(self.h)

    def set_wait_limit(self, cycles):
        """pgb6_hermite_set_wait_limit: the SM cycles after which a wait of the step kernel gives up."""
        self._check(self.L.pgb6_hermite_set_wait_limit(self.h, int(cycles)), "set_wait_limit")

    def wait_status(self):
        """(a wait gave up, CTAs returned from the step kernel so far, CTAs per launch)."""
        g, e, n = C.c_int(), C.c_int(), C.c_int()
        self._check(self.L.pgb6_hermite_wait_status(self.h, C.byref(g), C.byref(e), C.byref(n)), "wait_status")
        return g.value, e.value, n.value

    def get(self):
        n = self.n
        st = dict(t=np.zeros(n), dt=np.zeros(n), pos=np.zeros((n, 3)), vel=np.zeros((n, 3)),
                  acc=np.zeros((n, 3)), jrk=np.zeros((n, 3)), pot=np.zeros(n))
        self._check(self.L.pgb6_hermite_get(self.h, *(ptr(st[k]) for k in ("t", "dt", "pos", "vel", "acc", "jrk",
                                                                             "pot"))), "get")
        return st

    def last_step(self):
        n = self.n
        act = np.zeros(n, np.int32)
        acc, jrk, pot = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
        ni = self.L.pgb6_hermite_last_step(self.h, ptr(act, C.c_int), ptr(acc), ptr(jrk), ptr(pot))
        if ni < 0:
            raise RuntimeError(f"pgb6_hermite_last_step failed ({ni}): {self.g6.last_error()}")
        return act[:ni], acc[:ni], jrk[:ni], pot[:ni]

    def energy(self):
        ek, ew = C.c_double(), C.c_double()
        self._check(self.L.pgb6_hermite_energy(self.h, C.byref(ek), C.byref(ew)), "energy")
        return ek.value, ew.value

    def counts(self):
        p, b = C.c_longlong(), C.c_longlong()
        self.L.pgb6_hermite_counts(self.h, C.byref(p), C.byref(b))
        return p.value, b.value

    @property
    def stream(self):
        return self.L.pgb6_hermite_stream(self.h)

    def stats(self):
        """(pair interactions so far, steps by force i-tile 16 / 32 / 64 / 128 / 512)."""
        pairs, by = C.c_longlong(), (C.c_longlong * 5)()
        self.L.pgb6_hermite_stats(self.h, C.byref(pairs), by)
        return pairs.value, list(by)

    def close(self):
        if self.h:
            self.L.pgb6_hermite_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bind_noalloc(g6: "G6"):
    """Bind pgb6_force_noalloc (the allocation-free force call) on a G6 instance's library."""
    _sig(g6.L, "pgb6_force_noalloc", [vp, C.c_int, vp, C.c_int, C.c_double, vp, C.c_int, vp], C.c_int)
    return g6.L.pgb6_force_noalloc
