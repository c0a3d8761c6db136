"""Drive the unmodified reference libraries (oracle/_ref/*.so) through their own C APIs.

TEST INFRASTRUCTURE ONLY (checker and CPU baseline).  Each helper follows the call
sequence of the reference's sample drivers:

* newton:  PG5/newton/direct/direct.c:133-176 (g5_set_xmj, g5_set_eps_to_all, g5_set_n,
  g5_calculate_force_on_x)
* table:   PG5/table/force_prof/force_prof.c (g5_open builds the S2 table; a custom shape is
  installed with pg5_gen_force_table after g5_open, pg5_table.h:38-40)
* quad:    PG5/newton_quad/source.cpp:847-866 (g5c_set_xmjMC, g5c_set_nMC,
  g5c_calculate_force_on_xMC)
* hermite: PG6/banana/hermite.c:214-252 (g6_set_ti, g6calc_firsthalf, g6calc_lasthalf*)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as _o

D = np.float64
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)
fp = C.POINTER(C.c_float)


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


class RefG5:
    """GRAPE-5 newton library (libpg5_ref.so or the SYMMETRIC build)."""

    def __init__(self, symmetric: bool = False):
        self.sym = symmetric
        self.L = _o.load_ref("libpg5sym_ref.so" if symmetric else "libpg5_ref.so")
        L = self.L
        L.g5_open.restype = None
        L.g5_set_eps_to_all.argtypes = [C.c_double]
        L.g5_set_n.argtypes = [C.c_int]
        if symmetric:
            L.g5_set_xmj.argtypes = [C.c_int, C.c_int, dp, dp, dp]
        else:
            L.g5_set_xmj.argtypes = [C.c_int, C.c_int, dp, dp]
        L.g5_calculate_force_on_x.argtypes = [dp, dp, dp, C.c_int]
        L.g5_calculate_force_on_xe.argtypes = [dp, dp, dp, dp, C.c_int]
        L.g5_get_jmemsize.restype = C.c_int
        L.g5_open()

    def force(self, xj, mj, eps, xi, eps2j=None, eps2i=None):
        xj = np.ascontiguousarray(xj, D)
        mj = np.ascontiguousarray(mj, D)
        xi = np.ascontiguousarray(xi, D)
        nj, ni = len(xj), len(xi)
        if self.sym:
            e = np.ascontiguousarray(np.broadcast_to(eps2j, (nj,)), D)
            self.L.g5_set_xmj(0, nj, _p(xj), _p(mj), _p(e))
        else:
            self.L.g5_set_xmj(0, nj, _p(xj), _p(mj))
        self.L.g5_set_eps_to_all(eps)
        self.L.g5_set_n(nj)
        acc = np.zeros((ni, 3), D)
        pot = np.zeros(ni, D)
        if eps2i is not None:
            e2 = np.ascontiguousarray(np.broadcast_to(eps2i, (ni,)), D)
            self.L.g5_calculate_force_on_xe(_p(xi), _p(e2), _p(acc), _p(pot), ni)
        else:
            self.L.g5_calculate_force_on_x(_p(xi), _p(acc), _p(pot), ni)
        return acc, pot


class RefG5Table:
    """GRAPE-5 table (cutoff-force) library, libpg5table_ref.so (512-entry table)."""

    EXP_BIT, FRC_BIT = 4, 5

    def __init__(self):
        L = self.L = _o.load_ref("libpg5table_ref.so")
        L.g5_open.restype = None
        L.g5_set_n.argtypes = [C.c_int]
        L.g5_set_xmj.argtypes = [C.c_int, C.c_int, dp, dp]
        L.g5_calculate_force_on_x.argtypes = [dp, dp, dp, C.c_int]
        L.pg5_gen_force_table.argtypes = [C.c_void_p, C.c_double]
        L.g5_open()
        self._cb = None

    def set_table(self, func, rcut):
        self._cb = _o.FORCE_FN(func)
        self.L.pg5_gen_force_table(C.cast(self._cb, C.c_void_p), rcut)

    def table(self):
        """The library's Force_table[512][2] (exported data symbol)."""
        arr = (C.c_float * (2 << (self.EXP_BIT + self.FRC_BIT))).in_dll(self.L, "Force_table")
        return np.frombuffer(arr, np.float32).reshape(-1, 2).copy()

    def force(self, xj, mj, xi):
        xj = np.ascontiguousarray(xj, D)
        mj = np.ascontiguousarray(mj, D)
        xi = np.ascontiguousarray(xi, D)
        self.L.g5_set_xmj(0, len(xj), _p(xj), _p(mj))
        self.L.g5_set_n(len(xj))
        acc = np.zeros((len(xi), 3), D)
        pot = np.zeros(len(xi), D)
        self.L.g5_calculate_force_on_x(_p(xi), _p(acc), _p(pot), len(xi))
        return acc, pot


class RefQuad:
    """newton_quad library (g5_* monopole + g5c_* quadrupole cells), libquad_ref.so."""

    def __init__(self):
        L = self.L = _o.load_ref("libquad_ref.so")
        L.g5_open.restype = None
        L.g5_set_eps_to_all.argtypes = [C.c_double]
        L.g5_set_xmjMC.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp]
        L.g5_set_nMC.argtypes = [C.c_int, C.c_int]
        L.g5_calculate_force_on_xMC.argtypes = [C.c_int, dp, dp, dp, C.c_int]
        L.g5c_set_xmjMC.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp]
        L.g5c_set_nMC.argtypes = [C.c_int, C.c_int]
        L.g5c_calculate_force_on_xMC.argtypes = [C.c_int, dp, dp, dp, C.c_int]
        L.g5_open()

    def force(self, eps, xi, xj, mj, xc, mc, qc, devid=0):
        """Returns (acc_mono, pot_mono, acc_quad, pot_quad) exactly as the API returns them."""
        xi = np.ascontiguousarray(xi, D)
        ni = len(xi)
        self.L.g5_set_eps_to_all(eps)
        out = []
        xj = np.ascontiguousarray(xj, D)
        mj = np.ascontiguousarray(mj, D)
        self.L.g5_set_xmjMC(devid, 0, len(xj), _p(xj), _p(mj))
        self.L.g5_set_nMC(devid, len(xj))
        a = np.zeros((ni, 3), D)
        p = np.zeros(ni, D)
        self.L.g5_calculate_force_on_xMC(devid, _p(xi), _p(a), _p(p), ni)
        out += [a, p]
        xc = np.ascontiguousarray(xc, D)
        mc = np.ascontiguousarray(mc, D)
        qc = np.ascontiguousarray(qc, D)
        self.L.g5c_set_xmjMC(devid, 0, len(xc), _p(xc), _p(mc), _p(qc))
        self.L.g5c_set_nMC(devid, len(xc))
        a = np.zeros((ni, 3), D)
        p = np.zeros(ni, D)
        self.L.g5c_calculate_force_on_xMC(devid, _p(xi), _p(a), _p(p), ni)
        out += [a, p]
        return tuple(out)


class RefG6:
    """GRAPE-6 library, libpg6_ref.so (AVX2 + OpenMP)."""

    NPIPES = 48

    def __init__(self):
        L = self.L = _o.load_ref("libpg6_ref.so")
        L.g6_open.argtypes = [C.c_int]
        L.g6_npipes.restype = C.c_int
        L.g6_set_j_particle.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                        dp, dp, dp, dp, dp]
        L.g6_set_ti.argtypes = [C.c_int, C.c_double]
        fh = [C.c_int, C.c_int, C.c_int, ip, dp, dp, dp, dp, dp, C.c_double, dp]
        L.g6calc_firsthalf.argtypes = fh
        base = [C.c_int, C.c_int, C.c_int, ip, dp, dp, C.c_double, dp, dp, dp, dp]
        L.g6calc_lasthalf.argtypes = base
        L.g6calc_lasthalf2.argtypes = base + [ip]
        L.g6calc_lasthalf2p.argtypes = base + [ip, fp]
        L.g6calc_lasthalfn.argtypes = base
        L.g6calc_lasthalf2n.argtypes = base + [ip]
        L.g6calc_lasthalf2np.argtypes = base + [ip, fp]
        L.g6_read_neighbour_list.argtypes = [C.c_int]
        L.g6_get_neighbour_list.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip]
        L.g6_open(0)

    def set_j(self, pos, vel, acc2, jrk6, mass, tj, idx=None):
        n = len(pos)
        pos, vel, acc2, jrk6 = (np.ascontiguousarray(a, D) for a in (pos, vel, acc2, jrk6))
        snp = np.zeros(3, D)
        for j in range(n):
            self.L.g6_set_j_particle(0, j, int(idx[j]) if idx is not None else j, float(tj[j]), 0.0,
                                     float(mass[j]), _p(snp), _p(jrk6[j]), _p(acc2[j]), _p(vel[j]),
                                     _p(pos[j]))

    def set_j_at(self, adr, pos, vel, acc2, jrk6, mass, tj):
        """g6_set_j_particle for the j addresses adr (records taken from the full arrays)."""
        pos, vel, acc2, jrk6 = (np.ascontiguousarray(a, D) for a in (pos, vel, acc2, jrk6))
        snp = np.zeros(3, D)
        for j in adr:
            j = int(j)
            self.L.g6_set_j_particle(0, j, j, float(tj[j]), 0.0, float(mass[j]), _p(snp), _p(jrk6[j]),
                                     _p(acc2[j]), _p(vel[j]), _p(pos[j]))

    def calc(self, ti, nj, xi, vi, idi, eps2, h2=None, variant="2p"):
        """One g6_set_ti + chunked firsthalf/lasthalf<variant> over all i (chunks of npipes)."""
        xi = np.ascontiguousarray(xi, D)
        vi = np.ascontiguousarray(vi, D)
        idi = np.ascontiguousarray(idi, np.int32)
        ni = len(xi)
        h2 = np.ascontiguousarray(np.zeros(ni) if h2 is None else np.broadcast_to(h2, (ni,)), D)
        acc = np.zeros((ni, 3), D)
        jrk = np.zeros((ni, 3), D)
        pot = np.zeros(ni, D)
        nnb = np.zeros(ni, np.int32)
        rnnb = np.zeros(ni, np.float32)
        nbl = {}
        self.L.g6_set_ti(0, ti)
        npipe = self.NPIPES
        fn = getattr(self.L, "g6calc_lasthalf" + ("" if variant == "plain" else variant))
        for i0 in range(0, ni, npipe):
            n = min(npipe, ni - i0)
            sl = slice(i0, i0 + n)
            args = [0, nj, n, _p(idi[sl], C.c_int), _p(xi[sl]), _p(vi[sl])]
            self.L.g6calc_firsthalf(*args, _p(acc[sl]), _p(jrk[sl]), _p(pot[sl]), eps2, _p(h2[sl]))
            rest = [eps2, _p(h2[sl]), _p(acc[sl]), _p(jrk[sl]), _p(pot[sl])]
            if variant in ("2", "2n"):
                rest.append(_p(nnb[sl], C.c_int))
            if variant in ("2p", "2np"):
                rest += [_p(nnb[sl], C.c_int), _p(rnnb[sl], C.c_float)]
            fn(*args, *rest)
            if variant in ("n", "2n", "2np"):
                err = self.L.g6_read_neighbour_list(0)
                for ii in range(n):
                    cnt = C.c_int()
                    buf = np.zeros(1024, np.int32)
                    rc = self.L.g6_get_neighbour_list(0, ii, 1024, C.byref(cnt), _p(buf, C.c_int))
                    nbl[i0 + ii] = (rc, err, buf[:cnt.value].copy() if rc == 0 else None)
        return dict(acc=acc, jrk=jrk, pot=pot, nnb=nnb, rnnb=rnnb, nbl=nbl)
