"""The rest of the drop-in surface: the Fortran twins and g5_set_cutoff_table.

* Fortran twins (``g5_*_`` of PG5/newton/libpg5/pg5_fortran.c:1-119, ``g6*_`` of
  PG6/libpg6/phantom_g6.c): every argument by pointer.  A GRAPE-5 direct sum and a GRAPE-6
  block-step call made through the twins give the C entry points' results bit for bit (GPU).
* ``g5_set_cutoff_table(ffunc, fcut, fcor, pfunc, pcut, pcor)``: a stub in the reference
  (PG5/table/libpg5/phantom_g5.c:79-84); here it installs ffunc as the cutoff-force shape.  The
  table it builds equals the one pg5_gen_force_table(ffunc, fcut) builds, in this library and
  in the reference's own build (oracle/_ref/libpg5table_ref.so), bit for bit (CPU: table
  generation is host work).
"""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import pgb, gpu_available
from oracle import oracle as O

dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def _shape(r):
    return math.erfc(r / 0.02) / (r * r + 1e-4) ** 1.5 if r > 0 else 1e6


def test_cutoff_table_equals_gen_force_table():
    tab = pgb.ffi.G5Table()
    L = tab.L
    L.g5_set_cutoff_table.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_double, C.c_double]
    L.g5_set_cutoff_table.restype = None
    cb = pgb.ffi.FORCE_FN(_shape)
    try:
        L.pg5_set_table_bits(4, 5)
        L.g5_set_cutoff_table(C.cast(cb, C.c_void_p), 0.05, 0.0, None, 0.0, 0.0)
        t_cut, xs_cut = tab.table()
        tab.set_table(_shape, 0.05)
        t_gen, xs_gen = tab.table()
        assert t_cut.tobytes() == t_gen.tobytes() and xs_cut == xs_gen
        # a different shape replaces it
        tab.set_table(lambda r: 1.0 / (r * r + 1e-3) ** 1.5, 0.05)
        assert tab.table()[0].tobytes() != t_cut.tobytes()
        L.g5_set_cutoff_table(C.cast(cb, C.c_void_p), 0.05, 0.0, None, 0.0, 0.0)
        assert tab.table()[0].tobytes() == t_cut.tobytes()
        if O.ref_available("libpg5table_ref.so"):
            from oracle import refapi
            R = refapi.RefG5Table()
            R.set_table(_shape, 0.05)
            assert R.table().tobytes() == t_cut.tobytes()
    finally:
        L.pg5_set_table_bits(4, 5)


@pytest.mark.gpu
def test_fortran_twins_match_the_c_entry_points():
    if not gpu_available():
        pytest.skip("no GPU")
    W = pgb.workloads
    # GRAPE-5 direct sum (direct.c:133-176 sequence) through both ABIs
    g5 = pgb.ffi.G5()
    L = g5.L
    for name, args in (("g5_open_", []), ("g5_set_xmj_", [ip, ip, dp, dp]), ("g5_set_eps_to_all_", [dp]),
                       ("g5_set_n_", [ip]), ("g5_calculate_force_on_x_", [dp, dp, dp, ip]),
                       ("g5_get_number_of_pipelines_", []), ("g5_get_jmemsize_", [])):
        getattr(L, name).argtypes = args
    L.g5_get_number_of_pipelines_.restype = C.c_int
    L.g5_get_jmemsize_.restype = C.c_int
    s = W.plummer_g5(2000, seed=W.SEED0 + 40)
    x = np.ascontiguousarray(s.x)
    m = np.ascontiguousarray(s.m)
    n = len(m)
    a_c, p_c = g5.force(x, m, s.eps, x)
    a_f, p_f = np.zeros((n, 3)), np.zeros(n)
    L.g5_open_()
    L.g5_set_xmj_(C.byref(C.c_int(0)), C.byref(C.c_int(n)), _p(x), _p(m))
    L.g5_set_eps_to_all_(C.byref(C.c_double(s.eps)))
    L.g5_set_n_(C.byref(C.c_int(n)))
    L.g5_calculate_force_on_x_(_p(x), _p(a_f), _p(p_f), C.byref(C.c_int(n)))
    assert a_f.tobytes() == a_c.tobytes() and p_f.tobytes() == p_c.tobytes()
    assert L.g5_get_number_of_pipelines_() == L.g5_get_number_of_pipelines()
    assert L.g5_get_jmemsize_() == L.g5_get_jmemsize()

    # GRAPE-6: j-memory, set_ti, firsthalf + lasthalf2p (hermite.c:214-252) through both ABIs
    g6 = pgb.ffi.G6()
    L6 = g6.L
    st = W.hermite_state(3000, seed=W.SEED0 + 41)
    act = np.arange(0, 3000, 71, dtype=np.int32)[:48]
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    L6.g6_open_.argtypes = [ip]
    L6.g6_set_j_particle_.argtypes = [ip, ip, ip, dp, dp, dp, dp, dp, dp, dp, dp]
    L6.g6_set_ti_.argtypes = [ip, dp]
    L6.g6calc_firsthalf_.argtypes = [ip, ip, ip, ip, dp, dp, dp, dp, dp, dp, dp]
    L6.g6calc_lasthalf2p_.argtypes = [ip, ip, ip, ip, dp, dp, dp, dp, dp, dp, dp, ip, C.POINTER(C.c_float)]
    L6.g6calc_lasthalf2p_.restype = C.c_int
    L6.g6_npipes_.restype = C.c_int
    L6.g6_open_(C.byref(C.c_int(0)))
    zero = C.c_int(0)
    snp = np.zeros(3)
    for j in range(3000):
        L6.g6_set_j_particle_(C.byref(zero), C.byref(C.c_int(j)), C.byref(C.c_int(int(st.idx[j]))),
                              C.byref(C.c_double(st.tj[j])), C.byref(C.c_double(0.0)),
                              C.byref(C.c_double(st.mass[j])), _p(snp), _p(st.jrk6[j]), _p(st.acc2[j]),
                              _p(st.vel[j]), _p(st.pos[j]))
    ni = len(act)
    xi, vi = np.ascontiguousarray(xp[act]), np.ascontiguousarray(vp[act])
    idi = np.ascontiguousarray(st.idx[act])
    acc, jrk, pot = np.zeros((ni, 3)), np.zeros((ni, 3)), np.zeros(ni)
    h2 = np.zeros(ni)
    nnb = np.zeros(ni, np.int32)
    rnnb = np.zeros(ni, np.float32)
    L6.g6_set_ti_(C.byref(zero), C.byref(C.c_double(st.t_now)))
    nj, nic, e2 = C.c_int(3000), C.c_int(ni), C.c_double(st.eps2)
    L6.g6calc_firsthalf_(C.byref(zero), C.byref(nj), C.byref(nic), _p(idi, C.c_int), _p(xi), _p(vi), _p(acc),
                         _p(jrk), _p(pot), C.byref(e2), _p(h2))
    rc = L6.g6calc_lasthalf2p_(C.byref(zero), C.byref(nj), C.byref(nic), _p(idi, C.c_int), _p(xi), _p(vi),
                               C.byref(e2), _p(h2), _p(acc), _p(jrk), _p(pot), _p(nnb, C.c_int),
                               _p(rnnb, C.c_float))
    assert rc == 0
    assert L6.g6_npipes_() == L6.g6_npipes()
    res = g6.calc(st.t_now, 3000, xi, vi, idi, st.eps2, variant="2p")
    assert acc.tobytes() == res["acc"].tobytes() and jrk.tobytes() == res["jrk"].tobytes()
    assert pot.tobytes() == res["pot"].tobytes()
    assert np.array_equal(nnb, res["nnb"]) and rnnb.tobytes() == res["rnnb"].astype(np.float32).tobytes()
