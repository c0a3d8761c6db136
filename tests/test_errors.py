"""Error reporting of the C ABI (CPU only: every case is refused before any GPU work).

The reference asserts (or writes out of bounds); these libraries record an error code and a
message (pgb5_last_error / pgb6_last_error) and, by default, abort like assert().  With abort
switched off the call returns without doing anything.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import pgb

ARG, CAPACITY = 2, 3


@pytest.fixture
def g5():
    lib = pgb.ffi.G5()
    lib.set_abort(False)
    lib.clear_error()
    yield lib
    lib.clear_error()
    lib.set_abort(True)


@pytest.fixture
def g6():
    lib = pgb.ffi.G6()
    lib.set_abort(False)
    lib.clear_error()
    yield lib
    lib.clear_error()
    lib.set_abort(True)


def test_g5_negative_address_is_refused(g5):
    x = np.zeros((4, 3))
    m = np.zeros(4)
    g5.L.g5_set_xmj(-1, 4, pgb.ffi.ptr(x), pgb.ffi.ptr(m))
    code, msg = g5.last_error()
    assert code == ARG and "adr -1" in msg


def test_g5_unknown_batched_kind_is_refused(g5):
    h = C.c_void_p()
    items = np.zeros((1, 4), np.int32)
    rc = g5.L.pgb5_plan_create(C.byref(h), 7, 1, pgb.ffi.ptr(items, C.c_int))
    assert rc == ARG and g5.last_error()[0] == ARG and not h.value


def test_g6_negative_address_and_oversized_call_are_refused(g6):
    v = np.zeros(3)
    g6.L.g6_set_j_particle(0, -5, 0, 0.0, 0.0, 1.0, pgb.ffi.ptr(v), pgb.ffi.ptr(v), pgb.ffi.ptr(v),
                           pgb.ffi.ptr(v), pgb.ffi.ptr(v))
    assert g6.last_error()[0] == ARG
    g6.clear_error()
    ni = g6.L.g6_npipes() + 1          # more i-particles than pipelines (phantom_g6.c: NPIPES)
    x = np.zeros((ni, 3))
    idx = np.arange(ni, dtype=np.int32)
    out = np.zeros((ni, 3))
    pot = np.zeros(ni)
    rc = g6.L.g6calc_lasthalf(0, 10, ni, pgb.ffi.ptr(idx, C.c_int), pgb.ffi.ptr(x), pgb.ffi.ptr(x), 1e-4,
                              pgb.ffi.ptr(pot), pgb.ffi.ptr(out), pgb.ffi.ptr(out), pgb.ffi.ptr(pot))
    code, msg = g6.last_error()
    assert rc == 0 and code == ARG and "pipes" in msg


def test_g6_batched_plan_rejects_negative_items(g6):
    h = C.c_void_p()
    items = np.array([[0, 10, 0, -1]], np.int32)
    rc = g6.L.pgb6_plan_create(C.byref(h), 1, pgb.ffi.ptr(items, C.c_int), 0)
    assert rc == ARG and not h.value


def test_g5_plan_update_refuses_a_null_plan(g5):
    items = np.zeros((1, 4), np.int32)
    assert g5.L.pgb5_plan_update(None, 1, pgb.ffi.ptr(items, C.c_int)) == ARG
    code, msg = g5.last_error()
    assert code == ARG and "pgb5_plan_update" in msg


def test_g6_plan_update_and_set_config_refuse_a_null_plan(g6):
    items = np.zeros((1, 4), np.int32)
    assert g6.L.pgb6_plan_update(None, 1, pgb.ffi.ptr(items, C.c_int)) == ARG
    assert "pgb6_plan_update" in g6.last_error()[1]
    g6.clear_error()
    assert g6.L.pgb6_plan_set_config(None, 0) == ARG
