"""PG5 table (cutoff-force, TreePM PP) path: lib/libpg5table.so.

CPU tests (no GPU): the force-shape table the library generates is bit-identical to the one
the reference library builds (oracle/_ref/libpg5table_ref.so, Force_table) and to the oracle's
restatement, for the default S2 table and for a custom shape.

GPU tests: forces against the FP64 evaluation of the same table + linear interpolation
(oracle.g5_table) with rms relative error <= 1e-6, and against the reference's AVX2 kernel
(max relative 1e-4: both use the same FP32 table; the reference sums in FP32).
"""
import math

import numpy as np
import pytest

from conftest import pgb, gpu_available
from oracle import oracle as O

W = pgb.workloads
S2_PP, S2_PM = 0.1 / 64, 3.0 / 64   # PG5/table/libpg5/pppm.h:4-6


def rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def rms(x):
    return float(np.sqrt(np.mean(np.square(x))))


@pytest.fixture(scope="module")
def tab():
    return pgb.ffi.G5Table()


def test_default_s2_table_matches_reference_bits(tab):
    tab.L.pg5_set_table_bits(4, 5)
    tab.L.pg5_gen_s2_force_table(S2_PP, S2_PM)
    t, xs = tab.table()
    assert t.shape == (512, 2)
    o, oxs = O.gen_force_table(4, 5, lambda r: O.s2_force(r, S2_PP, S2_PM), S2_PM)
    assert t.tobytes() == o.tobytes() and xs == oxs
    if O.ref_available("libpg5table_ref.so"):
        from oracle import refapi
        ref = refapi.RefG5Table()       # g5_open builds the S2 table
        assert ref.table().tobytes() == t.tobytes()


def test_custom_table_1024_entries_matches_oracle(tab):
    n = 1 << 20
    rs = 1.25 / n ** (1 / 3)
    f = W.gaussian_split_force(rs, 4.5 * rs, 0.1 / n ** (1 / 3))
    tab.set_table(f, 4.5 * rs, frc_bit=6)
    t, xs = tab.table()
    assert t.shape == (1024, 2)
    o, oxs = O.gen_force_table(4, 6, f, 4.5 * rs)
    assert t.tobytes() == o.tobytes() and xs == oxs
    assert t[-1, 0] == 0.0 and t[-1, 1] == 0.0   # zero force at and beyond the cutoff
    tab.L.pg5_set_table_bits(4, 5)


@pytest.mark.skipif(not O.ref_available("libpg5table_ref.so"), reason="reference not built")
def test_custom_table_512_matches_reference_bits(tab):
    from oracle import refapi
    f = W.gaussian_split_force(0.01, 0.045, 0.001)
    tab.set_table(f, 0.045, frc_bit=5)
    ref = refapi.RefG5Table()
    ref.set_table(f, 0.045)
    assert ref.table().tobytes() == tab.table()[0].tobytes()


def _box(n, seed):
    rng = W.Rng(seed)
    return rng.uniform(3 * n).reshape(-1, 3).astype(np.float32).astype(np.float64)


@pytest.mark.gpu
def test_s2_forces_vs_fp64_table_and_reference(tab):
    if not gpu_available():
        pytest.skip("no GPU")
    tab.L.pg5_set_table_bits(4, 5)
    tab.L.g5_open()
    t, xs = tab.table()
    xj = 0.2 * _box(6000, 3)
    mj = np.full(len(xj), 1.0 / 6000)
    xi = xj[::5].copy()
    a, p = tab.force(xj, mj, xi)
    assert np.all(p == 0.0)
    # the API rounds the scaled coordinates to float (j: (float)x * (float)xscale, i: through
    # double, PG5/table/libpg5/phantom_g5.c:96-128); the FP64 oracle gets those same inputs
    xj_s = (xj.astype(np.float32) * np.float32(xs)).astype(np.float64) / xs
    xi_s = (xi.astype(np.float32).astype(np.float64) * xs).astype(np.float32).astype(np.float64) / xs
    ao = O.g5_table(xi_s, xj_s, mj, t, 4, 5, xs)
    assert rms(rel(a, ao)) <= 1e-6, rms(rel(a, ao))
    if O.ref_available("libpg5table_ref.so"):
        from oracle import refapi
        ar, _ = refapi.RefG5Table().force(xj, mj, xi)
        assert rel(a, ar).max() <= 1e-4


@pytest.mark.gpu
def test_treepm_groups_batched_vs_fp64(tab):
    """Small TreePM set: every group's forces from one batched launch vs the FP64 table oracle."""
    if not gpu_available():
        pytest.skip("no GPU")
    import torch
    ts = W.treepm_groups(1 << 15, mesh=32, block=8, nmax=512)
    f = W.gaussian_split_force(ts.rs, ts.rcut, ts.eps)
    tab.set_table(f, ts.rcut, frc_bit=6)
    t, xs = tab.table()
    # device records are in table units: x' = x * xscale (j in float arithmetic, as set_xmj does)
    ip = np.zeros((len(ts.xi), 4), np.float32)
    ip[:, :3] = (ts.xi * xs).astype(np.float32)
    jp = np.zeros((len(ts.xj), 4), np.float32)
    jp[:, :3] = ts.xj.astype(np.float32) * np.float32(xs)
    jp[:, 3] = ts.mj
    dev = torch.device("cuda")
    d_i = torch.from_numpy(ip).to(dev)
    d_j = torch.from_numpy(jp).to(dev)
    d_o = torch.zeros((len(ts.xi), 4), dtype=torch.float64, device=dev)
    plan = tab.plan_create(ts.items)
    outs = []
    try:
        # the kernel configurations the table kind can use (CTAs of <= 256 threads); the others
        # are refused
        for cfg in range(11):
            if cfg in (2, 3, 4, 8, 9, 10):   # 8-10: the j-paired form (point masses and cells only)
                tab.set_abort(False)
                try:
                    assert tab.L.pgb5_plan_set_config(plan, cfg) != 0
                finally:
                    tab.set_abort(True)
                continue
            rc = tab.L.pgb5_plan_set_config(plan, cfg)
            assert rc == 0
            tab.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), d_o.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            outs.append(d_o.cpu().numpy().copy())
    finally:
        tab.plan_destroy(plan)
    out = outs[0]
    for o in outs[1:]:
        assert rms(rel(o[:, :3], out[:, :3])) <= 1e-6
    errs = []
    for k in range(0, len(ts.items), 7):
        i0, ni, j0, nj = ts.items[k]
        ao = O.g5_table(ip[i0:i0 + ni, :3].astype(np.float64) / xs, jp[j0:j0 + nj, :3].astype(np.float64) / xs,
                        ts.mj[j0:j0 + nj], t, 4, 6, xs)
        errs.append(rel(out[i0:i0 + ni, :3], ao))
    assert rms(np.concatenate(errs)) <= 1e-6
    # the plain per-group API gives the same forces as the batched launch
    k = 3
    i0, ni, j0, nj = ts.items[k]
    a, _ = tab.force(ts.xj[j0:j0 + nj], ts.mj[j0:j0 + nj], ts.xi[i0:i0 + ni])
    assert rms(rel(a, out[i0:i0 + ni, :3])) <= 1e-6
    tab.L.pg5_set_table_bits(4, 5)
