"""GPU parity of the Barnes-Hut quadrupole workload (newton_quad): interaction lists from the
host tree (drivers/pgb_bhtree.c) evaluated by the batched index-list launches (a PG5 newton
plan over the point-mass lists, a quadrupole plan over the cell lists) and by the per-group
drop-in calls (g5_*MC + g5c_*MC, as PG5/newton_quad/source.cpp:813-866 makes them).

Tolerances:
  * vs FP64 on the same lists (orc_g5_newton + orc_g5_quad on the same float32 inputs):
    rms relative acc and potential error <= 1e-6;
  * drop-in calls vs batched launches: rms relative <= 1e-6;
  * vs the full FP64 direct sum (multipole truncation at theta = 0.5, reported, not a parity
    bar): rms relative acc error <= 2e-3 -- a wrong sign or a missing term is far larger.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import pgb, gpu_available
from oracle import oracle as O

pytestmark = pytest.mark.gpu
W = pgb.workloads


def rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def rms(x):
    return float(np.sqrt(np.mean(np.square(x))))


@pytest.fixture(scope="module")
def g5():
    if not gpu_available():
        pytest.skip("no GPU")
    lib = pgb.ffi.G5()
    lib.L.g5_open()
    return lib


@pytest.fixture(scope="module")
def bh():
    return W.bh_hernquist(1 << 15)


def batched(g5, bh, cfg_p=None, cfg_c=None, tune=False):
    import torch
    dev = torch.device("cuda")
    ip, pp, cp, cq = bh.records()
    d_i, d_p = torch.from_numpy(ip).to(dev), torch.from_numpy(pp).to(dev)
    d_c, d_q = torch.from_numpy(cp).to(dev), torch.from_numpy(cq).to(dev)
    d_pi = torch.from_numpy(bh.pidx).to(dev)
    d_ci = torch.from_numpy(bh.cidx).to(dev)
    o_p = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    o_c = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    pl_p = g5.plan_create(g5.NEWTON, bh.items("p"))
    pl_c = g5.plan_create(g5.QUAD, bh.items("c"))
    try:
        if cfg_p is not None:
            assert g5.L.pgb5_plan_set_config(pl_p, cfg_p) == 0
        if cfg_c is not None:
            assert g5.L.pgb5_plan_set_config(pl_c, cfg_c) == 0
        if tune:
            g5.plan_tune_indexed(pl_p, d_i.data_ptr(), d_p.data_ptr(), None, d_pi.data_ptr(), o_p.data_ptr(), s)
            g5.plan_tune_indexed(pl_c, d_i.data_ptr(), d_c.data_ptr(), d_q.data_ptr(), d_ci.data_ptr(), o_c.data_ptr(),
                                 s)
        g5.plan_launch_indexed(pl_p, d_i.data_ptr(), d_p.data_ptr(), None, d_pi.data_ptr(), o_p.data_ptr(), s)
        g5.plan_launch_indexed(pl_c, d_i.data_ptr(), d_c.data_ptr(), d_q.data_ptr(), d_ci.data_ptr(), o_c.data_ptr(), s)
        torch.cuda.synchronize()
        op, oc = o_p.cpu().numpy(), o_c.cpu().numpy()
    finally:
        g5.plan_destroy(pl_p)
        g5.plan_destroy(pl_c)
    # acc = monopole + quadrupole parts; phi = -sum m/r - sum(phi_p + phi_q)
    return op[:, :3] + oc[:, :3], op[:, 3] - oc[:, 3]


def fp64_lists(bh, groups):
    """FP64 on the same lists and the same float32 inputs, for the given groups."""
    ip, pp, cp, cq = (a.astype(np.float64) for a in bh.records())
    acc, phi, idx = [], [], []
    for g in groups:
        s = slice(bh.gfirst[g], bh.gfirst[g] + bh.gcount[g])
        pl = bh.pidx[bh.poff[g]:bh.poff[g + 1]]
        cl = bh.cidx[bh.coff[g]:bh.coff[g + 1]]
        a1, p1 = O.g5_newton(ip[s, :3], ip[s, 3], pp[pl, :3], pp[pl, 3])
        a2, p2 = O.g5_quad(ip[s, :3], ip[s, 3], cp[cl, :3], cp[cl, 3], cq[cl, :6])
        acc.append(a1 + a2)
        phi.append(-p1 - p2)
        idx.append(np.arange(s.start, s.stop))
    return np.concatenate(acc), np.concatenate(phi), np.concatenate(idx)


def test_batched_index_lists_vs_fp64_same_lists(g5, bh):
    acc, phi = batched(g5, bh)
    groups = range(0, bh.ngroups, 3)
    ra, rp, idx = fp64_lists(bh, groups)
    assert rms(rel(acc[idx], ra)) <= 1e-6, rms(rel(acc[idx], ra))
    assert rms((phi[idx] - rp) / rp) <= 1e-6


def test_every_configuration_gives_the_same_forces(g5, bh):
    ref_a, ref_p = batched(g5, bh)
    for cp_, cc_ in ((0, 0), (1, 1), (2, 2), (3, 4), (4, 5), (5, 6), (6, 7), (7, 1), (8, 8), (7, 8), (8, 7), (10, 10), (9, 8)):
        a, p = batched(g5, bh, cfg_p=cp_, cfg_c=cc_)
        assert rms(rel(a, ref_a)) <= 1e-6 and rms((p - ref_p) / ref_p) <= 1e-6, (cp_, cc_)
    a, p = batched(g5, bh, tune=True)
    assert rms(rel(a, ref_a)) <= 1e-6


def test_dropin_group_calls_match_batched(g5, bh):
    acc_b, phi_b = batched(g5, bh)
    L = C.CDLL(pgb.ffi.lib_path("libpgbdrv.so"), mode=os.RTLD_LOCAL)
    vp, dp, ip_, lp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_longlong)
    L.g5drv_open.argtypes = [C.c_char_p]
    L.g5drv_open.restype = vp
    L.g5drv_bh.argtypes = [vp, C.c_int, C.c_int, ip_, ip_, dp, dp, dp, lp, ip_, dp, dp, dp, lp, ip_, C.c_double, dp, dp,
                           C.c_int]
    L.g5drv_bh.restype = C.c_double
    h = L.g5drv_open(pgb.ffi.lib_path("libpg5.so").encode())
    assert h
    ip, pp, cp, cq = (a.astype(np.float64) for a in bh.records())
    xi = np.ascontiguousarray(ip[:, :3])
    xp = np.ascontiguousarray(pp[:, :3])
    mp = np.ascontiguousarray(pp[:, 3])
    cpos = np.ascontiguousarray(cp[:, :3])
    cm = np.ascontiguousarray(cp[:, 3])
    cqq = np.ascontiguousarray(cq[:, :6])
    acc = np.zeros((len(mp), 3))
    phi = np.zeros(len(mp))
    P = lambda a, t=dp: a.ctypes.data_as(t)  # noqa: E731
    sec = L.g5drv_bh(h, 0, bh.ngroups, P(bh.gfirst, ip_), P(bh.gcount, ip_), P(xi), P(xp), P(mp), P(bh.poff, lp),
                     P(bh.pidx, ip_), P(cpos), P(cm), P(cqq), P(bh.coff, lp), P(bh.cidx, ip_), bh.eps, P(acc), P(phi),
                     4)
    assert sec > 0
    assert rms(rel(acc, acc_b)) <= 1e-6
    assert rms((phi - phi_b) / phi_b) <= 1e-6


def test_multipole_error_vs_direct_sum(g5, bh):
    acc, phi = batched(g5, bh)
    sample = np.sort(W.Rng(77).permutation(len(bh.m))[:512])
    eps2 = bh.eps * bh.eps
    ad, pd = O.g5_newton(bh.x[sample], eps2, bh.x, bh.m)
    err = rel(acc[sample], ad)
    assert rms(err) <= 2e-3, rms(err)


def _launch(g5, bh, pl_p, pl_c):
    import torch
    dev = torch.device("cuda")
    ip, pp, cp, cq = bh.records()
    d = [torch.from_numpy(a).to(dev) for a in (ip, pp, cp, cq, bh.pidx, bh.cidx)]
    o_p = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    o_c = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    g5.plan_launch_indexed(pl_p, d[0].data_ptr(), d[1].data_ptr(), None, d[4].data_ptr(), o_p.data_ptr(), s)
    g5.plan_launch_indexed(pl_c, d[0].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), d[5].data_ptr(), o_c.data_ptr(), s)
    torch.cuda.synchronize()
    op, oc = o_p.cpu().numpy(), o_c.cpu().numpy()
    return op[:, :3] + oc[:, :3], op[:, 3] - oc[:, 3]


@pytest.mark.parametrize("cfg", [7, 1])
def test_plan_update_matches_fresh_plans(g5, cfg):
    """pgb5_plan_update on the lists of other trees (more groups, then fewer) gives the results
    of plans created for them with the same configuration, bit for bit."""
    sets = [W.bh_hernquist(1 << 14, seed=W.SEED0 + 61), W.bh_hernquist(1 << 16, seed=W.SEED0 + 62),
            W.bh_hernquist(3000, seed=W.SEED0 + 63)]
    pl_p = pl_c = None
    try:
        for k, bh in enumerate(sets):
            if pl_p is None:
                pl_p, pl_c = g5.plan_create(g5.NEWTON, bh.items("p")), g5.plan_create(g5.QUAD, bh.items("c"))
                assert g5.L.pgb5_plan_set_config(pl_p, cfg) == 0 and g5.L.pgb5_plan_set_config(pl_c, cfg) == 0
            else:
                g5.plan_update(pl_p, bh.items("p"))
                g5.plan_update(pl_c, bh.items("c"))
            assert g5.L.pgb5_plan_config(pl_p) == cfg and g5.L.pgb5_plan_config(pl_c) == cfg
            assert g5.L.pgb5_plan_interactions(pl_c) == int(np.sum(np.diff(bh.coff) * bh.gcount))
            a, p = _launch(g5, bh, pl_p, pl_c)
            a0, p0 = batched(g5, bh, cfg_p=cfg, cfg_c=cfg)
            np.testing.assert_array_equal(a, a0, err_msg=f"set {k}")
            np.testing.assert_array_equal(p, p0, err_msg=f"set {k}")
    finally:
        if pl_p is not None:
            g5.plan_destroy(pl_p)
            g5.plan_destroy(pl_c)


def test_graph_captured_plans_replay_and_update(g5):
    """Both launches captured in a CUDA graph replay the stream launches' results bit for bit;
    after the replays have finished the same plans take another tree's lists."""
    import torch
    dev = torch.device("cuda")
    bh, bh2 = W.bh_hernquist(1 << 14, seed=W.SEED0 + 71), W.bh_hernquist(1 << 15, seed=W.SEED0 + 72)
    ip, pp, cp, cq = bh.records()
    d = [torch.from_numpy(a).to(dev) for a in (ip, pp, cp, cq, bh.pidx, bh.cidx)]
    o_p = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    o_c = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    pl_p, pl_c = g5.plan_create(g5.NEWTON, bh.items("p")), g5.plan_create(g5.QUAD, bh.items("c"))
    try:
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            g5.plan_launch_indexed(pl_p, d[0].data_ptr(), d[1].data_ptr(), None, d[4].data_ptr(), o_p.data_ptr(),
                                   s.cuda_stream)
            g5.plan_launch_indexed(pl_c, d[0].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), d[5].data_ptr(),
                                   o_c.data_ptr(), s.cuda_stream)
        s.synchronize()
        ref_p, ref_c = o_p.clone(), o_c.clone()
        o_p.zero_()
        o_c.zero_()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            g5.plan_launch_indexed(pl_p, d[0].data_ptr(), d[1].data_ptr(), None, d[4].data_ptr(), o_p.data_ptr(),
                                   s.cuda_stream)
            g5.plan_launch_indexed(pl_c, d[0].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), d[5].data_ptr(),
                                   o_c.data_ptr(), s.cuda_stream)
        for _ in range(3):
            graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(o_p, ref_p) and torch.equal(o_c, ref_c)
        del graph
        g5.plan_update(pl_p, bh2.items("p"))
        g5.plan_update(pl_c, bh2.items("c"))
        a, p = _launch(g5, bh2, pl_p, pl_c)
        cfg_p, cfg_c = g5.L.pgb5_plan_config(pl_p), g5.L.pgb5_plan_config(pl_c)
        a0, p0 = batched(g5, bh2, cfg_p=cfg_p, cfg_c=cfg_c)
        np.testing.assert_array_equal(a, a0)
        np.testing.assert_array_equal(p, p0)
    finally:
        g5.plan_destroy(pl_p)
        g5.plan_destroy(pl_c)


@pytest.mark.parametrize("cfg", [7, 8])
def test_64_thread_configurations_vs_fp64_same_lists(g5, bh, cfg):
    """The 64-thread CTAs of both kinds -- 7: one, two or three i per thread by the task's size
    (j-lanes for tasks of <= 32 i, 3 i x 4 lanes for 33..48, 2 i x 2 lanes above), 8: the
    j-paired form -- on the tree's lists against FP64 on the same lists, every group (ragged
    tiles and every task layout occur)."""
    acc, phi = batched(g5, bh, cfg_p=cfg, cfg_c=cfg)
    ra, rp, idx = fp64_lists(bh, range(bh.ngroups))
    assert rms(rel(acc[idx], ra)) <= 1e-6, rms(rel(acc[idx], ra))
    assert rms((phi[idx] - rp) / rp) <= 1e-6
    sizes = np.asarray(bh.gcount) % 64
    assert np.any((sizes > 32) & (sizes <= 48)) and np.any((sizes > 0) & (sizes <= 32)) and np.any(sizes > 48)
