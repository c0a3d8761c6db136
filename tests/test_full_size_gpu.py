"""GPU parity at the benchmark configurations' full sizes.

Each test builds the configuration's seeded synthetic input at its full size, runs the batched
launch (the path the benchmark times) over all of it, and checks a sample against the FP64
oracle on the same inputs; a smaller sample is also checked against the reference's own AVX2
library where it was compiled here (oracle/_ref).  Tolerances, as in the smaller tests:

* vs FP64: rms relative acc (and jerk, potential) error <= 1e-6; Hermite nearest neighbour
  identical wherever the FP64 first and second neighbours differ by more than 1e-5 (relative,
  in r^2);
* vs the reference's AVX2 result (12-bit rsqrt + one Newton step): PG6 acc <= 5e-6, jerk <= 1e-4,
  pot <= 2e-7 relative (max; 5e-7 on C5's smallest, 256-body cluster, where single particles'
  128-term FP32 block sums reach a few 1e-7); PG5 table acc <= 1e-4 (max); quadrupole tree code
  rms 1e-3;
* Barnes-Hut against the full FP64 direct sum (multipole truncation at theta = 0.5) on 4096
  sampled particles: rms <= 2e-3 (reported by the benchmark, checked here against gross errors).

C2: PG6 Hermite N = 65536, the schedule's largest call (all 65536 active against all j).
C3: PG5 table, N = 2^20 uniform periodic box, 128^3 cell mesh, 1024-entry Gaussian-split table.
C4: Barnes-Hut with quadrupole cells, N = 2^22 Hernquist sphere, theta 0.5, groups <= 256.
C5: 1024 independent Plummer clusters, N log-uniform in [256, 16384].
"""
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


def f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


@pytest.fixture(scope="module")
def torch_dev():
    if not gpu_available():
        pytest.skip("no GPU")
    import torch
    return torch, torch.device("cuda")


def _g6_rows(out):
    acc = np.stack([out["ax"], out["ay"], out["az"]], 1)
    jrk = np.stack([out["jx"], out["jy"], out["jz"]], 1)
    return acc, jrk, out["pot"]


def test_c2_hermite_65536_largest_call(torch_dev):
    torch, dev = torch_dev
    g6 = pgb.ffi.G6()
    g6.L.g6_open(0)

    def gpu_force(x, v, m, eps2):
        idx = np.arange(len(x), dtype=np.int32)
        r = g6.batch_host([[0, len(x), 0, len(x)]], x, v, idx, x, v, m, idx, eps2, nn=False)
        return r["acc"], r["jrk"]

    n = 65536
    st = W.hermite_state(n, seed=W.SEED0 + 1, force_fn=gpu_force)
    ti = st.t_now + 15 * 2.0 ** -20
    xp, vp = O.g6_predict(ti, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    ptcl = np.zeros(n, pgb.ffi.G6PTCL)
    ptcl["pos"], ptcl["vel"], ptcl["acc2"], ptcl["jrk6"] = st.pos, st.vel, st.acc2, st.jrk6
    ptcl["mass"], ptcl["tim"], ptcl["idx"] = st.mass, st.tj, st.idx
    d_ptcl = torch.from_numpy(ptcl.view(np.uint8)).to(dev)
    d_pred = torch.zeros(n * pgb.ffi.G6PREDJ.itemsize, dtype=torch.uint8, device=dev)
    d_i = torch.from_numpy(pgb.ffi.g6_irecords(xp, vp, st.idx).view(np.uint8)).to(dev)
    d_o = torch.zeros(n * pgb.ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    assert g6.L.pgb6_predict(d_ptcl.data_ptr(), n, ti, d_pred.data_ptr(), 0, s) == 0
    plan = g6.plan_create([[0, n, 0, n]], nn=True)
    try:
        g6.plan_tune(plan, d_i.data_ptr(), d_pred.data_ptr(), st.eps2, d_o.data_ptr(), s)
        d_o.zero_()
        g6.plan_launch(plan, d_i.data_ptr(), d_pred.data_ptr(), st.eps2, d_o.data_ptr(), s)
        torch.cuda.synchronize()
    finally:
        g6.plan_destroy(plan)
    out = d_o.cpu().numpy().view(pgb.ffi.G6OUT)
    sel = np.arange(0, n, 64)
    ref = O.g6_force(xp[sel], f32(vp[sel]), st.idx[sel], np.float32(st.eps2), xp, f32(vp), f32(st.mass), st.idx)
    acc, jrk, pot = _g6_rows(out[sel])
    assert rms(rel(acc, ref["acc"])) <= 1e-6
    assert rms(rel(jrk, ref["jrk"])) <= 1e-6
    assert rms((pot - ref["pot"]) / np.abs(ref["pot"])) <= 1e-6
    clear = ref["r2nn2"] / ref["r2nn"] - 1.0 > 1e-5
    assert np.array_equal(st.idx[out["jadr"][sel]][clear], ref["nnb"][clear])
    np.testing.assert_allclose(-2.0 / out["key"][sel], ref["rnnb"], rtol=1e-6)
    if O.ref_available("libpg6_ref.so"):
        from oracle import refapi
        R = refapi.RefG6()
        R.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
        few = sel[::8]
        r = R.calc(ti, n, xp[few], vp[few], st.idx[few], st.eps2, variant="2p")
        a2, j2, p2 = _g6_rows(out[few])
        assert rel(a2, r["acc"]).max() <= 5e-6
        assert rel(j2, r["jrk"]).max() <= 1e-4
        assert (np.abs(p2 - r["pot"]) / np.abs(r["pot"])).max() <= 2e-7


def test_c3_treepm_2e20_groups(torch_dev):
    torch, dev = torch_dev
    tab = pgb.ffi.G5Table()
    ts = W.treepm_groups(seed=W.SEED0 + 2)
    assert len(ts.xi) == 1 << 20
    f = W.gaussian_split_force(ts.rs, ts.rcut, ts.eps)
    try:
        tab.set_table(f, ts.rcut, frc_bit=6)
        t, xs = tab.table()
        ip = np.zeros((len(ts.xi), 4), np.float32)
        ip[:, :3] = (ts.xi.astype(np.float32).astype(np.float64) * xs).astype(np.float32)
        jp = np.zeros((len(ts.xj), 4), np.float32)
        jp[:, :3] = ts.xj.astype(np.float32) * np.float32(xs)
        jp[:, 3] = ts.mj
        d_i, d_j = torch.from_numpy(ip).to(dev), torch.from_numpy(jp).to(dev)
        d_o = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
        plan = tab.plan_create(ts.items)
        try:
            tab.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), d_o.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
        finally:
            tab.plan_destroy(plan)
        out = d_o.cpu().numpy()
        errs = []
        for k in range(0, len(ts.items), 64):
            i0, ni, j0, nj = (int(v) for v in ts.items[k])
            ao = O.g5_table(ip[i0:i0 + ni, :3].astype(np.float64) / xs, jp[j0:j0 + nj, :3].astype(np.float64) / xs,
                            ts.mj[j0:j0 + nj], t, 4, 6, xs)
            errs.append(rel(out[i0:i0 + ni, :3], ao))
        assert rms(np.concatenate(errs)) <= 1e-6
        if O.ref_available("libpg5table_ref.so"):
            # the reference's table is 512 entries (fixed at its compile time): the same force
            # shape in a 512-entry table on both sides, a few groups through the plain API
            from oracle import refapi
            R = refapi.RefG5Table()
            R.set_table(f, ts.rcut)
            tab.set_table(f, ts.rcut, frc_bit=5)
            for k in (0, len(ts.items) // 2, len(ts.items) - 1):
                i0, ni, j0, nj = (int(v) for v in ts.items[k])
                a, _ = tab.force(ts.xj[j0:j0 + nj], ts.mj[j0:j0 + nj], ts.xi[i0:i0 + ni])
                ar, _ = R.force(ts.xj[j0:j0 + nj], ts.mj[j0:j0 + nj], ts.xi[i0:i0 + ni])
                assert rel(a, ar).max() <= 1e-4
    finally:
        tab.L.pg5_set_table_bits(4, 5)


def test_c4_barnes_hut_2e22(torch_dev):
    torch, dev = torch_dev
    g5 = pgb.ffi.G5()
    g5.L.g5_open()
    bh = W.bh_hernquist(1 << 22, seed=W.SEED0 + 3)
    ip, pp, cp, cq = bh.records()
    d = [torch.from_numpy(a).to(dev) for a in (ip, pp, cp, cq, bh.pidx, bh.cidx)]
    o_p = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    o_c = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    pl_p, pl_c = g5.plan_create(g5.NEWTON, bh.items("p")), g5.plan_create(g5.QUAD, bh.items("c"))
    try:
        g5.plan_launch_indexed(pl_p, d[0].data_ptr(), d[1].data_ptr(), None, d[4].data_ptr(), o_p.data_ptr(), s)
        g5.plan_launch_indexed(pl_c, d[0].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), d[5].data_ptr(),
                               o_c.data_ptr(), s)
        torch.cuda.synchronize()
    finally:
        g5.plan_destroy(pl_p)
        g5.plan_destroy(pl_c)
    op, oc = o_p.cpu().numpy(), o_c.cpu().numpy()
    acc, phi = op[:, :3] + oc[:, :3], op[:, 3] - oc[:, 3]
    del d, o_p, o_c
    ip64, pp64, cp64, cq64 = (a.astype(np.float64) for a in (ip, pp, cp, cq))
    ea, ep = [], []
    for g in range(0, bh.ngroups, 97):
        sl = slice(bh.gfirst[g], bh.gfirst[g] + bh.gcount[g])
        pl = bh.pidx[bh.poff[g]:bh.poff[g + 1]]
        cl = bh.cidx[bh.coff[g]:bh.coff[g + 1]]
        a1, p1 = O.g5_newton(ip64[sl, :3], ip64[sl, 3], pp64[pl, :3], pp64[pl, 3])
        a2, p2 = O.g5_quad(ip64[sl, :3], ip64[sl, 3], cp64[cl, :3], cp64[cl, 3], cq64[cl, :6])
        ea.append(rel(acc[sl], a1 + a2))
        ep.append((phi[sl] + p1 + p2) / (p1 + p2))
    assert rms(np.concatenate(ea)) <= 1e-6
    assert rms(np.concatenate(ep)) <= 1e-6
    smp = np.sort(W.Rng(4096).permutation(len(bh.m))[:4096])
    ad, _ = O.g5_newton(ip64[smp, :3], float(ip64[0, 3]), pp64[:, :3], pp64[:, 3])
    assert rms(rel(acc[smp], ad)) <= 2e-3
    if O.ref_available("libquad_ref.so"):
        from oracle import refapi
        R = refapi.RefQuad()
        ra, rq = [], []
        for g in (0, bh.ngroups // 3, bh.ngroups - 1):
            sl = slice(bh.gfirst[g], bh.gfirst[g] + bh.gcount[g])
            pl = bh.pidx[bh.poff[g]:bh.poff[g + 1]]
            cl = bh.cidx[bh.coff[g]:bh.coff[g + 1]]
            am, _, aq, _ = R.force(bh.eps, ip64[sl, :3], pp64[pl, :3], pp64[pl, 3], cp64[cl, :3], cp64[cl, 3],
                                   cq64[cl, :6])
            ra.append(rel(acc[sl], am + aq))
        assert rms(np.concatenate(ra)) <= 1e-3


def test_c5_1024_clusters(torch_dev):
    torch, dev = torch_dev
    g6 = pgb.ffi.G6()
    g6.L.g6_open(0)
    cs = W.cluster_set(seed=W.SEED0 + 4)
    assert len(cs.sizes) == 1024
    n = len(cs.mass)
    idx = np.arange(n, dtype=np.int32)
    d_i = torch.from_numpy(pgb.ffi.g6_irecords(cs.pos, cs.vel, idx).view(np.uint8)).to(dev)
    d_j = torch.from_numpy(pgb.ffi.g6_jrecords(cs.pos, cs.vel, cs.mass, idx).view(np.uint8)).to(dev)
    d_o = torch.zeros(n * pgb.ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
    items = np.stack([cs.offsets[:-1], cs.sizes, cs.offsets[:-1], cs.sizes], 1)
    plan = g6.plan_create(items, nn=True)
    try:
        s = torch.cuda.current_stream().cuda_stream
        g6.plan_tune(plan, d_i.data_ptr(), d_j.data_ptr(), cs.eps2, d_o.data_ptr(), s)
        d_o.zero_()
        g6.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), cs.eps2, d_o.data_ptr(), s)
        torch.cuda.synchronize()
    finally:
        g6.plan_destroy(plan)
    out = d_o.cpu().numpy().view(pgb.ffi.G6OUT)
    ea, ej, ep = [], [], []
    for k in range(0, 1024, 64):
        sl = slice(int(cs.offsets[k]), int(cs.offsets[k + 1]))
        ref = O.g6_force(cs.pos[sl], f32(cs.vel[sl]), idx[sl], np.float32(cs.eps2), cs.pos[sl], f32(cs.vel[sl]),
                         f32(cs.mass[sl]), idx[sl])
        acc, jrk, pot = _g6_rows(out[sl])
        ea.append(rel(acc, ref["acc"]))
        ej.append(rel(jrk, ref["jrk"]))
        ep.append((pot - ref["pot"]) / np.abs(ref["pot"]))
        clear = ref["r2nn2"] / ref["r2nn"] - 1.0 > 1e-5
        assert np.array_equal(idx[out["jadr"][sl]][clear], ref["nnb"][clear]), k
    assert rms(np.concatenate(ea)) <= 1e-6
    assert rms(np.concatenate(ej)) <= 1e-6
    assert rms(np.concatenate(ep)) <= 1e-6
    if O.ref_available("libpg6_ref.so"):
        from oracle import refapi
        k = int(np.argmin(cs.sizes))
        sl = slice(int(cs.offsets[k]), int(cs.offsets[k + 1]))
        nk = int(cs.sizes[k])
        R = refapi.RefG6()
        z = np.zeros((nk, 3))
        R.set_j(cs.pos[sl], cs.vel[sl], z, z, cs.mass[sl], np.zeros(nk), np.arange(nk, dtype=np.int32))
        r = R.calc(0.0, nk, cs.pos[sl], cs.vel[sl], np.arange(nk, dtype=np.int32), cs.eps2, variant="2p")
        acc, jrk, pot = _g6_rows(out[sl])
        assert rel(acc, r["acc"]).max() <= 5e-6
        assert rel(jrk, r["jrk"]).max() <= 1e-4
        # the reference returns the potential as float (FP64 sums of 12-bit rsqrt + Newton terms);
        # ours sums 128-term FP32 blocks into FP64: a few 1e-7 on single particles of a 256-body
        # cluster (rms against FP64 3e-8, checked above)
        assert (np.abs(pot - r["pot"]) / np.abs(r["pot"])).max() <= 5e-7
