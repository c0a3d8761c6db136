"""GPU parity of the GRAPE-6 Hermite path (lib/libpg6.so).

Reference for every case: the FP64 oracle (FP64 predictor + FP64 force/jerk/pot/NN,
oracle/pg_oracle.c) on the same j-memory; where the reference library was compiled here
(oracle/_ref/libpg6_ref.so), also the reference's own AVX2 result through the same API calls.
Tolerances:
  * vs FP64: rms relative |da|/|a| <= 1e-6, |dj|/|j| <= 1e-6 (rms), pot <= 1e-6 (rms)
  * vs reference AVX2: acc <= 5e-6, jerk <= 1e-4, pot <= 2e-7 relative (max over particles),
    the reference's own FP64 error being rms 6.8e-8 / 1.8e-6 / 3.3e-8
  * nearest neighbour: index identical wherever the FP64 first and second softened r^2
    differ by more than 1e-5 relative; rnnb (softened r) within 1e-6 relative.
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


def fp64_force(x, v, m, eps2):
    idx = np.arange(len(x), dtype=np.int32)
    r = O.g6_force(x, v, idx, eps2, x, v, m, idx)
    return r["acc"], r["jrk"]


# the default build (q = -2/r from the MUFU rsqrt alone) and the reference's rsqrt form (one
# Newton step): every case holds for both
@pytest.fixture(scope="module", params=["libpg6.so", "libpg6_newton.so"])
def g6(request):
    if not gpu_available():
        pytest.skip("no GPU")
    lib = pgb.ffi.G6(request.param)
    lib.L.g6_open(0)
    return lib


@pytest.fixture(scope="module")
def state():
    return W.hermite_state(8192, seed=W.SEED0 + 1, force_fn=fp64_force)


def oracle_call(st, active, ti, h2=None, maxlen=1024):
    xp, vp = O.g6_predict(ti, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    # the GRAPE-6 path carries predicted velocities and masses as float (gravity.c:43-47)
    vpf = vp.astype(np.float32).astype(np.float64)
    mf = st.mass.astype(np.float32).astype(np.float64)
    return O.g6_force(xp[active], vpf[active], st.idx[active], np.float32(st.eps2), xp, vpf, mf, st.idx,
                      h2=h2, maxlen=maxlen), xp, vp


def check_nn(res, ref):
    sep = ref["r2nn2"] / ref["r2nn"] - 1.0
    clear = sep > 1e-5
    assert np.array_equal(res["nnb"][clear], ref["nnb"][clear])
    np.testing.assert_allclose(res["rnnb"], ref["rnnb"], rtol=1e-6)


def test_hermite_api_vs_fp64(g6, state):
    st = state
    g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    active = np.sort(W.Rng(5).permutation(len(st.mass))[:1000]).astype(np.int32)
    ref, xp, vp = oracle_call(st, active, st.t_now)
    res = g6.calc(st.t_now, len(st.mass), xp[active], vp[active], st.idx[active], st.eps2, variant="2p")
    ea, ej = rel(res["acc"], ref["acc"]), rel(res["jrk"], ref["jrk"])
    ep = np.abs(res["pot"] - ref["pot"]) / np.abs(ref["pot"])
    assert rms(ea) <= 1e-6, (rms(ea), ea.max())
    assert rms(ej) <= 1e-6, (rms(ej), ej.max())
    assert rms(ep) <= 1e-6
    check_nn(res, ref)


def test_hermite_plain_and_nnb_variants_agree(g6, state):
    st = state
    g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    active = np.arange(0, 300, dtype=np.int32)
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    a = g6.calc(st.t_now, len(st.mass), xp[active], vp[active], active, st.eps2, variant="plain")
    b = g6.calc(st.t_now, len(st.mass), xp[active], vp[active], active, st.eps2, variant="2")
    c = g6.calc(st.t_now, len(st.mass), xp[active], vp[active], active, st.eps2, variant="2p")
    for k in ("acc", "jrk", "pot"):
        np.testing.assert_array_equal(a[k], b[k])
        np.testing.assert_array_equal(a[k], c[k])
    np.testing.assert_array_equal(b["nnb"], c["nnb"])


@pytest.mark.skipif(not O.ref_available("libpg6_ref.so"), reason="reference not built")
def test_hermite_vs_reference_avx2(g6):
    from oracle import refapi
    st = W.hermite_state(4096, seed=W.SEED0 + 7, force_fn=fp64_force)
    active = np.sort(W.Rng(8).permutation(4096)[:600]).astype(np.int32)
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    res = g6.calc(st.t_now, 4096, xp[active], vp[active], active, st.eps2, variant="2p")
    R = refapi.RefG6()
    R.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    ref = R.calc(st.t_now, 4096, xp[active], vp[active], active, st.eps2, variant="2p")
    assert rel(res["acc"], ref["acc"]).max() <= 5e-6
    assert rel(res["jrk"], ref["jrk"]).max() <= 1e-4
    assert (np.abs(res["pot"] - ref["pot"]) / np.abs(ref["pot"])).max() <= 2e-7
    fp, _, _ = oracle_call(st, active, st.t_now)
    clear = fp["r2nn2"] / fp["r2nn"] - 1.0 > 1e-5
    assert np.array_equal(res["nnb"][clear], ref["nnb"][clear])
    np.testing.assert_allclose(res["rnnb"], ref["rnnb"], rtol=1e-6)


@pytest.mark.parametrize("ni,nj", [(1, 1), (5, 100), (16, 300), (17, 700), (31, 1500), (32, 8192), (33, 999),
                                   (47, 4097), (48, 8192), (48, 129)])
def test_small_call_shapes_vs_fp64(g6, state, ni, nj):
    """One g6calc_lasthalf2p call of ni <= 48 i-particles against the first nj j-particles: the
    small-call kernel's i-slot variants (16/32/48), single-CTA calls (nj < 256) and clusters of
    2, 4 and 8 CTAs (j-chunks of >= 128 j), each against the FP64 oracle."""
    st = state
    g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    active = np.sort(W.Rng(100 + ni).permutation(nj)[:ni]).astype(np.int32)
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    vpf = vp.astype(np.float32).astype(np.float64)
    mf = st.mass.astype(np.float32).astype(np.float64)
    ref = O.g6_force(xp[active], vpf[active], st.idx[active], np.float32(st.eps2), xp[:nj], vpf[:nj], mf[:nj],
                     st.idx[:nj])
    res = g6.calc(st.t_now, nj, xp[active], vp[active], st.idx[active], st.eps2, variant="2p")
    if nj == 1:
        assert np.all(res["acc"] == 0) and np.all(res["pot"] == 0)
        return
    ea, ej = rel(res["acc"], ref["acc"]), rel(res["jrk"], ref["jrk"])
    ep = np.abs(res["pot"] - ref["pot"]) / np.abs(ref["pot"])
    # rms as for the full calls; the max bounds catch a lost or doubled j-chunk (an O(1e-2) error)
    assert ea.max() <= 1e-4 and ej.max() <= 1e-2 and ep.max() <= 1e-4, (ea.max(), ej.max(), ep.max())
    assert rms(ea) <= 1e-6 and rms(ej) <= 1e-5 and rms(ep) <= 1e-6
    check_nn(res, ref)


def test_neighbour_lists_vs_fp64(g6, state):
    st = state
    g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    active = np.sort(W.Rng(15).permutation(len(st.mass))[:200]).astype(np.int32)
    h2 = np.full(len(active), 0.02)   # banana's neighbour radius^2 (hermite.c:372)
    ref, xp, vp = oracle_call(st, active, st.t_now, h2=h2)
    res = g6.calc(st.t_now, len(st.mass), xp[active], vp[active], st.idx[active], st.eps2, h2=h2,
                  variant="2np")
    xr = xp
    for k, i in enumerate(active):
        rc, err, lst = res["nbl"][k]
        n_ref = ref["nbcount"][k]
        assert rc == 0 and err == 0
        ref_list = ref["nblist"][k, :n_ref]
        # j within 1e-5 (relative, in r^2) of the radius may legitimately differ in FP32
        d2 = np.sum((xr - xr[i]) ** 2, axis=1) + st.eps2
        edge = set(np.nonzero(np.abs(d2 / 0.02 - 1.0) < 1e-5)[0].tolist())
        assert set(lst.tolist()) - edge == set(ref_list.tolist()) - edge
        assert list(lst) == sorted(lst)  # j-address order (ids == addresses here)
    check_nn(res, ref)


def test_neighbour_list_overflow_is_reported(g6, state):
    st = state
    g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    active = np.arange(5, dtype=np.int32)
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    res = g6.calc(st.t_now, len(st.mass), xp[active], vp[active], active, st.eps2, h2=np.full(5, 1e4),
                  variant="n", maxlen=1024)
    # every particle is a neighbour of every other: 8191 > 1024 entries
    for k in range(5):
        rc, err, lst = res["nbl"][k]
        assert rc == 1 and err == 1 and lst is None


def test_single_particle_and_self_only(g6):
    """ni = nj = 1: only the self pair exists; reference semantics: zero force, nnb = self."""
    one = np.zeros((1, 3))
    g6.set_j(one + 0.5, one, one, one, np.array([1.0]), np.array([0.0]), np.array([7]))
    res = g6.calc(0.0, 1, one + 0.5, one, np.array([7]), 1e-4, variant="2p")
    assert np.all(res["acc"] == 0) and np.all(res["jrk"] == 0) and res["pot"][0] == 0
    assert res["nnb"][0] == 7


def test_j_updates_between_block_steps(g6, state):
    """Corrector-style updates of a few j between two g6_set_ti calls are seen by the next call."""
    st = state
    g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    active = np.arange(100, 164, dtype=np.int32)
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    g6.calc(st.t_now, len(st.mass), xp[active], vp[active], active, st.eps2)
    pos2 = st.pos.copy()
    pos2[active] += 1e-3
    tj2 = st.tj.copy()
    tj2[active] = st.t_now
    g6.set_j(pos2[active], st.vel[active], st.acc2[active], st.jrk6[active], st.mass[active], tj2[active],
             st.idx[active], addr=active)
    t2 = st.t_now + 1.0 / 256
    st2 = W.HermiteState(pos=pos2, vel=st.vel, acc2=st.acc2, jrk6=st.jrk6, mass=st.mass, tj=tj2, idx=st.idx,
                         eps2=st.eps2, t_now=t2)
    ref, xq, vq = oracle_call(st2, active, t2)
    res = g6.calc(t2, len(st.mass), xq[active], vq[active], active, st.eps2, variant="2p")
    assert rms(rel(res["acc"], ref["acc"])) <= 1e-6
    assert rms(rel(res["jrk"], ref["jrk"])) <= 1e-6


def test_batched_clusters_vs_fp64(g6):
    cs = W.cluster_set(ncl=12, nmin=64, nmax=3000, seed=99)
    idx = np.arange(len(cs.mass), dtype=np.int32)
    items = np.stack([cs.offsets[:-1], cs.sizes, cs.offsets[:-1], cs.sizes], 1)
    res = g6.batch_host(items, cs.pos, cs.vel, idx, cs.pos, cs.vel, cs.mass, idx, cs.eps2)
    vf = cs.vel.astype(np.float32).astype(np.float64)
    mf = cs.mass.astype(np.float32).astype(np.float64)
    for c in range(len(cs.sizes)):
        s = slice(cs.offsets[c], cs.offsets[c + 1])
        ref = O.g6_force(cs.pos[s], vf[s], idx[s], np.float32(cs.eps2), cs.pos[s], vf[s], mf[s], idx[s])
        assert rms(rel(res["acc"][s], ref["acc"])) <= 1e-6
        assert rms(rel(res["jrk"][s], ref["jrk"])) <= 1e-6
        np.testing.assert_allclose(res["pot"][s], ref["pot"], rtol=1e-5)
        check_nn({"nnb": res["nnb"][s], "rnnb": res["rnnb"][s]}, ref)


@pytest.mark.parametrize("ff", [True, False])
def test_device_plan_graph_capture(g6, ff):
    """The batched plan launches from a captured CUDA graph and replays with identical bits, for
    both position layouts; both layouts agree with the FP64 oracle."""
    import torch
    cs = W.cluster_set(ncl=6, nmin=100, nmax=2000, seed=123)
    n = len(cs.mass)
    idx = np.arange(n, dtype=np.int32)
    irec = pgb.ffi.g6_irecords(cs.pos, cs.vel, idx, ff=ff)
    jrec = pgb.ffi.g6_jrecords(cs.pos, cs.vel, cs.mass, idx, ff=ff)
    dev = torch.device("cuda")
    d_i = torch.from_numpy(irec.view(np.uint8)).to(dev)
    d_j = torch.from_numpy(jrec.view(np.uint8)).to(dev)
    d_o = torch.zeros(n * pgb.ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
    items = np.stack([cs.offsets[:-1], cs.sizes, cs.offsets[:-1], cs.sizes], 1)
    plan = g6.plan_create(items, nn=True, f64=not ff)
    try:
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            g6.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), cs.eps2, d_o.data_ptr(), s.cuda_stream)
        s.synchronize()
        first = d_o.cpu().numpy().view(pgb.ffi.G6OUT).copy()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            g6.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), cs.eps2, d_o.data_ptr(), s.cuda_stream)
        for _ in range(3):
            d_o.zero_()
            graph.replay()
        torch.cuda.synchronize()
        again = d_o.cpu().numpy().view(pgb.ffi.G6OUT)
        assert first.tobytes() == again.tobytes()
        del graph
        vf = cs.vel.astype(np.float32).astype(np.float64)
        mf = cs.mass.astype(np.float32).astype(np.float64)
        for c in range(len(cs.sizes)):
            sl = slice(cs.offsets[c], cs.offsets[c + 1])
            ref = O.g6_force(cs.pos[sl], vf[sl], idx[sl], np.float32(cs.eps2), cs.pos[sl], vf[sl], mf[sl], idx[sl])
            acc = np.stack([first["ax"][sl], first["ay"][sl], first["az"][sl]], 1)
            assert rms(rel(acc, ref["acc"])) <= 1e-6
    finally:
        g6.plan_destroy(plan)


def test_plan_update_matches_fresh_plans(g6):
    """pgb6_plan_update with other cluster sets (more items, then fewer, then one large item)
    gives the results of plans created for them with the same configuration, bit for bit."""
    import torch
    dev = torch.device("cuda")
    sets = [W.cluster_set(ncl=6, nmin=100, nmax=2000, seed=131), W.cluster_set(ncl=20, nmin=64, nmax=3000, seed=132),
            W.cluster_set(ncl=3, nmin=50, nmax=500, seed=133), W.cluster_set(ncl=1, nmin=9000, nmax=9000, seed=134)]
    plan = None
    try:
        for k, cs in enumerate(sets):
            n = len(cs.mass)
            idx = np.arange(n, dtype=np.int32)
            d_i = torch.from_numpy(pgb.ffi.g6_irecords(cs.pos, cs.vel, idx).view(np.uint8)).to(dev)
            d_j = torch.from_numpy(pgb.ffi.g6_jrecords(cs.pos, cs.vel, cs.mass, idx).view(np.uint8)).to(dev)
            items = np.stack([cs.offsets[:-1], cs.sizes, cs.offsets[:-1], cs.sizes], 1)
            if plan is None:
                plan = g6.plan_create(items, nn=True)
            else:
                g6.plan_update(plan, items)
            cfg = g6.L.pgb6_plan_config(plan)
            assert g6.L.pgb6_plan_interactions(plan) == int(np.sum(cs.sizes.astype(np.int64) ** 2))
            out = []
            for p in (plan, None):
                d_o = torch.zeros(n * pgb.ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
                q = p
                if q is None:   # a fresh plan pinned to the same configuration
                    q = g6.plan_create(items, nn=True)
                    assert g6.L.pgb6_plan_set_config(q, cfg) == 0
                g6.plan_launch(q, d_i.data_ptr(), d_j.data_ptr(), cs.eps2, d_o.data_ptr(), 0)
                torch.cuda.synchronize()
                out.append(d_o.cpu().numpy().view(pgb.ffi.G6OUT).copy())
                if p is None:
                    assert g6.L.pgb6_plan_config(q) == cfg
                    g6.plan_destroy(q)
            assert out[0].tobytes() == out[1].tobytes(), f"set {k}"
    finally:
        if plan is not None:
            g6.plan_destroy(plan)


def test_every_configuration_vs_fp64(g6, state):
    """Every kernel configuration of the batched Hermite path (pinned with pgb6_plan_set_config;
    both position layouts, with and without the nearest neighbour) on items that exercise the
    per-tile self test (i-particles inside their own j-range and outside it), ragged j-tiles
    (j counts that are not multiples of 4 or of the tile) and single-j items, against the FP64
    oracle: rms relative acc / pot <= 1e-6 per item, jerk rms <= 1e-6 over the launch's particles
    and <= 2e-5 for every particle (the jerk's two terms cancel: one ill-conditioned particle of
    a 37-particle item carries 5.9e-6 with the MUFU rsqrt alone, 1.4e-6 with the Newton step; the
    reference's own jerk error is rms 1.8e-6), nearest neighbour identical wherever the FP64 first
    and second neighbours are separated."""
    import torch
    st = state
    n = len(st.mass)
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    vpf = vp.astype(np.float32).astype(np.float64)
    mf = st.mass.astype(np.float32).astype(np.float64)
    rng = W.Rng(77)
    act = np.sort(rng.permutation(n)[:3000]).astype(np.int32)
    # (i indices, j range): all j; a ragged j-range; a single j (the i-set excludes it); i
    # outside their j-range; a j-range that holds every i
    cases = [(act, 0, n), (act[:37], 0, 4099), (np.arange(10, 60, dtype=np.int32), 5, 1),
             (np.arange(5000, 5300, dtype=np.int32), 0, 130), (np.arange(200, 457, dtype=np.int32), 190, 1003)]
    ii = np.concatenate([c[0] for c in cases])
    ioff = np.concatenate([[0], np.cumsum([len(c[0]) for c in cases])]).astype(np.int64)
    items = np.array([[ioff[k], len(c[0]), c[1], c[2]] for k, c in enumerate(cases)], np.int32)
    refs = [O.g6_force(xp[c[0]], vpf[c[0]], st.idx[c[0]], np.float32(st.eps2), xp[c[1]:c[1] + c[2]],
                       vpf[c[1]:c[1] + c[2]], mf[c[1]:c[1] + c[2]], st.idx[c[1]:c[1] + c[2]]) for c in cases]
    dev = torch.device("cuda")
    ncfg = 0
    for ff in (True, False):
        d_i = torch.from_numpy(pgb.ffi.g6_irecords(xp[ii], vp[ii], st.idx[ii], ff=ff).view(np.uint8)).to(dev)
        d_j = torch.from_numpy(pgb.ffi.g6_jrecords(xp, vp, st.mass, st.idx, ff=ff).view(np.uint8)).to(dev)
        d_o = torch.zeros(len(ii) * pgb.ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
        for nn in (True, False):
            plan = g6.plan_create(items, nn=nn, f64=not ff)
            try:
                g6.set_abort(False)
                cfg = 0
                while g6.L.pgb6_plan_set_config(plan, cfg) == 0:
                    d_o.fill_(0xFF)
                    g6.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), st.eps2, d_o.data_ptr(), 0)
                    torch.cuda.synchronize()
                    out = d_o.cpu().numpy().view(pgb.ffi.G6OUT)
                    ej_all = []
                    for k, (c, ref) in enumerate(zip(cases, refs)):
                        o = out[ioff[k]:ioff[k + 1]]
                        tag = (ff, nn, cfg, k)
                        acc = np.stack([o["ax"], o["ay"], o["az"]], 1)
                        jrk = np.stack([o["jx"], o["jy"], o["jz"]], 1)
                        assert rms(rel(acc, ref["acc"])) <= 1e-6, tag
                        ej = rel(jrk, ref["jrk"])
                        assert ej.max() <= 2e-5, tag
                        ej_all.append(ej)
                        assert rms((o["pot"] - ref["pot"]) / np.abs(ref["pot"])) <= 1e-6, tag
                        if nn:
                            clear = ref["r2nn2"] / ref["r2nn"] - 1.0 > 1e-5 if c[2] > 1 else np.ones(len(o), bool)
                            jadr = o["jadr"]
                            assert np.all((jadr >= c[1]) & (jadr < c[1] + c[2])), tag
                            assert np.array_equal(st.idx[jadr][clear], ref["nnb"][clear]), tag
                            np.testing.assert_allclose(-2.0 / o["key"], ref["rnnb"], rtol=1e-6, err_msg=str(tag))
                    assert rms(np.concatenate(ej_all)) <= 1e-6, (ff, nn, cfg)
                    cfg += 1
                ncfg = max(ncfg, cfg)
            finally:
                g6.clear_error()
                g6.set_abort(True)
                g6.plan_destroy(plan)
    assert ncfg >= 10


def test_tuned_chunk_count_and_deferred_lookups(g6, state):
    """A one-item plan (the batched path of one block-step call) after pgb6_plan_tune, which picks
    the kernel configuration and, for one item, the j-chunk count: results against the FP64
    oracle (acc / jerk / pot rms relative <= 1e-6; the nearest neighbour's address identical
    wherever the FP64 first and second neighbours are separated, and never a deferred-lookup tile
    mark), the reported chunk and kernel counts (split i-tiles of the tile-minimum configurations
    add the lookup kernel), and a new plan of the same shape taking the tuned configuration and
    chunk count."""
    import torch
    st = state
    n = len(st.mass)
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    vpf = vp.astype(np.float32).astype(np.float64)
    mf = st.mass.astype(np.float32).astype(np.float64)
    act = np.sort(W.Rng(91).permutation(n)[:4096]).astype(np.int32)
    ref = O.g6_force(xp[act], vpf[act], st.idx[act], np.float32(st.eps2), xp, vpf, mf, st.idx)
    dev = torch.device("cuda")
    d_i = torch.from_numpy(pgb.ffi.g6_irecords(xp[act], vp[act], st.idx[act]).view(np.uint8)).to(dev)
    d_j = torch.from_numpy(pgb.ffi.g6_jrecords(xp, vp, st.mass, st.idx).view(np.uint8)).to(dev)
    d_o = torch.zeros(len(act) * pgb.ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
    items = np.array([[0, len(act), 0, n]], np.int32)
    ipt = [1, 1, 2, 1, 4, 2, 2, 2, 4, 2]   # i per thread of each configuration (pgb_g6.cu CFG_IPT)
    plan = g6.plan_create(items, nn=True)
    plan2 = None
    try:
        cfg, ms = g6.plan_tune(plan, d_i.data_ptr(), d_j.data_ptr(), st.eps2, d_o.data_ptr(), 0)
        chunks = g6.L.pgb6_plan_chunks(plan)
        kernels = g6.L.pgb6_plan_kernels(plan)
        assert g6.L.pgb6_plan_config(plan) == cfg and ms > 0
        assert 1 <= chunks <= n // 128
        assert kernels == (2 if chunks > 1 and ipt[cfg] % 2 == 0 else 1), (cfg, chunks, kernels)
        d_o.fill_(0xFF)
        g6.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), st.eps2, d_o.data_ptr(), 0)
        torch.cuda.synchronize()
        o = d_o.cpu().numpy().view(pgb.ffi.G6OUT)
        acc = np.stack([o["ax"], o["ay"], o["az"]], 1)
        jrk = np.stack([o["jx"], o["jy"], o["jz"]], 1)
        assert rms(rel(acc, ref["acc"])) <= 1e-6
        assert rms(rel(jrk, ref["jrk"])) <= 1e-6
        assert rms((o["pot"] - ref["pot"]) / np.abs(ref["pot"])) <= 1e-6
        jadr = o["jadr"]
        assert np.all((jadr >= 0) & (jadr < n))   # resolved addresses: no (1 << 30) tile mark
        clear = ref["r2nn2"] / ref["r2nn"] - 1.0 > 1e-5
        assert np.array_equal(st.idx[jadr][clear], ref["nnb"][clear])
        plan2 = g6.plan_create(items, nn=True)
        assert g6.L.pgb6_plan_config(plan2) == cfg
        assert g6.L.pgb6_plan_chunks(plan2) == chunks
    finally:
        g6.plan_destroy(plan)
        if plan2 is not None:
            g6.plan_destroy(plan2)
