"""GPU parity of the Barnes-Hut tree builder (lib/libpgbtree.so, pgbt_*) with the host builder.

The host builder (drivers/pgb_bhtree.c) follows the reference tree code's rules
(PG5/newton_quad/source.cpp) and is itself checked by tests/test_bhtree.py.  The device build
must give the same tree bit for bit: particle order, every node's range, centre, half side and
children (pre-order numbering), the FP64 moments, the groups and every group's point-mass and
cell list.  Cases: Hernquist spheres (the benchmark's distribution) of 2^12, 2^16 and 2^20
particles with different leaf / group sizes and opening angles, a uniform cube, and sets with
coincident particles (the 40-level depth cap) and a single particle.
"""
import numpy as np
import pytest

from conftest import gpu_available, pgb

pytestmark = pytest.mark.gpu
W = pgb.workloads

FIELDS = ("perm", "x", "m", "nfirst", "ncount", "nhalf", "ncentre", "nchild", "ccom", "cmass", "cquad", "gfirst",
          "gcount", "gcentre", "ghalf", "poff", "pidx", "coff", "cidx")


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if not gpu_available():
        pytest.skip("no GPU")


def hernquist(n, seed):
    rng = W.Rng(seed)
    x = W._isotropic(rng, W.hernquist_radii(rng, n, 100.0)).astype(np.float32).astype(np.float64)
    return x, np.full(n, np.float32(1.0 / n), np.float64)


def check_same(x, m, theta, nleaf, ncrit):
    host = W.bh_tree(x, m, theta, nleaf, ncrit)
    t = W.GpuTree(x, m, theta, nleaf, ncrit)
    try:
        dev = t.set()
    finally:
        t.close()
    for f in FIELDS:
        a, b = getattr(dev, f), getattr(host, f)
        assert a.shape == b.shape, (f, a.shape, b.shape)
        if not np.array_equal(a, b):
            bad = np.nonzero((a != b).reshape(len(a), -1).any(axis=1))[0]
            raise AssertionError(f"{f}: {len(bad)} rows differ, first {bad[:5]}")
    return host


@pytest.mark.parametrize("n,theta,nleaf,ncrit", [(1 << 12, 0.5, 8, 64), (1 << 16, 0.6, 16, 256),
                                                 (1 << 20, 0.5, 16, 256)])
def test_hernquist_trees_match_the_host_builder(n, theta, nleaf, ncrit):
    x, m = hernquist(n, W.SEED0 + 3)
    host = check_same(x, m, theta, nleaf, ncrit)
    assert len(host.gfirst) > 1 and len(host.cidx) > 0


def test_uniform_cube_and_unequal_masses():
    rng = W.Rng(W.SEED0 + 41)
    x = (rng.uniform(3 * 20000).reshape(-1, 3) * 2.0 - 1.0) * 3.7
    m = rng.uniform(20000) + 0.5
    check_same(x, m, 0.7, 4, 32)


def test_coincident_particles_hit_the_depth_cap():
    rng = W.Rng(W.SEED0 + 42)
    x = rng.uniform(3 * 3000).reshape(-1, 3) - 0.5
    x[100:160] = [0.123, -0.25, 0.0625]      # 60 particles at one point: a 40-level chain
    x[2000:2005] = x[7]
    m = np.full(len(x), 1.0 / len(x))
    host = check_same(x, m, 0.5, 16, 128)
    assert host.ncount.max() > 16 and (host.nchild < 0).all(axis=1).any()


def test_single_particle_and_tiny_sets():
    check_same(np.array([[0.3, -0.2, 0.1]]), np.array([1.0]), 0.5, 16, 256)
    rng = W.Rng(W.SEED0 + 43)
    check_same(rng.uniform(3 * 17).reshape(-1, 3), np.full(17, 1.0 / 17), 0.5, 16, 256)


def test_device_records_follow_the_tree():
    x, m = hernquist(1 << 14, W.SEED0 + 5)
    t = W.GpuTree(x, m, 0.5, 16, 256)
    try:
        s = t.set()
        p, c, q = t.records()
        d = t.device()
        assert all(v for v in d.values())
        assert t.build_ms > 0
        items_p, items_c = t.items()
        np.testing.assert_array_equal(items_p, s.items("p"))
        np.testing.assert_array_equal(items_c, s.items("c"))
        import torch
        irec = torch.empty((len(m), 4), dtype=torch.float32, device="cuda")
        t.irecords(1e-6, irec.data_ptr())
        ir = irec.cpu().numpy()
        np.testing.assert_array_equal(ir[:, :3], s.x.astype(np.float32))
        np.testing.assert_array_equal(ir[:, 3], np.float32(1e-6))
    finally:
        t.close()
    np.testing.assert_array_equal(p[:, :3], s.x.astype(np.float32))
    np.testing.assert_array_equal(p[:, 3], s.m.astype(np.float32))
    np.testing.assert_array_equal(c[:, :3], s.ccom.astype(np.float32))
    np.testing.assert_array_equal(c[:, 3], s.cmass.astype(np.float32))
    np.testing.assert_array_equal(q[:, :6], s.cquad.astype(np.float32))
    np.testing.assert_array_equal(q[:, 6:], 0.0)


def test_repeated_builds_release_their_scratch():
    import torch
    x, m = hernquist(1 << 18, W.SEED0 + 6)
    W.GpuTree(x, m, 0.5, 16, 256).close()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        W.GpuTree(x, m, 0.5, 16, 256).close()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < (64 << 20), (free0, free1)


def test_rebuild_reuses_the_tree_object():
    """pgbt_rebuild on other particles (more, then fewer) gives the host builder's tree."""
    t = None
    try:
        for n, seed in ((1 << 14, 7), (1 << 16, 8), (3000, 9)):
            x, m = hernquist(n, W.SEED0 + seed)
            if t is None:
                t = W.GpuTree(x, m, 0.5, 16, 256)
            else:
                t.rebuild(x, m)
            dev, host = t.set(), W.bh_tree(x, m, 0.5, 16, 256)
            for f in FIELDS:
                np.testing.assert_array_equal(getattr(dev, f), getattr(host, f), err_msg=f"{f} (n {n})")
    finally:
        if t is not None:
            t.close()
