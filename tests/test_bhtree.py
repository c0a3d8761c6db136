"""The Barnes-Hut workload's host tree (phantom-grape_b200/drivers/pgb_bhtree.c), CPU only.

The tree, groups and interaction lists are checked against the rules of the reference's tree
code (PG5/newton_quad/source.cpp): groups tile the particles, every group's list accounts for
each particle exactly once (as itself or inside one cell), the lists are exactly what a plain
restatement of make_interaction_list (source.cpp:581-707) produces from the same tree, and the
cell moments equal their direct FP64 sums.
"""
import numpy as np
import pytest

from conftest import pgb

W = pgb.workloads


@pytest.fixture(scope="module")
def bh():
    return W.bh_hernquist(1 << 12, theta=0.5, nleaf=8, ncrit=64)


def test_tree_order_and_groups_tile_the_particles(bh):
    rng = W.Rng(W.SEED0 + 3)
    x0 = W._isotropic(rng, W.hernquist_radii(rng, 1 << 12)).astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(bh.x, x0[bh.perm])
    assert sorted(bh.perm.tolist()) == list(range(1 << 12))
    # groups: consecutive tree-order ranges covering every particle once, each <= ncrit
    assert bh.gfirst[0] == 0
    np.testing.assert_array_equal(bh.gfirst[1:], bh.gfirst[:-1] + bh.gcount[:-1])
    assert bh.gfirst[-1] + bh.gcount[-1] == len(bh.m)
    assert bh.gcount.max() <= bh.ncrit


def test_every_list_accounts_for_all_the_mass(bh):
    total = bh.m.sum()
    for g in range(bh.ngroups):
        pl = bh.pidx[bh.poff[g]:bh.poff[g + 1]]
        cl = bh.cidx[bh.coff[g]:bh.coff[g + 1]]
        assert len(set(pl.tolist())) == len(pl)
        # particles inside the listed cells and the listed particles: disjoint, all of them
        covered = np.zeros(len(bh.m), np.int32)
        covered[pl] += 1
        for c in cl:
            covered[bh.nfirst[c]:bh.nfirst[c] + bh.ncount[c]] += 1
        assert np.all(covered == 1), g
        assert abs(bh.m[pl].sum() + bh.cmass[cl].sum() - total) < 1e-12


def _walk(bh, v, g, h, th2, pl, cl):
    """make_interaction_list restated over the exported node arrays."""
    if bh.ncount[v] <= bh.nleaf or np.all(bh.nchild[v] < 0):
        pl.extend(range(bh.nfirst[v], bh.nfirst[v] + bh.ncount[v]))
        return
    for w in bh.nchild[v]:
        if w < 0:
            continue
        if bh.ncount[w] == 1:
            pl.append(bh.nfirst[w])
            continue
        d = np.maximum(np.abs(bh.ccom[w] - g) - h, 0.0)
        if (d @ d) * th2 > (2.0 * bh.nhalf[w]) ** 2:
            cl.append(w)
        else:
            _walk(bh, w, g, h, th2, pl, cl)


def test_lists_follow_the_opening_rule(bh):
    th2 = bh.theta ** 2
    for g in range(bh.ngroups):
        pl, cl = [], []
        _walk(bh, 0, bh.gcentre[g], bh.ghalf[g], th2, pl, cl)
        np.testing.assert_array_equal(bh.pidx[bh.poff[g]:bh.poff[g + 1]], pl)
        np.testing.assert_array_equal(bh.cidx[bh.coff[g]:bh.coff[g + 1]], cl)


def test_cell_moments_are_direct_sums(bh):
    for v in range(0, len(bh.cmass), 7):
        s = slice(bh.nfirst[v], bh.nfirst[v] + bh.ncount[v])
        m, x = bh.m[s], bh.x[s]
        M = m.sum()
        com = (m[:, None] * x).sum(0) / M
        assert abs(bh.cmass[v] - M) <= 1e-12 * M
        np.testing.assert_allclose(bh.ccom[v], com, rtol=0, atol=1e-12 * max(1.0, np.abs(com).max()))
        if bh.ncount[v] == 1:
            continue
        d = x - com
        dd = (d * d).sum(1)
        q = np.array([(m * (3 * d[:, 0] * d[:, 0] - dd)).sum(), (m * 3 * d[:, 0] * d[:, 1]).sum(),
                      (m * 3 * d[:, 0] * d[:, 2]).sum(), (m * (3 * d[:, 1] * d[:, 1] - dd)).sum(),
                      (m * 3 * d[:, 1] * d[:, 2]).sum(), (m * (3 * d[:, 2] * d[:, 2] - dd)).sum()])
        scale = (m * dd).sum() * 3 + 1e-300
        np.testing.assert_allclose(bh.cquad[v], q, rtol=0, atol=1e-10 * scale)


def test_group_is_the_first_node_at_or_below_ncrit(bh):
    parent = np.full(len(bh.ncount), -1)
    for v in range(len(bh.ncount)):
        for w in bh.nchild[v]:
            if w >= 0:
                parent[w] = v
    node_of = {}   # the topmost node of each particle range (a chain of one-child nodes shares it)
    for v in range(len(bh.ncount)):
        key = (int(bh.nfirst[v]), int(bh.ncount[v]))
        if key not in node_of or bh.nhalf[v] > bh.nhalf[node_of[key]]:
            node_of[key] = v
    for g in range(bh.ngroups):
        v = node_of[(int(bh.gfirst[g]), int(bh.gcount[g]))]
        assert bh.ncount[v] <= bh.ncrit
        assert parent[v] < 0 or bh.ncount[parent[v]] > bh.ncrit
