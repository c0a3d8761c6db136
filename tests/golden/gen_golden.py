"""Generate the golden vectors under tests/golden/ from the reference itself.

Runs the unmodified reference libraries (oracle/_ref/*.so, built from the reference's own
sources by `make -C oracle ref`) through their C APIs on small seeded inputs and stores inputs
plus outputs as .npz.  The fixtures pin the FP64 oracle (tests/test_oracle_golden.py) and give
the GPU tests a reference-produced answer on machines where the reference is not built.

    python tests/golden/gen_golden.py        # rewrites the .npz files
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

import conftest  # noqa: E402  (loads the package as phantom_grape_b200)
from oracle import oracle as O  # noqa: E402
from oracle import refapi  # noqa: E402

W = conftest.pgb.workloads


def g5_newton():
    s = W.plummer_g5(1024, seed=W.SEED0 + 1000)
    a, p = refapi.RefG5().force(s.x, s.m, s.eps, s.x)
    return dict(x=s.x, m=s.m, eps=s.eps, acc=a, pot=p)


def g5_symmetric():
    s = W.plummer_g5(512, seed=W.SEED0 + 1001)
    rng = W.Rng(1002)
    e2 = ((0.005 + 0.02 * rng.uniform(512)) ** 2).astype(np.float32).astype(np.float64)
    a, p = refapi.RefG5(symmetric=True).force(s.x, s.m, 0.0, s.x, eps2j=e2, eps2i=e2)
    return dict(x=s.x, m=s.m, eps2=e2, acc=a, pot=p)


def g5_quad():
    rng = W.Rng(1003)
    nc = 300
    xc = (4.0 * (rng.uniform(3 * nc).reshape(-1, 3) - 0.5)).astype(np.float32).astype(np.float64)
    mc = (0.5 + rng.uniform(nc)).astype(np.float32).astype(np.float64)
    q = 0.01 * (rng.uniform(6 * nc).reshape(-1, 6) - 0.5)
    q[:, 5] = -(q[:, 0] + q[:, 3])
    qc = q.astype(np.float32).astype(np.float64)
    xi = (0.3 * (rng.uniform(3 * 200).reshape(-1, 3) - 0.5)).astype(np.float32).astype(np.float64)
    eps = 1e-3
    am, pm, aq, pq = refapi.RefQuad().force(eps, xi, xc[:40], mc[:40], xc, mc, qc)
    return dict(xi=xi, xc=xc, mc=mc, qc=qc, eps=eps, acc_mono=am, pot_mono=pm, acc_quad=aq, pot_quad=pq)


def g5_table():
    R = refapi.RefG5Table()   # g5_open: default S2 table, 512 entries
    table = R.table()
    rng = W.Rng(1004)
    xj = 0.2 * rng.uniform(3 * 2000).reshape(-1, 3).astype(np.float32).astype(np.float64)
    mj = np.full(2000, 1.0 / 2000)
    xi = xj[::7].copy()
    a, p = R.force(xj, mj, xi)
    # a custom shape installed with pg5_gen_force_table (TreePM Gaussian split, 512 entries)
    f = W.gaussian_split_force(0.01, 0.045, 0.001)
    R.set_table(f, 0.045)
    table_gs = R.table()
    a_gs, _ = R.force(xj / 4.0, mj, xi / 4.0)
    return dict(xi=xi, xj=xj, mj=mj, table_s2=table, acc_s2=a, pot_s2=p, table_gs=table_gs, acc_gs=a_gs)


def g6_hermite():
    def fp64_force(x, v, m, eps2):
        idx = np.arange(len(x), dtype=np.int32)
        r = O.g6_force(x, v, idx, eps2, x, v, m, idx)
        return r["acc"], r["jrk"]

    st = W.hermite_state(1024, seed=W.SEED0 + 1005, force_fn=fp64_force)
    active = np.sort(W.Rng(1006).permutation(1024)[:200]).astype(np.int32)
    xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
    R = refapi.RefG6()
    R.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
    r = R.calc(st.t_now, 1024, xp[active], vp[active], active, st.eps2, h2=0.02, variant="2np")
    counts = np.array([len(r["nbl"][k][2]) for k in range(len(active))], np.int32)
    lists = np.concatenate([r["nbl"][k][2] for k in range(len(active))]).astype(np.int32)
    return dict(pos=st.pos, vel=st.vel, acc2=st.acc2, jrk6=st.jrk6, mass=st.mass, tj=st.tj, idx=st.idx,
                eps2=st.eps2, t_now=st.t_now, active=active, xi=xp[active], vi=vp[active], h2=0.02,
                acc=r["acc"], jrk=r["jrk"], pot=r["pot"], nnb=r["nnb"], rnnb=r["rnnb"],
                nb_counts=counts, nb_lists=lists)


CASES = dict(g5_newton=g5_newton, g5_symmetric=g5_symmetric, g5_quad=g5_quad, g5_table=g5_table,
             g6_hermite=g6_hermite)


def main():
    if not O.ref_available("libpg6_ref.so"):
        raise SystemExit("build the reference first: make -C oracle ref")
    for name, fn in CASES.items():
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **fn())
        print("wrote", name)


if __name__ == "__main__":
    main()
