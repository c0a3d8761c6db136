"""Pin the FP64 oracle against golden vectors produced by the reference itself (CPU only).

tests/golden/*.npz hold the outputs of the unmodified reference libraries (built from the
reference's own sources, tests/golden/gen_golden.py).  The FP64 oracle must agree with them
within the reference's own measured error against FP64 (raw 12-bit rsqrt for PG5,
Newton-refined for PG6): that is what makes the oracle a valid checker of the GPU path.
Where the reference is built here, the fixtures are also regenerated and must match bit for bit.
"""
import os

import numpy as np
import pytest

from conftest import pgb
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def rms(x):
    return float(np.sqrt(np.mean(np.square(x))))


def test_g5_newton_oracle_vs_reference():
    g = load("g5_newton")
    a, p = O.g5_newton(g["x"], np.float32(float(g["eps"]) ** 2), g["x"], g["m"])
    e = rel(g["acc"], a)
    assert rms(e) < 2e-4 and e.max() < 3e-3          # reference AVX2: rms 4.3e-5, max 1.1e-3
    assert np.abs(g["pot"] / p - 1).max() < 3e-5       # pot returned positive (+sum m/r)


def test_g5_symmetric_oracle_vs_reference():
    g = load("g5_symmetric")
    a, p = O.g5_newton(g["x"], g["eps2"], g["x"], g["m"], eps2j=g["eps2"])
    assert rms(rel(g["acc"], a)) < 2e-4
    assert np.abs(g["pot"] / p - 1).max() < 3e-4      # GravityKernel0's raw rsqrt: measured 1.3e-4


def test_g5_quad_oracle_vs_reference():
    g = load("g5_quad")
    eps2 = np.float32(float(g["eps"]) ** 2)
    a, p = O.g5_quad(g["xi"], eps2, g["xc"], g["mc"], g["qc"])
    e = rel(g["acc_quad"], a)
    assert rms(e) < 2e-3 and e.max() < 2e-2
    # the API returns the quadrupole potential negated (quad_g5c.c:292 via g5_get_forceMC)
    assert np.abs(-g["pot_quad"] / p - 1).max() < 5e-4
    am, pm = O.g5_newton(g["xi"], eps2, g["xc"][:40], g["mc"][:40])
    assert rms(rel(g["acc_mono"], am)) < 3e-3           # 40 j only, near-cancelling: measured 7.5e-4


def test_g5_table_oracle_vs_reference():
    g = load("g5_table")
    t = g["table_s2"]
    o, xs = O.gen_force_table(4, 5, lambda r: O.s2_force(r, 0.1 / 64, 3.0 / 64), 3.0 / 64)
    assert o.tobytes() == t.tobytes()                   # bit-identical table generation
    a = O.g5_table(g["xi"], g["xj"], g["mj"], t, 4, 5, xs)
    e = rel(g["acc_s2"], a)
    assert rms(e) < 1e-5 and e.max() < 1e-3
    assert np.all(g["pot_s2"] == 0)
    f = pgb.workloads.gaussian_split_force(0.01, 0.045, 0.001)
    o2, xs2 = O.gen_force_table(4, 5, f, 0.045)
    assert o2.tobytes() == g["table_gs"].tobytes()
    a2 = O.g5_table(g["xi"] / 4, g["xj"] / 4, g["mj"], o2, 4, 5, xs2)
    assert rms(rel(g["acc_gs"], a2)) < 1e-5


def test_g6_hermite_oracle_vs_reference():
    g = load("g6_hermite")
    xp, vp = O.g6_predict(float(g["t_now"]), g["pos"], g["vel"], g["acc2"], g["jrk6"], g["tj"])
    act = g["active"]
    np.testing.assert_allclose(xp[act], g["xi"], rtol=0, atol=1e-14)
    vf = vp.astype(np.float32).astype(np.float64)
    r = O.g6_force(xp[act], vf[act], g["idx"][act], np.float32(float(g["eps2"])), xp, vf,
                   g["mass"].astype(np.float32).astype(np.float64), g["idx"], h2=np.full(len(act), 0.02),
                   maxlen=1024)
    assert rel(g["acc"], r["acc"]).max() < 5e-6       # reference: acc rms 6.8e-8
    assert rel(g["jrk"], r["jrk"]).max() < 1e-4       # jerk rms 1.8e-6
    assert (np.abs(g["pot"] - r["pot"]) / np.abs(r["pot"])).max() < 2e-7
    clear = r["r2nn2"] / r["r2nn"] - 1 > 1e-5
    assert np.array_equal(g["nnb"][clear], r["nnb"][clear])
    np.testing.assert_allclose(g["rnnb"], r["rnnb"], rtol=1e-6)
    # neighbour lists: same sets (in j order) except j within 1e-5 of the radius
    off = 0
    for k, i in enumerate(act):
        n = int(g["nb_counts"][k])
        got = g["nb_lists"][off:off + n]
        off += n
        want = r["nblist"][k, :r["nbcount"][k]]
        d2 = np.sum((xp - xp[i]) ** 2, axis=1) + float(g["eps2"])
        edge = set(np.nonzero(np.abs(d2 / 0.02 - 1) < 1e-5)[0].tolist())
        assert set(got.tolist()) - edge == set(want.tolist()) - edge
        assert list(got) == sorted(got)


@pytest.mark.skipif(not O.ref_available("libpg6_ref.so"), reason="reference not built here")
def test_fixtures_regenerate_bit_exact():
    import importlib.util
    spec = importlib.util.spec_from_file_location("gen_golden", os.path.join(GOLD, "gen_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    for name in ("g5_newton", "g5_table", "g6_hermite"):
        new = gen.CASES[name]()
        old = load(name)
        for k, v in new.items():
            assert np.asarray(v).tobytes() == old[k].tobytes(), (name, k)
