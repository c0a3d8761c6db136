"""Pin the oracle's Hermite block-timestep integrator against the reference's own (CPU only).

tests/golden/banana_pl001k.npz holds the output of the reference's sample integrator
PG6/banana (tests/golden/gen_banana.py: built from the reference's sources with its -DNORMAL
setting, run on its 1024-body Plummer initial conditions to t = 0.5 for eps = 0 and 1/64).
The oracle's predictor, corrector, start-up step, block selection and time reset
(oracle/pg_oracle.c, orc_hermite_*) driven by oracle.hermite_run must reproduce it:

* with the reference's own GRAPE-6 library for the forces (where it is built here): the same
  particle and block steps per output interval, the printed energies to their 8 decimals, every
  particle's final dt bit for bit and its final position to 1e-12 and velocity to 1e-10;
* with the FP64 force oracle (always): the same block count per interval, particle steps
  within 0.1 %, energies within 3e-8 and final positions within 1e-6 (the forces differ from
  the reference's float-rounded ones in the last bits, which moves a few step-size decisions).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "banana_pl001k.npz")
CASES = ("eps0", "eps64")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def _params(g, case):
    epsinv, eta, eta_s, dtmax, tend = g[f"{case}_params"]
    eps2 = 0.0 if epsinv == 0 else 1.0 / (epsinv * epsinv)
    return eps2, eta, eta_s, dtmax, tend


def _run(g, case, force_of):
    eps2, eta, eta_s, dtmax, tend = _params(g, case)
    st = O.HermiteState(g["pos"], g["vel"], g["mass"], dtmax)
    outs = []
    t = O.hermite_run(st, force_of(st, eps2), eta, eta_s, dtmax, tend, outs)
    assert t == pytest.approx(tend)
    return st, np.array(outs)


def _fp64_force(st, eps2):
    idx = np.arange(st.n, dtype=np.int32)

    def force(act, t_gl, xp, vp, changed):
        pos, vel, a2, j6, m, tj = st.jmem()
        xj, vj = O.g6_predict(t_gl, pos, vel, a2, j6, tj)
        r = O.g6_force(xp, vp, act, eps2, xj, vj, m, idx)
        return r["acc"], r["jrk"], r["pot"]
    return force


def test_golden_fixture_is_consistent(gold):
    for case in CASES:
        assert len(gold[f"{case}_times"]) == 5
        np.testing.assert_allclose(gold[f"{case}_times"], np.arange(5) * 0.125)
        # printed total = kinetic + potential, and the snapshot's full-precision energies agree
        e = gold[f"{case}_energies"]
        np.testing.assert_allclose(e[:, 0], e[:, 1] + e[:, 2], atol=2e-8)
        ei, ep, etot, ek, ew = gold[f"{case}_snap_energy"]
        assert abs(etot - e[-1, 0]) < 1e-8 and abs(ek - e[-1, 2]) < 1e-8 and abs(ew - e[-1, 1]) < 1e-8
        assert np.all(gold[f"{case}_snap_t"] + gold[f"{case}_snap_dt"] <= 0.125 + 1e-15)


@pytest.mark.parametrize("case", CASES)
def test_integrator_matches_reference_with_fp64_forces(gold, case):
    st, outs = _run(gold, case, _fp64_force)
    e = gold[f"{case}_energies"]
    np.testing.assert_allclose(outs[:, 1], e[:, 0], rtol=0, atol=3e-8)
    np.testing.assert_allclose(outs[:, 2], e[:, 2], rtol=0, atol=3e-8)
    np.testing.assert_allclose(outs[:, 3], e[:, 1], rtol=0, atol=3e-8)
    np.testing.assert_array_equal(outs[:, 5], gold[f"{case}_blocks"])
    np.testing.assert_allclose(outs[:, 4], gold[f"{case}_steps"], rtol=1e-3)
    np.testing.assert_allclose(st.pos, gold[f"{case}_snap_pos"], rtol=0, atol=1e-6)
    assert np.mean(st.dt == gold[f"{case}_snap_dt"]) > 0.99


@pytest.mark.skipif(not O.ref_available("libpg6_ref.so"), reason="reference not built here")
@pytest.mark.parametrize("case", CASES)
def test_integrator_reproduces_reference_with_its_own_forces(gold, case):
    from oracle import refapi
    R = refapi.RefG6()

    def force_of(st, eps2):
        def force(act, t_gl, xp, vp, changed):
            R.set_j_at(changed, *st.jmem())
            r = R.calc(t_gl, st.n, xp, vp, act, eps2, variant="plain")
            return r["acc"], r["jrk"], r["pot"]
        return force

    st, outs = _run(gold, case, force_of)
    e = gold[f"{case}_energies"]
    np.testing.assert_array_equal(outs[:, 4], gold[f"{case}_steps"])
    np.testing.assert_array_equal(outs[:, 5], gold[f"{case}_blocks"])
    np.testing.assert_array_equal(np.round(outs[:, 1:4], 8), e[:, [0, 2, 1]])
    np.testing.assert_array_equal(st.dt, gold[f"{case}_snap_dt"])
    np.testing.assert_array_equal(st.t, gold[f"{case}_snap_t"])
    np.testing.assert_allclose(st.pos, gold[f"{case}_snap_pos"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(st.vel, gold[f"{case}_snap_vel"], rtol=0, atol=1e-10)
    np.testing.assert_array_equal(st.jrk, gold[f"{case}_snap_jrk"])
