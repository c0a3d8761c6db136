"""GPU parity of the device Hermite block-time-step integrator (pgb6_hermite_*, libpg6).

Every step is replayed on the CPU by the oracle's integrator functions (oracle/pg_oracle.c
orc_hermite_*, pinned to the reference's own PG6/banana integrator by test_hermite_oracle.py),
fed with the force the GPU computed for that step:

* the block time and the active set equal the oracle's selection exactly;
* the new state (t, dt, pos, vel, acc, jerk, pot of every particle) equals the oracle's corrector
  (or start-up step) bit for bit -- the integrator's arithmetic is the reference's FP64 formulas
  evaluated without fused multiply-adds;
* the force of every step matches the FP64 force oracle on the same predicted positions
  (rms relative 1e-6 over all steps and particles, as the force kernel's own tests).

Over whole runs (the reference's 1024-body Plummer sphere to t = 0.5) the energies at every
output time and the step counts stay within the spread that force rounding causes between the
reference and the FP64 oracle (tolerances in the tests).  Sizes: 1024 bodies (one selection
segment, small-call force kernel) and 16384 (eight segments, regular-mode force kernel).
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import gpu_available, pgb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "banana_pl001k.npz")
W = pgb.workloads


@pytest.fixture(scope="module")
def g6():
    if not gpu_available():
        pytest.skip("no GPU")
    g = pgb.ffi.G6()
    g.L.g6_open(0)
    return g


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def _params(g, case):
    epsinv, eta, eta_s, dtmax, tend = g[f"{case}_params"]
    return (0.0 if epsinv == 0 else 1.0 / (epsinv * epsinv)), eta, eta_s, dtmax, tend


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def _assert_state_equal(H, st, what):
    s = H.get()
    for k in ("t", "dt", "pos", "vel", "acc", "jrk", "pot"):
        a, b = s[k], getattr(st, k)
        if not np.array_equal(a, b):
            bad = np.nonzero((a != b).reshape(len(a), -1).any(axis=1))[0]
            raise AssertionError(f"{what}: {k} differs for {len(bad)} particles, first {bad[:5]}: "
                                 f"{a[bad[:3]]} vs {b[bad[:3]]}")


class ForceCheck:
    """FP64 force oracle on the step's predicted positions; collects relative errors."""

    def __init__(self, st, eps2):
        self.st, self.eps2 = st, eps2
        self.ea, self.ej, self.ep = [], [], []
        self.idx = np.arange(st.n, dtype=np.int32)
        self.mf = st.mass.astype(np.float32).astype(np.float64)

    def add(self, t_gl, act, xp, vp, acc, jrk, pot):
        pos, vel, a2, j6, m, tj = self.st.jmem()
        xj, vj = O.g6_predict(t_gl, pos, vel, a2, j6, tj)
        f32 = lambda a: a.astype(np.float32).astype(np.float64)
        ref = O.g6_force(xp, f32(vp), act, np.float32(self.eps2), xj, f32(vj), self.mf, self.idx)
        self.ea.append(_rel(acc, ref["acc"]))
        self.ej.append(_rel(jrk, ref["jrk"]))
        self.ep.append(np.abs(pot - ref["pot"]) / np.abs(ref["pot"]))

    def check(self, rms_tol=1e-6, max_tol=1e-4):
        for name, e in (("acc", self.ea), ("jrk", self.ej), ("pot", self.ep)):
            e = np.concatenate(e)
            rms = float(np.sqrt(np.mean(e * e)))
            assert rms <= rms_tol and e.max() <= max_tol, (name, rms, e.max())


def _replay(g6, mass, pos, vel, eps2, eta, eta_s, dtmax, nsteps):
    """Run the GPU integrator step by step, replaying each step with the oracle."""
    H = pgb.ffi.Hermite(g6, mass, pos, vel, eps2, eta, eta_s, dtmax)
    st = O.HermiteState(pos, vel, mass, dtmax)
    fc = ForceCheck(st, eps2)
    try:
        act, acc, jrk, pot = H.last_step()
        np.testing.assert_array_equal(act, np.arange(st.n))
        xp, vp = O.hermite_predict(st, act, 0.0)
        fc.add(0.0, act, xp, vp, acc, jrk, pot)
        assert O.hermite_startup(st, act, acc, jrk, pot, eta_s, dtmax) == 0
        _assert_state_equal(H, st, "start-up")
        resets = 0
        for k in range(nsteps):
            time, ni = H.step()
            t_gl, act_o = O.hermite_select(st)
            act, acc, jrk, pot = H.last_step()
            assert ni == len(act)
            np.testing.assert_array_equal(act, act_o, err_msg=f"step {k}")
            xp, vp = O.hermite_predict(st, act, t_gl)
            fc.add(t_gl, act, xp, vp, acc, jrk, pot)
            O.hermite_correct(st, act, t_gl, xp, vp, acc, jrk, pot, eta, dtmax)
            if t_gl - int(t_gl * (1.0 / dtmax)) * dtmax == 0.0:
                st.t[:] = 0.0
                resets += 1
                assert time == resets * dtmax
            else:
                assert time == resets * dtmax + t_gl
            _assert_state_equal(H, st, f"step {k} (t_gl {t_gl}, ni {ni})")
        fc.check()
        ek, ew = H.energy()
        e_o, ek_o, ew_o = st.energy()
        assert ek == pytest.approx(ek_o, rel=1e-13) and ew == pytest.approx(ew_o, rel=1e-13)
        return resets
    finally:
        H.close()


@pytest.mark.parametrize("case", ["eps0", "eps64"])
def test_steps_replay_bit_exact_pl001k(g6, gold, case):
    eps2, eta, eta_s, dtmax, tend = _params(gold, case)
    resets = _replay(g6, gold["mass"], gold["pos"], gold["vel"], eps2, eta, eta_s, dtmax, 420)
    assert resets >= 1   # the replay crossed a time reset


def test_steps_replay_bit_exact_16k(g6):
    x, v, m, _ = W.plummer_hermite(16384, W.SEED0 + 21)
    _replay(g6, m, x, v, 1.0 / 64 ** 2, 0.2, 0.01, 0.125, 60)


@pytest.mark.parametrize("case", ["eps0", "eps64"])
def test_run_to_half_matches_reference_energies(g6, gold, case):
    eps2, eta, eta_s, dtmax, tend = _params(gold, case)
    H = pgb.ffi.Hermite(g6, gold["mass"], gold["pos"], gold["vel"], eps2, eta, eta_s, dtmax)
    try:
        e_ref = gold[f"{case}_energies"]
        steps, blocks = [], []
        for k in range(1, 5):
            p, b = H.advance(k * dtmax)
            assert H.time == pytest.approx(k * dtmax, abs=0)
            steps.append(p)
            blocks.append(b)
            ek, ew = H.energy()
            # the printed energies have 8 decimals; the FP64-force oracle stays within 2e-8
            assert abs(ek + ew - e_ref[k, 0]) < 5e-8, (k, ek + ew, e_ref[k, 0])
            assert abs(ek - e_ref[k, 2]) < 5e-8 and abs(ew - e_ref[k, 1]) < 5e-8, (k, ek, ew, e_ref[k])
        np.testing.assert_allclose(steps, gold[f"{case}_steps"][1:], rtol=0.005)
        np.testing.assert_allclose(blocks, gold[f"{case}_blocks"][1:], rtol=0.02)
        s = H.get()
        np.testing.assert_array_equal(s["t"], 0.0)   # the run ended on a reset
        np.testing.assert_allclose(s["pos"], gold[f"{case}_snap_pos"], rtol=0, atol=1e-5)
        p, b = H.counts()
        assert p == sum(steps) + len(gold["mass"]) and b == sum(blocks) + 1
    finally:
        H.close()


def test_bad_arguments_are_refused(g6):
    g6.set_abort(False)
    try:
        with pytest.raises(RuntimeError):
            pgb.ffi.Hermite(g6, np.ones(1), np.zeros((1, 3)), np.zeros((1, 3)), 0.0, 0.2, 0.01, 0.125)
        x, v, m, _ = W.plummer_hermite(64, W.SEED0 + 5)
        with pytest.raises(RuntimeError):
            pgb.ffi.Hermite(g6, m, x, v, 1e-4, -1.0, 0.01, 0.125)
    finally:
        g6.clear_error()
        g6.set_abort(True)


def test_bounded_wait_gives_up_and_every_cta_returns(g6):
    """The step kernel's waits are bounded.  With the limit lowered to 100 SM cycles, a wait of
    an ordinary advance (the first grid barrier: 296 CTAs do not all arrive within 100 cycles)
    runs out: the error word is set, every CTA of the launch returns (the exit count grows by
    the grid), the call reports PGB_ERR_DEVICE, and the context stays usable (a fresh integrator
    with the default limit runs afterwards).  Nothing hangs: every wait ends after its limit."""
    x, v, m = W.plummer_henon(2048, W.SEED0 + 31)
    H = pgb.ffi.Hermite(g6, m, x, v, 1.0 / 64 ** 2, 0.2, 0.01, 0.125)
    try:
        gave_up, exits0, grid = H.wait_status()
        assert gave_up == 0 and exits0 == grid > 0          # the start-up launch
        H.set_wait_limit(100)
        g6.set_abort(False)
        g6.clear_error()
        p, b = C.c_longlong(), C.c_longlong()
        rc = g6.L.pgb6_hermite_advance(H.h, 0.125, C.byref(p), C.byref(b))
        code, msg = g6.last_error()
        assert rc == 4 and code == 4 and "timed out" in msg   # PGB_ERR_DEVICE
        gave_up, exits1, _ = H.wait_status()
        assert gave_up == 1 and exits1 == exits0 + grid
    finally:
        g6.clear_error()
        g6.set_abort(True)
        H.close()
    H2 = pgb.ffi.Hermite(g6, m, x, v, 1.0 / 64 ** 2, 0.2, 0.01, 0.125)
    try:
        H2.advance(0.125)
        assert H2.time == 0.125
        assert H2.wait_status()[0] == 0
    finally:
        H2.close()
