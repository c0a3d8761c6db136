"""Python access to the CPU checker: the FP64 restatement (liboracle.so, pg_oracle.c) and
the unmodified reference libraries compiled from their own sources (_ref/*.so).

TEST INFRASTRUCTURE ONLY.  Only the test suite, ``__graft_entry__.smoke()`` and the
benchmark's CPU-baseline / reference leg import this module; the CUDA force engine never
does.  Each reference library is loaded with RTLD_LOCAL because the GRAPE-5 newton and table
libraries export the same ``g5_*`` names.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_SRC = os.environ.get("PGB_REFERENCE", "/root/reference")   # the reference source tree

_lock = threading.Lock()
_lib = None

D = np.float64
F = np.float32
I32 = np.int32


def _p(a, ctype=C.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def build(ref: bool | None = None) -> None:
    """Compile liboracle.so, and the reference libraries when the reference tree exists."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref is None:
        ref = os.path.isdir(REF_SRC)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)


def lib() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            path = os.path.join(HERE, "liboracle.so")
            if not os.path.exists(path):
                subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
            L = C.CDLL(path)
            dp, fp, ip = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int)
            L.orc_g5_newton.argtypes = [C.c_int, dp, dp, C.c_int, dp, dp, dp, dp, dp]
            L.orc_g5_newton.restype = None
            L.orc_pg5_gen_force_table.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_double, fp, dp]
            L.orc_pg5_gen_force_table.restype = None
            L.orc_s2_force.argtypes = [C.c_double, C.c_double, C.c_double]
            L.orc_s2_force.restype = C.c_double
            L.orc_g5_table.argtypes = [C.c_int, dp, C.c_int, dp, dp, fp, C.c_int, C.c_int, C.c_double, dp]
            L.orc_g5_table.restype = None
            L.orc_g5_quad.argtypes = [C.c_int, dp, dp, C.c_int, dp, dp, dp, dp, dp]
            L.orc_g5_quad.restype = None
            L.orc_g6_predict.argtypes = [C.c_int, C.c_double, dp, dp, dp, dp, dp, dp, dp]
            L.orc_g6_predict.restype = None
            L.orc_g6_force.argtypes = [C.c_int, dp, dp, ip, C.c_double, dp, C.c_int, dp, dp, dp, ip,
                                       dp, dp, dp, ip, dp, dp, dp, ip, ip, C.c_int]
            L.orc_g6_force.restype = C.c_int
            L.orc_hermite_select.argtypes = [C.c_int, dp, dp, dp, ip]
            L.orc_hermite_select.restype = C.c_int
            L.orc_hermite_predict.argtypes = [C.c_int, ip, C.c_double, dp, dp, dp, dp, dp, dp, dp]
            L.orc_hermite_predict.restype = None
            L.orc_hermite_correct.argtypes = [C.c_int, ip, C.c_double, dp, dp, dp, dp, dp, C.c_double, C.c_double,
                                              dp, dp, dp, dp, dp, dp, dp]
            L.orc_hermite_correct.restype = None
            L.orc_hermite_startup.argtypes = [C.c_int, ip, dp, dp, dp, C.c_double, C.c_double, dp, dp, dp, dp, dp]
            L.orc_hermite_startup.restype = C.c_int
            L.orc_potential_energy.argtypes = [C.c_int, dp, dp, C.c_double]
            L.orc_potential_energy.restype = C.c_double
            _lib = L
    return _lib


FORCE_FN = C.CFUNCTYPE(C.c_double, C.c_double)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def g5_newton(xi, eps2i, xj, mj, eps2j=None):
    """FP64 GRAPE-5 direct sum: returns (acc[ni,3], pot[ni]) with pot = +sum m/r (self incl.)."""
    xi, xj, mj = _c(xi, D), _c(xj, D), _c(mj, D)
    ni, nj = len(xi), len(xj)
    eps2i = _c(np.broadcast_to(eps2i, (ni,)), D)
    if eps2j is not None:
        eps2j = _c(np.broadcast_to(eps2j, (nj,)), D)
    acc = np.zeros((ni, 3), D)
    pot = np.zeros(ni, D)
    lib().orc_g5_newton(ni, _p(xi), _p(eps2i), nj, _p(xj), _p(mj), _p(eps2j), _p(acc), _p(pot))
    return acc, pot


def s2_force(r, sft_pp, sft_pm):
    return lib().orc_s2_force(r, sft_pp, sft_pm)


def gen_force_table(exp_bit, frc_bit, func, rcut):
    """Reference-identical float table for force shape ``func(r)`` -> (table[tbl,2] f32, xscale)."""
    tbl = 1 << (exp_bit + frc_bit)
    table = np.zeros((tbl, 2), F)
    xs = C.c_double()
    cb = FORCE_FN(func)
    lib().orc_pg5_gen_force_table(exp_bit, frc_bit, C.cast(cb, C.c_void_p), rcut,
                                  _p(table, C.c_float), C.byref(xs))
    return table, xs.value


def g5_table(xi, xj, mj, table, exp_bit, frc_bit, xscale):
    """FP64 evaluation of the table force with the same table + lerp: returns acc[ni,3]."""
    xi, xj, mj = _c(xi, D), _c(xj, D), _c(mj, D)
    table = _c(table, F)
    acc = np.zeros((len(xi), 3), D)
    lib().orc_g5_table(len(xi), _p(xi), len(xj), _p(xj), _p(mj), _p(table, C.c_float),
                       exp_bit, frc_bit, xscale, _p(acc))
    return acc


def g5_quad(xi, eps2i, xc, mc, qc):
    """FP64 quadrupole cells: returns (acc[ni,3], pot[ni]) with pot = +sum(phi_p + phi_q)."""
    xi, xc, mc, qc = _c(xi, D), _c(xc, D), _c(mc, D), _c(qc, D)
    ni = len(xi)
    eps2i = _c(np.broadcast_to(eps2i, (ni,)), D)
    acc = np.zeros((ni, 3), D)
    pot = np.zeros(ni, D)
    lib().orc_g5_quad(ni, _p(xi), _p(eps2i), len(xc), _p(xc), _p(mc), _p(qc), _p(acc), _p(pot))
    return acc, pot


def g6_predict(ti, pos, vel, acc2, jrk6, tj):
    pos, vel, acc2, jrk6, tj = (_c(a, D) for a in (pos, vel, acc2, jrk6, tj))
    n = len(pos)
    xp = np.zeros((n, 3), D)
    vp = np.zeros((n, 3), D)
    lib().orc_g6_predict(n, ti, _p(pos), _p(vel), _p(acc2), _p(jrk6), _p(tj), _p(xp), _p(vp))
    return xp, vp


def g6_force(xi, vi, idi, eps2, xj, vj, mj, idj, h2=None, maxlen=0):
    """FP64 Hermite force.  Returns a dict with acc, jrk, pot (=-sum m/r), nnb, rnnb
    (softened r), r2nn, r2nn2 (second nearest), and nbcount/nblist/overflow when h2 given."""
    xi, vi, xj, vj, mj = (_c(a, D) for a in (xi, vi, xj, vj, mj))
    idi, idj = _c(idi, I32), _c(idj, I32)
    ni, nj = len(xi), len(xj)
    out = dict(acc=np.zeros((ni, 3), D), jrk=np.zeros((ni, 3), D), pot=np.zeros(ni, D),
               nnb=np.zeros(ni, I32), rnnb=np.zeros(ni, D), r2nn=np.zeros(ni, D),
               r2nn2=np.zeros(ni, D))
    nbc = nbl = None
    if h2 is not None:
        h2 = _c(np.broadcast_to(h2, (ni,)), D)
        nbc = np.zeros(ni, I32)
        nbl = np.zeros((ni, max(maxlen, 1)), I32)
    ov = lib().orc_g6_force(ni, _p(xi), _p(vi), _p(idi, C.c_int), eps2, _p(h2), nj, _p(xj), _p(vj),
                            _p(mj), _p(idj, C.c_int), _p(out["acc"]), _p(out["jrk"]), _p(out["pot"]),
                            _p(out["nnb"], C.c_int), _p(out["rnnb"]), _p(out["r2nn"]),
                            _p(out["r2nn2"]), _p(nbc, C.c_int), _p(nbl, C.c_int), maxlen)
    if h2 is not None:
        out.update(nbcount=nbc, nblist=nbl, overflow=ov)
    return out


def potential_energy(x, m, eps2):
    x, m = _c(x, D), _c(m, D)
    return lib().orc_potential_energy(len(x), _p(x), _p(m), eps2)


# ----------------------------------------------------------------------------------------
# The reference libraries themselves (compiled from the reference's own sources).

def ref_path(name: str) -> str:
    return os.path.join(REF_DIR, name)


def ref_available(name: str = "libpg5_ref.so") -> bool:
    return os.path.exists(ref_path(name))


def load_ref(name: str) -> C.CDLL:
    """Load one reference library privately (RTLD_LOCAL), a fresh handle per call site."""
    return C.CDLL(ref_path(name), mode=os.RTLD_LOCAL | os.RTLD_NOW)


# ------------------------------------------------------------------------------------------
# Hermite block-time-step integrator (PG6/banana): see pg_oracle.c orc_hermite_*.

class HermiteState:
    """The integrator's particle state in the reference's storage precision (struct Particle,
    PG6/banana/particle.h): t, dt, pos, vel, acc in FP64; jrk, mass, pot as floats (held in
    float64 arrays with float values)."""

    def __init__(self, pos, vel, mass, dtmax):
        n = len(mass)
        self.n = n
        self.t = np.zeros(n)
        self.dt = np.full(n, float(dtmax))
        self.pos = np.ascontiguousarray(pos, D).copy()
        self.vel = np.ascontiguousarray(vel, D).copy()
        self.acc = np.zeros((n, 3))
        self.jrk = np.zeros((n, 3))
        self.mass = np.asarray(mass, F).astype(D)
        self.pot = np.zeros(n)

    def copy(self):
        o = HermiteState.__new__(HermiteState)
        o.n = self.n
        for k in ("t", "dt", "pos", "vel", "acc", "jrk", "mass", "pot"):
            setattr(o, k, getattr(self, k).copy())
        return o

    def jmem(self):
        """The j-memory records the integrator writes (g6_set_j_particle arguments,
        hermite.c:240-265): acc/2 and jrk*(1/6)."""
        return self.pos, self.vel, self.acc * 0.5, self.jrk * (1.0 / 6.0), self.mass, self.t

    def energy(self):
        """calc_energy.c:9-33: kinetic sum m v^2 / 2 and potential sum m pot / 2."""
        ek = 0.5 * float(np.sum(self.mass * np.sum(self.vel * self.vel, axis=1)))
        ew = 0.5 * float(np.sum(self.mass * self.pot))
        return ek + ew, ek, ew


def hermite_select(st: HermiteState):
    t_gl = C.c_double()
    act = np.empty(st.n, I32)
    ni = lib().orc_hermite_select(st.n, _p(st.t), _p(st.dt), C.byref(t_gl), _p(act, C.c_int))
    return t_gl.value, act[:ni].copy()


def hermite_predict(st: HermiteState, act, t_gl):
    act = np.ascontiguousarray(act, I32)
    xp = np.empty((len(act), 3))
    vp = np.empty((len(act), 3))
    lib().orc_hermite_predict(len(act), _p(act, C.c_int), t_gl, _p(st.t), _p(st.pos), _p(st.vel), _p(st.acc),
                              _p(st.jrk), _p(xp), _p(vp))
    return xp, vp


def hermite_correct(st: HermiteState, act, t_gl, xp, vp, acc1, jrk1, pot1, eta, dtmax):
    act = np.ascontiguousarray(act, I32)
    lib().orc_hermite_correct(len(act), _p(act, C.c_int), t_gl, _p(_c(xp, D)), _p(_c(vp, D)), _p(_c(acc1, D)),
                              _p(_c(jrk1, D)), _p(_c(pot1, D)), eta, dtmax, _p(st.t), _p(st.dt), _p(st.pos),
                              _p(st.vel), _p(st.acc), _p(st.jrk), _p(st.pot))


def hermite_startup(st: HermiteState, act, acc1, jrk1, pot1, eta_s, dtmax):
    act = np.ascontiguousarray(act, I32)
    return lib().orc_hermite_startup(len(act), _p(act, C.c_int), _p(_c(acc1, D)), _p(_c(jrk1, D)),
                                     _p(_c(pot1, D)), eta_s, dtmax, _p(st.t), _p(st.dt), _p(st.acc),
                                     _p(st.jrk), _p(st.pot))


def hermite_run(st: HermiteState, force, eta, eta_s, dtmax, tend, outputs=None, on_step=None):
    """The sample integrator's main loop (PG6/banana/banana01.c:96-183) restated over the
    functions above: the start-up step at t = 0 with every particle active, then block steps
    while the global time t_mod*dtmax + t_gl < tend.  After a step whose t_gl is a multiple of
    dtmax the output is taken (outputs.append((time, e, ek, ew, particle_steps, block_steps)))
    and the times are reset (reset_time, timestep.c:127-135).
    force(act, t_gl, xp, vp, changed) -> (acc, jrk, pot) evaluates the active i-particles
    (predicted xp, vp) against the j-memory; `changed` lists the particles whose j-memory record
    (HermiteState.jmem) changed since the previous call.  on_step(t_gl, act) is called after
    every block step."""
    n = st.n
    act = np.arange(n, dtype=I32)
    xp, vp = hermite_predict(st, act, 0.0)
    a, j, p = force(act, 0.0, xp, vp, act)
    bad = hermite_startup(st, act, a, j, p, eta_s, dtmax)
    if bad:
        raise RuntimeError("start-up step below dtmin")
    steps, blocks = n, 1
    if outputs is not None:
        outputs.append((0.0, *st.energy(), steps, blocks))
        steps = blocks = 0
    changed = act
    t_mod, t_gl = 0, 0.0
    while t_mod * dtmax + t_gl < tend:
        t_gl, act = hermite_select(st)
        xp, vp = hermite_predict(st, act, t_gl)
        a, j, p = force(act, t_gl, xp, vp, changed)
        hermite_correct(st, act, t_gl, xp, vp, a, j, p, eta, dtmax)
        changed = act
        steps += len(act)
        blocks += 1
        if on_step is not None:
            on_step(t_gl, act)
        if t_gl - int(t_gl * (1.0 / dtmax)) * dtmax == 0.0:
            if outputs is not None:
                outputs.append((t_mod * dtmax + t_gl, *st.energy(), steps, blocks))
                steps = blocks = 0
            t_mod += 1
            t_gl = 0.0
            st.t[:] = 0.0
            changed = np.arange(n, dtype=I32)
    return t_mod * dtmax + t_gl
