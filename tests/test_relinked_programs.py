"""The drop-in, proven with the reference's own programs: its sample N-body codes, compiled
unmodified from their sources, linked once against the reference library and once against this
repository's B200 library (oracle/Makefile: direct_ref / direct_b200, banana01 / banana01_b200),
run on the same input, must print the same physics.

* PG5/newton/direct (leapfrog, dt = 0.01, eps = 0.02, 1000 steps, g5_set_xmj + g5_set_eps_to_all
  + g5_set_n + g5_calculate_force_on_x per step; direct.c:133-176): a seeded 1024-body Plummer
  sphere written in its input format.  The total energy it prints every 100 steps agrees within
  5e-5 relative (the integration's own energy error is ~1e-5; the two force paths differ by
  FP32 rounding, and the reference's by its rsqrt bias factors), and the first output's kinetic
  and potential energies within 1e-4.
* PG6/banana (4th-order Hermite block time steps through g6_set_j_particle, g6_set_ti,
  g6calc_firsthalf, g6calc_lasthalf per 48 i): the reference's own 1024-body Plummer initial
  conditions (stored in tests/golden/banana_pl001k.npz by gen_banana.py) to t = 0.5 with the
  reference's input.list parameters; every printed energy agrees with the reference-linked run
  within 1e-6 relative, and the step counts within 1 %.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, gpu_available

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden", "banana_pl001k.npz")


def _need(*names):
    if not gpu_available():
        pytest.skip("no GPU")
    missing = [n for n in names if not os.path.exists(os.path.join(REF, n))]
    if missing:
        pytest.skip(f"not built: {missing} (make -C oracle ref)")


def _plummer_text(path, n=1024):
    from conftest import pgb
    W = pgb.workloads
    x, v, m = W.plummer_henon(n, W.SEED0 + 21)
    with open(path, "w") as f:
        f.write(f"{n}\n3\n0.0\n")
        f.writelines(f"{a:.17g}\n" for a in m)
        f.writelines(f"{r[0]:.17g} {r[1]:.17g} {r[2]:.17g}\n" for r in x)
        f.writelines(f"{r[0]:.17g} {r[1]:.17g} {r[2]:.17g}\n" for r in v)


def _run(prog, args, cwd, threads=4):
    r = subprocess.run([os.path.join(REF, prog)] + args, cwd=cwd, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
    assert r.returncode == 0, (prog, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def test_direct_relinked_against_the_b200_library():
    _need("direct_ref", "direct_b200")
    with tempfile.TemporaryDirectory() as d:
        _plummer_text(os.path.join(d, "pl1k"))
        outs = [_run(p, ["pl1k", p + ".out"], d) for p in ("direct_ref", "direct_b200")]
    parsed = []
    for out in outs:
        e = np.array(re.findall(r"^e: ([-+0-9.e]+) de: ([-+0-9.e]+)", out, re.M), dtype=np.float64)
        kp = np.array(re.findall(r"^ke: ([-+0-9.e]+) pe: ([-+0-9.e]+)", out, re.M), dtype=np.float64)
        steps = re.findall(r"^step: (\d+)", out, re.M)
        parsed.append((e, kp, steps))
    (e0, kp0, s0), (e1, kp1, s1) = parsed
    assert len(s0) == len(s1) == 9 and s0 == s1
    np.testing.assert_allclose(e1[:, 0], e0[:, 0], rtol=5e-5)
    np.testing.assert_allclose(kp1[0], kp0[0], rtol=1e-4)


def test_banana_relinked_against_the_b200_library():
    _need("banana01", "banana01_b200")
    g = np.load(GOLDEN)
    with tempfile.TemporaryDirectory() as d:
        init = os.path.join(d, "pl001k.init")
        with open(init, "w") as f:
            m, x, v = g["mass"], g["pos"], g["vel"]
            f.write(f"0.0\n{len(m)}\n")
            for i in range(len(m)):
                f.write(f"{i + 1}\n{m[i]:.17g}\n{x[i, 0]:.17g} {x[i, 1]:.17g} {x[i, 2]:.17g}\n"
                        f"{v[i, 0]:.17g} {v[i, 1]:.17g} {v[i, 2]:.17g}\n")
        with open(os.path.join(d, "input.list"), "w") as f:
            f.write(f"0 0.5 0.5\n0.0\n0.2 0.01 8.0\n{init}\nsnap\n")
        outs = [_run(p, [], d) for p in ("banana01", "banana01_b200")]
    res = []
    for out in outs:
        en = np.array(re.findall(r"^tot: ([-+0-9.]+) w: ([-+0-9.]+) k: ([-+0-9.]+)", out, re.M), dtype=np.float64)
        st = np.array([float(b) for _, b in re.findall(r"niave: ([0-9.e+-]+) ([0-9.e+-]+)", out)])
        res.append((en, st))
    (en0, st0), (en1, st1) = res
    assert len(en0) == len(en1) >= 4
    np.testing.assert_allclose(en1, en0, rtol=1e-6)
    np.testing.assert_allclose(en0, g["eps0_energies"][:len(en0)], rtol=1e-7)   # the reference run is the golden one
    assert np.all(np.abs(st1 - st0) <= 0.01 * st0 + 1)
