"""GPU parity of the GRAPE-6 API with more pipelines than the reference's 48.

g6_npipes() is an environment setting of this library (PGB_G6_NPIPES, read once per process),
so the case runs in a child process.  With 1024 pipelines a g6calc_lasthalf2p call carries up
to 1024 i-particles: the call no longer fits the parameter-block launch of small calls and
takes the staged path (i-records uploaded, several i-tiles, two-level reduction of the j-chunk
partial sums).  Tolerances as in test_g6_gpu.py (vs the FP64 oracle: rms relative 1e-6).
"""
import os
import subprocess
import sys

import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from conftest import pgb
from oracle import oracle as O
W = pgb.workloads
g6 = pgb.ffi.G6()
g6.L.g6_open(0)
assert g6.L.g6_npipes() == 1024, g6.L.g6_npipes()

def fp64_force(x, v, m, eps2):
    idx = np.arange(len(x), dtype=np.int32)
    r = O.g6_force(x, v, idx, eps2, x, v, m, idx)
    return r["acc"], r["jrk"]

st = W.hermite_state(8192, seed=W.SEED0 + 3, force_fn=fp64_force)
g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
active = np.sort(W.Rng(11).permutation(len(st.mass))[:3000]).astype(np.int32)
xp, vp = O.g6_predict(st.t_now, st.pos, st.vel, st.acc2, st.jrk6, st.tj)
vpf = vp.astype(np.float32).astype(np.float64)
mf = st.mass.astype(np.float32).astype(np.float64)
ref = O.g6_force(xp[active], vpf[active], st.idx[active], np.float32(st.eps2), xp, vpf, mf, st.idx)
res = g6.calc(st.t_now, len(st.mass), xp[active], vp[active], st.idx[active], st.eps2, variant="2p")
rel = lambda a, b: np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
rms = lambda x: float(np.sqrt(np.mean(np.square(x))))
ea, ej = rel(res["acc"], ref["acc"]), rel(res["jrk"], ref["jrk"])
ep = np.abs(res["pot"] - ref["pot"]) / np.abs(ref["pot"])
assert rms(ea) <= 1e-6 and rms(ej) <= 1e-6 and rms(ep) <= 1e-6, (rms(ea), rms(ej), rms(ep))
sep = ref["r2nn2"] / ref["r2nn"] - 1.0
clear = sep > 1e-5
assert np.array_equal(res["nnb"][clear], ref["nnb"][clear])
np.testing.assert_allclose(res["rnnb"], ref["rnnb"], rtol=1e-6)
print("ok", rms(ea), rms(ej), rms(ep))
"""


def test_hermite_api_1024_pipes():
    if not gpu_available():
        pytest.skip("no GPU")
    env = dict(os.environ, PGB_G6_NPIPES="1024")
    r = subprocess.run([sys.executable, "-c", CHILD, HERE], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert r.stdout.startswith("ok"), r.stdout
