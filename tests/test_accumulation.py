"""Summation error of the kernels' accumulation scheme (CPU, numpy float32 arithmetic).

The force kernels sum each i's FP32 pair terms in FP32 over blocks of at most 128 terms
(G5_FOLD / G6_FOLD in csrc/pgb_g5_kernels.cuh and pgb_g6_kernels.cuh) and add the block sums
into FP64.  On the acceleration terms of a Plummer sphere (the C2 distribution, eps^2 = 1e-8)
this keeps the rounding of the summation near that of the FP32 pair arithmetic itself, where
FP32 sums over a whole long j-range are two orders of magnitude worse; a compensated
(two-sum) FP32 sum is more accurate still but costs three more FP32 operations per
accumulator and pair.  The test pins these relations (relative rms errors against the exact
sum of the same FP32 terms, and against the FP64 force for the pair arithmetic).
"""
import numpy as np

from conftest import pgb

W = pgb.workloads
F32 = np.float32


def _terms(n=32768, ni=32):
    x, _, m, _ = W.plummer_hermite(n, W.SEED0 + 1)
    I = np.random.default_rng(3).choice(n, ni, replace=False)
    dx = (x[None, :, :] - x[I][:, None, :]).astype(F32)          # FP64 difference rounded to FP32
    r2 = (dx[..., 0] * dx[..., 0] + dx[..., 1] * dx[..., 1] + dx[..., 2] * dx[..., 2] + F32(1e-8)).astype(F32)
    q = (F32(-2.0) / np.sqrt(r2)).astype(F32)
    q[np.arange(ni), I] = 0
    mq3 = (m.astype(F32)[None, :] * q * (q * q)).astype(F32)
    t = (mq3[..., None] * dx).astype(F32)                          # -8 m dx / r^3, FP32 terms
    d64 = x[None, :, :] - x[I][:, None, :]
    r = np.sqrt((d64 * d64).sum(-1) + 1e-8)
    r[np.arange(ni), I] = np.inf
    true = (-8.0 * (m[None, :] / r ** 3)[..., None] * d64).sum(1)
    return t, true


def _rms_rel(a, b):
    e = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
    return float(np.sqrt(np.mean(e * e)))


def _blocked(t, block):
    s = np.zeros(t.shape[::2])
    for j0 in range(0, t.shape[1], block):
        s += np.cumsum(t[:, j0:j0 + block], axis=1, dtype=F32)[:, -1].astype(np.float64)
    return s


def test_blocked_fp32_sums_stay_at_the_pair_arithmetic_level():
    t, true = _terms()
    exact = t.astype(np.float64).sum(axis=1)
    pair = _rms_rel(exact, true)                       # FP32 pair arithmetic, exact summation
    b128 = _rms_rel(_blocked(t, 128), exact)
    b1024 = _rms_rel(_blocked(t, 1024), exact)
    whole = _rms_rel(np.cumsum(t, axis=1, dtype=F32)[:, -1].astype(np.float64), exact)
    assert pair < 5e-8
    assert b128 < 2.0 * pair                           # the kernels' blocks
    assert b1024 > 1.5 * b128                          # a whole 1024-record tile
    assert whole > 30 * b128                           # plain FP32 over the whole j-range
    # compensated (Kahan) FP32 summation, for comparison: below the blocked sum
    s = np.zeros(t.shape[::2], F32)
    c = np.zeros_like(s)
    for j in range(t.shape[1]):
        y = (t[:, j] - c).astype(F32)
        u = (s + y).astype(F32)
        c = ((u - s).astype(F32) - y).astype(F32)
        s = u
    assert _rms_rel(s.astype(np.float64) - c.astype(np.float64), exact) < b128
