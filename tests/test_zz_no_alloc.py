"""The allocation-free force call, pgb6_force_noalloc (lib/libpg6.so).

It exists for callers that cannot let the library allocate GPU memory -- codes that own all of
their device memory through their own pool, and step loops that cannot pay the device-wide
synchronisation of cudaMalloc / cudaFree.  Its scratch (work list, counters, partial sums) is a
fixed array in the library's static device memory, shared by every call.

Checked here through the C ABI:
* two calls in a row give the same forces, jerks, potentials and nearest neighbours as the
  allocating entry point (a one-item plan) within the tolerance of the other GPU tests (rms
  relative 1e-6), and bit-identical results to each other;
* both calls agree with the FP64 direct sum of the oracle on the same inputs (rms relative
  acc / jerk / pot <= 1e-6, nearest neighbour identical wherever the FP64 first and second
  neighbours are separated), so a defect shared by both entry points is caught too;
* the device's free memory is the same before and after the two calls (nothing allocated);
* an i count beyond the fixed scratch is refused with PGB_ERR_CAPACITY instead of being run
  (its buffers are sized for that count, so a regression gives a wrong return code, not an
  out-of-bounds access).
The file is named so that pytest collects it last; it also runs alone in a fresh process.
"""
import numpy as np
import pytest

from conftest import pgb, gpu_available

pytestmark = pytest.mark.gpu

PGB_ERR_CAPACITY = 3


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def _rms(x):
    return float(np.sqrt(np.mean(np.square(x))))


def _cols(out, prefix):
    return np.stack([out[prefix + c] for c in "xyz"], 1)


@pytest.fixture(scope="module")
def setup():
    if not gpu_available():
        pytest.skip("no GPU")
    import torch
    g6 = pgb.ffi.G6()
    g6.L.g6_open(0)
    fn = pgb.ffi.bind_noalloc(g6)
    cs = pgb.workloads.cluster_set(ncl=1, nmin=20000, nmax=20000, seed=2027)
    n = len(cs.mass)
    idx = np.arange(n, dtype=np.int32)
    ni = 3001   # a ragged i count (not a multiple of any i-tile)
    irec = pgb.ffi.g6_irecords(cs.pos[:ni], cs.vel[:ni], idx[:ni])
    jrec = pgb.ffi.g6_jrecords(cs.pos, cs.vel, cs.mass, idx)
    dev = torch.device("cuda")
    d_i = torch.from_numpy(irec.view(np.uint8)).to(dev)
    d_j = torch.from_numpy(jrec.view(np.uint8)).to(dev)
    outs = [torch.zeros(ni * pgb.ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev) for _ in range(3)]
    return dict(torch=torch, g6=g6, fn=fn, n=n, ni=ni, eps2=cs.eps2, d_i=d_i, d_j=d_j, outs=outs, cs=cs, idx=idx)


def test_noalloc_matches_allocating_entry_point_twice(setup):
    S = setup
    torch, g6, fn = S["torch"], S["g6"], S["fn"]
    stream = torch.cuda.current_stream().cuda_stream
    # reference answer from the allocating path: a one-item plan
    plan = g6.plan_create([[0, S["ni"], 0, S["n"]]], nn=True)
    try:
        g6.plan_launch(plan, S["d_i"].data_ptr(), S["d_j"].data_ptr(), S["eps2"], S["outs"][0].data_ptr(), stream)
    finally:
        g6.plan_destroy(plan)
    torch.cuda.synchronize()
    # a warm-up call: the first call on a device resolves the scratch array's address and the
    # library's kernels are loaded; after it, free device memory must not change
    assert fn(S["d_i"].data_ptr(), S["ni"], S["d_j"].data_ptr(), S["n"], S["eps2"], S["outs"][1].data_ptr(),
              g6.NN, stream) == 0, g6.last_error()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    res = []
    for k in (1, 2):  # two calls in a row
        S["outs"][k].fill_(0xFF)
        rc = fn(S["d_i"].data_ptr(), S["ni"], S["d_j"].data_ptr(), S["n"], S["eps2"], S["outs"][k].data_ptr(),
                g6.NN, stream)
        assert rc == 0, g6.last_error()
        torch.cuda.synchronize()
        res.append(S["outs"][k].cpu().numpy().view(pgb.ffi.G6OUT))
    assert torch.cuda.mem_get_info()[0] == free_before, "the allocation-free call changed the free device memory"
    ref = S["outs"][0].cpu().numpy().view(pgb.ffi.G6OUT)
    for r in res:
        assert _rms(_rel(_cols(r, "a"), _cols(ref, "a"))) <= 1e-6
        assert _rms(_rel(_cols(r, "j"), _cols(ref, "j"))) <= 1e-6
        np.testing.assert_allclose(r["pot"], ref["pot"], rtol=1e-6)
        np.testing.assert_array_equal(r["jadr"], ref["jadr"])
        np.testing.assert_allclose(r["key"], ref["key"], rtol=1e-6)
    assert res[0].tobytes() == res[1].tobytes()

    # against the FP64 direct sum on the same inputs (velocities and masses as the float records
    # carry them)
    from oracle import oracle as O
    cs, idx, ni = S["cs"], S["idx"], S["ni"]
    f = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    o = O.g6_force(cs.pos[:ni], f(cs.vel[:ni]), idx[:ni], np.float32(S["eps2"]), cs.pos, f(cs.vel), f(cs.mass), idx)
    for r in res:
        assert _rms(_rel(_cols(r, "a"), o["acc"])) <= 1e-6
        assert _rms(_rel(_cols(r, "j"), o["jrk"])) <= 1e-6
        assert _rms((r["pot"] - o["pot"]) / np.abs(o["pot"])) <= 1e-6
        clear = o["r2nn2"] / o["r2nn"] - 1.0 > 1e-5
        assert clear.sum() > 0.9 * ni
        np.testing.assert_array_equal(idx[r["jadr"][clear]], o["nnb"][clear])


def test_noalloc_refuses_sizes_beyond_its_scratch(setup):
    S = setup
    torch, g6, fn = S["torch"], S["g6"], S["fn"]
    too_many = 4096 * 512 + 1   # more i-tiles than the fixed scratch holds, for any tile size
    dev = torch.device("cuda")
    # buffers sized for too_many records, so that even a failed capacity check stays in bounds
    d_i = torch.zeros(too_many * pgb.ffi.G6IREC.itemsize, dtype=torch.uint8, device=dev)
    d_o = torch.zeros(too_many * pgb.ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
    g6.set_abort(False)
    try:
        g6.clear_error()
        rc = fn(d_i.data_ptr(), too_many, S["d_j"].data_ptr(), S["n"], S["eps2"], d_o.data_ptr(), g6.NN,
                torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        code, msg = g6.last_error()
        assert rc == PGB_ERR_CAPACITY and code == PGB_ERR_CAPACITY and "scratch" in msg
    finally:
        g6.clear_error()
        g6.set_abort(True)
