#!/usr/bin/env python
"""Benchmark of the B200 pairwise-force engine (one JSON line on stdout from rank 0).

Workload (default, ``--workload hermite``): the PG6 4th-order Hermite force path on a
N = 65536 Plummer sphere (distribution-function velocities, FP64 state, eps = 1e-4) in a
block-time-step state; one step = 64 force calls with active sets of 2^k particles
(k uniform in 4..16), each call = j-prediction of all 65536 particles to the call's time +
force / jerk / potential / nearest neighbour of the active set against all j.
About 4.1e10 pair interactions per step (60-flop convention, PG6/banana/banana01.h:9).

Numbers:
* ``value``   Gint/s of the batched device path (pgb6 plans: one persistent launch per call,
              the 64 calls captured in one CUDA graph; inputs resident in HBM), device time
              from CUDA events, L2 flushed (256 MiB write) between steps.
* ``e2e``     the same schedule through the drop-in GRAPE-6 API (g6_set_ti,
              g6calc_firsthalf / g6calc_lasthalf2p per npipes chunk, g6_set_j_particle of the
              active set) with host buffers, timed on the host clock; the same driver replays
              the reference library's identical call sequence for ``--impl reference``.
* ``roofline`` the Hermite force kernel against the FP32 pipe: achieved = 60 flop x pairs / the
              kernel's CUDA-event time; peak = 148 SMs x 128 lanes x 2 x SM clock.
* ``cpu_baseline`` the reference's own AVX2 + OpenMP library (oracle/_ref) on the host cores,
              on a bounded sample of the same schedule.

Other workloads (``--workload``): ``direct`` (PG5 newton, N = 16384 Plummer, all i vs all j),
``clusters`` (1024 independent Plummer clusters, N log-uniform in [256, 16384], one Hermite
force evaluation each; batched vs 1024 sequences of plain calls), ``treepm`` (PG5 table, N=2^20
uniform periodic box, 1024-entry table, 4096 i-groups with their j-lists in one launch).

Multi-GPU (torchrun): every rank runs the full per-GPU workload on its own replica (the work
items are independent: no data-path collective), ``scaling`` is "weak", ``value`` is the sum
over ranks divided by the slowest rank's time (max over ranks via an NCCL all-reduce).
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SM_COUNT = 148
# DRAM bytes (read + write) of one launch of the roofline kernel, from the committed ncu captures
# (dram__bytes_read.sum + dram__bytes_write.sum); the bench cannot run ncu itself.
G5_CFG_NAMES = ["128x4", "256x2", "512x2", "1024x1", "384x2", "128x2", "128x1", "64x1"]   # pgb5 configurations (threads x i/thread)
PROFILED_TRAFFIC = {
    "hermite": {"bytes": 6_485_760 + 17_935_104,
                "source": "profiles/g6_kernel_hermite_65536x65536.md (128x2 configuration, paired accumulations)"},
    "direct": {"bytes": 542_720, "pairs": 268_435_456, "source": "profiles/g5_kernels_direct_treepm_bh.md (1024x1)"},
    "treepm": {"bytes": 557_901_056 + 35_891_456, "pairs": 4_463_983_086,
               "source": "profiles/g5_kernels_direct_treepm_bh.md (64x1)"},
    # captured at N = 2^20 (both launches of a step); scaled to the run's pairs
    "bh": {"bytes": 132_306_688 + 27_293_184 + 228_275_200 + 31_873_536, "pairs": 4_462_862_693,
           "source": "profiles/g5_kernels_direct_treepm_bh.md (64x1, N=2^20 capture scaled by pairs)"},
}


def profiled_traffic(workload, pairs):
    """DRAM bytes of one step's roofline kernel launches from the committed capture, scaled to
    `pairs` when the run's size differs from the capture's (traffic grows with the lists)."""
    e = PROFILED_TRAFFIC.get(workload)
    if not e:
        return None, None
    if "pairs" in e and pairs != e["pairs"]:
        return int(e["bytes"] * pairs / e["pairs"]), e["source"]
    return e["bytes"], e["source"]
FP32_LANES = 128


def load_pkg():
    name = "phantom_grape_b200"
    if name in sys.modules:
        return sys.modules[name]
    d = os.path.join(ROOT, "phantom-grape_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {"sm_max_mhz": 1965.0, "hbm_gbs": 6650.0}


# ----------------------------------------------------------------------------------------
# clocks sampled during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # the sampler is running (its first line written) before the timed region starts
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ----------------------------------------------------------------------------------------
# distributed plumbing

def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws, local, backend="nccl"):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if ws > 1:
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return dist


def reduce_max(value: float, ws: int, device) -> float:
    """Max over ranks (NCCL all-reduce on a one-element tensor); identity on one rank."""
    if ws <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, ws: int, device) -> float:
    if ws <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------------------------------
# Hermite workload (PG6 API)

def predict_np(t, st):
    """FP64 j-prediction (the library's own predictor formula, used here only to prepare the
    i-particles of each call as a host integrator's predictor would, hermite.c:39-60)."""
    dt = (t - st.tj)[:, None]
    x = st.pos + st.vel * dt + st.acc2 * dt * dt + st.jrk6 * dt ** 3
    v = st.vel + 2.0 * st.acc2 * dt + 3.0 * st.jrk6 * dt * dt
    return x, v


def hermite_workload(pgb, g6, n=65536, ncalls=64, seed_offset=0):
    W = pgb.workloads

    def gpu_force(x, v, m, eps2):
        idx = np.arange(len(x), dtype=np.int32)
        r = g6.batch_host([[0, len(x), 0, len(x)]], x, v, idx, x, v, m, idx, eps2, nn=False)
        return r["acc"], r["jrk"]

    st = W.hermite_state(n, seed=W.SEED0 + 1 + seed_offset, force_fn=gpu_force)
    sets = W.hermite_schedule(n, ncalls, seed=W.SEED0 + 101 + seed_offset)
    t_calls = st.t_now + np.arange(ncalls) * 2.0 ** -20
    set_off = np.concatenate([[0], np.cumsum([len(s) for s in sets])]).astype(np.int32)
    set_idx = np.concatenate(sets).astype(np.int32)
    xi = np.empty((len(set_idx), 3))
    vi = np.empty((len(set_idx), 3))
    for c, s in enumerate(sets):
        x, v = predict_np(t_calls[c], st)
        xi[set_off[c]:set_off[c + 1]] = x[s]
        vi[set_off[c]:set_off[c + 1]] = v[s]
    return dict(st=st, sets=sets, t_calls=t_calls, set_off=set_off, set_idx=set_idx, xi=xi, vi=vi, n=n,
                pairs=int(len(set_idx)) * n)


class Driver:
    """ctypes view of lib/libpgbdrv.so (drivers/pgb_drivers.c)."""

    def __init__(self, pgb):
        L = self.L = C.CDLL(pgb.ffi.lib_path("libpgbdrv.so"), mode=os.RTLD_LOCAL | os.RTLD_NOW)
        dp, ip, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
        L.g6drv_open.argtypes = [C.c_char_p]
        L.g6drv_open.restype = vp
        L.g6drv_npipes.argtypes = [vp]
        L.g6drv_npipes.restype = C.c_int
        L.g6drv_set_j.argtypes = [vp, C.c_int, dp, dp, dp, dp, dp, dp, ip, ip]
        L.g6drv_set_j.restype = C.c_double
        L.g6drv_schedule.argtypes = [vp, C.c_int, C.c_int, ip, ip, dp, dp, dp, C.c_double, C.c_int, C.c_int,
                                     dp, dp, dp, dp, dp, dp, ip, dp, dp, dp, ip, C.POINTER(C.c_float)]
        L.g6drv_schedule.restype = C.c_double
        L.g5drv_open.argtypes = [C.c_char_p]
        L.g5drv_open.restype = vp
        L.g5drv_direct.argtypes = [vp, C.c_int, dp, dp, C.c_double, dp, dp]
        L.g5drv_direct.restype = C.c_double
        L.g5drv_groups.argtypes = [vp, C.c_int, ip, dp, dp, dp, C.c_double, dp, dp, C.c_int]
        L.g5drv_groups.restype = C.c_double
        lp = C.POINTER(C.c_longlong)
        L.g5drv_bh.argtypes = [vp, C.c_int, C.c_int, ip, ip, dp, dp, dp, lp, ip, dp, dp, dp, lp, ip, C.c_double, dp, dp,
                               C.c_int]
        L.g5drv_bh.restype = C.c_double

    @staticmethod
    def p(a, t=C.c_double):
        return None if a is None else a.ctypes.data_as(C.POINTER(t))

    def g6_open(self, path):
        h = self.L.g6drv_open(path.encode())
        if not h:
            raise RuntimeError(f"cannot open {path}")
        return h

    def g6_set_j(self, h, st):
        p = self.p
        return self.L.g6drv_set_j(h, len(st.mass), p(st.pos), p(st.vel), p(st.acc2), p(st.jrk6), p(st.mass),
                                  p(st.tj), p(st.idx, C.c_int), None)

    def g6_schedule(self, h, wl, calls=None, resend=True, outputs=False):
        """Run calls [0, calls) of the schedule; returns (seconds, pairs, outputs or None)."""
        st, p = wl["st"], self.p
        ncalls = len(wl["sets"]) if calls is None else calls
        off = wl["set_off"]
        nact = int(off[ncalls])
        out = None
        if outputs:
            out = dict(acc=np.zeros((nact, 3)), jrk=np.zeros((nact, 3)), pot=np.zeros(nact),
                       nnb=np.zeros(nact, np.int32), rnnb=np.zeros(nact, np.float32))
        o = out or {}
        sec = self.L.g6drv_schedule(h, wl["n"], ncalls, p(off, C.c_int), p(wl["set_idx"], C.c_int), p(wl["t_calls"]),
                                    p(wl["xi"]), p(wl["vi"]), st.eps2, 1, 1 if resend else 0, p(st.pos), p(st.vel),
                                    p(st.acc2), p(st.jrk6), p(st.mass), p(st.tj), p(st.idx, C.c_int),
                                    p(o.get("acc")), p(o.get("jrk")), p(o.get("pot")), p(o.get("nnb"), C.c_int),
                                    p(o.get("rnnb"), C.c_float))
        return sec, nact * wl["n"], out


def ref_lib(name):
    """The reference's own build (oracle/_ref), compiled here when the reference is present."""
    path = os.path.join(ROOT, "oracle", "_ref", name)
    if not os.path.exists(path) and os.path.isdir("/root/reference"):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=False)
    return path if os.path.exists(path) else None


def cpu_sample_calls(wl, target_pairs):
    """Smallest prefix of the schedule with at least target_pairs interactions."""
    cum = np.cumsum([len(s) * wl["n"] for s in wl["sets"]])
    return int(min(len(cum), np.searchsorted(cum, target_pairs) + 1))


def cpu_baseline_hermite(pgb, wl, target_pairs=1.2e10):
    path = ref_lib("libpg6_ref.so")
    if path is None:
        return {"value": None, "unit": "Gint/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "unavailable: reference library not built"}
    drv = Driver(pgb)
    h = drv.g6_open(path)
    drv.g6_set_j(h, wl["st"])
    calls = cpu_sample_calls(wl, target_pairs)
    drv.g6_schedule(h, wl, calls=1)                 # warm-up (OpenMP pool, page faults)
    sec, pairs, _ = drv.g6_schedule(h, wl, calls=calls)
    return {"value": pairs / sec / 1e9, "unit": "Gint/s", "cores": os.cpu_count(), "kind": "reference",
            "sample": f"first {calls} of 64 block-step calls ({pairs:.3e} pairs, {sec:.1f} s), "
                      f"libpg6 AVX2 + OpenMP (PG6/libpg6 built from its sources), npipes 48"}


def run_hermite(args, pgb, ws, rank, local):
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ffi = pgb.ffi
    g6 = ffi.G6()
    g6.L.g6_open(0)
    wl = hermite_workload(pgb, g6, seed_offset=rank)
    st, n, sets = wl["st"], wl["n"], wl["sets"]
    if args.profile_api:
        # profiling target: the drop-in API's full-size call (npipes = 48 i-particles against all
        # n j-particles) through g6_set_ti + g6calc_firsthalf + g6calc_lasthalf2p, four times; no
        # timing.  The second force launch is the one to capture.
        g6.set_j(st.pos, st.vel, st.acc2, st.jrk6, st.mass, st.tj, st.idx)
        ni = g6.L.g6_npipes()
        for _ in range(4):
            g6.calc(st.t_now, n, st.pos[:ni], st.vel[:ni], st.idx[:ni], st.eps2, variant="2p")
        return {"profile": "drop-in API call", "ni": ni, "nj": n, "calls": 4}

    # device-resident inputs: j-memory records, the i-records of every call, outputs
    ptcl = np.zeros(n, ffi.G6PTCL)
    ptcl["pos"], ptcl["vel"], ptcl["acc2"], ptcl["jrk6"] = st.pos, st.vel, st.acc2, st.jrk6
    ptcl["mass"], ptcl["tim"], ptcl["idx"] = st.mass, st.tj, st.idx
    nact = len(wl["set_idx"])
    ff = not args.f64_positions
    pflags = 0 if ff else g6.POS_F64
    irec = ffi.g6_irecords(wl["xi"], wl["vi"], st.idx[wl["set_idx"]], ff=ff)
    d_ptcl = torch.from_numpy(ptcl.view(np.uint8)).to(dev)
    d_irec = torch.from_numpy(irec.view(np.uint8)).to(dev)
    d_pred = torch.zeros(n * ffi.G6PREDJ.itemsize, dtype=torch.uint8, device=dev)
    d_out = torch.zeros(nact * ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
    off = wl["set_off"]
    plans = [g6.plan_create([[int(off[c]), len(sets[c]), 0, n]], nn=True, f64=not ff) for c in range(len(sets))]
    s = torch.cuda.Stream(device=dev)

    def step_launches():
        for c in range(len(sets)):
            rc = g6.L.pgb6_predict(d_ptcl.data_ptr(), n, float(wl["t_calls"][c]), d_pred.data_ptr(), pflags,
                                   s.cuda_stream)
            assert rc == 0
            g6.plan_launch(plans[c], d_irec.data_ptr(), d_pred.data_ptr(), st.eps2, d_out.data_ptr(), s.cuda_stream)

    with torch.cuda.stream(s):
        step_launches()
    s.synchronize()
    tuned = {}
    if not args.no_tune and not args.profile_largest:
        # autotune the kernel configuration once per active-set size, on the real data
        for c in range(len(sets)):
            if len(sets[c]) in tuned:
                continue
            g6.L.pgb6_predict(d_ptcl.data_ptr(), n, float(wl["t_calls"][c]), d_pred.data_ptr(), pflags,
                              s.cuda_stream)
            cfg, ms = g6.plan_tune(plans[c], d_irec.data_ptr(), d_pred.data_ptr(), st.eps2, d_out.data_ptr(),
                                   s.cuda_stream)
            tuned[len(sets[c])] = cfg
        for c in range(len(sets)):   # re-create the plans so that every plan picks up its tuned shape
            g6.plan_destroy(plans[c])
            plans[c] = g6.plan_create([[int(off[c]), len(sets[c]), 0, n]], nn=True, f64=not ff)
        with torch.cuda.stream(s):
            step_launches()
        s.synchronize()
    if args.profile_largest:
        # profiling target: after the warm pass above (1 + 64 force launches), the largest call's
        # force launch three times; nothing else allocated, no timing
        big = max(range(len(sets)), key=lambda c: len(sets[c]))
        with torch.cuda.stream(s):
            g6.L.pgb6_predict(d_ptcl.data_ptr(), n, float(wl["t_calls"][big]), d_pred.data_ptr(), pflags,
                                   s.cuda_stream)
            for _ in range(3):
                g6.plan_launch(plans[big], d_irec.data_ptr(), d_pred.data_ptr(), st.eps2, d_out.data_ptr(),
                               s.cuda_stream)
        s.synchronize()
        for p_ in plans:
            g6.plan_destroy(p_)
        return {"profile": "largest Hermite call", "call": big, "active": len(sets[big]), "nj": n,
                "force_launches_before": 1 + len(sets)}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        step_launches()

    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks.start()
    barrier(ws)
    torch.cuda.synchronize()
    for k in range(args.steps):
        with torch.cuda.stream(s):
            ev[k][0].record(s)
            graph.replay()
            ev[k][1].record(s)
            flush.fill_(k & 0xFF)   # 256 MiB write between steps: L2 (126 MB) flushed
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_local = sum(step_ms) / 1e3
    t_max = reduce_max(t_local, ws, dev)
    pairs_total = reduce_sum(float(wl["pairs"]) * args.steps, ws, dev)
    value = pairs_total / t_max / 1e9

    # roofline pass (after the timed region): each force launch timed alone with CUDA events
    fev = []
    with torch.cuda.stream(s):
        for c in range(len(sets)):
            g6.L.pgb6_predict(d_ptcl.data_ptr(), n, float(wl["t_calls"][c]), d_pred.data_ptr(), pflags,
                                   s.cuda_stream)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            g6.plan_launch(plans[c], d_irec.data_ptr(), d_pred.data_ptr(), st.eps2, d_out.data_ptr(), s.cuda_stream)
            b.record(s)
            fev.append((a, b, len(sets[c]) * n))
    torch.cuda.synchronize()
    kern_s = sum(a.elapsed_time(b) for a, b, _ in fev) / 1e3
    kern_pairs = sum(p for _, _, p in fev)
    big = max(fev, key=lambda e: e[2])
    big_ms = big[0].elapsed_time(big[1])

    # end to end through the GRAPE-6 API with host buffers (same driver as the reference arm)
    drv = Driver(pgb)
    h = drv.g6_open(pgb.ffi.lib_path("libpg6.so"))
    drv.g6_set_j(h, st)
    drv.g6_schedule(h, wl, calls=4)   # warm-up
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    torch.cuda.synchronize()
    barrier(ws)
    e2e_t = 0.0
    for _ in range(e2e_steps):
        sec, _, _ = drv.g6_schedule(h, wl)
        e2e_t += sec
    e2e_max = reduce_max(e2e_t, ws, dev)
    e2e_val = reduce_sum(float(wl["pairs"]) * e2e_steps, ws, dev) / e2e_max / 1e9
    npipe = g6.L.g6_npipes()
    nchunks = sum((len(x) + npipe - 1) // npipe for x in sets)
    h2d = nact * (ffi.G6IREC.itemsize + ffi.G6PTCL.itemsize + 4) + nchunks * 16 + len(sets) * 0
    d2h = nact * ffi.G6OUT.itemsize

    pk = peaks()
    sm_mhz = clk.get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
    fp32_peak_tf = SM_COUNT * FP32_LANES * 2 * sm_mhz * 1e6 / 1e12
    fp32_peak_max = SM_COUNT * FP32_LANES * 2 * pk.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    # roofline of the dominant kernel, on its largest launch (65536 x 65536), timed alone with CUDA
    # events on its stream; all 64 force launches together are reported beside it
    achieved_tf = big[2] * 60 / (big_ms / 1e3) / 1e12
    achieved_all_tf = kern_pairs * 60 / kern_s / 1e12
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_hermite(pgb, wl)
        # the FP64 check of the batched results of the largest call (the kernel configuration
        # that dominates the time), on every 64th of its active particles
        rows = d_out.cpu().numpy().view(ffi.G6OUT)
        c = int(np.argmax([len(x) for x in sets]))
        a0, a1 = int(off[c]), int(off[c + 1])
        sel = np.arange(a0, a1, max(1, (a1 - a0) // 1024))
        xp_c, vp_c = predict_np(wl["t_calls"][c], st)
        cpu["fp64_check"] = fp64_check_g6(rows[sel], wl["xi"][sel], wl["vi"][sel],
                                          st.idx[wl["set_idx"][sel]], st.eps2, xp_c, vp_c, st.mass, st.idx)
        cpu["fp64_check"]["call"] = f"call {c} ({a1 - a0} active x {n} j), every {max(1, (a1 - a0) // 1024)}th active particle"
    for p_ in plans:
        g6.plan_destroy(p_)
    del graph
    line = {
        "metric": "Gint/s (PG6 Hermite force+jerk+pot+NN, batched)",
        "value": round(value, 2),
        "unit": "Gint/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_max / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (f64 predictor, " + ("double-float" if ff else "f64") + " x_j-x_i, f64 cross-tile sums)",
        "data": "synthetic (seeded Plummer, DF velocities; no dataset)",
        "config": {"workload": "PG6 Hermite N=65536 Plummer eps=1e-4, 64 block-step calls of 2^k active "
                               "(k=4..16), force+jerk+pot+nearest neighbour",
                   "pairs_per_step": wl["pairs"], "flop_per_pair": 60, "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"replicas x{ws} (independent schedules, no data-path collective)",
                   "graph": "64 x (predict + persistent force launch) in one CUDA graph",
                   "relative_coordinates": "double-float (hi+lo FP32)" if ff else "FP64 subtract + F2F"},
        "frac_fp32": round(value * 1e9 * 60 / 1e12 / fp32_peak_tf, 4),
        "roofline": {"bound": "fp32", "achieved": round(achieved_tf, 2), "peak": round(fp32_peak_tf, 2),
                     "unit": "TFLOP/s", "frac": round(achieved_tf / fp32_peak_tf, 4),
                     "traffic": PROFILED_TRAFFIC["hermite"]["bytes"] if ff else None,
                     "traffic_source": PROFILED_TRAFFIC["hermite"]["source"] if ff else None,
                     "kernel": "pgb::g6_kernel (autotuned configuration), largest call of the step "
                               f"({big[2]:.3e} pairs, {big_ms:.3f} ms)",
                     "achieved_all_launches": round(achieved_all_tf, 2),
                     "peak_source": f"148 SM x 128 FP32 lanes x 2 x median SM clock {sm_mhz:.0f} MHz sampled "
                                    f"in the timed region ({fp32_peak_max:.1f} TFLOP/s at sm_max_mhz)"},
        "e2e": {"value": round(e2e_val, 2), "unit": "Gint/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "api": "GRAPE-6 drop-in (g6_set_ti, g6calc_firsthalf, "
                "g6calc_lasthalf2p per npipes chunk, g6_set_j_particle of the active set), host buffers",
                "npipes": npipe, "steps": e2e_steps},
        "gpu_launches": args.steps * 2 * len(sets),
        "autotune": {str(k): int(v) for k, v in sorted(tuned.items())},
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    return line


# ----------------------------------------------------------------------------------------
# other workloads (PG5 direct, PG5 table / TreePM, independent Hermite clusters)

def _err_stats(got, ref, vec=True):
    """rms and max relative error of got against ref (per row for vectors)."""
    if vec:
        e = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    else:
        e = np.abs(got - ref) / np.abs(ref)
    return {"rms": float(np.sqrt(np.mean(e * e))), "max": float(e.max())}


def fp64_check_g6(out_rows, xi, vi, idi, eps2, xj, vj, mj, idj, jadr_base=0):
    """Hermite results (G6OUT rows) against the FP64 oracle on the same inputs: acc, jerk and pot
    errors, and NN index mismatches where the FP64 first and second neighbours differ by
    > 1e-5 (relative, in r^2).  The GRAPE-6 path carries velocities and masses as float.
    jadr_base: j address of xj[0] in the launch (the NN result is an absolute j address)."""
    from oracle import oracle as O
    f = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    ref = O.g6_force(xi, f(vi), idi, np.float32(eps2), xj, f(vj), f(mj), idj)
    acc = np.stack([out_rows["ax"], out_rows["ay"], out_rows["az"]], 1)
    jrk = np.stack([out_rows["jx"], out_rows["jy"], out_rows["jz"]], 1)
    clear = ref["r2nn2"] / ref["r2nn"] - 1.0 > 1e-5
    nn = out_rows["jadr"].astype(np.int64) - jadr_base
    nn_id = np.where((nn >= 0) & (nn < len(idj)), idj[np.clip(nn, 0, len(idj) - 1)], -1)
    return {"acc": _err_stats(acc, ref["acc"]), "jerk": _err_stats(jrk, ref["jrk"]),
            "pot": _err_stats(out_rows["pot"], ref["pot"], vec=False),
            "nn_mismatch": int(np.sum(nn_id[clear] != ref["nnb"][clear])), "particles": int(len(xi)),
            "oracle": "FP64 direct sum on the same inputs (oracle/pg_oracle.c)"}


def _timed_launches(torch, s, launch, steps, warmup, flush):
    for _ in range(warmup):
        with torch.cuda.stream(s):
            launch()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        with torch.cuda.stream(s):
            ev[k][0].record(s)
            launch()
            ev[k][1].record(s)
            flush.fill_(k & 0xFF)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) / 1e3 for a, b in ev]


def _line(args, ws, metric, value, t_step, pairs, flop, workload, dtype, achieved_tf, clk, e2e, cpu, launches,
          extra=None, kernel=""):
    traffic, tsrc = profiled_traffic(args.workload, pairs)
    pk = peaks()
    sm_mhz = clk.get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
    peak_tf = SM_COUNT * FP32_LANES * 2 * sm_mhz * 1e6 / 1e12
    line = {
        "metric": metric, "value": round(value, 2), "unit": "Gint/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_step * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded; no dataset)",
        "config": {"workload": workload, "pairs_per_step": pairs, "flop_per_pair": flop,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{ws}"},
        "frac_fp32": round((value * 1e9 * flop / 1e12 if isinstance(flop, (int, float)) else achieved_tf) / peak_tf, 4),
        "roofline": {"bound": "fp32", "achieved": round(achieved_tf, 2), "peak": round(peak_tf, 2), "unit": "TFLOP/s",
                     "frac": round(achieved_tf / peak_tf, 4), "traffic": traffic, "traffic_source": tsrc,
                     "kernel": kernel,
                     "peak_source": f"148 SM x 128 FP32 lanes x 2 x median SM clock {sm_mhz:.0f} MHz"},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk, "cpu_baseline": cpu,
    }
    if extra:
        line.update(extra)
    return line


def run_direct(args, pgb, ws, rank, local):
    """PG5 newton direct sum, N=16384 Plummer (eps=0.01), all i against all j (38 flop/pair)."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W = pgb.workloads
    g5 = pgb.ffi.G5()
    g5.L.g5_open()
    st = W.plummer_g5(16384, seed=W.SEED0 + rank)
    n = len(st.m)
    ipos = np.concatenate([st.x, np.full((n, 1), st.eps ** 2)], 1).astype(np.float32)
    jpos = np.concatenate([st.x, st.m[:, None]], 1).astype(np.float32)
    d_i = torch.from_numpy(ipos).to(dev)
    d_j = torch.from_numpy(jpos).to(dev)
    d_o = torch.zeros((n, 4), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    plan = g5.plan_create(g5.NEWTON, [[0, n, 0, n]])
    s = torch.cuda.Stream(device=dev)
    if not args.no_tune and not args.profile_largest:
        g5.plan_tune(plan, d_i.data_ptr(), d_j.data_ptr(), None, d_o.data_ptr(), s.cuda_stream)
    dcfg = g5.L.pgb5_plan_config(plan)
    launch = lambda: g5.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), None, d_o.data_ptr(), s.cuda_stream)  # noqa
    if args.profile_largest:
        # profiling target: the evaluation's force launch four times; no timing
        for _ in range(4):
            launch()
        s.synchronize()
        g5.plan_destroy(plan)
        return {"profile": "PG5 direct evaluation", "n": n, "launches": 4}
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    # one evaluation takes ~0.2 ms: at least 2000 of them, so that the clock sampler (every
    # 200 ms) sees the timed region
    ts = _timed_launches(torch, s, launch, max(args.steps, 2000), args.warmup, flush)
    barrier(ws)
    clk = clocks.stop()
    t_local = sum(ts)
    t_max = reduce_max(t_local, ws, dev)
    pairs = n * n
    value = reduce_sum(float(pairs) * len(ts), ws, dev) / t_max / 1e9
    achieved = pairs * len(ts) * 38 / t_local / 1e12
    drv = Driver(pgb)
    h = drv.L.g5drv_open(pgb.ffi.lib_path("libpg5.so").encode())
    acc = np.zeros((n, 3))
    pot = np.zeros(n)
    x = np.ascontiguousarray(st.x)
    m = np.ascontiguousarray(st.m)
    drv.L.g5drv_direct(h, n, Driver.p(x), Driver.p(m), st.eps, Driver.p(acc), Driver.p(pot))
    e2e_t = sum(drv.L.g5drv_direct(h, n, Driver.p(x), Driver.p(m), st.eps, Driver.p(acc), Driver.p(pot))
                for _ in range(args.e2e_steps * 5))
    e2e_val = reduce_sum(float(pairs) * args.e2e_steps * 5, ws, dev) / reduce_max(e2e_t, ws, dev) / 1e9
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        path = ref_lib("libpg5_ref.so")
        if path:
            hr = drv.L.g5drv_open(path.encode())
            drv.L.g5drv_direct(hr, n, Driver.p(x), Driver.p(m), st.eps, Driver.p(acc), Driver.p(pot))
            reps = 3
            tr = sum(drv.L.g5drv_direct(hr, n, Driver.p(x), Driver.p(m), st.eps, Driver.p(acc), Driver.p(pot))
                     for _ in range(reps))
            cpu = {"value": pairs * reps / tr / 1e9, "unit": "Gint/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"{reps} full evaluations, PG5/newton/libpg5 AVX2 + OpenMP (g5_calculate_force_on_x)"}
        from oracle import oracle as O
        smp = np.sort(W.Rng(1024).permutation(n)[:1024])
        f64 = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
        ao, po = O.g5_newton(f64(ipos[smp, :3]), f64(ipos[smp, 3]), f64(jpos[:, :3]), f64(jpos[:, 3]))
        og = d_o.cpu().numpy()[smp]
        if cpu is None:
            cpu = {}
        cpu["fp64_check"] = {"acc": _err_stats(og[:, :3], ao), "pot": _err_stats(-og[:, 3], po, vec=False),
                             "particles": 1024, "oracle": "FP64 direct sum on the same float32 inputs"}
    g5.plan_destroy(plan)
    return _line(args, ws, "Gint/s (PG5 newton direct sum, batched)", value, t_max / len(ts), pairs, 38,
                 "PG5 newton N=16384 Plummer eps=0.01, all i vs all j (acc + pot)", "f32 (f64 cross-tile sums)",
                 achieved, clk,
                 {"value": round(e2e_val, 2), "unit": "Gint/s", "h2d_bytes_per_step": n * 16 * 2,
                  "d2h_bytes_per_step": n * 32, "api": "g5_set_xmj + g5_set_eps_to_all + g5_set_n + "
                  "g5_calculate_force_on_x (direct.c:133-176), host buffers"},
                 cpu, len(ts), extra={"steps": len(ts)},
                 kernel=f"pgb::g5_kernel<NEWTON,{G5_CFG_NAMES[dcfg]}> (autotuned)")


def run_clusters(args, pgb, ws, rank, local):
    """1024 independent Plummer clusters, N log-uniform in [256, 16384], one Hermite force+jerk+pot+NN
    evaluation each: one batched launch vs 1024 sequences of plain g6 calls."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W = pgb.workloads
    ffi = pgb.ffi
    g6 = ffi.G6()
    g6.L.g6_open(0)
    cs = W.cluster_set(seed=W.SEED0 + 4 + rank)
    n = len(cs.mass)
    idx = np.arange(n, dtype=np.int32)
    irec = ffi.g6_irecords(cs.pos, cs.vel, idx)
    jrec = ffi.g6_jrecords(cs.pos, cs.vel, cs.mass, idx)
    d_i = torch.from_numpy(irec.view(np.uint8)).to(dev)
    d_j = torch.from_numpy(jrec.view(np.uint8)).to(dev)
    d_o = torch.zeros(n * ffi.G6OUT.itemsize, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    items = np.stack([cs.offsets[:-1], cs.sizes, cs.offsets[:-1], cs.sizes], 1)
    plan = g6.plan_create(items, nn=True)
    s = torch.cuda.Stream(device=dev)
    launch = lambda: g6.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), cs.eps2, d_o.data_ptr(), s.cuda_stream)  # noqa
    cfg = None
    if not args.no_tune:
        cfg, _ = g6.plan_tune(plan, d_i.data_ptr(), d_j.data_ptr(), cs.eps2, d_o.data_ptr(), s.cuda_stream)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    ts = _timed_launches(torch, s, launch, args.steps, args.warmup, flush)
    barrier(ws)
    clk = clocks.stop()
    t_local = sum(ts)
    t_max = reduce_max(t_local, ws, dev)
    pairs = int((cs.sizes.astype(np.int64) ** 2).sum())
    value = reduce_sum(float(pairs) * len(ts), ws, dev) / t_max / 1e9
    achieved = pairs * len(ts) * 60 / t_local / 1e12
    # plain: 1024 x (g6_set_j_particle x N_k, g6_set_ti, npipes chunks of firsthalf/lasthalf2p)
    drv = Driver(pgb)
    p = Driver.p
    drv.L.g6drv_clusters.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double] + \
        [C.POINTER(C.c_double)] * 3 + [C.POINTER(C.c_int), C.POINTER(C.c_float)]
    drv.L.g6drv_clusters.restype = C.c_double
    offs = cs.offsets.astype(np.int32)
    pos, vel, mass = (np.ascontiguousarray(a) for a in (cs.pos, cs.vel, cs.mass))
    h = drv.g6_open(pgb.ffi.lib_path("libpg6.so"))
    drv.L.g6drv_clusters(h, 0, 8, p(offs, C.c_int), p(pos), p(vel), p(mass), cs.eps2, None, None, None, None, None)
    e2e_t = drv.L.g6drv_clusters(h, 0, len(cs.sizes), p(offs, C.c_int), p(pos), p(vel), p(mass), cs.eps2,
                                 None, None, None, None, None)
    e2e_val = reduce_sum(float(pairs), ws, dev) / reduce_max(e2e_t, ws, dev) / 1e9
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        path = ref_lib("libpg6_ref.so")
        if path:
            hr = drv.g6_open(path)
            # bounded sample: the first clusters up to ~4e9 pairs
            cum = np.cumsum(cs.sizes.astype(np.int64) ** 2)
            ncl = int(np.searchsorted(cum, 4e9) + 1)
            drv.L.g6drv_clusters(hr, 0, 2, p(offs, C.c_int), p(pos), p(vel), p(mass), cs.eps2, None, None, None,
                                 None, None)
            tr = drv.L.g6drv_clusters(hr, 0, ncl, p(offs, C.c_int), p(pos), p(vel), p(mass), cs.eps2, None, None,
                                      None, None, None)
            cpu = {"value": float(cum[ncl - 1]) / tr / 1e9, "unit": "Gint/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": f"first {ncl} of 1024 clusters ({cum[ncl - 1]:.3e} pairs), "
                   "PG6/libpg6 AVX2 + OpenMP through the same plain call sequence"}
        # FP64 check of the batched results of every 64th cluster
        rows = d_o.cpu().numpy().view(ffi.G6OUT)
        ck = {"acc": [], "jerk": [], "pot": [], "nn": 0, "n": 0}
        nsel = 0
        for k in range(0, len(cs.sizes), 64):
            o, m_ = int(cs.offsets[k]), int(cs.sizes[k])
            sl = slice(o, o + m_)
            r = fp64_check_g6(rows[sl], cs.pos[sl], cs.vel[sl], idx[sl], cs.eps2, cs.pos[sl], cs.vel[sl],
                              cs.mass[sl], idx[sl], jadr_base=o)
            for key in ("acc", "jerk", "pot"):
                ck[key].append((r[key]["rms"] ** 2 * r["particles"], r[key]["max"]))
            ck["nn"] += r["nn_mismatch"]
            ck["n"] += r["particles"]
            nsel += 1
        if cpu is None:
            cpu = {}
        cpu["fp64_check"] = {key: {"rms": float(np.sqrt(sum(a for a, _ in ck[key]) / ck["n"])),
                                   "max": float(max(b for _, b in ck[key]))} for key in ("acc", "jerk", "pot")}
        cpu["fp64_check"].update({"nn_mismatch": ck["nn"], "particles": ck["n"],
                                  "clusters": f"every 64th of 1024 ({nsel})",
                                  "oracle": "FP64 direct sum on the same inputs (oracle/pg_oracle.c)"})
    g6.plan_destroy(plan)
    return _line(args, ws, "Gint/s (independent Hermite clusters, batched)", value, t_max / len(ts), pairs, 60,
                 "1024 Plummer clusters, N log-uniform [256,16384], eps=1e-4, one force+jerk+pot+NN each",
                 "f32 (double-float x_j-x_i, f64 cross-tile sums)", achieved, clk,
                 {"value": round(e2e_val, 3), "unit": "Gint/s", "h2d_bytes_per_step": n * (128 + 48),
                  "d2h_bytes_per_step": n * 64, "api": "plain GRAPE-6 calls per cluster (g6_set_j_particle x N_k, "
                  "g6_set_ti, g6calc_firsthalf/lasthalf2p per npipes), host buffers"},
                 cpu, len(ts), extra={"autotune": cfg, "batched_vs_plain": round(value / e2e_val, 1)},
                 kernel="pgb::g6_kernel (autotuned configuration)")


def split_force_np(r, ts_):
    """The analytic TreePM force shape (workloads.gaussian_split_force) on an array of r."""
    from scipy.special import erfc
    rs, eps = ts_.rs, ts_.eps
    g = erfc(r / (2.0 * rs)) + r / (np.sqrt(np.pi) * rs) * np.exp(-r * r / (4.0 * rs * rs))
    return np.where(r >= ts_.rcut * (1.0 - 1e-6), 0.0, g / (r * r + eps * eps) ** 1.5)


def run_treepm(args, pgb, ws, rank, local):
    """PG5 table cutoff force (TreePM PP part): N=2^20 uniform periodic box, 1024-entry table,
    4096 i-groups of 203-325 particles with their j-lists (4.0-4.5k entries) in one launch."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W = pgb.workloads
    tab = pgb.ffi.G5Table()
    ts_ = W.treepm_groups(seed=W.SEED0 + 2 + rank)
    f = W.gaussian_split_force(ts_.rs, ts_.rcut, ts_.eps)
    tab.set_table(f, ts_.rcut, frc_bit=6)
    _, xs = tab.table()
    # table units: j in float arithmetic as g5_set_xmj does, i through double as g5_set_xi does
    ip = np.zeros((len(ts_.xi), 4), np.float32)
    ip[:, :3] = (ts_.xi.astype(np.float32).astype(np.float64) * xs).astype(np.float32)
    jp = np.zeros((len(ts_.xj), 4), np.float32)
    jp[:, :3] = ts_.xj.astype(np.float32) * np.float32(xs)
    jp[:, 3] = ts_.mj
    d_i = torch.from_numpy(ip).to(dev)
    d_j = torch.from_numpy(jp).to(dev)
    d_o = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    plan = tab.plan_create(ts_.items)
    s = torch.cuda.Stream(device=dev)
    tcfg = None
    if not args.no_tune and not args.profile_largest:
        tcfg, _ = tab.plan_tune(plan, d_i.data_ptr(), d_j.data_ptr(), d_o.data_ptr(), s.cuda_stream)
    tcfg = tab.L.pgb5_plan_config(plan)
    launch = lambda: tab.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), d_o.data_ptr(), s.cuda_stream)  # noqa
    if args.profile_largest:
        # profiling target: the batch's launch four times (configuration: PGB_G5_CFG or the default)
        for _ in range(4):
            launch()
        s.synchronize()
        tab.plan_destroy(plan)
        return {"profile": "PG5 table TreePM batch", "config": G5_CFG_NAMES[tcfg], "launches": 4}
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    tms = _timed_launches(torch, s, launch, args.steps, args.warmup, flush)
    barrier(ws)
    clk = clocks.stop()
    t_local = sum(tms)
    t_max = reduce_max(t_local, ws, dev)
    pairs = ts_.interactions
    value = reduce_sum(float(pairs) * len(tms), ws, dev) / t_max / 1e9
    achieved = pairs * len(tms) * 38 / t_local / 1e12
    drv = Driver(pgb)
    p = Driver.p
    items = np.ascontiguousarray(ts_.items, np.int32)
    xi, xj, mj = (np.ascontiguousarray(a) for a in (ts_.xi, ts_.xj, ts_.mj))
    acc = np.zeros((len(xi), 3))
    pot = np.zeros(len(xi))
    h = drv.L.g5drv_open(pgb.ffi.lib_path("libpg5table.so").encode())
    tab.set_table(f, ts_.rcut, frc_bit=6)    # this process's library instance is the same .so
    nthr = min(os.cpu_count() or 1, 16)
    drv.L.g5drv_groups(h, 16, p(items, C.c_int), p(xi), p(xj), p(mj), 0.0, p(acc), p(pot), nthr)
    e2e_t = drv.L.g5drv_groups(h, len(items), p(items, C.c_int), p(xi), p(xj), p(mj), 0.0, p(acc), p(pot), nthr)
    e2e_val = reduce_sum(float(pairs), ws, dev) / reduce_max(e2e_t, ws, dev) / 1e9
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        path = ref_lib("libpg5table_ref.so")
        if path:
            hr = drv.L.g5drv_open(path.encode())
            # the same force shape in the reference's table (dlopen of the same file: same instance)
            Lr = C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
            Lr.pg5_gen_force_table.argtypes = [C.c_void_p, C.c_double]
            cb = pgb.ffi.FORCE_FN(f)
            Lr.pg5_gen_force_table(C.cast(cb, C.c_void_p), ts_.rcut)
            ng = 1024
            tr = drv.L.g5drv_groups(hr, ng, p(items, C.c_int), p(xi), p(xj), p(mj), 0.0, p(acc), p(pot),
                                    min(os.cpu_count() or 1, 24))
            sp = int((items[:ng, 1].astype(np.int64) * items[:ng, 3]).sum())
            cpu = {"value": sp / tr / 1e9, "unit": "Gint/s", "cores": min(os.cpu_count() or 1, 24),
                   "kind": "reference", "sample": f"first {ng} of {len(items)} groups ({sp:.3e} pairs), "
                   "PG5/table/libpg5 (512-entry table: the table size is fixed at compile time there), "
                   "OpenMP over groups with g5_*MC(devid) as source.cpp does"}
        # FP64 check: the same table and lerp evaluated in FP64 on every 64th group's inputs, and
        # the table's own error against the analytic force shape on the same pairs
        from oracle import oracle as O
        tab.set_table(f, ts_.rcut, frc_bit=6)
        t_, _ = tab.table()
        og = d_o.cpu().numpy()
        got, ref, ana = [], [], []
        for k in range(0, len(ts_.items), 64):
            i0, ni_, j0, nj_ = (int(v) for v in ts_.items[k])
            xi_ = ip[i0:i0 + ni_, :3].astype(np.float64) / xs
            xj_ = jp[j0:j0 + nj_, :3].astype(np.float64) / xs
            ref.append(O.g5_table(xi_, xj_, ts_.mj[j0:j0 + nj_], t_, 4, 6, xs))
            got.append(og[i0:i0 + ni_, :3])
            d = xj_[None, :, :] - xi_[:, None, :]
            r = np.sqrt((d * d).sum(2))
            ana.append((ts_.mj[j0:j0 + nj_][None, :, None] * d * split_force_np(r, ts_)[:, :, None]).sum(1))
        got, ref, ana = np.concatenate(got), np.concatenate(ref), np.concatenate(ana)
        if cpu is None:
            cpu = {}
        cpu["fp64_check"] = {"acc": _err_stats(got, ref), "table_vs_analytic_acc": _err_stats(ref, ana),
                             "particles": int(len(got)),
                             "oracle": "FP64 evaluation of the same 1024-entry table and lerp on the same inputs"}
    tab.plan_destroy(plan)
    return _line(args, ws, "Gint/s (PG5 table cutoff force, TreePM PP, batched)", value, t_max / len(tms), pairs, 38,
                 "PG5 table N=2^20 uniform periodic box, 1024-entry Gaussian-split table, 4096 i-groups",
                 "f32 (f64 cross-tile sums)", achieved, clk,
                 {"value": round(e2e_val, 2), "unit": "Gint/s",
                  "h2d_bytes_per_step": int(len(xj) * 16 + len(xi) * 16), "d2h_bytes_per_step": int(len(xi) * 32),
                  "api": f"per group g5_set_xmjMC + g5_set_nMC + g5_calculate_force_on_xMC, {nthr} host threads "
                         "(one devid each), host buffers"},
                 cpu, len(tms), kernel=f"pgb::g5_kernel<TABLE,{G5_CFG_NAMES[tcfg]}> (autotuned)")


def run_bh(args, pgb, ws, rank, local):
    """Barnes-Hut with quadrupole cells (newton_quad): N = 2^22 Hernquist sphere, theta = 0.5,
    groups of <= 256, leaves of <= 16 particles; per evaluation one index-list launch over every
    group's point-mass list (PG5 newton, 38 flop/pair) and one over every group's cell list
    (quadrupole kernel, 60 flop/pair)."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W = pgb.workloads
    g5 = pgb.ffi.G5()
    g5.L.g5_open()
    if args.profile_tree:
        # profiling target: the GPU tree of the workload's particles built twice; no timing
        rng = W.Rng(W.SEED0 + 3 + rank)
        x = W._isotropic(rng, W.hernquist_radii(rng, args.bh_n, 100.0)).astype(np.float32).astype(np.float64)
        m = np.full(args.bh_n, np.float32(1.0 / args.bh_n), np.float64)
        for _ in range(2):
            W.GpuTree(x, m, 0.5, 16, 256).close()
        return {"profile": "GPU tree build", "n": args.bh_n, "builds": 2}
    bh = W.bh_hernquist(args.bh_n, seed=W.SEED0 + 3 + rank)
    ip, pp, cp, cq = bh.records()
    d_i, d_p = torch.from_numpy(ip).to(dev), torch.from_numpy(pp).to(dev)
    d_c, d_q = torch.from_numpy(cp).to(dev), torch.from_numpy(cq).to(dev)
    d_pi, d_ci = torch.from_numpy(bh.pidx).to(dev), torch.from_numpy(bh.cidx).to(dev)
    o_p = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    o_c = torch.zeros((len(ip), 4), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    s = torch.cuda.Stream(device=dev)
    pl_p = g5.plan_create(g5.NEWTON, bh.items("p"))
    pl_c = g5.plan_create(g5.QUAD, bh.items("c"))
    args_p = (d_i.data_ptr(), d_p.data_ptr(), None, d_pi.data_ptr(), o_p.data_ptr(), s.cuda_stream)
    args_c = (d_i.data_ptr(), d_c.data_ptr(), d_q.data_ptr(), d_ci.data_ptr(), o_c.data_ptr(), s.cuda_stream)
    if not args.no_tune and not args.profile_largest:
        g5.plan_tune_indexed(pl_p, *args_p)
        g5.plan_tune_indexed(pl_c, *args_c)
    cfg_p, cfg_c = g5.L.pgb5_plan_config(pl_p), g5.L.pgb5_plan_config(pl_c)
    if args.profile_largest:
        # profiling target: (point-mass launch, cell launch) twice (configuration: PGB_G5_CFG or
        # the default)
        for _ in range(2):
            g5.plan_launch_indexed(pl_p, *args_p)
            g5.plan_launch_indexed(pl_c, *args_c)
        s.synchronize()
        g5.plan_destroy(pl_p)
        g5.plan_destroy(pl_c)
        return {"profile": "Barnes-Hut batch", "config": [G5_CFG_NAMES[cfg_p], G5_CFG_NAMES[cfg_c]], "launches": 4}

    def launch():
        g5.plan_launch_indexed(pl_p, *args_p)
        g5.plan_launch_indexed(pl_c, *args_c)

    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        launch()   # outside capture once (lazy module loading)
    torch.cuda.synchronize()
    with torch.cuda.graph(graph, stream=s):
        launch()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(ws)
    tms = _timed_launches(torch, s, graph.replay, args.steps, args.warmup, flush)
    barrier(ws)
    clk = clocks.stop()
    t_local = sum(tms)
    t_max = reduce_max(t_local, ws, dev)
    pairs = bh.p_pairs + bh.c_pairs
    value = reduce_sum(float(pairs) * len(tms), ws, dev) / t_max / 1e9
    flops = bh.p_pairs * 38 + bh.c_pairs * 60
    achieved = flops * len(tms) / t_local / 1e12
    # each kind's launch alone (CUDA events on its stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    with torch.cuda.stream(s):
        ev[0].record(s)
        g5.plan_launch_indexed(pl_p, *args_p)
        ev[1].record(s)
        g5.plan_launch_indexed(pl_c, *args_c)
        ev[2].record(s)
    torch.cuda.synchronize()
    ms_p, ms_c = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    acc_b = (o_p[:, :3] + o_c[:, :3]).cpu().numpy()
    phi_b = (o_p[:, 3] - o_c[:, 3]).cpu().numpy()
    del graph

    # end to end through the batched API with host buffers: every step copies the records and
    # both index lists from pinned host memory, launches both plans and reads both results back
    h_in = [torch.from_numpy(a).pin_memory() for a in (ip, pp, cp, cq, bh.pidx, bh.cidx)]
    d_in = [d_i, d_p, d_c, d_q, d_pi, d_ci]
    h_out = [torch.empty_like(o_p, device="cpu").pin_memory() for _ in range(2)]
    e2e_ms = []
    for k in range(args.warmup + args.e2e_steps):
        a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            a_.record(s)
            for d_, h_ in zip(d_in, h_in):
                d_.copy_(h_, non_blocking=True)
            launch()
            h_out[0].copy_(o_p, non_blocking=True)
            h_out[1].copy_(o_c, non_blocking=True)
            b_.record(s)
        s.synchronize()
        if k >= args.warmup:
            e2e_ms.append(a_.elapsed_time(b_))
    e2e_val = reduce_sum(float(pairs) * len(e2e_ms), ws, dev) / reduce_max(sum(e2e_ms) / 1e3, ws, dev) / 1e9
    h2d = sum(t.numel() * t.element_size() for t in h_in)
    d2h = sum(t.numel() * t.element_size() for t in h_out)

    # a whole tree-code step through this repository's API, from particles in host memory to
    # forces in host memory: the tree, moments, groups and lists built on the GPU
    # (lib/libpgbtree.so), both plans created from its group table, both launches, both results
    # read back -- every step; host clock
    # the step's inputs in pinned host memory (input order), as a code would keep its particles
    x_in = torch.empty(bh.x.shape, dtype=torch.float64).pin_memory().numpy()
    m_in = torch.empty(bh.m.shape, dtype=torch.float64).pin_memory().numpy()
    x_in[bh.perm], m_in[bh.perm] = bh.x, bh.m
    t0 = time.perf_counter()
    W.bh_tree(x_in, m_in, bh.theta, bh.nleaf, bh.ncrit, bh.eps)
    host_build_s = time.perf_counter() - t0
    d_i2 = torch.empty_like(d_i)
    s2 = torch.cuda.Stream(device=dev)
    ev_p = torch.cuda.Event()
    step_s, build_ms, same = [], [], True
    tr = q_p = q_c = None
    for k in range(args.warmup + args.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if tr is None:
            tr = W.GpuTree(x_in, m_in, bh.theta, bh.nleaf, bh.ncrit, bh.eps)
        else:
            tr.rebuild(x_in, m_in)    # a code that steps rebuilds its tree object
        dv = tr.device()
        it_p, it_c = tr.items()
        tr.irecords(bh.eps * bh.eps, d_i2.data_ptr())
        # one plan per kind for the run (the tuned configurations pinned at creation), given the
        # step's lists by pgb5_plan_update
        if q_p is None:
            q_p = g5.plan_create(g5.NEWTON, it_p)
            g5.L.pgb5_plan_set_config(q_p, cfg_p)
        else:
            g5.plan_update(q_p, it_p)
        g5.plan_launch_indexed(q_p, d_i2.data_ptr(), dv["part"], None, dv["pidx"], o_p.data_ptr(), s.cuda_stream)
        ev_p.record(s)
        # the cell plan is made on the host while the point-mass launch runs
        if q_c is None:
            q_c = g5.plan_create(g5.QUAD, it_c)
            g5.L.pgb5_plan_set_config(q_c, cfg_c)
        else:
            g5.plan_update(q_c, it_c)
        g5.plan_launch_indexed(q_c, d_i2.data_ptr(), dv["cell"], dv["cquad"], dv["cidx"], o_c.data_ptr(),
                               s.cuda_stream)
        s2.wait_event(ev_p)
        with torch.cuda.stream(s2):
            h_out[0].copy_(o_p, non_blocking=True)    # read back while the cell launch runs
        with torch.cuda.stream(s):
            h_out[1].copy_(o_c, non_blocking=True)
        s.synchronize()
        s2.synchronize()
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            step_s.append(dt)
            build_ms.append(tr.build_ms)
    g5.plan_destroy(q_p)
    g5.plan_destroy(q_c)
    tr.close()
    same = bool(np.array_equal((h_out[0][:, :3] + h_out[1][:, :3]).numpy(), acc_b))
    tree_val = reduce_sum(float(pairs) * len(step_s), ws, dev) / reduce_max(sum(step_s), ws, dev) / 1e9

    # the per-group drop-in calls with host buffers (source.cpp:813-866 call sequence)
    drv = Driver(pgb)
    p = Driver.p
    lp = C.POINTER(C.c_longlong)
    f64 = lambda a: np.ascontiguousarray(a, np.float64)  # noqa: E731
    xi, xp, mp = f64(ip[:, :3]), f64(pp[:, :3]), f64(pp[:, 3])
    cpos, cm, cqq = f64(cp[:, :3]), f64(cp[:, 3]), f64(cq[:, :6])
    acc = np.zeros((len(mp), 3))
    phi = np.zeros(len(mp))
    nthr = min(os.cpu_count() or 1, 32)

    def dropin(h, g0, g1, threads):
        return drv.L.g5drv_bh(h, g0, g1, p(bh.gfirst, C.c_int), p(bh.gcount, C.c_int), p(xi), p(xp), p(mp),
                              p(bh.poff, C.c_longlong), p(bh.pidx, C.c_int), p(cpos), p(cm), p(cqq),
                              p(bh.coff, C.c_longlong), p(bh.cidx, C.c_int), bh.eps, p(acc), p(phi), threads)

    h = drv.L.g5drv_open(pgb.ffi.lib_path("libpg5.so").encode())
    dropin(h, 0, min(64, bh.ngroups), nthr)   # warm-up
    dropin_t = dropin(h, 0, bh.ngroups, nthr)
    dropin_val = reduce_sum(float(pairs), ws, dev) / reduce_max(dropin_t, ws, dev) / 1e9
    dropin_rms = float(np.sqrt(np.mean(np.sum((acc - acc_b) ** 2, 1) / np.sum(acc_b ** 2, 1))))
    errors = {"dropin_vs_batched_rms": dropin_rms}
    if rank == 0 and ws == 1 and not args.no_errors and not args.no_cpu_baseline:
        from oracle import oracle as O
        # FP64 on the same lists and inputs (every 97th group), and the full FP64 direct sum
        # (multipole truncation) on 4096 sampled particles
        e1 = []
        for g in range(0, bh.ngroups, 97):
            sl = slice(bh.gfirst[g], bh.gfirst[g] + bh.gcount[g])
            pl = bh.pidx[bh.poff[g]:bh.poff[g + 1]]
            cl = bh.cidx[bh.coff[g]:bh.coff[g + 1]]
            a1, _ = O.g5_newton(xi[sl], float(ip[0, 3]), xp[pl], mp[pl])
            a2, _ = O.g5_quad(xi[sl], float(ip[0, 3]), cpos[cl], cm[cl], cqq[cl])
            ref = a1 + a2
            e1.append(np.linalg.norm(acc_b[sl] - ref, axis=1) / np.linalg.norm(ref, axis=1))
        e1 = np.concatenate(e1)
        smp = np.sort(W.Rng(4096).permutation(len(mp))[:4096])
        ad, _ = O.g5_newton(xi[smp], float(ip[0, 3]), xp, mp)
        e2 = np.linalg.norm(acc_b[smp] - ad, axis=1) / np.linalg.norm(ad, axis=1)
        errors.update({"same_lists_fp64": {"rms": float(np.sqrt(np.mean(e1 ** 2))), "max": float(e1.max()),
                                           "particles": int(len(e1))},
                       "direct_sum_fp64": {"rms": float(np.sqrt(np.mean(e2 ** 2))), "max": float(e2.max()),
                                           "particles": 4096}})
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        path = ref_lib("libquad_ref.so")
        if path:
            hr = drv.L.g5drv_open(path.encode())
            ng = min(bh.ngroups, 4000)
            cores = min(os.cpu_count() or 1, 128)
            tr = dropin(hr, 0, ng, cores)
            sp = int((bh.gcount[:ng].astype(np.int64) * (np.diff(bh.poff)[:ng] + np.diff(bh.coff)[:ng])).sum())
            cpu = {"value": sp / tr / 1e9, "unit": "Gint/s", "cores": cores, "kind": "reference",
                   "sample": f"first {ng} of {bh.ngroups} groups ({sp:.3e} pairs), PG5/newton_quad libraries "
                   "(libpg5 + quad, AVX2) built from their sources, OpenMP over groups with g5_*MC / g5c_*MC"}
    g5.plan_destroy(pl_p)
    g5.plan_destroy(pl_c)
    return _line(args, ws, "Gint/s (Barnes-Hut point masses + quadrupole cells, batched)", value, t_max / len(tms),
                 pairs, "38 (point mass) / 60 (quadrupole cell)", f"Barnes-Hut N={args.bh_n} Hernquist (a=1, r<=100) eps=1e-3, theta=0.5, ncrit=256, "
                 f"nleaf=16: {bh.ngroups} groups, {bh.p_pairs:.3e} point-mass + {bh.c_pairs:.3e} cell pairs",
                 "f32 (f64 cross-tile sums)", achieved, clk,
                 {"value": round(tree_val, 2), "unit": "Gint/s", "h2d_bytes_per_step": int(x_in.nbytes + m_in.nbytes),
                  "d2h_bytes_per_step": int(d2h), "steps": len(step_s),
                  "api": "whole step from host particles to host forces: pgbt_rebuild (octree, moments, groups, "
                         "lists on the GPU, the tree object reused) + pgbt_group_table + pgbt_irecords + "
                         "pgb5_plan_update x 2 (one plan per kind for the run; the cell plan made while the "
                         "point-mass launch runs) + pgb5_plan_launch_indexed x 2, both results read back (the "
                         "first while the second launch runs); host clock",
                  "forces_equal_batched": same,
                  "lists_copied": {"value": round(e2e_val, 2), "unit": "Gint/s", "h2d_bytes_per_step": int(h2d),
                                   "d2h_bytes_per_step": int(d2h), "steps": len(e2e_ms),
                                   "api": "pgb5_plan_launch_indexed x 2 with the host-built records and index lists "
                                          "copied from pinned host memory and both results read back every step"}},
                 cpu, 2 * len(tms),
                 extra={"dropin": {"value": round(dropin_val, 2), "unit": "Gint/s", "threads": nthr,
                                   "api": "per group g5_set_xmjMC + g5_set_nMC + g5_calculate_force_on_xMC and "
                                          "g5c_set_xmjMC + g5c_set_nMC + g5c_calculate_force_on_xMC, one devid per "
                                          "host thread, host buffers; list gathers inside the timed loop"},
                        "launch_ms": {"point_masses": round(ms_p, 3), "cells": round(ms_c, 3)},
                        "autotune": {"point_masses": G5_CFG_NAMES[cfg_p], "cells": G5_CFG_NAMES[cfg_c]},
                        "tree_build": {"gpu_ms": round(float(np.median(build_ms)), 2),
                                       "host_s": round(host_build_s, 2),
                                       "gpu": "lib/libpgbtree.so pgbt_rebuild of the step's tree object (device time, CUDA events)",
                                       "host": "drivers/pgb_bhtree.c bh_build (OpenMP lists)",
                                       "identical": "tests/test_bhtree_gpu.py"},
                        "errors": errors},
                 kernel=f"pgb::g5_kernel<NEWTON,{G5_CFG_NAMES[cfg_p]}> + <QUAD,{G5_CFG_NAMES[cfg_c]}> (index lists)")


# ----------------------------------------------------------------------------------------
# reference arm

INT_PARAMS = dict(epsinv=0.0, eta=0.2, eta_s=0.01, dtstarinv=8.0)   # PG6/banana/input.list defaults


def integrator_ics(pgb, n, rank=0):
    """Initial conditions of the integrator workload: a seeded Plummer sphere in Henon units (the
    units and shape of the reference's own PG6/banana/init/pl016k.init), equal masses 1/n."""
    W = pgb.workloads
    return W.plummer_henon(n, W.SEED0 + 31 + rank)


def write_banana_init(path, m, x, v):
    """The reference integrator's input format (PG6/banana/io.c:18-26): time, n, then per
    particle: index, mass, position, velocity."""
    with open(path, "w") as f:
        f.write(f"0.0\n{len(m)}\n")
        for i in range(len(m)):
            f.write(f"{i + 1}\n{m[i]:.17g}\n{x[i, 0]:.17g} {x[i, 1]:.17g} {x[i, 2]:.17g}\n"
                    f"{v[i, 0]:.17g} {v[i, 1]:.17g} {v[i, 2]:.17g}\n")


def run_banana(path, m, x, v, intervals, threads=None):
    """Run the reference's own Hermite integrator (oracle/_ref/banana01, PG6/banana built from its
    sources with -DNORMAL) from t = 0 for `intervals` output intervals of 1/8.  Returns the wall
    time of each interval (host clock at the arrival of its output line; line-buffered stdout),
    the particle steps and block steps of each, the energies, and the start-up time."""
    import re
    dts = 1.0 / INT_PARAMS["dtstarinv"]
    with tempfile.TemporaryDirectory() as d:
        init = os.path.join(d, "ics.init")
        write_banana_init(init, m, x, v)
        with open(os.path.join(d, "input.list"), "w") as f:
            f.write(f"0 {intervals * dts} 1000000\n{INT_PARAMS['epsinv']}\n"
                    f"{INT_PARAMS['eta']} {INT_PARAMS['eta_s']} {INT_PARAMS['dtstarinv']}\n{init}\nsnap\n")
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        cmd = ([ "stdbuf", "-oL"] if subprocess.run(["which", "stdbuf"], capture_output=True).returncode == 0
               else []) + [path]
        t0 = time.perf_counter()
        proc = subprocess.Popen(cmd, cwd=d, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env)
        stamps, lines = [], []
        for line in proc.stdout:
            lines.append(line)
            if line.startswith("Time:"):
                stamps.append(time.perf_counter() - t0)
        proc.wait()
        if proc.returncode != 0:
            raise RuntimeError(f"banana01 exited {proc.returncode}: {proc.stderr.read()[-500:]}")
    out = "".join(lines)
    st = re.findall(r"niave: ([0-9.e+-]+) ([0-9.e+-]+)", out)
    steps = [float(b) for _, b in st]
    blocks = [round(float(b) / float(a)) if float(a) > 0 else 0 for a, b in st]
    en = [float(e) for e in re.findall(r"^tot: ([-+0-9.]+)", out, re.M)]
    times = np.diff(stamps).tolist()
    return dict(times=times, steps=steps[1:], blocks=blocks[1:], energies=en, startup=stamps[0] if stamps else None,
                threads=threads or os.cpu_count())


def run_integrator(args, pgb, ws, rank, local):
    """PG6 Hermite block-time-step integration on the device (pgb6_hermite_*): the reference
    sample integrator's run (PG6/banana with its input.list: eps = 0, eta = 0.2, eta_s = 0.01,
    dtstar = 1/8) of an N = 16384 Plummer sphere; one step = one output interval of 1/8."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ffi = pgb.ffi
    g6 = ffi.G6()
    g6.L.g6_open(0)
    n = args.int_n
    x, v, m = integrator_ics(pgb, n, rank)
    eps2 = 0.0 if INT_PARAMS["epsinv"] == 0 else 1.0 / INT_PARAMS["epsinv"] ** 2
    dts = 1.0 / INT_PARAMS["dtstarinv"]
    H = ffi.Hermite(g6, m, x, v, eps2, INT_PARAMS["eta"], INT_PARAMS["eta_s"], dts)
    if args.profile_largest:
        # profiling target: the start-up step and two intervals of 1/8 (one launch each); no timing
        H.advance(dts)
        H.advance(2 * dts)
        torch.cuda.synchronize()
        H.close()
        return {"profile": "integrator launches", "n": n, "launches": 3}
    ek0, ew0 = H.energy()
    s = torch.cuda.ExternalStream(H.stream, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for k in range(args.warmup):
        H.advance((k + 1) * dts)
    torch.cuda.synchronize()
    fp0, tiles0 = H.stats()
    clocks = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks.start()
    barrier(ws)
    torch.cuda.synchronize()
    psteps = blocks = 0
    for k in range(args.steps):
        ev[k][0].record(s)
        p_, b_ = H.advance((args.warmup + k + 1) * dts)
        ev[k][1].record(s)
        with torch.cuda.stream(s):
            flush.fill_(k & 0xFF)   # 256 MiB write between steps: L2 (126 MB) flushed
        psteps += p_
        blocks += b_
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    t_local = sum(a.elapsed_time(b) for a, b in ev) / 1e3
    t_max = reduce_max(t_local, ws, dev)
    value = reduce_sum(float(psteps) * n, ws, dev) / t_max / 1e9
    fp1, tiles1 = H.stats()
    force_pairs = fp1 - fp0
    tiles = [b - a for a, b in zip(tiles0, tiles1)]
    ek, ew = H.energy()
    de = ((ek + ew) - (ek0 + ew0)) / abs(ek0 + ew0)
    H.close()

    # end to end through the C ABI with host buffers: create (upload + start-up step), the same
    # number of intervals from t = 0, the final state back to the host
    e2e_int = max(1, min(args.steps, args.e2e_steps))
    torch.cuda.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    H2 = ffi.Hermite(g6, m, x, v, eps2, INT_PARAMS["eta"], INT_PARAMS["eta_s"], dts)
    H2.advance(e2e_int * dts)
    st2 = H2.get()
    e2e_t = time.perf_counter() - t0
    p2, b2 = H2.counts()
    H2.close()
    e2e_val = reduce_sum(float(p2) * n, ws, dev) / reduce_max(e2e_t, ws, dev) / 1e9

    pk = peaks()
    sm_mhz = clk.get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
    fp32_peak_tf = SM_COUNT * FP32_LANES * 2 * sm_mhz * 1e6 / 1e12
    # the whole step runs in one persistent kernel: its roofline is the pair arithmetic over the
    # kernel's CUDA-event time (selection, prediction and corrector included)
    achieved_tf = force_pairs * 60 / t_local / 1e12
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        path = ref_lib("banana01")
        if path is None:
            cpu = {"value": None, "unit": "Gint/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": "unavailable: oracle/_ref/banana01 not built"}
        else:
            r = run_banana(path, m, x, v, 2)
            cpu = {"value": round(sum(r["steps"]) * n / sum(r["times"]) / 1e9, 3), "unit": "Gint/s",
                   "cores": r["threads"], "kind": "reference",
                   "sample": f"the first 2 intervals (t = 0 to 1/4: {int(sum(r['steps']))} particle steps, "
                             f"{sum(r['blocks'])} block steps, {sum(r['times']):.2f} s), PG6/banana with libpg6 "
                             "AVX2 + OpenMP built from the reference's sources",
                   "energies": r["energies"]}
    line = {
        "metric": "Gint/s (PG6 Hermite block-time-step integration: particle steps x N per second)",
        "value": round(value, 2), "unit": "Gint/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_max / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 integrator, f32 force (double-float x_j-x_i, f64 sums)",
        "data": "synthetic (seeded Plummer in Henon units; no dataset)",
        "config": {"workload": f"PG6 Hermite integration N={n} Plummer, eps=0, eta=0.2, eta_s=0.01, dtstar=1/8 "
                               "(PG6/banana input.list); one step = one interval of 1/8",
                   "particle_steps": psteps, "block_steps": blocks, "interactions": psteps * n,
                   "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"replicas x{ws} (independent systems, no data-path collective)",
                   "energy_error": de, "time": (args.warmup + args.steps) * dts},
        "roofline": {"bound": "fp32", "achieved": round(achieved_tf, 2), "peak": round(fp32_peak_tf, 2),
                     "unit": "TFLOP/s", "frac": round(achieved_tf / fp32_peak_tf, 4), "traffic": None,
                     "kernel": f"pgb::hm_run_kernel (one cooperative launch per interval: selection, prediction, "
                               f"force, corrector), {force_pairs:.3e} pairs in {t_local * 1e3:.2f} ms, 60 flop per "
                               "pair; block steps by force i-tile 16/32/64/128/512: " + "/".join(map(str, tiles)),
                     "peak_source": f"148 SM x 128 FP32 lanes x 2 x median SM clock {sm_mhz:.0f} MHz"},
        "e2e": {"value": round(e2e_val, 2), "unit": "Gint/s",
                "h2d_bytes_per_step": int(n * 56 / e2e_int), "d2h_bytes_per_step": int(n * 136 / e2e_int),
                "api": "pgb6_hermite_create (upload + start-up step) + pgb6_hermite_advance + "
                       "pgb6_hermite_get, host buffers, host clock", "steps": e2e_int,
                "particle_steps": p2, "block_steps": b2},
        "gpu_launches": args.steps,   # one cooperative launch of pgb::hm_run_kernel per interval
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    return line


def run_reference_integrator(args, pgb, ws, rank):
    path = ref_lib("banana01")
    if path is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/banana01 (the reference integrator) not built"}
    n = args.int_n
    x, v, m = integrator_ics(pgb, n)
    r = run_banana(path, m, x, v, args.warmup + args.steps)
    times = r["times"][args.warmup:]
    steps = r["steps"][args.warmup:]
    val = sum(steps) * n / sum(times) / 1e9
    return {
        "metric": "Gint/s (PG6 Hermite block-time-step integration: particle steps x N per second)",
        "value": round(val, 3), "unit": "Gint/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(sum(times) / len(times) * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 integrator, f32 force", "data": "synthetic",
        "config": {"workload": f"PG6 Hermite integration N={n} Plummer, eps=0, eta=0.2, eta_s=0.01, dtstar=1/8 "
                               "(PG6/banana input.list); one step = one interval of 1/8",
                   "particle_steps": int(sum(steps)), "block_steps": int(sum(r["blocks"][args.warmup:]))},
        "impl": "reference",
        "cpu_baseline": {"value": round(val, 3), "unit": "Gint/s", "cores": r["threads"], "kind": "reference",
                         "sample": f"intervals {args.warmup + 1}-{args.warmup + args.steps} of the run "
                                   "(PG6/banana banana01 + libpg6 AVX2 + OpenMP, built from the reference's "
                                   "sources; per-interval host time at its output lines)"},
        "e2e": {"value": round(val, 3), "unit": "Gint/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference(args, pgb, ws, rank):
    if rank != 0:
        return None
    if args.workload == "integrator":
        return run_reference_integrator(args, pgb, ws, rank)
    path = ref_lib("libpg6_ref.so")
    if path is None:
        return {"impl": "reference", "unavailable": "reference library (oracle/_ref/libpg6_ref.so) not built"}
    W = pgb.workloads
    drv = Driver(pgb)
    h = drv.g6_open(path)
    # same workload; a = j from an FP64-free source is not needed for timing: use the engine's
    # own force only if a GPU is present, else zero acc/jerk (prediction cost is the same)
    st = W.hermite_state(65536, seed=W.SEED0 + 1)
    sets = W.hermite_schedule(65536, 64, seed=W.SEED0 + 101)
    t_calls = st.t_now + np.arange(64) * 2.0 ** -20
    set_off = np.concatenate([[0], np.cumsum([len(s) for s in sets])]).astype(np.int32)
    set_idx = np.concatenate(sets).astype(np.int32)
    xi = np.empty((len(set_idx), 3))
    vi = np.empty((len(set_idx), 3))
    for c, s in enumerate(sets):
        x, v = predict_np(t_calls[c], st)
        xi[set_off[c]:set_off[c + 1]] = x[s]
        vi[set_off[c]:set_off[c + 1]] = v[s]
    wl = dict(st=st, sets=sets, t_calls=t_calls, set_off=set_off, set_idx=set_idx, xi=xi, vi=vi, n=65536)
    drv.g6_set_j(h, st)
    calls = cpu_sample_calls(wl, args.ref_pairs)
    for _ in range(args.warmup):
        drv.g6_schedule(h, wl, calls=calls)
    tot, pairs = 0.0, 0
    for _ in range(args.steps):
        sec, p_, _ = drv.g6_schedule(h, wl, calls=calls)
        tot += sec
        pairs += p_
    val = pairs / tot / 1e9
    sample = (f"first {calls} of the 64 block-step calls per step ({pairs // args.steps:.3e} pairs), "
              f"PG6/libpg6 AVX2 + OpenMP built from its own sources, npipes 48")
    return {
        "metric": "Gint/s (PG6 Hermite force+jerk+pot+NN, batched)",
        "value": round(val, 3), "unit": "Gint/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tot / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (f64 predictor + x_j-x_i)", "data": "synthetic",
        "config": {"workload": "PG6 Hermite N=65536 Plummer eps=1e-4, 64 block-step calls of 2^k active "
                               "(k=4..16), force+jerk+pot+nearest neighbour (sampled prefix)",
                   "flop_per_pair": 60},
        "impl": "reference",
        "cpu_baseline": {"value": round(val, 3), "unit": "Gint/s", "cores": os.cpu_count(), "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(val, 3), "unit": "Gint/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ----------------------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["hermite", "direct", "clusters", "treepm", "bh", "integrator"],
                    default="hermite")
    ap.add_argument("--int-n", type=int, default=16384, help="particles of the integrator workload")
    ap.add_argument("--bh-n", type=int, default=1 << 22, help="particles of the Barnes-Hut workload")
    ap.add_argument("--no-errors", action="store_true", help="bh: skip the FP64 error report")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--ref-pairs", type=float, default=4e9, help="pairs per reference-arm step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the kernel-configuration autotuner")
    ap.add_argument("--f64-positions", action="store_true",
                    help="FP64 x_j - x_i (DADD + F2F) instead of the double-float subtraction")
    ap.add_argument("--profile-largest", action="store_true",
                    help="profiling target: set up, warm, then run the largest call's force launch 3 times "
                         "(direct, treepm: the batch's launch 4 times; bh: both launches twice)")
    ap.add_argument("--profile-tree", action="store_true",
                    help="profiling target (--workload bh): build the GPU tree of the workload twice and exit")
    ap.add_argument("--profile-api", action="store_true",
                    help="profiling target: four full-size drop-in API calls (48 i x N j) and exit")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_setup()
    pgb = load_pkg()
    if args.impl == "reference":
        line = run_reference(args, pgb, ws, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    dist = dist_init(ws, local)
    runner = {"hermite": run_hermite, "direct": run_direct, "clusters": run_clusters, "treepm": run_treepm,
              "bh": run_bh, "integrator": run_integrator}
    line = runner[args.workload](args, pgb, ws, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
