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
# the reference source tree (only to build the checker when its build is missing)
REF_SRC = os.environ.get("PGB_REFERENCE", "/root/reference")
# DRAM bytes (read + write) of one launch of the roofline kernel, from the committed ncu captures
# (dram__bytes_read.sum + dram__bytes_write.sum); the bench cannot run ncu itself.
G6_CFG_NAMES = ["512x1 (8 j-lanes)", "256x1 (2 j-lanes)", "128x2 i-paired", "128x1", "128x4 i-paired",
                "256x2 i-paired", "128x2 j-paired", "256x2 j-paired", "128x4 j-paired",
                "128x2 j-paired stage-ordered"]   # pgb6 configurations
G5_CFG_NAMES = ["128x4", "256x2", "512x2", "1024x1", "384x2", "128x2", "128x1", "64x1", "64x1 j-paired",
                "1024x1 j-paired", "256x1 j-paired"]   # pgb5 configurations (threads x i/thread)
PROFILED_TRAFFIC = {
    # the largest Hermite call by the configuration that runs it (6: 128x2 j-paired, 2: 128x2 i-paired)
    "hermite": {"bytes": 6_564_864 + 13_965_568,
                "source": "profiles/g6_kernel_hermite_65536x65536.md (128x2 j-paired, 15 chunks)"},
    "hermite_cfg9": {"bytes": 6_416_384 + 72_704,
                     "source": "profiles/g6_kernel_hermite_65536x65536.md (128x2 j-paired, stage-ordered, 8 chunks)"},
    "hermite_cfg2": {"bytes": 6_578_944 + 17_873_152,
                     "source": "profiles/g6_kernel_hermite_65536x65536.md (128x2 i-paired)"},
    "direct": {"bytes": 540_928, "pairs": 268_435_456,
               "source": "profiles/g5_kernels_direct_treepm_bh.md (1024x1 j-paired)"},
    "treepm": {"bytes": 557_901_056 + 35_891_456, "pairs": 4_463_983_086,
               "source": "profiles/g5_kernels_direct_treepm_bh.md (64x1)"},
    # captured at N = 2^20 (both launches of a step); scaled to the run's pairs
    "bh": {"bytes": 131_828_224 + 26_739_456 + 227_582_208 + 31_331_072, "pairs": 4_462_862_693,
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
HERMITE_STREAMS = 3   # streams of the batched Hermite schedule (see hermite_batched; C2 step:
                      # 818 Gint/s on one stream, 858 on two, 866 on three)


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


_PIPE_PEAKS = {}


def pipe_peaks(pgb, stream_ptr=0):
    """Measured FP32 FFMA and MUFU rsqrt throughput of this GPU (lib/libpgbpeak.so: independent
    FFMA / rsqrt.approx chains on every SM, best of 5 CUDA-event-timed launches), with the SM
    clock sampled while they run.  Cached per process (measured once, right after the first
    workload's timed region)."""
    if _PIPE_PEAKS:
        return _PIPE_PEAKS
    L = C.CDLL(pgb.ffi.lib_path("libpgbpeak.so"), mode=os.RTLD_LOCAL | os.RTLD_NOW)
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.pgb_peak_fp32.argtypes = [C.c_int, C.c_void_p, dp, dp, ip]
    L.pgb_peak_mufu.argtypes = [C.c_int, C.c_void_p, dp, dp, ip]
    tf, ms, g = C.c_double(), C.c_double(), C.c_int()
    mg, mms, mgr = C.c_double(), C.c_double(), C.c_int()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    rc1 = L.pgb_peak_fp32(20000, C.c_void_p(stream_ptr), C.byref(tf), C.byref(ms), C.byref(g))
    rc2 = L.pgb_peak_mufu(2500, C.c_void_p(stream_ptr), C.byref(mg), C.byref(mms), C.byref(mgr))
    clk = clocks.stop()
    if rc1 == 0:
        _PIPE_PEAKS.update({"fp32_tflops": round(tf.value, 2), "fp32_ms": round(ms.value, 3), "fp32_ctas": g.value})
    L.pgb_peak_fp32_mix.argtypes = [C.c_int, C.c_int, C.c_void_p, dp, dp]
    mix = {}
    for kind, name in ((0, "ffma2_only"), (1, "ffma2_ffma_1to2"), (2, "ffma2_ffma_1to6")):
        t2, m2 = C.c_double(), C.c_double()
        if L.pgb_peak_fp32_mix(kind, 20000, C.c_void_p(stream_ptr), C.byref(t2), C.byref(m2)) == 0:
            mix[name] = round(t2.value, 2)
    if mix:
        _PIPE_PEAKS["fp32_mix_tflops"] = mix
    # the Hermite kernel's j-paired pair loop alone on a resident shared-memory tile (no j
    # staging, scheduling or partial rows): the rate its arithmetic sustains
    L.pgb_peak_g6_loop.argtypes = [C.c_int, C.c_int, C.c_void_p, dp, dp, ip]
    loop = {}
    for form, name in ((1, "jpair"), (2, "jquad2")):
        gp, lm, rg = C.c_double(), C.c_double(), C.c_int()
        if L.pgb_peak_g6_loop(form, 400, C.c_void_p(stream_ptr), C.byref(gp), C.byref(lm), C.byref(rg)) == 0:
            loop[name] = {"gpairs": round(gp.value, 1), "registers": rg.value}
    if loop:
        _PIPE_PEAKS["g6_pair_loop"] = loop
    # the relative error of the kernels' scale q = -2/r over every float r2 in [1, 4): the MUFU
    # estimate alone (the default build) and refined by the reference's Newton step
    L.pgb_peak_rsqrt_error.argtypes = [C.c_void_p, dp, dp]
    emax, erms = (C.c_double * 2)(), (C.c_double * 2)()
    if L.pgb_peak_rsqrt_error(C.c_void_p(stream_ptr), emax, erms) == 0:
        _PIPE_PEAKS["rsqrt_rel_error"] = {
            "mufu": {"max": float(emax[0]), "rms": float(erms[0])},
            "newton": {"max": float(emax[1]), "rms": float(erms[1])},
            "how": "q = -2/r against FP64 for every float r2 in [1, 4) (lib/libpgbpeak.so pgb_peak_rsqrt_error)"}
    if rc2 == 0:
        _PIPE_PEAKS.update({"mufu_grsqrt_s": round(mg.value, 1), "mufu_ms": round(mms.value, 3),
                            "mufu_per_sm_clk": round(mg.value * 1e9 / SM_COUNT / ((clk.get("sm_mhz") or 1965.0) * 1e6), 2)})
    _PIPE_PEAKS["sm_mhz"] = clk.get("sm_mhz")
    _PIPE_PEAKS["how"] = ("lib/libpgbpeak.so: 8 independent FFMA (rsqrt.approx.ftz.f32) chains per thread, 256-thread "
                          "CTAs at full occupancy on every SM, best of 5 launches (CUDA events)")
    return _PIPE_PEAKS


def pair_loop_ceiling(fp32_tf, kernel_gpairs):
    """The Hermite pair loop's own rate on a resident tile (pipe_peaks) beside the force kernel's:
    the part of the gap to the FFMA peak that the arithmetic itself leaves, and the part the
    kernel's staging, scheduling and reductions add."""
    loop = _PIPE_PEAKS.get("g6_pair_loop")
    if not loop:
        return None
    best = max(v["gpairs"] for v in loop.values())
    return {"forms": loop, "best_gpairs": best, "frac_of_peak": round(best * 1e9 * 60 / 1e12 / fp32_tf, 4),
            "kernel_vs_loop": round(kernel_gpairs / best, 4),
            "how": "lib/libpgbpeak.so pgb_peak_g6_loop: the j-paired inner loop (two i per thread, NN tile "
                   "minimum, FP64 folds every 128 j) over one 128-record tile staged once, a wave of resident "
                   "CTAs, best of 5 launches"}


def fp32_peak(pgb, clk, stream_ptr=0):
    """The FP32 roofline denominator: the measured FFMA throughput (TFLOP/s) when the
    microbenchmark ran, else 148 SMs x 128 lanes x 2 x the sampled SM clock; with its source."""
    pk = peaks()
    sm_mhz = clk.get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
    nominal = SM_COUNT * FP32_LANES * 2 * sm_mhz * 1e6 / 1e12
    pp = pipe_peaks(pgb, stream_ptr)
    if pp.get("fp32_tflops"):
        return pp["fp32_tflops"], nominal, (f"measured: {pp['fp32_tflops']} TFLOP/s FFMA microbenchmark "
                                            f"(lib/libpgbpeak.so) at {pp.get('sm_mhz')} MHz; nominal 148 SM x 128 "
                                            f"lanes x 2 x {sm_mhz:.0f} MHz (timed-region clock) = {nominal:.1f}")
    return nominal, nominal, f"nominal: 148 SM x 128 FP32 lanes x 2 x median SM clock {sm_mhz:.0f} MHz"


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
        L.g6drv_schedule2.argtypes = [vp, C.c_int, C.c_int, ip, ip, dp, dp, dp, C.c_double, C.c_int, C.c_int, ip, ip,
                                      dp, dp, dp, dp, dp, dp, ip, dp, dp, dp, ip, C.POINTER(C.c_float)]
        L.g6drv_schedule2.restype = C.c_double
        L.g6drv_call_time.argtypes = [vp, C.c_int, C.c_int, C.c_int, dp, dp, ip, C.c_double]
        L.g6drv_call_time.restype = C.c_double
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

    def g6_schedule(self, h, wl, calls=None, resend=True, outputs=False, resend_sets=None):
        """Run calls [0, calls) of the schedule; returns (seconds, pairs, outputs or None).
        resend_sets: {"off", "idx"} of the particles re-sent after each call (default: the
        call's own active set)."""
        st, p = wl["st"], self.p
        ncalls = len(wl["sets"]) if calls is None else calls
        off = wl["set_off"]
        nact = int(off[ncalls])
        out = None
        if outputs:
            out = dict(acc=np.zeros((nact, 3)), jrk=np.zeros((nact, 3)), pot=np.zeros(nact),
                       nnb=np.zeros(nact, np.int32), rnnb=np.zeros(nact, np.float32))
        o = out or {}
        rs = resend_sets or {}
        sec = self.L.g6drv_schedule2(h, wl["n"], ncalls, p(off, C.c_int), p(wl["set_idx"], C.c_int),
                                     p(wl["t_calls"]), p(wl["xi"]), p(wl["vi"]), st.eps2, 1, 1 if resend else 0,
                                     p(rs.get("off"), C.c_int), p(rs.get("idx"), C.c_int), p(st.pos), p(st.vel),
                                     p(st.acc2), p(st.jrk6), p(st.mass), p(st.tj), p(st.idx, C.c_int),
                                     p(o.get("acc")), p(o.get("jrk")), p(o.get("pot")), p(o.get("nnb"), C.c_int),
                                     p(o.get("rnnb"), C.c_float))
        return sec, nact * wl["n"], out


def ref_lib(name):
    """The reference's own build (oracle/_ref), compiled here when the reference is present."""
    path = os.path.join(ROOT, "oracle", "_ref", name)
    if not os.path.exists(path) and os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF_SRC}"], check=False)
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


def hermite_shard(pgb, wl, ws, rank):
    """This rank's part of the schedule: a contiguous slice of every call's active set
    (phantom-grape_b200/shard.py).  Returns (sub-schedule, its rows in the schedule's order,
    [(call, local offset, count)], rows of every rank)."""
    S = pgb.shard
    sizes = [len(x) for x in wl["sets"]]
    sl = S.shard_schedule(sizes, ws, rank)
    off = wl["set_off"]
    rows, calls, loc = [], [], 0
    for c, (lo, hi) in enumerate(sl):
        rows.append(np.arange(off[c] + lo, off[c] + hi))
        calls.append((c, loc, int(hi - lo)))
        loc += int(hi - lo)
    rows = np.concatenate(rows).astype(np.int64)
    sub = dict(wl)
    sub["sets"] = [wl["sets"][c][lo:hi] for c, (lo, hi) in enumerate(sl)]
    sub["set_off"] = np.concatenate([[0], np.cumsum([len(x) for x in sub["sets"]])]).astype(np.int32)
    sub["set_idx"] = np.ascontiguousarray(wl["set_idx"][rows], np.int32)
    sub["xi"], sub["vi"] = np.ascontiguousarray(wl["xi"][rows]), np.ascontiguousarray(wl["vi"][rows])
    sub["pairs"] = len(rows) * wl["n"]
    _, nrows = S.rank_major_order(sizes, ws)
    return sub, rows, calls, nrows


def hermite_batched(args, pgb, g6, wl, sub, calls, dev, s, ff, tune, steps, warmup, flush, ws, nrows, dist,
                    clocks=None):
    """The batched device path of the schedule (this rank's share): j-memory, i-records and
    results resident in HBM, one plan per call, the calls' (predict + force) launches captured in
    one CUDA graph; with several ranks the step ends with the all-gather of every rank's results.
    Consecutive calls alternate between HERMITE_STREAMS streams and predicted j-sets, so that a call's
    predictor and nearest-neighbour lookups can run in the tail of the neighbouring call's force
    launch (each stream keeps its own calls in order, which makes reusing its j-set safe).
    Times `steps` replays (CUDA events on the launching stream, L2 flushed in between), then each
    force launch alone.  Returns a dict of the figures and the resident buffers."""
    import torch
    ffi = pgb.ffi
    st, n = wl["st"], wl["n"]
    ptcl = np.zeros(n, ffi.G6PTCL)
    ptcl["pos"], ptcl["vel"], ptcl["acc2"], ptcl["jrk6"] = st.pos, st.vel, st.acc2, st.jrk6
    ptcl["mass"], ptcl["tim"], ptcl["idx"] = st.mass, st.tj, st.idx
    nrow = len(sub["set_idx"])
    pflags = 0 if ff else g6.POS_F64
    irec = ffi.g6_irecords(sub["xi"], sub["vi"], st.idx[sub["set_idx"]], ff=ff)
    d_ptcl = torch.from_numpy(ptcl.view(np.uint8)).to(dev)
    d_irec = torch.from_numpy(irec.view(np.uint8)).to(dev)
    d_pred = torch.zeros(n * ffi.G6PREDJ.itemsize, dtype=torch.uint8, device=dev)
    # the streams the calls alternate between (the launching stream first), each with its own
    # predicted j-set
    lanes = [(s, d_pred)] + [(torch.cuda.Stream(device=dev), torch.zeros_like(d_pred))
                             for _ in range(HERMITE_STREAMS - 1)]
    d_out = torch.zeros((max(nrow, 1), ffi.G6OUT.itemsize), dtype=torch.uint8, device=dev)
    live = [(c, loc, cnt) for c, loc, cnt in calls if cnt > 0]
    plans = {c: g6.plan_create([[loc, cnt, 0, n]], nn=True, f64=not ff) for c, loc, cnt in live}

    def predict(c, buf=None, stream=None):
        buf = d_pred if buf is None else buf
        stream = s if stream is None else stream
        rc = g6.L.pgb6_predict(d_ptcl.data_ptr(), n, float(wl["t_calls"][c]), buf.data_ptr(), pflags,
                               stream.cuda_stream)
        assert rc == 0, g6.last_error()

    def step_launches():
        fork = torch.cuda.Event()
        fork.record(s)
        for st2, _ in lanes[1:]:
            st2.wait_event(fork)
        for k, (c, _, _) in enumerate(live):
            stream, buf = lanes[k % len(lanes)]
            predict(c, buf, stream)
            g6.plan_launch(plans[c], d_irec.data_ptr(), buf.data_ptr(), st.eps2, d_out.data_ptr(), stream.cuda_stream)
        for st2, _ in lanes[1:]:
            join = torch.cuda.Event()
            join.record(st2)
            s.wait_event(join)

    with torch.cuda.stream(s):
        step_launches()
    s.synchronize()
    tuned = {}
    if tune:
        # autotune the kernel configuration once per active-set size, on the real data
        for c, loc, cnt in live:
            if cnt in tuned:
                continue
            predict(c)
            cfg, _ = g6.plan_tune(plans[c], d_irec.data_ptr(), d_pred.data_ptr(), st.eps2, d_out.data_ptr(),
                                  s.cuda_stream)
            tuned[cnt] = cfg
        for c, loc, cnt in live:   # re-create the plans so that every plan picks up its tuned shape
            g6.plan_destroy(plans[c])
            plans[c] = g6.plan_create([[loc, cnt, 0, n]], nn=True, f64=not ff)
        with torch.cuda.stream(s):
            step_launches()
        s.synchronize()
    tuned_chunks = {str(cnt): int(g6.L.pgb6_plan_chunks(plans[c])) for c, _, cnt in sorted(live, key=lambda t: t[2])}
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        step_launches()

    def step():
        graph.replay()
        if ws > 1:
            pgb.shard.gather_rows(d_out[:nrow], nrows, dist)

    with torch.cuda.stream(s):
        for _ in range(warmup):
            step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if clocks:
        clocks.start()
    barrier(ws)
    torch.cuda.synchronize()
    # the timed steps inside an NVTX range, so that a profiler's launch list can select them
    # (ncu --nvtx --nvtx-include "pgb_timed_steps/")
    torch.cuda.nvtx.range_push("pgb_timed_steps")
    with torch.cuda.stream(s):
        for k in range(steps):
            ev[k][0].record(s)
            step()
            ev[k][1].record(s)
            flush.fill_(k & 0xFF)   # 256 MiB write between steps: L2 (126 MB) flushed
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier(ws)
    clk = clocks.stop() if clocks else {}
    step_ms = [a.elapsed_time(b) for a, b in ev]
    # roofline pass (after the timed region): each force launch timed alone with CUDA events,
    # three launches after its predictor, the median taken
    fev = []
    with torch.cuda.stream(s):
        for c, _, cnt in live:
            predict(c)
            evs = []
            for _ in range(3):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(s)
                g6.plan_launch(plans[c], d_irec.data_ptr(), d_pred.data_ptr(), st.eps2, d_out.data_ptr(),
                               s.cuda_stream)
                b.record(s)
                evs.append((a, b))
            fev.append((evs, cnt * n, c))
    torch.cuda.synchronize()
    fms = [(float(np.median([a.elapsed_time(b) for a, b in evs])), p, c) for evs, p, c in fev]
    kern_s = sum(ms for ms, _, _ in fms) / 1e3
    kern_pairs = sum(p for _, p, _ in fms)
    big = max(fms, key=lambda e: e[1])
    return dict(step_ms=step_ms, clk=clk, tuned=tuned, tuned_chunks=tuned_chunks, graph=graph, plans=plans,
                d_ptcl=d_ptcl, d_irec=d_irec,
                d_out=d_out, ptcl=ptcl, irec=irec, nrow=nrow, kern_s=kern_s, kern_pairs=kern_pairs,
                big_pairs=big[1], big_ms=big[0], big_call=big[2], step=step,
                launches_per_step=sum(1 + g6.L.pgb6_plan_kernels(plans[c]) for c, _, _ in live))


def hermite_fp64_check(pgb, wl, sub, calls, out_rows, ff_label=""):
    """FP64 oracle check of the batched results of the largest call (every 64th active particle)."""
    st, n = wl["st"], wl["n"]
    c, loc, cnt = max(calls, key=lambda t: t[2])
    sel = np.arange(loc, loc + cnt, max(1, cnt // 1024))
    xp_c, vp_c = predict_np(wl["t_calls"][c], st)
    ck = fp64_check_g6(out_rows[sel], sub["xi"][sel], sub["vi"][sel], st.idx[sub["set_idx"][sel]], st.eps2,
                       xp_c, vp_c, st.mass, st.idx)
    ck["call"] = f"call {c} ({cnt} active x {n} j), every {max(1, cnt // 1024)}th active particle{ff_label}"
    return ck


def run_hermite(args, pgb, ws, rank, local):
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    dist = None
    if ws > 1:
        import torch.distributed as dist
    ffi = pgb.ffi
    g6 = ffi.G6()
    g6.L.g6_open(0)
    # one problem on every rank (strong scaling over the ranks' slices of each call)
    wl = hermite_workload(pgb, g6)
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
    sub, rows, calls, nrows = hermite_shard(pgb, wl, ws, rank)
    s = torch.cuda.Stream(device=dev)
    ff = not args.f64_positions
    if args.profile_largest:
        # profiling target: after the warm pass (1 + 64 force launches), the largest call's force
        # launch three times; nothing else allocated, no timing
        live = [(c, loc, cnt) for c, loc, cnt in calls if cnt > 0]
        ffi_ = pgb.ffi
        ptcl = np.zeros(n, ffi_.G6PTCL)
        ptcl["pos"], ptcl["vel"], ptcl["acc2"], ptcl["jrk6"] = st.pos, st.vel, st.acc2, st.jrk6
        ptcl["mass"], ptcl["tim"], ptcl["idx"] = st.mass, st.tj, st.idx
        irec = ffi_.g6_irecords(sub["xi"], sub["vi"], st.idx[sub["set_idx"]], ff=ff)
        d_ptcl = torch.from_numpy(ptcl.view(np.uint8)).to(dev)
        d_irec = torch.from_numpy(irec.view(np.uint8)).to(dev)
        d_pred = torch.zeros(n * ffi_.G6PREDJ.itemsize, dtype=torch.uint8, device=dev)
        d_out = torch.zeros(len(rows) * ffi_.G6OUT.itemsize, dtype=torch.uint8, device=dev)
        pflags = 0 if ff else g6.POS_F64
        plans = {c: g6.plan_create([[loc, cnt, 0, n]], nn=True, f64=not ff) for c, loc, cnt in live}
        with torch.cuda.stream(s):
            for c, _, _ in live:
                g6.L.pgb6_predict(d_ptcl.data_ptr(), n, float(wl["t_calls"][c]), d_pred.data_ptr(), pflags,
                                  s.cuda_stream)
                g6.plan_launch(plans[c], d_irec.data_ptr(), d_pred.data_ptr(), st.eps2, d_out.data_ptr(),
                               s.cuda_stream)
            big = max(live, key=lambda t: t[2])[0]
            g6.L.pgb6_predict(d_ptcl.data_ptr(), n, float(wl["t_calls"][big]), d_pred.data_ptr(), pflags,
                              s.cuda_stream)
            for _ in range(3):
                g6.plan_launch(plans[big], d_irec.data_ptr(), d_pred.data_ptr(), st.eps2, d_out.data_ptr(),
                               s.cuda_stream)
        s.synchronize()
        for p_ in plans.values():
            g6.plan_destroy(p_)
        return {"profile": "largest Hermite call", "call": big, "active": len(sets[big]), "nj": n,
                "force_launches_before": 1 + len(live)}

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    clocks = ClockSampler(local)
    B = hermite_batched(args, pgb, g6, wl, sub, calls, dev, s, ff, not args.no_tune, args.steps, args.warmup, flush,
                        ws, nrows, dist, clocks=clocks)
    clk = B["clk"]
    t_local = sum(B["step_ms"]) / 1e3
    t_max = reduce_max(t_local, ws, dev)
    value = float(wl["pairs"]) * args.steps / t_max / 1e9      # the whole schedule per step
    fp32_tf, fp32_nominal, peak_src = fp32_peak(pgb, clk, s.cuda_stream)
    achieved_tf = B["big_pairs"] * 60 / (B["big_ms"] / 1e3) / 1e12
    # DRAM traffic of the largest launch from the committed capture of the configuration it runs
    big_cfg = g6.L.pgb6_plan_config(B["plans"][B["big_call"]])
    tkey = ({6: "hermite", 9: "hermite_cfg9", 2: "hermite_cfg2"}.get(big_cfg)) if ff and ws == 1 else None
    tkey = tkey if tkey in PROFILED_TRAFFIC else None
    achieved_all_tf = B["kern_pairs"] * 60 / B["kern_s"] / 1e12

    # the batched path end to end with host buffers: every step copies the j-memory and the
    # i-records of every call from pinned host memory, replays the graph (and gathers), and
    # reads every result back; CUDA events on the stream around copies and compute
    h_ptcl = torch.from_numpy(B["ptcl"].view(np.uint8)).pin_memory()
    h_irec = torch.from_numpy(B["irec"].view(np.uint8)).pin_memory()
    tot_rows = int(sum(nrows))
    h_out = torch.empty((tot_rows, ffi.G6OUT.itemsize), dtype=torch.uint8).pin_memory()
    e2e_b_ms = []
    for k in range(args.warmup + args.e2e_steps):
        a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            a_.record(s)
            B["d_ptcl"].copy_(h_ptcl, non_blocking=True)
            B["d_irec"].copy_(h_irec, non_blocking=True)
            B["graph"].replay()
            res = B["d_out"][:B["nrow"]]
            if ws > 1:
                res = pgb.shard.gather_rows(res, nrows, dist)
            h_out.copy_(res, non_blocking=True)
            b_.record(s)
        s.synchronize()
        if k >= args.warmup:
            e2e_b_ms.append(a_.elapsed_time(b_))
    e2e_b = float(wl["pairs"]) * len(e2e_b_ms) / reduce_max(sum(e2e_b_ms) / 1e3, ws, dev) / 1e9
    h2d_b = h_ptcl.numel() + h_irec.numel()
    d2h_b = h_out.numel()

    # end to end through the GRAPE-6 API with host buffers (same driver as the reference arm);
    # with several ranks each runs the calls' slices it owns, re-sends every active particle (its
    # j-memory is complete) and the results are gathered
    drv = Driver(pgb)
    h = drv.g6_open(pgb.ffi.lib_path("libpg6.so"))
    drv.g6_set_j(h, st)
    drv.g6_schedule(h, sub, calls=4)   # warm-up
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    rs = dict(off=wl["set_off"], idx=wl["set_idx"])
    outs = None
    torch.cuda.synchronize()
    barrier(ws)
    e2e_t = 0.0
    for _ in range(e2e_steps):
        sec, _, outs = drv.g6_schedule(h, sub, outputs=ws > 1, resend_sets=rs)
        if ws > 1:
            t0 = time.perf_counter()
            loc_rows = np.concatenate([outs["acc"], outs["jrk"], outs["pot"][:, None]], 1)
            pgb.shard.gather_rows(torch.from_numpy(loc_rows).to(dev), nrows, dist).cpu()
            sec += time.perf_counter() - t0
        e2e_t += sec
    e2e_max = reduce_max(e2e_t, ws, dev)
    e2e_val = float(wl["pairs"]) * e2e_steps / e2e_max / 1e9
    # the same calls' device time alone (events around each call's device work in the library)
    g6.L.pgb6_call_device_ms(1)
    g6.L.pgb6_set_call_timing(1)
    sec_t, _, _ = drv.g6_schedule(h, sub, resend_sets=rs)
    g6.L.pgb6_set_call_timing(0)
    plain_dev_s = reduce_max(g6.L.pgb6_call_device_ms(1) / 1e3, ws, dev)
    plain_dev = float(wl["pairs"]) / plain_dev_s / 1e9 if plain_dev_s > 0 else None
    npipe = g6.L.g6_npipes()
    nact = len(sub["set_idx"])
    nchunks = sum((len(x) + npipe - 1) // npipe for x in sub["sets"])
    h2d = nact * (ffi.G6IREC.itemsize + 4) + len(wl["set_idx"]) * ffi.G6PTCL.itemsize + nchunks * 16
    d2h = nact * ffi.G6OUT.itemsize

    cpu = None
    out_rows = B["d_out"][:B["nrow"]].cpu().numpy().reshape(-1).view(ffi.G6OUT)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_hermite(pgb, wl)
        cpu["fp64_check"] = hermite_fp64_check(pgb, wl, sub, calls, out_rows)
    # the FP64 relative coordinate (DADD + F2F, the reference's own split), same schedule, same timing
    f64line = None
    if ws == 1 and not args.no_f64_line and ff:
        s64 = torch.cuda.Stream(device=dev)
        clk64 = ClockSampler(local)
        B64 = hermite_batched(args, pgb, g6, wl, sub, calls, dev, s64, False, not args.no_tune,
                              max(3, min(args.steps, 10)), args.warmup, flush, ws, nrows, dist, clocks=clk64)
        v64 = float(wl["pairs"]) * len(B64["step_ms"]) / (sum(B64["step_ms"]) / 1e3) / 1e9
        f64line = {"value": round(v64, 2), "unit": "Gint/s", "steps": len(B64["step_ms"]),
                   "largest_launch_ms": round(B64["big_ms"], 3),
                   "roofline_frac": round(B64["big_pairs"] * 60 / (B64["big_ms"] / 1e3) / 1e12 / fp32_tf, 4),
                   "relative_coordinates": "FP64 subtract + F2F (the reference's own split, gravity.c:316-333)",
                   "clocks": B64["clk"]}
        if rank == 0 and not args.no_cpu_baseline:
            rows64 = B64["d_out"][:B64["nrow"]].cpu().numpy().reshape(-1).view(ffi.G6OUT)
            f64line["fp64_check"] = hermite_fp64_check(pgb, wl, sub, calls, rows64, " (FP64 x_j - x_i)")
        for p_ in B64["plans"].values():
            g6.plan_destroy(p_)
        del B64
    # the reference's rsqrt form (the MUFU estimate refined by one Newton step,
    # lib/libpg6_newton.so), same schedule, same timing
    nline = None
    if ws == 1 and not args.no_newton_line:
        g6n = ffi.G6("libpg6_newton.so")
        sn = torch.cuda.Stream(device=dev)
        clkn = ClockSampler(local)
        Bn = hermite_batched(args, pgb, g6n, wl, sub, calls, dev, sn, ff, not args.no_tune,
                             max(3, min(args.steps, 10)), args.warmup, flush, ws, nrows, dist, clocks=clkn)
        vn = float(wl["pairs"]) * len(Bn["step_ms"]) / (sum(Bn["step_ms"]) / 1e3) / 1e9
        nline = {"value": round(vn, 2), "unit": "Gint/s", "steps": len(Bn["step_ms"]),
                 "largest_launch_ms": round(Bn["big_ms"], 3),
                 "roofline_frac": round(Bn["big_pairs"] * 60 / (Bn["big_ms"] / 1e3) / 1e12 / fp32_tf, 4),
                 "rsqrt": "rsqrt.approx + one Newton step, q = y (r2 y^2 - 3) (the reference's form, "
                          "gravity.c:341-346), lib/libpg6_newton.so",
                 "clocks": Bn["clk"]}
        if rank == 0 and not args.no_cpu_baseline:
            rowsn = Bn["d_out"][:Bn["nrow"]].cpu().numpy().reshape(-1).view(ffi.G6OUT)
            nline["fp64_check"] = hermite_fp64_check(pgb, wl, sub, calls, rowsn, " (Newton-refined rsqrt)")
        for p_ in Bn["plans"].values():
            g6n.plan_destroy(p_)
        del Bn
    for p_ in B["plans"].values():
        g6.plan_destroy(p_)
    del B["graph"]
    line = {
        "metric": "Gint/s (PG6 Hermite force+jerk+pot+NN, batched)",
        "value": round(value, 2),
        "unit": "Gint/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_max / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak",
        "vs_baseline": None,
        "dtype": "f32 (f64 predictor, " + ("double-float" if ff else "f64") + " x_j-x_i, f64 cross-tile sums)",
        "data": "synthetic (seeded Plummer, DF velocities; no dataset)",
        "config": hermite_config(wl["pairs"], ws),
        "setup": {"sharding": (f"i-partition x{ws}: every rank predicts all j and computes a contiguous slice of "
                               "each call's active set; results all-gathered (NCCL) inside the timed step")
                  if ws > 1 else "one GPU",
                  "graph": "64 x (predict + persistent force launch) in one CUDA graph, consecutive calls on "
                           f"{HERMITE_STREAMS} streams with a predicted j-set each",
                  "relative_coordinates": "double-float (hi+lo FP32)" if ff else "FP64 subtract + F2F",
                  "rsqrt": "rsqrt.approx alone, q = -2 y (lib/libpg6.so)"},
        "frac_fp32": round(value * 1e9 * 60 / 1e12 / fp32_tf, 4),
        "roofline": {"bound": "fp32", "achieved": round(achieved_tf, 2), "peak": round(fp32_tf, 2),
                     "unit": "TFLOP/s", "frac": round(achieved_tf / fp32_tf, 4),
                     "traffic": PROFILED_TRAFFIC[tkey]["bytes"] if tkey else None,
                     "traffic_source": PROFILED_TRAFFIC[tkey]["source"] if tkey else None,
                     "kernel": f"pgb::g6_kernel (autotuned configuration {big_cfg}: "
                               f"{G6_CFG_NAMES[big_cfg] if 0 <= big_cfg < len(G6_CFG_NAMES) else '?'}), largest "
                               f"call of the step ({B['big_pairs']:.3e} pairs, {B['big_ms']:.3f} ms)",
                     "achieved_all_launches": round(achieved_all_tf, 2),
                     "peak_source": peak_src, "peak_nominal": round(fp32_nominal, 2),
                     "mufu_peak_grsqrt_s": _PIPE_PEAKS.get("mufu_grsqrt_s"),
                     "mufu_per_sm_clk": _PIPE_PEAKS.get("mufu_per_sm_clk"),
                     "fp32_mix_tflops": _PIPE_PEAKS.get("fp32_mix_tflops"),
                     "pair_loop_ceiling": pair_loop_ceiling(fp32_tf, B["big_pairs"] / (B["big_ms"] / 1e3) / 1e9),
                     "rsqrt_rel_error": _PIPE_PEAKS.get("rsqrt_rel_error")},
        "e2e": {"value": round(e2e_val, 2), "unit": "Gint/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "api": "GRAPE-6 drop-in (g6_set_ti, g6calc_firsthalf, "
                "g6calc_lasthalf2p per npipes chunk, g6_set_j_particle of the active set), host buffers",
                "npipes": npipe, "steps": e2e_steps,
                "device_only": {"value": round(plain_dev, 2) if plain_dev else None, "unit": "Gint/s",
                                "how": "the same calls' device time (pgb6_call_device_ms: CUDA events around each "
                                       "call's j update + prediction and force launch)"},
                "batched": {"value": round(e2e_b, 2), "unit": "Gint/s", "h2d_bytes_per_step": int(h2d_b),
                            "d2h_bytes_per_step": int(d2h_b), "steps": len(e2e_b_ms),
                            "api": "pgb6_predict + pgb6_plan_launch per call (one CUDA graph) with the j-memory and "
                                   "every call's i-records copied from pinned host memory and every result read "
                                   "back each step; CUDA events on the stream"}},
        "batched_vs_plain": {"device": round(value / plain_dev, 2) if plain_dev else None,
                             "end_to_end": round(e2e_b / e2e_val, 2)},
        "gpu_launches": args.steps * B["launches_per_step"],
        "autotune": {str(k): int(v) for k, v in sorted(B["tuned"].items())},
        "autotune_chunks": B["tuned_chunks"],
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    if f64line:
        line["f64_positions"] = f64line
    if nline:
        line["newton_rsqrt"] = nline
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
          extra=None, kernel="", parallelism=None):
    traffic, tsrc = profiled_traffic(args.workload, pairs)
    peak_tf, nominal_tf, peak_src = fp32_peak(load_pkg(), clk)
    line = {
        "metric": metric, "value": round(value, 2), "unit": "Gint/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_step * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded; no dataset)",
        "config": {"workload": workload, "pairs_per_step": pairs, "flop_per_pair": flop,
                   "l2": "flushed between steps (256 MiB write)",
                   "parallelism": parallelism or (f"replicas x{ws}" if ws > 1 else "one GPU")},
        "frac_fp32": round((value * 1e9 * flop / 1e12 if isinstance(flop, (int, float)) else achieved_tf) / peak_tf, 4),
        "roofline": {"bound": "fp32", "achieved": round(achieved_tf, 2), "peak": round(peak_tf, 2), "unit": "TFLOP/s",
                     "frac": round(achieved_tf / peak_tf, 4), "traffic": traffic, "traffic_source": tsrc,
                     "kernel": kernel, "peak_source": peak_src, "peak_nominal": round(nominal_tf, 2)},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk, "cpu_baseline": cpu,
    }
    if extra:
        line.update(extra)
    nl = line.get("newton_rsqrt")
    if nl and "achieved_tflops" in nl:
        nl["roofline_frac"] = round(nl["achieved_tflops"] / peak_tf, 4)
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
    # the reference's rsqrt form (the MUFU estimate refined by one Newton step,
    # lib/libpg5_newton.so): same inputs, same timing
    nline, d_on = None, None
    if ws == 1 and not args.no_newton_line:
        g5n = pgb.ffi.G5("libpg5_newton.so")
        g5n.L.g5_open()
        d_on = torch.zeros_like(d_o)
        pn = g5n.plan_create(g5n.NEWTON, [[0, n, 0, n]])
        if not args.no_tune:
            g5n.plan_tune(pn, d_i.data_ptr(), d_j.data_ptr(), None, d_on.data_ptr(), s.cuda_stream)
        tn = _timed_launches(torch, s, lambda: g5n.plan_launch(pn, d_i.data_ptr(), d_j.data_ptr(), None,
                                                               d_on.data_ptr(), s.cuda_stream),
                             max(args.steps, 2000), args.warmup, flush)
        nline = {"value": round(pairs * len(tn) / sum(tn) / 1e9, 2), "unit": "Gint/s", "launches": len(tn),
                 "achieved_tflops": round(pairs * len(tn) * 38 / sum(tn) / 1e12, 2),
                 "rsqrt": "rsqrt.approx + one Newton step (the reference's form), lib/libpg5_newton.so"}
        g5n.plan_destroy(pn)
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
        if nline:
            on = d_on.cpu().numpy()[smp]
            nline["fp64_check"] = {"acc": _err_stats(on[:, :3], ao), "pot": _err_stats(-on[:, 3], po, vec=False),
                                   "particles": 1024}
    g5.plan_destroy(plan)
    return _line(args, ws, "Gint/s (PG5 newton direct sum, batched)", value, t_max / len(ts), pairs, 38,
                 "PG5 newton N=16384 Plummer eps=0.01, all i vs all j (acc + pot)", "f32 (f64 cross-tile sums)",
                 achieved, clk,
                 {"value": round(e2e_val, 2), "unit": "Gint/s", "h2d_bytes_per_step": n * 16 * 2,
                  "d2h_bytes_per_step": n * 32, "api": "g5_set_xmj + g5_set_eps_to_all + g5_set_n + "
                  "g5_calculate_force_on_x (direct.c:133-176), host buffers"},
                 cpu, len(ts), extra={"steps": len(ts), **({"newton_rsqrt": nline} if nline else {})},
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
    # one cluster set on every rank; with several ranks each takes a contiguous range of
    # clusters of about equal cost (N_k^2) and the step ends with the all-gather of the results
    cs = W.cluster_set(seed=W.SEED0 + 4)
    n = len(cs.mass)
    idx = np.arange(n, dtype=np.int32)
    bnd = pgb.shard.contiguous_partition(cs.sizes.astype(np.float64) ** 2, ws)
    c0, c1 = int(bnd[rank]), int(bnd[rank + 1])
    p0, p1 = int(cs.offsets[c0]), int(cs.offsets[c1])
    nrows = [int(cs.offsets[bnd[r + 1]] - cs.offsets[bnd[r]]) for r in range(ws)]
    irec = ffi.g6_irecords(cs.pos[p0:p1], cs.vel[p0:p1], idx[p0:p1])
    jrec = ffi.g6_jrecords(cs.pos[p0:p1], cs.vel[p0:p1], cs.mass[p0:p1], idx[p0:p1])
    d_i = torch.from_numpy(irec.view(np.uint8)).to(dev)
    d_j = torch.from_numpy(jrec.view(np.uint8)).to(dev)
    d_o = torch.zeros((max(p1 - p0, 1), ffi.G6OUT.itemsize), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    items = np.stack([cs.offsets[c0:c1] - p0, cs.sizes[c0:c1], cs.offsets[c0:c1] - p0, cs.sizes[c0:c1]], 1)
    plan = g6.plan_create(items, nn=True)
    s = torch.cuda.Stream(device=dev)
    dist = None
    if ws > 1:
        import torch.distributed as dist

    def launch():
        g6.plan_launch(plan, d_i.data_ptr(), d_j.data_ptr(), cs.eps2, d_o.data_ptr(), s.cuda_stream)
        if ws > 1:
            pgb.shard.gather_rows(d_o[:p1 - p0], nrows, dist)

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
    my_pairs = int((cs.sizes[c0:c1].astype(np.int64) ** 2).sum())
    value = float(pairs) * len(ts) / t_max / 1e9
    achieved = my_pairs * len(ts) * 60 / t_local / 1e12
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
    drv.L.g6drv_clusters(h, c0, min(c0 + 8, c1), p(offs, C.c_int), p(pos), p(vel), p(mass), cs.eps2, None, None,
                         None, None, None)
    e2e_t = drv.L.g6drv_clusters(h, c0, c1, p(offs, C.c_int), p(pos), p(vel), p(mass), cs.eps2,
                                 None, None, None, None, None)
    e2e_val = float(pairs) / reduce_max(e2e_t, ws, dev) / 1e9
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
        rows = d_o.cpu().numpy().reshape(-1).view(ffi.G6OUT)
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
    kernels_per_launch = max(1, g6.L.pgb6_plan_kernels(plan))
    g6.plan_destroy(plan)
    return _line(args, ws, "Gint/s (independent Hermite clusters, batched)", value, t_max / len(ts), pairs, 60,
                 "1024 Plummer clusters, N log-uniform [256,16384], eps=1e-4, one force+jerk+pot+NN each",
                 "f32 (double-float x_j-x_i, f64 cross-tile sums)", achieved, clk,
                 {"value": round(e2e_val, 3), "unit": "Gint/s", "h2d_bytes_per_step": n * (128 + 48),
                  "d2h_bytes_per_step": n * 64, "api": "plain GRAPE-6 calls per cluster (g6_set_j_particle x N_k, "
                  "g6_set_ti, g6calc_firsthalf/lasthalf2p per npipes), host buffers"},
                 cpu, len(ts) * kernels_per_launch, extra={"autotune": cfg, "batched_vs_plain": round(value / e2e_val, 1),
                                      "scaling": "strong" if ws > 1 else "weak"},
                 kernel="pgb::g6_kernel (autotuned configuration)",
                 parallelism=(f"contiguous cost partition of the clusters x{ws}, results all-gathered in the step"
                              if ws > 1 else "one GPU"))


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
    # the reference's rsqrt form (the MUFU estimate refined by one Newton step,
    # lib/libpg5_newton.so): the same two launches, same timing
    nline, acc_n = None, None
    if ws == 1 and not args.no_newton_line:
        g5n = pgb.ffi.G5("libpg5_newton.so")
        g5n.L.g5_open()
        qn_p, qn_c = g5n.plan_create(g5n.NEWTON, bh.items("p")), g5n.plan_create(g5n.QUAD, bh.items("c"))
        on_p, on_c = torch.zeros_like(o_p), torch.zeros_like(o_c)
        an_p = (d_i.data_ptr(), d_p.data_ptr(), None, d_pi.data_ptr(), on_p.data_ptr(), s.cuda_stream)
        an_c = (d_i.data_ptr(), d_c.data_ptr(), d_q.data_ptr(), d_ci.data_ptr(), on_c.data_ptr(), s.cuda_stream)
        if not args.no_tune:
            g5n.plan_tune_indexed(qn_p, *an_p)
            g5n.plan_tune_indexed(qn_c, *an_c)

        def launch_n():
            g5n.plan_launch_indexed(qn_p, *an_p)
            g5n.plan_launch_indexed(qn_c, *an_c)

        gn = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            launch_n()
        torch.cuda.synchronize()
        with torch.cuda.graph(gn, stream=s):
            launch_n()
        tn = _timed_launches(torch, s, gn.replay, args.steps, args.warmup, flush)
        del gn
        acc_n = (on_p[:, :3] + on_c[:, :3]).cpu().numpy()
        nline = {"value": round(pairs * len(tn) / sum(tn) / 1e9, 2), "unit": "Gint/s", "steps": len(tn),
                 "achieved_tflops": round(flops * len(tn) / sum(tn) / 1e12, 2),
                 "rsqrt": "rsqrt.approx + one Newton step (the reference's form), lib/libpg5_newton.so"}
        g5n.plan_destroy(qn_p)
        g5n.plan_destroy(qn_c)

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
        e1, en = [], []
        for g in range(0, bh.ngroups, 97):
            sl = slice(bh.gfirst[g], bh.gfirst[g] + bh.gcount[g])
            pl = bh.pidx[bh.poff[g]:bh.poff[g + 1]]
            cl = bh.cidx[bh.coff[g]:bh.coff[g + 1]]
            a1, _ = O.g5_newton(xi[sl], float(ip[0, 3]), xp[pl], mp[pl])
            a2, _ = O.g5_quad(xi[sl], float(ip[0, 3]), cpos[cl], cm[cl], cqq[cl])
            ref = a1 + a2
            e1.append(np.linalg.norm(acc_b[sl] - ref, axis=1) / np.linalg.norm(ref, axis=1))
            if acc_n is not None:
                en.append(np.linalg.norm(acc_n[sl] - ref, axis=1) / np.linalg.norm(ref, axis=1))
        e1 = np.concatenate(e1)
        if nline:
            en = np.concatenate(en)
            nline["fp64_check"] = {"acc": {"rms": float(np.sqrt(np.mean(en ** 2))), "max": float(en.max()),
                                           "particles": int(len(en))}, "oracle": "FP64 on the same lists"}
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
    if "same_lists_fp64" in errors:
        cpu = cpu if cpu is not None else {}
        cpu["fp64_check"] = {"acc": errors["same_lists_fp64"], "direct_sum_acc": errors["direct_sum_fp64"],
                             "oracle": "FP64 on the same interaction lists and float32 inputs (every 97th group); "
                                       "the full FP64 direct sum on 4096 sampled particles measures the multipole "
                                       "truncation at theta = 0.5"}
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
                        "errors": errors, **({"newton_rsqrt": nline} if nline else {})},
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


def hermite_config(pairs, ws):
    """The configuration both arms of the Hermite benchmark report (identical by construction)."""
    return {"workload": "PG6 Hermite N=65536 Plummer eps=1e-4, 64 block-step calls of 2^k active (k=4..16), "
                        "force+jerk+pot+nearest neighbour",
            "pairs_per_step": int(pairs), "flop_per_pair": 60, "calls_per_step": 64,
            "l2": "flushed between steps (256 MiB write); the CPU arm's working set exceeds its caches",
            "parallelism": f"i-partition x{ws} (strong)" if ws > 1 else "one device"}


def run_reference(args, pgb, ws, rank):
    if rank != 0:
        return None
    if args.workload == "integrator":
        return run_reference_integrator(args, pgb, ws, rank)
    path = ref_lib("libpg6_ref.so")
    if path is None:
        return {"impl": "reference", "unavailable": "reference library (oracle/_ref/libpg6_ref.so) not built"}
    from oracle import refapi
    W = pgb.workloads

    def ref_force(x, v, m, eps2):
        # the state's acceleration and jerk from the reference library itself (all particles
        # active, npipes chunks), so that no part of this arm runs on the GPU engine
        R = refapi.RefG6()
        idx = np.arange(len(x), dtype=np.int32)
        z = np.zeros_like(x)
        R.set_j(x, v, z, z, m, np.full(len(x), 1.0), idx)
        r = R.calc(1.0, len(x), x, v, idx, eps2, variant="plain")
        return r["acc"], r["jrk"]

    drv = Driver(pgb)
    h = drv.g6_open(path)
    st = W.hermite_state(65536, seed=W.SEED0 + 1, force_fn=ref_force)
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
    # warm-up steps: one call each (OpenMP thread pool, page faults); timed steps: the whole
    # 64-call schedule, as the GPU arm's step
    for _ in range(args.warmup):
        drv.g6_schedule(h, wl, calls=1)
    tot, pairs = 0.0, 0
    for _ in range(args.steps):
        sec, p_, _ = drv.g6_schedule(h, wl)
        tot += sec
        pairs += p_
    val = pairs / tot / 1e9
    sample = (f"the whole 64-call schedule per step ({pairs // args.steps:.3e} pairs), PG6/libpg6 AVX2 + OpenMP "
              f"built from its own sources, npipes 48, the same call sequence as the GPU arm's e2e")
    return {
        "metric": "Gint/s (PG6 Hermite force+jerk+pot+NN, batched)",
        "value": round(val, 3), "unit": "Gint/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tot / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak",
        "vs_baseline": None, "dtype": "f32 (f64 predictor + x_j-x_i)", "data": "synthetic (seeded Plummer, DF velocities; no dataset)",
        "config": hermite_config(pairs // args.steps, ws),
        "impl": "reference",
        "cpu_baseline": {"value": round(val, 3), "unit": "Gint/s", "cores": os.cpu_count(), "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(val, 3), "unit": "Gint/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ----------------------------------------------------------------------------------------

def run_api_floor(pgb):
    """The drop-in API's per-call wall time for several (i, j) shapes on the C2 state (C caller:
    drivers/pgb_drivers.c g6drv_call_time, g6calc_firsthalf + g6calc_lasthalf2p, best of three runs
    of 2000 calls) and the floor of a launch and its completion (lib/libpgbpeak.so
    pgb_peak_launch_floor: empty kernels waited for by stream synchronisation or by a polled
    flag in mapped host memory)."""
    g6 = pgb.ffi.G6()
    g6.L.g6_open(0)
    wl = hermite_workload(pgb, g6)
    st, n = wl["st"], wl["n"]
    drv = Driver(pgb)
    h = drv.g6_open(pgb.ffi.lib_path("libpg6.so"))
    drv.g6_set_j(h, st)
    g6.L.g6_set_ti(0, float(wl["t_calls"][0]))
    sel = np.arange(0, 48 * 97, 97) % n
    xi, vi = np.ascontiguousarray(st.pos[sel]), np.ascontiguousarray(st.vel[sel])
    idi = np.ascontiguousarray(st.idx[sel], np.int32)
    calls = {}
    for ni, nj in ((48, n), (16, n), (1, n), (48, 16384), (48, 1024), (1, 128)):
        t = drv.L.g6drv_call_time(h, ni, nj, 2000, Driver.p(xi), Driver.p(vi), Driver.p(idi, C.c_int), st.eps2)
        calls[f"{ni}x{nj}"] = round(t * 1e6, 2)
    L = C.CDLL(pgb.ffi.lib_path("libpgbpeak.so"), mode=os.RTLD_LOCAL | os.RTLD_NOW)
    L.pgb_peak_launch_floor.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_double)]
    floor = {}
    for kind, name in ((0, "stream_sync"), (1, "flag_poll")):
        for grid in (1, 264):
            us = C.c_double()
            if L.pgb_peak_launch_floor(kind, grid, 3000, None, C.byref(us)) == 0:
                floor[f"{name}_grid{grid}"] = round(us.value, 2)
    return {"api_call_us": calls, "empty_launch_us": floor, "npipes": int(g6.L.g6_npipes()),
            "how": "µs per drop-in call (firsthalf + lasthalf2p) by i x j shape on the C2 state, host clock; "
                   "empty-kernel launch + completion for comparison"}


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
    ap.add_argument("--no-f64-line", action="store_true",
                    help="hermite: skip the second batched run with FP64 relative coordinates")
    ap.add_argument("--no-newton-line", action="store_true",
                    help="skip the second run with the reference's Newton-refined rsqrt (lib*_newton.so)")
    ap.add_argument("--no-workloads", action="store_true",
                    help="hermite on one GPU: skip the other configurations' lines (C1, C3, C4, C5)")
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
    ap.add_argument("--api-floor", action="store_true",
                    help="per-call time of the GRAPE-6 drop-in API by call shape, beside the launch and "
                         "completion floor of empty kernels; one JSON line")
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
    if args.api_floor:
        print(json.dumps(run_api_floor(pgb)), flush=True)
        return
    dist = dist_init(ws, local)
    runner = {"hermite": run_hermite, "direct": run_direct, "clusters": run_clusters, "treepm": run_treepm,
              "bh": run_bh, "integrator": run_integrator}
    line = runner[args.workload](args, pgb, ws, rank, local)
    profiling = args.profile_largest or args.profile_tree or args.profile_api
    if args.workload == "hermite" and ws == 1 and not args.no_workloads and not profiling:
        # the other configurations of the benchmark, each with its own value, roofline, e2e,
        # CPU baseline and FP64 check, in the same run
        import copy
        import torch
        wls = {}
        for key, name in (("C1", "direct"), ("C3", "treepm"), ("C4", "bh"), ("C5", "clusters")):
            torch.cuda.empty_cache()
            sub_args = copy.copy(args)
            sub_args.workload = name
            t0 = time.perf_counter()
            try:
                sub = runner[name](sub_args, pgb, ws, rank, local)
            except Exception as e:   # reported in the line; the headline stands
                sub = {"error": f"{type(e).__name__}: {e}"}
            sub["wall_s"] = round(time.perf_counter() - t0, 1)
            wls[key] = sub
        line["workloads"] = wls
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
