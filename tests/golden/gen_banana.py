"""Generate tests/golden/banana_pl001k.npz from the reference's own Hermite integrator.

Runs the unmodified sample integrator PG6/banana (oracle/_ref/banana01, compiled from the
reference's sources by `make -C oracle ref`, with its setting.mk's -DNORMAL and linked against
the reference libpg6) on the reference's own initial conditions PG6/banana/init/pl001k.init
(1024-body Plummer sphere), for two parameter sets, and stores:

  * the initial conditions (mass, pos, vel) read from the init file;
  * per output time (every dtstar = 1/8): total, potential and kinetic energy as the integrator
    prints them (8 decimals), the particle steps and block steps of the interval;
  * the final snapshot (t = 0.5): energies in full precision and every particle's t, dt, pos,
    vel, acc, jrk, pot.

    python tests/golden/gen_banana.py
"""
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("PGB_REFERENCE", "/root/reference")
BANANA = os.path.join(ROOT, "oracle", "_ref", "banana01")
INIT = os.path.join(REF, "PG6", "banana", "init", "pl001k.init")

# (name, epsinv, eta, eta_s, dtstarinv, tend): the reference input.list's defaults (eps = 0)
# and the same with a softening length of 1/64
CASES = [("eps0", 0.0, 0.2, 0.01, 8.0, 0.5), ("eps64", 64.0, 0.2, 0.01, 8.0, 0.5)]

# struct Particle (PG6/banana/particle.h) as written by output_snapshot (x86-64 layout)
PARTICLE = np.dtype([("t", "<f8"), ("dt", "<f8"), ("mass", "<f4"), ("pot", "<f4"), ("pos", "<f8", 3),
                     ("vel", "<f8", 3), ("acc", "<f8", 3), ("jrk", "<f4", 3), ("id", "<u4"), ("in", "<u4"),
                     ("nn", "<i4"), ("nptr", "<u8")])
assert PARTICLE.itemsize == 128


def read_init(path):
    tok = open(path).read().split()
    n = int(tok[1])
    rec = np.array(tok[2:2 + 8 * n], dtype=np.float64).reshape(n, 8)
    return rec[:, 1], rec[:, 2:5], rec[:, 5:8]


def run(epsinv, eta, eta_s, dtstarinv, tend):
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input.list"), "w") as f:
            f.write(f"0 {tend} {tend}\n{epsinv}\n{eta} {eta_s} {dtstarinv}\n{INIT}\nsnap\n")
        out = subprocess.run([BANANA], cwd=d, capture_output=True, text=True, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS="4")).stdout
        raw = open(os.path.join(d, "snap.bin.0000"), "rb").read()
    times = [float(x) for x in re.findall(r"^Time:\s+([0-9.]+)", out, re.M)]
    en = np.array(re.findall(r"^tot: ([-+0-9.]+) w: ([-+0-9.]+) k: ([-+0-9.]+)", out, re.M), dtype=np.float64)
    st = re.findall(r"niave: ([0-9.e+-]+) ([0-9.e+-]+)", out)
    steps = np.array([float(b) for _, b in st])
    blocks = np.array([round(float(b) / float(a)) if float(a) > 0 else 0 for a, b in st])
    # snapshot: Globaltime (16 B), n (int), particles, Energy (5 doubles)
    n = int(np.frombuffer(raw, "<i4", 1, 16)[0])
    parts = np.frombuffer(raw, PARTICLE, n, 20)
    energy = np.frombuffer(raw, "<f8", 5, 20 + n * PARTICLE.itemsize)
    return dict(times=np.array(times), energies=en, steps=steps, blocks=blocks, snap_t=parts["t"].copy(),
                snap_dt=parts["dt"].copy(), snap_pos=parts["pos"].copy(), snap_vel=parts["vel"].copy(),
                snap_acc=parts["acc"].copy(), snap_jrk=parts["jrk"].astype(np.float64),
                snap_pot=parts["pot"].astype(np.float64), snap_energy=energy.copy())


def main():
    mass, pos, vel = read_init(INIT)
    out = dict(mass=mass, pos=pos, vel=vel)
    for name, epsinv, eta, eta_s, dtsi, tend in CASES:
        r = run(epsinv, eta, eta_s, dtsi, tend)
        out[f"{name}_params"] = np.array([epsinv, eta, eta_s, 1.0 / dtsi, tend])
        for k, v in r.items():
            out[f"{name}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "banana_pl001k.npz"), **out)


if __name__ == "__main__":
    main()
