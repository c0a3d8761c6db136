"""Seeded synthetic particle sets for the force-engine workloads.

All randomness comes from a counter-based splitmix64 stream (``Rng``), so every harness
(tests, benchmark, fixture scripts) gets identical bits on any machine.  Seeds are
``20261203 + config index`` by default.  The sets stand in for the reference's sample
inputs (Plummer spheres, uniform boxes, cluster sets) with the same shapes, sizes and
distributions; no data file is read.

Workloads
---------
* ``plummer_g5``      PG5 newton direct sum: N=16384 equal-mass Plummer sphere, G=1, a=1,
                      radii truncated at 22.8 a, float32-rounded positions, eps = 0.01.
* ``hermite_state``   PG6 Hermite: Plummer sphere with distribution-function velocities,
                      FP64, eps = 1e-4, block time-step state (levels 3..12, t_j lagging
                      t_now by 0, 1/2 or 1 of the particle's step).
* ``hermite_schedule``64 force calls with active sets of 2^k particles, k uniform in 4..16.
* ``cluster_set``     1024 independent Plummer clusters, N log-uniform in [256, 16384].
* ``treepm_groups``  PG5 table (TreePM PP): N=2^20 uniform periodic box, i-groups from a
                      128^3 cell mesh, j-lists within r_cut with explicit periodic shifts;
                      ``gaussian_split_force`` is the matching force shape for the table.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SEED0 = 20261203
_GOLD = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


class Rng:
    """Counter-based splitmix64: value k of stream s is mix(s + (k+1) * golden)."""

    def __init__(self, seed: int):
        self.state = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.k = 0

    def u64(self, n: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            ks = np.arange(self.k + 1, self.k + 1 + n, dtype=np.uint64)
            z = self.state + ks * _GOLD
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
            z = z ^ (z >> np.uint64(31))
        self.k += n
        return z

    def uniform(self, n: int) -> np.ndarray:
        """Uniform doubles in [0, 1) with 53 random bits."""
        return (self.u64(n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)

    def integers(self, lo: int, hi: int, n: int) -> np.ndarray:
        """Integers in [lo, hi) (hi - lo small; bias < 2^-40)."""
        return lo + (self.u64(n) % np.uint64(hi - lo)).astype(np.int64)

    def permutation(self, n: int) -> np.ndarray:
        return np.argsort(self.u64(n), kind="stable")


def _isotropic(rng: Rng, r: np.ndarray) -> np.ndarray:
    n = len(r)
    cth = 2.0 * rng.uniform(n) - 1.0
    phi = 2.0 * math.pi * rng.uniform(n)
    sth = np.sqrt(np.maximum(0.0, 1.0 - cth * cth))
    return np.stack([r * sth * np.cos(phi), r * sth * np.sin(phi), r * cth], axis=1)


def plummer_radii(rng: Rng, n: int, rmax: float = 22.8) -> np.ndarray:
    out = np.empty(0)
    while len(out) < n:
        u = rng.uniform(2 * (n - len(out)) + 16)
        u = u[u > 0]
        r = 1.0 / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        out = np.concatenate([out, r[r <= rmax]])
    return out[:n]


def plummer_speeds(rng: Rng, r: np.ndarray) -> np.ndarray:
    """Aarseth-Henon-Wielen rejection: q on g(q) = q^2 (1-q^2)^(7/2), v = q sqrt(2) (1+r^2)^(-1/4)."""
    n = len(r)
    q = np.empty(0)
    while len(q) < n:
        m = 4 * (n - len(q)) + 16
        x = rng.uniform(m)
        y = 0.1 * rng.uniform(m)
        ok = y < x * x * (1.0 - x * x) ** 3.5
        q = np.concatenate([q, x[ok]])
    q = q[:n]
    return q * math.sqrt(2.0) * (1.0 + r * r) ** -0.25


@dataclass
class G5Set:
    x: np.ndarray        # [n,3] float64 (float32-representable)
    m: np.ndarray        # [n]   float64 (float32-representable)
    eps: float


def plummer_g5(n: int = 16384, seed: int = SEED0 + 0, eps: float = 0.01) -> G5Set:
    rng = Rng(seed)
    x = _isotropic(rng, plummer_radii(rng, n))
    x = x.astype(np.float32).astype(np.float64)
    m = np.full(n, np.float64(np.float32(1.0 / n)))
    return G5Set(x=x, m=m, eps=eps)


@dataclass
class HermiteState:
    pos: np.ndarray      # [n,3] FP64 at t_j
    vel: np.ndarray      # [n,3]
    acc2: np.ndarray     # [n,3] acc / 2   (the library's predictor convention)
    jrk6: np.ndarray     # [n,3] jerk / 6
    mass: np.ndarray     # [n]
    tj: np.ndarray       # [n]  particle times
    idx: np.ndarray      # [n]  int32 ids
    eps2: float
    t_now: float


def plummer_hermite(n: int, seed: int, rmax: float = 22.8):
    rng = Rng(seed)
    r = plummer_radii(rng, n, rmax)
    x = _isotropic(rng, r)
    v = _isotropic(rng, plummer_speeds(rng, r))
    # centre of mass / momentum at rest
    x -= x.mean(axis=0)
    v -= v.mean(axis=0)
    return x, v, np.full(n, 1.0 / n), rng


def plummer_henon(n: int, seed: int):
    """Plummer sphere in Henon units (G = M = 1, E = -1/4: scale radius 3 pi / 16), equal
    masses 1/n, centre of mass at rest -- the units of the reference sample integrator's
    initial conditions (PG6/banana/init/pl*.init).  Returns (x, v, m)."""
    x, v, m, _ = plummer_hermite(n, seed)
    a = 3.0 * np.pi / 16.0
    return x * a, v / np.sqrt(a), m


def hermite_state(n: int = 65536, seed: int = SEED0 + 1, eps: float = 1e-4,
                  force_fn=None, t_now: float = 1.0) -> HermiteState:
    """Block time-step state.  ``force_fn(x, v, m, eps2) -> (acc, jrk)`` supplies the
    instantaneous acceleration and jerk (an FP64 direct sum in tests, the GPU engine in the
    benchmark); with ``None`` they are zero (pure drift prediction)."""
    x, v, m, rng = plummer_hermite(n, seed)
    eps2 = eps * eps
    if force_fn is not None:
        a, j = force_fn(x, v, m, eps2)
    else:
        a = np.zeros_like(x)
        j = np.zeros_like(x)
    lev = rng.integers(3, 13, n)
    dt = np.ldexp(1.0, -lev)
    u = rng.integers(0, 3, n) * 0.5
    tj = t_now - dt * u
    # positions at t_j consistent with the Taylor expansion about t_now (back-extrapolated)
    h = (tj - t_now)[:, None]
    pos = x + v * h + 0.5 * a * h * h + j * h ** 3 / 6.0
    vel = v + a * h + 0.5 * j * h * h
    acc = a + j * h
    return HermiteState(pos=pos, vel=vel, acc2=0.5 * acc, jrk6=j / 6.0, mass=m, tj=tj,
                        idx=np.arange(n, dtype=np.int32), eps2=eps2, t_now=t_now)


def hermite_schedule(n: int = 65536, ncalls: int = 64, kmin: int = 4, kmax: int = 16,
                     seed: int = SEED0 + 101):
    """List of active sets (int32 index arrays) of size 2^k, k uniform in [kmin, kmax]."""
    rng = Rng(seed)
    ks = rng.integers(kmin, kmax + 1, ncalls)
    sets = []
    for k in ks:
        size = min(1 << int(k), n)
        perm = rng.permutation(n)
        sets.append(np.sort(perm[:size]).astype(np.int32))
    return sets


@dataclass
class ClusterSet:
    offsets: np.ndarray  # [ncl+1] particle offsets
    pos: np.ndarray      # [N,3] FP64
    vel: np.ndarray
    mass: np.ndarray
    eps2: float
    sizes: np.ndarray = field(default=None)


def cluster_set(ncl: int = 1024, nmin: int = 256, nmax: int = 16384,
                seed: int = SEED0 + 4, eps: float = 1e-4, spacing: float = 64.0) -> ClusterSet:
    rng = Rng(seed)
    u = rng.uniform(ncl)
    sizes = np.rint(np.exp(math.log(nmin) + u * (math.log(nmax) - math.log(nmin)))).astype(np.int64)
    sizes = np.clip(sizes, nmin, nmax)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    pos = np.empty((offs[-1], 3))
    vel = np.empty((offs[-1], 3))
    mass = np.empty(offs[-1])
    for c in range(ncl):
        x, v, m, _ = plummer_hermite(int(sizes[c]), seed * 7919 + c)
        centre = np.array([spacing * (c % 32), spacing * ((c // 32) % 32), spacing * (c // 1024)])
        s = slice(offs[c], offs[c + 1])
        pos[s] = x + centre
        vel[s] = v
        mass[s] = m
    return ClusterSet(offsets=offs, pos=pos, vel=vel, mass=mass, eps2=eps * eps, sizes=sizes)


# ------------------------------------------------------------------------------------------
# PG5 table (TreePM particle-particle part)

def gaussian_split_force(rs: float, rcut: float, eps: float):
    """Force shape over r of the TreePM short-range part, for pg5_gen_force_table:
    f(r) = g(r) / (r^2 + eps^2)^(3/2) with g(r) = erfc(r / 2 rs) + r / (sqrt(pi) rs) exp(-r^2 / 4 rs^2),
    and f = 0 at r >= rcut so that the table's last entry (the clamp value) is zero; the
    table's last node sits at rcut up to float rounding, hence the 1e-6 relative margin.
    The Plummer-softened denominator keeps entry 0 (r = 0) finite."""
    inv_sqrt_pi = 1.0 / math.sqrt(math.pi)
    rzero = rcut * (1.0 - 1e-6)

    def f(r):
        if r >= rzero:
            return 0.0
        g = math.erfc(r / (2.0 * rs)) + r * inv_sqrt_pi / rs * math.exp(-r * r / (4.0 * rs * rs))
        return g / (r * r + eps * eps) ** 1.5

    return f


@dataclass
class TreePMSet:
    x: np.ndarray        # [n,3] particle positions in the unit box (float32-representable)
    m: np.ndarray        # [n]
    xi: np.ndarray       # [n,3] i-particles ordered by group
    order: np.ndarray    # xi = x[order]
    items: np.ndarray    # [ngroups,4] int32: i_offset, i_count, j_offset, j_count
    xj: np.ndarray       # [nj_total,3] j-lists, periodic images already shifted
    mj: np.ndarray       # [nj_total]
    rs: float
    rcut: float
    eps: float

    @property
    def interactions(self) -> int:
        return int((self.items[:, 1].astype(np.int64) * self.items[:, 3]).sum())


def treepm_groups(n: int = 1 << 20, seed: int = SEED0 + 2, mesh: int = 128, block: int = 8,
                  nmax: int = 512) -> TreePMSet:
    """Uniform periodic unit box; i-groups are blocks of block^3 cells of a mesh^3 cell mesh,
    split into octants while they hold more than nmax particles; each group's j-list holds every
    particle (or periodic image) within rcut of the group's box.  Candidates come from the 27
    blocks around the group's block (a block is at least rcut wide)."""
    rng = Rng(seed)
    x = rng.uniform(3 * n).reshape(n, 3).astype(np.float32).astype(np.float64)
    m = np.full(n, 1.0 / n)
    rs = 1.25 / n ** (1.0 / 3.0)
    rcut = 4.5 * rs
    eps = 0.1 / n ** (1.0 / 3.0)
    nb = mesh // block
    assert block / mesh >= rcut, "blocks must be at least rcut wide"
    cell = np.minimum((x * mesh).astype(np.int64), mesh - 1)
    blk = cell // block
    bid = (blk[:, 0] * nb + blk[:, 1]) * nb + blk[:, 2]
    border = np.argsort(bid, kind="stable")
    bstart = np.searchsorted(bid[border], np.arange(nb ** 3 + 1))

    order, items, xjs, mjs = [], [], [], []
    ioff = joff = 0
    for bx in range(nb):
        for by in range(nb):
            for bz in range(nb):
                b = (bx * nb + by) * nb + bz
                members = border[bstart[b]:bstart[b + 1]]
                # neighbour candidates with periodic shifts
                cand, shifts = [], []
                for ox in (-1, 0, 1):
                    for oy in (-1, 0, 1):
                        for oz in (-1, 0, 1):
                            wx, wy, wz = bx + ox, by + oy, bz + oz
                            nbid = ((wx % nb) * nb + (wy % nb)) * nb + (wz % nb)
                            sl = border[bstart[nbid]:bstart[nbid + 1]]
                            cand.append(sl)
                            shifts.append(np.broadcast_to(
                                np.array([wx // nb, wy // nb, wz // nb], np.float64), (len(sl), 3)))
                cand = np.concatenate(cand)
                pc = x[cand] + np.concatenate(shifts)
                # split the block into octants while a group is too large
                todo = [(np.array([bx, by, bz]) * block, block, members)]
                while todo:
                    lo, size, mem = todo.pop(0)
                    if len(mem) > nmax and size > 1:
                        h = size // 2
                        cm = cell[mem]
                        for ox in (0, h):
                            for oy in (0, h):
                                for oz in (0, h):
                                    o = lo + np.array([ox, oy, oz])
                                    sel = np.all((cm >= o) & (cm < o + h), axis=1)
                                    todo.append((o, h, mem[sel]))
                        continue
                    if len(mem) == 0:
                        continue
                    blo, bhi = lo / mesh, (lo + size) / mesh
                    d = np.maximum(0.0, np.maximum(blo - pc, pc - bhi))
                    keep = (d * d).sum(axis=1) <= rcut * rcut
                    order.append(mem)
                    xjs.append(pc[keep])
                    mjs.append(m[cand[keep]])
                    items.append((ioff, len(mem), joff, int(keep.sum())))
                    ioff += len(mem)
                    joff += int(keep.sum())
    order = np.concatenate(order)
    return TreePMSet(x=x, m=m, xi=x[order], order=order, items=np.array(items, np.int32),
                     xj=np.concatenate(xjs), mj=np.concatenate(mjs), rs=rs, rcut=rcut, eps=eps)


# ------------------------------------------------------------------------------------------
# Barnes-Hut with quadrupole cells (newton_quad)

def hernquist_radii(rng: Rng, n: int, rmax: float = 100.0) -> np.ndarray:
    """Hernquist (a = 1) radii by inverting M(<r)/M = r^2/(1+r)^2: r = sqrt(U)/(1 - sqrt(U)),
    rejecting r > rmax."""
    out = np.empty(0)
    while len(out) < n:
        s = np.sqrt(rng.uniform(2 * (n - len(out)) + 16))
        s = s[s < 1.0]
        r = s / (1.0 - s)
        out = np.concatenate([out, r[r <= rmax]])
    return out[:n]


@dataclass
class BHSet:
    """A Barnes-Hut force evaluation: particles in tree order, the tree's cells and every
    group's interaction list (point masses: indices into the particles; cells: indices into
    the cell arrays).  Built by drivers/pgb_bhtree.c."""
    x: np.ndarray        # [n,3] tree-order positions (float32-representable)
    m: np.ndarray        # [n]
    perm: np.ndarray     # [n] tree order -> sampling order
    gfirst: np.ndarray   # [ng] int32 first particle of each group (tree order)
    gcount: np.ndarray   # [ng] int32
    gcentre: np.ndarray  # [ng,3] group cell centre
    ghalf: np.ndarray    # [ng] group cell half side
    poff: np.ndarray     # [ng+1] int64 point-mass list offsets
    pidx: np.ndarray     # [np] int32
    coff: np.ndarray     # [ng+1] int64 cell list offsets
    cidx: np.ndarray     # [nc] int32
    ccom: np.ndarray     # [ncell,3] cell centre of mass
    cmass: np.ndarray    # [ncell]
    cquad: np.ndarray    # [ncell,6] (xx, xy, xz, yy, yz, zz), traceless
    nfirst: np.ndarray   # [ncell] the tree's nodes (= the cells): particle range, half side,
    ncount: np.ndarray   #   geometric centre and children (-1: empty octant)
    nhalf: np.ndarray
    ncentre: np.ndarray
    nchild: np.ndarray   # [ncell,8]
    eps: float
    theta: float
    nleaf: int
    ncrit: int

    @property
    def ngroups(self) -> int:
        return len(self.gfirst)

    @property
    def p_pairs(self) -> int:
        return int((self.gcount.astype(np.int64) * np.diff(self.poff)).sum())

    @property
    def c_pairs(self) -> int:
        return int((self.gcount.astype(np.int64) * np.diff(self.coff)).sum())

    def records(self):
        """float32 records of the batched path: i (x, y, z, eps^2), particles (x, y, z, m), cells
        (centre of mass, mass) and their quadrupole words (xx xy xz yy)(yz zz 0 0)."""
        n, nc = len(self.m), len(self.cmass)
        ip = np.empty((n, 4), np.float32)
        ip[:, :3] = self.x
        ip[:, 3] = np.float32(self.eps * self.eps)
        pp = np.empty((n, 4), np.float32)
        pp[:, :3] = self.x
        pp[:, 3] = self.m
        cp = np.empty((nc, 4), np.float32)
        cp[:, :3] = self.ccom
        cp[:, 3] = self.cmass
        cq = np.zeros((nc, 8), np.float32)
        cq[:, :6] = self.cquad
        return ip, pp, cp, cq

    def items(self, kind: str) -> np.ndarray:
        """Work items (i_offset, i_count, j_offset, j_count) of the point-mass ('p') or cell
        ('c') lists, j offsets into the index list."""
        off = self.poff if kind == "p" else self.coff
        return np.stack([self.gfirst, self.gcount, off[:-1], np.diff(off)], 1).astype(np.int32)


def _bh_read(L, pre, h, x, m, eps, theta, nleaf, ncrit):
    """Read a built tree through the accessors <pre>n, <pre>groups, ... of library L."""
    import ctypes as C
    vp, dp, ip, lp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_longlong)
    for f, r in (("ngroups", C.c_int), ("nnodes", C.c_int), ("np", C.c_longlong), ("nc", C.c_longlong)):
        getattr(L, pre + f).argtypes = [vp]
        getattr(L, pre + f).restype = r
    getattr(L, pre + "perm").argtypes = [vp, ip]
    getattr(L, pre + "groups").argtypes = [vp, ip, ip, dp, dp]
    getattr(L, pre + "cells").argtypes = [vp, dp, dp, dp]
    getattr(L, pre + "lists").argtypes = [vp, lp, ip, lp, ip]
    getattr(L, pre + "nodes").argtypes = [vp, ip, ip, dp, dp, ip]
    n = len(m)
    fn = lambda name: getattr(L, pre + name)  # noqa: E731
    ng, nn, npl, ncl = fn("ngroups")(h), fn("nnodes")(h), fn("np")(h), fn("nc")(h)
    perm = np.empty(n, np.int32)
    fn("perm")(h, perm.ctypes.data_as(ip))
    gfirst, gcount = np.empty(ng, np.int32), np.empty(ng, np.int32)
    gcentre, ghalf = np.empty((ng, 3)), np.empty(ng)
    fn("groups")(h, gfirst.ctypes.data_as(ip), gcount.ctypes.data_as(ip), gcentre.ctypes.data_as(dp),
                 ghalf.ctypes.data_as(dp))
    ccom, cmass, cquad = np.empty((nn, 3)), np.empty(nn), np.empty((nn, 6))
    fn("cells")(h, ccom.ctypes.data_as(dp), cmass.ctypes.data_as(dp), cquad.ctypes.data_as(dp))
    poff, coff = np.empty(ng + 1, np.int64), np.empty(ng + 1, np.int64)
    pidx, cidx = np.empty(max(npl, 1), np.int32), np.empty(max(ncl, 1), np.int32)
    fn("lists")(h, poff.ctypes.data_as(lp), pidx.ctypes.data_as(ip), coff.ctypes.data_as(lp), cidx.ctypes.data_as(ip))
    nfirst, ncount, nhalf = np.empty(nn, np.int32), np.empty(nn, np.int32), np.empty(nn)
    ncentre, nchild = np.empty((nn, 3)), np.empty((nn, 8), np.int32)
    fn("nodes")(h, nfirst.ctypes.data_as(ip), ncount.ctypes.data_as(ip), nhalf.ctypes.data_as(dp),
                ncentre.ctypes.data_as(dp), nchild.ctypes.data_as(ip))
    return BHSet(x=x[perm], m=m[perm], perm=perm, gfirst=gfirst, gcount=gcount, gcentre=gcentre, ghalf=ghalf,
                 poff=poff, pidx=pidx[:npl], coff=coff, cidx=cidx[:ncl], ccom=ccom, cmass=cmass, cquad=cquad,
                 nfirst=nfirst, ncount=ncount, nhalf=nhalf, ncentre=ncentre, nchild=nchild, eps=eps, theta=theta,
                 nleaf=nleaf, ncrit=ncrit)


def bh_tree(x: np.ndarray, m: np.ndarray, theta: float = 0.5, nleaf: int = 16, ncrit: int = 256,
            eps: float = 1e-3) -> BHSet:
    """Octree, moments and interaction lists of particles x (n x 3), m (n) with the reference's
    rules, built on the host (drivers/pgb_bhtree.c)."""
    import ctypes as C
    from . import ffi
    L = C.CDLL(ffi.lib_path("libpgbdrv.so"), mode=C.RTLD_LOCAL)
    dp = C.POINTER(C.c_double)
    L.bh_build.argtypes = [C.c_int, dp, dp, C.c_double, C.c_int, C.c_int]
    L.bh_build.restype = C.c_void_p
    L.bh_free.argtypes = [C.c_void_p]
    x = np.ascontiguousarray(x, np.float64)
    m = np.ascontiguousarray(m, np.float64)
    h = L.bh_build(len(m), x.ctypes.data_as(dp), m.ctypes.data_as(dp), theta, nleaf, ncrit)
    if not h:
        raise MemoryError("bh_build failed")
    try:
        return _bh_read(L, "bh_", h, x, m, eps, theta, nleaf, ncrit)
    finally:
        L.bh_free(h)


class GpuTree:
    """The same tree built on the GPU (lib/libpgbtree.so, pgbt_*): .set() reads it back as a
    BHSet, .device() gives the device pointers of the batched force launch, .build_ms the
    device time of the build."""

    def __init__(self, x: np.ndarray, m: np.ndarray, theta: float = 0.5, nleaf: int = 16, ncrit: int = 256,
                 eps: float = 1e-3):
        import ctypes as C
        from . import ffi
        self.L = L = C.CDLL(ffi.lib_path("libpgbtree.so"), mode=C.RTLD_LOCAL)
        dp, vp = C.POINTER(C.c_double), C.c_void_p
        L.pgbt_build.argtypes = [C.c_int, dp, dp, C.c_double, C.c_int, C.c_int]
        L.pgbt_build.restype = vp
        L.pgbt_free.argtypes = [vp]
        L.pgbt_build_ms.argtypes = [vp]
        L.pgbt_build_ms.restype = C.c_float
        L.pgbt_device.argtypes = [vp] + [C.POINTER(vp)] * 7
        L.pgbt_last_error.argtypes = [C.c_char_p, C.c_int]
        L.pgbt_nnodes.argtypes = [vp]
        L.pgbt_nnodes.restype = C.c_int
        L.pgbt_ngroups.argtypes = [vp]
        L.pgbt_ngroups.restype = C.c_int
        self.x = np.ascontiguousarray(x, np.float64)
        self.m = np.ascontiguousarray(m, np.float64)
        self.args = (eps, theta, nleaf, ncrit)
        self.h = L.pgbt_build(len(self.m), self.x.ctypes.data_as(dp), self.m.ctypes.data_as(dp), theta, nleaf, ncrit)
        if not self.h:
            buf = C.create_string_buffer(512)
            L.pgbt_last_error(buf, 512)
            raise RuntimeError(f"pgbt_build failed: {buf.value.decode()}")
        self.build_ms = L.pgbt_build_ms(self.h)

    def rebuild(self, x: np.ndarray, m: np.ndarray):
        """Rebuild the tree for new particles (same parameters), reusing its device buffers."""
        import ctypes as C
        dp = C.POINTER(C.c_double)
        self.L.pgbt_rebuild.argtypes = [C.c_void_p, C.c_int, dp, dp]
        self.x = np.ascontiguousarray(x, np.float64)
        self.m = np.ascontiguousarray(m, np.float64)
        if self.L.pgbt_rebuild(self.h, len(self.m), self.x.ctypes.data_as(dp), self.m.ctypes.data_as(dp)):
            raise RuntimeError("pgbt_rebuild failed")
        self.build_ms = self.L.pgbt_build_ms(self.h)

    def set(self) -> BHSet:
        return _bh_read(self.L, "pgbt_", self.h, self.x, self.m, *self.args)

    def records(self):
        """Host copies of the force-launch records: particles (n, 4), cells (nn, 4), quadrupoles (nn, 8)."""
        import ctypes as C
        nn = self.L.pgbt_nnodes(self.h)
        part = np.empty((len(self.m), 4), np.float32)
        cell, cquad = np.empty((nn, 4), np.float32), np.empty((nn, 8), np.float32)
        fp = C.POINTER(C.c_float)
        self.L.pgbt_records.argtypes = [C.c_void_p, fp, fp, fp]
        self.L.pgbt_records(self.h, part.ctypes.data_as(fp), cell.ctypes.data_as(fp), cquad.ctypes.data_as(fp))
        return part, cell, cquad

    def irecords(self, eps2: float, out_ptr: int):
        """Write the i-records float4 (x, y, z, eps2) in tree order to device memory out_ptr."""
        import ctypes as C
        self.L.pgbt_irecords.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
        if self.L.pgbt_irecords(self.h, eps2, out_ptr):
            raise RuntimeError("pgbt_irecords failed")

    def items(self):
        """Work items (i_offset, i_count, j_offset, j_count) of the point-mass and the cell lists."""
        import ctypes as C
        ng = self.L.pgbt_ngroups(self.h)
        first, count = np.empty(ng, np.int32), np.empty(ng, np.int32)
        poff, coff = np.empty(ng + 1, np.int64), np.empty(ng + 1, np.int64)
        ip, lp = C.POINTER(C.c_int), C.POINTER(C.c_longlong)
        self.L.pgbt_group_table.argtypes = [C.c_void_p, ip, ip, lp, lp]
        self.L.pgbt_group_table(self.h, first.ctypes.data_as(ip), count.ctypes.data_as(ip), poff.ctypes.data_as(lp),
                                coff.ctypes.data_as(lp))
        mk = lambda off: np.stack([first, count, off[:-1], np.diff(off)], 1).astype(np.int32)  # noqa: E731
        return mk(poff), mk(coff)

    def device(self):
        import ctypes as C
        ptrs = [C.c_void_p() for _ in range(7)]
        self.L.pgbt_device(self.h, *[C.byref(p) for p in ptrs])
        return dict(zip(("part", "cell", "cquad", "poff", "pidx", "coff", "cidx"), (p.value for p in ptrs)))

    def close(self):
        if self.h:
            self.L.pgbt_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bh_hernquist(n: int = 1 << 22, seed: int = SEED0 + 3, theta: float = 0.5, nleaf: int = 16, ncrit: int = 256,
                 eps: float = 1e-3, rmax: float = 100.0) -> BHSet:
    """Hernquist sphere (a = 1, M = 1, truncated at rmax), equal masses, float32-rounded
    positions; octree with theta = 0.5, groups of <= ncrit = 256 and leaves of <= nleaf = 16
    particles (the reference leaves nleaf to the user, source.cpp:1287-1289)."""
    rng = Rng(seed)
    x = _isotropic(rng, hernquist_radii(rng, n, rmax)).astype(np.float32).astype(np.float64)
    m = np.full(n, np.float32(1.0 / n), np.float64)
    return bh_tree(x, m, theta, nleaf, ncrit, eps)
