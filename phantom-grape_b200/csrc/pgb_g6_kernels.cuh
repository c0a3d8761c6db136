// pgb_g6_kernels.cuh -- PG6 (GRAPE-6) j-predictor and 4th-order Hermite force / jerk /
// potential / nearest-neighbour / neighbour-list kernels for sm_100a.
//
// Precision layout (the reference's, PG6/libpg6/gravity.c:311-420): the predictor and the
// relative position x_j - x_i are FP64; the difference is rounded to FP32 and everything after
// it (r^2, rsqrt, velocity difference, products) is FP32.  Sums are FP32 over at most 128
// terms (G6_FOLD) and then added into FP64 sums; split j-ranges are reduced in FP64 in chunk
// order.
//
// Per pair, with the pair scale s of 1/r (pgb::pair_scale: the MUFU estimate 1/r, or -2/r in the
// reference's Newton-refined form; self pair masked by index):
//   pot_sum += m s, acc_sum += (m s^3) dx, jrk_sum += (m s^3) (dv + S_JERK s^2 (dx.dv) dx)
// and finally acc = S_ACC acc_sum, jerk = S_ACC jrk_sum, pot = S_POT pot_sum (for s = -2/r:
// -1/8, -1/8, 1/2 and S_JERK = -3/4, phantom_g6.c:200-208), i.e.
//   acc = sum m dx/r^3, jerk = sum m (dv/r^3 - 3 (dx.dv) dx/r^5), pot = -sum m/r.
// Nearest neighbour: the smallest key k = nn_key(s) over j != i (reported as q = -2/r_soft);
// ties -> smallest j address.  Neighbour list: j with k <= key of h_i (softened r <= h_i),
// appended with an atomic counter.
#pragma once

#include "pgb_common.cuh"

namespace pgb {

// j-memory record as stored by g6_set_j_particle (gravity.c:31-40): a2 = acc/2, j6 = jerk/6.
struct G6Ptcl {
    double pos[3], vel[3], acc2[3], jrk6[3];
    double mass, tim;
    int idx, pad[3];
};

// A position as stored for the force kernel: FP64 (x, y, z), or -- the layout of the kernel's
// double-float variant -- a pair of floats per coordinate, hi = fl32(x), lo = fl32(x - hi),
// which represents x to ~2^-48 relative.
union __align__(8) Pos3 {
    struct { double x, y, z; } d;
    struct { float xh, yh, zh, xl, yl, zl; } f;
};

// Predicted j record in HBM and shared memory: 48 bytes, three 16-byte words.
struct __align__(16) G6PredJ {
    Pos3 p;               // words 0-1
    float m;
    int id;
    float vx, vy, vz;     // word 2
    float pad;
};

// i-particle record: 48 bytes.
struct __align__(16) G6I {
    Pos3 p;
    float vx, vy, vz;
    int id;
    float h2;             // neighbour radius^2 (0: no neighbours)
    float pad;
};

__host__ __device__ inline void split_ff(double x, float& hi, float& lo) {
    hi = (float)x;
    lo = (float)(x - (double)hi);
}

__host__ __device__ inline void store_pos(Pos3& p, double x, double y, double z, bool ff) {
    if (ff) {
        split_ff(x, p.f.xh, p.f.xl);
        split_ff(y, p.f.yh, p.f.yl);
        split_ff(z, p.f.zh, p.f.zl);
    } else {
        p.d.x = x;
        p.d.y = y;
        p.d.z = z;
    }
}

// jadr of a split i-tile's result before g6_resolve_kernel: the start of the j-tile that holds
// the nearest neighbour, with this bit set (j addresses stay below it; -1: no candidate).
constexpr int G6_NN_TILE = 1 << 30;

// Per-i result (final or partial).  key/jadr: nearest-neighbour key and j address.
struct __align__(16) G6Out {
    double ax, ay, az;
    double jx, jy, jz;
    double pot;
    float key;
    int jadr;
};

struct G6Args {
    const G6I* ipart;
    const G6PredJ* jpred;
    float eps2;
    const Task* tasks;
    int ntasks;
    int* task_counter;
    const Group* groups;
    int* group_counters;
    G6Out* partial;        // [rows][itile]
    G6Out* out;            // [.] indexed by absolute i
    int itile;
    // neighbour lists (NBL variant): per absolute i, count and up to maxlen j addresses
    int* nb_count;
    int* nb_list;
    int nb_maxlen;
    // regular mode (tasks == nullptr): one item of reg_ni i against reg_nj j, split into
    // ceil(reg_ni/itile) i-tiles x reg_nch j-chunks, task t = (i-tile t / nch, chunk t % nch)
    int reg_ni = 0, reg_nj = 0, reg_nch = 1;
    // per partial row (zero, self-cleaning): arrival counters of the two-level reduction of
    // groups with many chunks; nullptr: every group is reduced in one level
    int* bundle_counters = nullptr;
    // leave the partial rows of split j-ranges unreduced (the caller's next kernel sums them in
    // chunk order): no arrival counters, fences or last-CTA reduction in this launch
    bool partial_only = false;
    // records in jpred (bounds the nearest-neighbour address lookups of split groups)
    int jn = 0;
};

// The task and group of regular mode (the same decomposition plan_item() writes out).
__device__ __forceinline__ Task regular_task(const G6Args& A, int t) {
    const int nch = A.reg_nch;
    const int it = t / nch, c = t % nch;
    const int i0 = it * A.itile;
    const int nii = min(A.itile, A.reg_ni - i0);
    if (nch == 1) return Task{i0, nii, 0, A.reg_nj, -1, 0, -1, 0};
    const int j0 = (int)((long long)c * A.reg_nj / nch);
    const int j1 = (int)((long long)(c + 1) * A.reg_nj / nch);
    return Task{i0, nii, j0, j1 - j0, it, c, it * nch + c, 0};
}

__device__ __forceinline__ Group regular_group(const G6Args& A, int g) {
    const int i0 = g * A.itile;
    return Group{i0, min(A.itile, A.reg_ni - i0), A.reg_nch, g * A.reg_nch};
}

// FP64 predictor: one thread per j (gravity.c:149-193; velocity stored as float, :168-173).
// ff: store the predicted position in the double-float layout.
__global__ void g6_predict_kernel(const G6Ptcl* __restrict__ p, int nj, double ti, G6PredJ* __restrict__ out,
                                  bool ff) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nj) return;
    const G6Ptcl& P = p[j];
    double dt = ti - P.tim;
    double dt2 = dt * dt, dt3 = dt2 * dt;
    G6PredJ o;
    store_pos(o.p, P.pos[0] + P.vel[0] * dt + P.acc2[0] * dt2 + P.jrk6[0] * dt3,
              P.pos[1] + P.vel[1] * dt + P.acc2[1] * dt2 + P.jrk6[1] * dt3,
              P.pos[2] + P.vel[2] * dt + P.acc2[2] * dt2 + P.jrk6[2] * dt3, ff);
    o.vx = (float)(P.vel[0] + 2.0 * P.acc2[0] * dt + 3.0 * P.jrk6[0] * dt2);
    o.vy = (float)(P.vel[1] + 2.0 * P.acc2[1] * dt + 3.0 * P.jrk6[1] * dt2);
    o.vz = (float)(P.vel[2] + 2.0 * P.acc2[2] * dt + 3.0 * P.jrk6[2] * dt2);
    o.m = (float)P.mass;
    o.id = P.idx;
    o.pad = 0.f;
    out[j] = o;
}

// Sparse j-memory update: jd[idx[k]] = rec[k] (addresses checked against the capacity).
__global__ void g6_scatter_kernel(const G6Ptcl* __restrict__ rec, const int* __restrict__ idx, int n, int cap,
                                  G6Ptcl* __restrict__ jd) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int a = idx[k];
    if (a >= 0 && a < cap) jd[a] = rec[k];
}

// Neighbour lists after the force launch: each i's entries were appended by atomics in
// arrival order; this kernel (one CTA per i) sorts a list of count <= nbmax entries by j address
// in shared memory (bitonic network over P >= count slots, P a power of two) and replaces every
// address by the id stored in the j-memory, so that the list is the reference's (j-address
// order, gravity.c:888-900, ids).  A list longer than nbmax kept only its count and is left
// alone (the host reports the overflow).
__global__ void g6_nb_sort_kernel(const int* __restrict__ nb_count, int* __restrict__ nb_list, int nbmax, int P,
                                  const G6Ptcl* __restrict__ jmem) {
    extern __shared__ int sh_nb[];
    const int c = nb_count[blockIdx.x];
    if (c > nbmax || c <= 0) return;
    int* row = nb_list + (size_t)blockIdx.x * nbmax;
    for (int k = threadIdx.x; k < P; k += blockDim.x) sh_nb[k] = k < c ? row[k] : 0x7fffffff;
    __syncthreads();
    for (int size = 2; size <= P; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int k = threadIdx.x; k < P; k += blockDim.x) {
                const int q = k ^ stride;
                if (q > k) {
                    const bool up = (k & size) == 0;
                    const int a = sh_nb[k], b = sh_nb[q];
                    if ((a > b) == up) {
                        sh_nb[k] = b;
                        sh_nb[q] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int k = threadIdx.x; k < c; k += blockDim.x) row[k] = jmem[sh_nb[k]].idx;
}

// FP32 partial sums cover at most G6_FOLD terms (per thread and i) before they are added into
// the FP64 sums.  Rounding error of the blocked sum alone, acc of a 65536-body Plummer sphere
// (rms relative, against the exact sum of the same FP32 terms): 2.1e-8 for 128 terms, 3.3e-8
// for 256, against 1.7e-8 for the FP32 pair arithmetic itself.  Measured on the largest
// Hermite call (256 x 2 configuration): acc 6.7e-8 -> 5.4e-8 rms against FP64 with no change in
// speed; 64-term blocks (5.0e-8) cost 7 %.
constexpr int G6_FOLD = 128;

struct G6Acc {
    float ax, ay, az, jx, jy, jz, pot;
};

// x_j - x_i rounded to FP32.  FP64 layout: an FP64 subtraction and a conversion (DADD + F2F,
// the reference's own split, gravity.c:316-333).  Double-float layout: (xjh - xih) + (xjl - xil)
// in FP32 -- the hi difference is exact whenever the two positions are within a factor 2
// (Sterbenz), i.e. for every close pair, so the result is fl32(x_j - x_i) to within 1 ulp,
// with three FP32 adds instead of an FP64 add and an F2F on the XU pipe shared with MUFU.
template <bool FF>
__device__ __forceinline__ float rel1(const Pos3& j, const Pos3& i, int c) {
    if constexpr (FF) {
        const float* jf = &j.f.xh;
        const float* iff = &i.f.xh;
        return __fadd_rn(__fsub_rn(jf[c], iff[c]), __fsub_rn(jf[c + 3], iff[c + 3]));
    } else {
        const double* jd = &j.d.x;
        const double* id = &i.d.x;
        return __double2float_rn(jd[c] - id[c]);
    }
}

// The initial nearest-neighbour key (gravity_kernel2's 10 in the reported scale) and the key
// bound of an i-particle's neighbour radius h (gravity.c:688-695: -2/h, or -1e10 when h2 == 0:
// no neighbours; none for a padding slot), both in the kernels' key scale.
constexpr float G6_KEY0 = 10.0f / KEY_OUT;
__device__ __forceinline__ float g6_hkey(bool real, float h2) {
    if (!real) return -INFINITY;
    return h2 == 0.0f ? -1e10f / KEY_OUT : (-2.0f / KEY_OUT) / sqrtf(h2);
}

// The nearest-neighbour key of one pair: nn_key of the pair scale, that of s = 0 for the self
// pair.  Every path of the kernels computes it with exactly these operations, so a key found by
// one pass can be looked up again by another (g6_rescan).
template <bool FF>
__device__ __forceinline__ float g6_key(const G6PredJ& J, const Pos3& I, int idi, float eps2) {
    const float dx = rel1<FF>(J.p, I, 0), dy = rel1<FF>(J.p, I, 1), dz = rel1<FF>(J.p, I, 2);
    const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, eps2)));
    const float s = pair_scale(r2);
    return nn_key((J.id == idi) ? 0.0f : s);
}

// Nearest-neighbour bookkeeping per pair, two forms:
//  * select (NN, !TILEMIN): kmin/kadr updated per pair with strict '<' in j order;
//  * tile minimum (TILEMIN): only tmin = min(tmin, k) per pair (one FMNMX); the caller keeps,
//    per j-tile, whether the tile improved the running minimum and recovers the address of the
//    best tile's first minimal key afterwards (g6_rescan) -- the same (key, smallest address)
//    result with one instruction per pair instead of three.
// SELF: the j-tile may hold the i-particle itself (its id), so the key is masked to 0 for it;
// tiles that cannot hold it skip the compare and select.
template <bool FF, bool NN, bool NBL, bool SELF = true, bool TILEMIN = false>
__device__ __forceinline__ void g6_pair(const G6PredJ& J, int jadr, const Pos3& I, float vxi,
                                        float vyi, float vzi, int idi, float eps2, float hinv, G6Acc& a,
                                        float& kmin, int& kadr, int* nbc, int* nbl, int nbmax) {
    float dx = rel1<FF>(J.p, I, 0);
    float dy = rel1<FF>(J.p, I, 1);
    float dz = rel1<FF>(J.p, I, 2);
    float dvx = J.vx - vxi, dvy = J.vy - vyi, dvz = J.vz - vzi;
    float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, eps2)));
    float s = pair_scale(r2);
    if constexpr (SELF) s = (J.id == idi) ? 0.0f : s;
    if constexpr (NN && TILEMIN) {
        kmin = fminf(kmin, nn_key(s));
    } else if constexpr (NN) {
        const float k = nn_key(s);
        bool lt = k < kmin;
        kmin = lt ? k : kmin;
        kadr = lt ? jadr : kadr;
    }
    if constexpr (NBL) {
        if (nn_key(s) <= hinv) {
            int slot = atomicAdd(nbc, 1);
            if (slot < nbmax) nbl[slot] = jadr;
        }
    }
    a.pot = __fmaf_rn(J.m, s, a.pot);
    float rv = __fmaf_rn(dz, dvz, __fmaf_rn(dy, dvy, dx * dvx));
    float ms = J.m * s;
    float s2 = s * s;
    float mq3 = ms * s2;
    float c = S_JERK * s2 * rv;
    a.ax = __fmaf_rn(mq3, dx, a.ax);
    a.ay = __fmaf_rn(mq3, dy, a.ay);
    a.az = __fmaf_rn(mq3, dz, a.az);
    a.jx = __fmaf_rn(mq3, __fmaf_rn(c, dx, dvx), a.jx);
    a.jy = __fmaf_rn(mq3, __fmaf_rn(c, dy, dvy), a.jy);
    a.jz = __fmaf_rn(mq3, __fmaf_rn(c, dz, dvz), a.jz);
}

// Two i-particles of a thread against one j: the per-i chains exactly as in g6_pair, with the
// accumulations (acc and both jerk products: nine FMAs for the two i) issued as paired FP32
// instructions (FFMA2: each lane rounded exactly as the scalar FFMA, so the results are
// bit-identical to g6_pair).  Paired instructions execute on the heavy half of the FMA pipe
// only; pairing the accumulations alone lowers the issued instructions without making that half
// the bottleneck (pairing the r^2 and dx.dv chains as well measured slower).
struct G6Acc2 {
    float2 ax, ay, az, jx, jy, jz;
    float pot[2];
};

template <bool FF, bool NN, bool NBL, bool SELF = true, bool TILEMIN = false>
__device__ __forceinline__ void g6_pair2(const G6PredJ& J, int jadr, const Pos3* I, const float* vxi,
                                         const float* vyi, const float* vzi, const int* idi, float eps2,
                                         const float* hinv, G6Acc2& a, float* kmin, int* kadr, int* const* nbc,
                                         int* const* nbl, int nbmax) {
    float dx[2], dy[2], dz[2], dvx[2], dvy[2], dvz[2], mq3[2], c[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        dx[k] = rel1<FF>(J.p, I[k], 0);
        dy[k] = rel1<FF>(J.p, I[k], 1);
        dz[k] = rel1<FF>(J.p, I[k], 2);
        dvx[k] = J.vx - vxi[k];
        dvy[k] = J.vy - vyi[k];
        dvz[k] = J.vz - vzi[k];
        float r2 = __fmaf_rn(dz[k], dz[k], __fmaf_rn(dy[k], dy[k], __fmaf_rn(dx[k], dx[k], eps2)));
        float s = pair_scale(r2);
        if constexpr (SELF) s = (J.id == idi[k]) ? 0.0f : s;
        if constexpr (NN && TILEMIN) {
            kmin[k] = fminf(kmin[k], nn_key(s));
        } else if constexpr (NN) {
            const float kk = nn_key(s);
            bool lt = kk < kmin[k];
            kmin[k] = lt ? kk : kmin[k];
            kadr[k] = lt ? jadr : kadr[k];
        }
        if constexpr (NBL) {
            if (nn_key(s) <= hinv[k]) {
                int slot = atomicAdd(nbc[k], 1);
                if (slot < nbmax) nbl[k][slot] = jadr;
            }
        }
        a.pot[k] = __fmaf_rn(J.m, s, a.pot[k]);
        float rv = __fmaf_rn(dz[k], dvz[k], __fmaf_rn(dy[k], dvy[k], dx[k] * dvx[k]));
        float ms = J.m * s;
        float s2 = s * s;
        mq3[k] = ms * s2;
        c[k] = S_JERK * s2 * rv;
    }
    const float2 M = make_float2(mq3[0], mq3[1]), C = make_float2(c[0], c[1]);
    const float2 DX = make_float2(dx[0], dx[1]), DY = make_float2(dy[0], dy[1]), DZ = make_float2(dz[0], dz[1]);
    a.ax = __ffma2_rn(M, DX, a.ax);
    a.ay = __ffma2_rn(M, DY, a.ay);
    a.az = __ffma2_rn(M, DZ, a.az);
    a.jx = __ffma2_rn(M, __ffma2_rn(C, DX, make_float2(dvx[0], dvx[1])), a.jx);
    a.jy = __ffma2_rn(M, __ffma2_rn(C, DY, make_float2(dvy[0], dvy[1])), a.jy);
    a.jz = __ffma2_rn(M, __ffma2_rn(C, DZ, make_float2(dvz[0], dvz[1])), a.jz);
}

// ---- j-paired form ------------------------------------------------------------------------
// One i-particle against two consecutive j (a "j-pair"), with the j-tile in shared memory as
// one array per field (G6TileSoA), so that a 16-byte shared load returns a field of four
// consecutive j: every paired FP32 operand is then a natural register pair -- (j, j+1) for the
// j fields, a loop-invariant (v, v) for the i fields.  The double-float relative coordinates
// (nine FADD2 per j-pair), the velocity differences (three), r^2 and dx.dv (three FFMA2 each),
// the potential and the factors m s, s^2, m s^3 and S_JERK s^2 (dx.dv) (six) and the nine
// accumulations issue paired: 33 paired FP32 instructions per j-pair, only the rsqrt (and the
// Newton step's 3 operations), the self select and the key minimum stay per lane.  Measured on
// the largest Hermite call: 4.69 ms, against 4.75 ms with the potential scalar, 4.82 ms with
// all six factors scalar, 4.93 ms with r^2 and dx.dv scalar as well, 4.99 ms with the velocity
// differences scalar too and 5.10 ms with the relative coordinates scalar also.
// The two lanes of each accumulator sum the even and the odd j of the tile; they are added
// into the FP64 sums one after the other at every fold.  Per pair the key q is bit-identical
// to g6_key (FADD2 rounds each lane as FADD does).
struct G6IPair {
    float2 nxh, nyh, nzh, nxl, nyl, nzl;   // -x_i (hi, lo) of each coordinate, in both lanes
    float vx, vy, vz;
    int id;
};

template <int NT>
struct G6TileSoA {
    float xh[NT], yh[NT], zh[NT], xl[NT], yl[NT], zl[NT];
    float m[NT], vx[NT], vy[NT], vz[NT];
    int id[NT];
};

template <bool NN, bool SELF>
__device__ __forceinline__ void g6_jpair(float2 xh, float2 yh, float2 zh, float2 xl, float2 yl, float2 zl,
                                         float2 m, float2 vx, float2 vy, float2 vz, int2 jid,
                                         const G6IPair& I, float eps2, G6Acc2& a, float& tmin) {
    const float2 dx = __fadd2_rn(__fadd2_rn(xh, I.nxh), __fadd2_rn(xl, I.nxl));
    const float2 dy = __fadd2_rn(__fadd2_rn(yh, I.nyh), __fadd2_rn(yl, I.nyl));
    const float2 dz = __fadd2_rn(__fadd2_rn(zh, I.nzh), __fadd2_rn(zl, I.nzl));
    // v_j - v_i as v_j + (-v_i): each lane rounded as the scalar subtraction
    const float2 dvx = __fadd2_rn(vx, make_float2(-I.vx, -I.vx));
    const float2 dvy = __fadd2_rn(vy, make_float2(-I.vy, -I.vy));
    const float2 dvz = __fadd2_rn(vz, make_float2(-I.vz, -I.vz));
    // r^2 and dx.dv of both j, paired
    const float2 r2v = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, make_float2(eps2, eps2))));
    const float2 rvv = __ffma2_rn(dz, dvz, __ffma2_rn(dy, dvy, __fmul2_rn(dx, dvx)));
    float2 sv;
    const float* mp = &m.x;
    const int* idp = &jid.x;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        float s = pair_scale((&r2v.x)[h]);
        if constexpr (SELF) s = (idp[h] == I.id) ? 0.0f : s;
        if constexpr (NN) tmin = fminf(tmin, nn_key(s));
        (&sv.x)[h] = s;
    }
    {
        float2 P = make_float2(a.pot[0], a.pot[1]);
        P = __ffma2_rn(m, sv, P);
        a.pot[0] = P.x;
        a.pot[1] = P.y;
    }
    const float2 s2 = __fmul2_rn(sv, sv);
    const float2 mq3 = __fmul2_rn(__fmul2_rn(m, sv), s2);
    const float2 c = __fmul2_rn(__fmul2_rn(make_float2(S_JERK, S_JERK), s2), rvv);
    a.ax = __ffma2_rn(mq3, dx, a.ax);
    a.ay = __ffma2_rn(mq3, dy, a.ay);
    a.az = __ffma2_rn(mq3, dz, a.az);
    a.jx = __ffma2_rn(mq3, __ffma2_rn(c, dx, dvx), a.jx);
    a.jy = __ffma2_rn(mq3, __ffma2_rn(c, dy, dvy), a.jy);
    a.jz = __ffma2_rn(mq3, __ffma2_rn(c, dz, dvz), a.jz);
}

// The j-paired form for two i, stage-ordered: the four j-pair chains of a j-quad (two i x two
// j-pairs) advanced together stage by stage -- relative coordinates, dv and r^2, the eight
// rsqrt and the scales s, the paired potential, factors and accumulations -- which hands the scheduler
// independent work in every stage (largest Hermite call 5.65 against 5.77 ms for the chain-by-
// chain order of g6_jpair; the autotuner chooses between them per call size).  The same
// operations as g6_jpair on the same values: bit-identical results.
template <bool NN, bool SELF>
__device__ __forceinline__ void g6_jquad2(const float4& XH, const float4& YH, const float4& ZH, const float4& XL,
                                          const float4& YL, const float4& ZL, const float4& M, const float4& VX,
                                          const float4& VY, const float4& VZ, const int4& ID, const G6IPair* IP,
                                          float eps2, G6Acc2* a, float* tmin) {
    float2 dx[4], dy[4], dz[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const G6IPair& I = IP[c >> 1];
        const bool hi = c & 1;
        const float2 xh = hi ? make_float2(XH.z, XH.w) : make_float2(XH.x, XH.y);
        const float2 yh = hi ? make_float2(YH.z, YH.w) : make_float2(YH.x, YH.y);
        const float2 zh = hi ? make_float2(ZH.z, ZH.w) : make_float2(ZH.x, ZH.y);
        const float2 xl = hi ? make_float2(XL.z, XL.w) : make_float2(XL.x, XL.y);
        const float2 yl = hi ? make_float2(YL.z, YL.w) : make_float2(YL.x, YL.y);
        const float2 zl = hi ? make_float2(ZL.z, ZL.w) : make_float2(ZL.x, ZL.y);
        dx[c] = __fadd2_rn(__fadd2_rn(xh, I.nxh), __fadd2_rn(xl, I.nxl));
        dy[c] = __fadd2_rn(__fadd2_rn(yh, I.nyh), __fadd2_rn(yl, I.nyl));
        dz[c] = __fadd2_rn(__fadd2_rn(zh, I.nzh), __fadd2_rn(zl, I.nzl));
    }
    const float vxs[4] = {VX.x, VX.y, VX.z, VX.w}, vys[4] = {VY.x, VY.y, VY.z, VY.w}, vzs[4] = {VZ.x, VZ.y, VZ.z, VZ.w};
    const float ms[4] = {M.x, M.y, M.z, M.w};
    const int ids[4] = {ID.x, ID.y, ID.z, ID.w};
    float r2[8], dvx[8], dvy[8], dvz[8];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const G6IPair& I = IP[c >> 1];
        const int j0 = (c & 1) << 1;
        const float2 vx = __fadd2_rn(make_float2(vxs[j0], vxs[j0 + 1]), make_float2(-I.vx, -I.vx));
        const float2 vy = __fadd2_rn(make_float2(vys[j0], vys[j0 + 1]), make_float2(-I.vy, -I.vy));
        const float2 vz = __fadd2_rn(make_float2(vzs[j0], vzs[j0 + 1]), make_float2(-I.vz, -I.vz));
        dvx[2 * c] = vx.x; dvx[2 * c + 1] = vx.y;
        dvy[2 * c] = vy.x; dvy[2 * c + 1] = vy.y;
        dvz[2 * c] = vz.x; dvz[2 * c + 1] = vz.y;
    }
    float rvv[8];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float2 r = __ffma2_rn(dz[c], dz[c], __ffma2_rn(dy[c], dy[c], __ffma2_rn(dx[c], dx[c], make_float2(eps2, eps2))));
        r2[2 * c] = r.x;
        r2[2 * c + 1] = r.y;
        const float2 v = __ffma2_rn(dz[c], make_float2(dvz[2 * c], dvz[2 * c + 1]),
                                    __ffma2_rn(dy[c], make_float2(dvy[2 * c], dvy[2 * c + 1]),
                                               __fmul2_rn(dx[c], make_float2(dvx[2 * c], dvx[2 * c + 1]))));
        rvv[2 * c] = v.x;
        rvv[2 * c + 1] = v.y;
    }
    float y[8];
#pragma unroll
    for (int l = 0; l < 8; l++) y[l] = mufu_rsqrt(r2[l]);
    float sv[8];
#pragma unroll
    for (int l = 0; l < 8; l++) {
        const int c = l >> 1, h = l & 1;
        const G6IPair& I = IP[c >> 1];
        const int jj = ((c & 1) << 1) + h;
        float s = pair_scale_from_rsqrt(r2[l], y[l]);
        if constexpr (SELF) s = (ids[jj] == I.id) ? 0.0f : s;
        if constexpr (NN) tmin[c >> 1] = fminf(tmin[c >> 1], nn_key(s));
        sv[l] = s;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        G6Acc2& A = a[c >> 1];
        const int j0 = (c & 1) << 1;
        const float2 S = make_float2(sv[2 * c], sv[2 * c + 1]), MJ = make_float2(ms[j0], ms[j0 + 1]);
        {
            float2 P = make_float2(A.pot[0], A.pot[1]);
            P = __ffma2_rn(MJ, S, P);
            A.pot[0] = P.x;
            A.pot[1] = P.y;
        }
        const float2 S2 = __fmul2_rn(S, S);
        const float2 M3 = __fmul2_rn(__fmul2_rn(MJ, S), S2);
        const float2 C2 = __fmul2_rn(__fmul2_rn(make_float2(S_JERK, S_JERK), S2), make_float2(rvv[2 * c], rvv[2 * c + 1]));
        A.ax = __ffma2_rn(M3, dx[c], A.ax);
        A.ay = __ffma2_rn(M3, dy[c], A.ay);
        A.az = __ffma2_rn(M3, dz[c], A.az);
        A.jx = __ffma2_rn(M3, __ffma2_rn(C2, dx[c], make_float2(dvx[2 * c], dvx[2 * c + 1])), A.jx);
        A.jy = __ffma2_rn(M3, __ffma2_rn(C2, dy[c], make_float2(dvy[2 * c], dvy[2 * c + 1])), A.jy);
        A.jz = __ffma2_rn(M3, __ffma2_rn(C2, dz[c], make_float2(dvz[2 * c], dvz[2 * c + 1])), A.jz);
    }
}

// The address of the first j of tile [jb, jb + ne) (every JL-th from lane jl) whose key equals
// kmin -- the nearest neighbour found by a tile-minimum pass (see g6_pair).  The records are read
// again from the predicted j-set (L2-resident).  Returns -1 if none matches, which cannot
// happen for a key that the same arithmetic produced.
template <bool FF>
__device__ __forceinline__ int g6_rescan(const G6PredJ* __restrict__ jpred, int jb, int ne, const Pos3& I, int idi,
                                         float eps2, float kmin) {
    int j = 0;
    for (; j + 3 < ne; j += 4) {
        G6PredJ J[4];
#pragma unroll
        for (int u = 0; u < 4; u++) J[u] = jpred[jb + j + u];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (g6_key<FF>(J[u], I, idi, eps2) == kmin) return jb + j + u;
    }
    for (; j < ne; j++)
        if (g6_key<FF>(jpred[jb + j], I, idi, eps2) == kmin) return jb + j;
    return -1;
}

__device__ __forceinline__ G6Out g6_finish(const G6Out& s) {
    G6Out o;
    o.ax = S_ACC * s.ax;
    o.ay = S_ACC * s.ay;
    o.az = S_ACC * s.az;
    o.jx = S_ACC * s.jx;
    o.jy = S_ACC * s.jy;
    o.jz = S_ACC * s.jz;
    o.pot = S_POT * s.pot;
    o.key = key_out(s.key);
    o.jadr = s.jadr;
    return o;
}

// (key, j address) order of the nearest-neighbour search: smaller key, ties to the smaller
// address -- independent of the order in which partial results are combined.
__device__ __forceinline__ bool nn_better(float k1, int a1, float k0, int a0) {
    return k1 < k0 || (k1 == k0 && (unsigned)a1 < (unsigned)a0);
}

__device__ __forceinline__ void out_add(G6Out& s, const G6Out& v) {
    s.ax += v.ax; s.ay += v.ay; s.az += v.az;
    s.jx += v.jx; s.jy += v.jy; s.jz += v.jz;
    s.pot += v.pot;
    if (nn_better(v.key, v.jadr, s.key, s.jadr)) {
        s.key = v.key;
        s.jadr = v.jadr;
    }
}

// Chunks per bundle of the two-level group reduction: ceil(sqrt(nchunk)) for groups of more
// than 16 chunks (when bundle counters exist), else the whole group in one level.
__device__ __forceinline__ int bundle_size(int nchunk, bool two_level) {
    if (!two_level || nchunk <= 16) return nchunk;
    int b = (int)sqrtf((float)nchunk);
    while (b * b < nchunk) b++;
    return b;
}

// A G6Out is four 16-byte words: (ax, ay) (az, jx) (jy, jz) (pot, key|jadr).  Word 3's second
// half packs the nearest-neighbour key (low 32 bits) and j address (high 32 bits).
__device__ __forceinline__ double2 word_add(double2 s, double2 v, bool w3) {
    s.x += v.x;
    if (!w3) {
        s.y += v.y;
    } else {
        const long long a = __double_as_longlong(s.y), b = __double_as_longlong(v.y);
        if (nn_better(__int_as_float((int)(b & 0xffffffffLL)), (int)(b >> 32),
                      __int_as_float((int)(a & 0xffffffffLL)), (int)(a >> 32)))
            s.y = v.y;
    }
    return s;
}

__device__ __forceinline__ double2 word_zero(bool w3) {
    // word 3: key +inf, address -1 (every real candidate is better)
    return make_double2(0.0, w3 ? __longlong_as_double((long long)0xffffffff7f800000ULL) : 0.0);
}

// A finished result word: the sums times the scale's constants, the key as reported.
__device__ __forceinline__ double2 word_finish(double2 v, bool w3) {
    if (!w3) return make_double2(S_ACC * v.x, S_ACC * v.y);
    const long long b = __double_as_longlong(v.y);
    const float k = key_out(__int_as_float((int)(b & 0xffffffffLL)));
    const long long packed = (b & ~0xffffffffLL) | (long long)(unsigned)__float_as_int(k);
    return make_double2(S_POT * v.x, __longlong_as_double(packed));
}

// Sum `nrows` partial rows (row r at base + r*stride G6Out) word by word over the words
// [wbeg, wbeg + nw) of a row (4 words per G6Out): thread (g, f) of R <= NT/nw row groups sums word
// f of rows g, g+R, ... (coalesced 16-byte loads through L2, up to eight rows in flight), then
// the R group sums are added in group order through shared memory W (NT words).  The order is
// fixed for a given (NT, nw, nrows): deterministic.  finish: write the final scaled result (acc,
// jerk x -1/8, pot x 1/2) instead of the raw sum.  dst (same word indexing) may be row 0 itself:
// every word is read before it is written.
template <int NT>
__device__ __forceinline__ void reduce_rows(const G6Out* base, size_t stride, int nrows, int wbeg, int nw,
                                            G6Out* dst, bool finish, double2* W) {
    // row groups: as many as the threads allow, but no more than the rows and at most 8 (their
    // sums are combined serially)
    const int R = (2 * nw <= NT) ? min(min(NT / nw, nrows), 8) : 1;
    const double2* src = reinterpret_cast<const double2*>(base);
    double2* out = reinterpret_cast<double2*>(dst);
    const size_t wstride = 4 * stride;
    for (int k0 = 0; k0 < nw; k0 += (R > 1 ? nw : NT)) {
        const int g = (R > 1) ? threadIdx.x / nw : 0;
        const int k = (R > 1) ? threadIdx.x % nw : k0 + threadIdx.x;
        const int f = wbeg + k;
        const bool w3 = (f & 3) == 3;
        double2 s0 = word_zero(w3);
        if (g < R && k < nw) {
            double2 s1 = s0, s2 = s0, s3 = s0;
            const double2* col = src + f;
            int r = g;
            // eight rows' loads in flight (L2 latency bound), four running sums
            for (; r + 7 * R < nrows; r += 8 * R) {
                double2 v[8];
#pragma unroll
                for (int u = 0; u < 8; u++) v[u] = __ldcg(col + (size_t)(r + u * R) * wstride);
                s0 = word_add(word_add(s0, v[0], w3), v[4], w3);
                s1 = word_add(word_add(s1, v[1], w3), v[5], w3);
                s2 = word_add(word_add(s2, v[2], w3), v[6], w3);
                s3 = word_add(word_add(s3, v[3], w3), v[7], w3);
            }
            for (; r + 3 * R < nrows; r += 4 * R) {
                const double2 v0 = __ldcg(col + (size_t)r * wstride);
                const double2 v1 = __ldcg(col + (size_t)(r + R) * wstride);
                const double2 v2 = __ldcg(col + (size_t)(r + 2 * R) * wstride);
                const double2 v3 = __ldcg(col + (size_t)(r + 3 * R) * wstride);
                s0 = word_add(s0, v0, w3);
                s1 = word_add(s1, v1, w3);
                s2 = word_add(s2, v2, w3);
                s3 = word_add(s3, v3, w3);
            }
            for (; r < nrows; r += R) s0 = word_add(s0, __ldcg(col + (size_t)r * wstride), w3);
            s0 = word_add(s0, s1, w3);
            s0 = word_add(s0, s2, w3);
            s0 = word_add(s0, s3, w3);
        }
        if (R > 1) {
            __syncthreads();
            W[threadIdx.x] = s0;
            __syncthreads();
            if (threadIdx.x >= nw) continue;
            for (int q = 1; q < R; q++) s0 = word_add(s0, W[q * nw + threadIdx.x], w3);
        } else if (k >= nw) {
            continue;
        }
        if (finish) s0 = word_finish(s0, w3);
        out[f] = s0;
    }
}

template <bool B>
struct BoolC {
    static constexpr bool value = B;
};

// Shared memory of a g6_kernel CTA: the j-tile (as records, or as field arrays in the j-paired
// form, which also keeps its threads' FP64 sums there: 7 per i) and, after the tile loop, NT
// G6Out for the lane and group reductions.
template <int NT, int IPT, bool JP>
constexpr int g6_smem_bytes() {
    return JP ? (int)((sizeof(G6TileSoA<NT>) + 15) / 16 * 16 + 7 * IPT * NT * sizeof(double))
              : NT * (int)sizeof(G6Out);
}

// Thread layout of a CTA: NT threads = JL j-lanes x ISL i-slots (ISL = NT/JL, whole warps per
// lane so that the shared-memory j reads stay warp-broadcasts).  A thread owns IPT i-particles
// li = slot + k*ISL of the task's i-tile (ITILE = ISL*IPT) and every JL-th j of each j-tile.
// The j-lanes are summed in lane order through shared memory at the end of the task.
//
// g6_task: one task (an i-tile against a j-range) by the whole CTA; smem holds NT G6Out.  A task
// of a split j-range (T.group >= 0) writes its partial sums to partial row T.slot; otherwise the
// final result to A.out.  Returns with the CTA's shared memory free for reuse after a barrier.
//
// Per j-tile the CTA first tests whether the tile can hold one of the task's i-particles
// (a j id inside the i-tile's id range, one __syncthreads_or at the staging barrier); only such
// tiles run the self-pair mask.  With two i per thread (IPT even) the nearest neighbour is
// found as a tile minimum (see g6_pair) and its address recovered once per i and task by
// g6_rescan.  JP selects the j-paired form (1: g6_jpair, 2: g6_jquad2 for two i per thread;
// double-float positions, no neighbour lists, one j-lane); otherwise the j-tile is an array of
// G6PredJ records.
template <int NT, int IPT, int JL, bool FF, bool NN, bool NBL, int JP = 0>
__device__ __forceinline__ void g6_task(const G6Args& A, const Task& T, unsigned char* smem) {
    static_assert(JL == 1 || IPT == 1, "j-lanes are used with one i per thread");
    constexpr int ISL = NT / JL;
    constexpr bool PAIRED = (IPT % 2 == 0);
    constexpr bool USE_JP = JP && FF && !NBL && (IPT == 2 || IPT == 4) && JL == 1;
    constexpr bool TILEMIN = NN && !NBL && PAIRED;
    G6PredJ* sj = reinterpret_cast<G6PredJ*>(smem);
    G6TileSoA<NT>* sa = reinterpret_cast<G6TileSoA<NT>*>(smem);
    // j-paired form: the FP64 sums of thread t, i k, component c at Ssh[(k * 7 + c) * NT + t]
    // (updated once per G6_FOLD j; kept out of the registers)
    double* Ssh = reinterpret_cast<double*>(smem + (sizeof(G6TileSoA<NT>) + 15) / 16 * 16);
    G6Out* red = reinterpret_cast<G6Out*>(smem);
    __shared__ int s_idr[2];
    const int slot = threadIdx.x % ISL;
    const int jl = threadIdx.x / ISL;

    Pos3 pi[IPT];
    float vxi[IPT], vyi[IPT], vzi[IPT], hinv[IPT];
    int idi[IPT];
    double S[IPT][7];
    float kmin[IPT], tmin[IPT];
    int kadr[IPT], ktile[IPT];
#pragma unroll
    for (int k = 0; k < IPT; k++) {
        int li = slot + k * ISL;
        int ii = T.i0 + (li < T.ni ? li : 0);
        const G6I P = A.ipart[ii];
        pi[k] = P.p;
        vxi[k] = P.vx; vyi[k] = P.vy; vzi[k] = P.vz;
        idi[k] = P.id;
        // gravity.c:688-695: -2/h, or -1e10 when h2 == 0 (no neighbours); padding lanes none
        hinv[k] = g6_hkey(li < T.ni, P.h2);
#pragma unroll
        for (int c = 0; c < 7; c++) S[k][c] = 0.0;
        kmin[k] = G6_KEY0;   // gravity_kernel2 starts its key at 10 and index at -1 (:495-496)
        kadr[k] = -1;
        tmin[k] = G6_KEY0;
        ktile[k] = -1;
    }
    // the i-tile's id range (padding slots repeat the tile's first i): published to the CTA by
    // the first barrier of the tile loop
    {
        int lo = idi[0], hi = idi[0];
#pragma unroll
        for (int k = 1; k < IPT; k++) {
            lo = min(lo, idi[k]);
            hi = max(hi, idi[k]);
        }
        lo = __reduce_min_sync(0xffffffffu, lo);
        hi = __reduce_max_sync(0xffffffffu, hi);
        __syncthreads();
        if (threadIdx.x == 0) {
            s_idr[0] = 0x7fffffff;
            s_idr[1] = (int)0x80000000;
        }
        __syncthreads();
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_idr[0], lo);
            atomicMax(&s_idr[1], hi);
        }
    }
    G6IPair IP[USE_JP ? IPT : 1];
    if constexpr (USE_JP) {
#pragma unroll
        for (int c = 0; c < 7 * IPT; c++) Ssh[c * NT + threadIdx.x] = 0.0;
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            IP[k].nxh = make_float2(-pi[k].f.xh, -pi[k].f.xh);
            IP[k].nyh = make_float2(-pi[k].f.yh, -pi[k].f.yh);
            IP[k].nzh = make_float2(-pi[k].f.zh, -pi[k].f.zh);
            IP[k].nxl = make_float2(-pi[k].f.xl, -pi[k].f.xl);
            IP[k].nyl = make_float2(-pi[k].f.yl, -pi[k].f.yl);
            IP[k].nzl = make_float2(-pi[k].f.zl, -pi[k].f.zl);
            IP[k].vx = vxi[k];
            IP[k].vy = vyi[k];
            IP[k].vz = vzi[k];
            IP[k].id = idi[k];
        }
    }

    for (int jt = 0; jt < T.nj; jt += NT) {
        const int nt = min(NT, T.nj - jt);
        __syncthreads();
        const int idlo = s_idr[0], idhi = s_idr[1];
        bool mine = false;
        int nt4 = nt;
        if constexpr (USE_JP) {
            // fields of the tile's records, padded to a multiple of 4 with massless copies of
            // the tile's first record (they add exact zeros, and their key repeats that record's)
            nt4 = (nt + 3) & ~3;
            if (threadIdx.x < nt4) {
                const bool real = threadIdx.x < nt;
                const G6PredJ r = A.jpred[T.j0 + jt + (real ? threadIdx.x : 0)];
                sa->xh[threadIdx.x] = r.p.f.xh;
                sa->yh[threadIdx.x] = r.p.f.yh;
                sa->zh[threadIdx.x] = r.p.f.zh;
                sa->xl[threadIdx.x] = r.p.f.xl;
                sa->yl[threadIdx.x] = r.p.f.yl;
                sa->zl[threadIdx.x] = r.p.f.zl;
                sa->m[threadIdx.x] = real ? r.m : 0.0f;
                sa->vx[threadIdx.x] = r.vx;
                sa->vy[threadIdx.x] = r.vy;
                sa->vz[threadIdx.x] = r.vz;
                sa->id[threadIdx.x] = r.id;
                mine = real && r.id >= idlo && r.id <= idhi;
            }
        } else {
            if (threadIdx.x < nt) {
                const G6PredJ r = A.jpred[T.j0 + jt + threadIdx.x];
                sj[threadIdx.x] = r;
                mine = r.id >= idlo && r.id <= idhi;
            }
        }
        const bool self_tile = __syncthreads_or(mine) != 0;
        if constexpr (TILEMIN) {
#pragma unroll
            for (int k = 0; k < IPT; k++) tmin[k] = kmin[k];
        }

        auto run_tile = [&](auto self_c) {
            constexpr bool SELF = decltype(self_c)::value;
            if constexpr (USE_JP) {
                // a full tile that cannot hold one of the task's i runs every fold block with a
                // constant trip count (FULL); self and partial tiles with the run-time count
                constexpr bool FULL = !SELF && NT % G6_FOLD == 0;
                for (int j0 = 0; j0 < (FULL ? NT : nt4); j0 += G6_FOLD) {
                    const int j1 = FULL ? j0 + G6_FOLD : min(j0 + G6_FOLD, nt4);
                    G6Acc2 a[IPT];
                    const float2 z2 = make_float2(0.f, 0.f);
#pragma unroll
                    for (int k = 0; k < IPT; k++) a[k] = G6Acc2{z2, z2, z2, z2, z2, z2, {0.f, 0.f}};
#pragma unroll 1
                    for (int j = j0; j < j1; j += 4) {
                        const float4 XH = *reinterpret_cast<const float4*>(&sa->xh[j]);
                        const float4 YH = *reinterpret_cast<const float4*>(&sa->yh[j]);
                        const float4 ZH = *reinterpret_cast<const float4*>(&sa->zh[j]);
                        const float4 XL = *reinterpret_cast<const float4*>(&sa->xl[j]);
                        const float4 YL = *reinterpret_cast<const float4*>(&sa->yl[j]);
                        const float4 ZL = *reinterpret_cast<const float4*>(&sa->zl[j]);
                        const float4 M = *reinterpret_cast<const float4*>(&sa->m[j]);
                        const float4 VX = *reinterpret_cast<const float4*>(&sa->vx[j]);
                        const float4 VY = *reinterpret_cast<const float4*>(&sa->vy[j]);
                        const float4 VZ = *reinterpret_cast<const float4*>(&sa->vz[j]);
                        int4 ID = make_int4(0, 0, 0, 0);
                        if constexpr (SELF) ID = *reinterpret_cast<const int4*>(&sa->id[j]);
                        if constexpr (JP == 2 && IPT == 2) {
                            g6_jquad2<NN, SELF>(XH, YH, ZH, XL, YL, ZL, M, VX, VY, VZ, ID, IP, A.eps2, a, tmin);
                        } else {
#pragma unroll
                        for (int k = 0; k < IPT; k++) {
                            g6_jpair<NN, SELF>(make_float2(XH.x, XH.y), make_float2(YH.x, YH.y),
                                               make_float2(ZH.x, ZH.y), make_float2(XL.x, XL.y),
                                               make_float2(YL.x, YL.y), make_float2(ZL.x, ZL.y),
                                               make_float2(M.x, M.y), make_float2(VX.x, VX.y),
                                               make_float2(VY.x, VY.y), make_float2(VZ.x, VZ.y),
                                               make_int2(ID.x, ID.y), IP[k], A.eps2, a[k], tmin[k]);
                            g6_jpair<NN, SELF>(make_float2(XH.z, XH.w), make_float2(YH.z, YH.w),
                                               make_float2(ZH.z, ZH.w), make_float2(XL.z, XL.w),
                                               make_float2(YL.z, YL.w), make_float2(ZL.z, ZL.w),
                                               make_float2(M.z, M.w), make_float2(VX.z, VX.w),
                                               make_float2(VY.z, VY.w), make_float2(VZ.z, VZ.w),
                                               make_int2(ID.z, ID.w), IP[k], A.eps2, a[k], tmin[k]);
                        }
                        }
                    }
#pragma unroll
                    for (int k = 0; k < IPT; k++) {
                        const float2* v = &a[k].ax;
#pragma unroll
                        for (int c = 0; c < 6; c++) {
                            double& d = Ssh[(k * 7 + c) * NT + threadIdx.x];
                            d = d + (double)v[c].x + (double)v[c].y;
                        }
                        double& d = Ssh[(k * 7 + 6) * NT + threadIdx.x];
                        d = d + (double)a[k].pot[0] + (double)a[k].pot[1];
                    }
                }
            } else if constexpr (PAIRED) {
                constexpr int NP = IPT / 2;
                int* nbc[IPT];
                int* nbl[IPT];
#pragma unroll
                for (int k = 0; k < IPT; k++) {
                    int li = slot + k * ISL;
                    int gi = T.i0 + (li < T.ni ? li : 0);
                    nbc[k] = NBL ? A.nb_count + gi : nullptr;
                    nbl[k] = NBL ? A.nb_list + (size_t)gi * A.nb_maxlen : nullptr;
                }
                for (int j0 = 0; j0 < nt; j0 += G6_FOLD) {
                    const int j1 = min(j0 + G6_FOLD, nt);
                    G6Acc2 a[NP];
                    const float2 z2 = make_float2(0.f, 0.f);
#pragma unroll
                    for (int p = 0; p < NP; p++) a[p] = G6Acc2{z2, z2, z2, z2, z2, z2, {0.f, 0.f}};
#pragma unroll 2
                    for (int j = j0; j < j1; j++) {
                        const G6PredJ J = sj[j];
                        const int jadr = T.j0 + jt + j;
#pragma unroll
                        for (int p = 0; p < NP; p++)
                            g6_pair2<FF, NN, NBL, SELF, TILEMIN>(J, jadr, pi + 2 * p, vxi + 2 * p, vyi + 2 * p,
                                                                 vzi + 2 * p, idi + 2 * p, A.eps2, hinv + 2 * p, a[p],
                                                                 (TILEMIN ? tmin : kmin) + 2 * p, kadr + 2 * p,
                                                                 nbc + 2 * p, nbl + 2 * p, A.nb_maxlen);
                    }
#pragma unroll
                    for (int p = 0; p < NP; p++) {
                        const float2* v = &a[p].ax;
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int k = 2 * p + h;
#pragma unroll
                            for (int c = 0; c < 6; c++) S[k][c] += (double)(h ? v[c].y : v[c].x);
                            S[k][6] += (double)a[p].pot[h];
                        }
                    }
                }
            } else {
                // blocks of G6_FOLD terms per lane
                for (int j0 = 0; j0 < nt; j0 += G6_FOLD * JL) {
                    const int j1 = min(j0 + G6_FOLD * JL, nt);
                    G6Acc a[IPT];
#pragma unroll
                    for (int k = 0; k < IPT; k++) a[k] = G6Acc{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
                    for (int j = j0 + jl; j < j1; j += JL) {
                        const G6PredJ J = sj[j];
                        const int jadr = T.j0 + jt + j;
#pragma unroll
                        for (int k = 0; k < IPT; k++) {
                            int li = slot + k * ISL;
                            int gi = T.i0 + (li < T.ni ? li : 0);
                            g6_pair<FF, NN, NBL, SELF>(J, jadr, pi[k], vxi[k], vyi[k], vzi[k], idi[k], A.eps2,
                                                       hinv[k], a[k], kmin[k], kadr[k],
                                                       NBL ? A.nb_count + gi : nullptr,
                                                       NBL ? A.nb_list + (size_t)gi * A.nb_maxlen : nullptr,
                                                       A.nb_maxlen);
                        }
                    }
#pragma unroll
                    for (int k = 0; k < IPT; k++) {
                        S[k][0] += (double)a[k].ax;
                        S[k][1] += (double)a[k].ay;
                        S[k][2] += (double)a[k].az;
                        S[k][3] += (double)a[k].jx;
                        S[k][4] += (double)a[k].jy;
                        S[k][5] += (double)a[k].jz;
                        S[k][6] += (double)a[k].pot;
                    }
                }
            }
        };
        if (USE_JP ? (self_tile || nt4 != NT) : self_tile) run_tile(BoolC<true>{});
        else run_tile(BoolC<false>{});

        if constexpr (TILEMIN) {
#pragma unroll
            for (int k = 0; k < IPT; k++)
                if (tmin[k] < kmin[k]) {
                    kmin[k] = tmin[k];
                    ktile[k] = jt;
                }
        }
    }
    if constexpr (TILEMIN) {
        // the address of each i's nearest neighbour: the first j of its best tile with that key
        // (the j-paired form reads its i-record again rather than keep it in registers).  A task
        // of a split j-range leaves the start of its best tile instead, marked G6_NN_TILE: the
        // group's reduction keeps the best (key, tile start) over the chunks -- the same winner
        // as over addresses, the chunks being consecutive j-ranges -- and g6_resolve_kernel
        // looks up that one tile per i after the launch (one lookup per i instead of one per i
        // and chunk, spread over the whole GPU instead of the CTA that completes the group).
        const bool defer = T.group >= 0 && !A.partial_only && A.jn < G6_NN_TILE;
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int li = slot + k * ISL;
            if (defer) {
                if (ktile[k] >= 0) kadr[k] = (T.j0 + ktile[k]) | G6_NN_TILE;
            } else if (li < T.ni && ktile[k] >= 0) {
                if constexpr (USE_JP) {
                    const G6I P = A.ipart[T.i0 + li];
                    kadr[k] = g6_rescan<FF>(A.jpred, T.j0 + ktile[k], min(NT, T.nj - ktile[k]), P.p, P.id, A.eps2,
                                            kmin[k]);
                } else {
                    kadr[k] = g6_rescan<FF>(A.jpred, T.j0 + ktile[k], min(NT, T.nj - ktile[k]), pi[k], idi[k],
                                            A.eps2, kmin[k]);
                }
            }
        }
    }
    if constexpr (USE_JP) {
#pragma unroll
        for (int k = 0; k < IPT; k++)
#pragma unroll
            for (int c = 0; c < 7; c++) S[k][c] = Ssh[(k * 7 + c) * NT + threadIdx.x];
    }

    G6Out* dst_row = (T.group < 0) ? nullptr : A.partial + (size_t)T.slot * A.itile;
#pragma unroll
    for (int k = 0; k < IPT; k++) {
        G6Out o;
        o.ax = S[k][0]; o.ay = S[k][1]; o.az = S[k][2];
        o.jx = S[k][3]; o.jy = S[k][4]; o.jz = S[k][5];
        o.pot = S[k][6];
        o.key = kmin[k];
        o.jadr = kadr[k];
        if constexpr (JL > 1) {
            // sum the j-lanes in lane order (lane 0 holds the CTA's result afterwards)
            __syncthreads();
            red[threadIdx.x] = o;
            __syncthreads();
            if (jl != 0) continue;
            for (int l = 1; l < JL; l++) out_add(o, red[slot + l * ISL]);
        }
        int li = slot + k * ISL;
        if (li >= T.ni) continue;
        if (dst_row) dst_row[li] = o;
        else A.out[T.i0 + li] = g6_finish(o);
    }
}

// The minBlocks of the launch bounds (0: unstated, ptxas's own register choice).  Measured on
// the largest Hermite call (128-thread CTAs), with run-to-run spread of about 1 %: the i-paired
// form takes 5.83 ms with minBlocks 1 (ptxas then uses 128 registers), 6.15 ms unstated (104)
// and 6.09 ms with 4 (123); the j-paired form 5.78 ms unstated (164 registers), 5.91 ms with 3
// (166) and 6.03 ms capped at 128 (spills).  Four i per thread is slower in both forms (6.55 ms).
template <int NT, int IPT, bool JPE>
constexpr int g6_min_ctas() {
    return (!JPE && IPT == 2) ? (NT <= 128 ? 1 : 512 / NT) : 0;   // 256 threads: <= 128 registers, 2 CTAs
}

template <int NT, int IPT, int JL, bool FF, bool NN, bool NBL, int JP = 0>
__global__ void __launch_bounds__(NT, g6_min_ctas<NT, IPT, JP && FF && !NBL && (IPT == 2 || IPT == 4) && JL == 1>())
    g6_kernel(const G6Args A) {
    // j tile during the loop, per-thread results (G6Out) after it
    __shared__ __align__(16) unsigned char
        smem[g6_smem_bytes<NT, IPT, JP && FF && !NBL && (IPT == 2 || IPT == 4) && JL == 1>()];
    __shared__ int s_task, s_flag;

    for (bool first = true;; first = false) {
        int t = next_task(A.task_counter, &s_task, A.ntasks, first);
        if (t >= A.ntasks) break;
        const Task T = A.tasks ? A.tasks[t] : regular_task(A, t);
        g6_task<NT, IPT, JL, FF, NN, NBL, JP>(A, T, smem);
        if (T.group < 0 || A.partial_only) continue;
        const Group G = A.groups ? A.groups[T.group] : regular_group(A, T.group);
        double2* W = reinterpret_cast<double2*>(smem);
        const int B = bundle_size(G.nchunk, A.bundle_counters != nullptr);
        if (B < G.nchunk) {
            // two levels: the last CTA of each bundle of B consecutive chunks sums the bundle's
            // rows into the bundle's first row, the last bundle of the group sums those
            const int b = T.chunk / B;
            const int r0 = G.slot0 + b * B;
            const int nbk = min(B, G.nchunk - b * B);
            if (!group_arrive(A.bundle_counters, r0, nbk, &s_flag)) continue;
            G6Out* row0 = A.partial + (size_t)r0 * A.itile;
            reduce_rows<NT>(row0, (size_t)A.itile, nbk, 0, 4 * G.ni, row0, false, W);
            const int nb = (G.nchunk + B - 1) / B;
            if (!group_arrive(A.group_counters, T.group, nb, &s_flag)) continue;
            reduce_rows<NT>(A.partial + (size_t)G.slot0 * A.itile, (size_t)B * A.itile, nb, 0, 4 * G.ni, A.out + G.i0, true,
                            W);
        } else {
            if (!group_arrive(A.group_counters, T.group, G.nchunk, &s_flag)) continue;
            reduce_rows<NT>(A.partial + (size_t)G.slot0 * A.itile, (size_t)A.itile, G.nchunk, 0, 4 * G.ni, A.out + G.i0,
                            true, W);
        }
    }
}

// The nearest-neighbour addresses of split i-tiles (the tasks' deferred lookups, see g6_task):
// for every result row of a split group whose jadr carries G6_NN_TILE, the first j of the
// marked tile (ntile records, bounded by A.jn) whose key equals the row's key.  G6_RES_LANES
// threads per row each scan ntile / G6_RES_LANES records with all their loads in flight at once
// (one L2 round trip for a 128-record tile), and the smallest match wins.  Block b covers the
// 128 / G6_RES_LANES rows of group b / (itile / rows per block) from row (b % that) x rows.
constexpr int G6_RES_LANES = 16;

template <bool FF>
__global__ void __launch_bounds__(128) g6_resolve_kernel(const G6Args A, int ngroups, int ntile) {
    constexpr int RPB = 128 / G6_RES_LANES;   // rows per block
    const int per_group = (A.itile + RPB - 1) / RPB;
    const int g = blockIdx.x / per_group;
    if (g >= ngroups) return;
    const Group G = A.groups ? A.groups[g] : regular_group(A, g);
    const int li = (blockIdx.x % per_group) * RPB + (int)(threadIdx.x / G6_RES_LANES);
    const int q = threadIdx.x % G6_RES_LANES;
    int tile = -1;
    float key = 0.f;
    if (li < G.ni && G.nchunk > 1) {
        const G6Out& o = A.out[G.i0 + li];
        const int a = o.jadr;
        if (a >= 0 && (a & G6_NN_TILE)) {
            tile = a & (G6_NN_TILE - 1);
            key = key_in(o.key);
        }
    }
    int found = 0x7fffffff;
    if (tile >= 0) {
        const int per = (ntile + G6_RES_LANES - 1) / G6_RES_LANES;
        const int b = tile + q * per, e = min(min(b + per, tile + ntile), A.jn);
        const G6I P = A.ipart[G.i0 + li];
        for (int j0 = b; j0 < e && found == 0x7fffffff; j0 += 8) {
            G6PredJ J[8];
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (j0 + u < e) J[u] = A.jpred[j0 + u];
#pragma unroll
            for (int u = 7; u >= 0; u--)
                if (j0 + u < e && g6_key<FF>(J[u], P.p, P.id, A.eps2) == key) found = j0 + u;
        }
    }
    // the smallest match of the row's lanes (consecutive lanes of one warp)
#pragma unroll
    for (int m = 1; m < G6_RES_LANES; m <<= 1) found = min(found, __shfl_xor_sync(0xffffffffu, found, m));
    if (tile >= 0 && q == 0) A.out[G.i0 + li].jadr = found == 0x7fffffff ? -1 : found;
}

}  // namespace pgb
