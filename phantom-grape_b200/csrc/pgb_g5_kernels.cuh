// pgb_g5_kernels.cuh -- PG5 Newtonian (plain and symmetric softening) and quadrupole-cell
// interaction kernels for sm_100a.
//
// Work decomposition (all kernels): a persistent grid of CTAs pulls Tasks (i-tile x j-chunk)
// from a global counter.  A CTA of NT threads owns NT*IPT i-particles (IPT per thread, kept
// in registers), streams its j-chunk through shared memory in tiles of NT records (one
// coalesced 16-byte load per thread per record word), and every thread reads each j record
// with a broadcast LDS.128.  Sums are accumulated in FP32 over at most 128 terms (G5_FOLD) and
// then added into FP64 accumulators (the cross-block reduction runs in FP64).  Split j-ranges
// write FP64 partial rows; the last CTA of a group reduces them in chunk order.
//
// Formulae, with the pair scale s of 1/r (pgb::pair_scale: the MUFU estimate 1/r by default,
// -2/r in the reference's Newton-refined form with PGB_RSQRT_NEWTON):
//   pot_sum += m s,  acc_sum += (m s^3) dx,  acc = S_ACC acc_sum,  pot_raw = S_POT pot_sum
//   = -sum m/r
// i.e. the reference's GravityKernel accumulators (PG5/newton/libpg5/gravity_avx2.c:95-153:
// phi -= m/r, acc += m dx / r^3) without its 12-bit rsqrt.
#pragma once

#include "pgb_common.cuh"

namespace pgb {

struct G5Args {
    const float4* ipos;     // [.] x, y, z, eps2 of each i-particle
    const float4* jpos;     // [.] x, y, z, m of each j-particle (or cell word 0)
    const float4* jaux;     // symmetric: [.] eps2_j in .x; quad: [2*nc] (q0 q1 q2 q3)(q4 q5 - -)
    const int* jidx;        // nullptr: task j-ranges address jpos/jaux directly; else they address
                            // this index list (interaction lists of a tree: j = jidx[k])
    const Task* tasks;
    int ntasks;
    int* task_counter;      // zero before launch
    const Group* groups;
    int* group_counters;    // zero at allocation, self-cleaning
    double4* partial;       // [rows][itile]
    double4* out;           // [.] (ax, ay, az, pot_raw) per i, indexed by absolute i
    int itile;              // NT*IPT
    // table kind only: force-shape table (f, df/ds) in s = 2 + |dx'|^2, 2^(EXP+FRC) entries
    const float2* table;
    int tbl_size;
    int tbl_shift;          // 23 - FRC_BIT
    float r2cut;            // float with bits (1<<30) | ((tbl_size-1) << tbl_shift)
    double ascale;          // 1 / xscale
};

// kinds
enum { G5_NEWTON = 0, G5_SYMMETRIC = 1, G5_QUAD = 2, G5_TABLE = 3 };
constexpr int G5_TBL_MAX = 4096;   // largest table held in shared memory (32 KB)
// FP32 partial sums cover at most G5_FOLD terms (per thread and i) before they are added into
// the FP64 sums: the rounding of a 128-term FP32 sum stays near the level of the FP32 pair
// arithmetic, a whole 1024-record tile (the direct sum's CTA) adds several times more
// (acc 1.4e-7 rms against FP64 with 1024-term sums, 4.7e-8 with 64-term sums on N = 16384)
constexpr int G5_FOLD = 128;

template <int KIND>
struct JWords { static constexpr int n = (KIND == G5_SYMMETRIC) ? 2 : (KIND == G5_QUAD ? 3 : 1); };

// FP32 block sums per i: (acc, pot) for the point-mass and table kinds; the quadrupole kind
// keeps [0..2] sum (w dr + K s^5 v), [3] sum m s, [4] sum K s^5 D (g5_quad_pair), which g5_fold
// scales and combines into (acc, phi_p + phi_q).
template <int KIND>
struct NAcc { static constexpr int n = KIND == G5_QUAD ? 5 : 4; };

// The cells' moments as staged in shared memory, Q' = G5_QSCALE Q, and the constant K of the
// (Q dr) r^-5 term (g5_quad_pair).  For s = -2/r: Q' = (5/32) Q, which makes the coefficient of
// the monopole and of the D s^7 term of the acceleration the same, and K = -8/5 puts the
// (Q dr) r^-5 term into the same sums; the sums are scaled by G5_QACC (acc) and G5_QP3, G5_QP4
// (phi_p + phi_q = G5_QP3 a[3] + G5_QP4 a[4]).  For s = 1/r the moments are staged 16 times
// larger and K is a quarter: every term is the same term times an exact power of two (K is the
// FP32 -8/5 divided by 4), and the constants remove them.
#ifdef PGB_RSQRT_NEWTON
constexpr float G5_QSCALE = 0.15625f;
constexpr float G5_QK = -1.6f;
constexpr double G5_QACC = -0.125, G5_QP3 = -0.5, G5_QP4 = -(0.1 / (double)(-1.6f));
#else
constexpr float G5_QSCALE = 2.5f;
constexpr float G5_QK = -0.4f;
constexpr double G5_QACC = 1.0, G5_QP3 = 1.0, G5_QP4 = 8.0 * (0.1 / (double)(-1.6f));
#endif

__device__ __forceinline__ float4 scale4(float4 v, float f) {
    return make_float4(f * v.x, f * v.y, f * v.z, f * v.w);
}

// One FP32 block sum (a[NAcc]) into the FP64 sums S = (ax, ay, az, pot) -- pot as each kind's
// raw sum (the quadrupole kind's +sum(phi_p + phi_q), which needs no finishing).
template <int KIND>
__device__ __forceinline__ void g5_fold(double (&S)[4], const float* a) {
    if constexpr (KIND == G5_QUAD) {
#pragma unroll
        for (int c = 0; c < 3; c++) S[c] += G5_QACC * (double)a[c];
        S[3] += G5_QP3 * (double)a[3] + G5_QP4 * (double)a[4];
    } else {
#pragma unroll
        for (int c = 0; c < 4; c++) S[c] += (double)a[c];
    }
}

// The same for paired sums: lane k of each a2[c] (k < 0: both lanes, x then y).
template <int KIND>
__device__ __forceinline__ void g5_fold2(double (&S)[4], const float2* a2, int k) {
    float a[2][NAcc<KIND>::n];
#pragma unroll
    for (int c = 0; c < NAcc<KIND>::n; c++) {
        a[0][c] = k == 1 ? a2[c].y : a2[c].x;
        a[1][c] = a2[c].y;
    }
    if (k < 0) {
        if constexpr (KIND == G5_QUAD) {
#pragma unroll
            for (int c = 0; c < 3; c++) S[c] += G5_QACC * ((double)a[0][c] + (double)a[1][c]);
            S[3] += G5_QP3 * ((double)a[0][3] + (double)a[1][3]) + G5_QP4 * ((double)a[0][4] + (double)a[1][4]);
        } else {
#pragma unroll
            for (int c = 0; c < 4; c++) S[c] = S[c] + (double)a[0][c] + (double)a[1][c];
        }
    } else {
        g5_fold<KIND>(S, a[0]);
    }
}

// A cell's two moment words into shared memory (word 1 at sq[0], word 2 at sq[1]), scaled.
__device__ __forceinline__ void g5_stage_quad(float4* sq, const float4* jaux, int jj) {
    sq[0] = scale4(jaux[2 * jj], G5_QSCALE);
    sq[1] = scale4(jaux[2 * jj + 1], G5_QSCALE);
}

// Table lookup of the cutoff force (PG5/table/libpg5/gravity_kernel_avx2.c:70-124):
// s = min(2 + |dx'|^2, r2cut); the table bin is the float bit pattern of s shifted right by
// 23-FRC_BIT (the exponent and FRC_BIT leading mantissa bits); the bin's node is s with its
// low bits cleared; f = T[bin].x + (s - node) T[bin].y.  `tab` is pre-offset by the bin of 2.0
// so that it can be indexed by the shifted bits directly.  s >= 2 and the clamp (fminf returns
// r2cut for a NaN s) keep every index inside the table.
__device__ __forceinline__ void g5_table_pair(float4 J, float xi, float yi, float zi, const float2* tab,
                                              int shift, float r2cut, float (&a)[4]) {
    float dx = J.x - xi, dy = J.y - yi, dz = J.z - zi;
    float s = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, 2.0f)));
    s = fminf(s, r2cut);
    unsigned u = __float_as_uint(s);
    float node = __uint_as_float((u >> shift) << shift);
    float2 T = tab[u >> shift];
    float f = __fmaf_rn(s - node, T.y, T.x);
    float mf = J.w * f;
    a[0] = __fmaf_rn(mf, dx, a[0]);
    a[1] = __fmaf_rn(mf, dy, a[1]);
    a[2] = __fmaf_rn(mf, dz, a[2]);
}

// The quadrupole cell (c_GravityKernel, PG5/newton_quad/quad/quad_avx2.c:35-149; FP64 form
// source.cpp:1160-1184): with the pair scale s (below q; 1/r by default) and the moments staged
// as Q' = G5_QSCALE Q,
//   v = Q' dr,  D = dr . v,  w = s^3 (m + D s^4),  p = K s^5
//   acc = dr (m r^-3 + (5/2) (dr.Q.dr) r^-7) - (Q dr) r^-5 = G5_QACC (w dr + p v)
//   phi_p + phi_q = m r^-1 + (1/2) (dr.Q.dr) r^-5 = G5_QP3 (m s) + G5_QP4 (p D)
// (s = 1/r: Q' = (5/2) Q, K = -2/5, G5_QACC = 1, G5_QP3 = 1, G5_QP4 = -1/2; s = -2/r: (5/32) Q,
// -8/5, -1/8, -1/2, -1/(10 K)).  34 FP32 operations per pair with s = 1/r (36 with the Newton
// step; the r^-1, r^-2, r^-5 form takes 38); the block sums of w dr + p v, m s and p D are
// scaled and combined in FP64 by g5_fold.  K rounded to FP32 weighs the (Q dr) term 1.5e-8
// (relative) heavier.
__device__ __forceinline__ void g5_quad_pair(float dx, float dy, float dz, float m, float4 Q0, float4 Q1,
                                             float e, float (&a)[5]) {
    // Q0 = q00 q01 q02 q11, Q1 = q12 q22 - -
    const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, e)));
    const float q = pair_scale(r2);
    const float vx = __fmaf_rn(Q0.z, dz, __fmaf_rn(Q0.y, dy, Q0.x * dx));
    const float vy = __fmaf_rn(Q1.x, dz, __fmaf_rn(Q0.w, dy, Q0.y * dx));
    const float vz = __fmaf_rn(Q1.y, dz, __fmaf_rn(Q1.x, dy, Q0.z * dx));
    const float D = __fmaf_rn(dz, vz, __fmaf_rn(dy, vy, dx * vx));
    const float q2 = q * q, q3 = q2 * q, q4 = q2 * q2, p = q4 * (G5_QK * q);
    const float w = q3 * __fmaf_rn(D, q4, m);
    a[0] = __fmaf_rn(w, dx, __fmaf_rn(p, vx, a[0]));
    a[1] = __fmaf_rn(w, dy, __fmaf_rn(p, vy, a[1]));
    a[2] = __fmaf_rn(w, dz, __fmaf_rn(p, vz, a[2]));
    a[3] = __fmaf_rn(m, q, a[3]);
    a[4] = __fmaf_rn(p, D, a[4]);
}

template <int KIND, int NT>
__device__ __forceinline__ void g5_interact(const float4* sj, int j, float xi, float yi, float zi,
                                            float ei, float (&a)[NAcc<KIND>::n]) {
    float4 J = sj[j];
    float dx = J.x - xi, dy = J.y - yi, dz = J.z - zi;
    if constexpr (KIND == G5_QUAD) {
        g5_quad_pair(dx, dy, dz, J.w, sj[NT + 2 * j], sj[NT + 2 * j + 1], ei, a);
    } else {
        float e = ei;
        if constexpr (KIND == G5_SYMMETRIC) e += sj[NT + j].x;  // GravityKernel0
        float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, e)));
        float q = pair_scale(r2);
        float mq = J.w * q;
        float q2 = q * q;
        float mq3 = mq * q2;
        a[3] += mq;
        a[0] = __fmaf_rn(mq3, dx, a[0]);
        a[1] = __fmaf_rn(mq3, dy, a[1]);
        a[2] = __fmaf_rn(mq3, dz, a[2]);
    }
}

__device__ __forceinline__ float& lane_of(float2& v, int k) { return k ? v.y : v.x; }

// Two i-particles of a thread (configurations with IPT >= 2, and the 64-thread CTAs' full
// tiles) against one j record: the per-i chains exactly as g5_interact / g5_table_pair, the
// accumulations of the two i issued as paired FP32 instructions (FFMA2 / FADD2, each lane rounded
// as the scalar instruction: results bit-identical to two g5_interact calls), except the
// quadrupole kind's, whose sums stay scalar (g5_quad_pair per i: its many other FMAs already
// load the FMA pipe's heavy half, which alone executes paired instructions; paired sums measured
// 2 % slower).  a2[c] holds component c of both i.
template <int KIND, int NT>
__device__ __forceinline__ void g5_interact2(const float4* sj, int j, const float* xi, const float* yi,
                                             const float* zi, const float* ei, const float2* tab, int shift,
                                             float r2cut, float2 (&a2)[NAcc<KIND>::n]) {
    const float4 J = sj[j];
    if constexpr (KIND == G5_QUAD) {
        const float4 Q0 = sj[NT + 2 * j];
        const float4 Q1 = sj[NT + 2 * j + 1];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            float a[5];
#pragma unroll
            for (int c = 0; c < 5; c++) a[c] = lane_of(a2[c], k);
            g5_quad_pair(J.x - xi[k], J.y - yi[k], J.z - zi[k], J.w, Q0, Q1, ei[k], a);
#pragma unroll
            for (int c = 0; c < 5; c++) lane_of(a2[c], k) = a[c];
        }
    } else {
        float dx[2], dy[2], dz[2], s0[2], s3[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            dx[k] = J.x - xi[k];
            dy[k] = J.y - yi[k];
            dz[k] = J.z - zi[k];
            if constexpr (KIND == G5_TABLE) {
                float s = __fmaf_rn(dz[k], dz[k], __fmaf_rn(dy[k], dy[k], __fmaf_rn(dx[k], dx[k], 2.0f)));
                s = fminf(s, r2cut);
                unsigned u = __float_as_uint(s);
                float node = __uint_as_float((u >> shift) << shift);
                float2 T = tab[u >> shift];
                float f = __fmaf_rn(s - node, T.y, T.x);
                s0[k] = J.w * f;
            } else {
                float e = ei[k];
                if constexpr (KIND == G5_SYMMETRIC) e += sj[NT + j].x;
                float r2 = __fmaf_rn(dz[k], dz[k], __fmaf_rn(dy[k], dy[k], __fmaf_rn(dx[k], dx[k], e)));
                float q = pair_scale(r2);
                float mq = J.w * q;
                float q2 = q * q;
                s3[k] = mq;
                s0[k] = mq * q2;
            }
        }
        const float2 M = make_float2(s0[0], s0[1]);
        a2[0] = __ffma2_rn(M, make_float2(dx[0], dx[1]), a2[0]);
        a2[1] = __ffma2_rn(M, make_float2(dy[0], dy[1]), a2[1]);
        a2[2] = __ffma2_rn(M, make_float2(dz[0], dz[1]), a2[2]);
        if constexpr (KIND != G5_TABLE) a2[3] = __fadd2_rn(a2[3], make_float2(s3[0], s3[1]));
    }
}

// ---- j-paired form (the 64-thread tree-code CTAs) ------------------------------------------
// One i-particle against two consecutive j records (a "j-pair"), the j-tile held in shared memory
// as one array per field (G5TileSoA), so that a 16-byte shared load returns a field of four
// consecutive j and every paired FP32 operand is a natural register pair: (j, j+1) for the j
// fields, a loop-invariant (v, v) for the i position.  The relative coordinates and the
// accumulations -- and for cells the Q.dr products and D -- issue as paired FP32 instructions on
// the heavy half of the FMA pipe, the rest of the chain stays scalar, loading the two halves
// about equally.  Per pair the arithmetic is g5_interact's, operation for operation (FADD2 /
// FFMA2 round each lane as FADD / FFMA): the two lanes of an accumulator sum the even and the
// odd j.
template <int NT>
struct G5TileSoA {
    float x[NT], y[NT], z[NT], m[NT];
    float q[6][NT];   // cells: G5_QSCALE (q00 q01 q02 q11 q12 q22)
};

__device__ __forceinline__ void g5_newton_jpair(float2 X, float2 Y, float2 Z, float2 M, float2 nx, float2 ny,
                                                float2 nz, float e, float2 (&a)[4]) {
    const float2 dx = __fadd2_rn(X, nx), dy = __fadd2_rn(Y, ny), dz = __fadd2_rn(Z, nz);
    float2 mq, q;
    const float* dxp = &dx.x;
    const float* dyp = &dy.x;
    const float* dzp = &dz.x;
    const float* mp = &M.x;
    float* mqp = &mq.x;
    float* qp = &q.x;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const float r2 = __fmaf_rn(dzp[h], dzp[h], __fmaf_rn(dyp[h], dyp[h], __fmaf_rn(dxp[h], dxp[h], e)));
        qp[h] = pair_scale(r2);
        mqp[h] = mp[h] * qp[h];
    }
    const float2 mq3 = __fmul2_rn(mq, __fmul2_rn(q, q));
    a[3] = __fadd2_rn(a[3], mq);
    a[0] = __ffma2_rn(mq3, dx, a[0]);
    a[1] = __ffma2_rn(mq3, dy, a[1]);
    a[2] = __ffma2_rn(mq3, dz, a[2]);
}

// Q = (q00 q01 q02 q11 q12 q22) of the two cells, as pairs, staged as Q' = G5_QSCALE Q: the
// arithmetic of g5_quad_pair with every FP32 operation paired (the moment products, D, r^2, the
// factors q^2 .. w and the sums; only the rsqrt runs per lane), each lane rounded as the scalar
// operation.  An earlier form computed r^2 and the factors per lane (23 paired + 2 x 10 scalar
// instructions per j-pair); pairing them as well (33 paired) follows the Hermite j-paired forms,
// where the same move made the largest call 5 % faster.
__device__ __forceinline__ void g5_quad_jpair(float2 X, float2 Y, float2 Z, float2 M, const float2 (&Q)[6], float2 nx,
                                              float2 ny, float2 nz, float e, float2 (&a)[5]) {
    const float2 dx = __fadd2_rn(X, nx), dy = __fadd2_rn(Y, ny), dz = __fadd2_rn(Z, nz);
    const float2 vx = __ffma2_rn(Q[2], dz, __ffma2_rn(Q[1], dy, __fmul2_rn(Q[0], dx)));
    const float2 vy = __ffma2_rn(Q[4], dz, __ffma2_rn(Q[3], dy, __fmul2_rn(Q[1], dx)));
    const float2 vz = __ffma2_rn(Q[5], dz, __ffma2_rn(Q[4], dy, __fmul2_rn(Q[2], dx)));
    const float2 D = __ffma2_rn(dz, vz, __ffma2_rn(dy, vy, __fmul2_rn(dx, vx)));
    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, make_float2(e, e))));
    const float2 q = make_float2(pair_scale(r2.x), pair_scale(r2.y));
    const float2 q2 = __fmul2_rn(q, q), q3 = __fmul2_rn(q2, q), q4 = __fmul2_rn(q2, q2);
    const float2 p = __fmul2_rn(q4, __fmul2_rn(make_float2(G5_QK, G5_QK), q));
    const float2 w = __fmul2_rn(q3, __ffma2_rn(D, q4, M));
    a[0] = __ffma2_rn(w, dx, __ffma2_rn(p, vx, a[0]));
    a[1] = __ffma2_rn(w, dy, __ffma2_rn(p, vy, a[1]));
    a[2] = __ffma2_rn(w, dz, __ffma2_rn(p, vz, a[2]));
    a[3] = __ffma2_rn(M, q, a[3]);
    a[4] = __ffma2_rn(p, D, a[4]);
}

// Final scaling of the FP64 sums into (acc, pot_raw).
template <int KIND>
__device__ __forceinline__ double4 g5_finish(double4 s, double ascale) {
    if constexpr (KIND == G5_QUAD) return s;  // quad sums are already (acc, +sum(phi_p+phi_q))
    if constexpr (KIND == G5_TABLE)           // acc *= 1/xscale (gravity_kernel_avx2.c:127-129)
        return make_double4(ascale * s.x, ascale * s.y, ascale * s.z, 0.0);
    return make_double4(S_ACC * s.x, S_ACC * s.y, S_ACC * s.z, S_POT * s.w);
}

__device__ __forceinline__ double4 add4(double4 a, double4 b) {
    return make_double4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// One lane's pass over a j tile: records first, first + STRIDE, ... < nt (STRIDE 0: the
// runtime stride `nl`), accumulated in that order.
template <int KIND, int NT, int IPT, int STRIDE>
__device__ __forceinline__ void g5_jloop(const float4* sj, int first, int nt, const float* xi, const float* yi,
                                         const float* zi, const float* ei, const float2* tab, int shift, float r2cut,
                                         float (&a)[IPT][NAcc<KIND>::n], int nl = 1) {
    const int step = STRIDE > 0 ? STRIDE : nl;
#pragma unroll 4
    for (int j = first; j < nt; j += step) {
        if constexpr (KIND == G5_TABLE) {
            const float4 J = sj[j];
#pragma unroll
            for (int k = 0; k < IPT; k++) g5_table_pair(J, xi[k], yi[k], zi[k], tab, shift, r2cut, a[k]);
        } else {
#pragma unroll
            for (int k = 0; k < IPT; k++) g5_interact<KIND, NT>(sj, j, xi[k], yi[k], zi[k], ei[k], a[k]);
        }
    }
}

template <int KIND, int NT, int IPT, bool JP = false>
__global__ void __launch_bounds__(NT) g5_kernel(G5Args A) {
    constexpr int W = JWords<KIND>::n;   // 16-byte words per j record
    constexpr bool LANES = (IPT == 1 && NT <= 64);
    // the j-paired form: newton point masses and quadrupole cells, one i per thread (the
    // 64-thread CTAs run two for tasks of more than 32 i)
    constexpr bool USE_JP = JP && IPT == 1 && (KIND == G5_NEWTON || KIND == G5_QUAD);
    constexpr int KM = LANES ? 2 : 1;   // i per thread at most in the j-paired form
    constexpr int SJ_RECS = NT * (W > 2 ? W : 2);
    constexpr int SJ_SOA = USE_JP ? (int)((sizeof(G5TileSoA<NT>) + 15) / 16) : 0;
    __shared__ float4 sj[SJ_RECS > SJ_SOA ? SJ_RECS : SJ_SOA];  // also the reduction buffer (double4 x NT)
    __shared__ int s_task, s_flag;
    // table kind: the force table in dynamic shared memory sized to the table (A.tbl_size
    // entries, 8 KB for 1024) for the lifetime of the CTA; the other kinds launch without any
    extern __shared__ float2 g5_dyn_tab[];
    const float2* tab = g5_dyn_tab;
    int shift = 0;
    if constexpr (KIND == G5_TABLE) {
        for (int k = threadIdx.x; k < A.tbl_size; k += NT) g5_dyn_tab[k] = A.table[k];
        shift = A.tbl_shift;
        tab = g5_dyn_tab - (0x40000000u >> shift);  // index by (bits of s) >> shift directly
        __syncthreads();
    }

    // Tasks of more than NT/2 i in the 64-thread one-i-per-thread CTAs: two i per thread
    // (slot and slot + NT/2) and two j-lanes (even and odd records of each tile), so that every
    // j record loaded from shared memory serves two i and their sums take paired FP32
    // instructions; the two lanes' sums are added in lane order.
    auto lanes_pair_task = [&](const Task& T) {
        constexpr int H = NT / 2;
        const int slot = (int)threadIdx.x % H, lane = (int)threadIdx.x / H;
        float xi[2], yi[2], zi[2], ei[2];
        double S[2][4];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int li = slot + k * H;
            const float4 p = A.ipos[T.i0 + (li < T.ni ? li : 0)];
            xi[k] = p.x; yi[k] = p.y; zi[k] = p.z; ei[k] = p.w;
            S[k][0] = S[k][1] = S[k][2] = S[k][3] = 0.0;
        }
        for (int jt = 0; jt < T.nj; jt += NT) {
            const int nt = min(NT, T.nj - jt);
            __syncthreads();
            if (threadIdx.x < nt) {
                const int jk = T.j0 + jt + threadIdx.x;
                const int jj = A.jidx ? __ldg(A.jidx + jk) : jk;
                sj[threadIdx.x] = A.jpos[jj];
                if constexpr (W == 2) sj[NT + threadIdx.x] = A.jaux[jj];
                if constexpr (W == 3) g5_stage_quad(sj + NT + 2 * threadIdx.x, A.jaux, jj);
            }
            __syncthreads();
            // one block: a lane sees at most NT/2 <= G5_FOLD records of a tile
            float2 a2[NAcc<KIND>::n];
#pragma unroll
            for (int c = 0; c < NAcc<KIND>::n; c++) a2[c] = make_float2(0.f, 0.f);
#pragma unroll 4
            for (int j = lane; j < nt; j += 2)
                g5_interact2<KIND, NT>(sj, j, xi, yi, zi, ei, tab, shift, A.r2cut, a2);
#pragma unroll
            for (int k = 0; k < 2; k++) g5_fold2<KIND>(S[k], a2, k);
        }
        // lane 1's sums into lane 0's, one i per round through the j-tile buffer
        double4* red = reinterpret_cast<double4*>(sj);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            __syncthreads();
            red[threadIdx.x] = make_double4(S[k][0], S[k][1], S[k][2], S[k][3]);
            __syncthreads();
            if (lane == 0) {
                const double4 v = red[slot + H];
                S[k][0] += v.x;
                S[k][1] += v.y;
                S[k][2] += v.z;
                S[k][3] += v.w;
            }
        }
        if (lane != 0) return;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int li = slot + k * H;
            if (li >= T.ni) continue;
            const double4 v = make_double4(S[k][0], S[k][1], S[k][2], S[k][3]);
            if (T.group < 0) A.out[T.i0 + li] = g5_finish<KIND>(v, A.ascale);
            else A.partial[(size_t)T.slot * A.itile + li] = v;
        }
    };

    // Tasks of 33..48 i in the 64-thread CTAs: three i per thread (slot, slot + 16, slot + 32)
    // over four j-lanes, so that such a task occupies 48 i-slots instead of the pair layout's 64
    // (tree-code groups of 33..63 i leave a third of those idle); each lane's records are read
    // once for its three i.  The lanes' sums are added in lane order.
    auto lanes_triple_task = [&](const Task& T) {
        constexpr int H = NT / 4;
        const int slot = (int)threadIdx.x % H, lane = (int)threadIdx.x / H;
        float xi[3], yi[3], zi[3], ei[3];
        double S[3][4];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int li = slot + k * H;
            const float4 p = A.ipos[T.i0 + (li < T.ni ? li : 0)];
            xi[k] = p.x; yi[k] = p.y; zi[k] = p.z; ei[k] = p.w;
            S[k][0] = S[k][1] = S[k][2] = S[k][3] = 0.0;
        }
        for (int jt = 0; jt < T.nj; jt += NT) {
            const int nt = min(NT, T.nj - jt);
            __syncthreads();
            if (threadIdx.x < nt) {
                const int jk = T.j0 + jt + threadIdx.x;
                const int jj = A.jidx ? __ldg(A.jidx + jk) : jk;
                sj[threadIdx.x] = A.jpos[jj];
                if constexpr (W == 2) sj[NT + threadIdx.x] = A.jaux[jj];
                if constexpr (W == 3) g5_stage_quad(sj + NT + 2 * threadIdx.x, A.jaux, jj);
            }
            __syncthreads();
            // one block: a lane sees at most NT/4 <= G5_FOLD records of a tile
            float a[3][NAcc<KIND>::n];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int c = 0; c < NAcc<KIND>::n; c++) a[k][c] = 0.f;
            g5_jloop<KIND, NT, 3, 4>(sj, lane, nt, xi, yi, zi, ei, tab, shift, A.r2cut, a);
#pragma unroll
            for (int k = 0; k < 3; k++) g5_fold<KIND>(S[k], a[k]);
        }
        double4* red = reinterpret_cast<double4*>(sj);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            __syncthreads();
            red[threadIdx.x] = make_double4(S[k][0], S[k][1], S[k][2], S[k][3]);
            __syncthreads();
            if (lane == 0) {
                for (int l = 1; l < 4; l++) {
                    const double4 v = red[slot + l * H];
                    S[k][0] += v.x;
                    S[k][1] += v.y;
                    S[k][2] += v.z;
                    S[k][3] += v.w;
                }
            }
        }
        if (lane != 0) return;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int li = slot + k * H;
            if (li >= T.ni) continue;
            const double4 v = make_double4(S[k][0], S[k][1], S[k][2], S[k][3]);
            if (T.group < 0) A.out[T.i0 + li] = g5_finish<KIND>(v, A.ascale);
            else A.partial[(size_t)T.slot * A.itile + li] = v;
        }
    };

    // The j-paired task (USE_JP).  In the 64-thread CTAs a task of more than NT/2 i runs two i
    // per thread (slot and slot + NT/2) over two j-lanes, a smaller one one i per thread over
    // nl = NT / isl lanes (isl = ni rounded up to 16, as the other form); lane l takes the tile's
    // j-quads l, l + nl, ...  Larger CTAs: one i per thread, one lane.  The tile is staged as
    // field arrays padded to a multiple of 4 with massless copies of its first record (and zero
    // moments for cells), which add exact zeros.  FP32 sums are folded into FP64 every G5_FOLD
    // j of a lane; the lanes' sums are added in lane order.
    auto jp_task = [&](const Task& T) {
        G5TileSoA<NT>* sa = reinterpret_cast<G5TileSoA<NT>*>(sj);
        const bool two = LANES && T.ni > NT / 2;
        int nl = 1, isl = NT;
        if (two) {
            nl = 2;
            isl = NT / 2;
        } else if (LANES) {
            const int need = (T.ni + 15) & ~15;
            nl = NT / (need > 0 ? need : 32);
            isl = NT / nl;
        }
        const int slot = (int)threadIdx.x % isl, lane = (int)threadIdx.x / isl;
        const int nik = two ? 2 : 1;
        float2 nx[KM], ny[KM], nz[KM];
        float ei[KM];
        double S[KM][4];
#pragma unroll
        for (int k = 0; k < KM; k++) {
            const int li = slot + k * isl;
            const float4 p = A.ipos[T.i0 + (li < T.ni ? li : 0)];
            nx[k] = make_float2(-p.x, -p.x);
            ny[k] = make_float2(-p.y, -p.y);
            nz[k] = make_float2(-p.z, -p.z);
            ei[k] = p.w;
            S[k][0] = S[k][1] = S[k][2] = S[k][3] = 0.0;
        }
        for (int jt = 0; jt < T.nj; jt += NT) {
            const int nt = min(NT, T.nj - jt);
            const int nt4 = (nt + 3) & ~3;
            __syncthreads();
            if ((int)threadIdx.x < nt4) {
                const bool real = (int)threadIdx.x < nt;
                const int jk = T.j0 + jt + (real ? (int)threadIdx.x : 0);
                const int jj = A.jidx ? __ldg(A.jidx + jk) : jk;
                const float4 J = A.jpos[jj];
                sa->x[threadIdx.x] = J.x;
                sa->y[threadIdx.x] = J.y;
                sa->z[threadIdx.x] = J.z;
                sa->m[threadIdx.x] = real ? J.w : 0.0f;
                if constexpr (KIND == G5_QUAD) {
                    const float4 Q0 = A.jaux[2 * jj], Q1 = A.jaux[2 * jj + 1];
                    const float f = real ? G5_QSCALE : 0.0f;
                    sa->q[0][threadIdx.x] = f * Q0.x;
                    sa->q[1][threadIdx.x] = f * Q0.y;
                    sa->q[2][threadIdx.x] = f * Q0.z;
                    sa->q[3][threadIdx.x] = f * Q0.w;
                    sa->q[4][threadIdx.x] = f * Q1.x;
                    sa->q[5][threadIdx.x] = f * Q1.y;
                }
            }
            __syncthreads();
            for (int jb = 0; jb < nt4; jb += G5_FOLD * nl) {
            const int je = min(jb + G5_FOLD * nl, nt4);
            float2 a2[KM][NAcc<KIND>::n];
#pragma unroll
            for (int k = 0; k < KM; k++)
#pragma unroll
                for (int c = 0; c < NAcc<KIND>::n; c++) a2[k][c] = make_float2(0.f, 0.f);
            for (int j = jb + 4 * lane; j < je; j += 4 * nl) {
                const float4 X = *reinterpret_cast<const float4*>(&sa->x[j]);
                const float4 Y = *reinterpret_cast<const float4*>(&sa->y[j]);
                const float4 Z = *reinterpret_cast<const float4*>(&sa->z[j]);
                const float4 M = *reinterpret_cast<const float4*>(&sa->m[j]);
                if constexpr (KIND == G5_QUAD) {
                    float4 Qv[6];
#pragma unroll
                    for (int c = 0; c < 6; c++) Qv[c] = *reinterpret_cast<const float4*>(&sa->q[c][j]);
                    float2 Qa[6], Qb[6];
#pragma unroll
                    for (int c = 0; c < 6; c++) {
                        Qa[c] = make_float2(Qv[c].x, Qv[c].y);
                        Qb[c] = make_float2(Qv[c].z, Qv[c].w);
                    }
#pragma unroll
                    for (int k = 0; k < KM; k++) {
                        if (k < nik) {
                            g5_quad_jpair(make_float2(X.x, X.y), make_float2(Y.x, Y.y), make_float2(Z.x, Z.y),
                                          make_float2(M.x, M.y), Qa, nx[k], ny[k], nz[k], ei[k], a2[k]);
                            g5_quad_jpair(make_float2(X.z, X.w), make_float2(Y.z, Y.w), make_float2(Z.z, Z.w),
                                          make_float2(M.z, M.w), Qb, nx[k], ny[k], nz[k], ei[k], a2[k]);
                        }
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < KM; k++) {
                        if (k < nik) {
                            g5_newton_jpair(make_float2(X.x, X.y), make_float2(Y.x, Y.y), make_float2(Z.x, Z.y),
                                            make_float2(M.x, M.y), nx[k], ny[k], nz[k], ei[k], a2[k]);
                            g5_newton_jpair(make_float2(X.z, X.w), make_float2(Y.z, Y.w), make_float2(Z.z, Z.w),
                                            make_float2(M.z, M.w), nx[k], ny[k], nz[k], ei[k], a2[k]);
                        }
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < KM; k++) g5_fold2<KIND>(S[k], a2[k], -1);
            }
        }
        // lane sums in lane order, one i per round through the j-tile buffer
        double4* red = reinterpret_cast<double4*>(sj);
#pragma unroll
        for (int k = 0; k < KM; k++) {
            if (k < nik && nl > 1) {
                __syncthreads();
                red[threadIdx.x] = make_double4(S[k][0], S[k][1], S[k][2], S[k][3]);
                __syncthreads();
                if (lane == 0) {
                    for (int l = 1; l < nl; l++) {
                        const double4 v = red[slot + l * isl];
                        S[k][0] += v.x;
                        S[k][1] += v.y;
                        S[k][2] += v.z;
                        S[k][3] += v.w;
                    }
                }
            }
        }
        if (lane != 0) return;
#pragma unroll
        for (int k = 0; k < KM; k++) {
            const int li = slot + k * isl;
            if (k >= nik || li >= T.ni) continue;
            const double4 v = make_double4(S[k][0], S[k][1], S[k][2], S[k][3]);
            if (T.group < 0) A.out[T.i0 + li] = g5_finish<KIND>(v, A.ascale);
            else A.partial[(size_t)T.slot * A.itile + li] = v;
        }
    };

    // The last CTA to finish a task of a split group reduces the group's partial rows.
    auto group_done = [&](const Task& T) {
        const Group G = A.groups[T.group];
        if (group_arrive(A.group_counters, T.group, G.nchunk, &s_flag)) {
            // Cooperative reduction of the group's partial rows: P threads per i, each summing a
            // fixed strided subset of the rows, then the P sums in thread order (deterministic
            // for a given group shape).  `red` reuses the j-tile buffer.
            double4* red = reinterpret_cast<double4*>(sj);
            static_assert(sizeof(float4) * NT * (W > 2 ? W : 2) >= sizeof(double4) * NT, "reduction buffer");
            int P = 1;
            while (P * 2 * G.ni <= NT) P *= 2;
            const int per = NT / P;
            for (int base = 0; base < G.ni; base += per) {
                const int li = base + threadIdx.x / P, p = threadIdx.x % P;
                double4 s = make_double4(0, 0, 0, 0);
                if (li < G.ni) {
                    // four independent partial sums keep four rows' loads in flight; combined in
                    // a fixed order (deterministic)
                    const double4* col = A.partial + (size_t)G.slot0 * A.itile + li;
                    auto ld = [&](int c) {
                        const double4* r = col + (size_t)c * A.itile;
                        return make_double4(__ldcg(&r->x), __ldcg(&r->y), __ldcg(&r->z), __ldcg(&r->w));
                    };
                    double4 s1 = s, s2 = s, s3 = s;
                    int c = p;
                    for (; c + 3 * P < G.nchunk; c += 4 * P) {
                        double4 v0 = ld(c), v1 = ld(c + P), v2 = ld(c + 2 * P), v3 = ld(c + 3 * P);
                        s = add4(s, v0);
                        s1 = add4(s1, v1);
                        s2 = add4(s2, v2);
                        s3 = add4(s3, v3);
                    }
                    for (; c < G.nchunk; c += P) s = add4(s, ld(c));
                    s = add4(add4(s, s1), add4(s2, s3));
                }
                __syncthreads();
                red[threadIdx.x] = s;
                __syncthreads();
                if (p == 0 && li < G.ni) {
                    for (int q = 1; q < P; q++) s = add4(s, red[threadIdx.x + q]);
                    A.out[G.i0 + li] = g5_finish<KIND>(s, A.ascale);
                }
            }
        }
    };

    for (bool first = true;; first = false) {
        int t = next_task(A.task_counter, &s_task, A.ntasks, first);
        if (t >= A.ntasks) break;
        const Task T = A.tasks[t];
        if constexpr (USE_JP) {
            jp_task(T);
            if (T.group >= 0) group_done(T);
            continue;
        }
        if constexpr (LANES) {
            if (NT == 64 && T.ni > NT / 2 && T.ni <= 3 * NT / 4) {
                lanes_triple_task(T);
                if (T.group >= 0) group_done(T);
                continue;
            }
            if (T.ni > NT / 2) {
                lanes_pair_task(T);
                if (T.group >= 0) group_done(T);
                continue;
            }
        }
        // j-lanes (the 64-thread one-i-per-thread CTAs): a task of few i takes half-warps of
        // i-slots (isl = ni rounded up to 16; the two half-warps of a warp then read two j records,
        // which a 16-byte shared load serves in the same two wavefronts as a broadcast) and
        // splits each j-tile over the nl = NT / isl lanes of slots; the lanes' sums are added in
        // lane order at the end.  Large tasks: nl = 1.
        int nl = 1, isl = NT;
        if constexpr (LANES) {
            const int need = (T.ni + 15) & ~15;
            nl = NT / (need > 0 ? need : 32);
            isl = NT / nl;
        }
        const int slot = LANES ? (int)threadIdx.x % isl : (int)threadIdx.x;
        const int lane = LANES ? (int)threadIdx.x / isl : 0;

        float xi[IPT], yi[IPT], zi[IPT], ei[IPT];
        double S[IPT][4];
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            int li = slot + k * NT;
            int ii = T.i0 + (li < T.ni ? li : 0);
            float4 p = A.ipos[ii];
            xi[k] = p.x; yi[k] = p.y; zi[k] = p.z; ei[k] = p.w;
            S[k][0] = S[k][1] = S[k][2] = S[k][3] = 0.0;
        }

        for (int jt = 0; jt < T.nj; jt += NT) {
            const int nt = min(NT, T.nj - jt);
            __syncthreads();
            if (threadIdx.x < nt) {
                const int jk = T.j0 + jt + threadIdx.x;
                const int jj = A.jidx ? __ldg(A.jidx + jk) : jk;
                sj[threadIdx.x] = A.jpos[jj];
                if constexpr (W == 2) sj[NT + threadIdx.x] = A.jaux[jj];
                if constexpr (W == 3) g5_stage_quad(sj + NT + 2 * threadIdx.x, A.jaux, jj);
            }
            __syncthreads();
            if constexpr (IPT % 2 == 0) {
                for (int j0 = 0; j0 < nt; j0 += G5_FOLD) {
                    const int j1 = min(j0 + G5_FOLD, nt);
                    float2 a2[IPT / 2][NAcc<KIND>::n];
#pragma unroll
                    for (int p = 0; p < IPT / 2; p++)
#pragma unroll
                        for (int c = 0; c < NAcc<KIND>::n; c++) a2[p][c] = make_float2(0.f, 0.f);
#pragma unroll 4
                    for (int j = j0; j < j1; j++) {
#pragma unroll
                        for (int p = 0; p < IPT / 2; p++)
                            g5_interact2<KIND, NT>(sj, j, xi + 2 * p, yi + 2 * p, zi + 2 * p, ei + 2 * p, tab, shift,
                                                   A.r2cut, a2[p]);
                    }
#pragma unroll
                    for (int k = 0; k < IPT; k++) g5_fold2<KIND>(S[k], a2[k / 2], k % 2);
                }
            } else {
            // blocks of G5_FOLD terms per lane (one block when a tile has no more: NT <= G5_FOLD);
            // the lane stride as a template constant, so that the unrolled loop addresses its j
            // records with immediate offsets (64-thread CTAs have 1, 2 or 4 lanes)
            const int nlanes = LANES ? nl : 1;
            auto block = [&](int j0, int j1) {
                float a[IPT][NAcc<KIND>::n];
#pragma unroll
                for (int k = 0; k < IPT; k++)
#pragma unroll
                    for (int c = 0; c < NAcc<KIND>::n; c++) a[k][c] = 0.f;
                if (nlanes == 1) g5_jloop<KIND, NT, IPT, 1>(sj, j0 + lane, j1, xi, yi, zi, ei, tab, shift, A.r2cut, a);
                else if (nlanes == 2) g5_jloop<KIND, NT, IPT, 2>(sj, j0 + lane, j1, xi, yi, zi, ei, tab, shift, A.r2cut, a);
                else if (nlanes == 4) g5_jloop<KIND, NT, IPT, 4>(sj, j0 + lane, j1, xi, yi, zi, ei, tab, shift, A.r2cut, a);
                else g5_jloop<KIND, NT, IPT, 0>(sj, j0 + lane, j1, xi, yi, zi, ei, tab, shift, A.r2cut, a, nlanes);
#pragma unroll
                for (int k = 0; k < IPT; k++) g5_fold<KIND>(S[k], a[k]);
            };
            if constexpr (NT <= G5_FOLD) {
                block(0, nt);
            } else {
                for (int j0 = 0; j0 < nt; j0 += G5_FOLD * nlanes) block(j0, min(j0 + G5_FOLD * nlanes, nt));
            }
            }
        }

        bool lane0 = true;
        if constexpr (LANES) {
            if (nl > 1) {
                // lane sums in lane order through the j-tile buffer (IPT == 1)
                double4* red = reinterpret_cast<double4*>(sj);
                __syncthreads();
                red[threadIdx.x] = make_double4(S[0][0], S[0][1], S[0][2], S[0][3]);
                __syncthreads();
                lane0 = lane == 0;
                if (lane0) {
                    for (int l = 1; l < nl; l++) {
                        const double4 v = red[slot + l * isl];
                        S[0][0] += v.x;
                        S[0][1] += v.y;
                        S[0][2] += v.z;
                        S[0][3] += v.w;
                    }
                }
            }
        }
        if (T.group < 0) {
#pragma unroll
            for (int k = 0; k < IPT; k++) {
                int li = slot + k * NT;
                if (lane0 && li < T.ni)
                    A.out[T.i0 + li] = g5_finish<KIND>(make_double4(S[k][0], S[k][1], S[k][2], S[k][3]), A.ascale);
            }
            continue;
        }
        double4* row = A.partial + (size_t)T.slot * A.itile;
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            int li = slot + k * NT;
            if (lane0 && li < T.ni) row[li] = make_double4(S[k][0], S[k][1], S[k][2], S[k][3]);
        }
        group_done(T);
    }
}

}  // namespace pgb
