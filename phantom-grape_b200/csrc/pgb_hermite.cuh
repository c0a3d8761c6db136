// pgb_hermite.cuh -- the PG6 sample integrator's 4th-order Hermite block-time-step scheme on
// the device: block selection, i- and j-prediction, corrector and new step, start-up step.
//
// Reference: PG6/banana (built with -DNORMAL, its setting): timestep.c:87-98 global_time
// (block time and active set), hermite.c:39-63 predict_exmotion (i predictor), hermite.c:67-108
// correct + 143-205 correct_sgmotion (corrector, new state), timestep.c:53-85 dt_criterion
// (Aarseth criterion, step halved or doubled on the power-of-two grid), hermite.c:110-141
// startup_sgmotion + timestep.c:24-51 dt_startup, timestep.c:127-135 reset_time,
// timestep.c:137-150 calc_modulus.  The j-memory that the reference re-sends with
// g6_set_j_particle after every step (hermite.c:240-265: pos, vel, acc/2, jerk/6, mass, t) is the
// particle state itself here: the j predictor reads the state arrays, so nothing is re-sent.
//
// State in HBM, one array per field of struct Particle (PG6/banana/particle.h): t, dt, pot,
// mass [n] and pos, vel, acc, jrk [n][3], all FP64 (jrk and pot hold float values: the
// reference stores them as float).  One block step is five launches:
//   hm_tmin_kernel   min over i of t_i + dt_i (the block time t_gl), atomicMin on the bits
//                    (t + dt >= 0, so the bit patterns order like the values); with `reset`,
//                    first sets every t_i = 0 (reset_time after a step that ended on a
//                    multiple of dtmax);
//   hm_count_kernel  active particles (t_i + dt_i == t_gl) per segment of SEG particles; the
//                    last segment to arrive scans the counts in order and publishes (ni, t_gl)
//                    to the host through mapped memory, so the host can size the force launch;
//   hm_build_kernel  j-prediction of every particle to t_gl (the library's FP64 predictor,
//                    gravity.c:149-193) and, for the active ones in index order, the active
//                    list and the predicted i-records;
//   the force kernel (pgb_g6_kernels.cuh / pgb_g6_small.cuh) on the ni i-records;
//   hm_correct_kernel (or hm_startup_kernel for the first step) per active particle.
// The i-predictor and the corrector use the reference's formulas and constants in the order
// its C source evaluates them, with every FP64 multiply and add rounded separately (no fused
// multiply-add): given the same forces the new state equals a plain C evaluation bit for bit.
#pragma once

#include "pgb_g6_kernels.cuh"

namespace pgb {

constexpr int HM_NT = 256;            // threads per CTA of the step kernels
constexpr int HM_PER = 8;             // particles per thread
constexpr int HM_SEG = HM_NT * HM_PER;  // particles per segment (one CTA)

struct HmState {
    double *t, *dt, *pos, *vel, *acc, *jrk, *pot, *mass;
    int n;
};

// Published by hm_count_kernel into mapped host memory: the step's block time and active count.
struct HmHostCtl {
    unsigned seq;
    int ni;
    double t_gl;
};

struct HmWork {
    unsigned long long* tmin;  // atomic min of the bits of t + dt; all ones between steps
    int* ticket;               // arrivals on hm_count_kernel (self-resetting)
    int* bcnt;                 // active count per segment
    int* boff;                 // exclusive prefix of bcnt
    int* ni;                   // the step's active count
    double* t_gl;              // the step's block time
    int* bad;                  // start-up steps below dtmin
    int* active;               // [n] active particles in index order
    G6I* irec;                 // [n] their predicted i-records
    G6PredJ* jpred;            // [n] every particle predicted to t_gl
    G6Out* out;                // [n] force, jerk, potential of the active particles
    HmHostCtl* host;           // device address of the mapped control block
};

__device__ __forceinline__ double hm_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double hm_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double hm_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double hm_float(double a) { return (double)__double2float_rn(a); }

// predict_exmotion's constants as its source spells them (hermite.h)
constexpr double HM_SECOND = 5e-1;
constexpr double HM_THIRD = 1.666666666666667e-1;
constexpr double HM_FOURTH = 4.166666666666667e-2;
constexpr double HM_FIFTH = 8.333333333333333e-3;

// i predictor (hermite.c:47-56): x + v d + a d^2 (1/2) + j d^3 (1/6), v + a d + j d^2 (1/2)
__device__ __forceinline__ void hm_predict_i(const HmState& P, int i, double t_gl, double xp[3], double vp[3]) {
    const double d = hm_sub(t_gl, P.t[i]);
    const double d2 = hm_mul(d, d), d3 = hm_mul(d, d2);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const double x = P.pos[3 * i + c], v = P.vel[3 * i + c], a = P.acc[3 * i + c], j = P.jrk[3 * i + c];
        xp[c] = hm_add(hm_add(hm_add(x, hm_mul(v, d)), hm_mul(hm_mul(a, d2), HM_SECOND)),
                       hm_mul(hm_mul(j, d3), HM_THIRD));
        vp[c] = hm_add(hm_add(v, hm_mul(a, d)), hm_mul(hm_mul(j, d2), HM_SECOND));
    }
}

// calc_modulus (timestep.c:137-150): what is left of num after removing the largest
// power-of-two multiples down to mod; zero when num is a multiple of mod on dtmax's grid.
__device__ __forceinline__ double hm_modulus(double num, double mod, double modmax) {
    double tmpmod = modmax;
    for (int it = 0; num > 0.0 && it < 4096; it++) {
        for (int k = 0; tmpmod > num && k < 2048; k++) tmpmod *= 0.5;
        if (tmpmod < mod) break;
        num = hm_sub(num, tmpmod);
    }
    return num;
}

template <int NT>
__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v, unsigned long long* sm) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    v = sm[0];
#pragma unroll
    for (int w = 1; w < NT / 32; w++) v = sm[w] < v ? sm[w] : v;
    return v;
}

__global__ void __launch_bounds__(HM_NT) hm_tmin_kernel(HmState P, HmWork W, int reset) {
    __shared__ unsigned long long sm[HM_NT / 32];
    const int seg0 = blockIdx.x * HM_SEG;
    unsigned long long m = ~0ull;
#pragma unroll 4
    for (int r = 0; r < HM_PER; r++) {
        const int i = seg0 + r * HM_NT + (int)threadIdx.x;
        if (i >= P.n) break;
        double t = P.t[i];
        if (reset) {
            t = 0.0;
            P.t[i] = 0.0;
        }
        const unsigned long long b = (unsigned long long)__double_as_longlong(hm_add(t, P.dt[i]));
        m = b < m ? b : m;
    }
    m = block_min_u64<HM_NT>(m, sm);
    if (threadIdx.x == 0) atomicMin(W.tmin, m);
}

// Inclusive scan of v over the CTA (warp shuffles, then the warp totals); *total = the sum.
template <int NT>
__device__ __forceinline__ int block_scan(int v, int* sw, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    __syncthreads();
    if (lane == 31) sw[w] = v;
    __syncthreads();
    int base = 0, all = 0;
#pragma unroll
    for (int k = 0; k < NT / 32; k++) {
        base += k < w ? sw[k] : 0;
        all += sw[k];
    }
    *total = all;
    return v + base;
}

__global__ void __launch_bounds__(HM_NT) hm_count_kernel(HmState P, HmWork W, unsigned seq) {
    __shared__ int sw[HM_NT / 32];
    __shared__ int s_last;
    const double tg = __longlong_as_double((long long)*W.tmin);
    const int seg0 = blockIdx.x * HM_SEG;
    int c = 0;
#pragma unroll 4
    for (int r = 0; r < HM_PER; r++) {
        const int i = seg0 + r * HM_NT + (int)threadIdx.x;
        if (i >= P.n) break;
        c += hm_add(P.t[i], P.dt[i]) == tg;
    }
    int tot;
    block_scan<HM_NT>(c, sw, &tot);
    if (threadIdx.x == 0) W.bcnt[blockIdx.x] = tot;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(W.ticket, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    // the last segment: every count is written; scan them in segment order
    __threadfence();
    int run = 0;
    for (int b0 = 0; b0 < (int)gridDim.x; b0 += HM_NT) {
        const int b = b0 + (int)threadIdx.x;
        const int v = b < (int)gridDim.x ? __ldcg(W.bcnt + b) : 0;
        int sum;
        const int inc = block_scan<HM_NT>(v, sw, &sum);
        if (b < (int)gridDim.x) W.boff[b] = run + inc - v;
        run += sum;
    }
    if (threadIdx.x == 0) {
        *W.ni = run;
        *W.t_gl = tg;
        *W.tmin = ~0ull;   // every segment has read it
        *W.ticket = 0;
        W.host->ni = run;
        W.host->t_gl = tg;
        __threadfence_system();
        *(volatile unsigned*)&W.host->seq = seq;
    }
}

__global__ void __launch_bounds__(HM_NT) hm_build_kernel(HmState P, HmWork W, bool ff) {
    __shared__ int sw[HM_NT / 32];
    const double tg = *W.t_gl;
    const int seg0 = blockIdx.x * HM_SEG;
    int base = W.boff[blockIdx.x];
    for (int r = 0; r < HM_PER; r++) {
        const int i = seg0 + r * HM_NT + (int)threadIdx.x;
        const bool in = i < P.n;
        bool act = false;
        if (in) {
            // j predictor of the library (gravity.c:149-193) on (pos, vel, acc/2, jerk/6, t)
            const double d = tg - P.t[i], d2 = d * d, d3 = d2 * d;
            double x[3];
            float v[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const double a2 = P.acc[3 * i + c] * 0.5, j6 = P.jrk[3 * i + c] * (1.0 / 6.0);
                x[c] = P.pos[3 * i + c] + P.vel[3 * i + c] * d + a2 * d2 + j6 * d3;
                v[c] = (float)(P.vel[3 * i + c] + 2.0 * a2 * d + 3.0 * j6 * d2);
            }
            G6PredJ o;
            store_pos(o.p, x[0], x[1], x[2], ff);
            o.m = (float)P.mass[i];
            o.id = i;
            o.vx = v[0];
            o.vy = v[1];
            o.vz = v[2];
            o.pad = 0.f;
            W.jpred[i] = o;
            act = hm_add(P.t[i], P.dt[i]) == tg;
        }
        int tot;
        const int inc = block_scan<HM_NT>(act ? 1 : 0, sw, &tot);
        if (act) {
            const int k = base + inc - 1;
            W.active[k] = i;
            double xp[3], vp[3];
            hm_predict_i(P, i, tg, xp, vp);
            G6I rec;
            store_pos(rec.p, xp[0], xp[1], xp[2], ff);
            rec.vx = (float)vp[0];
            rec.vy = (float)vp[1];
            rec.vz = (float)vp[2];
            rec.id = i;
            rec.h2 = 0.f;
            rec.pad = 0.f;
            W.irec[k] = rec;
        }
        base += tot;
    }
}

// Corrector and new step of active particle k (hermite.c:67-108, 143-205; timestep.c:53-85),
// given its new acceleration (FP64), jerk and potential (rounded to float as the reference's
// struct NewAccJerk stores them).
__global__ void hm_correct_kernel(HmState P, HmWork W, int ni, double eta, double dtmax) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ni) return;
    const int i = W.active[k];
    const double tg = *W.t_gl;
    const double dtmin = dtmax / 2251799813685248.0;  // dtmax / 2^51
    double x1[3], v1[3];
    hm_predict_i(P, i, tg, x1, v1);
    const G6Out F = W.out[k];
    const double a1[3] = {F.ax, F.ay, F.az};
    const double j1[3] = {hm_float(F.jx), hm_float(F.jy), hm_float(F.jz)};
    const double dts = P.dt[i], dtsinv = 1.0 / dts;
    double s0[3], c0[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const double a0 = P.acc[3 * i + c], j0 = P.jrk[3 * i + c];
        const double da = hm_sub(a0, a1[c]);
        s0[c] = hm_mul(hm_mul(hm_mul(2.0, hm_sub(hm_mul(-3.0, da), hm_mul(hm_add(hm_mul(2.0, j0), j1[c]), dts))),
                              dtsinv),
                       dtsinv);
        c0[c] = hm_mul(hm_mul(hm_mul(hm_mul(6.0, hm_add(hm_mul(2.0, da), hm_mul(hm_add(j0, j1[c]), dts))), dtsinv),
                              dtsinv),
                       dtsinv);
        const double s4 = hm_mul(hm_mul(hm_mul(hm_mul(hm_mul(s0[c], dts), dts), dts), dts), HM_FOURTH);
        const double c5 = hm_mul(hm_mul(hm_mul(hm_mul(hm_mul(hm_mul(c0[c], dts), dts), dts), dts), dts), HM_FIFTH);
        x1[c] = hm_add(x1[c], hm_add(s4, c5));
        const double s3 = hm_mul(hm_mul(hm_mul(hm_mul(s0[c], dts), dts), dts), HM_THIRD);
        const double c4 = hm_mul(hm_mul(hm_mul(hm_mul(hm_mul(c0[c], dts), dts), dts), dts), HM_FOURTH);
        v1[c] = hm_add(v1[c], hm_add(s3, c4));
    }
    // dt_criterion at t_gl with the old step
    double a = 0.0, jj = 0.0, sn = 0.0, cr = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const double s1 = hm_add(s0[c], hm_mul(c0[c], dts));
        a = hm_add(a, hm_mul(a1[c], a1[c]));
        jj = hm_add(jj, hm_mul(j1[c], j1[c]));
        sn = hm_add(sn, hm_mul(s1, s1));
        cr = hm_add(cr, hm_mul(c0[c], c0[c]));
    }
    a = sqrt(a);
    jj = sqrt(jj);
    sn = sqrt(sn);
    cr = sqrt(cr);
    const double dti = hm_mul(eta, sqrt(hm_add(hm_mul(a, sn), hm_mul(jj, jj)) / hm_add(hm_mul(jj, cr), hm_mul(sn, sn))));
    double dnew = dts;
    if (dti < dnew) {
        for (int it = 0; dnew > dti && dnew > dtmin && it < 64; it++) dnew *= 0.5;
    } else if (dti > 2.0 * dnew) {
        if (hm_modulus(tg, 2.0 * dnew, dtmax) == 0.0) dnew = 2.0 * dnew;
    }
    P.t[i] = tg;
    P.dt[i] = dnew;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        P.pos[3 * i + c] = x1[c];
        P.vel[3 * i + c] = v1[c];
        P.acc[3 * i + c] = a1[c];
        P.jrk[3 * i + c] = j1[c];
    }
    P.pot[i] = hm_float(F.pot);
}

// Start-up step (hermite.c:110-141, timestep.c:24-51): every particle active at t = 0; the new
// force becomes the state and the first step is the largest power-of-two fraction of dtmax
// below eta_s |a|/|j| that divides t.  Counts the steps that fell below dtmin into *W.bad.
__global__ void hm_startup_kernel(HmState P, HmWork W, int ni, double eta_s, double dtmax) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ni) return;
    const int i = W.active[k];
    const double dtmin = dtmax / 2251799813685248.0;
    const G6Out F = W.out[k];
    const double a1[3] = {F.ax, F.ay, F.az};
    const double j1[3] = {hm_float(F.jx), hm_float(F.jy), hm_float(F.jz)};
    double a = 0.0, jj = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        P.acc[3 * i + c] = a1[c];
        P.jrk[3 * i + c] = j1[c];
        a = hm_add(a, hm_mul(a1[c], a1[c]));
        jj = hm_add(jj, hm_mul(j1[c], j1[c]));
    }
    P.pot[i] = hm_float(F.pot);
    const double dtcrit = hm_mul(eta_s, sqrt(a / jj));
    double d = dtmax;
    for (int it = 0; d > dtcrit && d > dtmin && it < 64; it++) d *= 0.5;
    for (int it = 0; hm_modulus(P.t[i], d, dtmax) != 0.0 && it < 64; it++) {
        d *= 0.5;
        if (d < dtmin) {
            atomicAdd(W.bad, 1);
            break;
        }
    }
    P.dt[i] = d;
}

// reset_time (timestep.c:127-135) on its own, for reads of the state between steps.
__global__ void hm_reset_kernel(HmState P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P.n) P.t[i] = 0.0;
}

// Kinetic and potential energy (calc_energy.c:9-33): ek = sum m v^2 / 2, ew = sum m pot / 2.
// One CTA, fixed summation order: the result does not depend on the launch.
__global__ void __launch_bounds__(1024) hm_energy_kernel(HmState P, double* out) {
    __shared__ double sk[1024], sp[1024];
    double k = 0.0, w = 0.0;
    for (int i = threadIdx.x; i < P.n; i += 1024) {
        const double vx = P.vel[3 * i], vy = P.vel[3 * i + 1], vz = P.vel[3 * i + 2];
        k += P.mass[i] * (vx * vx + vy * vy + vz * vz);
        w += P.mass[i] * P.pot[i];
    }
    sk[threadIdx.x] = k;
    sp[threadIdx.x] = w;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sk[threadIdx.x] += sk[threadIdx.x + o];
            sp[threadIdx.x] += sp[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = 0.5 * sk[0];
        out[1] = 0.5 * sp[0];
    }
}

}  // namespace pgb
