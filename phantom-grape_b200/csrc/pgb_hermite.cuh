// pgb_hermite.cuh -- the PG6 sample integrator's 4th-order Hermite block-time-step scheme on
// the device: block selection, i- and j-prediction, force, corrector and new step, start-up
// step, time reset -- one persistent kernel runs whole block steps back to back.
//
// Reference: PG6/banana (built with -DNORMAL, its setting): timestep.c:87-98 global_time
// (block time and active set), hermite.c:39-63 predict_exmotion (i predictor), hermite.c:67-108
// correct + 143-205 correct_sgmotion (corrector, new state), timestep.c:53-85 dt_criterion
// (Aarseth criterion, step halved or doubled on the power-of-two grid), hermite.c:110-141
// startup_sgmotion + timestep.c:24-51 dt_startup, timestep.c:127-135 reset_time,
// timestep.c:137-150 calc_modulus, banana01.c:119-179 the main loop.  The j-memory that the
// reference re-sends with g6_set_j_particle after every step (hermite.c:240-265: pos, vel,
// acc/2, jerk/6, mass, t) is the particle state itself here: the j predictor reads the state
// arrays, so nothing is re-sent.
//
// State in HBM, one array per field of struct Particle (PG6/banana/particle.h): t, dt, pot,
// mass [n] and pos, vel, acc, jrk [n][3], all FP64 (jrk and pot hold float values: the
// reference stores them as float).
//
// hm_run_kernel is a cooperative launch (every CTA resident) that loops over block steps until
// the global time reaches tend.  Segments of HM_SEG particles belong to CTAs (segment s to CTA
// s mod grid) in every phase.  Once per launch, then after every step:
//   A  per segment: the minimum of t_i + dt_i and how many particles sit at it; the global
//      minimum by atomicMin.
// Each step is then three phases; one grid barrier closes the step, and within it CTAs wait
// only for the data they read (per-segment and per-task flags tagged with the step number):
//   B  every CTA reads the block time t_gl (the global minimum) and computes every segment's
//      offset of active particles; it predicts its own segments' particles to t_gl (the
//      library's FP64 j predictor, gravity.c:149-193) and writes their active ones, in index
//      order, to the active list with predicted i-records; CTA 0 advances the clock;
//   C  the force: the GRAPE-6 pair kernel's tasks (pgb_g6_kernels.cuh g6_task) over an
//      i-tile x j-chunk decomposition of the ni x n pairs, each task once the segments of its
//      i- and j-ranges are built; split j-ranges left as partial rows;
//   D  per own segment, once the tasks of its active particles' i-tiles are done, one warp per
//      active particle: its partial rows summed in chunk order, the corrector (or the start-up
//      step); then reset_time if the step ended on a multiple of dtmax, and A for the segment.
// Data read across CTAs within a step is double-buffered by step parity where the next step
// could overwrite it before a slow CTA has read it (segment minima); everything else is
// rewritten only after the closing barrier.
// Every CTA derives the step's decisions (block time, ni, decomposition, end of the run) from
// the same data, so they agree without further communication.  The barriers are bounded: a
// barrier that waits longer than about a second (a limit the host may lower) sets an error word
// and the kernel returns.
// The i-predictor and the corrector use the reference's formulas and constants in the order
// its C source evaluates them, with every FP64 multiply and add rounded separately (no fused
// multiply-add): given the same forces the new state equals a plain C evaluation bit for bit.
#pragma once

#include "pgb_g6_kernels.cuh"

namespace pgb {

constexpr int HM_NT = 256;       // threads per CTA
constexpr int HM_SEG = 256;      // particles per segment of the selection (one per thread)
constexpr int HM_MAXSEG = 4096;  // segments at most: n <= 2^20

struct HmState {
    double *t, *dt, *pos, *vel, *acc, *jrk, *pot, *mass;
    int n;
};

// The integrator's clock and counters in device memory (banana01.c:119-179 bookkeeping): the
// last step's block time and active count, the global time after it (t_mod * dtmax + t_gl, or
// t_mod * dtmax after a reset), the completed dtmax intervals, the particle / block steps, the
// pair interactions and the steps by force decomposition.
struct HmClock {
    double t_gl;
    double time;
    long long psteps, bsteps;
    long long force_pairs;
    long long variant_steps[5];   // steps by force decomposition (i-tile 16, 32, 64, 128, 512)
    long long spin_limit;         // SM cycles a wait may last (0: HM_SPIN_LIMIT)
    int t_mod;
    int ni;       // the last step's active count
    int nch;      // its force decomposition: j-chunks and i-tile
    int itile;
    int bad;      // start-up steps below dtmin
    int err;      // a wait gave up
    int exits;    // CTAs that have returned from the step kernel (all launches)
    int pad;
};

// Default limit of every wait of the step kernel: about a second of SM clock.
constexpr long long HM_SPIN_LIMIT = 2000000000LL;

// Grid barrier state: the generation CTA 0 last released, the step number (the tag of the
// flags below) at the end of the last launch, and per CTA the generation it last arrived at
// (32-bit words 128 bytes apart so that arrivals do not share a line).
constexpr int HM_ARRIVE_STRIDE = 32;
struct HmSync {
    unsigned gen;
    unsigned step;
    unsigned pad[HM_ARRIVE_STRIDE - 2];
    unsigned arrive[1];   // [grid * HM_ARRIVE_STRIDE]
};

struct HmWork {
    unsigned long long* bmin;  // [2][nseg] per segment: the minimum of t + dt (bits), by step parity
    int* bcnt;                 // [2][nseg] per segment: particles at that minimum
    unsigned long long* gmin;  // [3] the global minimum, by step number mod 3 (atomicMin)
    unsigned* seg_flag;        // [nseg] step number of the segment's last build (phase B)
    unsigned* task_flag;       // [task_cap] step number of the force task's last completion
    int task_cap;
    HmClock* clk;
    HmSync* sync;
    int* active;               // [n] active particles in index order
    G6I* irec;                 // [n] their predicted i-records
    G6PredJ* jpred;            // [n] every particle predicted to t_gl
    G6Out* out;                // [n] force, jerk, potential of the active particles (final)
    G6Out* partial;            // partial rows of split j-ranges, part_cap entries
    long long part_cap;
};

struct HmRun {
    HmState P;
    HmWork W;
    float eps2;
    double eta, eta_s, dtmax, tend;
    int startup;     // take the start-up step only
    int max_steps;   // block steps of this launch at most
    int nseg;
    int minj;        // j per chunk at least
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

// The force of active particle k, by the whole warp: with nch > 1 the sum of its nch j-chunk
// partial rows in a fixed order (lane l takes chunks l, l+32, ..., then a butterfly; lane 0's
// sum is the result) scaled as the force kernel's final stage does, written to out[k]; with
// nch == 1 the force kernel's final result out[k].
__device__ __forceinline__ G6Out hm_force_of(const HmWork& W, int k, int nch, int itile) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    if (nch == 1) return W.out[k];
    const int it = k / itile, li = k - it * itile;
    const double2* row = reinterpret_cast<const double2*>(W.partial + (size_t)it * nch * itile + li);
    const size_t stride = (size_t)itile * 4;   // double2 words per partial row
    double s[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int c = lane; c < nch; c += 32) {
        const double2* r = row + (size_t)c * stride;
        const double2 w0 = __ldcg(r), w1 = __ldcg(r + 1), w2 = __ldcg(r + 2), w3 = __ldcg(r + 3);
        s[0] += w0.x; s[1] += w0.y; s[2] += w1.x; s[3] += w1.y; s[4] += w2.x; s[5] += w2.y; s[6] += w3.x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < 7; q++) s[q] += __shfl_xor_sync(full, s[q], o);
#pragma unroll
    for (int q = 0; q < 7; q++) s[q] = __shfl_sync(full, s[q], 0);
    G6Out F;
    F.ax = S_ACC * s[0]; F.ay = S_ACC * s[1]; F.az = S_ACC * s[2];
    F.jx = S_ACC * s[3]; F.jy = S_ACC * s[4]; F.jz = S_ACC * s[5];
    F.pot = S_POT * s[6];
    F.key = 0.f;
    F.jadr = -1;
    if (lane == 0) W.out[k] = F;
    return F;
}

// Corrector and new step of active particle k (hermite.c:67-108, 143-205; timestep.c:53-85),
// given its new acceleration (FP64), jerk and potential (rounded to float as the reference's
// struct NewAccJerk stores them).
__device__ __forceinline__ void hm_correct(const HmState& P, int i, double tg, const G6Out& F, double eta, double dtmax) {
    const double dtmin = dtmax / 2251799813685248.0;  // dtmax / 2^51
    double x1[3], v1[3];
    hm_predict_i(P, i, tg, x1, v1);
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
// below eta_s |a|/|j| that divides t.  Counts the steps that fell below dtmin into W.clk->bad.
__device__ __forceinline__ void hm_startup(const HmState& P, const HmWork& W, int i, const G6Out& F, double eta_s,
                                           double dtmax) {
    const double dtmin = dtmax / 2251799813685248.0;
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
            atomicAdd(&W.clk->bad, 1);
            break;
        }
    }
    P.dt[i] = d;
}

// Grid barrier for a cooperative launch.  Each CTA publishes the barrier's generation number
// in its own arrival word; CTA 0's threads watch the arrival words, and once every CTA is in
// they release the generation, for which the other CTAs wait.  No atomics, no shared counter.
// Release/acquire through the fences around the flag stores and loads.  A wait gives up after
// about a second of SM clock (C->spin_limit cycles when set; error word set); returns false on
// error (the caller returns).
__device__ __forceinline__ bool hm_spin_until(volatile unsigned* w, unsigned target, HmClock* C) {
    const long long t0 = clock64();
    const long long lim = C->spin_limit > 0 ? C->spin_limit : HM_SPIN_LIMIT;
    while (*w != target) {
        if (clock64() - t0 > lim) {
            atomicExch(&C->err, 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ bool hm_grid_sync(HmSync* S, HmClock* C, unsigned target) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        __threadfence();
        *(volatile unsigned*)&S->arrive[blockIdx.x * HM_ARRIVE_STRIDE] = target;
    }
    if (blockIdx.x == 0) {
        int ok = 1;
        for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x)
            ok &= hm_spin_until(&S->arrive[k * HM_ARRIVE_STRIDE], target, C);
        ok = __syncthreads_and(ok);
        if (threadIdx.x == 0) {
            __threadfence();
            *(volatile unsigned*)&S->gen = target;
            if (!ok) s_ok = 0;
        }
    } else if (threadIdx.x == 0) {
        if (!hm_spin_until(&S->gen, target, C)) s_ok = 0;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (*(volatile int*)&C->err) s_ok = 0;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ unsigned long long hm_globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Phase A for one segment: its minimum of t + dt (bits) and count at the minimum, into the
// parity-p slots; the minimum also into the global minimum *gmin.
__device__ __forceinline__ void hm_segment_min(const HmRun& R, int seg, int reset, int p, unsigned long long* gmin,
                                               unsigned long long* sm) {
    const HmState& P = R.P;
    const int i = seg * HM_SEG + (int)threadIdx.x;
    unsigned long long b = ~0ull;
    if (i < P.n) {
        double t = P.t[i];
        if (reset) {
            t = 0.0;
            P.t[i] = 0.0;
        }
        b = (unsigned long long)__double_as_longlong(hm_add(t, P.dt[i]));
    }
    const unsigned long long m = block_min_u64<HM_NT>(b, sm);
    const int c = __syncthreads_count(i < P.n && b == m);
    if (threadIdx.x == 0) {
        R.W.bmin[p * R.nseg + seg] = m;
        R.W.bcnt[p * R.nseg + seg] = c;
        atomicMin(gmin, m);
    }
}

// Phase B for one segment: j-prediction of its particles; its active ones (in index order from
// offset base) into the active list with their predicted i-records.
__device__ __forceinline__ void hm_segment_build(const HmRun& R, int seg, double tg, int base, bool ff, int* sw) {
    const HmState& P = R.P;
    const HmWork& W = R.W;
    const int i = seg * HM_SEG + (int)threadIdx.x;
    bool act = false;
    if (i < P.n) {
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
}

// The force decomposition of a step with ni active particles (identical in every CTA): the pair
// kernel's shape by ni (i-tile of 16, 32, 64, 128 or 512: j-lanes 16, 8, 4, 2 or two i per
// thread), j-chunks for about one task per CTA, at least minj j per chunk, partial rows and
// task flags within their buffers.
struct HmShape {
    int variant, itile, itiles, nch, ntasks;
};
__device__ __forceinline__ HmShape hm_shape(const HmRun& R, int ni) {
    HmShape h;
    h.variant = ni <= 16 ? 0 : ni <= 32 ? 1 : ni <= 64 ? 2 : ni <= 2048 ? 3 : 4;
    h.itile = h.variant == 4 ? 512 : (16 << h.variant);
    h.itiles = (ni + h.itile - 1) / h.itile;
    const int nj = R.P.n;
    int nch = ((int)gridDim.x + h.itiles - 1) / h.itiles;
    const int by_j = nj / R.minj > 1 ? nj / R.minj : 1;
    nch = nch < by_j ? nch : by_j;
    const long long cap = R.W.part_cap / ((long long)h.itiles * h.itile);
    if (nch > cap) nch = cap > 1 ? (int)cap : 1;
    const int tcap = R.W.task_cap / h.itiles;
    if (nch > tcap) nch = tcap > 1 ? tcap : 1;
    h.nch = nch < 1 ? 1 : nch;
    h.ntasks = h.itiles * h.nch;
    return h;
}

// Wait (all threads of the CTA) until every flag[k] for which need(k) holds equals tag; then the
// data published before those flags is visible to the CTA.  False if a wait gave up.
template <class Need>
__device__ __forceinline__ bool hm_wait_flags(unsigned* flag, int nflag, unsigned tag, HmClock* C, Need need) {
    int ok = 1;
    for (int k = threadIdx.x; k < nflag; k += HM_NT)
        if (need(k)) ok &= hm_spin_until(flag + k, tag, C);
    __threadfence();
    return __syncthreads_and(ok) != 0;
}

// Publish (thread 0, after the CTA's writes): flag = tag.
__device__ __forceinline__ void hm_publish(unsigned* flag, unsigned tag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        *(volatile unsigned*)flag = tag;
    }
}

template <bool FF>
__device__ __forceinline__ void hm_run_body(const HmRun& R) {
    __shared__ __align__(16) unsigned char smem[HM_NT * sizeof(G6Out)];
    __shared__ int s_boff[HM_MAXSEG + 1];   // offsets of every segment's active particles (+ ni)
    __shared__ unsigned long long sm[HM_NT / 32];
    __shared__ int sw[HM_NT / 32];
    const HmWork& W = R.W;
    HmClock* C = W.clk;
    const int G = (int)gridDim.x, nseg = R.nseg;
    unsigned epoch = *(volatile unsigned*)&W.sync->gen;   // both stable between launches
    unsigned E = *(volatile unsigned*)&W.sync->step;
    // A (once per launch): segment minima of the current state and their global minimum
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        W.gmin[E % 3] = ~0ull;
        W.gmin[(E + 1) % 3] = ~0ull;
    }
    if (!hm_grid_sync(W.sync, C, ++epoch)) return;
    for (int seg = blockIdx.x; seg < nseg; seg += G) {
        hm_segment_min(R, seg, 0, E & 1, W.gmin + E % 3, sm);
        __syncthreads();
    }
    if (!hm_grid_sync(W.sync, C, ++epoch)) return;
    for (int step = 0;; step++) {
        // the loop condition of banana01.c:146 on the clock written before the last barrier
        if (R.startup ? step >= 1 : (!(*(volatile double*)&C->time < R.tend) || step >= R.max_steps)) break;
        const int p = E & 1;
        // B: the block time, every segment's active offset, own segments' predictions and
        // i-records (published per segment)
        const unsigned long long g = *(volatile unsigned long long*)(W.gmin + E % 3);
        int run = 0;
        for (int b0 = 0; b0 < nseg; b0 += HM_NT) {
            const int k = b0 + (int)threadIdx.x;
            const int v = (k < nseg && W.bmin[p * nseg + k] == g) ? W.bcnt[p * nseg + k] : 0;
            int sum;
            const int inc = block_scan<HM_NT>(v, sw, &sum);
            if (k < nseg) s_boff[k] = run + inc - v;
            run += sum;
        }
        const int ni = run;
        if (threadIdx.x == 0) s_boff[nseg] = ni;
        const double tg = __longlong_as_double((long long)g);
        for (int seg = blockIdx.x; seg < nseg; seg += G) {
            __syncthreads();
            hm_segment_build(R, seg, tg, s_boff[seg], FF, sw);
            hm_publish(W.seg_flag + seg, E);
        }
        __syncthreads();
        const HmShape sh = hm_shape(R, ni);
        // banana01.c:161-179: after a step that ends on a multiple of dtmax the times restart
        // (reset_time, applied with the corrector below) and t_mod counts the interval
        int rs = 0;
        if (!R.startup) {
            const double q = (double)__double2int_rz(hm_mul(tg, 1.0 / R.dtmax));
            rs = hm_sub(tg, hm_mul(q, R.dtmax)) == 0.0;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            W.gmin[(E + 2) % 3] = ~0ull;   // read last in step E-1, next atomicMin in step E+1
            C->t_gl = tg;
            C->ni = ni;
            C->nch = sh.nch;
            C->itile = sh.itile;
            C->psteps += ni;
            C->bsteps += 1;
            C->force_pairs += (long long)ni * R.P.n;
            C->variant_steps[sh.variant] += 1;
            if (!R.startup) {
                const int tm = C->t_mod + rs;
                C->t_mod = tm;
                C->time = rs ? hm_add(hm_mul((double)tm, R.dtmax), 0.0) : hm_add(hm_mul((double)tm, R.dtmax), tg);
            }
        }
        // C: force tasks, each after the segments it reads are built
        {
            G6Args a;
            a.ipart = W.irec;
            a.jpred = W.jpred;
            a.eps2 = R.eps2;
            a.tasks = nullptr;
            a.ntasks = sh.ntasks;
            a.task_counter = nullptr;
            a.groups = nullptr;
            a.group_counters = nullptr;
            a.partial = W.partial;
            a.out = W.out;
            a.itile = sh.itile;
            a.nb_count = nullptr;
            a.nb_list = nullptr;
            a.nb_maxlen = 0;
            a.reg_ni = ni;
            a.reg_nj = R.P.n;
            a.reg_nch = sh.nch;
            a.partial_only = true;
            for (int t = blockIdx.x; t < sh.ntasks; t += G) {
                const Task T = regular_task(a, t);
                const int js0 = T.j0 / HM_SEG, js1 = (T.j0 + T.nj - 1) / HM_SEG;
                const int k0 = T.i0, k1 = T.i0 + T.ni;
                const bool ok = hm_wait_flags(W.seg_flag, nseg, E, C, [&](int s) {
                    return (s >= js0 && s <= js1) || (s_boff[s] < k1 && s_boff[s + 1] > k0);
                });
                if (!ok) return;
                switch (sh.variant) {
                    case 0: g6_task<HM_NT, 1, 16, FF, false, false>(a, T, smem); break;
                    case 1: g6_task<HM_NT, 1, 8, FF, false, false>(a, T, smem); break;
                    case 2: g6_task<HM_NT, 1, 4, FF, false, false>(a, T, smem); break;
                    case 3: g6_task<HM_NT, 1, 2, FF, false, false>(a, T, smem); break;
                    default: g6_task<HM_NT, 2, 1, FF, false, false>(a, T, smem); break;
                }
                hm_publish(W.task_flag + t, E);
            }
        }
        // D + next A, segment by segment (the CTA that built it): after the force tasks of its
        // active particles' i-tiles, the corrector (or start-up step) of each, one warp each;
        // the time reset; the segment's new minimum
        const int wpc = HM_NT / 32;
        for (int seg = blockIdx.x; seg < nseg; seg += G) {
            const int k0 = s_boff[seg], k1 = s_boff[seg + 1];
            if (k1 > k0) {
                const int it0 = k0 / sh.itile, it1 = (k1 - 1) / sh.itile;
                const bool ok = hm_wait_flags(W.task_flag, sh.ntasks, E, C,
                                              [&](int t) { return t / sh.nch >= it0 && t / sh.nch <= it1; });
                if (!ok) return;
            }
            for (int k = k0 + (int)(threadIdx.x >> 5); k < k1; k += wpc) {
                const G6Out F = hm_force_of(W, k, sh.nch, sh.itile);
                if ((threadIdx.x & 31) == 0) {
                    const int i = W.active[k];
                    if (R.startup) hm_startup(R.P, W, i, F, R.eta_s, R.dtmax);
                    else hm_correct(R.P, i, tg, F, R.eta, R.dtmax);
                }
            }
            __syncthreads();   // the segment's updated t, dt
            hm_segment_min(R, seg, rs, p ^ 1, W.gmin + (E + 1) % 3, sm);
            __syncthreads();
        }
        if (!hm_grid_sync(W.sync, C, ++epoch)) return;
        E++;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) W.sync->step = E;
}

// The step kernel: the body above, then every CTA counts its return (on every path, the early
// returns of a wait that gave up included), so the host can tell that the whole grid has left.
template <bool FF>
__global__ void __launch_bounds__(HM_NT, 2) hm_run_kernel(const HmRun R) {
    hm_run_body<FF>(R);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&R.W.clk->exits, 1);
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
