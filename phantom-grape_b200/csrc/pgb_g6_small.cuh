// pgb_g6_small.cuh -- the Hermite force kernel of the drop-in API's small calls: at most 64
// i-particles (the reference's g6calc_lasthalf* take at most NPIPES = 48 per call,
// PG6/libpg6/avx_type.h:1) against the whole j-memory.
//
// Such a call has far too few i-particles to fill the GPU by i, so the j-range is cut into one
// chunk per CTA (gridDim.x chunks, every CTA resident) and the partial sums are reduced in
// three fixed-order stages, none of which round-trips through a task scheduler:
//   1. the JL j-lanes of the CTA, word by word through shared memory (lane order);
//   2. the CTAs of a thread-block cluster (CL consecutive chunks), through distributed shared
//      memory: CTA `rank` sums its slice of the words over the cluster's CTAs (rank order) and
//      writes the cluster's row of partial sums;
//   3. the cluster rows: slice r of the words of every row is written by rank r of each
//      cluster, and the rank-r CTA that arrives last on a per-slice counter sums the slice over
//      the rows (reduce_rows: fixed row order) and writes the final scaled result -- CL CTAs
//      share the final stage and no cluster waits for another.
// The i-records come in the parameter block (no upload; staged to shared memory with
// broadcast reads) and the j-chunks are a pure function of (blockIdx, nj, gridDim), so a call
// is one launch.  The result is deterministic for a given
// grid and cluster size.  Per pair the arithmetic is g6_pair(), identical to g6_kernel.
#pragma once

#include <cooperative_groups.h>

#include "pgb_g6_kernels.cuh"

namespace pgb {

struct G6SmallArgs {
    const G6PredJ* jpred;
    float eps2;
    int ni, nj;        // i-particles (<= ISL) and j-records [0, nj)
    G6Out* partial;    // [gridDim.x / CL][ISL] cluster sums
    int* counter;      // [cluster size] arrivals per word slice; zero at launch, reset by the last
    G6Out* out;        // [ni] final results
    int* nb_count;     // neighbour lists (NBL), indexed by i
    int* nb_list;
    int nb_maxlen;
    // completion flags in mapped host memory (nullptr: none): the CTA that writes word slice r
    // of the results sets done[r] = seq after them, so the host can wait for the results by
    // polling instead of synchronising the stream
    volatile unsigned* done;
    unsigned seq;
};

// Publish a final slice: every thread's result writes are made visible to the host before
// thread 0 sets the slice's completion flag.
__device__ __forceinline__ void publish_done(const G6SmallArgs& A, int slice) {
    if (!A.done) return;
    __threadfence_system();
    __syncthreads();
    if (threadIdx.x == 0) A.done[slice] = A.seq;
}

constexpr int G6_SMALL_MAXI = 64;

// The i-records of a small call, passed by value in the kernel's parameter block: no separate
// upload (and no host-to-device copy latency) for a call of up to G6_SMALL_MAXI i-particles.
struct G6IBlock {
    G6I rec[G6_SMALL_MAXI];
};

template <int ISL, int JL, bool FF, bool NN, bool NBL>
__global__ void __launch_bounds__(ISL * JL, 2)
    g6_small_kernel(const G6SmallArgs A, const __grid_constant__ G6IBlock ib) {
    namespace cg = cooperative_groups;
    constexpr int NT = ISL * JL;
    static_assert(ISL <= G6_SMALL_MAXI, "i-slots within the i-block");
    __shared__ __align__(16) unsigned char smem[NT * sizeof(G6Out)];  // j tile, then per-thread sums
    __shared__ double2 cta_w[4 * ISL];                                 // this CTA's sums, by word
    __shared__ G6I s_i[ISL];
    __shared__ int s_flag;
    G6PredJ* sj = reinterpret_cast<G6PredJ*>(smem);
    const int slot = threadIdx.x % ISL, jl = threadIdx.x / ISL;
    const int nch = gridDim.x, c = blockIdx.x;
    const int j0 = (int)((long long)c * A.nj / nch), j1 = (int)((long long)(c + 1) * A.nj / nch);

    // the first j tile's loads go out first; meanwhile the i-records are staged from the
    // parameter block into shared memory with warp-uniform (broadcast) constant-bank reads --
    // per-thread reads of different records would serialise in the constant cache
    int jt = j0;
    int nt = min(NT, j1 - jt);
    G6PredJ jr;
    if (threadIdx.x < nt) jr = A.jpred[jt + threadIdx.x];
    for (int r = threadIdx.x / 32; r < A.ni; r += NT / 32) {
        const uint4* src = reinterpret_cast<const uint4*>(&ib.rec[r]);
        const uint4 w0 = src[0], w1 = src[1], w2 = src[2];
        if ((threadIdx.x & 31) == 0) {
            uint4* d = reinterpret_cast<uint4*>(&s_i[r]);
            d[0] = w0;
            d[1] = w1;
            d[2] = w2;
        }
    }
    if (threadIdx.x < nt) sj[threadIdx.x] = jr;
    __syncthreads();

    const int ii = slot < A.ni ? slot : 0;
    const G6I P = s_i[ii];
    const float hinv = g6_hkey(slot < A.ni, P.h2);
    double S[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    float kmin = G6_KEY0;  // gravity_kernel2's initial key and index (:495-496)
    int kadr = -1;
    int* nbc = NBL ? A.nb_count + ii : nullptr;
    int* nbl = NBL ? A.nb_list + (size_t)ii * A.nb_maxlen : nullptr;

    for (;;) {
        G6Acc a{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
        for (int j = jl; j < nt; j += JL)
            g6_pair<FF, NN, NBL>(sj[j], jt + j, P.p, P.vx, P.vy, P.vz, P.id, A.eps2, hinv, a, kmin, kadr, nbc, nbl,
                                 A.nb_maxlen);
        S[0] += (double)a.ax;
        S[1] += (double)a.ay;
        S[2] += (double)a.az;
        S[3] += (double)a.jx;
        S[4] += (double)a.jy;
        S[5] += (double)a.jz;
        S[6] += (double)a.pot;
        jt += NT;
        if (jt >= j1) break;
        nt = min(NT, j1 - jt);
        __syncthreads();
        if (threadIdx.x < nt) sj[threadIdx.x] = A.jpred[jt + threadIdx.x];
        __syncthreads();
    }

    // 1. j-lanes: thread w = 4 slot + word sums that word over the lanes in order
    __syncthreads();
    {
        G6Out o;
        o.ax = S[0]; o.ay = S[1]; o.az = S[2];
        o.jx = S[3]; o.jy = S[4]; o.jz = S[5];
        o.pot = S[6];
        o.key = kmin;
        o.jadr = kadr;
        reinterpret_cast<G6Out*>(smem)[threadIdx.x] = o;
    }
    __syncthreads();
    const int nw = 4 * A.ni;
    const double2* rw = reinterpret_cast<const double2*>(smem);
    if (threadIdx.x < nw) {
        const bool w3 = (threadIdx.x & 3) == 3;
        const int s = threadIdx.x >> 2, wd = threadIdx.x & 3;
        double2 v = rw[4 * s + wd];
        for (int l = 1; l < JL; l++) v = word_add(v, rw[4 * (l * ISL + s) + wd], w3);
        if (nch == 1) {
            // the whole call in one CTA: final result directly
            reinterpret_cast<double2*>(A.out)[threadIdx.x] = word_finish(v, w3);
        }
        cta_w[threadIdx.x] = v;
    }
    if (nch == 1) {
        publish_done(A, 0);
        return;
    }

    // 2. the cluster: CTA `rank` reduces words [f0, f1) over the cluster's CTAs, in rank order,
    //    into the cluster's row
    cg::cluster_group cl = cg::this_cluster();
    const int CL = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    cl.sync();
    const int f0 = rank * nw / CL, f1 = (rank + 1) * nw / CL;
    const int f = f0 + (int)threadIdx.x;
    if (f < f1) {
        const bool w3 = (f & 3) == 3;
        double2 v = *cl.map_shared_rank(&cta_w[f], 0);
        for (int q = 1; q < CL; q++) v = word_add(v, *cl.map_shared_rank(&cta_w[f], q), w3);
        reinterpret_cast<double2*>(A.partial + (size_t)(c / CL) * ISL)[f] = v;
    }

    // 3. slice `rank` of every cluster row was written by that cluster's CTA `rank`: those CTAs
    //    arrive on counter[rank], and the last of them sums the slice over the rows in order
    const int nclus = nch / CL;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const int prev = atomicAdd(&A.counter[rank], 1);
        const int last = (prev == nclus - 1);
        if (last) atomicExch(&A.counter[rank], 0);
        s_flag = last;
    }
    __syncthreads();
    if (s_flag) {
        __threadfence();
        reduce_rows<NT>(A.partial, (size_t)ISL, nclus, f0, f1 - f0, A.out, true, reinterpret_cast<double2*>(smem));
        publish_done(A, rank);
    }
    cl.sync();  // no CTA leaves while a peer may still read its cta_w
}

}  // namespace pgb
