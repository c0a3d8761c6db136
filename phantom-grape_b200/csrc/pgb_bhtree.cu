// pgb_bhtree.cu -- lib/libpgbtree.so: the Barnes-Hut octree, its multipole moments, the i-groups
// and every group's interaction list, built on the GPU.
//
// Reference: the tree code that drives PG5/newton_quad's g5_* / g5c_* calls
// (PG5/newton_quad/source.cpp): octree construction (source.cpp:418-514, childindex :177-197),
// cell moments (:215-248, 544-576), group selection (:477-482, 510-514) and
// make_interaction_list / calc_dist (:581-707).  The rules are the ones the host builder
// drivers/pgb_bhtree.c restates (and tests/test_bhtree.py checks against a plain restatement of
// make_interaction_list); this library produces the same tree -- particle order, node numbering,
// moments, groups and lists, bit for bit -- on the device, so the batched force launch can take
// its lists without a host round trip:
//  * root: the cube centred on the origin whose half side is the smallest power of two above
//    every |coordinate|;
//  * a node holding more than nleaf particles (and less than 40 levels deep) is split; a
//    particle goes to the octant ((x > c_x) << 2 | (y > c_y) << 1 | (z > c_z)) of the node centre
//    c, the particles of each child keep their order (stable partition);
//  * nodes are numbered in depth-first pre-order, children in octant order (the recursion's
//    creation order);
//  * moments in FP64: a leaf from its particles in tree order, an internal node from its
//    children in octant order (mass, centre of mass, traceless quadrupole by the parallel-axis
//    shift), every multiply and add rounded separately (no fused multiply-add), as the C code;
//  * groups: the first node on each root-to-leaf path with at most ncrit particles or no
//    children, in pre-order;
//  * lists: the depth-first walk of the host builder (particles of small nodes and single-
//    particle children, quadrupole cells that pass theta^2 d^2 > side^2 with d the distance from
//    the cell's centre of mass to the group's cube).
//
// Construction is level by level: at each level the particles of every splitting node are
// cut into tiles (of HT_TILE for a CTA, or of HT_TILE_W for a warp where the level's nodes are
// many and small); one kernel computes octants and per-tile octant counts, a CTA, warp or thread
// per node scans its tiles in order (tile offsets, child sizes), children are allocated with a
// prefix sum, and a scatter kernel places each particle at child start + tile offset + its rank
// among the tile's particles of the same octant (warp ballots) -- a stable partition, as the
// host's counting sort.  Pre-order numbers follow from subtree sizes; moments are computed
// bottom-up one level at a time; lists by 64 threads per group (one per grandchild of the root,
// each walking the pre-order node array without a stack), a counting pass, a prefix sum and a
// filling pass.
#include "pgb_common.cuh"

using namespace pgb;

namespace {

const char* LIB = "libpgbtree";
ErrorSlot g_err;

constexpr int HT_MAXDEPTH = 40;   // the host builder's depth cap
constexpr int HT_TILE = 2048;     // particles per tile of the partition kernels (a CTA per tile)
constexpr int HT_TILE_W = 512;    // the same for a warp per tile
constexpr int HT_NT = 256;        // threads per CTA of the tile kernels
constexpr int HT_SMALL_LEVEL = 4096;     // levels of at least this many nodes: a warp per tile
constexpr int HT_WARP_SCAN_LEVEL = 131072; // levels of 513 up to this many nodes: a warp per node

// ---- device helpers ---------------------------------------------------------------------

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }

// ---- exclusive prefix sum (any length) ----------------------------------------------------

constexpr int SC_NT = 256, SC_PER = 8, SC_TILE = SC_NT * SC_PER;

template <class T>
__device__ __forceinline__ T block_excl_scan(T v, T* sh, T* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T u = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += u;
    }
    __syncthreads();
    if (lane == 31) sh[w] = x;
    __syncthreads();
    T base = 0, all = 0;
#pragma unroll
    for (int k = 0; k < SC_NT / 32; k++) {
        base += k < w ? sh[k] : T(0);
        all += sh[k];
    }
    *total = all;
    return x - v + base;
}

template <class T>
__global__ void __launch_bounds__(SC_NT) scan_partial(const T* in, long long n, T* bsum) {
    __shared__ T sh[SC_NT / 32];
    const long long b0 = (long long)blockIdx.x * SC_TILE + (long long)threadIdx.x * SC_PER;
    T s = 0;
#pragma unroll
    for (int r = 0; r < SC_PER; r++)
        if (b0 + r < n) s += in[b0 + r];
    T tot;
    block_excl_scan<T>(s, sh, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

template <class T>
__global__ void __launch_bounds__(SC_NT) scan_final(const T* in, long long n, const T* boff, T* out) {
    __shared__ T sh[SC_NT / 32];
    const long long b0 = (long long)blockIdx.x * SC_TILE + (long long)threadIdx.x * SC_PER;
    T v[SC_PER];
    T s = 0;
#pragma unroll
    for (int r = 0; r < SC_PER; r++) {
        v[r] = (b0 + r < n) ? in[b0 + r] : T(0);
        s += v[r];
    }
    T tot;
    T run = block_excl_scan<T>(s, sh, &tot) + boff[blockIdx.x];
#pragma unroll
    for (int r = 0; r < SC_PER; r++) {
        if (b0 + r < n) out[b0 + r] = run;
        run += v[r];
    }
}

// out[k] = sum_{j<k} in[j] for k <= n (out has n + 1 entries; in and out may not alias).
// tmp: the block-sum buffers of the levels (two per level; the vector is sized once, before
// any reference into it is taken, so the recursion never reallocates it).
constexpr int SC_MAXLVL = 8;
template <class T>
bool excl_scan(const T* in, long long n, T* out, cudaStream_t s, std::vector<DevBuf<T>>& tmp, int lvl = 0) {
    const long long nb = (n + SC_TILE - 1) / SC_TILE;
    if (lvl == 0 && (int)tmp.size() < 2 * SC_MAXLVL) tmp.resize(2 * SC_MAXLVL);
    if (lvl >= SC_MAXLVL) {
        raise(g_err, LIB, PGB_ERR_CAPACITY, "prefix sum of %lld entries: too many levels", n);
        return false;
    }
    DevBuf<T>& bs = tmp[2 * lvl];
    DevBuf<T>& bo = tmp[2 * lvl + 1];
    PGB_CUDA_OR(g_err, LIB, bs.reserve((size_t)nb + 1), return false);
    PGB_CUDA_OR(g_err, LIB, bo.reserve((size_t)nb + 2), return false);
    if (n == 0) {
        PGB_CUDA_OR(g_err, LIB, cudaMemsetAsync(out, 0, sizeof(T), s), return false);
        return true;
    }
    scan_partial<T><<<(unsigned)nb, SC_NT, 0, s>>>(in, n, bs.p);
    if (nb == 1) {
        PGB_CUDA_OR(g_err, LIB, cudaMemsetAsync(bo.p, 0, sizeof(T), s), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(bo.p + 1, bs.p, sizeof(T), cudaMemcpyDeviceToDevice, s),
                    return false);
    } else if (!excl_scan<T>(bs.p, nb, bo.p, s, tmp, lvl + 1)) {
        return false;
    }
    scan_final<T><<<(unsigned)nb, SC_NT, 0, s>>>(in, n, bo.p, out);
    // the total
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(out + n, bo.p + nb, sizeof(T), cudaMemcpyDeviceToDevice, s), return false);
    PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return false);
    return true;
}

// ---- construction kernels -----------------------------------------------------------------

struct Nodes {   // breadth-first node arrays (construction order)
    int *first, *count, *parent, *child;   // child: [8] per node
    double *c, *half;                      // c: [3] per node
};

__device__ __forceinline__ bool splits(int count, int level, int nleaf) {
    return count > nleaf && level < HT_MAXDEPTH;
}

// Tiles of a level's splitting nodes: ntile[v - b] for nodes [b, e).
__global__ void k_ntiles(Nodes N, int b, int e, int level, int nleaf, int tile, int* ntile) {
    const int v = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= e) return;
    const int c = N.count[v];
    ntile[v - b] = splits(c, level, nleaf) ? (c + tile - 1) / tile : 0;
}

// The node of every tile: the last node i of the level whose first tile tile_off[i] <= t (a
// node without tiles has the same tile_off as the next node, so the last such is the owner).
__global__ void k_tile_nodes(int b, int cnt, const int* tile_off, const int* ntiles, int* tile_node) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *ntiles) return;
    int lo = 0, hi = cnt - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile_off[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    tile_node[t] = b + lo;
}

// Octant of every particle of a tile and the tile's octant counts.
__global__ void __launch_bounds__(HT_NT) k_octants(Nodes N, const int* tile_node, const int* tile_off, int b,
                                                   const int* ntiles, int tile, const double* x,
                                                   const int* perm, unsigned char* oct, int* tcount) {
    __shared__ int cnt[8];
    const int t = blockIdx.x;
    if (t >= *ntiles) return;
    const int v = tile_node[t];
    const int lt = t - tile_off[v - b];
    const int k0 = N.first[v] + lt * tile;
    const int k1 = min(N.first[v] + N.count[v], k0 + tile);
    if (threadIdx.x < 8) cnt[threadIdx.x] = 0;
    __syncthreads();
    const double cx = N.c[3 * v], cy = N.c[3 * v + 1], cz = N.c[3 * v + 2];
    for (int k = k0 + threadIdx.x; k < k1; k += HT_NT) {
        const double* p = x + 3 * (size_t)perm[k];
        const int o = ((p[0] > cx) << 2) | ((p[1] > cy) << 1) | (p[2] > cz);
        oct[k] = (unsigned char)o;
        atomicAdd(&cnt[o], 1);
    }
    __syncthreads();
    if (threadIdx.x < 8) tcount[8 * t + threadIdx.x] = cnt[threadIdx.x];
}

// The same with one warp per tile, for levels of many small nodes (a tile of a few dozen
// particles would leave most of a CTA idle): lane o < 8 keeps octant o's count.
__global__ void __launch_bounds__(HT_NT) k_octants_w(Nodes N, const int* tile_node, const int* tile_off, int b,
                                                     const int* ntiles, int tile, const double* x,
                                                     const int* perm, unsigned char* oct, int* tcount) {
    const int t = (int)((blockIdx.x * (unsigned)HT_NT + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= *ntiles) return; // whole warps
    const int v = tile_node[t];
    const int lt = t - tile_off[v - b];
    const int k0 = N.first[v] + lt * tile;
    const int k1 = min(N.first[v] + N.count[v], k0 + tile);
    const double cx = N.c[3 * v], cy = N.c[3 * v + 1], cz = N.c[3 * v + 2];
    int cnt = 0;
    for (int r0 = k0; r0 < k1; r0 += 32) {
        const int k = r0 + lane;
        int o = 8;
        if (k < k1) {
            const double* p = x + 3 * (size_t)perm[k];
            o = ((p[0] > cx) << 2) | ((p[1] > cy) << 1) | (p[2] > cz);
            oct[k] = (unsigned char)o;
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const unsigned m = __ballot_sync(0xffffffffu, o == q);
            if (lane == q) cnt += __popc(m);
        }
    }
    if (lane < 8) tcount[8 * t + lane] = cnt;
}

// Per splitting node: its tiles' offsets within each octant (in tile order), the child sizes
// and the number of non-empty children.
__global__ void k_node_scan(Nodes N, int b, int e, int level, int nleaf, const int* tile_off, const int* tcount,
                            int* tbase, int* ccount, int* nkids) {
    const int v = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= e) return;
    int run[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = tile_off[v - b]; t < tile_off[v - b + 1]; t++)
        for (int o = 0; o < 8; o++) {
            tbase[8 * t + o] = run[o];
            run[o] += tcount[8 * t + o];
        }
    int nk = 0;
    for (int o = 0; o < 8; o++) {
        ccount[8 * (v - b) + o] = run[o];
        nk += run[o] > 0;
    }
    nkids[v - b] = splits(N.count[v], level, nleaf) ? nk : 0;
}

// The same for a level of few nodes (the top of the tree, where a node has up to thousands of
// tiles): one CTA per node, HT_NT threads each over a contiguous run of its tiles -- the runs'
// octant sums, their exclusive scan in thread order through shared memory, then each thread's
// tiles' offsets.  Integer sums in tile order: the same offsets as k_node_scan.
__global__ void __launch_bounds__(HT_NT) k_node_scan_cta(Nodes N, int b, int level, int nleaf, const int* tile_off,
                                                         const int* tcount, int* tbase, int* ccount, int* nkids) {
    __shared__ int part[HT_NT][8];
    __shared__ int total[8];
    const int v = b + blockIdx.x;
    const int t0 = tile_off[v - b], t1 = tile_off[v - b + 1];
    const int per = (t1 - t0 + HT_NT - 1) / HT_NT;
    const int a = min(t0 + (int)threadIdx.x * per, t1), z = min(a + per, t1);
    int run[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = a; t < z; t++)
#pragma unroll
        for (int o = 0; o < 8; o++) run[o] += tcount[8 * t + o];
#pragma unroll
    for (int o = 0; o < 8; o++) part[threadIdx.x][o] = run[o];
    __syncthreads();
    if (threadIdx.x < 8) {
        // exclusive scan of column o over the threads, in thread order
        const int o = threadIdx.x;
        int acc = 0;
        for (int q = 0; q < HT_NT; q++) {
            const int c = part[q][o];
            part[q][o] = acc;
            acc += c;
        }
        total[o] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int o = 0; o < 8; o++) run[o] = part[threadIdx.x][o];
    for (int t = a; t < z; t++)
#pragma unroll
        for (int o = 0; o < 8; o++) {
            tbase[8 * t + o] = run[o];
            run[o] += tcount[8 * t + o];
        }
    if (threadIdx.x == 0) {
        int nk = 0;
        for (int o = 0; o < 8; o++) {
            ccount[8 * (v - b) + o] = total[o];
            nk += total[o] > 0;
        }
        nkids[v - b] = splits(N.count[v], level, nleaf) ? nk : 0;
    }
}

// The same for levels of a few thousand nodes (a dense centre leaves some of them hundreds of
// tiles): one warp per node, each lane over a contiguous run of its tiles, the runs' octant
// sums scanned across the lanes with shuffles.
__global__ void __launch_bounds__(256) k_node_scan_warp(Nodes N, int b, int e, int level, int nleaf,
                                                        const int* tile_off, const int* tcount, int* tbase,
                                                        int* ccount, int* nkids) {
    const int v = b + (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (v >= e) return; // whole warps
    const int t0 = tile_off[v - b], t1 = tile_off[v - b + 1];
    const int per = (t1 - t0 + 31) >> 5;
    const int a = min(t0 + lane * per, t1), z = min(a + per, t1);
    int run[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = a; t < z; t++)
#pragma unroll
        for (int o = 0; o < 8; o++) run[o] += tcount[8 * t + o];
    int nk = 0;
#pragma unroll
    for (int o = 0; o < 8; o++) {
        int x = run[o];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        const int total = __shfl_sync(0xffffffffu, x, 31);
        if (lane == 0) ccount[8 * (v - b) + o] = total;
        nk += total > 0;
        run[o] = x - run[o]; // exclusive
    }
    for (int t = a; t < z; t++)
#pragma unroll
        for (int o = 0; o < 8; o++) {
            tbase[8 * t + o] = run[o];
            run[o] += tcount[8 * t + o];
        }
    if (lane == 0) nkids[v - b] = splits(N.count[v], level, nleaf) ? nk : 0;
}

// Children of the level's splitting nodes, appended from index e + kid_off[v - b].
__global__ void k_children(Nodes N, int b, int e, int level, int nleaf, const int* ccount, const int* kid_off) {
    const int v = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= e) return;
    for (int o = 0; o < 8; o++) N.child[8 * v + o] = -1;
    if (!splits(N.count[v], level, nleaf)) return;
    const double half = 0.5 * N.half[v];
    int w = e + kid_off[v - b];
    int start = N.first[v];
    for (int o = 0; o < 8; o++) {
        const int c = ccount[8 * (v - b) + o];
        if (c == 0) continue;
        N.first[w] = start;
        N.count[w] = c;
        N.parent[w] = v;
        N.half[w] = half;
        N.c[3 * w] = N.c[3 * v] + ((o & 4) ? half : -half);
        N.c[3 * w + 1] = N.c[3 * v + 1] + ((o & 2) ? half : -half);
        N.c[3 * w + 2] = N.c[3 * v + 2] + ((o & 1) ? half : -half);
        N.child[8 * v + o] = w;
        start += c;
        w++;
    }
}

// Stable scatter of a tile's particles to their children: child start + the tile's offset in
// the octant + the particle's rank among the tile's earlier particles of the same octant.
__global__ void __launch_bounds__(HT_NT) k_scatter(Nodes N, const int* tile_node, const int* tile_off, int b,
                                                   const int* ntiles, int tile, const unsigned char* oct,
                                                   const int* tbase, const int* perm, int* perm2) {
    __shared__ int wcnt[HT_NT / 32][8];
    __shared__ int run[8];
    __shared__ int cstart[8];
    const int t = blockIdx.x;
    if (t >= *ntiles) return;
    const int v = tile_node[t];
    const int lt = t - tile_off[v - b];
    const int k0 = N.first[v] + lt * tile;
    const int k1 = min(N.first[v] + N.count[v], k0 + tile);
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    if (threadIdx.x < 8) {
        run[threadIdx.x] = tbase[8 * t + threadIdx.x];
        const int w = N.child[8 * v + threadIdx.x];
        cstart[threadIdx.x] = w >= 0 ? N.first[w] : 0;
    }
    __syncthreads();
    for (int r0 = k0; r0 < k1; r0 += HT_NT) {
        const int k = r0 + threadIdx.x;
        const bool in = k < k1;
        const int o = in ? oct[k] : 8;
        int rank = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const unsigned m = __ballot_sync(0xffffffffu, o == q);
            if (o == q) rank = __popc(m & ((1u << lane) - 1u));
            if (lane == 0) wcnt[wi][q] = __popc(m);
        }
        __syncthreads();
        if (in) {
            int before = 0;
            for (int w2 = 0; w2 < wi; w2++) before += wcnt[w2][o];
            perm2[cstart[o] + run[o] + before + rank] = perm[k];
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            int s = 0;
            for (int w2 = 0; w2 < HT_NT / 32; w2++) s += wcnt[w2][threadIdx.x];
            run[threadIdx.x] += s;
        }
        __syncthreads();
    }
}

// The same with one warp per tile: lane o < 8 keeps octant o's next destination (the child's
// start + the tile's offset in the octant + the octant's particles so far), ranks within a
// chunk of 32 from the octant's ballot.
__global__ void __launch_bounds__(HT_NT) k_scatter_w(Nodes N, const int* tile_node, const int* tile_off, int b,
                                                     const int* ntiles, int tile, const unsigned char* oct,
                                                     const int* tbase, const int* perm, int* perm2) {
    const int t = (int)((blockIdx.x * (unsigned)HT_NT + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= *ntiles) return; // whole warps
    const int v = tile_node[t];
    const int lt = t - tile_off[v - b];
    const int k0 = N.first[v] + lt * tile;
    const int k1 = min(N.first[v] + N.count[v], k0 + tile);
    int dst = 0;
    if (lane < 8) {
        const int w = N.child[8 * v + lane];
        dst = (w >= 0 ? N.first[w] : 0) + tbase[8 * t + lane];
    }
    const unsigned below = (1u << lane) - 1u;
    for (int r0 = k0; r0 < k1; r0 += 32) {
        const int k = r0 + lane;
        const bool in = k < k1;
        const int o = in ? oct[k] : 8;
        unsigned mine = 0;
        int add = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const unsigned m = __ballot_sync(0xffffffffu, o == q);
            if (o == q) mine = m;
            if (lane == q) add = __popc(m);
        }
        const int base = __shfl_sync(0xffffffffu, dst, o & 7);
        if (in) perm2[base + __popc(mine & below)] = perm[k];
        dst += add;
    }
}

// ---- pre-order numbering ------------------------------------------------------------------

__global__ void k_subtree(Nodes N, int b, int e, int* size) {
    const int v = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= e) return;
    int s = 1;
    for (int o = 0; o < 8; o++) {
        const int w = N.child[8 * v + o];
        if (w >= 0) s += size[w];
    }
    size[v] = s;
}

__global__ void k_preorder(Nodes N, int b, int e, const int* size, int* pre) {
    const int v = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= e) return;
    int run = pre[v] + 1;
    for (int o = 0; o < 8; o++) {
        const int w = N.child[8 * v + o];
        if (w < 0) continue;
        pre[w] = run;
        run += size[w];
    }
}

struct Tree {   // pre-order output arrays
    int *first, *count, *child;
    double *c, *half, *com, *mass, *quad;
};

__global__ void k_to_preorder(Nodes N, int nn, const int* pre, Tree T, const int* size, int* sizep) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    const int p = pre[v];
    sizep[p] = size[v];
    T.first[p] = N.first[v];
    T.count[p] = N.count[v];
    T.half[p] = N.half[v];
    for (int a = 0; a < 3; a++) T.c[3 * p + a] = N.c[3 * v + a];
    for (int o = 0; o < 8; o++) {
        const int w = N.child[8 * v + o];
        T.child[8 * p + o] = w >= 0 ? pre[w] : -1;
    }
}

__global__ void k_gather(int n, const int* perm, const double* x, const double* m, double* xt, double* mt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int p = perm[k];
    xt[3 * (size_t)k] = x[3 * (size_t)p];
    xt[3 * (size_t)k + 1] = x[3 * (size_t)p + 1];
    xt[3 * (size_t)k + 2] = x[3 * (size_t)p + 2];
    mt[k] = m[p];
}

// ---- moments ------------------------------------------------------------------------------

// q += m (3 d d - |d|^2 I) (xx, xy, xz, yy, yz), the host's operation order
__device__ __forceinline__ void quad_add(double q[6], double m, const double d[3]) {
    const double dd = da(da(dm(d[0], d[0]), dm(d[1], d[1])), dm(d[2], d[2]));
    q[0] = da(q[0], dm(m, ds(dm(dm(3.0, d[0]), d[0]), dd)));
    q[1] = da(q[1], dm(m, dm(dm(3.0, d[0]), d[1])));
    q[2] = da(q[2], dm(m, dm(dm(3.0, d[0]), d[2])));
    q[3] = da(q[3], dm(m, ds(dm(dm(3.0, d[1]), d[1]), dd)));
    q[4] = da(q[4], dm(m, dm(dm(3.0, d[1]), d[2])));
}

// Moments of the nodes of one level (pre-order indices in `list`), children already done.
__global__ void k_moments(Tree T, const int* list, int cnt, const double* xt, const double* mt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const int v = list[i];
    bool leaf = true;
    for (int o = 0; o < 8; o++) leaf = leaf && T.child[8 * v + o] < 0;
    double m = 0.0, s[3] = {0.0, 0.0, 0.0}, q[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, com[3];
    const int first = T.first[v], count = T.count[v];
    if (leaf) {
        for (int k = first; k < first + count; k++) {
            m = da(m, mt[k]);
            for (int a = 0; a < 3; a++) s[a] = da(s[a], dm(mt[k], xt[3 * (size_t)k + a]));
        }
        for (int a = 0; a < 3; a++) com[a] = s[a] / m;
        if (count > 1)
            for (int k = first; k < first + count; k++) {
                const double d[3] = {ds(xt[3 * (size_t)k], com[0]), ds(xt[3 * (size_t)k + 1], com[1]),
                                     ds(xt[3 * (size_t)k + 2], com[2])};
                quad_add(q, mt[k], d);
            }
    } else {
        for (int o = 0; o < 8; o++) {
            const int w = T.child[8 * v + o];
            if (w < 0) continue;
            m = da(m, T.mass[w]);
            for (int a = 0; a < 3; a++) s[a] = da(s[a], dm(T.mass[w], T.com[3 * w + a]));
        }
        for (int a = 0; a < 3; a++) com[a] = s[a] / m;
        for (int o = 0; o < 8; o++) {
            const int w = T.child[8 * v + o];
            if (w < 0) continue;
            const double d[3] = {ds(T.com[3 * w], com[0]), ds(T.com[3 * w + 1], com[1]), ds(T.com[3 * w + 2], com[2])};
            quad_add(q, T.mass[w], d);
            if (T.count[w] > 1)
                for (int k = 0; k < 5; k++) q[k] = da(q[k], T.quad[6 * w + k]);
        }
    }
    q[5] = -da(q[0], q[3]);
    T.mass[v] = m;
    for (int a = 0; a < 3; a++) T.com[3 * v + a] = com[a];
    for (int k = 0; k < 6; k++) T.quad[6 * v + k] = q[k];
}

// ---- groups and lists ---------------------------------------------------------------------

__device__ __forceinline__ bool is_leaf(const Tree& T, int v) {
    for (int o = 0; o < 8; o++)
        if (T.child[8 * v + o] >= 0) return false;
    return true;
}

// flag[p] = 1 for the group nodes (pre-order p); parent[] in pre-order
__global__ void k_group_flags(Tree T, const int* ppar, int nn, int ncrit, int* flag) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    const bool cond = T.count[v] <= ncrit || is_leaf(T, v);
    const int p = ppar[v];
    flag[v] = cond && (p < 0 || T.count[p] > ncrit);
}

__global__ void k_parent_pre(Tree T, int nn, int* ppar) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    if (v == 0) ppar[0] = -1;
    for (int o = 0; o < 8; o++) {
        const int w = T.child[8 * v + o];
        if (w >= 0) ppar[w] = v;
    }
}

__global__ void k_compact(const int* flag, const int* off, int nn, int* out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    if (flag[v]) out[off[v]] = v;
}

// What the list walk reads of a node, packed: centre of mass, side^2 (side = 2 x half side),
// particle range and kind (WK_ONE: a single particle; WK_PARTS: at most nleaf particles or
// no children -- the walk takes its particles; WK_SPLIT: walked further if not accepted), and
// the nodes in its subtree (itself included: in pre-order the subtree is [v, v + nsub)).
enum { WK_ONE = 0, WK_PARTS = 1, WK_SPLIT = 2 };
struct __align__(16) WalkNode {
    double com[3];
    double side2;
    int first, count, kind, nsub;
};

__global__ void k_walk_nodes(Tree T, int nn, int nleaf, const int* sizep, WalkNode* wn) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    WalkNode w;
    for (int a = 0; a < 3; a++) w.com[a] = T.com[3 * v + a];
    const double side = 2.0 * T.half[v];
    w.side2 = dm(side, side);
    w.first = T.first[v];
    w.count = T.count[v];
    w.kind = w.count == 1 ? WK_ONE : ((w.count <= nleaf || is_leaf(T, v)) ? WK_PARTS : WK_SPLIT);
    w.nsub = sizep[v];
    wn[v] = w;
}

// distance^2 from point p to the cube (centre g, half side h), calc_dist's order
__device__ __forceinline__ double box_d2(const double* p, const double g[3], double h) {
    double d2 = 0.0;
    for (int a = 0; a < 3; a++) {
        const double d = ds(fabs(ds(p[a], g[a])), h);
        if (d > 0) d2 = da(d2, dm(d, d));
    }
    return d2;
}

// The interaction lists are made by HT_UNITS work units per group, so that the walks spread
// over many threads: unit u, whose base-8 digits (o_1 .. o_D, most significant first) name a
// node D levels below the root, produces the part of the group's list that the host builder's
// depth-first walk (make_interaction_list) produces inside that node's subtree.  Where the walk
// takes a node of level l < D whole (its particle, itself as a cell, or its particles), the unit
// whose digits below l are zero emits it.  The units' lists, concatenated in unit order, are the
// group's list.  Most of a group's list lies in the few units around the group itself, so the
// depth sets how many threads share that work: at D = 2 the long walks of an N = 2^20 tree fill
// ~3 warps per SM.
constexpr int HT_UNIT_LEVELS = 2;
constexpr int HT_UNITS = 1 << (3 * HT_UNIT_LEVELS);
// threads per block of the list walks: a block stays resident until its slowest walk ends, so
// smaller blocks keep fewer finished warps idle (N = 2^22 build: 12.3 ms with 128, 12.7 with
// 64, 13.0 with 256 threads)
constexpr int HT_WALK_NT = 128;

// The count walk's output: the numbers of point-mass and cell entries.
struct ListCount {
    long long a = 0, b = 0;
    __device__ __forceinline__ void part(int) { a++; }
    __device__ __forceinline__ void parts(int, int n) { a += n; }
    __device__ __forceinline__ void cell(int) { b++; }
    __device__ __forceinline__ void flush() {}
};

// One list of the fill walk, written in aligned 16-byte chunks: the entries of the current chunk
// wait in the thread's four staging slots in shared memory (slot j at sm[j * HT_WALK_NT], so that
// the lanes' slots lie in distinct banks) and go out as one vector store when the last slot is
// filled.  The first chunk's slots before the list's start, and the last chunk's slots after its
// end, belong to the neighbouring units' lists: a partial chunk is written entry by entry.  A lane
// stores one sector per four entries instead of one per entry.
struct ChunkOut {
    int* c;  // the current chunk (16-byte aligned)
    int* sm; // the staging slots
    int s;   // the next entry's slot
    int s0;  // the current chunk's first slot that belongs to this list
    __device__ __forceinline__ ChunkOut(int* q, int* stage) : sm(stage) {
        s = s0 = (int)((reinterpret_cast<unsigned long long>(q) >> 2) & 3);
        c = q - s;
    }
    __device__ __forceinline__ void out() {
        if (s0 == 0) {
            *reinterpret_cast<int4*>(c) = make_int4(sm[0], sm[HT_WALK_NT], sm[2 * HT_WALK_NT], sm[3 * HT_WALK_NT]);
        } else {
            for (int j = s0; j < 4; j++) c[j] = sm[j * HT_WALK_NT];
        }
        c += 4;
        s = s0 = 0;
    }
    __device__ __forceinline__ void push(int k) {
        sm[s * HT_WALK_NT] = k;
        if (++s == 4) out();
    }
    // the n consecutive entries k, k + 1, ...: pushed one by one up to a chunk boundary (where
    // the chunk before has just gone out, or the list starts), then whole chunks stored directly
    __device__ __forceinline__ void push_range(int k, int n) {
        for (; n > 0 && s != 0; n--) push(k++);
        for (; n >= 4; n -= 4, k += 4, c += 4) *reinterpret_cast<int4*>(c) = make_int4(k, k + 1, k + 2, k + 3);
        for (; n > 0; n--) push(k++);
    }
    // the pending entries: slots s0 .. s - 1 of the current chunk
    __device__ __forceinline__ void flush() {
        for (int j = s0; j < s; j++) c[j] = sm[j * HT_WALK_NT];
    }
};

struct ListFill {
    ChunkOut P, C; // point-mass and cell entries
    __device__ __forceinline__ void part(int k) { P.push(k); }
    __device__ __forceinline__ void parts(int k, int n) { P.push_range(k, n); }
    __device__ __forceinline__ void cell(int w) { C.push(w); }
    __device__ __forceinline__ void flush() {
        P.flush();
        C.flush();
    }
};

// A node the walk reaches: its particle (one particle), itself as a cell (theta^2 d^2 >
// side^2), its particles (at most nleaf or no children) -- or false: the walk descends.
template <class ListOut>
__device__ __forceinline__ bool take_node(const WalkNode& C, int w, const double g[3], double h, double th2,
                                          ListOut& L) {
    if (C.kind == WK_ONE) {
        L.part(C.first);
        return true;
    }
    if (dm(box_d2(C.com, g, h), th2) > C.side2) {
        L.cell(w);
        return true;
    }
    if (C.kind == WK_PARTS) {
        L.parts(C.first, C.count);
        return true;
    }
    return false;
}

// Depth-first walk below node v (descended into), children in octant order.  The nodes are in
// pre-order, so the walk needs no stack: a node taken whole is followed by the node after its
// subtree (w + nsub), a node descended into by its first child (w + 1), and the walk ends at
// the end of v's subtree -- the same nodes in the same order as a recursive walk over the
// children, one node record read per step.
template <class ListOut>
__device__ void walk_below(const Tree& T, const WalkNode* __restrict__ wn, int v, const double g[3], double h,
                           double th2, ListOut& L) {
    (void)T;
    const int end = v + wn[v].nsub;
    for (int w = v + 1; w < end;) {
        const WalkNode C = wn[w];
        w += take_node(C, w, g, h, th2, L) ? C.nsub : 1;
    }
}

// Work unit u of the group with node gv.  The root: the group's list is the root as one cell
// when the root passes the opening test (group_list of the host builder), the root's particles
// when it has at most nleaf particles or no children; unit 0 emits either.
template <class ListOut>
__device__ void unit_walk(const Tree& T, const WalkNode* __restrict__ wn, int gv, int u, double th2, ListOut& L) {
    const double g[3] = {T.c[3 * gv], T.c[3 * gv + 1], T.c[3 * gv + 2]};
    const double h = T.half[gv];
    const WalkNode R = wn[0];
    if (!(dm(box_d2(R.com, g, h), th2) < R.side2)) {
        if (u == 0) L.cell(0);
        return;
    }
    if (R.kind != WK_SPLIT) {
        if (u == 0) L.parts(R.first, R.count);
        return;
    }
    int v = 0; // a node the walk descends into
#pragma unroll
    for (int l = 1; l <= HT_UNIT_LEVELS; l++) {
        const int below = 3 * (HT_UNIT_LEVELS - l);
        const int c = T.child[8 * v + ((u >> below) & 7)];
        if (c < 0) return;
        const WalkNode C = wn[c];
        if (l == HT_UNIT_LEVELS) {
            if (!take_node(C, c, g, h, th2, L)) walk_below(T, wn, c, g, h, th2, L);
            return;
        }
        if (C.kind != WK_SPLIT || dm(box_d2(C.com, g, h), th2) > C.side2) {
            if ((u & ((1 << below) - 1)) == 0) take_node(C, c, g, h, th2, L);
            return;
        }
        v = c;
    }
}

// The unit whose node (HT_UNIT_LEVELS levels below the root) holds the group's node gv: its
// octant digits from the centres, as the partition assigns them (a point above a node's centre
// on an axis goes to the upper half).  A group above that depth takes the digits down to itself
// and zeros below.
__device__ __forceinline__ int home_unit(const Tree& T, int gv) {
    const double cx = T.c[3 * gv], cy = T.c[3 * gv + 1], cz = T.c[3 * gv + 2];
    int u = 0, v = 0;
#pragma unroll
    for (int l = 0; l < HT_UNIT_LEVELS; l++) {
        int o = 0;
        if (v >= 0 && v != gv) {
            o = ((cx > T.c[3 * v]) << 2) | ((cy > T.c[3 * v + 1]) << 1) | (int)(cz > T.c[3 * v + 2]);
            v = T.child[8 * v + o];
        }
        u = (u << 3) | o;
    }
    return u;
}

// Thread q takes rank q / ng of group q % ng: the lanes of a warp take the same rank of
// neighbouring groups, whose walks are alike.  Rank r is unit r ^ home: rank 0 is the unit
// around the group (the longest walk), ranks 1-7 its siblings, then the units under the other
// children of the root -- so the long walks start first and the grid's last blocks are short.
// Counts and offsets are stored group-major (g * HT_UNITS + u), the order of the lists.
__global__ void __launch_bounds__(HT_WALK_NT) k_list_count(Tree T, const WalkNode* wn, const int* gnode, int ng,
                                                          double th2, long long* np, long long* nc) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)ng * HT_UNITS) return;
    const int g = (int)(q % ng), gv = gnode[g];
    const int u = (int)(q / ng) ^ home_unit(T, gv);
    ListCount L;
    unit_walk(T, wn, gv, u, th2, L);
    np[(long long)g * HT_UNITS + u] = L.a;
    nc[(long long)g * HT_UNITS + u] = L.b;
}

__global__ void __launch_bounds__(HT_WALK_NT) k_list_fill(Tree T, const WalkNode* wn, const int* gnode, int ng,
                                                         double th2, const long long* uoffp, const long long* uoffc,
                                                         int* pidx, int* cidx) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)ng * HT_UNITS) return;
    const int g = (int)(q % ng), gv = gnode[g];
    const int u = (int)(q / ng) ^ home_unit(T, gv);
    const long long r = (long long)g * HT_UNITS + u;
    __shared__ int stage[2][4][HT_WALK_NT];
    ListFill L{ChunkOut(pidx + uoffp[r], &stage[0][0][threadIdx.x]), ChunkOut(cidx + uoffc[r], &stage[1][0][threadIdx.x])};
    unit_walk(T, wn, gv, u, th2, L);
    L.flush();
}

// per-group offsets from the per-unit offsets (entry ng: the totals)
__global__ void k_group_offsets(int ng, const long long* uoffp, const long long* uoffc, long long* poff,
                                long long* coff) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g > ng) return;
    poff[g] = uoffp[(long long)g * HT_UNITS];
    coff[g] = uoffc[(long long)g * HT_UNITS];
}

__global__ void k_iota(int n, int* p) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) p[k] = k;
}

__global__ void k_maxabs(const double* x, long long n3, unsigned long long* out) {
    double mx = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n3; k += (long long)gridDim.x * blockDim.x)
        mx = fmax(mx, fabs(x[k]));
    // non-negative doubles order like their bit patterns
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}

// Particle and cell records of the batched force launch: float4 (x, y, z, m) in tree order,
// cells float4 (com, mass) + two float4 of the quadrupole (xx, xy, xz, yy) (yz, zz, 0, 0).
__global__ void k_records(int n, int nn, const double* xt, const double* mt, Tree T, float4* part, float4* cell,
                          float4* cquad) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        part[k] = make_float4((float)xt[3 * (size_t)k], (float)xt[3 * (size_t)k + 1], (float)xt[3 * (size_t)k + 2],
                              (float)mt[k]);
    if (k < nn) {
        cell[k] = make_float4((float)T.com[3 * k], (float)T.com[3 * k + 1], (float)T.com[3 * k + 2], (float)T.mass[k]);
        cquad[2 * k] = make_float4((float)T.quad[6 * k], (float)T.quad[6 * k + 1], (float)T.quad[6 * k + 2],
                                   (float)T.quad[6 * k + 3]);
        cquad[2 * k + 1] = make_float4((float)T.quad[6 * k + 4], (float)T.quad[6 * k + 5], 0.f, 0.f);
    }
}

int g_device = -1;
std::mutex g_init_mu;

bool ensure_device() {
    std::lock_guard<std::mutex> g(g_init_mu);
    if (g_device < 0) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
            raise(g_err, LIB, PGB_ERR_NOGPU, "no CUDA device available");
            return false;
        }
        const char* e = std::getenv("PGB_DEVICE");
        int d = e ? std::atoi(e) : 0;
        if (d < 0 || d >= n) d = 0;
        g_device = d;
    }
    PGB_CUDA_OR(g_err, LIB, cudaSetDevice(g_device), return false);
    return true;
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

struct pgbt_tree {
    int n = 0, nn = 0, ng = 0, nleaf = 0, ncrit = 0;
    double theta = 0.0;
    long long np = 0, nc = 0;
    float build_ms = 0.f;
    cudaStream_t s = nullptr;
    DevBuf<double> x, m, xt, mt;
    DevBuf<int> perm, perm2;
    // breadth-first construction arrays
    DevBuf<int> bfirst, bcount, bparent, bchild;
    DevBuf<double> bc, bhalf;
    // pre-order tree
    DevBuf<int> first, count, child, ppar, gnode;
    DevBuf<double> c, half, com, mass, quad;
    DevBuf<long long> poff, coff;
    DevBuf<int> pidx, cidx;
    // force-launch records
    DevBuf<float4> part, cell, cquad;
    // build scratch, kept for the next pgbt_rebuild (released by pgbt_free)
    std::vector<DevBuf<int>> stmp;
    std::vector<DevBuf<long long>> ltmp;
    DevBuf<unsigned long long> mx;
    DevBuf<int> ntile, tile_off, tile_node, tcount, tbase, ccount, nkids, kid_off;
    DevBuf<unsigned char> oct;
    DevBuf<int> size, pre, lvl_pre, gflag, goff;
    DevBuf<int> sizep;   // subtree sizes (nodes) in pre-order, for the stackless list walks
    DevBuf<long long> unp, unc, uoffp, uoffc;
    DevBuf<unsigned char> wn;   // WalkNode records
    // device staging of pgbt_groups / pgbt_group_table (kept: no allocation when a step loop
    // asks every step)
    DevBuf<int> gt_first, gt_count;
    DevBuf<double> gt_centre, gt_half;
};

namespace {

bool grow_nodes(pgbt_tree* T, size_t need, size_t keep) {
    if (need <= T->bfirst.n) return true;
    const size_t want = std::max(need, 2 * T->bfirst.n);
    PGB_CUDA_OR(g_err, LIB, T->bfirst.grow_keep(want, keep, T->s), return false);
    PGB_CUDA_OR(g_err, LIB, T->bcount.grow_keep(want, keep, T->s), return false);
    PGB_CUDA_OR(g_err, LIB, T->bparent.grow_keep(want, keep, T->s), return false);
    PGB_CUDA_OR(g_err, LIB, T->bchild.grow_keep(8 * want, 8 * keep, T->s), return false);
    PGB_CUDA_OR(g_err, LIB, T->bc.grow_keep(3 * want, 3 * keep, T->s), return false);
    PGB_CUDA_OR(g_err, LIB, T->bhalf.grow_keep(want, keep, T->s), return false);
    return true;
}

Nodes bfs(pgbt_tree* T) {
    return Nodes{T->bfirst.p, T->bcount.p, T->bparent.p, T->bchild.p, T->bc.p, T->bhalf.p};
}

template <class V>
bool to_host(V* dst, const V* src, size_t cnt, cudaStream_t s) {
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(dst, src, cnt * sizeof(V), cudaMemcpyDeviceToHost, s), return false);
    return true;
}

bool build(pgbt_tree* T, const double* xh, const double* mh) {
    const int n = T->n;
    cudaStream_t s = T->s;
    std::vector<DevBuf<int>>& stmp = T->stmp;
    std::vector<DevBuf<long long>>& ltmp = T->ltmp;
    PGB_CUDA_OR(g_err, LIB, T->x.reserve(3 * (size_t)n), return false);
    PGB_CUDA_OR(g_err, LIB, T->m.reserve((size_t)n), return false);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(T->x.p, xh, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s),
                return false);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(T->m.p, mh, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s),
                return false);
    cudaEvent_t e0, e1;
    PGB_CUDA_OR(g_err, LIB, cudaEventCreate(&e0), return false);
    PGB_CUDA_OR(g_err, LIB, cudaEventCreate(&e1), return false);
    PGB_CUDA_OR(g_err, LIB, cudaEventRecord(e0, s), return false);

    // root cube: the smallest power of two above every |coordinate|
    DevBuf<unsigned long long>& mx = T->mx;
    PGB_CUDA_OR(g_err, LIB, mx.reserve(1), return false);
    PGB_CUDA_OR(g_err, LIB, mx.zero_fill(s), return false);
    k_maxabs<<<592, 256, 0, s>>>(T->x.p, 3LL * n, mx.p);
    unsigned long long mbits = 0;
    if (!to_host(&mbits, mx.p, 1, s)) return false;
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(s), return false);
    double maxabs;
    std::memcpy(&maxabs, &mbits, sizeof maxabs);
    double R = 1.0;
    if (maxabs > 0) {
        while (R <= maxabs) R *= 2.0;
        while (R * 0.5 > maxabs) R *= 0.5;
    }

    // level-by-level partition
    PGB_CUDA_OR(g_err, LIB, T->perm.reserve((size_t)n), return false);
    PGB_CUDA_OR(g_err, LIB, T->perm2.reserve((size_t)n), return false);
    k_iota<<<nblk(n, 256), 256, 0, s>>>(n, T->perm.p);
    if (!grow_nodes(T, std::max<size_t>(1024, (size_t)n / 4), 0)) return false;
    {
        const int zero = 0, neg = -1;
        const double c0[3] = {0.0, 0.0, 0.0};
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(T->bfirst.p, &zero, sizeof(int), cudaMemcpyHostToDevice, s), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(T->bcount.p, &n, sizeof(int), cudaMemcpyHostToDevice, s), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(T->bparent.p, &neg, sizeof(int), cudaMemcpyHostToDevice, s), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(T->bc.p, c0, sizeof c0, cudaMemcpyHostToDevice, s), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(T->bhalf.p, &R, sizeof(double), cudaMemcpyHostToDevice, s), return false);
        PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(s), return false);
    }
    // per-level scratch, sized once: a level has at most n nodes, at most n / (nleaf + 1) of
    // them split, and their tiles number at most n / tile plus one per splitting node
    DevBuf<int>&ntile = T->ntile, &tile_off = T->tile_off, &tile_node = T->tile_node, &tcount = T->tcount,
                &tbase = T->tbase, &ccount = T->ccount, &nkids = T->nkids, &kid_off = T->kid_off;
    DevBuf<unsigned char>& oct = T->oct;
    const size_t tcap = (size_t)n / HT_TILE_W + (size_t)n / ((size_t)T->nleaf + 1) + 2;
    PGB_CUDA_OR(g_err, LIB, oct.reserve((size_t)n), return false);
    PGB_CUDA_OR(g_err, LIB, ntile.reserve((size_t)n + 1), return false);
    PGB_CUDA_OR(g_err, LIB, tile_off.reserve((size_t)n + 1), return false);
    PGB_CUDA_OR(g_err, LIB, ccount.reserve(8 * (size_t)n), return false);
    PGB_CUDA_OR(g_err, LIB, nkids.reserve((size_t)n + 1), return false);
    PGB_CUDA_OR(g_err, LIB, kid_off.reserve((size_t)n + 1), return false);
    PGB_CUDA_OR(g_err, LIB, tile_node.reserve(tcap), return false);
    PGB_CUDA_OR(g_err, LIB, tcount.reserve(8 * tcap), return false);
    PGB_CUDA_OR(g_err, LIB, tbase.reserve(8 * tcap), return false);
    std::vector<int> lvl = {0, 1};   // level ranges [lvl[L], lvl[L+1])
    for (int L = 0;; L++) {
        const int b = lvl[L], e = lvl[L + 1], cnt = e - b;
        if (cnt <= 0) break;
        Nodes N = bfs(T);
        // a level of many nodes has small ones: a warp per tile of HT_TILE_W instead of a CTA
        // per tile of HT_TILE
        const bool small = cnt >= HT_SMALL_LEVEL;
        const int tile = small ? HT_TILE_W : HT_TILE;
        k_ntiles<<<nblk(cnt, 256), 256, 0, s>>>(N, b, e, L, T->nleaf, tile, ntile.p);
        if (!excl_scan<int>(ntile.p, cnt, tile_off.p, s, stmp)) return false;
        // the tile kernels run on a grid that covers every possible tile; the count itself
        // stays on the device (tile_off[cnt])
        const unsigned tgrid = (unsigned)std::min<size_t>(tcap, (size_t)n / tile + (size_t)cnt + 2);
        k_tile_nodes<<<nblk(tgrid, 256), 256, 0, s>>>(b, cnt, tile_off.p, tile_off.p + cnt, tile_node.p);
        if (small)
            k_octants_w<<<nblk(tgrid, HT_NT / 32), HT_NT, 0, s>>>(N, tile_node.p, tile_off.p, b, tile_off.p + cnt,
                                                                 tile, T->x.p, T->perm.p, oct.p, tcount.p);
        else
            k_octants<<<tgrid, HT_NT, 0, s>>>(N, tile_node.p, tile_off.p, b, tile_off.p + cnt, tile, T->x.p,
                                             T->perm.p, oct.p, tcount.p);
        // the tile scans: a CTA per node where a level has few nodes (the top, whose nodes hold
        // many tiles), a warp per node below, a thread per node where the nodes are small
        if (cnt <= 512)
            k_node_scan_cta<<<cnt, HT_NT, 0, s>>>(N, b, L, T->nleaf, tile_off.p, tcount.p, tbase.p, ccount.p, nkids.p);
        else if (cnt <= HT_WARP_SCAN_LEVEL)
            k_node_scan_warp<<<nblk(cnt, 256 / 32), 256, 0, s>>>(N, b, e, L, T->nleaf, tile_off.p, tcount.p, tbase.p,
                                                                ccount.p, nkids.p);
        else
            k_node_scan<<<nblk(cnt, 128), 128, 0, s>>>(N, b, e, L, T->nleaf, tile_off.p, tcount.p, tbase.p, ccount.p,
                                                      nkids.p);
        if (!excl_scan<int>(nkids.p, cnt, kid_off.p, s, stmp)) return false;
        int nnew = 0;
        if (!to_host(&nnew, kid_off.p + cnt, 1, s)) return false;
        PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(s), return false);
        if (!grow_nodes(T, (size_t)e + nnew, (size_t)e)) return false;
        N = bfs(T);
        // children are created (child[] = -1 for the rest) even when nothing splits
        k_children<<<nblk(cnt, 128), 128, 0, s>>>(N, b, e, L, T->nleaf, ccount.p, kid_off.p);
        if (nnew > 0) {
            PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(T->perm2.p, T->perm.p, (size_t)n * sizeof(int),
                                                    cudaMemcpyDeviceToDevice, s), return false);
            if (small)
                k_scatter_w<<<nblk(tgrid, HT_NT / 32), HT_NT, 0, s>>>(N, tile_node.p, tile_off.p, b, tile_off.p + cnt,
                                                                     tile, oct.p, tbase.p, T->perm.p, T->perm2.p);
            else
                k_scatter<<<tgrid, HT_NT, 0, s>>>(N, tile_node.p, tile_off.p, b, tile_off.p + cnt, tile, oct.p,
                                                 tbase.p, T->perm.p, T->perm2.p);
            std::swap(T->perm.p, T->perm2.p);
            std::swap(T->perm.n, T->perm2.n);
        }
        PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return false);
        lvl.push_back(e + nnew);
        if (nnew == 0) break;
    }
    const int nn = lvl.back();
    const int nlev = (int)lvl.size() - 1;
    T->nn = nn;
    Nodes N = bfs(T);

    // pre-order numbering: subtree sizes bottom-up, numbers top-down
    DevBuf<int>&size = T->size, &pre = T->pre;
    PGB_CUDA_OR(g_err, LIB, size.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, pre.reserve((size_t)nn), return false);
    for (int L = nlev - 1; L >= 0; L--)
        if (lvl[L + 1] > lvl[L]) k_subtree<<<nblk(lvl[L + 1] - lvl[L], 256), 256, 0, s>>>(N, lvl[L], lvl[L + 1], size.p);
    PGB_CUDA_OR(g_err, LIB, cudaMemsetAsync(pre.p, 0, sizeof(int), s), return false);
    for (int L = 0; L < nlev; L++)
        if (lvl[L + 1] > lvl[L]) k_preorder<<<nblk(lvl[L + 1] - lvl[L], 256), 256, 0, s>>>(N, lvl[L], lvl[L + 1], size.p, pre.p);
    PGB_CUDA_OR(g_err, LIB, T->first.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->count.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->child.reserve(8 * (size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->ppar.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->c.reserve(3 * (size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->half.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->com.reserve(3 * (size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->mass.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->quad.reserve(6 * (size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->sizep.reserve((size_t)nn), return false);
    Tree P{T->first.p, T->count.p, T->child.p, T->c.p, T->half.p, T->com.p, T->mass.p, T->quad.p};
    k_to_preorder<<<nblk(nn, 256), 256, 0, s>>>(N, nn, pre.p, P, size.p, T->sizep.p);

    // tree-order particles
    PGB_CUDA_OR(g_err, LIB, T->xt.reserve(3 * (size_t)n), return false);
    PGB_CUDA_OR(g_err, LIB, T->mt.reserve((size_t)n), return false);
    k_gather<<<nblk(n, 256), 256, 0, s>>>(n, T->perm.p, T->x.p, T->m.p, T->xt.p, T->mt.p);

    // moments, deepest level first: the pre-order indices of each level
    DevBuf<int>& lvl_pre = T->lvl_pre;
    PGB_CUDA_OR(g_err, LIB, lvl_pre.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(lvl_pre.p, pre.p, (size_t)nn * sizeof(int), cudaMemcpyDeviceToDevice, s),
                return false);
    for (int L = nlev - 1; L >= 0; L--) {
        const int cnt = lvl[L + 1] - lvl[L];
        if (cnt > 0) k_moments<<<nblk(cnt, 128), 128, 0, s>>>(P, lvl_pre.p + lvl[L], cnt, T->xt.p, T->mt.p);
    }

    // groups in pre-order
    k_parent_pre<<<nblk(nn, 256), 256, 0, s>>>(P, nn, T->ppar.p);
    DevBuf<int>&gflag = T->gflag, &goff = T->goff;
    PGB_CUDA_OR(g_err, LIB, gflag.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, goff.reserve((size_t)nn + 1), return false);
    k_group_flags<<<nblk(nn, 256), 256, 0, s>>>(P, T->ppar.p, nn, T->ncrit, gflag.p);
    if (!excl_scan<int>(gflag.p, nn, goff.p, s, stmp)) return false;
    int ng = 0;
    if (!to_host(&ng, goff.p + nn, 1, s)) return false;
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(s), return false);
    T->ng = ng;
    PGB_CUDA_OR(g_err, LIB, T->gnode.reserve((size_t)ng + 1), return false);
    k_compact<<<nblk(nn, 256), 256, 0, s>>>(gflag.p, goff.p, nn, T->gnode.p);

    // interaction lists: count, prefix sums, fill
    DevBuf<long long>&unp = T->unp, &unc = T->unc, &uoffp = T->uoffp, &uoffc = T->uoffc;
    const long long nu = (long long)ng * HT_UNITS;
    PGB_CUDA_OR(g_err, LIB, unp.reserve((size_t)nu + 1), return false);
    PGB_CUDA_OR(g_err, LIB, unc.reserve((size_t)nu + 1), return false);
    PGB_CUDA_OR(g_err, LIB, uoffp.reserve((size_t)nu + 1), return false);
    PGB_CUDA_OR(g_err, LIB, uoffc.reserve((size_t)nu + 1), return false);
    PGB_CUDA_OR(g_err, LIB, T->poff.reserve((size_t)ng + 1), return false);
    PGB_CUDA_OR(g_err, LIB, T->coff.reserve((size_t)ng + 1), return false);
    const double th2 = T->theta * T->theta;
    PGB_CUDA_OR(g_err, LIB, T->wn.reserve((size_t)nn * sizeof(WalkNode)), return false);
    WalkNode* wn = reinterpret_cast<WalkNode*>(T->wn.p);
    k_walk_nodes<<<nblk(nn, 256), 256, 0, s>>>(P, nn, T->nleaf, T->sizep.p, wn);
    k_list_count<<<nblk(nu, HT_WALK_NT), HT_WALK_NT, 0, s>>>(P, wn, T->gnode.p, ng, th2, unp.p, unc.p);
    if (!excl_scan<long long>(unp.p, nu, uoffp.p, s, ltmp)) return false;
    if (!excl_scan<long long>(unc.p, nu, uoffc.p, s, ltmp)) return false;
    k_group_offsets<<<nblk((long long)ng + 1, 256), 256, 0, s>>>(ng, uoffp.p, uoffc.p, T->poff.p, T->coff.p);
    long long tot[2] = {0, 0};
    if (!to_host(&tot[0], T->poff.p + ng, 1, s) || !to_host(&tot[1], T->coff.p + ng, 1, s)) return false;
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(s), return false);
    T->np = tot[0];
    T->nc = tot[1];
    PGB_CUDA_OR(g_err, LIB, T->pidx.reserve((size_t)std::max(1LL, T->np)), return false);
    PGB_CUDA_OR(g_err, LIB, T->cidx.reserve((size_t)std::max(1LL, T->nc)), return false);
    k_list_fill<<<nblk(nu, HT_WALK_NT), HT_WALK_NT, 0, s>>>(P, wn, T->gnode.p, ng, th2, uoffp.p, uoffc.p, T->pidx.p, T->cidx.p);
    // force-launch records
    PGB_CUDA_OR(g_err, LIB, T->part.reserve((size_t)n), return false);
    PGB_CUDA_OR(g_err, LIB, T->cell.reserve((size_t)nn), return false);
    PGB_CUDA_OR(g_err, LIB, T->cquad.reserve(2 * (size_t)nn), return false);
    k_records<<<nblk(std::max(n, nn), 256), 256, 0, s>>>(n, nn, T->xt.p, T->mt.p, P, T->part.p, T->cell.p, T->cquad.p);
    PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return false);
    PGB_CUDA_OR(g_err, LIB, cudaEventRecord(e1, s), return false);
    PGB_CUDA_OR(g_err, LIB, cudaEventSynchronize(e1), return false);
    cudaEventElapsedTime(&T->build_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return true;
}

void tree_free(pgbt_tree* T) {
    if (!T) return;
    if (T->s) cudaStreamSynchronize(T->s);
    DevBuf<double>* d[] = {&T->x, &T->m, &T->xt, &T->mt, &T->bc, &T->bhalf, &T->c, &T->half, &T->com, &T->mass, &T->quad};
    for (auto* b : d) b->release();
    DevBuf<int>* i[] = {&T->perm, &T->perm2, &T->bfirst, &T->bcount, &T->bparent, &T->bchild, &T->first, &T->count,
                        &T->child, &T->ppar, &T->gnode, &T->pidx, &T->cidx};
    for (auto* b : i) b->release();
    T->poff.release();
    T->coff.release();
    T->part.release();
    T->cell.release();
    T->cquad.release();
    for (auto& b : T->stmp) b.release();
    for (auto& b : T->ltmp) b.release();
    T->mx.release();
    DevBuf<int>* sc[] = {&T->ntile, &T->tile_off, &T->tile_node, &T->tcount, &T->tbase, &T->ccount, &T->nkids,
                         &T->kid_off, &T->size, &T->pre, &T->lvl_pre, &T->gflag, &T->goff, &T->sizep};
    for (auto* b : sc) b->release();
    T->oct.release();
    T->wn.release();
    T->gt_first.release();
    T->gt_count.release();
    T->gt_centre.release();
    T->gt_half.release();
    T->unp.release();
    T->unc.release();
    T->uoffp.release();
    T->uoffc.release();
    if (T->s) cudaStreamDestroy(T->s);
    delete T;
}
}  // namespace

// ---- C ABI (the host builder's bh_* accessors, drivers/pgb_bhtree.c, on device-built trees) --

PGB_EXPORT int pgbt_last_error(char* buf, int len) {
    std::lock_guard<std::mutex> g(g_err.mu);
    if (buf && len > 0) {
        std::strncpy(buf, g_err.msg.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return g_err.code;
}
PGB_EXPORT void pgbt_clear_error(void) {
    std::lock_guard<std::mutex> g(g_err.mu);
    g_err.code = 0;
    g_err.msg.clear();
}
PGB_EXPORT void pgbt_set_abort(int on) {
    std::lock_guard<std::mutex> g(g_err.mu);
    g_err.abort_on_error = on ? 1 : 0;
}

// Build the tree of n particles (x: n x 3, m: n, host arrays) and every group's interaction
// list on the GPU.  Returns NULL on bad arguments or failure (pgbt_last_error).
PGB_EXPORT pgbt_tree* pgbt_build(int n, const double* x, const double* m, double theta, int nleaf, int ncrit) {
    if (n <= 0 || !x || !m || nleaf < 1 || ncrit < 1 || !(theta > 0)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgbt_build: bad arguments (n %d, nleaf %d, ncrit %d, theta %g)", n, nleaf,
              ncrit, theta);
        return nullptr;
    }
    if (!ensure_device()) return nullptr;
    auto* T = new pgbt_tree();
    T->n = n;
    T->nleaf = nleaf;
    T->ncrit = ncrit;
    T->theta = theta;
    if (cudaStreamCreateWithFlags(&T->s, cudaStreamNonBlocking) != cudaSuccess) {
        raise(g_err, LIB, PGB_ERR_CUDA, "pgbt_build: stream creation failed");
        delete T;
        return nullptr;
    }
    if (!build(T, x, m)) {
        tree_free(T);
        return nullptr;
    }
    return T;
}

// Rebuild an existing tree for n new particles (same theta, nleaf, ncrit), reusing its device
// buffers: a code that builds a tree every step avoids the allocations of a fresh build.
// Returns PGB_OK, or an error code (the tree is then unusable: pgbt_free it).
PGB_EXPORT int pgbt_rebuild(pgbt_tree* T, int n, const double* x, const double* m) {
    if (!T || n <= 0 || !x || !m) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgbt_rebuild: bad arguments (n %d)", n);
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    T->n = n;
    return build(T, x, m) ? PGB_OK : PGB_ERR_CUDA;
}

PGB_EXPORT void pgbt_free(pgbt_tree* T) {
    if (g_device >= 0) cudaSetDevice(g_device);
    tree_free(T);
}

PGB_EXPORT int pgbt_n(const pgbt_tree* T) { return T ? T->n : 0; }
PGB_EXPORT int pgbt_ngroups(const pgbt_tree* T) { return T ? T->ng : 0; }
PGB_EXPORT int pgbt_nnodes(const pgbt_tree* T) { return T ? T->nn : 0; }
PGB_EXPORT long long pgbt_np(const pgbt_tree* T) { return T ? T->np : 0; }
PGB_EXPORT long long pgbt_nc(const pgbt_tree* T) { return T ? T->nc : 0; }
// device time of the build (ms, CUDA events from the first kernel to the records)
PGB_EXPORT float pgbt_build_ms(const pgbt_tree* T) { return T ? T->build_ms : 0.f; }

namespace {
template <class V>
int copy_out(pgbt_tree* T, V* dst, const V* src, size_t cnt) {
    if (!dst || !cnt) return PGB_OK;
    if (!ensure_device()) return PGB_ERR_NOGPU;
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(dst, src, cnt * sizeof(V), cudaMemcpyDeviceToHost, T->s), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(T->s), return PGB_ERR_CUDA);
    return PGB_OK;
}

// per group: one entry of a pre-order node field
__global__ void k_group_fields(Tree P, const int* gnode, int ng, int* first, int* count, double* centre, double* half) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    const int v = gnode[g];
    first[g] = P.first[v];
    count[g] = P.count[v];
    for (int a = 0; a < 3; a++) centre[3 * g + a] = P.c[3 * v + a];
    half[g] = P.half[v];
}
}  // namespace

// perm[n]: tree order -> input index
PGB_EXPORT int pgbt_perm(pgbt_tree* T, int* perm) { return T ? copy_out(T, perm, T->perm.p, (size_t)T->n) : PGB_ERR_ARG; }

// per group: first particle (tree order), count, cell centre (3), half side
PGB_EXPORT int pgbt_groups(pgbt_tree* T, int* first, int* count, double* centre, double* half) {
    if (!T) return PGB_ERR_ARG;
    if (!ensure_device()) return PGB_ERR_NOGPU;
    const int ng = T->ng;
    auto &f = T->gt_first, &c = T->gt_count;
    auto &ce = T->gt_centre, &h = T->gt_half;
    PGB_CUDA_OR(g_err, LIB, f.reserve((size_t)ng + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, c.reserve((size_t)ng + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, ce.reserve(3 * (size_t)ng + 3), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, h.reserve((size_t)ng + 1), return PGB_ERR_CUDA);
    Tree P{T->first.p, T->count.p, T->child.p, T->c.p, T->half.p, T->com.p, T->mass.p, T->quad.p};
    k_group_fields<<<nblk(ng, 256), 256, 0, T->s>>>(P, T->gnode.p, ng, f.p, c.p, ce.p, h.p);
    int rc = copy_out(T, first, f.p, (size_t)ng);
    if (!rc) rc = copy_out(T, count, c.p, (size_t)ng);
    if (!rc) rc = copy_out(T, centre, ce.p, 3 * (size_t)ng);
    if (!rc) rc = copy_out(T, half, h.p, (size_t)ng);
    return rc;
}

// per node: centre of mass (3), mass, quadrupole (6)
PGB_EXPORT int pgbt_cells(pgbt_tree* T, double* com, double* mass, double* quad) {
    if (!T) return PGB_ERR_ARG;
    int rc = copy_out(T, com, T->com.p, 3 * (size_t)T->nn);
    if (!rc) rc = copy_out(T, mass, T->mass.p, (size_t)T->nn);
    if (!rc) rc = copy_out(T, quad, T->quad.p, 6 * (size_t)T->nn);
    return rc;
}

// per node: particle range (tree order), half side, centre (3), children (8, -1 = empty)
PGB_EXPORT int pgbt_nodes(pgbt_tree* T, int* first, int* count, double* half, double* centre, int* child) {
    if (!T) return PGB_ERR_ARG;
    int rc = copy_out(T, first, T->first.p, (size_t)T->nn);
    if (!rc) rc = copy_out(T, count, T->count.p, (size_t)T->nn);
    if (!rc) rc = copy_out(T, half, T->half.p, (size_t)T->nn);
    if (!rc) rc = copy_out(T, centre, T->c.p, 3 * (size_t)T->nn);
    if (!rc) rc = copy_out(T, child, T->child.p, 8 * (size_t)T->nn);
    return rc;
}

// list offsets (ngroup + 1 each) and entries
PGB_EXPORT int pgbt_lists(pgbt_tree* T, long long* poff, int* pidx, long long* coff, int* cidx) {
    if (!T) return PGB_ERR_ARG;
    int rc = copy_out(T, poff, T->poff.p, (size_t)T->ng + 1);
    if (!rc) rc = copy_out(T, coff, T->coff.p, (size_t)T->ng + 1);
    if (!rc) rc = copy_out(T, pidx, T->pidx.p, (size_t)T->np);
    if (!rc) rc = copy_out(T, cidx, T->cidx.p, (size_t)T->nc);
    return rc;
}

namespace {
__global__ void k_irecords(int n, const double* xt, float eps2, float4* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        out[k] = make_float4((float)xt[3 * (size_t)k], (float)xt[3 * (size_t)k + 1], (float)xt[3 * (size_t)k + 2], eps2);
}
}  // namespace

// i-records of the batched force launch into the caller's device buffer out[n]: float4
// (x, y, z, eps2) in tree order, on the tree's stream (complete when the call returns).
PGB_EXPORT int pgbt_irecords(pgbt_tree* T, double eps2, void* out) {
    if (!T || !out) return PGB_ERR_ARG;
    if (!ensure_device()) return PGB_ERR_NOGPU;
    k_irecords<<<nblk(T->n, 256), 256, 0, T->s>>>(T->n, T->xt.p, (float)eps2, (float4*)out);
    PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(T->s), return PGB_ERR_CUDA);
    return PGB_OK;
}

// Host copies of the groups' particle ranges and list offsets only (first, count: ngroup;
// poff, coff: ngroup + 1; any pointer may be NULL): what a batched launch's work items need.
PGB_EXPORT int pgbt_group_table(pgbt_tree* T, int* first, int* count, long long* poff, long long* coff) {
    if (!T) return PGB_ERR_ARG;
    if (!ensure_device()) return PGB_ERR_NOGPU;
    const int ng = T->ng;
    auto &f = T->gt_first, &c = T->gt_count;
    auto &ce = T->gt_centre, &h = T->gt_half;
    PGB_CUDA_OR(g_err, LIB, f.reserve((size_t)ng + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, c.reserve((size_t)ng + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, ce.reserve(3 * (size_t)ng + 3), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, h.reserve((size_t)ng + 1), return PGB_ERR_CUDA);
    Tree P{T->first.p, T->count.p, T->child.p, T->c.p, T->half.p, T->com.p, T->mass.p, T->quad.p};
    k_group_fields<<<nblk(ng, 256), 256, 0, T->s>>>(P, T->gnode.p, ng, f.p, c.p, ce.p, h.p);
    int rc = copy_out(T, first, f.p, (size_t)ng);
    if (!rc) rc = copy_out(T, count, c.p, (size_t)ng);
    if (!rc) rc = copy_out(T, poff, T->poff.p, (size_t)ng + 1);
    if (!rc) rc = copy_out(T, coff, T->coff.p, (size_t)ng + 1);
    return rc;
}

// Host copies of the force-launch records (layouts as pgbt_device; any pointer may be NULL):
// part [n][4], cell [nnodes][4], cquad [nnodes][8] floats.
PGB_EXPORT int pgbt_records(pgbt_tree* T, float* part, float* cell, float* cquad) {
    if (!T) return PGB_ERR_ARG;
    int rc = copy_out(T, (float4*)part, T->part.p, (size_t)T->n);
    if (!rc) rc = copy_out(T, (float4*)cell, T->cell.p, (size_t)T->nn);
    if (!rc) rc = copy_out(T, (float4*)cquad, T->cquad.p, 2 * (size_t)T->nn);
    return rc;
}

// Device pointers for a batched force launch (valid until pgbt_free): particles float4
// (x, y, z, m) in tree order [n]; cells float4 (com, mass) [nnodes] and their quadrupoles,
// two float4 per cell (xx, xy, xz, yy) (yz, zz, 0, 0); the groups' list offsets (int64,
// ngroup + 1) and entries (int32: tree-order particle indices, pre-order cell indices).
PGB_EXPORT int pgbt_device(pgbt_tree* T, void** part, void** cell, void** cquad, void** poff, void** pidx, void** coff,
                           void** cidx) {
    if (!T) return PGB_ERR_ARG;
    if (part) *part = T->part.p;
    if (cell) *cell = T->cell.p;
    if (cquad) *cquad = T->cquad.p;
    if (poff) *poff = T->poff.p;
    if (pidx) *pidx = T->pidx.p;
    if (coff) *coff = T->coff.p;
    if (cidx) *cidx = T->cidx.p;
    return PGB_OK;
}
