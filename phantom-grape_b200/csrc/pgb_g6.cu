// pgb_g6.cu -- GRAPE-6 API of libpg6 on the B200 engine, plus the batched pgb6_* path.
//
// Drop-in for PG6/libpg6 (gp6util.h:1-101, phantom_g6.c, gravity.c).  Semantics kept:
//  * g6_set_j_particle stores (pos, vel, acc/2, jerk/6, mass, t, id) at address padr
//    (phantom_g6.c:118-125, gravity.c:95-115); the caller supplies acc/2 and jerk/6
//    (banana01.c:206-212).
//  * g6_set_ti sets the prediction time and a flag; the first g6calc_firsthalf after it
//    predicts all nj j-particles to t_i in FP64 (phantom_g6.c:138-164, gravity.c:149-193).
//  * g6calc_lasthalf* evaluate ni <= g6_npipes() i-particles against the nj predicted
//    j-particles, excluding the pair whose id equals the i id, and return
//    acc = sum m dx/r^3, jerk = sum m (dv/r^3 - 3 (dx.dv) dx/r^5), pot = -sum m/r
//    (the reference's -1/8 and 1/2 rescaling, phantom_g6.c:13-14, 200-208), nnb = id of the
//    nearest neighbour, rnnb = its softened distance (-2/key, gravity.c:651-657).
//  * lasthalfn / 2n / 2np also build neighbour lists (softened r <= h_i, gravity.c:788-793),
//    read back with g6_read_neighbour_list / g6_get_neighbour_list (phantom_g6.c:482-504),
//    lists in j-address order as the reference produces them.
//  * g6_set_tunit/xunit/reset/reset_fofpga/setup_njdata are no-ops, as in the reference.
// Deliberate differences:
//  * the self pair is excluded by an exact int id compare (the reference compares ids
//    converted to float, gravity.c:347-351: identical below 2^24 ids);
//  * pot is returned with FP64 precision (the reference stores it as float, avx_type.h:19);
//  * nearest-neighbour ties go to the smallest j address (the reference: lane j%4 first);
//  * a neighbour list longer than the capacity (1024, PGB_G6_NBMAX) is counted, flagged by
//    g6_read_neighbour_list and refused by g6_get_neighbour_list, never written out of bounds
//    (gravity.c:896-906 writes before it checks).
#include <atomic>
#include <chrono>

#include "pgb_g6_kernels.cuh"
#include "pgb_g6_small.cuh"
#include "pgb_hermite.cuh"

using namespace pgb;

namespace {

const char* LIB = "libpg6";
ErrorSlot g_err;

int env_int(const char* name, int dflt, int lo, int hi) {
    const char* s = std::getenv(name);
    if (!s || !*s) return dflt;
    int v = std::atoi(s);
    return v < lo ? lo : (v > hi ? hi : v);
}

int npipes() {
    static int v = env_int("PGB_G6_NPIPES", 48, 1, 1 << 20);
    return v;
}
int jmemsize() {
    static int v = env_int("PGB_G6_JMEMSIZE", 1 << 22, 1024, 1 << 26);
    return v;
}
// neighbour-list capacity per i-particle (the lists are sorted on the device in shared memory:
// at most 8192 entries)
int nbmax() {
    static int v = env_int("PGB_G6_NBMAX", 1024, 1, 1 << 13);
    return v;
}

std::mutex g_init_mu;
int g_device = -1;

bool ensure_device() {
    if (g_device >= 0) {
        PGB_CUDA_OR(g_err, LIB, cudaSetDevice(g_device), return false);
        return true;
    }
    std::lock_guard<std::mutex> g(g_init_mu);
    if (g_device < 0) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
            raise(g_err, LIB, PGB_ERR_NOGPU, "no CUDA device available");
            return false;
        }
        int d = env_int("PGB_DEVICE", 0, 0, n - 1);
        PGB_CUDA_OR(g_err, LIB, cudaSetDevice(d), return false);
        g_device = d;
    }
    PGB_CUDA_OR(g_err, LIB, cudaSetDevice(g_device), return false);
    return true;
}

// ------------------------------------------------------------------------------------------
// kernel configurations: (threads per CTA, i per thread, j-lanes); i-tile = NT/JL*IPT

enum Cfg {
    CFG_SMALL = 0, CFG_MED = 1, CFG_LARGE = 2, CFG_128x1 = 3, CFG_128x4 = 4, CFG_256x2 = 5,
    CFG_128x2J = 6, CFG_256x2J = 7, CFG_128x4J = 8, CFG_128x2JS = 9, NCFG = 10
};
constexpr int CFG_NT[NCFG] = {512, 256, 128, 128, 128, 256, 128, 256, 128, 128};
constexpr int CFG_IPT[NCFG] = {1, 1, 2, 1, 4, 2, 2, 2, 4, 2};
constexpr int CFG_JL[NCFG] = {8, 2, 1, 1, 1, 1, 1, 1, 1, 1};
// j-paired form (1: g6_jpair, 2: stage-ordered g6_jquad2): used with double-float positions and
// without neighbour lists; the other variants of these configurations run the i-paired form
constexpr int CFG_JP[NCFG] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 2};
inline int cfg_itile(int c) { return CFG_NT[c] / CFG_JL[c] * CFG_IPT[c]; }
constexpr int ITILE_MAX = 512;

template <int NT, int IPT, int JL, bool FF, int JP = 0>
int occ_of(bool nn, bool nbl) {
    static int v[4] = {0, 0, 0, 0};
    int k = (nn ? 1 : 0) + (nbl ? 2 : 0);
    if (!v[k]) {
        int b = 0;
        if (k == 0)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, g6_kernel<NT, IPT, JL, FF, false, false, JP>, NT, 0);
        if (k == 1)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, g6_kernel<NT, IPT, JL, FF, true, false, JP>, NT, 0);
        if (k == 2)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, g6_kernel<NT, IPT, JL, FF, false, true, JP>, NT, 0);
        if (k == 3)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, g6_kernel<NT, IPT, JL, FF, true, true, JP>, NT, 0);
        v[k] = b > 0 ? b : 1;
    }
    return v[k];
}

template <bool FF>
int occupancy_ff(int cfg, bool nn, bool nbl) {
    switch (cfg) {
        case CFG_SMALL: return occ_of<512, 1, 8, FF>(nn, nbl);
        case CFG_MED: return occ_of<256, 1, 2, FF>(nn, nbl);
        case CFG_128x1: return occ_of<128, 1, 1, FF>(nn, nbl);
        case CFG_128x4: return occ_of<128, 4, 1, FF>(nn, nbl);
        case CFG_256x2: return occ_of<256, 2, 1, FF>(nn, nbl);
        case CFG_128x2J: return occ_of<128, 2, 1, FF, 1>(nn, nbl);
        case CFG_256x2J: return occ_of<256, 2, 1, FF, 1>(nn, nbl);
        case CFG_128x4J: return occ_of<128, 4, 1, FF, 1>(nn, nbl);
        case CFG_128x2JS: return occ_of<128, 2, 1, FF, 2>(nn, nbl);
        default: return occ_of<128, 2, 1, FF>(nn, nbl);
    }
}

int occupancy(int cfg, bool ff, bool nn, bool nbl) {
    return ff ? occupancy_ff<true>(cfg, nn, nbl) : occupancy_ff<false>(cfg, nn, nbl);
}

template <int NT, int IPT, int JL, bool FF, int JP = 0>
void launch_cfg(bool nn, bool nbl, int grid, const G6Args& a, cudaStream_t s) {
    if (nn && nbl) g6_kernel<NT, IPT, JL, FF, true, true, JP><<<grid, NT, 0, s>>>(a);
    else if (nn) g6_kernel<NT, IPT, JL, FF, true, false, JP><<<grid, NT, 0, s>>>(a);
    else if (nbl) g6_kernel<NT, IPT, JL, FF, false, true, JP><<<grid, NT, 0, s>>>(a);
    else g6_kernel<NT, IPT, JL, FF, false, false, JP><<<grid, NT, 0, s>>>(a);
}

template <bool FF>
void launch_ff(int cfg, bool nn, bool nbl, int grid, const G6Args& a, cudaStream_t s) {
    switch (cfg) {
        case CFG_SMALL: launch_cfg<512, 1, 8, FF>(nn, nbl, grid, a, s); break;
        case CFG_MED: launch_cfg<256, 1, 2, FF>(nn, nbl, grid, a, s); break;
        case CFG_128x1: launch_cfg<128, 1, 1, FF>(nn, nbl, grid, a, s); break;
        case CFG_128x4: launch_cfg<128, 4, 1, FF>(nn, nbl, grid, a, s); break;
        case CFG_256x2: launch_cfg<256, 2, 1, FF>(nn, nbl, grid, a, s); break;
        case CFG_128x2J: launch_cfg<128, 2, 1, FF, 1>(nn, nbl, grid, a, s); break;
        case CFG_256x2J: launch_cfg<256, 2, 1, FF, 1>(nn, nbl, grid, a, s); break;
        case CFG_128x4J: launch_cfg<128, 4, 1, FF, 1>(nn, nbl, grid, a, s); break;
        case CFG_128x2JS: launch_cfg<128, 2, 1, FF, 2>(nn, nbl, grid, a, s); break;
        default: launch_cfg<128, 2, 1, FF>(nn, nbl, grid, a, s); break;
    }
}

cudaError_t launch_kernel(int cfg, bool ff, bool nn, bool nbl, int grid, const G6Args& a, cudaStream_t s) {
    if (ff) launch_ff<true>(cfg, nn, nbl, grid, a, s);
    else launch_ff<false>(cfg, nn, nbl, grid, a, s);
    return cudaGetLastError();
}

// Whether a force launch of this shape leaves nearest-neighbour lookups to g6_resolve_kernel:
// the tile-minimum search (two or four i per thread; one j-lane), split i-tiles (ngroups > 0),
// j addresses below the G6_NN_TILE mark (g6_task's `defer`).
bool needs_resolve(int cfg, bool nn, bool nbl, int ngroups, int jn) {
    return nn && !nbl && ngroups > 0 && CFG_IPT[cfg] % 2 == 0 && CFG_JL[cfg] == 1 && jn < G6_NN_TILE;
}

// The deferred nearest-neighbour lookups of a force launch (after it, on the same stream).
cudaError_t launch_resolve(int cfg, bool ff, bool nn, bool nbl, int ngroups, const G6Args& a, cudaStream_t s) {
    if (!needs_resolve(cfg, nn, nbl, ngroups, a.jn)) return cudaSuccess;
    constexpr int rpb = 128 / G6_RES_LANES;
    const long long grid = (long long)ngroups * ((a.itile + rpb - 1) / rpb);
    if (ff) g6_resolve_kernel<true><<<(unsigned)grid, 128, 0, s>>>(a, ngroups, CFG_NT[cfg]);
    else g6_resolve_kernel<false><<<(unsigned)grid, 128, 0, s>>>(a, ngroups, CFG_NT[cfg]);
    return cudaGetLastError();
}

// The small-call cluster kernel (pgb_g6_small.cuh): i-slots x j-lanes by the call's i count.
struct SmallShape {
    int isl, jl;
};
inline SmallShape small_shape(int ni) {
    if (ni <= 16) return {16, 32};
    if (ni <= 32) return {32, 16};
    if (ni <= 48) return {48, 10};
    return {64, 8};
}
// CTAs per cluster: 71 co-resident clusters of 4 (284 CTAs) leave 12 of the 148 SMs with one
// CTA, where the 33 clusters of 8 left 32 (the others, with two, set the call's time): the
// 48 x 65536 call 27.2 -> 26.6 us, 48 x 16384 23.0 -> 19.7 us
constexpr int SMALL_CL = 4;

template <int ISL, int JL, bool FF, bool NN, bool NBL>
cudaError_t small_launch(int grid, int cl, const G6SmallArgs& a, const G6IBlock& ib, cudaStream_t s,
                         int* max_clusters) {
    auto kern = g6_small_kernel<ISL, JL, FF, NN, NBL>;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(ISL * JL);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (max_clusters) return cudaOccupancyMaxActiveClusters(max_clusters, (void*)kern, &cfg);
    return cudaLaunchKernelEx(&cfg, kern, a, ib);
}

template <int ISL, int JL, bool FF>
cudaError_t small_launch_nn(bool nn, bool nbl, int grid, int cl, const G6SmallArgs& a,
                            const G6IBlock& ib, cudaStream_t s, int* mc) {
    if (nn && nbl) return small_launch<ISL, JL, FF, true, true>(grid, cl, a, ib, s, mc);
    if (nn) return small_launch<ISL, JL, FF, true, false>(grid, cl, a, ib, s, mc);
    if (nbl) return small_launch<ISL, JL, FF, false, true>(grid, cl, a, ib, s, mc);
    return small_launch<ISL, JL, FF, false, false>(grid, cl, a, ib, s, mc);
}

template <bool FF>
cudaError_t small_launch_ff(SmallShape sh, bool nn, bool nbl, int grid, int cl, const G6SmallArgs& a,
                            const G6IBlock& ib, cudaStream_t s, int* mc) {
    if (sh.isl == 16) return small_launch_nn<16, 32, FF>(nn, nbl, grid, cl, a, ib, s, mc);
    if (sh.isl == 32) return small_launch_nn<32, 16, FF>(nn, nbl, grid, cl, a, ib, s, mc);
    if (sh.isl == 48) return small_launch_nn<48, 10, FF>(nn, nbl, grid, cl, a, ib, s, mc);
    return small_launch_nn<64, 8, FF>(nn, nbl, grid, cl, a, ib, s, mc);
}

// Launch (mc == nullptr) or query the co-resident clusters of cl CTAs (into *mc).
cudaError_t small_kernel(SmallShape sh, bool ff, bool nn, bool nbl, int grid, int cl, const G6SmallArgs& a,
                         const G6IBlock& ib, cudaStream_t s, int* mc) {
    return ff ? small_launch_ff<true>(sh, nn, nbl, grid, cl, a, ib, s, mc)
              : small_launch_ff<false>(sh, nn, nbl, grid, cl, a, ib, s, mc);
}

// Chunks (= CTAs, all co-resident) and cluster size of a small call over nj j-records: at least
// 128 j per chunk, at most the co-resident clusters' CTAs (queried once per kernel variant).
void small_grid(SmallShape sh, bool ff, bool nn, bool nbl, int nj, int& grid, int& cl) {
    static int cache[4][2][2][2] = {};
    const int v = sh.isl / 16 - 1;
    int& mc = cache[v][ff][nn][nbl];
    if (!mc) {
        G6SmallArgs a{};
        G6IBlock ib{};
        int n = 0;
        if (small_kernel(sh, ff, nn, nbl, SMALL_CL, SMALL_CL, a, ib, nullptr, &n) != cudaSuccess || n < 1) {
            cudaGetLastError();
            n = sm_count(g_device) / SMALL_CL;
        }
        mc = n;
    }
    static const int forced = env_int("PGB_G6_SMALL_CTAS", 0, 0, 1 << 16);
    int by_j = nj / 128;
    int want = mc * SMALL_CL;
    if (forced) want = std::min(want, forced);
    want = std::min(want, by_j);
    if (want < 1) want = 1;
    cl = 1;
    while (cl < SMALL_CL && cl * 2 <= want) cl *= 2;
    grid = want / cl * cl;
}

// Relative-coordinate arithmetic of the library's own calls: double-float (default) or FP64
// subtraction + conversion (PGB_G6_DX=f64), see rel1() in pgb_g6_kernels.cuh.
bool dx_ff() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("PGB_G6_DX");
        v = (e && std::strcmp(e, "f64") == 0) ? 0 : 1;
    }
    return v == 1;
}

// Forced configuration for tuning sweeps (PGB_G6_CFG = 0..3), else by i count.
int pick_cfg(long long ni_max) {
    static int forced = env_int("PGB_G6_CFG", -1, -1, NCFG - 1);
    if (forced >= 0) return forced;
    if (ni_max <= 64) return CFG_SMALL;
    if (ni_max <= 4096) return CFG_MED;
    return CFG_LARGE;
}

// Plan one batch of items ([k][4] = i_off, i_cnt, j_off, j_cnt) for a configuration:
// about 4 tasks per resident CTA, chunks of at least 128 j, at most 512 chunks per i-tile
// (their partial rows are summed by the cooperative reduction of the group's last CTA).
long long plan_items(std::vector<Task>& tasks, std::vector<Group>& groups, int& rows, int nitem, const int* items,
                     int cfg, bool ff, bool nn, bool nbl, int nch_fixed = 0) {
    int slots = sm_count(g_device) * occupancy(cfg, ff, nn, nbl);
    int itile = cfg_itile(cfg);
    long long work = 0;
    for (int k = 0; k < nitem; k++) {
        long long ni = items[4 * k + 1];
        long long tiles = (ni + itile - 1) / itile;
        work += tiles * itile * (long long)items[4 * k + 3];
    }
    // about 4 tasks per resident CTA for load balance of uneven items; a single item (equal
    // tasks) or a small call (the drop-in API's npipes-sized calls) instead gets one wave of one
    // fat task per resident CTA, which keeps the number of partial rows (the reduction depth) low
    long long per_task = (cfg == CFG_SMALL || nitem == 1) ? work / slots + 1 : work / (4LL * slots) + 1;
    long long inter = 0;
    rows = 0;
    static const long long maxch = env_int("PGB_G6_MAXCHUNKS", 512, 1, 4096);
    for (int k = 0; k < nitem; k++) {
        int ni = items[4 * k + 1], nj = items[4 * k + 3];
        long long jc;
        if (nitem == 1) {
            // one item of equal tasks: the chunk count that minimises the wave quantisation, or
            // the autotuner's (nch_fixed)
            long long itiles = (ni + itile - 1) / itile;
            static const int forced_nch = env_int("PGB_G6_NCH", 0, 0, 4096);   // profiling: a pinned count
            int nch = forced_nch > 0 ? forced_nch : nch_fixed > 0 ? nch_fixed : best_nch(itiles, nj, slots, (int)maxch);
            jc = (nj + nch - 1) / nch;
        } else {
            jc = per_task / itile;
            if (jc < 128) jc = 128;
            if (jc * maxch < nj) jc = (nj + maxch - 1) / maxch;
        }
        if (jc > nj) jc = nj > 0 ? nj : 1;
        rows += plan_item(tasks, groups, items[4 * k], ni, items[4 * k + 2], nj, itile, (int)jc, rows);
        inter += (long long)ni * nj;
    }
    std::stable_sort(tasks.begin(), tasks.end(), [](const Task& a, const Task& b) {
        return (long long)a.ni * a.nj > (long long)b.ni * b.nj;
    });
    return inter;
}

// The chunk counts the autotuner tries for a single item besides the wave model's choice m:
// m x 3/4, 5/4, 3/2, and the counts whose chunks are whole 128-record j-tiles (nj / nch a
// multiple of 128) between m/2 and 2m.  Measured on the largest Hermite calls, the time moves
// by up to 5 % from one count to the next (the persistent CTAs' last wave; counts whose chunks
// are whole tiles were within 1 % of the best and never bimodal), which the model cannot predict.
std::vector<int> chunk_candidates(int m, int nj, int maxch) {
    std::vector<int> c;
    auto add = [&](long long v) {
        const long long hi = std::max<long long>(1, std::min<long long>(maxch, nj / 128));
        v = std::max<long long>(1, std::min<long long>(v, hi));
        if (std::find(c.begin(), c.end(), (int)v) == c.end()) c.push_back((int)v);
    };
    add(m);
    add((3LL * m + 2) / 4);
    add((5LL * m + 2) / 4);
    add((3LL * m + 1) / 2);
    for (long long n = std::max(1, m / 2); n <= 2LL * m; n++)
        if (nj % n == 0 && (nj / n) % 128 == 0) add(n);
    return c;
}

// ------------------------------------------------------------------------------------------
// library state (the reference keeps one global j-memory, gravity.c:31-47)

struct State {
    std::mutex mu;
    bool ready = false;
    cudaStream_t stream = nullptr;
    HostBuf<G6Ptcl> jh;
    DevBuf<G6Ptcl> jd;
    DevBuf<G6PredJ> pred;
    int jcap = 0, jdirty_lo = 1 << 30, jdirty_hi = 0;
    // sparse updates (a block step re-sends only its active particles): dirty addresses
    std::vector<int> dirty;
    std::vector<unsigned char> dirty_flag;
    bool all_dirty = true;
    HostBuf<G6Ptcl> sbuf;   // packed dirty records
    HostBuf<int> sidx;      // their addresses
    DevBuf<G6Ptcl> sbuf_d;
    DevBuf<int> sidx_d;
    double ti = 0.0;
    int predict_flag = 0;
    HostBuf<G6I> ibuf;
    HostBuf<G6Out> outh;    // mapped: the kernel writes the final results into it
    G6Out* outh_dev = nullptr;            // its device address (looked up once per allocation)
    const G6Out* outh_seen = nullptr;     // the allocation outh_dev belongs to
    DevBuf<int> pcnt;       // self-resetting counters of the parameter-block launches
    G6IBlock iblk;  // their i-records
    DevBuf<G6Out> spart;    // cluster rows of the small-call kernel
    HostBuf<unsigned> flags;  // mapped completion flags of the small-call kernel
    unsigned* flags_dev = nullptr;
    unsigned seq = 0;         // sequence number of the last flagged call
    int wait_flags = 0;       // flags the next wait_results() polls (0: synchronise the stream)
    Stager<G6I, G6Out> st;
    // neighbour lists of the last lasthalf*n call
    DevBuf<int> nbc_d, nbl_d;
    HostBuf<int> nbc_h, nbl_h;
    std::vector<std::vector<int>> nblists;
    std::vector<int> nbcounts;
    // device-time accounting of the drop-in calls (pgb6_set_call_timing): CUDA events around the
    // j-update + prediction of g6calc_firsthalf and the force launch of g6calc_lasthalf*
    bool time_calls = false;
    cudaEvent_t tev[2] = {nullptr, nullptr};
    double dev_ms = 0.0;
    int nb_ni = 0, nb_error = 0;
};
State S;

bool init_state() {
    if (!ensure_device()) return false;
    if (!S.ready) {
        PGB_CUDA_OR(g_err, LIB, cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking), return false);
        S.ready = true;
    }
    return true;
}

bool grow_j(int need) {
    if (need > jmemsize()) {
        raise(g_err, LIB, PGB_ERR_CAPACITY, "j-memory overflow: address %d >= jmemsize %d", need - 1, jmemsize());
        return false;
    }
    if (need <= S.jcap) return true;
    int cap = S.jcap ? S.jcap : 8192;
    while (cap < need) cap *= 2;
    if (cap > jmemsize()) cap = jmemsize();
    PGB_CUDA_OR(g_err, LIB, S.jh.reserve(cap, true), return false);
    std::memset((void*)(S.jh.p + S.jcap), 0, (size_t)(cap - S.jcap) * sizeof(G6Ptcl));
    S.dirty_flag.resize(cap, 0);
    S.all_dirty = true;  // new device buffer: upload everything
    S.jdirty_lo = 0;
    S.jdirty_hi = cap;
    S.jcap = cap;
    return true;
}

void mark_dirty(int padr) {
    if (padr < S.jdirty_lo) S.jdirty_lo = padr;
    if (padr + 1 > S.jdirty_hi) S.jdirty_hi = padr + 1;
    if (!S.all_dirty && !S.dirty_flag[padr]) {
        S.dirty_flag[padr] = 1;
        S.dirty.push_back(padr);
    }
}

// Upload the j-memory changes: the contiguous dirty range, or, when the changed records are
// sparse in it (a block step's active set), only those records plus a scatter on the device.
bool flush_j() {
    if (S.jdirty_hi <= S.jdirty_lo) return true;
    PGB_CUDA_OR(g_err, LIB, S.jd.reserve(S.jcap), return false);
    size_t lo = S.jdirty_lo, range = (size_t)(S.jdirty_hi - S.jdirty_lo), n = S.dirty.size();
    if (!S.all_dirty && n * 4 < range) {
        PGB_CUDA_OR(g_err, LIB, S.sbuf.reserve(n), return false);
        PGB_CUDA_OR(g_err, LIB, S.sidx.reserve(n), return false);
        PGB_CUDA_OR(g_err, LIB, S.sbuf_d.reserve(n), return false);
        PGB_CUDA_OR(g_err, LIB, S.sidx_d.reserve(n), return false);
        for (size_t k = 0; k < n; k++) {
            S.sbuf.p[k] = S.jh.p[S.dirty[k]];
            S.sidx.p[k] = S.dirty[k];
        }
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(S.sbuf_d.p, S.sbuf.p, n * sizeof(G6Ptcl), cudaMemcpyHostToDevice,
                                                S.stream), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(S.sidx_d.p, S.sidx.p, n * sizeof(int), cudaMemcpyHostToDevice,
                                                S.stream), return false);
        g6_scatter_kernel<<<(int)((n + 255) / 256), 256, 0, S.stream>>>(S.sbuf_d.p, S.sidx_d.p, (int)n, S.jcap,
                                                                         S.jd.p);
        PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return false);
    } else {
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(S.jd.p + lo, S.jh.p + lo, range * sizeof(G6Ptcl),
                                                cudaMemcpyHostToDevice, S.stream), return false);
    }
    for (int a : S.dirty) S.dirty_flag[a] = 0;
    S.dirty.clear();
    S.all_dirty = false;
    S.jdirty_lo = 1 << 30;
    S.jdirty_hi = 0;
    return true;
}

// Call timing: start / stop marks on the library's stream; stop adds the device time between
// them once the stop mark has completed.
bool time_mark(int k) {
    if (!S.time_calls) return true;
    if (!S.tev[k]) PGB_CUDA_OR(g_err, LIB, cudaEventCreate(&S.tev[k]), return false);
    PGB_CUDA_OR(g_err, LIB, cudaEventRecord(S.tev[k], S.stream), return false);
    return true;
}

bool time_add() {
    if (!S.time_calls) return true;
    float ms = 0.f;
    PGB_CUDA_OR(g_err, LIB, cudaEventSynchronize(S.tev[1]), return false);
    PGB_CUDA_OR(g_err, LIB, cudaEventElapsedTime(&ms, S.tev[0], S.tev[1]), return false);
    S.dev_ms += ms;
    return true;
}

bool flush_and_predict(int nj) {
    if (nj <= 0) return true;
    if (!grow_j(nj) || !time_mark(0) || !flush_j()) return false;
    PGB_CUDA_OR(g_err, LIB, S.pred.reserve(S.jcap), return false);
    g6_predict_kernel<<<(nj + 255) / 256, 256, 0, S.stream>>>(S.jd.p, nj, S.ti, S.pred.p, dx_ff());
    PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return false);
    if (!time_mark(1)) return false;
    // j-memory is read asynchronously from the pinned mirror: later set_j calls wait for it
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(S.stream), return false);
    return time_add();
}

// The small-call path: one launch of the cluster kernel (i-records in its parameter block),
// results into the mapped buffer; the call is one launch and one stream synchronisation.
bool run_small(int nj, int ni, float eps2, bool nn, bool nbl, G6Out* out_dev) {
    const bool ff = dx_ff();
    const SmallShape sh = small_shape(ni);
    int grid = 1, cl = 1;
    small_grid(sh, ff, nn, nbl, nj, grid, cl);
    PGB_CUDA_OR(g_err, LIB, S.spart.reserve((size_t)(grid / cl) * sh.isl), return false);
    if (!S.pcnt.p) {
        PGB_CUDA_OR(g_err, LIB, S.pcnt.reserve(SMALL_CL), return false);
        PGB_CUDA_OR(g_err, LIB, S.pcnt.zero_fill(S.stream), return false);
    }
    G6SmallArgs a;
    a.jpred = S.pred.p;
    a.eps2 = eps2;
    a.ni = ni;
    a.nj = nj;
    a.partial = S.spart.p;
    a.counter = S.pcnt.p;
    a.out = out_dev;
    a.nb_count = nullptr;
    a.nb_list = nullptr;
    a.nb_maxlen = nbmax();
    if (nbl) {
        PGB_CUDA_OR(g_err, LIB, S.nbc_d.reserve(ni), return false);
        PGB_CUDA_OR(g_err, LIB, S.nbl_d.reserve((size_t)ni * nbmax()), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemsetAsync(S.nbc_d.p, 0, (size_t)ni * sizeof(int), S.stream), return false);
        a.nb_count = S.nbc_d.p;
        a.nb_list = S.nbl_d.p;
    }
    // completion flags (mapped host memory, one per word slice of the final stage)
    a.done = nullptr;
    a.seq = 0;
    if (!nbl) {
        if (!S.flags.p) {
            PGB_CUDA_OR(g_err, LIB, S.flags.reserve(SMALL_CL, false, cudaHostAllocPortable | cudaHostAllocMapped),
                        return false);
            std::memset((void*)S.flags.p, 0, SMALL_CL * sizeof(unsigned));
            PGB_CUDA_OR(g_err, LIB, cudaHostGetDevicePointer((void**)&S.flags_dev, S.flags.p, 0), return false);
        }
        a.done = S.flags_dev;
        a.seq = ++S.seq;
        if (a.seq == 0) a.seq = ++S.seq;   // 0 is the flags' initial value
        S.wait_flags = cl;
    }
    std::memcpy(S.iblk.rec, S.ibuf.p, (size_t)ni * sizeof(G6I));
    PGB_CUDA_OR(g_err, LIB, small_kernel(sh, ff, nn, nbl, grid, cl, a, S.iblk, S.stream, nullptr), return false);
    return true;
}

// Wait for the results of the last call: by its completion flags when it has them (a bounded
// spin, then the stream synchronisation that reports a failed launch), else the stream.
bool wait_results() {
    if (S.wait_flags > 0) {
        const int n = S.wait_flags;
        S.wait_flags = 0;
        const unsigned seq = S.seq;
        volatile unsigned* f = S.flags.p;
        auto t0 = std::chrono::steady_clock::now();
        for (long it = 0;; it++) {
            bool all = true;
            for (int k = 0; k < n; k++) all = all && f[k] == seq;
            if (all) return true;
            if ((it & 1023) == 1023 && std::chrono::steady_clock::now() - t0 > std::chrono::seconds(5)) break;
        }
    }
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(S.stream), return false);
    return true;
}

// One drop-in API call: ni i-particles (in S.ibuf) against j-records [0, nj), results into
// the mapped pinned buffer S.outh (the kernel writes them there: no device-to-host copy).
// Up to G6_SMALL_MAXI i-particles (the reference's 48 pipes): the small-call cluster kernel, one
// launch.  More (PGB_G6_NPIPES > 64): the general kernel in regular mode -- it derives its i-tile
// x j-chunk tasks from the shape, so only the i-records are uploaded, and its task counter
// resets itself.
bool run_force(int nj, int ni, float eps2, bool nn, bool nbl) {
    PGB_CUDA_OR(g_err, LIB, S.outh.reserve(ni, false, cudaHostAllocPortable | cudaHostAllocMapped), return false);
    if (S.outh_seen != S.outh.p) {
        PGB_CUDA_OR(g_err, LIB, cudaHostGetDevicePointer((void**)&S.outh_dev, S.outh.p, 0), return false);
        S.outh_seen = S.outh.p;
    }
    G6Out* out_dev = S.outh_dev;
    if (ni <= G6_SMALL_MAXI && nj > 0) return run_small(nj, ni, eps2, nn, nbl, out_dev);
    const int cfg = pick_cfg(ni);
    const bool ff = dx_ff();
    const int itile = cfg_itile(cfg);
    const int slots = sm_count(g_device) * occupancy(cfg, ff, nn, nbl);
    static const int maxch = env_int("PGB_G6_MAXCHUNKS", 512, 1, 4096);
    const int itiles = (ni + itile - 1) / itile;
    int nch = best_nch(itiles, nj, slots, maxch);
    if (nch > nj) nch = nj > 0 ? nj : 1;
    const int rows = nch > 1 ? itiles * nch : 0;
    static const std::vector<Task> no_tasks;
    static const std::vector<Group> no_groups;
    PGB_CUDA_OR(g_err, LIB, S.st.stage(S.stream, no_tasks, no_groups, rows, ITILE_MAX, S.ibuf.p, ni, (size_t)itiles),
                return false);
    G6Args a;
    a.ipart = S.st.irecs();
    a.jpred = S.pred.p;
    a.eps2 = eps2;
    a.tasks = nullptr;
    a.ntasks = itiles * nch;
    a.task_counter = S.st.counter();
    a.groups = nullptr;
    a.group_counters = S.st.dgcnt.p;
    a.partial = S.st.dpart.p;
    a.out = out_dev;
    a.itile = itile;
    a.bundle_counters = S.st.bundle_counters();
    a.nb_count = nullptr;
    a.nb_list = nullptr;
    a.nb_maxlen = nbmax();
    a.reg_ni = ni;
    a.reg_nj = nj;
    a.reg_nch = nch;
    a.jn = nj;
    if (nbl) {
        PGB_CUDA_OR(g_err, LIB, S.nbc_d.reserve(ni), return false);
        PGB_CUDA_OR(g_err, LIB, S.nbl_d.reserve((size_t)ni * nbmax()), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemsetAsync(S.nbc_d.p, 0, (size_t)ni * sizeof(int), S.stream), return false);
        a.nb_count = S.nbc_d.p;
        a.nb_list = S.nbl_d.p;
    }
    if (a.ntasks == 0) return true;
    const int grid = a.ntasks < slots ? a.ntasks : slots;
    PGB_CUDA_OR(g_err, LIB, launch_kernel(cfg, ff, nn, nbl, grid, a, S.stream), return false);
    PGB_CUDA_OR(g_err, LIB, launch_resolve(cfg, ff, nn, nbl, nch > 1 ? itiles : 0, a, S.stream), return false);
    return true;
}

// Counts + lists back to the host; each list is sorted by j address (the reference's order,
// gravity.c:888-900) and mapped to particle ids.  Lists longer than the capacity keep only
// their count and set the overflow flag.
void nblist_collect(int ni) {
    S.nb_ni = ni;
    S.nb_error = 0;
    S.nbcounts.assign(ni, 0);
    S.nblists.assign(ni, {});
    // every list in j-address order, addresses replaced by ids, on the device
    int P = 1;
    while (P < nbmax()) P <<= 1;
    if (ni > 0) {
        g6_nb_sort_kernel<<<ni, 256, (size_t)P * sizeof(int), S.stream>>>(S.nbc_d.p, S.nbl_d.p, nbmax(), P, S.jd.p);
        PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return);
    }
    if (S.nbc_h.reserve(ni) != cudaSuccess || S.nbl_h.reserve((size_t)ni * nbmax()) != cudaSuccess) {
        raise(g_err, LIB, PGB_ERR_CUDA, "pinned neighbour-list buffer allocation failed");
        return;
    }
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(S.nbc_h.p, S.nbc_d.p, (size_t)ni * sizeof(int), cudaMemcpyDeviceToHost,
                                            S.stream), return);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(S.nbl_h.p, S.nbl_d.p, (size_t)ni * nbmax() * sizeof(int),
                                            cudaMemcpyDeviceToHost, S.stream), return);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(S.stream), return);
    for (int i = 0; i < ni; i++) {
        int c = S.nbc_h.p[i];
        S.nbcounts[i] = c;
        if (c > nbmax()) {
            S.nb_error = 1;
            continue;
        }
        // sorted by j address and mapped to ids on the device (g6_nb_sort_kernel)
        S.nblists[i].assign(S.nbl_h.p + (size_t)i * nbmax(), S.nbl_h.p + (size_t)i * nbmax() + c);
    }
}

// The common body of every g6calc_lasthalf* variant.
int lasthalf_impl(int nj, int ni, const int* pidx, const double (*pos)[3], const double (*vel)[3], double eps2,
                  const double* h2, double (*acc)[3], double (*jrk)[3], double* pot, int* nnb, float* rnnb,
                  bool nbl) {
    if (ni < 0 || ni > npipes()) {
        raise(g_err, LIB, PGB_ERR_ARG, "ni = %d outside [0, %d] pipes", ni, npipes());
        return 0;
    }
    if (nj < 0) {
        raise(g_err, LIB, PGB_ERR_ARG, "nj = %d is negative", nj);
        return 0;
    }
    if (ni == 0) return 0;
    std::lock_guard<std::mutex> g(S.mu);
    // checked under the lock: a concurrent g6_set_j_particle may grow the j store
    if (nj > S.jcap) {
        raise(g_err, LIB, PGB_ERR_ARG, "nj = %d but only %d j-particles were set", nj, S.jcap);
        return 0;
    }
    if (!init_state()) return 0;
    if (S.ibuf.reserve(ni) != cudaSuccess) {
        raise(g_err, LIB, PGB_ERR_CUDA, "pinned i-buffer allocation failed");
        return 0;
    }
    for (int i = 0; i < ni; i++) {
        G6I& r = S.ibuf.p[i];
        store_pos(r.p, pos[i][0], pos[i][1], pos[i][2], dx_ff());
        r.vx = (float)vel[i][0];
        r.vy = (float)vel[i][1];
        r.vz = (float)vel[i][2];
        r.id = pidx[i];
        r.h2 = (nbl && h2) ? (float)h2[i] : 0.f;
        r.pad = 0.f;
    }
    bool nn = (nnb != nullptr);
    // eps2 is a per-call scalar, used as float (phantom_g6.c:191)
    S.wait_flags = 0;
    if (!time_mark(0)) return 0;
    if (!run_force(nj, ni, (float)eps2, nn, nbl)) return 0;
    if (!time_mark(1)) return 0;
    if (!wait_results() || !time_add()) return 0;
    for (int i = 0; i < ni; i++) {
        const G6Out& o = S.outh.p[i];
        acc[i][0] = o.ax;
        acc[i][1] = o.ay;
        acc[i][2] = o.az;
        jrk[i][0] = o.jx;
        jrk[i][1] = o.jy;
        jrk[i][2] = o.jz;
        pot[i] = o.pot;
        if (nnb) nnb[i] = (o.jadr >= 0 && o.jadr < S.jcap) ? S.jh.p[o.jadr].idx : -1;
        if (rnnb) rnnb[i] = -2.0f / o.key;
    }
    if (nbl) nblist_collect(ni);
    return 0;
}

}  // namespace

// ============================================================================================
// GRAPE-6 API (PG6/libpg6/gp6util.h:1-101)

PGB_EXPORT void g6_open(int gpid) {
    (void)gpid;
    std::lock_guard<std::mutex> g(S.mu);
    init_state();
}
PGB_EXPORT void g6_close(int gpid) {
    (void)gpid;
    std::lock_guard<std::mutex> g(S.mu);
    if (!S.ready) return;
    cudaSetDevice(g_device);
    cudaStreamSynchronize(S.stream);
    S.jd.release();
    S.pred.release();
    S.st.release();
    S.pcnt.release();
    S.spart.release();
    S.wait_flags = 0;
    S.nbc_d.release();
    S.nbl_d.release();
    S.sbuf_d.release();
    S.sidx_d.release();
    for (int a : S.dirty) S.dirty_flag[a] = 0;
    S.dirty.clear();
    S.all_dirty = true;
    S.jdirty_lo = 0;
    S.jdirty_hi = S.jcap;
}
PGB_EXPORT void g6_set_tunit(int) {}
PGB_EXPORT void g6_set_xunit(int) {}
PGB_EXPORT void g6_reset(int) {}
PGB_EXPORT void g6_reset_fofpga(int) {}
PGB_EXPORT int g6_npipes(void) { return npipes(); }
PGB_EXPORT void g6_setup_njdata(int, int) {}

PGB_EXPORT void g6_set_j_particle(int gpid, int padr, int pidx, double t, double dt, double mss, double* snp,
                                  double* jrk, double* acc, double* vel, double* pos) {
    (void)gpid;
    (void)dt;
    (void)snp;
    if (padr < 0) {
        raise(g_err, LIB, PGB_ERR_ARG, "g6_set_j_particle: negative address %d", padr);
        return;
    }
    std::lock_guard<std::mutex> g(S.mu);
    if (!grow_j(padr + 1)) return;
    G6Ptcl& p = S.jh.p[padr];
    for (int d = 0; d < 3; d++) {
        p.pos[d] = pos[d];
        p.vel[d] = vel[d];
        p.acc2[d] = acc[d];
        p.jrk6[d] = jrk[d];
    }
    p.mass = mss;
    p.tim = t;
    p.idx = pidx;
    mark_dirty(padr);
}

PGB_EXPORT void g6_set_ti(int gpid, double time) {
    (void)gpid;
    std::lock_guard<std::mutex> g(S.mu);
    S.ti = time;
    S.predict_flag = 1;
}

PGB_EXPORT void g6calc_firsthalf(int gpid, int nj, int ni, int* pidx, double (*pos)[3], double (*vel)[3],
                                 double (*acc)[3], double (*jrk)[3], double* pot, double eps2, double* h2) {
    (void)gpid; (void)ni; (void)pidx; (void)pos; (void)vel; (void)acc; (void)jrk; (void)pot; (void)eps2; (void)h2;
    std::lock_guard<std::mutex> g(S.mu);
    if (!init_state()) return;
    if (S.predict_flag == 1) {
        if (!flush_and_predict(nj)) return;
        S.predict_flag = 0;
    }
    S.nb_error = 0;  // avx_initialize_neighbourlist (gravity.c:123-128)
}

#define LASTHALF_ARGS int gpid, int nj, int ni, int *pidx, double(*pos)[3], double(*vel)[3], double eps2, double *h2, \
                      double(*acc)[3], double(*jrk)[3], double *pot

PGB_EXPORT int g6calc_lasthalf(LASTHALF_ARGS) {
    (void)gpid;
    return lasthalf_impl(nj, ni, pidx, pos, vel, eps2, h2, acc, jrk, pot, nullptr, nullptr, false);
}
PGB_EXPORT int g6calc_lasthalf2(LASTHALF_ARGS, int* nnb) {
    (void)gpid;
    return lasthalf_impl(nj, ni, pidx, pos, vel, eps2, h2, acc, jrk, pot, nnb, nullptr, false);
}
PGB_EXPORT int g6calc_lasthalf2p(LASTHALF_ARGS, int* nnb, float* rnnb) {
    (void)gpid;
    return lasthalf_impl(nj, ni, pidx, pos, vel, eps2, h2, acc, jrk, pot, nnb, rnnb, false);
}
PGB_EXPORT int g6calc_lasthalfn(LASTHALF_ARGS) {
    (void)gpid;
    return lasthalf_impl(nj, ni, pidx, pos, vel, eps2, h2, acc, jrk, pot, nullptr, nullptr, true);
}
PGB_EXPORT int g6calc_lasthalf2n(LASTHALF_ARGS, int* nnb) {
    (void)gpid;
    return lasthalf_impl(nj, ni, pidx, pos, vel, eps2, h2, acc, jrk, pot, nnb, nullptr, true);
}
PGB_EXPORT int g6calc_lasthalf2np(LASTHALF_ARGS, int* nnb, float* rnnb) {
    (void)gpid;
    return lasthalf_impl(nj, ni, pidx, pos, vel, eps2, h2, acc, jrk, pot, nnb, rnnb, true);
}

// 0: success, 1: a list of the last lasthalf*n call overflowed (phantom_g6.c:482-486)
PGB_EXPORT int g6_read_neighbour_list(int gpid) {
    (void)gpid;
    return S.nb_error;
}

// 0: success, 1: nb > maxlen (phantom_g6.c:495-499, gravity.c:135-147)
PGB_EXPORT int g6_get_neighbour_list(int gpid, int ipipe, int maxlen, int* nblen, int* nbl) {
    (void)gpid;
    if (ipipe < 0 || ipipe >= S.nb_ni) {
        raise(g_err, LIB, PGB_ERR_ARG, "g6_get_neighbour_list: ipipe %d outside [0, %d)", ipipe, S.nb_ni);
        return 1;
    }
    if (S.nbcounts[ipipe] > maxlen || S.nbcounts[ipipe] > nbmax()) return 1;
    const std::vector<int>& v = S.nblists[ipipe];
    *nblen = (int)v.size();
    for (size_t k = 0; k < v.size(); k++) nbl[k] = v[k];
    return 0;
}

PGB_EXPORT void g6_debugfunc(int tmp) {
    FILE* fp = std::fopen("dump.dat", "a");
    if (!fp) return;
    std::fprintf(fp, "%d\n", tmp);
    std::fclose(fp);
}
PGB_EXPORT void g6_debugfunc_double(double tmp) {
    FILE* fp = std::fopen("dump.dat", "a");
    if (!fp) return;
    std::fprintf(fp, "%+e\n", tmp);
    std::fclose(fp);
}
PGB_EXPORT void g6_dump(double tim, int n, double* m, double (*x)[3], double (*v)[3]) {
    char out[64];
    std::snprintf(out, sizeof out, "dump.dat.%05d", (int)tim);
    FILE* fp = std::fopen(out, "w");
    if (!fp) return;
    for (int i = 0; i < n; i++) {
        std::fprintf(fp, "%+.16e", m[i]);
        std::fprintf(fp, " %+.16e %+.16e %+.16e", x[i][0], x[i][1], x[i][2]);
        std::fprintf(fp, " %+.16e %+.16e %+.16e", v[i][0], v[i][1], v[i][2]);
        std::fprintf(fp, "\n");
    }
    std::fclose(fp);
}

// Fortran twins (phantom_g6.c: every entry point has a `_` variant taking pointers)
PGB_EXPORT void g6_open_(int* gpid) { g6_open(*gpid); }
PGB_EXPORT void g6_close_(int* gpid) { g6_close(*gpid); }
PGB_EXPORT void g6_set_tunit_(int* v) { g6_set_tunit(*v); }
PGB_EXPORT void g6_set_xunit_(int* v) { g6_set_xunit(*v); }
PGB_EXPORT void g6_reset_(int* v) { g6_reset(*v); }
PGB_EXPORT void g6_reset_fofpga_(int* v) { g6_reset_fofpga(*v); }
PGB_EXPORT int g6_npipes_(void) { return g6_npipes(); }
PGB_EXPORT void g6_setup_njdata_(int* gpid, int* nj) { g6_setup_njdata(*gpid, *nj); }
PGB_EXPORT void g6_set_j_particle_(int* gpid, int* padr, int* pidx, double* t, double* dt, double* mss, double* snp,
                                   double* jrk, double* acc, double* vel, double* pos) {
    g6_set_j_particle(*gpid, *padr, *pidx, *t, *dt, *mss, snp, jrk, acc, vel, pos);
}
PGB_EXPORT void g6_set_ti_(int* gpid, double* t) { g6_set_ti(*gpid, *t); }
PGB_EXPORT void g6calc_firsthalf_(int* gpid, int* nj, int* ni, int* pidx, double (*pos)[3], double (*vel)[3],
                                  double (*acc)[3], double (*jrk)[3], double* pot, double* eps2, double* h2) {
    g6calc_firsthalf(*gpid, *nj, *ni, pidx, pos, vel, acc, jrk, pot, *eps2, h2);
}
#define LASTHALF_FARGS int *gpid, int *nj, int *ni, int *pidx, double(*pos)[3], double(*vel)[3], double *eps2, \
                       double *h2, double(*acc)[3], double(*jrk)[3], double *pot
#define LASTHALF_FCALL *gpid, *nj, *ni, pidx, pos, vel, *eps2, h2, acc, jrk, pot
PGB_EXPORT int g6calc_lasthalf_(LASTHALF_FARGS) { return g6calc_lasthalf(LASTHALF_FCALL); }
PGB_EXPORT int g6calc_lasthalf2_(LASTHALF_FARGS, int* nnb) { return g6calc_lasthalf2(LASTHALF_FCALL, nnb); }
PGB_EXPORT int g6calc_lasthalf2p_(LASTHALF_FARGS, int* nnb, float* rnnb) {
    return g6calc_lasthalf2p(LASTHALF_FCALL, nnb, rnnb);
}
PGB_EXPORT int g6calc_lasthalfn_(LASTHALF_FARGS) { return g6calc_lasthalfn(LASTHALF_FCALL); }
PGB_EXPORT int g6calc_lasthalf2n_(LASTHALF_FARGS, int* nnb) { return g6calc_lasthalf2n(LASTHALF_FCALL, nnb); }
PGB_EXPORT int g6calc_lasthalf2np_(LASTHALF_FARGS, int* nnb, float* rnnb) {
    return g6calc_lasthalf2np(LASTHALF_FCALL, nnb, rnnb);
}
PGB_EXPORT int g6_read_neighbour_list_(int* gpid) { return g6_read_neighbour_list(*gpid); }
PGB_EXPORT int g6_get_neighbour_list_(int* gpid, int* ipipe, int* maxlen, int* nblen, int* nbl) {
    return g6_get_neighbour_list(*gpid, *ipipe, *maxlen, nblen, nbl);
}
PGB_EXPORT void g6_debugfunc_(int* v) { g6_debugfunc(*v); }
PGB_EXPORT void g6_debugfunc_double_(double* v) { g6_debugfunc_double(*v); }
PGB_EXPORT void g6_dump_(double* tim, int* n, double* m, double (*x)[3], double (*v)[3]) { g6_dump(*tim, *n, m, x, v); }

// ============================================================================================
// Library status and the batched path (no reference counterpart; declared in include/pgb_g6.h)

PGB_EXPORT int pgb6_last_error(char* buf, int len) {
    std::lock_guard<std::mutex> g(g_err.mu);
    if (buf && len > 0) {
        std::strncpy(buf, g_err.msg.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return g_err.code;
}
PGB_EXPORT void pgb6_clear_error(void) {
    std::lock_guard<std::mutex> g(g_err.mu);
    g_err.code = 0;
    g_err.msg.clear();
}
PGB_EXPORT void pgb6_set_abort(int on) {
    std::lock_guard<std::mutex> g(g_err.mu);
    g_err.abort_on_error = on ? 1 : 0;
}

// Sizes of the device record types, so callers can lay out device buffers:
// G6Ptcl (j-memory), G6PredJ (predicted j), G6I (i-particle), G6Out (result).
// Device-time accounting of the drop-in calls (no counterpart in the reference): with on != 0,
// every g6calc_firsthalf (j-memory update + prediction) and g6calc_lasthalf* (force launch)
// adds the device time between CUDA events recorded around its work on the library's stream
// to a running total; pgb6_call_device_ms returns that total in ms (and clears it when reset
// != 0).  It separates the device work of the plain API from its host overhead.
PGB_EXPORT void pgb6_set_call_timing(int on) {
    std::lock_guard<std::mutex> g(S.mu);
    S.time_calls = on != 0;
}

PGB_EXPORT double pgb6_call_device_ms(int reset) {
    std::lock_guard<std::mutex> g(S.mu);
    const double v = S.dev_ms;
    if (reset) S.dev_ms = 0.0;
    return v;
}

PGB_EXPORT void pgb6_record_sizes(int* ptcl, int* predj, int* irec, int* out) {
    if (ptcl) *ptcl = (int)sizeof(G6Ptcl);
    if (predj) *predj = (int)sizeof(G6PredJ);
    if (irec) *irec = (int)sizeof(G6I);
    if (out) *out = (int)sizeof(G6Out);
}

namespace {
// Autotune cache: work-item-table shape -> best kernel configuration measured by
// pgb6_plan_tune.  The shape key buckets the item count, the largest i and j counts (powers of
// two) and the variant flags, so plans of the same shape reuse a measured choice.
std::mutex g_tune_mu;
struct Tuned {
    int cfg, nch;   // nch 0: the wave model's chunk count
};
std::vector<std::pair<long long, Tuned>> g_tune;

int ilog2up(long long v) {
    int k = 0;
    while ((1LL << k) < v && k < 62) k++;
    return k;
}

long long shape_key(int nitem, const int* items, bool ff, bool nn) {
    long long nimax = 0, njmax = 0;
    for (int k = 0; k < nitem; k++) {
        nimax = std::max<long long>(nimax, items[4 * k + 1]);
        njmax = std::max<long long>(njmax, items[4 * k + 3]);
    }
    return ((long long)ilog2up(nitem + 1) << 24) | ((long long)ilog2up(nimax + 1) << 16) |
           ((long long)ilog2up(njmax + 1) << 8) | (ff ? 2 : 0) | (nn ? 1 : 0);
}

Tuned tuned_cfg(long long key) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    for (auto& e : g_tune)
        if (e.first == key) return e.second;
    return Tuned{-1, 0};
}

void set_tuned(long long key, Tuned t) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    for (auto& e : g_tune)
        if (e.first == key) {
            e.second = t;
            return;
        }
    g_tune.emplace_back(key, t);
}
}  // namespace

// The largest j_offset + j_count of an item table ([k][4] = i_off, i_cnt, j_off, j_cnt).
int items_jend(int nitem, const int* items) {
    long long e = 0;
    for (int k = 0; k < nitem; k++) e = std::max<long long>(e, (long long)items[4 * k + 2] + items[4 * k + 3]);
    return (int)std::min<long long>(e, 0x7fffffff);
}

struct pgb6_plan {
    int cfg;
    bool nn;
    bool ff;
    std::vector<int> items;    // the work-item table, kept for re-planning (autotuning)
    int jend = 0;              // the items' largest j_offset + j_count (the j records they read)
    long long shape_key = 0;   // autotune cache key of this work-item table
    int nch = 0;               // a single item's chunk count (0: the wave model's, see plan_items)
    std::vector<Task> tasks;
    std::vector<Group> groups;
    int rows = 0;
    long long interactions = 0;
    Stager<G6I, G6Out> st;
    cudaEvent_t launched = nullptr;   // recorded after every stream (not graph-captured) launch
};

enum { PGB6_NN = 1, PGB6_POS_F64 = 2 };

// items: [nitem][4] = (i_offset, i_count, j_offset, j_count) into the i- and j-arrays.
// flags: PGB6_NN (1) also computes the nearest neighbour (key, j address); PGB6_POS_F64 (2):
// the i/j records hold FP64 positions (default: double-float positions, see Pos3).
PGB_EXPORT int pgb6_plan_create(pgb6_plan** out, int nitem, const int* items, int flags) {
    if (!out || nitem < 0 || (nitem && !items)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_plan_create: bad arguments");
        return PGB_ERR_ARG;
    }
    for (int k = 0; k < nitem; k++)
        if (items[4 * k] < 0 || items[4 * k + 1] < 0 || items[4 * k + 2] < 0 || items[4 * k + 3] < 0) {
            raise(g_err, LIB, PGB_ERR_ARG, "pgb6_plan_create: item %d has a negative offset or count", k);
            return PGB_ERR_ARG;
        }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    auto* P = new pgb6_plan();
    P->nn = (flags & PGB6_NN) != 0;
    P->ff = (flags & PGB6_POS_F64) == 0;
    long long nimax = 0;
    for (int k = 0; k < nitem; k++) nimax = std::max<long long>(nimax, items[4 * k + 1]);
    // many small items fill the GPU with short tiles; large ones prefer 2 i per thread
    long long total_i = 0;
    for (int k = 0; k < nitem; k++) total_i += items[4 * k + 1];
    P->items.assign(items, items + 4 * (size_t)nitem);
    P->jend = items_jend(nitem, items);
    P->shape_key = shape_key(nitem, items, P->ff, P->nn);
    const Tuned tuned = tuned_cfg(P->shape_key);
    P->cfg = tuned.cfg >= 0 ? tuned.cfg : pick_cfg(nitem > 1 ? std::max<long long>(nimax, total_i / 4) : nimax);
    P->nch = tuned.cfg >= 0 ? tuned.nch : 0;
    P->interactions = plan_items(P->tasks, P->groups, P->rows, nitem, items, P->cfg, P->ff, P->nn, false, P->nch);
    cudaStream_t s = nullptr;
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && P->st.stage(s, P->tasks, P->groups, P->rows, ITILE_MAX, (const G6I*)nullptr, 0) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (s) cudaStreamDestroy(s);
    if (!ok) {
        P->st.release();
        delete P;
        raise(g_err, LIB, PGB_ERR_CUDA, "pgb6_plan_create: staging failed");
        return PGB_ERR_CUDA;
    }
    *out = P;
    return PGB_OK;
}

PGB_EXPORT long long pgb6_plan_interactions(const pgb6_plan* P) { return P ? P->interactions : 0; }
PGB_EXPORT int pgb6_plan_tasks(const pgb6_plan* P) { return P ? (int)P->tasks.size() : 0; }
PGB_EXPORT int pgb6_plan_config(const pgb6_plan* P) { return P ? P->cfg : -1; }
// j-chunks per i-tile of a one-item plan (1: the j-range unsplit); 0 for plans of several items.
PGB_EXPORT int pgb6_plan_chunks(const pgb6_plan* P) {
    if (!P || P->items.size() != 4 || P->tasks.empty()) return 0;
    return P->groups.empty() ? 1 : (int)(P->tasks.size() / P->groups.size());
}
// Kernels one pgb6_plan_launch issues: the force kernel, and the nearest-neighbour lookups of
// split i-tiles when the plan's configuration defers them.
PGB_EXPORT int pgb6_plan_kernels(const pgb6_plan* P) {
    if (!P || P->tasks.empty()) return 0;
    return 1 + (needs_resolve(P->cfg, P->nn, false, (int)P->groups.size(), P->jend) ? 1 : 0);
}

// Device-resident launch (capturable in a CUDA graph): ipart = G6I[], jpred = G6PredJ[],
// out = G6Out[] indexed by absolute i (acc, jerk, pot final; key = -2/r_soft of the nearest
// neighbour, jadr = its j address, when the plan has PGB6_NN).
PGB_EXPORT int pgb6_plan_launch(pgb6_plan* P, const void* ipart, const void* jpred, double eps2, void* out,
                                void* stream) {
    if (!P || !ipart || !jpred || !out) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_plan_launch: null argument");
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    if (P->st.ntasks == 0) return PGB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    G6Args a;
    a.ipart = (const G6I*)ipart;
    a.jpred = (const G6PredJ*)jpred;
    a.eps2 = (float)eps2;
    a.tasks = P->st.tasks();
    a.ntasks = P->st.ntasks;
    a.task_counter = P->st.counter();
    a.groups = P->st.groups();
    a.group_counters = P->st.dgcnt.p;
    a.partial = P->st.dpart.p;
    a.out = (G6Out*)out;
    a.itile = cfg_itile(P->cfg);
    a.bundle_counters = P->st.bundle_counters();
    a.nb_count = nullptr;
    a.nb_list = nullptr;
    a.nb_maxlen = 0;
    a.jn = P->jend;
    int slots = sm_count(g_device) * occupancy(P->cfg, P->ff, P->nn, false);
    int grid = a.ntasks < slots ? a.ntasks : slots;
    PGB_CUDA_OR(g_err, LIB, launch_kernel(P->cfg, P->ff, P->nn, false, grid, a, s), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, launch_resolve(P->cfg, P->ff, P->nn, false, (int)P->groups.size(), a, s),
                return PGB_ERR_CUDA);
    // completion marker for pgb6_plan_update (none for a launch captured into a CUDA graph)
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PGB_CUDA_OR(g_err, LIB, cudaStreamIsCapturing(s, &cap), return PGB_ERR_CUDA);
    if (cap == cudaStreamCaptureStatusNone) {
        if (!P->launched)
            PGB_CUDA_OR(g_err, LIB, cudaEventCreateWithFlags(&P->launched, cudaEventDisableTiming),
                        return PGB_ERR_CUDA);
        PGB_CUDA_OR(g_err, LIB, cudaEventRecord(P->launched, s), return PGB_ERR_CUDA);
    }
    return PGB_OK;
}

// Pin one kernel configuration (0 .. NCFG-1) and re-plan for it (after the plan's previous
// stream launches have finished).
PGB_EXPORT int pgb6_plan_set_config(pgb6_plan* P, int cfg) {
    if (!P || cfg < 0 || cfg >= NCFG) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_plan_set_config: configuration %d outside [0, %d)", cfg, (int)NCFG);
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    P->cfg = cfg;
    P->nch = 0;
    const int nitem = (int)(P->items.size() / 4);
    P->tasks.clear();
    P->groups.clear();
    P->interactions = plan_items(P->tasks, P->groups, P->rows, nitem, P->items.data(), cfg, P->ff, P->nn, false);
    if (P->launched) PGB_CUDA_OR(g_err, LIB, cudaEventSynchronize(P->launched), return PGB_ERR_CUDA);
    cudaStream_t s = nullptr;
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && P->st.stage(s, P->tasks, P->groups, P->rows, ITILE_MAX, (const G6I*)nullptr, 0) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (s) cudaStreamDestroy(s);
    if (!ok) {
        raise(g_err, LIB, PGB_ERR_CUDA, "pgb6_plan_set_config: staging failed");
        return PGB_ERR_CUDA;
    }
    return PGB_OK;
}

// New items for an existing plan (same flags; its configuration kept), re-planned on the host
// and staged into the plan's own buffers, which grow only when needed: a code whose active sets
// or clusters change every step keeps one plan instead of creating and destroying one per step
// (no device allocation, hence no device-wide synchronisation, in its step).  Waits until the
// plan's previous stream launches have finished reading its task list.
PGB_EXPORT int pgb6_plan_update(pgb6_plan* P, int nitem, const int* items) {
    if (!P || nitem < 0 || (nitem && !items)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_plan_update: null plan or bad item count %d", nitem);
        return PGB_ERR_ARG;
    }
    for (int k = 0; k < nitem; k++)
        if (items[4 * k] < 0 || items[4 * k + 1] < 0 || items[4 * k + 2] < 0 || items[4 * k + 3] < 0) {
            raise(g_err, LIB, PGB_ERR_ARG, "pgb6_plan_update: item %d has a negative offset or count", k);
            return PGB_ERR_ARG;
        }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    P->items.assign(items, items + 4 * (size_t)nitem);
    P->jend = items_jend(nitem, items);
    P->shape_key = shape_key(nitem, items, P->ff, P->nn);
    const Tuned tuned = tuned_cfg(P->shape_key);
    P->nch = (tuned.cfg == P->cfg) ? tuned.nch : 0;
    P->tasks.clear();
    P->groups.clear();
    P->interactions = plan_items(P->tasks, P->groups, P->rows, nitem, items, P->cfg, P->ff, P->nn, false, P->nch);
    if (P->launched) PGB_CUDA_OR(g_err, LIB, cudaEventSynchronize(P->launched), return PGB_ERR_CUDA);
    cudaStream_t s = nullptr;
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && P->st.stage(s, P->tasks, P->groups, P->rows, ITILE_MAX, (const G6I*)nullptr, 0) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (s) cudaStreamDestroy(s);
    if (!ok) {
        raise(g_err, LIB, PGB_ERR_CUDA, "pgb6_plan_update: staging failed");
        return PGB_ERR_CUDA;
    }
    return PGB_OK;
}

// Autotuner: launches the plan with every kernel configuration (threads per CTA x i per
// thread x j-lanes) on the caller's data -- a plan of one item also with the chunk counts of
// chunk_candidates for its three fastest configurations -- keeps the fastest (CUDA-event time,
// the median of three launches after a warm-up launch, so that a shape whose time alternates
// between launches is judged by its usual time), re-stages the plan with it and records it for
// plans of the same shape.  Returns the chosen configuration index; *best_ms (optional)
// receives its launch time.  Overwrites `out`.  Not capturable (it synchronises the stream).
PGB_EXPORT int pgb6_plan_tune(pgb6_plan* P, const void* ipart, const void* jpred, double eps2, void* out,
                              void* stream, float* best_ms) {
    if (!P || !ipart || !jpred || !out) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_plan_tune: null argument");
        return -1;
    }
    if (!ensure_device()) return -1;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    PGB_CUDA_OR(g_err, LIB, cudaEventCreate(&e0), return -1);
    PGB_CUDA_OR(g_err, LIB, cudaEventCreate(&e1), return -1);
    const int nitem = (int)(P->items.size() / 4);
    // one (configuration, chunk count): the median of three timed launches after a warm-up
    auto time_plan = [&](int cfg, int nch, float* t) -> bool {
        P->tasks.clear();
        P->groups.clear();
        P->cfg = cfg;
        P->nch = nch;
        plan_items(P->tasks, P->groups, P->rows, nitem, P->items.data(), cfg, P->ff, P->nn, false, nch);
        if (P->st.stage(s, P->tasks, P->groups, P->rows, ITILE_MAX, (const G6I*)nullptr, 0) != cudaSuccess) return false;
        if (pgb6_plan_launch(P, ipart, jpred, eps2, out, stream) != PGB_OK) return false;
        float ts[3];
        for (int rep = 0; rep < 3; rep++) {
            cudaEventRecord(e0, s);
            if (pgb6_plan_launch(P, ipart, jpred, eps2, out, stream) != PGB_OK) return false;
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) return false;
            cudaEventElapsedTime(&ts[rep], e0, e1);
        }
        std::sort(ts, ts + 3);
        *t = ts[1];
        return true;
    };
    std::vector<std::pair<float, int>> by_cfg;
    for (int cfg = 0; cfg < NCFG; cfg++) {
        float t;
        if (!time_plan(cfg, 0, &t)) break;
        by_cfg.emplace_back(t, cfg);
    }
    std::sort(by_cfg.begin(), by_cfg.end());
    Tuned best{P->cfg, 0};
    float best_t = 1e30f;
    if (!by_cfg.empty()) {
        best = Tuned{by_cfg[0].second, 0};
        best_t = by_cfg[0].first;
    }
    if (nitem == 1 && P->items[1] > 0 && P->items[3] > 0) {
        static const int maxch = env_int("PGB_G6_MAXCHUNKS", 512, 1, 4096);
        const int ni = P->items[1], nj = P->items[3];
        for (size_t r = 0; r < by_cfg.size() && r < 3; r++) {
            const int cfg = by_cfg[r].second;
            const int itile = cfg_itile(cfg);
            const int slots = sm_count(g_device) * occupancy(cfg, P->ff, P->nn, false);
            const int m = best_nch((ni + itile - 1) / itile, nj, slots, maxch);
            for (int nch : chunk_candidates(m, nj, maxch)) {
                if (nch == m) continue;   // timed above
                float t;
                if (!time_plan(cfg, nch, &t)) break;
                if (t < best_t) {
                    best_t = t;
                    best = Tuned{cfg, nch};
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P->tasks.clear();
    P->groups.clear();
    P->cfg = best.cfg;
    P->nch = best.nch;
    plan_items(P->tasks, P->groups, P->rows, nitem, P->items.data(), best.cfg, P->ff, P->nn, false, best.nch);
    PGB_CUDA_OR(g_err, LIB, P->st.stage(s, P->tasks, P->groups, P->rows, ITILE_MAX, (const G6I*)nullptr, 0),
                return -1);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(s), return -1);
    set_tuned(P->shape_key, best);
    if (best_ms) *best_ms = best_t;
    return best.cfg;
}

PGB_EXPORT void pgb6_plan_destroy(pgb6_plan* P) {
    if (!P) return;
    if (g_device >= 0) cudaSetDevice(g_device);
    P->st.release();
    if (P->launched) cudaEventDestroy(P->launched);
    delete P;
}

// FP64 predictor on device records: pred[j] = predict(ptcl[j], ti) for j < nj.
// flags: PGB6_POS_F64 (2) writes FP64 positions, else the double-float layout.
PGB_EXPORT int pgb6_predict(const void* ptcl, int nj, double ti, void* pred, int flags, void* stream) {
    if (nj < 0 || (nj > 0 && (!ptcl || !pred))) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_predict: bad arguments");
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    if (nj == 0) return PGB_OK;
    g6_predict_kernel<<<(nj + 255) / 256, 256, 0, (cudaStream_t)stream>>>((const G6Ptcl*)ptcl, nj, ti, (G6PredJ*)pred,
                                                                           (flags & PGB6_POS_F64) == 0);
    PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return PGB_ERR_CUDA);
    return PGB_OK;
}

namespace {
struct HostBatch {
    std::mutex mu;
    cudaStream_t s = nullptr;
    HostBuf<G6I> ih;
    HostBuf<G6PredJ> jh;
    HostBuf<G6Out> oh;
    DevBuf<G6I> id;
    DevBuf<G6PredJ> jd;
    DevBuf<G6Out> od;
};
HostBatch HB;
}  // namespace

// Host-buffer batch: the whole list of items in one launch, inputs and outputs in host memory
// (copies included).  Positions FP64; velocities, masses rounded to float as the GRAPE-6 path
// does.  nnb / rnnb may be NULL.
PGB_EXPORT int pgb6_batch_host(int nitem, const int* items, int ni, const double (*xi)[3], const double (*vi)[3],
                               const int* idi, int nj, const double (*xj)[3], const double (*vj)[3], const double* mj,
                               const int* idj, double eps2, double (*acc)[3], double (*jrk)[3], double* pot, int* nnb,
                               float* rnnb) {
    if (ni < 0 || nj < 0) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_batch_host: negative sizes");
        return PGB_ERR_ARG;
    }
    for (int k = 0; k < nitem; k++) {
        const int* it = items + 4 * k;
        if (it[0] < 0 || it[1] < 0 || it[2] < 0 || it[3] < 0 || it[0] + it[1] > ni || it[2] + it[3] > nj) {
            raise(g_err, LIB, PGB_ERR_ARG, "pgb6_batch_host: item %d outside the arrays", k);
            return PGB_ERR_ARG;
        }
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    std::lock_guard<std::mutex> g(HB.mu);
    if (!HB.s) PGB_CUDA_OR(g_err, LIB, cudaStreamCreateWithFlags(&HB.s, cudaStreamNonBlocking), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, HB.ih.reserve(ni + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, HB.jh.reserve(nj + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, HB.oh.reserve(ni + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, HB.id.reserve(ni + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, HB.jd.reserve(nj + 1), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, HB.od.reserve(ni + 1), return PGB_ERR_CUDA);
    for (int i = 0; i < ni; i++) {
        G6I& r = HB.ih.p[i];
        store_pos(r.p, xi[i][0], xi[i][1], xi[i][2], dx_ff());
        r.vx = (float)vi[i][0]; r.vy = (float)vi[i][1]; r.vz = (float)vi[i][2];
        r.id = idi[i];
        r.h2 = 0.f;
        r.pad = 0.f;
    }
    for (int j = 0; j < nj; j++) {
        G6PredJ& r = HB.jh.p[j];
        store_pos(r.p, xj[j][0], xj[j][1], xj[j][2], dx_ff());
        r.vx = (float)vj[j][0]; r.vy = (float)vj[j][1]; r.vz = (float)vj[j][2];
        r.m = (float)mj[j];
        r.id = idj[j];
        r.pad = 0.f;
    }
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(HB.id.p, HB.ih.p, (size_t)ni * sizeof(G6I), cudaMemcpyHostToDevice, HB.s),
                return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(HB.jd.p, HB.jh.p, (size_t)nj * sizeof(G6PredJ), cudaMemcpyHostToDevice, HB.s),
                return PGB_ERR_CUDA);
    pgb6_plan* P = nullptr;
    int rc = pgb6_plan_create(&P, nitem, items, ((nnb || rnnb) ? PGB6_NN : 0) | (dx_ff() ? 0 : PGB6_POS_F64));
    if (rc) return rc;
    rc = pgb6_plan_launch(P, HB.id.p, HB.jd.p, eps2, HB.od.p, HB.s);
    if (!rc && ni > 0)
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(HB.oh.p, HB.od.p, (size_t)ni * sizeof(G6Out), cudaMemcpyDeviceToHost, HB.s),
                    rc = PGB_ERR_CUDA);
    if (!rc) PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(HB.s), rc = PGB_ERR_CUDA);
    pgb6_plan_destroy(P);
    if (rc) return rc;
    // outputs only for i covered by an item
    for (int k = 0; k < nitem; k++) {
        for (int i = items[4 * k]; i < items[4 * k] + items[4 * k + 1]; i++) {
            const G6Out& o = HB.oh.p[i];
            acc[i][0] = o.ax; acc[i][1] = o.ay; acc[i][2] = o.az;
            jrk[i][0] = o.jx; jrk[i][1] = o.jy; jrk[i][2] = o.jz;
            pot[i] = o.pot;
            if (nnb) nnb[i] = (o.jadr >= 0 && o.jadr < nj) ? idj[o.jadr] : -1;
            if (rnnb) rnnb[i] = -2.0f / o.key;
        }
    }
    return PGB_OK;
}

// ============================================================================================
// Allocation-free Hermite force call (no counterpart in the reference).
//
// For callers that must not allocate GPU memory: codes whose device memory is owned by their
// own pool allocator (a simulation that reserves most of HBM at start-up and hands libraries
// fixed buffers), and time-step loops that cannot afford the device-wide synchronisation a
// cudaMalloc / cudaFree may cause.  pgb6_force_noalloc runs the same force kernel as the
// plans, but its work list, group counters and partial sums live in one fixed array in the
// library's own static device memory (g6_noalloc_scratch below, 16 MiB, held on every GPU the
// library is loaded on until the process exits).  It never calls cudaMalloc or cudaFree.
//
// Set-up: the first call on a device looks up the array's device address there (this first
// call should come before any stream capture).  Every call shares the array and leaves its
// contents behind; each call clears the counters it needs first.  Calls whose launches overlap
// on the GPU (different streams, or different host threads) race on the array and corrupt
// each other's results: serialise them.

namespace {
constexpr size_t NOALLOC_BYTES = size_t(16) << 20;     // the whole scratch array
constexpr int NOALLOC_MAX_ITILES = 4096;                // i-tiles (one group counter each)
constexpr int NOALLOC_MAX_TASKS = 16384;
constexpr size_t NA_OFF_GCNT = 256;                                        // task counter first
constexpr size_t NA_OFF_TASKS = NA_OFF_GCNT + sizeof(int) * NOALLOC_MAX_ITILES;
constexpr size_t NA_OFF_GROUPS = NA_OFF_TASKS + sizeof(Task) * NOALLOC_MAX_TASKS;
constexpr size_t NA_OFF_PART = (NA_OFF_GROUPS + sizeof(Group) * NOALLOC_MAX_ITILES + 255) & ~size_t(255);
constexpr size_t NOALLOC_MAX_PART = (NOALLOC_BYTES - NA_OFF_PART) / sizeof(G6Out);
}  // namespace

static __device__ __align__(256) unsigned char g6_noalloc_scratch[NOALLOC_BYTES];

namespace {
std::mutex g_na_mu;
void* g_na_addr[64];  // device address of g6_noalloc_scratch per device (set-up once)

// Regular decomposition of one (ni x nj) item into itiles x nch tasks, written to the scratch
// work list (the layout the force kernel reads from a staged plan).
__global__ void g6_regular_tasks(Task* tasks, Group* groups, int ni, int nj, int itile, int itiles, int nch) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= itiles * nch) return;
    int it = t / nch, c = t % nch;
    int i0 = it * itile;
    int nii = min(itile, ni - i0);
    int j0 = (int)((long long)c * nj / nch), j1 = (int)((long long)(c + 1) * nj / nch);
    if (nch == 1) {
        tasks[t] = Task{i0, nii, 0, nj, -1, 0, -1, 0};
        return;
    }
    tasks[t] = Task{i0, nii, j0, j1 - j0, it, c, it * nch + c, 0};
    if (c == 0) groups[it] = Group{i0, nii, nch, it * nch};
}
}  // namespace

// One item: ni i-records (G6I) against nj predicted j-records (G6PredJ), results G6Out per i
// in out (device pointers, caller-owned).  flags: PGB6_NN, PGB6_POS_F64 as for plans.
// Limits: ni <= 4096 i-tiles (1,048,576 particles with the 256-particle tile that large calls
// use); larger ni is refused
// with PGB_ERR_CAPACITY.  Returns PGB_OK or an error code (message in pgb6_last_error).
PGB_EXPORT int pgb6_force_noalloc(const void* ipart, int ni, const void* jpred, int nj, double eps2, void* out,
                                  int flags, void* stream) {
    if (ni < 0 || nj < 0 || (ni > 0 && (!ipart || !out)) || (nj > 0 && !jpred)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_force_noalloc: bad arguments (ni %d, nj %d)", ni, nj);
        return PGB_ERR_ARG;
    }
    if (ni == 0) return PGB_OK;
    if (!ensure_device()) return PGB_ERR_NOGPU;
    const bool nn = (flags & PGB6_NN) != 0, ff = (flags & PGB6_POS_F64) == 0;
    const int cfg = pick_cfg(ni);
    const int itile = cfg_itile(cfg);
    const long long itiles = (ni + (long long)itile - 1) / itile;
    if (itiles > NOALLOC_MAX_ITILES) {
        raise(g_err, LIB, PGB_ERR_CAPACITY, "pgb6_force_noalloc: ni = %d exceeds the fixed scratch (%d i-tiles of %d)",
              ni, NOALLOC_MAX_ITILES, itile);
        return PGB_ERR_CAPACITY;
    }
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> g(g_na_mu);
        if (g_device < 0 || g_device >= 64) {
            raise(g_err, LIB, PGB_ERR_NOGPU, "pgb6_force_noalloc: device %d outside the supported range [0, 64)",
                  g_device);
            return PGB_ERR_NOGPU;
        }
        if (!g_na_addr[g_device]) {
            cudaError_t e = cudaGetSymbolAddress(&g_na_addr[g_device], g6_noalloc_scratch);
            if (e != cudaSuccess) {
                g_na_addr[g_device] = nullptr;
                raise(g_err, LIB, PGB_ERR_CUDA, "pgb6_force_noalloc: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(e));
                return PGB_ERR_CUDA;
            }
        }
        base = g_na_addr[g_device];
    }
    // j-chunks per i-tile: about 4 tasks per resident CTA, at least 128 j per chunk, within
    // the scratch's task and partial-row capacity
    const int slots = sm_count(g_device) * occupancy(cfg, ff, nn, false);
    long long nch = (4LL * slots + itiles - 1) / itiles;
    nch = std::min<long long>(nch, std::max<long long>(1, nj / 128));
    nch = std::min<long long>(nch, 512);
    nch = std::min<long long>(nch, NOALLOC_MAX_TASKS / itiles);
    nch = std::min<long long>(nch, (long long)(NOALLOC_MAX_PART / ((size_t)itiles * itile)));
    if (nch < 1) nch = 1;
    const int ntasks = (int)(itiles * nch);
    unsigned char* b = (unsigned char*)base;
    cudaStream_t s = (cudaStream_t)stream;
    // the task counter and the group counters must start at zero
    PGB_CUDA_OR(g_err, LIB, cudaMemsetAsync(b, 0, NA_OFF_TASKS, s), return PGB_ERR_CUDA);
    g6_regular_tasks<<<(ntasks + 255) / 256, 256, 0, s>>>((Task*)(b + NA_OFF_TASKS), (Group*)(b + NA_OFF_GROUPS), ni,
                                                          nj, itile, (int)itiles, (int)nch);
    PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return PGB_ERR_CUDA);
    G6Args a;
    a.ipart = (const G6I*)ipart;
    a.jpred = (const G6PredJ*)jpred;
    a.eps2 = (float)eps2;
    a.tasks = (const Task*)(b + NA_OFF_TASKS);
    a.ntasks = ntasks;
    a.task_counter = (int*)b;
    a.groups = (const Group*)(b + NA_OFF_GROUPS);
    a.group_counters = (int*)(b + NA_OFF_GCNT);
    a.partial = (G6Out*)(b + NA_OFF_PART);
    a.out = (G6Out*)out;
    a.itile = itile;
    a.nb_count = nullptr;
    a.nb_list = nullptr;
    a.nb_maxlen = 0;
    a.jn = nj;
    int grid = ntasks < slots ? ntasks : slots;
    PGB_CUDA_OR(g_err, LIB, launch_kernel(cfg, ff, nn, false, grid, a, s), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, launch_resolve(cfg, ff, nn, false, nch > 1 ? (int)itiles : 0, a, s), return PGB_ERR_CUDA);
    return PGB_OK;
}

// ------------------------------------------------------------------------------------------
// Hermite block-time-step integrator on the device (pgb_hermite.cuh): the reference's sample
// integrator PG6/banana (hermite.c, timestep.c; banana01.c:96-183 main loop) with the particle
// state, the j-memory and the per-step bookkeeping resident in HBM.  One cooperative launch
// runs block steps until the global time reaches the caller's tend: the host launches once per
// call and reads the clock back.

struct pgb6_hermite {
    std::mutex mu;
    int n = 0, nseg = 0, grid = 0;
    double eps2 = 0.0, eta = 0.0, eta_s = 0.0, dtmax = 0.0;
    bool ff = true;
    cudaStream_t s = nullptr;
    DevBuf<double> state;          // t, dt, pot, mass [n]; pos, vel, acc, jrk [n][3]
    DevBuf<unsigned char> work;    // HmWork's arrays
    HmState P{};
    HmWork W{};
    double* energy = nullptr;      // [2] device
    HmClock clk{};                 // the device clock as of the last synchronisation
};

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Co-resident CTAs of the persistent kernel (its cooperative grid).
int hm_grid(bool ff) {
    static int cache[2] = {0, 0};
    int& g = cache[ff ? 1 : 0];
    if (!g) {
        int per = 0;
        cudaError_t e = ff ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, hm_run_kernel<true>, HM_NT, 0)
                           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, hm_run_kernel<false>, HM_NT, 0);
        if (e != cudaSuccess || per < 1) per = 1;
        g = per * sm_count(g_device);
    }
    return g;
}

bool hm_alloc(pgb6_hermite* H) {
    const size_t n = (size_t)H->n;
    PGB_CUDA_OR(g_err, LIB, H->state.reserve(16 * n), return false);
    double* b = H->state.p;
    H->P.n = H->n;
    H->P.t = b;
    H->P.dt = b + n;
    H->P.pot = b + 2 * n;
    H->P.mass = b + 3 * n;
    H->P.pos = b + 4 * n;
    H->P.vel = b + 7 * n;
    H->P.acc = b + 10 * n;
    H->P.jrk = b + 13 * n;
    H->nseg = (int)((n + HM_SEG - 1) / HM_SEG);
    H->grid = hm_grid(H->ff);
    // partial rows: at most (grid + i-tiles) rows of at most 512 entries; force tasks: at most
    // grid + i-tiles of at least 16
    const long long part_cap = (long long)H->grid * 512 + (long long)n + 512;
    const int task_cap = H->grid + (int)(n / 16) + 2;
    size_t off = 0;
    const size_t o_hdr = off;
    off = align256(off + sizeof(HmClock));
    const size_t o_sync = off;
    off = align256(off + sizeof(HmSync) + sizeof(unsigned) * (size_t)H->grid * HM_ARRIVE_STRIDE);
    const size_t o_gmin = off;
    off = align256(off + 3 * sizeof(unsigned long long));
    const size_t o_bmin = off;
    off = align256(off + sizeof(unsigned long long) * 2 * H->nseg);
    const size_t o_bcnt = off;
    off = align256(off + sizeof(int) * 2 * H->nseg);
    const size_t o_sflag = off;
    off = align256(off + sizeof(unsigned) * H->nseg);
    const size_t o_tflag = off;
    off = align256(off + sizeof(unsigned) * (size_t)task_cap);
    const size_t o_act = off;
    off = align256(off + sizeof(int) * n);
    const size_t o_irec = off;
    off = align256(off + sizeof(G6I) * n);
    const size_t o_jpred = off;
    off = align256(off + sizeof(G6PredJ) * n);
    const size_t o_out = off;
    off = align256(off + sizeof(G6Out) * n);
    const size_t o_part = off;
    off = align256(off + sizeof(G6Out) * (size_t)part_cap);
    const size_t o_en = off;
    off = align256(off + 2 * sizeof(double));
    PGB_CUDA_OR(g_err, LIB, H->work.reserve(off), return false);
    unsigned char* w = H->work.p;
    H->W.clk = (HmClock*)(w + o_hdr);
    H->W.sync = (HmSync*)(w + o_sync);
    H->W.gmin = (unsigned long long*)(w + o_gmin);
    H->W.bmin = (unsigned long long*)(w + o_bmin);
    H->W.bcnt = (int*)(w + o_bcnt);
    H->W.seg_flag = (unsigned*)(w + o_sflag);
    H->W.task_flag = (unsigned*)(w + o_tflag);
    H->W.task_cap = task_cap;
    H->W.active = (int*)(w + o_act);
    H->W.irec = (G6I*)(w + o_irec);
    H->W.jpred = (G6PredJ*)(w + o_jpred);
    H->W.out = (G6Out*)(w + o_out);
    H->W.partial = (G6Out*)(w + o_part);
    H->W.part_cap = part_cap;
    H->energy = (double*)(w + o_en);
    // clock, barrier and flags zero; the step numbers that tag the flags start at 1
    PGB_CUDA_OR(g_err, LIB, cudaMemsetAsync(w, 0, o_act, H->s), return false);
    const unsigned first_step = 1;
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(&H->W.sync->step, &first_step, sizeof first_step, cudaMemcpyHostToDevice,
                                            H->s), return false);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(H->s), return false);
    return true;
}

// Wait for the stream and read the device clock; a barrier that gave up is an error.
bool hm_sync_clock(pgb6_hermite* H) {
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(&H->clk, H->W.clk, sizeof(HmClock), cudaMemcpyDeviceToHost, H->s),
                return false);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(H->s), return false);
    if (H->clk.err) {
        raise(g_err, LIB, PGB_ERR_DEVICE, "hermite: a grid barrier of the step kernel timed out");
        return false;
    }
    return true;
}

// One cooperative launch: the start-up step, or block steps while the time is below tend (at
// most max_steps).
bool hm_launch(pgb6_hermite* H, bool startup, double tend, int max_steps) {
    HmRun R;
    R.P = H->P;
    R.W = H->W;
    R.eps2 = (float)H->eps2;
    R.eta = H->eta;
    R.eta_s = H->eta_s;
    R.dtmax = H->dtmax;
    R.tend = tend;
    R.startup = startup ? 1 : 0;
    R.max_steps = max_steps;
    R.nseg = H->nseg;
    // j per force chunk at least (fewer, longer tasks mean fewer partial rows for the owners
    // to sum; N = 16384 block steps: 64 -> 114, 128 -> 120, 256 -> 123, 512 -> 108 Gint/s)
    static const int minj = env_int("PGB_HM_MINJ", 256, 16, 1 << 20);
    R.minj = minj;
    void* args[] = {&R};
    const void* fn = H->ff ? (const void*)hm_run_kernel<true> : (const void*)hm_run_kernel<false>;
    PGB_CUDA_OR(g_err, LIB, cudaLaunchCooperativeKernel(fn, dim3(H->grid), dim3(HM_NT), args, 0, H->s),
                return false);
    return true;
}

void hm_free(pgb6_hermite* H) {
    if (H->s) cudaStreamSynchronize(H->s);
    H->state.release();
    H->work.release();
    if (H->s) cudaStreamDestroy(H->s);
    H->s = nullptr;
}

constexpr int HM_STEPS_PER_LAUNCH = 1 << 16;
}  // namespace

// Create an integrator for n particles (n >= 2) and take its start-up step: every particle's
// force, jerk and potential at t = 0 and its first step (startup_sgmotion).  eps2: softening^2;
// eta / eta_s: accuracy parameters of dt_criterion / dt_startup; dtmax: the largest step and the
// interval after which the times restart from 0 (the reference's dtstar).
PGB_EXPORT int pgb6_hermite_create(pgb6_hermite** out, int n, const double* mass, const double (*pos)[3],
                                   const double (*vel)[3], double eps2, double eta, double eta_s, double dtmax) {
    if (!out || n < 2 || n > HM_MAXSEG * HM_SEG || !mass || !pos || !vel || !(eps2 >= 0.0) || !(eta > 0.0) ||
        !(eta_s > 0.0) || !(dtmax > 0.0)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_create: bad arguments (n %d, eps2 %g, eta %g, eta_s %g, dtmax %g)",
              n, eps2, eta, eta_s, dtmax);
        return PGB_ERR_ARG;
    }
    *out = nullptr;
    if (!ensure_device()) return PGB_ERR_NOGPU;
    auto* H = new pgb6_hermite();
    H->n = n;
    H->eps2 = eps2;
    H->eta = eta;
    H->eta_s = eta_s;
    H->dtmax = dtmax;
    H->ff = dx_ff();
    bool ok = cudaStreamCreateWithFlags(&H->s, cudaStreamNonBlocking) == cudaSuccess;
    if (!ok) raise(g_err, LIB, PGB_ERR_CUDA, "pgb6_hermite_create: stream creation failed");
    ok = ok && hm_alloc(H);
    if (ok) {
        const size_t nn = (size_t)n;
        // t, dt, pot zero; acc, jrk zero; mass, pos, vel from the caller
        ok = cudaMemsetAsync(H->state.p, 0, 16 * nn * sizeof(double), H->s) == cudaSuccess &&
             cudaMemcpyAsync(H->P.mass, mass, nn * sizeof(double), cudaMemcpyHostToDevice, H->s) == cudaSuccess &&
             cudaMemcpyAsync(H->P.pos, pos, 3 * nn * sizeof(double), cudaMemcpyHostToDevice, H->s) == cudaSuccess &&
             cudaMemcpyAsync(H->P.vel, vel, 3 * nn * sizeof(double), cudaMemcpyHostToDevice, H->s) == cudaSuccess;
        if (!ok) raise(g_err, LIB, PGB_ERR_CUDA, "pgb6_hermite_create: upload failed");
    }
    ok = ok && hm_launch(H, true, 0.0, 1) && hm_sync_clock(H);
    const int bad = ok ? H->clk.bad : 0;
    if (ok && bad) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_create: the start-up step of %d particles is below dtmax/2^51",
              bad);
        hm_free(H);
        delete H;
        return PGB_ERR_ARG;
    }
    if (!ok) {
        hm_free(H);
        delete H;
        return PGB_ERR_CUDA;
    }
    *out = H;
    return PGB_OK;
}

// One block step: the particles with the smallest t + dt advance to it.  *time (optional): the
// global time after the step; *ni (optional): the number of particles advanced.
PGB_EXPORT int pgb6_hermite_step(pgb6_hermite* H, double* time, int* ni) {
    if (!H) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_step: null integrator");
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    std::lock_guard<std::mutex> g(H->mu);
    if (!hm_launch(H, false, INFINITY, 1) || !hm_sync_clock(H)) return H->clk.err ? PGB_ERR_DEVICE : PGB_ERR_CUDA;
    if (time) *time = H->clk.time;
    if (ni) *ni = H->clk.ni;
    return PGB_OK;
}

// Block steps while the global time is below tend (banana01.c:146 loop condition, evaluated on
// the device before every step).  *psteps / *bsteps (optional): the particle steps and block
// steps this call took.
PGB_EXPORT int pgb6_hermite_advance(pgb6_hermite* H, double tend, long long* psteps, long long* bsteps) {
    if (!H) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_advance: null integrator");
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    std::lock_guard<std::mutex> g(H->mu);
    const long long p0 = H->clk.psteps, b0 = H->clk.bsteps;
    while (H->clk.time < tend)
        if (!hm_launch(H, false, tend, HM_STEPS_PER_LAUNCH) || !hm_sync_clock(H))
            return H->clk.err ? PGB_ERR_DEVICE : PGB_ERR_CUDA;
    if (psteps) *psteps = H->clk.psteps - p0;
    if (bsteps) *bsteps = H->clk.bsteps - b0;
    return PGB_OK;
}

PGB_EXPORT double pgb6_hermite_time(pgb6_hermite* H) { return H ? H->clk.time : 0.0; }

// The limit, in SM cycles, of every wait of the step kernel (grid barriers, segment and task
// flags); cycles <= 0 restores the default (about a second).  A wait that runs out sets the
// integrator's error word: every CTA returns at its next wait, the call reports PGB_ERR_DEVICE
// and the integrator is unusable afterwards (its barrier state is no longer consistent).  For
// fault-handling tests; a production run keeps the default.
PGB_EXPORT int pgb6_hermite_set_wait_limit(pgb6_hermite* H, long long cycles) {
    if (!H) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_set_wait_limit: null integrator");
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    std::lock_guard<std::mutex> g(H->mu);
    const long long v = cycles > 0 ? cycles : 0;
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(&H->W.clk->spin_limit, &v, sizeof v, cudaMemcpyHostToDevice, H->s),
                return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(H->s), return PGB_ERR_CUDA);
    return PGB_OK;
}

// The step kernel's failure record, read from the device: *gave_up (a wait ran out, so the
// integrator is unusable), *exits (CTAs that have returned from the kernel, over every launch
// so far) and *grid (CTAs per launch).  Any pointer may be NULL.
PGB_EXPORT int pgb6_hermite_wait_status(pgb6_hermite* H, int* gave_up, int* exits, int* grid) {
    if (!H) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_wait_status: null integrator");
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    std::lock_guard<std::mutex> g(H->mu);
    HmClock c;
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(&c, H->W.clk, sizeof c, cudaMemcpyDeviceToHost, H->s),
                return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(H->s), return PGB_ERR_CUDA);
    if (gave_up) *gave_up = c.err;
    if (exits) *exits = c.exits;
    if (grid) *grid = H->grid;
    return PGB_OK;
}

// The particle state (any pointer may be NULL): t, dt, pos, vel, acc, jerk, pot as the
// reference's struct Particle holds them (jerk and pot with float values).
PGB_EXPORT int pgb6_hermite_get(pgb6_hermite* H, double* t, double* dt, double (*pos)[3], double (*vel)[3],
                                double (*acc)[3], double (*jrk)[3], double* pot) {
    if (!H) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_get: null integrator");
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    std::lock_guard<std::mutex> g(H->mu);
    const size_t n = (size_t)H->n;
    struct {
        void* dst;
        const double* src;
        size_t cnt;
    } cp[7] = {{t, H->P.t, n},           {dt, H->P.dt, n},          {pos, H->P.pos, 3 * n}, {vel, H->P.vel, 3 * n},
               {acc, H->P.acc, 3 * n},   {jrk, H->P.jrk, 3 * n},    {pot, H->P.pot, n}};
    for (auto& c : cp)
        if (c.dst)
            PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(c.dst, c.src, c.cnt * sizeof(double), cudaMemcpyDeviceToHost, H->s),
                        return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(H->s), return PGB_ERR_CUDA);
    return PGB_OK;
}

// The last block step's active particles (index order) and the force, jerk and potential the
// force phase returned for them (before the corrector's rounding of jerk and pot to float).
// Returns the number of active particles, or a negative error code.
PGB_EXPORT int pgb6_hermite_last_step(pgb6_hermite* H, int* active, double (*acc)[3], double (*jrk)[3],
                                      double* pot) {
    if (!H) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_last_step: null integrator");
        return -PGB_ERR_ARG;
    }
    if (!ensure_device()) return -PGB_ERR_NOGPU;
    std::lock_guard<std::mutex> g(H->mu);
    const int ni = H->clk.ni;
    std::vector<G6Out> o((size_t)ni);
    if (active)
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(active, H->W.active, ni * sizeof(int), cudaMemcpyDeviceToHost, H->s),
                    return -PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(o.data(), H->W.out, ni * sizeof(G6Out), cudaMemcpyDeviceToHost, H->s),
                return -PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(H->s), return -PGB_ERR_CUDA);
    for (int k = 0; k < ni; k++) {
        if (acc) {
            acc[k][0] = o[k].ax;
            acc[k][1] = o[k].ay;
            acc[k][2] = o[k].az;
        }
        if (jrk) {
            jrk[k][0] = o[k].jx;
            jrk[k][1] = o[k].jy;
            jrk[k][2] = o[k].jz;
        }
        if (pot) pot[k] = o[k].pot;
    }
    return ni;
}

// Kinetic and potential energy of the current state (calc_energy.c:9-33), FP64, fixed order.
PGB_EXPORT int pgb6_hermite_energy(pgb6_hermite* H, double* ek, double* ew) {
    if (!H) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb6_hermite_energy: null integrator");
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    std::lock_guard<std::mutex> g(H->mu);
    double e[2] = {0.0, 0.0};
    hm_energy_kernel<<<1, 1024, 0, H->s>>>(H->P, H->energy);
    PGB_CUDA_OR(g_err, LIB, cudaGetLastError(), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(e, H->energy, sizeof e, cudaMemcpyDeviceToHost, H->s), return PGB_ERR_CUDA);
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(H->s), return PGB_ERR_CUDA);
    if (ek) *ek = e[0];
    if (ew) *ew = e[1];
    return PGB_OK;
}

// Particle and block steps since creation (the start-up step counts n and 1).
PGB_EXPORT void pgb6_hermite_counts(pgb6_hermite* H, long long* psteps, long long* bsteps) {
    if (psteps) *psteps = H ? H->clk.psteps : 0;
    if (bsteps) *bsteps = H ? H->clk.bsteps : 0;
}

// The integrator's CUDA stream (for callers that time it with CUDA events or order their own
// work after it).
PGB_EXPORT void* pgb6_hermite_stream(pgb6_hermite* H) { return H ? (void*)H->s : nullptr; }

// Pair interactions of the force phases so far (active particles x n) and the steps taken with
// each force decomposition (i-tile 16, 32, 64, 128, 512); any pointer may be NULL.
PGB_EXPORT void pgb6_hermite_stats(pgb6_hermite* H, long long* pairs, long long* steps_by_tile) {
    if (pairs) *pairs = H ? H->clk.force_pairs : 0;
    for (int k = 0; k < 5; k++)
        if (steps_by_tile) steps_by_tile[k] = H ? H->clk.variant_steps[k] : 0;
}

PGB_EXPORT void pgb6_hermite_destroy(pgb6_hermite* H) {
    if (!H) return;
    if (g_device >= 0) cudaSetDevice(g_device);
    hm_free(H);
    delete H;
}
