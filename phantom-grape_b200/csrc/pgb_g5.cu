// pgb_g5.cu -- GRAPE-5 API (newton) and the newton_quad g5c_* API on the B200 engine.
//
// Drop-in for PG5/newton/libpg5 (gp5util.h:10-39, phantom_g5.c, pg5_fortran.c) and
// PG5/newton_quad/quad (quad_util.h:8-15, quad_g5c.c).  Built twice:
//   libpg5.so     plain softening   (g5_set_xmj(adr, nj, xj, mj))
//   libpg5sym.so  -DPGB_SYMMETRIC   (g5_set_xmj(adr, nj, xj, mj, epsj2), GravityKernel0)
//
// Semantics kept from the reference:
//  * set_* calls convert double -> float immediately (phantom_g5.c:100-205); j-records are
//    addressed absolutely (xj[adr..adr+nj) is read, as phantom_g5.c:193 does).
//  * g5_set_xi uses eps^2 = (float)(Eps*Eps) from g5_set_eps_to_all (phantom_g5.c:107);
//    g5_set_xei takes eps^2 per particle (phantom_g5.c:126).
//  * g5_get_force returns acc = sum m dx/r^3 and pot = +sum m/r (self pair included), the sign
//    the reference returns after Pot_correct (phantom_g5.c:251-259).  The reference's rsqrt
//    bias factors (1-3 bias, 1-bias) are NOT applied: they only undo the 12-bit rsqrt's mean
//    error, and the MUFU rsqrt (with or without the Newton step) has none to undo.
//  * g5c_* (quad_g5c.c:198-303) share the i-pipes of g5_set_xiMC and the output path of
//    g5_get_forceMC, so the quadrupole potential comes back as -sum(phi_p + phi_q) while the
//    monopole one comes back positive; callers reconcile this (source.cpp:854, 866).
// Deliberate differences:
//  * g5_calculate_force_on_x[e][MC] evaluate all ni in one launch instead of ni/4 calls.
//  * set_xmj does not write the zero padding at [nj, nj + (4 - nj%4)%4) (phantom_g5.c:199-204):
//    the kernels loop over exactly n j-records, and that padding can overwrite real records
//    when adr > 0.  set_xmjMC with an odd nj does not read xj[adr+nj] (quad_g5c.c:206-259,
//    phantom_g5.c:148-166 read one record past the end).
//  * j-memory capacity is 1 Mi records (PGB_G5_JMEMSIZE), not 64 Ki; exceeding it is an error,
//    not an out-of-bounds write.
#include "pgb_g5_kernels.cuh"

using namespace pgb;

namespace {

#if defined(PGB_TABLE)
const char* LIB = "libpg5table";
constexpr int PARTICLE_KIND = G5_TABLE;
#elif defined(PGB_SYMMETRIC)
const char* LIB = "libpg5sym";
constexpr int PARTICLE_KIND = G5_SYMMETRIC;
#else
const char* LIB = "libpg5";
constexpr int PARTICLE_KIND = G5_NEWTON;
#endif

ErrorSlot g_err;

constexpr int MAXDEV = 64;
// Kernel configurations: threads per CTA x i-particles per thread.  Large CTAs win on large
// single items (fewer, longer tasks), small i-tiles on batches of small groups (tree-code
// groups average well below their size limit: an i-tile much larger than the group idles
// most of its threads); the table
// kind keeps its force table in static shared memory (CTAs of <= 256 threads) and the quad
// kind stages three words per cell (<= 512 threads).  Plans pick one with pgb5_plan_tune.
// G5C_*J: the j-paired form (newton point masses and quadrupole cells only;
// pgb_g5_kernels.cuh g5_newton_jpair / g5_quad_jpair).
enum G5Cfg {
    G5C_128x4 = 0, G5C_256x2 = 1, G5C_512x2 = 2, G5C_1024x1 = 3, G5C_384x2 = 4, G5C_128x2 = 5, G5C_128x1 = 6,
    G5C_64x1 = 7, G5C_64x1J = 8, G5C_1024x1J = 9, G5C_256x1J = 10, G5_NCFG = 11
};
constexpr int G5C_NT[G5_NCFG] = {128, 256, 512, 1024, 384, 128, 128, 64, 64, 1024, 256};
constexpr int G5C_IPT[G5_NCFG] = {4, 2, 2, 1, 2, 2, 1, 1, 1, 1, 1};
inline bool cfg_jp(int c) { return c >= G5C_64x1J; }
constexpr int ITILE_MAX = 1024;
inline int cfg_itile(int c) { return G5C_NT[c] * G5C_IPT[c]; }
template <int KIND, int NT>
constexpr bool kind_fits() {
    return KIND == G5_TABLE ? NT <= 256 : (KIND == G5_QUAD ? NT <= 512 : true);
}
inline bool cfg_valid(int kind, int c) {
    if (cfg_jp(c)) return (kind == G5_NEWTON || kind == G5_QUAD) && (kind != G5_QUAD || G5C_NT[c] <= 512);
    return kind == G5_TABLE ? G5C_NT[c] <= 256 : (kind == G5_QUAD ? G5C_NT[c] <= 512 : true);
}
constexpr int MAXPIPE = 4096;

int env_int(const char* name, int dflt, int lo, int hi) {
    const char* s = std::getenv(name);
    if (!s || !*s) return dflt;
    int v = std::atoi(s);
    return v < lo ? lo : (v > hi ? hi : v);
}

int npipes() {
    static int v = env_int("PGB_G5_NPIPES", 4, 1, MAXPIPE);
    return v;
}
int jmemsize() {
    static int v = env_int("PGB_G5_JMEMSIZE", 1 << 20, 1024, 1 << 26);
    return v;
}

std::mutex g_init_mu;
int g_device = -1;
double g_eps = 0.0;  // phantom_g5.c:17, shared by all devids

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

// Launch (occ == nullptr) or query the resident CTAs per SM (into *occ) of one kernel.
template <int KIND, int NT, int IPT, bool JP = false>
cudaError_t launch_k(int grid, const G5Args& a, cudaStream_t s, int* occ) {
    if constexpr (!kind_fits<KIND, NT>() || (JP && KIND != G5_NEWTON && KIND != G5_QUAD)) {
        return cudaErrorInvalidConfiguration;
    } else {
        // the table kind's table lives in dynamic shared memory (a.tbl_size entries)
        const size_t dyn = (KIND == G5_TABLE) ? (size_t)a.tbl_size * sizeof(float2) : 0;
        if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, g5_kernel<KIND, NT, IPT, JP>, NT, dyn);
        g5_kernel<KIND, NT, IPT, JP><<<grid, NT, dyn, s>>>(a);
        return cudaGetLastError();
    }
}

template <int KIND>
cudaError_t launch_cfg(int cfg, int grid, const G5Args& a, cudaStream_t s, int* occ) {
    switch (cfg) {
        case G5C_256x2: return launch_k<KIND, 256, 2>(grid, a, s, occ);
        case G5C_512x2: return launch_k<KIND, 512, 2>(grid, a, s, occ);
        case G5C_1024x1: return launch_k<KIND, 1024, 1>(grid, a, s, occ);
        case G5C_384x2: return launch_k<KIND, 384, 2>(grid, a, s, occ);
        case G5C_128x2: return launch_k<KIND, 128, 2>(grid, a, s, occ);
        case G5C_128x1: return launch_k<KIND, 128, 1>(grid, a, s, occ);
        case G5C_64x1: return launch_k<KIND, 64, 1>(grid, a, s, occ);
        case G5C_64x1J: return launch_k<KIND, 64, 1, true>(grid, a, s, occ);
        case G5C_1024x1J: return launch_k<KIND, 1024, 1, true>(grid, a, s, occ);
        case G5C_256x1J: return launch_k<KIND, 256, 1, true>(grid, a, s, occ);
        default: return launch_k<KIND, 128, 4>(grid, a, s, occ);
    }
}

// The kinds each library serves: the table library the table kind, the others the particle
// kind of their build plus the quadrupole cells.
cudaError_t launch_kind(int kind, int cfg, int grid, const G5Args& a, cudaStream_t s, int* occ = nullptr) {
#ifdef PGB_TABLE
    (void)kind;
    return launch_cfg<G5_TABLE>(cfg, grid, a, s, occ);
#else
    if (kind == G5_QUAD) return launch_cfg<G5_QUAD>(cfg, grid, a, s, occ);
    return launch_cfg<PARTICLE_KIND>(cfg, grid, a, s, occ);
#endif
}

int table_entries();   // the table kind's current table size (0 in the other libraries)

// Resident CTAs per SM of a configuration (the table kind's depends on its table size).
int occupancy_of(int kind, int cfg) {
    static int cache[4][G5_NCFG] = {};
    static int cache_tbl[4][G5_NCFG] = {};
    const int tbl = (kind == G5_TABLE) ? table_entries() : 0;
    int& v = cache[kind & 3][cfg];
    if (!v || cache_tbl[kind & 3][cfg] != tbl) {
        int b = 0;
        G5Args a{};
        a.tbl_size = tbl;
        if (launch_kind(kind, cfg, 0, a, nullptr, &b) != cudaSuccess || b < 1) {
            cudaGetLastError();
            b = 1;
        }
        v = b;
        cache_tbl[kind & 3][cfg] = tbl;
    }
    return v;
}

// Default configuration of a call or plan whose largest item has ni i-particles (and
// PGB_G5_CFG forces one for sweeps): big CTAs for big items, 256-particle tiles for groups.
int pick_cfg(int kind, long long ni_max) {
    static int forced = env_int("PGB_G5_CFG", -1, -1, G5_NCFG - 1);
    if (forced >= 0 && cfg_valid(kind, forced)) return forced;
    if (kind == G5_TABLE || kind == G5_QUAD) return ni_max <= 256 ? G5C_128x2 : G5C_256x2;
    if (ni_max <= 256) return G5C_128x2;
    if (ni_max <= 2048) return G5C_256x2;
    return G5C_1024x1;
}

// Chunk length for one item: its tasks are all the same size, so one wave of tasks (one per
// resident CTA) balances, and fewer chunks keep the partial-row reduction short.
int choose_jchunk(long long itiles_total, int nj, int slots) {
    if (nj <= 0) return 1;
    int nch = best_nch(itiles_total > 0 ? itiles_total : 1, nj, slots, 512);
    return (nj + nch - 1) / nch;
}

// ------------------------------------------------------------------------------------------
// Force-shape table of the cutoff (TreePM PP) force: PG5/table/libpg5/pg5_table.c:43-113.
// One table per library, as the reference's global Force_table; uploaded when it changes.
struct TableState {
    std::mutex mu;
    int exp_bit = 4;           // pg5_table.h:7-8 (EXP_BIT 4, FRC_BIT 5 -> 512 entries)
    int frc_bit = -1;          // -1: PGB_G5T_FRC_BIT or 5
    std::vector<float> tab;    // [size][2] (f, df/ds)
    double xscale = 0.0;       // pg5_set_xscale (phantom_g5.c:43-50)
    bool built = false;
    int version = 0;
    DevBuf<float2> dev;
    int dev_version = -1;
};
TableState g_tab;

inline int tab_frc() {
    if (g_tab.frc_bit < 0) g_tab.frc_bit = env_int("PGB_G5T_FRC_BIT", 5, 1, 8);
    return g_tab.frc_bit;
}
inline int tab_size() { return 1 << (g_tab.exp_bit + tab_frc()); }
#ifdef PGB_TABLE
int table_entries() { return tab_size(); }
#else
int table_entries() { return 0; }
#endif

inline float bits_float(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t float_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Table generation in the reference's float arithmetic (bit-identical tables).
void gen_table_locked(double (*force_func)(double), double rcut) {
    const int frc = tab_frc(), tbl = tab_size();
    const uint32_t tick = 1u << (23 - frc);
    const float r2max = (float)(rcut * rcut);
    const float fmax = (float)((double)(1 << (1 << g_tab.exp_bit)) * (2.0 - 1.0 / (1 << frc)));
    const float r2scale = (fmax - 2.0f) / r2max;
    g_tab.tab.assign((size_t)tbl * 2, 0.f);
    uint32_t u = float_bits(2.0f);
    for (int i = 0; i < tbl; i++, u += tick) {
        float f = bits_float(u);
        float r2 = (float)(((double)f - 2.0) / (double)r2scale);
        float r = sqrtf(r2);
        g_tab.tab[2 * i] = (float)force_func((double)r);
    }
    u = float_bits(2.0f);
    int i;
    for (i = 0; i < tbl - 1; i++) {
        float x0 = bits_float(u);
        u += tick;
        float x1 = bits_float(u);
        float y0 = g_tab.tab[2 * i], y1 = g_tab.tab[2 * (i + 1)];
        g_tab.tab[2 * i + 1] = (y1 - y0) / (x1 - x0);
    }
    g_tab.tab[2 * i + 1] = 0.0f;
    g_tab.xscale = (double)sqrtf(r2scale);
    g_tab.built = true;
    g_tab.version++;
}

// S2 softening-difference shape, the table g5_open builds (pg5_table.c:8-35).
double reff(double sft, double r) {
    double eta = 2.0 * r / sft;
    if (eta < 1.0)
        return (224. + eta * eta * (-224. + eta * (70. + eta * (48. - eta * 21.)))) * 2.0 / (35.0 * std::pow(sft, 3));
    if (eta < 2.0)
        return (12. / (eta * eta) - 224. +
                eta * (896. + eta * (-840. + eta * (224. + eta * (70. + eta * (-48. + eta * 7.)))))) *
               2.0 / (35.0 * eta * std::pow(sft, 3));
    return 1.0 / std::pow(r, 3);
}
double g_sft_pp = 0.1 / 64, g_sft_pm = 3.0 / 64;  // pppm.h:4-6
double s2_force(double r) { return reff(g_sft_pp, r) - reff(g_sft_pm, r); }

void ensure_table_locked() {
    if (!g_tab.built) {
        g_sft_pp = 0.1 / 64;
        g_sft_pm = 3.0 / 64;
        gen_table_locked(s2_force, g_sft_pm);
    }
}

bool table_args(G5Args& a) {
    std::lock_guard<std::mutex> g(g_tab.mu);
    ensure_table_locked();
    const int tbl = tab_size(), frc = tab_frc();
    if (tbl > G5_TBL_MAX) {
        raise(g_err, LIB, PGB_ERR_CAPACITY, "table of %d entries > %d", tbl, G5_TBL_MAX);
        return false;
    }
    if (g_tab.dev_version != g_tab.version) {
        PGB_CUDA_OR(g_err, LIB, g_tab.dev.reserve(tbl), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemcpy(g_tab.dev.p, g_tab.tab.data(), (size_t)tbl * sizeof(float2),
                                           cudaMemcpyHostToDevice), return false);
        g_tab.dev_version = g_tab.version;
    }
    a.table = g_tab.dev.p;
    a.tbl_size = tbl;
    a.tbl_shift = 23 - frc;
    a.r2cut = bits_float((1u << 30) | ((uint32_t)(tbl - 1) << (23 - frc)));
    a.ascale = 1.0 / g_tab.xscale;
    return true;
}

#ifdef PGB_TABLE
// i and j coordinates of the table kind are pre-scaled by xscale: j in float arithmetic
// (phantom_g5.c:112-128: cvtpd2ps then * (float)xscale), i through double
// (phantom_g5.c:96-104: (float)x * Xscale rounded to float).
inline float scale_j(double x) {
    return (float)x * (float)g_tab.xscale;
}
inline float scale_i(double x) {
    return (float)((double)(float)x * g_tab.xscale);
}
#endif

// Staged work list + launch of one devid / plan.
struct Launcher {
    Stager<float4, double4> st;

    bool stage(cudaStream_t s, const std::vector<Task>& tasks, const std::vector<Group>& groups, int rows,
               const float4* i_host, int ni_host) {
        PGB_CUDA_OR(g_err, LIB, st.stage(s, tasks, groups, rows, ITILE_MAX, i_host, ni_host), return false);
        return true;
    }

    // Launch over the staged work list.  The kernel leaves its task counter at zero, so the same
    // staged list can be launched again (e.g. from a CUDA graph) without a reset.
    bool launch(int kind, int cfg, cudaStream_t s, const float4* i_dev, const float4* jpos, const float4* jaux,
                double4* out, const int* jidx = nullptr) {
        if (st.ntasks <= 0) return true;
        G5Args a;
        a.ipos = i_dev ? i_dev : st.irecs();
        a.jpos = jpos;
        a.jaux = jaux;
        a.jidx = jidx;
        a.tasks = st.tasks();
        a.ntasks = st.ntasks;
        a.task_counter = st.counter();
        a.groups = st.groups();
        a.group_counters = st.dgcnt.p;
        a.partial = st.dpart.p;
        a.out = out;
        a.itile = cfg_itile(cfg);
        a.table = nullptr;
        a.tbl_size = 0;
        a.tbl_shift = 0;
        a.r2cut = 0.f;
        a.ascale = 1.0;
        if (kind == G5_TABLE && !table_args(a)) return false;
        int slots = sm_count(g_device) * occupancy_of(kind, cfg);
        int grid = st.ntasks < slots ? st.ntasks : slots;
        PGB_CUDA_OR(g_err, LIB, launch_kind(kind, cfg, grid, a, s), return false);
        // completion marker for pgb5_plan_update; a launch captured into a CUDA graph records
        // none (its replays are the caller's to finish before the plan is updated)
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        PGB_CUDA_OR(g_err, LIB, cudaStreamIsCapturing(s, &cap), return false);
        if (cap == cudaStreamCaptureStatusNone) {
            if (!launched)
                PGB_CUDA_OR(g_err, LIB, cudaEventCreateWithFlags(&launched, cudaEventDisableTiming), return false);
            PGB_CUDA_OR(g_err, LIB, cudaEventRecord(launched, s), return false);
        }
        return true;
    }
    // the task list of the latest launch is no longer read once this returns
    bool wait_launched() {
        if (launched) PGB_CUDA_OR(g_err, LIB, cudaEventSynchronize(launched), return false);
        return true;
    }
    void release() {
        st.release();
        if (launched) cudaEventDestroy(launched);
        launched = nullptr;
    }
    cudaEvent_t launched = nullptr;   // recorded after every launch
};

struct Dev {
    std::mutex mu;
    bool ready = false;
    cudaStream_t stream = nullptr;
    // j-particles: host mirror (pinned) + device copy, dirty range uploaded lazily
    HostBuf<float4> jh;
    HostBuf<float4> jeh;  // symmetric: eps2_j in .x
    DevBuf<float4> jd, jed;
    int jdirty_lo = 1 << 30, jdirty_hi = 0, jcap = 0;
    int nbody = 0;
    // quadrupole cells: word 0 (x y z m) + 2 words of Q per cell
    HostBuf<float4> ch, cqh;
    DevBuf<float4> cd, cqd;
    int cdirty_lo = 1 << 30, cdirty_hi = 0, ccap = 0;
    int ncell = 0;
    // i pipes and results of g5_run / g5c_run
    float4 ip[MAXPIPE];
    DevBuf<double4> outd;
    HostBuf<double4> outh;
    HostBuf<float4> ibuf;
    int pending = 0;     // number of results of the last g5_run / g5c_run (0: none)
    bool inflight = false;  // a g5_run has not been synchronised yet
    Launcher L;
};

// Wait for an unsynchronised g5_run before the host mirrors it reads from are rewritten.
bool quiesce(Dev& d) {
    if (!d.inflight) return true;
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(d.stream), return false);
    d.inflight = false;
    return true;
}

Dev g_devs[MAXDEV];

Dev* get_dev(int devid) {
    if (devid < 0 || devid >= MAXDEV) {
        raise(g_err, LIB, PGB_ERR_ARG, "devid %d out of range [0, %d)", devid, MAXDEV);
        return nullptr;
    }
    if (!ensure_device()) return nullptr;
    Dev& d = g_devs[devid];
    if (!d.ready) {
        PGB_CUDA_OR(g_err, LIB, cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking), return nullptr);
        d.ready = true;
    }
    return &d;
}

bool grow_j(Dev& d, int need) {
    if (need > jmemsize()) {
        raise(g_err, LIB, PGB_ERR_CAPACITY, "j-memory overflow: %d records > jmemsize %d", need, jmemsize());
        return false;
    }
    if (need <= d.jcap) return true;
    int cap = d.jcap ? d.jcap : 4096;
    while (cap < need) cap *= 2;
    if (cap > jmemsize()) cap = jmemsize();
    PGB_CUDA_OR(g_err, LIB, d.jh.reserve(cap, true), return false);
    PGB_CUDA_OR(g_err, LIB, d.jeh.reserve(cap, true), return false);
    for (int j = d.jcap; j < cap; j++) {
        d.jh.p[j] = make_float4(0, 0, 0, 0);
        d.jeh.p[j] = make_float4(1, 0, 0, 0);
    }
    d.jdirty_lo = 0;  // new device buffer: upload everything written so far
    d.jdirty_hi = cap;
    d.jcap = cap;
    return true;
}

bool grow_c(Dev& d, int need) {
    if (need > jmemsize() / 2) {
        raise(g_err, LIB, PGB_ERR_CAPACITY, "cell-memory overflow: %d cells > %d", need, jmemsize() / 2);
        return false;
    }
    if (need <= d.ccap) return true;
    int cap = d.ccap ? d.ccap : 2048;
    while (cap < need) cap *= 2;
    PGB_CUDA_OR(g_err, LIB, d.ch.reserve(cap, true), return false);
    PGB_CUDA_OR(g_err, LIB, d.cqh.reserve(2 * (size_t)cap, true), return false);
    for (int j = d.ccap; j < cap; j++) {
        d.ch.p[j] = make_float4(0, 0, 0, 0);
        d.cqh.p[2 * j] = make_float4(0, 0, 0, 0);
        d.cqh.p[2 * j + 1] = make_float4(0, 0, 0, 0);
    }
    d.cdirty_lo = 0;
    d.cdirty_hi = cap;
    d.ccap = cap;
    return true;
}

bool flush_j(Dev& d) {
    if (d.jdirty_hi <= d.jdirty_lo) return true;
    PGB_CUDA_OR(g_err, LIB, d.jd.reserve(d.jcap), return false);
    size_t lo = d.jdirty_lo, n = (size_t)(d.jdirty_hi - d.jdirty_lo);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(d.jd.p + lo, d.jh.p + lo, n * sizeof(float4),
                                            cudaMemcpyHostToDevice, d.stream), return false);
    if (PARTICLE_KIND == G5_SYMMETRIC) {
        PGB_CUDA_OR(g_err, LIB, d.jed.reserve(d.jcap), return false);
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(d.jed.p + lo, d.jeh.p + lo, n * sizeof(float4),
                                                cudaMemcpyHostToDevice, d.stream), return false);
    }
    d.jdirty_lo = 1 << 30;
    d.jdirty_hi = 0;
    return true;
}

bool flush_c(Dev& d) {
    if (d.cdirty_hi <= d.cdirty_lo) return true;
    PGB_CUDA_OR(g_err, LIB, d.cd.reserve(d.ccap), return false);
    PGB_CUDA_OR(g_err, LIB, d.cqd.reserve(2 * (size_t)d.ccap), return false);
    size_t lo = d.cdirty_lo, n = (size_t)(d.cdirty_hi - d.cdirty_lo);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(d.cd.p + lo, d.ch.p + lo, n * sizeof(float4),
                                            cudaMemcpyHostToDevice, d.stream), return false);
    PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(d.cqd.p + 2 * lo, d.cqh.p + 2 * lo, 2 * n * sizeof(float4),
                                            cudaMemcpyHostToDevice, d.stream), return false);
    d.cdirty_lo = 1 << 30;
    d.cdirty_hi = 0;
    return true;
}

// Launch `kind` for ni i-records (host) against this devid's j-memory (nbody records) or cell
// memory (ncell cells).  Results land in d.outh after the stream synchronises.
bool compute(Dev& d, int kind, int ni, const float4* ih) {
    int nj = kind == G5_QUAD ? d.ncell : d.nbody;
    if (kind == G5_QUAD) {
        if (!grow_c(d, nj > 0 ? nj : 1) || !flush_c(d)) return false;
    } else {
        if (!grow_j(d, nj > 0 ? nj : 1) || !flush_j(d)) return false;
    }
    PGB_CUDA_OR(g_err, LIB, d.outd.reserve(ni > 0 ? ni : 1), return false);
    PGB_CUDA_OR(g_err, LIB, d.outh.reserve(ni > 0 ? ni : 1), return false);
    std::vector<Task> tasks;
    std::vector<Group> groups;
    const int cfg = pick_cfg(kind, ni);
    const int itile = cfg_itile(cfg);
    int slots = sm_count(g_device) * occupancy_of(kind, cfg);
    long long itiles = (ni + itile - 1) / itile;
    int jchunk = choose_jchunk(itiles, nj, slots);
    int rows = plan_item(tasks, groups, 0, ni, 0, nj, itile, jchunk, 0);
    const float4* jpos = kind == G5_QUAD ? d.cd.p : d.jd.p;
    const float4* jaux = kind == G5_QUAD ? d.cqd.p : (kind == G5_SYMMETRIC ? d.jed.p : nullptr);
    if (!d.L.stage(d.stream, tasks, groups, rows, ih, ni)) return false;
    if (!d.L.launch(kind, cfg, d.stream, nullptr, jpos, jaux, d.outd.p)) return false;
    if (ni > 0)
        PGB_CUDA_OR(g_err, LIB, cudaMemcpyAsync(d.outh.p, d.outd.p, (size_t)ni * sizeof(double4),
                                                cudaMemcpyDeviceToHost, d.stream), return false);
    return true;
}

bool sync_dev(Dev& d) {
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(d.stream), return false);
    d.inflight = false;
    return true;
}

void write_out(const double4* o, int ni, double (*a)[3], double* p) {
    for (int i = 0; i < ni; i++) {
        a[i][0] = o[i].x;
        a[i][1] = o[i].y;
        a[i][2] = o[i].z;
#ifdef PGB_TABLE
        p[i] = 0.0;      // the table kernel computes no potential (PG5/table phantom_g5.c:145-154)
#else
        p[i] = -o[i].w;  // GRAPE-5 return sign (phantom_g5.c:251-259)
#endif
    }
}

// The current xscale of the table library (building the default table on first use, as
// g5_open does); 0 for the other builds, which do not scale.
double current_xscale() {
#ifdef PGB_TABLE
    std::lock_guard<std::mutex> g(g_tab.mu);
    ensure_table_locked();
    return g_tab.xscale;
#else
    return 0.0;
#endif
}

inline float4 make_i(const double* x, float e2) {
#ifdef PGB_TABLE
    (void)e2;
    return make_float4(scale_i(x[0]), scale_i(x[1]), scale_i(x[2]), 0.f);
#else
    return make_float4((float)x[0], (float)x[1], (float)x[2], e2);
#endif
}

bool check_ni(int ni) {
    if (ni < 0 || ni > npipes()) {
        raise(g_err, LIB, PGB_ERR_ARG, "ni = %d outside [0, %d] pipelines", ni, npipes());
        return false;
    }
    return true;
}

void set_xi_impl(int devid, int ni, const double (*xi)[3], const double* eps2, bool per_i) {
    if (!check_ni(ni)) return;
    Dev* d = get_dev(devid);
    if (!d) return;
    current_xscale();
    std::lock_guard<std::mutex> g(d->mu);
    float e_all = (float)(g_eps * g_eps);
    for (int i = 0; i < ni; i++) d->ip[i] = make_i(xi[i], per_i ? (float)eps2[i] : e_all);
}

void run_impl(int devid, int kind) {
    Dev* d = get_dev(devid);
    if (!d) return;
    std::lock_guard<std::mutex> g(d->mu);
    int n = npipes();
    if (!quiesce(*d)) return;
    if (compute(*d, kind, n, d->ip)) {
        d->pending = n;
        d->inflight = true;
    }
}

void get_force_impl(int devid, int ni, double (*a)[3], double* p) {
    if (!check_ni(ni)) return;
    Dev* d = get_dev(devid);
    if (!d) return;
    std::lock_guard<std::mutex> g(d->mu);
    if (!d->pending) {
        raise(g_err, LIB, PGB_ERR_ARG, "g5_get_force without a preceding g5_run on devid %d", devid);
        return;
    }
    if (!sync_dev(*d)) return;
    write_out(d->outh.p, ni, a, p);
}

// All ni in one launch (the reference loops over npipes-wide calls, phantom_g5.c:276-300).
void calc_impl(int devid, int kind, const double (*x)[3], const double* eps2, double (*a)[3], double* p, int ni) {
    if (ni <= 0) return;
    current_xscale();
    Dev* d = get_dev(devid);
    if (!d) return;
    Dev* dj = d;
    std::lock_guard<std::mutex> g(dj->mu);
    if (!quiesce(*dj)) return;
    if (dj->ibuf.reserve(ni) != cudaSuccess) {
        raise(g_err, LIB, PGB_ERR_CUDA, "pinned i-buffer allocation failed (%d)", ni);
        return;
    }
    float e_all = (float)(g_eps * g_eps);
    for (int i = 0; i < ni; i++) dj->ibuf.p[i] = make_i(x[i], eps2 ? (float)eps2[i] : e_all);
    if (!compute(*dj, kind, ni, dj->ibuf.p) || !sync_dev(*dj)) return;
    write_out(dj->outh.p, ni, a, p);
}

}  // namespace

// ============================================================================================
// GRAPE-5 API (PG5/newton/libpg5/gp5util.h:10-39)

PGB_EXPORT int g5_get_number_of_pipelines(void) { return npipes(); }
PGB_EXPORT int g5_get_jmemsize(void) { return jmemsize(); }

#ifdef PGB_TABLE
extern "C" void pg5_gen_s2_force_table(double sft_for_PP, double sft_for_PM);
#endif

PGB_EXPORT void g5_open(void) {
    ensure_device();
#ifdef PGB_TABLE
    pg5_gen_s2_force_table(0.1 / 64, 3.0 / 64);  // g5_open builds the S2 table (phantom_g5.c:56-61)
#endif
}

PGB_EXPORT void g5_close(void) {
    if (g_device < 0) return;
    cudaSetDevice(g_device);
    for (auto& d : g_devs) {
        std::lock_guard<std::mutex> g(d.mu);
        if (d.ready) {
            cudaStreamSynchronize(d.stream);
            d.jd.release();
            d.jed.release();
            d.cd.release();
            d.cqd.release();
            d.outd.release();
            d.L.release();
            d.jdirty_lo = 0;
            d.jdirty_hi = d.jcap;
            d.cdirty_lo = 0;
            d.cdirty_hi = d.ccap;
            d.pending = 0;
        }
    }
}

PGB_EXPORT void g5_set_eps_to_all(double eps) { g_eps = eps; }

PGB_EXPORT void g5_set_epsMC(int devid, int ni, double* eps) {
    if (!check_ni(ni)) return;
    Dev* d = get_dev(devid);
    if (!d) return;
    std::lock_guard<std::mutex> g(d->mu);
    for (int i = 0; i < ni; i++) d->ip[i].w = (float)(eps[i] * eps[i]);  // phantom_g5.c:72-82
}
PGB_EXPORT void g5_set_eps(int ni, double* eps) { g5_set_epsMC(0, ni, eps); }

PGB_EXPORT void g5_set_nMC(int devid, int n) {
    Dev* d = get_dev(devid);
    if (!d) return;
    if (n < 0 || n > jmemsize()) {
        raise(g_err, LIB, PGB_ERR_CAPACITY, "g5_set_n(%d) outside [0, %d]", n, jmemsize());
        return;
    }
    std::lock_guard<std::mutex> g(d->mu);
    d->nbody = n;
}
PGB_EXPORT void g5_set_n(int n) { g5_set_nMC(0, n); }

PGB_EXPORT void g5_set_xiMC(int devid, int ni, double (*xi)[3]) { set_xi_impl(devid, ni, xi, nullptr, false); }
PGB_EXPORT void g5_set_xeiMC(int devid, int ni, double (*xi)[3], double* eps2) {
    set_xi_impl(devid, ni, xi, eps2, true);
}
PGB_EXPORT void g5_set_xi(int ni, double (*xi)[3]) { g5_set_xiMC(0, ni, xi); }
PGB_EXPORT void g5_set_xei(int ni, double (*xi)[3], double* eps2) { g5_set_xeiMC(0, ni, xi, eps2); }

#ifdef PGB_SYMMETRIC
PGB_EXPORT void g5_set_xmjMC(int devid, int adr, int nj, double (*xj)[3], double* mj, double* epsj2) {
#else
PGB_EXPORT void g5_set_xmjMC(int devid, int adr, int nj, double (*xj)[3], double* mj) {
#endif
    if (adr < 0 || nj < 0) {
        raise(g_err, LIB, PGB_ERR_ARG, "g5_set_xmj: adr %d nj %d", adr, nj);
        return;
    }
    current_xscale();
    Dev* d = get_dev(devid);
    if (!d) return;
    std::lock_guard<std::mutex> g(d->mu);
    if (!quiesce(*d) || !grow_j(*d, adr + nj)) return;
    for (int j = adr; j < adr + nj; j++) {
#ifdef PGB_TABLE
        d->jh.p[j] = make_float4(scale_j(xj[j][0]), scale_j(xj[j][1]), scale_j(xj[j][2]), (float)mj[j]);
#else
        d->jh.p[j] = make_float4((float)xj[j][0], (float)xj[j][1], (float)xj[j][2], (float)mj[j]);
#endif
#ifdef PGB_SYMMETRIC
        d->jeh.p[j] = make_float4((float)epsj2[j], 0, 0, 0);
#endif
    }
    if (nj > 0) {
        if (adr < d->jdirty_lo) d->jdirty_lo = adr;
        if (adr + nj > d->jdirty_hi) d->jdirty_hi = adr + nj;
    }
}

#ifdef PGB_SYMMETRIC
PGB_EXPORT void g5_set_xmj(int adr, int nj, double (*xj)[3], double* mj, double* epsj2) {
    g5_set_xmjMC(0, adr, nj, xj, mj, epsj2);
}
#else
PGB_EXPORT void g5_set_xmj(int adr, int nj, double (*xj)[3], double* mj) { g5_set_xmjMC(0, adr, nj, xj, mj); }
#endif

PGB_EXPORT void g5_runMC(int devid) { run_impl(devid, PARTICLE_KIND); }
PGB_EXPORT void g5_run(void) { g5_runMC(0); }

PGB_EXPORT void g5_get_forceMC(int devid, int ni, double (*a)[3], double* p) { get_force_impl(devid, ni, a, p); }
PGB_EXPORT void g5_get_force(int ni, double (*a)[3], double* p) { g5_get_forceMC(0, ni, a, p); }

PGB_EXPORT void g5_calculate_force_on_xMC(int devid, double (*x)[3], double (*a)[3], double* p, int ni) {
    calc_impl(devid, PARTICLE_KIND, x, nullptr, a, p, ni);
}
PGB_EXPORT void g5_calculate_force_on_xeMC(int devid, double (*x)[3], double* eps2, double (*a)[3], double* p,
                                           int ni) {
    calc_impl(devid, PARTICLE_KIND, x, eps2, a, p, ni);
}
PGB_EXPORT void g5_calculate_force_on_x(double (*x)[3], double (*a)[3], double* p, int ni) {
    g5_calculate_force_on_xMC(0, x, a, p, ni);
}
PGB_EXPORT void g5_calculate_force_on_xe(double (*x)[3], double* eps2, double (*a)[3], double* p, int ni) {
    g5_calculate_force_on_xeMC(0, x, eps2, a, p, ni);
}

#ifdef PGB_TABLE
// ============================================================================================
// Table (cutoff-force) API (PG5/table/libpg5/gp5util.h:9-35, pg5_table.h:38-40)

extern "C" {
// The reference exports its table as a global (pg5_table.h:31); this copy mirrors the current
// table (first 2^(EXP_BIT+FRC_BIT) rows) after every table generation.
__attribute__((visibility("default"))) float Force_table[G5_TBL_MAX][2];
}

namespace {
void mirror_table_locked() {
    int n = tab_size() < G5_TBL_MAX ? tab_size() : G5_TBL_MAX;
    std::memcpy(Force_table, g_tab.tab.data(), (size_t)n * 2 * sizeof(float));
}
}  // namespace

PGB_EXPORT void pg5_set_xscale(double xscale) {
    std::lock_guard<std::mutex> g(g_tab.mu);
    g_tab.xscale = xscale;  // phantom_g5.c:43-50
}

// f(r) is the force shape divided by r (an r^-3-like function); rcut the cutoff radius.
PGB_EXPORT void pg5_gen_force_table(double (*force_func)(double), double rcut) {
    if (!force_func || !(rcut > 0)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pg5_gen_force_table: null function or rcut <= 0");
        return;
    }
    std::lock_guard<std::mutex> g(g_tab.mu);
    gen_table_locked(force_func, rcut);
    mirror_table_locked();
}

PGB_EXPORT void pg5_gen_s2_force_table(double sft_for_PP, double sft_for_PM) {
    std::lock_guard<std::mutex> g(g_tab.mu);
    g_sft_pp = sft_for_PP;
    g_sft_pm = sft_for_PM;
    gen_table_locked(s2_force, sft_for_PM);
    mirror_table_locked();
}

// Table resolution: 2^(exp_bit + frc_bit) entries (the reference fixes EXP_BIT 4, FRC_BIT 5 at
// compile time, pg5_table.h:7-17).  Takes effect at the next table generation.
PGB_EXPORT int pg5_set_table_bits(int exp_bit, int frc_bit) {
    if (exp_bit != 4 || frc_bit < 1 || frc_bit > 8) {
        raise(g_err, LIB, PGB_ERR_ARG, "pg5_set_table_bits(%d, %d): EXP_BIT must be 4, FRC_BIT 1..8", exp_bit, frc_bit);
        return PGB_ERR_ARG;
    }
    std::lock_guard<std::mutex> g(g_tab.mu);
    g_tab.exp_bit = exp_bit;
    g_tab.frc_bit = frc_bit;
    g_tab.built = false;
    return PGB_OK;
}

// Copy of the current table: returns the number of entries, writes min(n, max_entries) rows.
PGB_EXPORT int pg5_get_table(float* out, int max_entries, double* xscale) {
    std::lock_guard<std::mutex> g(g_tab.mu);
    ensure_table_locked();
    int n = tab_size();
    if (out) std::memcpy(out, g_tab.tab.data(), (size_t)(n < max_entries ? n : max_entries) * 2 * sizeof(float));
    if (xscale) *xscale = g_tab.xscale;
    return n;
}

PGB_EXPORT void g5_set_range(double xmin, double xmax, double mmin) {
    (void)xmin; (void)xmax; (void)mmin;  // no-op, as phantom_g5.c:77-78
}
PGB_EXPORT void g5_set_eta(double eta) { (void)eta; }

// The reference leaves this a stub (phantom_g5.c:80-84, "please implement"): here it installs
// ffunc as the force shape with cutoff fcut (the table kernel has no potential, so pfunc,
// pcut and the corrections are ignored).
PGB_EXPORT void g5_set_cutoff_table(double (*ffunc)(double), double fcut, double fcor, double (*pfunc)(double),
                                    double pcut, double pcor) {
    (void)fcor; (void)pfunc; (void)pcut; (void)pcor;
    if (ffunc) pg5_gen_force_table(ffunc, fcut);
}
#else
// ============================================================================================
// Quadrupole j-cells (PG5/newton_quad/quad/quad_util.h:8-15)

PGB_EXPORT void g5c_set_nMC(int devid, int n) {
    Dev* d = get_dev(devid);
    if (!d) return;
    if (n < 0 || n > jmemsize() / 2) {
        raise(g_err, LIB, PGB_ERR_CAPACITY, "g5c_set_n(%d) outside [0, %d]", n, jmemsize() / 2);
        return;
    }
    std::lock_guard<std::mutex> g(d->mu);
    d->ncell = n;
}

// qj = (xx, xy, xz, yy, yz, zz) of the traceless moment sum m (3 d d - d^2 I) (source.cpp:215-248)
PGB_EXPORT void g5c_set_xmjMC(int devid, int adr, int nj, double (*xj)[3], double* mj, double (*qj)[6]) {
    if (adr < 0 || nj < 0) {
        raise(g_err, LIB, PGB_ERR_ARG, "g5c_set_xmj: adr %d nj %d", adr, nj);
        return;
    }
    Dev* d = get_dev(devid);
    if (!d) return;
    std::lock_guard<std::mutex> g(d->mu);
    if (!quiesce(*d) || !grow_c(*d, adr + nj)) return;
    for (int j = adr; j < adr + nj; j++) {
        d->ch.p[j] = make_float4((float)xj[j][0], (float)xj[j][1], (float)xj[j][2], (float)mj[j]);
        d->cqh.p[2 * j] = make_float4((float)qj[j][0], (float)qj[j][1], (float)qj[j][2], (float)qj[j][3]);
        d->cqh.p[2 * j + 1] = make_float4((float)qj[j][4], (float)qj[j][5], 0.f, 0.f);
    }
    if (nj > 0) {
        if (adr < d->cdirty_lo) d->cdirty_lo = adr;
        if (adr + nj > d->cdirty_hi) d->cdirty_hi = adr + nj;
    }
}
// The reference's structure-of-arrays variant (quad_g5c.c:19-196) computes the same sums.
PGB_EXPORT void g5c_set_xmjMC0(int devid, int adr, int nj, double (*xj)[3], double* mj, double (*qj)[6]) {
    g5c_set_xmjMC(devid, adr, nj, xj, mj, qj);
}

PGB_EXPORT void g5c_runMC(int devid) { run_impl(devid, G5_QUAD); }
PGB_EXPORT void g5c_runMC0(int devid) { g5c_runMC(devid); }

PGB_EXPORT void g5c_calculate_force_on_xMC(int devid, double (*x)[3], double (*a)[3], double* p, int ni) {
    calc_impl(devid, G5_QUAD, x, nullptr, a, p, ni);
}
PGB_EXPORT void g5c_calculate_force_on_xMC0(int devid, double (*x)[3], double (*a)[3], double* p, int ni) {
    g5c_calculate_force_on_xMC(devid, x, a, p, ni);
}

// ============================================================================================
// Fortran bindings (PG5/newton/libpg5/pg5_fortran.c:1-119)

PGB_EXPORT int g5_get_number_of_pipelines_(void) { return g5_get_number_of_pipelines(); }
PGB_EXPORT int g5_get_jmemsize_(void) { return g5_get_jmemsize(); }
PGB_EXPORT void g5_open_(void) { g5_open(); }
PGB_EXPORT void g5_close_(void) { g5_close(); }
PGB_EXPORT void g5_set_eps_to_all_(double* eps) { g5_set_eps_to_all(*eps); }
PGB_EXPORT void g5_set_n_(int* n) { g5_set_n(*n); }
PGB_EXPORT void g5_set_nMC_(int* devid, int* n) { g5_set_nMC(*devid, *n); }
PGB_EXPORT void g5_set_xi_(int* ni, double (*xi)[3]) { g5_set_xi(*ni, xi); }
PGB_EXPORT void g5_set_xei_(int* ni, double (*xi)[3], double* eps2) { g5_set_xei(*ni, xi, eps2); }
PGB_EXPORT void g5_set_xiMC_(int* devid, int* ni, double (*xi)[3]) { g5_set_xiMC(*devid, *ni, xi); }
PGB_EXPORT void g5_set_xeiMC_(int* devid, int* ni, double (*xi)[3], double* eps2) {
    g5_set_xeiMC(*devid, *ni, xi, eps2);
}
#ifdef PGB_SYMMETRIC
PGB_EXPORT void g5_set_xmj_(int* adr, int* nj, double (*xj)[3], double* mj, double* eps2) {
    g5_set_xmj(*adr, *nj, xj, mj, eps2);
}
PGB_EXPORT void g5_set_xmjMC_(int* devid, int* adr, int* nj, double (*xj)[3], double* mj, double* eps2) {
    g5_set_xmjMC(*devid, *adr, *nj, xj, mj, eps2);
}
#else
PGB_EXPORT void g5_set_xmj_(int* adr, int* nj, double (*xj)[3], double* mj) { g5_set_xmj(*adr, *nj, xj, mj); }
PGB_EXPORT void g5_set_xmjMC_(int* devid, int* adr, int* nj, double (*xj)[3], double* mj) {
    g5_set_xmjMC(*devid, *adr, *nj, xj, mj);
}
#endif
PGB_EXPORT void g5_run_(void) { g5_run(); }
PGB_EXPORT void g5_runMC_(int* devid) { g5_runMC(*devid); }
PGB_EXPORT void g5_get_force_(int* ni, double (*a)[3], double* p) { g5_get_force(*ni, a, p); }
PGB_EXPORT void g5_get_forceMC_(int* devid, int* ni, double (*a)[3], double* p) { g5_get_forceMC(*devid, *ni, a, p); }
PGB_EXPORT void g5_calculate_force_on_x_(double (*x)[3], double (*a)[3], double* p, int* ni) {
    g5_calculate_force_on_x(x, a, p, *ni);
}
PGB_EXPORT void g5_calculate_force_on_xe_(double (*x)[3], double* eps2, double (*a)[3], double* p, int* ni) {
    g5_calculate_force_on_xe(x, eps2, a, p, *ni);
}
PGB_EXPORT void g5_calculate_force_on_xMC_(int* devid, double (*x)[3], double (*a)[3], double* p, int* ni) {
    g5_calculate_force_on_xMC(*devid, x, a, p, *ni);
}
PGB_EXPORT void g5_calculate_force_on_xeMC_(int* devid, double (*x)[3], double* eps2, double (*a)[3], double* p,
                                            int* ni) {
    g5_calculate_force_on_xeMC(*devid, x, eps2, a, p, *ni);
}

#endif  // PGB_TABLE

// ============================================================================================
// Library status and the batched path (no reference counterpart; see include/pgb_g5.h)

PGB_EXPORT int pgb5_last_error(char* buf, int len) {
    std::lock_guard<std::mutex> g(g_err.mu);
    if (buf && len > 0) {
        std::strncpy(buf, g_err.msg.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return g_err.code;
}
PGB_EXPORT void pgb5_clear_error(void) {
    std::lock_guard<std::mutex> g(g_err.mu);
    g_err.code = 0;
    g_err.msg.clear();
}
PGB_EXPORT void pgb5_set_abort(int on) {
    std::lock_guard<std::mutex> g(g_err.mu);
    g_err.abort_on_error = on ? 1 : 0;
}

struct pgb5_plan {
    int kind;
    int cfg;
    std::vector<int> items;        // [nitem][4], kept for re-planning by the autotuner
    long long shape_key = 0;
    std::vector<Task> tasks;
    std::vector<Group> groups;
    int rows;
    long long interactions;
    Launcher L;
};

namespace {
bool check_kind(int kind) {
#ifdef PGB_TABLE
    if (kind != G5_TABLE) {
#else
    if (kind != G5_NEWTON && kind != G5_SYMMETRIC && kind != G5_QUAD) {
#endif
        raise(g_err, LIB, PGB_ERR_ARG, "unknown kind %d", kind);
        return false;
    }
    return true;
}

// Work list of a batch for one configuration.  A single item: one wave of equal tasks; many
// uneven items: about 4 tasks per resident CTA (j-chunks of >= 256 j, <= 512 chunks per item).
void plan_items(pgb5_plan* P) {
    const int nitem = (int)(P->items.size() / 4);
    const int* items = P->items.data();
    const int itile = cfg_itile(P->cfg);
    const int slots = sm_count(g_device) * occupancy_of(P->kind, P->cfg);
    long long work = 0;
    for (int k = 0; k < nitem; k++) work += (long long)items[4 * k + 1] * items[4 * k + 3];
    const long long per_task = work / ((nitem == 1 ? 1LL : 4LL) * slots) + 1;
    P->tasks.clear();
    P->groups.clear();
    P->rows = 0;
    P->interactions = 0;
    for (int k = 0; k < nitem; k++) {
        int ni = items[4 * k + 1], nj = items[4 * k + 3];
        long long tile_i = ni < itile ? ni : itile;
        long long jc;
        if (nitem == 1) {
            // one item of equal tasks: the chunk count that minimises the wave quantisation
            jc = choose_jchunk((ni + itile - 1) / itile, nj, slots);
        } else {
            jc = tile_i > 0 ? per_task / tile_i : nj;
            if (jc < 256) jc = 256;
            if (jc * 512 < nj) jc = (nj + 511) / 512;
        }
        if (jc > nj) jc = nj > 0 ? nj : 1;
        P->rows += plan_item(P->tasks, P->groups, items[4 * k], ni, items[4 * k + 2], nj, itile, (int)jc, P->rows);
        P->interactions += (long long)ni * nj;
    }
    // longest tasks first (persistent CTAs then finish together): a stable counting sort by the
    // power of two of the work, largest first -- linear in the task count, which matters for
    // plans made every step (a tree code's 1e5 tasks)
    {
        auto cls = [](const Task& t) {
            const unsigned long long w = (unsigned long long)t.ni * (unsigned long long)t.nj;
            return w ? 63 - __builtin_clzll(w) : 0;
        };
        size_t cnt[64] = {0};
        for (const Task& t : P->tasks) cnt[cls(t)]++;
        size_t pos[64], run = 0;
        for (int c = 63; c >= 0; c--) {
            pos[c] = run;
            run += cnt[c];
        }
        std::vector<Task> sorted(P->tasks.size());
        for (const Task& t : P->tasks) sorted[pos[cls(t)]++] = t;
        P->tasks.swap(sorted);
    }
}

// Autotune results by batch shape (kind, item count, largest item), shared by later plans.
std::mutex g_tune_mu;
std::vector<std::pair<long long, int>> g_tune;

int ilog2up(long long v) {
    int b = 0;
    while ((1LL << b) < v) b++;
    return b;
}

long long shape_key(int kind, int nitem, const int* items) {
    long long nimax = 0, njmax = 0;
    for (int k = 0; k < nitem; k++) {
        nimax = std::max<long long>(nimax, items[4 * k + 1]);
        njmax = std::max<long long>(njmax, items[4 * k + 3]);
    }
    return ((long long)ilog2up(nitem + 1) << 24) | ((long long)ilog2up(nimax + 1) << 16) |
           ((long long)ilog2up(njmax + 1) << 8) | kind;
}

int tuned_cfg(long long key) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    for (auto& e : g_tune)
        if (e.first == key) return e.second;
    return -1;
}

void set_tuned(long long key, int cfg) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    for (auto& e : g_tune)
        if (e.first == key) {
            e.second = cfg;
            return;
        }
    g_tune.emplace_back(key, cfg);
}

bool stage_plan(pgb5_plan* P, cudaStream_t s) {
    return P->L.stage(s, P->tasks, P->groups, P->rows, nullptr, 0);
}
}  // namespace

// items: [nitem][4] = (i_offset, i_count, j_offset, j_count) into the i- and j-arrays.
PGB_EXPORT int pgb5_plan_create(pgb5_plan** out, int kind, int nitem, const int* items) {
    if (!out || nitem < 0 || (nitem && !items) || !check_kind(kind)) return PGB_ERR_ARG;
    for (int k = 0; k < nitem; k++)
        if (items[4 * k + 1] < 0 || items[4 * k + 3] < 0 || items[4 * k] < 0 || items[4 * k + 2] < 0) {
            raise(g_err, LIB, PGB_ERR_ARG, "item %d has a negative offset or count", k);
            return PGB_ERR_ARG;
        }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    auto* P = new pgb5_plan();
    P->kind = kind;
    P->items.assign(items, items + 4 * (size_t)nitem);
    P->shape_key = shape_key(kind, nitem, items);
    long long nimax = 0;
    for (int k = 0; k < nitem; k++) nimax = std::max<long long>(nimax, items[4 * k + 1]);
    const int tuned = tuned_cfg(P->shape_key);
    P->cfg = tuned >= 0 ? tuned : pick_cfg(kind, nimax);
    plan_items(P);
    cudaStream_t s = nullptr;
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && stage_plan(P, s);
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (s) cudaStreamDestroy(s);
    if (!ok) {
        P->L.release();
        delete P;
        raise(g_err, LIB, PGB_ERR_CUDA, "plan staging failed");
        return PGB_ERR_CUDA;
    }
    *out = P;
    return PGB_OK;
}

// New items for an existing plan (same kind; the plan's configuration, chosen at creation, by
// the autotuner or pinned, is kept): the tasks are re-planned on the host and staged into the
// plan's own buffers, which grow only when the new list needs more.  A tree code whose lists
// change every step keeps one plan per kind instead of creating and destroying one per step
// (no device allocation, hence no device-wide synchronisation, in the step).  Waits until the
// plan's previous launches have finished reading its task list.
PGB_EXPORT int pgb5_plan_update(pgb5_plan* P, int nitem, const int* items) {
    if (!P || nitem < 0 || (nitem && !items)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb5_plan_update: null plan or bad item count %d", nitem);
        return PGB_ERR_ARG;
    }
    for (int k = 0; k < nitem; k++)
        if (items[4 * k + 1] < 0 || items[4 * k + 3] < 0 || items[4 * k] < 0 || items[4 * k + 2] < 0) {
            raise(g_err, LIB, PGB_ERR_ARG, "item %d has a negative offset or count", k);
            return PGB_ERR_ARG;
        }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    P->items.assign(items, items + 4 * (size_t)nitem);
    P->shape_key = shape_key(P->kind, nitem, items);
    plan_items(P);
    if (!P->L.wait_launched()) return g_err.code ? g_err.code : PGB_ERR_CUDA;
    cudaStream_t s = nullptr;
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && stage_plan(P, s);
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (s) cudaStreamDestroy(s);
    if (!ok) {
        raise(g_err, LIB, PGB_ERR_CUDA, "pgb5_plan_update: staging failed");
        return PGB_ERR_CUDA;
    }
    return PGB_OK;
}

PGB_EXPORT long long pgb5_plan_interactions(const pgb5_plan* P) { return P ? P->interactions : 0; }
PGB_EXPORT int pgb5_plan_tasks(const pgb5_plan* P) { return P ? (int)P->tasks.size() : 0; }

// Device-resident launch: ipos float4 (x,y,z,eps2), jpos float4 (x,y,z,m), jaux (symmetric:
// float4 eps2_j in .x; quad: two float4 of Q per cell), out double4 (ax,ay,az,pot_raw) where
// pot_raw = -sum m/r (newton/symmetric) or +sum(phi_p+phi_q) (quad).  stream: cudaStream_t.
PGB_EXPORT int pgb5_plan_launch(pgb5_plan* P, const void* ipos, const void* jpos, const void* jaux, void* out,
                                void* stream) {
    if (!P) return PGB_ERR_ARG;
    if (!ensure_device()) return PGB_ERR_NOGPU;
    cudaStream_t s = (cudaStream_t)stream;
    if (!ipos || !jpos || !out || ((P->kind == G5_SYMMETRIC || P->kind == G5_QUAD) && !jaux)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb5_plan_launch: null device pointer");
        return PGB_ERR_ARG;
    }
    if (!P->L.launch(P->kind, P->cfg, s, (const float4*)ipos, (const float4*)jpos, (const float4*)jaux,
                     (double4*)out))
        return g_err.code ? g_err.code : PGB_ERR_CUDA;
    return PGB_OK;
}

// As pgb5_plan_launch, with the items' j-ranges addressing the index list jidx (int32, device):
// record k of an item is jpos[jidx[j_offset + k]] (and its jaux words).  This runs the
// interaction lists of a tree code without copying records per group.
PGB_EXPORT int pgb5_plan_launch_indexed(pgb5_plan* P, const void* ipos, const void* jpos, const void* jaux,
                                        const int* jidx, void* out, void* stream) {
    if (!P) return PGB_ERR_ARG;
    if (!ensure_device()) return PGB_ERR_NOGPU;
    if (!ipos || !jpos || !out || !jidx || ((P->kind == G5_SYMMETRIC || P->kind == G5_QUAD) && !jaux)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb5_plan_launch_indexed: null device pointer");
        return PGB_ERR_ARG;
    }
    if (!P->L.launch(P->kind, P->cfg, (cudaStream_t)stream, (const float4*)ipos, (const float4*)jpos,
                     (const float4*)jaux, (double4*)out, jidx))
        return g_err.code ? g_err.code : PGB_ERR_CUDA;
    return PGB_OK;
}

namespace {
// The autotuner shared by pgb5_plan_tune and pgb5_plan_tune_indexed (jidx: nullptr or the
// index list the plan is launched with).
int tune_impl(pgb5_plan* P, const void* ipos, const void* jpos, const void* jaux, const int* jidx, void* out,
              void* stream, float* best_ms) {
    if (!P || !ipos || !jpos || !out) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb5_plan_tune: null argument");
        return -1;
    }
    if (!ensure_device()) return -1;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    PGB_CUDA_OR(g_err, LIB, cudaEventCreate(&e0), return -1);
    PGB_CUDA_OR(g_err, LIB, cudaEventCreate(&e1), return -1);
    int best = P->cfg;
    float best_t = 1e30f;
    for (int cfg = 0; cfg < G5_NCFG; cfg++) {
        if (!cfg_valid(P->kind, cfg)) continue;
        P->cfg = cfg;
        plan_items(P);
        if (!stage_plan(P, s)) break;
        float t = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
            cudaEventRecord(e0, s);
            const int rc = jidx ? pgb5_plan_launch_indexed(P, ipos, jpos, jaux, jidx, out, stream)
                                : pgb5_plan_launch(P, ipos, jpos, jaux, out, stream);
            if (rc != PGB_OK) break;
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0 && ms < t) t = ms;
        }
        if (t < best_t) {
            best_t = t;
            best = cfg;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P->cfg = best;
    plan_items(P);
    if (!stage_plan(P, s)) return -1;
    PGB_CUDA_OR(g_err, LIB, cudaStreamSynchronize(s), return -1);
    set_tuned(P->shape_key, best);
    if (best_ms) *best_ms = best_t;
    return best;
}
}  // namespace

// Autotuner: launches the plan with every kernel configuration valid for its kind on the
// caller's data, keeps the fastest (CUDA-event time, best of 2 after a warm-up launch),
// re-stages the plan with it and records it for later plans of the same shape.  Returns the
// chosen configuration index (-1 on error); *best_ms (optional) receives its launch time.
// Overwrites `out`.  Not capturable (it synchronises the stream).
PGB_EXPORT int pgb5_plan_tune(pgb5_plan* P, const void* ipos, const void* jpos, const void* jaux, void* out,
                              void* stream, float* best_ms) {
    return tune_impl(P, ipos, jpos, jaux, nullptr, out, stream, best_ms);
}

// The autotuner of a plan launched with pgb5_plan_launch_indexed (same index list).
PGB_EXPORT int pgb5_plan_tune_indexed(pgb5_plan* P, const void* ipos, const void* jpos, const void* jaux,
                                      const int* jidx, void* out, void* stream, float* best_ms) {
    if (!jidx) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb5_plan_tune_indexed: null index list");
        return -1;
    }
    return tune_impl(P, ipos, jpos, jaux, jidx, out, stream, best_ms);
}

PGB_EXPORT int pgb5_plan_config(const pgb5_plan* P) { return P ? P->cfg : -1; }

// Pin the plan's kernel configuration (0 .. PGB5_NCFG-1; not every one serves every kind) and
// re-stage its work list.
PGB_EXPORT int pgb5_plan_set_config(pgb5_plan* P, int cfg) {
    if (!P || cfg < 0 || cfg >= G5_NCFG || !cfg_valid(P->kind, cfg)) {
        raise(g_err, LIB, PGB_ERR_ARG, "pgb5_plan_set_config: configuration %d not valid for kind %d", cfg,
              P ? P->kind : -1);
        return PGB_ERR_ARG;
    }
    if (!ensure_device()) return PGB_ERR_NOGPU;
    P->cfg = cfg;
    plan_items(P);
    if (!P->L.wait_launched()) return g_err.code ? g_err.code : PGB_ERR_CUDA;
    cudaStream_t s = nullptr;
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && stage_plan(P, s);
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (s) cudaStreamDestroy(s);
    if (!ok) {
        raise(g_err, LIB, PGB_ERR_CUDA, "pgb5_plan_set_config: staging failed");
        return PGB_ERR_CUDA;
    }
    return PGB_OK;
}

PGB_EXPORT void pgb5_plan_destroy(pgb5_plan* P) {
    if (!P) return;
    if (g_device >= 0) {
        cudaSetDevice(g_device);
        cudaDeviceSynchronize();
    }
    P->L.release();
    delete P;
}
