// pgb_common.cuh -- shared host/device plumbing of the B200 force engine.
//
// * error recording: every C-ABI entry point records failures in a per-library error slot
//   (message + code) that `<lib>_last_error()` returns; by default a hard error (CUDA failure,
//   capacity overflow, ni > pipelines) also prints and aborts, which is what the reference's
//   assert() does (e.g. PG5/newton/libpg5/phantom_g5.c:77,105,246).
// * device buffers that grow on demand, pinned host staging buffers.
// * the work-list types shared by all kernels: a Task is one (i-tile, j-chunk) pair, a Group
//   collects the tasks whose partial sums are reduced, in chunk order, by the last CTA that
//   finishes one of them (deterministic; no second launch).
// * the MUFU reciprocal square root (PTX rsqrt.approx.ftz.f32) and the scale q = -2/r used by
//   every kernel: q = -2 y by default, or -- built with PGB_RSQRT_NEWTON -- the reference's
//   one-Newton-step form q = y (r2 y^2 - 3) ("rsqrt_1st_phantom", PG6/libpg6/gravity.c:341-346).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#define PGB_EXPORT extern "C" __attribute__((visibility("default")))

namespace pgb {

// ------------------------------------------------------------------------------------------
// errors

enum Status : int {
    PGB_OK = 0,
    PGB_ERR_CUDA = 1,       // a CUDA runtime call failed
    PGB_ERR_ARG = 2,        // bad argument (ni > pipelines, negative sizes, ...)
    PGB_ERR_CAPACITY = 3,   // j-memory / work-list capacity exceeded
    PGB_ERR_DEVICE = 4,     // the kernel reported an error word (bounded wait expired, ...)
    PGB_ERR_NOGPU = 5,      // no CUDA device
};

struct ErrorSlot {
    std::mutex mu;
    int code = 0;
    std::string msg;
    int abort_on_error = -1;  // -1: read PGB_NOABORT once
};

inline bool abort_enabled(ErrorSlot& e) {
    if (e.abort_on_error < 0) {
        const char* s = std::getenv("PGB_NOABORT");
        e.abort_on_error = (s && s[0] == '1') ? 0 : 1;
    }
    return e.abort_on_error == 1;
}

inline void raise(ErrorSlot& e, const char* lib, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    bool ab;
    {
        std::lock_guard<std::mutex> g(e.mu);
        e.code = code;
        e.msg = std::string(lib) + ": " + buf;
        ab = abort_enabled(e);
    }
    std::fprintf(stderr, "%s: error %d: %s\n", lib, code, buf);
    if (ab) std::abort();
}

#define PGB_CUDA_OR(slot, lib, call, onerr)                                                  \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess) {                                                             \
            ::pgb::raise(slot, lib, ::pgb::PGB_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
                         cudaGetErrorString(_e), __FILE__, __LINE__);                        \
            onerr;                                                                           \
        }                                                                                    \
    } while (0)

// ------------------------------------------------------------------------------------------
// buffers

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t want) {
        if (want <= n) return cudaSuccess;
        size_t m = n ? n : 256;
        while (m < want) m *= 2;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, m * sizeof(T));
        if (e == cudaSuccess) n = m;
        return e;
    }
    // grow while keeping the first `keep` elements (device-to-device copy)
    cudaError_t grow_keep(size_t want, size_t keep, cudaStream_t s) {
        if (want <= n) return cudaSuccess;
        size_t m = n ? n : 256;
        while (m < want) m *= 2;
        T* q = nullptr;
        cudaError_t e = cudaMalloc(&q, m * sizeof(T));
        if (e != cudaSuccess) return e;
        if (p && keep) {
            e = cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        }
        if (p) cudaFree(p);
        p = q;
        n = m;
        return e;
    }
    cudaError_t zero_fill(cudaStream_t s) {
        return n ? cudaMemsetAsync(p, 0, n * sizeof(T), s) : cudaSuccess;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

template <class T>
struct HostBuf {
    T* p = nullptr;
    size_t n = 0;
    // flags: cudaHostAllocMapped for a buffer that kernels write through its device address
    cudaError_t reserve(size_t want, bool keep = false, unsigned flags = cudaHostAllocPortable) {
        if (want <= n) return cudaSuccess;
        size_t m = n ? n : 256;
        while (m < want) m *= 2;
        T* q = nullptr;
        cudaError_t e = cudaHostAlloc(&q, m * sizeof(T), flags);
        if (e != cudaSuccess) return e;
        if (keep && p) std::memcpy(q, p, n * sizeof(T));
        if (p) cudaFreeHost(p);
        p = q;
        n = m;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
};

// ------------------------------------------------------------------------------------------
// work lists

// One unit of work for one CTA: i-particles [i0, i0+ni) against j-records [j0, j0+nj).
// `group` < 0: the task owns its i-particles outright and writes the final result.
// `group` >= 0: the task is chunk `chunk` of a split j-range; it writes its partial sums to
// partial row `slot` and the last finisher of the group reduces the rows in chunk order.
struct Task {
    int i0, ni, j0, nj;
    int group, chunk, slot, aux;
};

struct Group {
    int i0, ni;      // the i-particles the group's tasks share
    int nchunk;      // number of tasks (partial rows) in the group
    int slot0;       // first partial row; rows slot0 .. slot0+nchunk-1 in chunk order
};

// Number of j-chunks for one item of `itiles` equal i-tiles on `slots` resident CTAs: the
// persistent CTAs run ceil(itiles*nch/slots) waves of tasks of nj/nch pairs per i, so the time
// is proportional to waves/nch; a small penalty per chunk accounts for the partial-row
// reduction.  Chunks hold at least `minj` j and there are at most `maxch` of them.
inline int best_nch(long long itiles, long long nj, long long slots, int maxch, int minj = 128) {
    long long hi = nj / minj;
    if (hi > maxch) hi = maxch;
    if (hi < 1) return 1;
    double best = 1e300;
    int arg = 1;
    for (long long n = 1; n <= hi; n++) {
        long long waves = (itiles * n + slots - 1) / slots;
        double cost = (double)waves / (double)n * (1.0 + 0.002 * (double)n);
        if (cost < best) {
            best = cost;
            arg = (int)n;
        }
    }
    return arg;
}

// Split [0,ni) x [0,nj) into tasks of at most `itile` i and about `jchunk` j, appending to
// `tasks`/`groups`.  Offsets are added to i0/j0.  Returns the partial rows used.
inline int plan_item(std::vector<Task>& tasks, std::vector<Group>& groups, int i_off, int ni,
                     int j_off, int nj, int itile, int jchunk, int slot_base, int aux = 0) {
    if (ni <= 0) return 0;
    int nch = (nj + jchunk - 1) / jchunk;
    if (nch < 1) nch = 1;
    int used = 0;
    for (int it = 0; it < ni; it += itile) {
        int nii = ni - it < itile ? ni - it : itile;
        if (nch == 1) {
            tasks.push_back(Task{i_off + it, nii, j_off, nj, -1, 0, -1, aux});
            continue;
        }
        int g = (int)groups.size();
        groups.push_back(Group{i_off + it, nii, nch, slot_base + used});
        // near-equal chunks, each a multiple of 32 j where possible
        long long base = (long long)nj / nch;
        int rem = nj - (int)(base * nch);
        int j = 0;
        for (int c = 0; c < nch; c++) {
            int len = (int)base + (c < rem ? 1 : 0);
            tasks.push_back(Task{i_off + it, nii, j_off + j, len, g, c, slot_base + used + c, aux});
            j += len;
        }
        used += nch;
    }
    return used;
}


// ------------------------------------------------------------------------------------------
// Staging of one launch: the work list (+ optionally host i-records) is packed into pinned
// memory and copied to the device in one transfer; the device block is
//   [task counter (16 B) | tasks | groups | i-records].
// Partial rows (ORec x itile each) and group counters live beside it.
template <class IRec, class ORec>
struct Stager {
    DevBuf<unsigned char> dcall;
    DevBuf<int> dgcnt;             // group counters (zero at allocation, self-cleaning)
    DevBuf<ORec> dpart;            // partial rows, [rows][itile]
    HostBuf<unsigned char> hcall;  // pinned staging of the call block
    cudaEvent_t copied = nullptr;  // last H2D copy out of hcall
    size_t off_g = 0, off_i = 0, off_bc = 0;
    int ntasks = 0;

    cudaError_t stage(cudaStream_t s, const std::vector<Task>& tasks, const std::vector<Group>& groups, int rows,
                      int itile, const IRec* i_host, int ni_host, size_t min_groups = 0) {
        cudaError_t e;
        if (!copied && (e = cudaEventCreateWithFlags(&copied, cudaEventDisableTiming)) != cudaSuccess) return e;
        // the previous copy out of hcall must have left before hcall is rewritten
        if ((e = cudaEventSynchronize(copied)) != cudaSuccess) return e;
        const size_t off_t = 16;
        off_g = (off_t + tasks.size() * sizeof(Task) + 15) & ~size_t(15);
        off_i = (off_g + groups.size() * sizeof(Group) + 15) & ~size_t(15);
        size_t total = off_i + (size_t)ni_host * sizeof(IRec);
        if ((e = hcall.reserve(total)) != cudaSuccess) return e;
        if ((e = dcall.reserve(total)) != cudaSuccess) return e;
        std::memset(hcall.p, 0, 16);
        if (!tasks.empty()) std::memcpy(hcall.p + off_t, tasks.data(), tasks.size() * sizeof(Task));
        if (!groups.empty()) std::memcpy(hcall.p + off_g, groups.data(), groups.size() * sizeof(Group));
        if (ni_host) std::memcpy(hcall.p + off_i, i_host, (size_t)ni_host * sizeof(IRec));
        if ((e = reserve_scratch(s, rows, itile, std::max(groups.size(), min_groups))) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(dcall.p, hcall.p, total, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(copied, s)) != cudaSuccess) return e;
        ntasks = (int)tasks.size();
        return cudaSuccess;
    }
    // Partial rows and zeroed counters: one per group (`ngroups` includes groups that the
    // kernel derives itself, regular mode), then one per partial row for the two-level
    // reduction of long groups.  Enough for a launch that uploads nothing.
    cudaError_t reserve_scratch(cudaStream_t s, int rows, int itile, size_t ngroups) {
        cudaError_t e;
        off_bc = ngroups;
        const size_t old = dgcnt.n;
        if ((e = dgcnt.reserve(off_bc + (size_t)rows + 1)) != cudaSuccess) return e;
        if (dgcnt.n != old && (e = dgcnt.zero_fill(s)) != cudaSuccess) return e;
        if (rows > 0 && (e = dpart.reserve((size_t)rows * itile)) != cudaSuccess) return e;
        return cudaSuccess;
    }
    int* counter() const { return (int*)dcall.p; }
    const Task* tasks() const { return (const Task*)(dcall.p + 16); }
    const Group* groups() const { return (const Group*)(dcall.p + off_g); }
    const IRec* irecs() const { return (const IRec*)(dcall.p + off_i); }
    int* bundle_counters() const { return dgcnt.p + off_bc; }
    void release() {
        if (copied) cudaEventSynchronize(copied);
        dcall.release();
        dgcnt.release();
        dpart.release();
        hcall.release();
        if (copied) cudaEventDestroy(copied);
        copied = nullptr;
        ntasks = 0;
    }
};

// ------------------------------------------------------------------------------------------
// device helpers

__device__ __forceinline__ float mufu_rsqrt(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// q = -2/r from y = rsqrt.approx(r2).  By default q = -2 y: sm_100's MUFU estimate is already
// accurate to about an ulp, so a Newton step only adds rounding (and three FP32 operations per
// pair).  Built with PGB_RSQRT_NEWTON (the lib*_newton.so libraries), the reference's form: one
// Newton step folded into the scale, q = y (r2 y^2 - 3), which the AVX code needs to refine its
// 12-bit estimate.  Every operation is an explicit round-to-nearest intrinsic, so that the key
// is the same bit pattern wherever it is computed (the nearest-neighbour search recomputes it,
// see g6_task).
__device__ __forceinline__ float minus2_mufu(float y) { return __fmul_rn(-2.0f, y); }

__device__ __forceinline__ float minus2_newton(float r2, float y) {
    const float t = __fmul_rn(r2, y);
    const float u = __fmaf_rn(t, y, -3.0f);
    return __fmul_rn(u, y);
}

__device__ __forceinline__ float minus2_from_rsqrt(float r2, float y) {
#ifdef PGB_RSQRT_NEWTON
    return minus2_newton(r2, y);
#else
    (void)r2;
    return minus2_mufu(y);
#endif
}

__device__ __forceinline__ float minus2_over_r(float r2) { return minus2_from_rsqrt(r2, mufu_rsqrt(r2)); }

// The pair scale.  Every kernel forms its pair terms from one scale s of 1/r and removes the
// scale with FP64 constants where the sums are finished.  By default s = y, the MUFU estimate
// itself (no operation after the rsqrt); built with PGB_RSQRT_NEWTON, s = q = -2/r in the
// reference's Newton-refined form.  Every term is a product of powers of s, so the default's
// terms are those of s = -2 y (the MUFU estimate in the reference's scale) times exact powers
// of two, and the finished results are the same bit for bit.
//   PG6: pot = S_POT sum m s,  acc = S_ACC sum m s^3 dx,
//        jerk = S_ACC sum m s^3 (dv + S_JERK s^2 (dx.dv) dx)
//   PG5: pot_raw = S_POT sum m s (= -sum m/r),  acc = S_ACC sum m s^3 dx
// Nearest-neighbour key: k = nn_key(s), smaller is nearer; reported as q = -2/r_soft =
// key_out(k) = KEY_OUT k.
#ifdef PGB_RSQRT_NEWTON
constexpr double S_POT = 0.5, S_ACC = -0.125;
constexpr float S_JERK = -0.75f, KEY_OUT = 1.0f;
__device__ __forceinline__ float pair_scale_from_rsqrt(float r2, float y) { return minus2_newton(r2, y); }
__device__ __forceinline__ float nn_key(float s) { return s; }
#else
constexpr double S_POT = -1.0, S_ACC = 1.0;
constexpr float S_JERK = -3.0f, KEY_OUT = 2.0f;
__device__ __forceinline__ float pair_scale_from_rsqrt(float, float y) { return y; }
// -y: the negation is an operand modifier of the compare or min that consumes it
__device__ __forceinline__ float nn_key(float s) { return -s; }
#endif
__device__ __forceinline__ float pair_scale(float r2) { return pair_scale_from_rsqrt(r2, mufu_rsqrt(r2)); }
// KEY_OUT k, with a self-only key's -0 reported as +0 (the key of s = 0)
__device__ __forceinline__ float key_out(float k) { return __fmaf_rn(KEY_OUT, k, 0.0f); }
// a key as reported back to the kernels' scale (exact)
__device__ __forceinline__ float key_in(float q) { return q * (1.0f / KEY_OUT); }

// The persistent scheduler.  A CTA's first task is its block index; later ones are drawn from
// a global counter as gridDim.x + k.  Every CTA draws until it gets a task >= ntasks, so a
// launch draws exactly ntasks times (the ntasks - min(grid, ntasks) extra tasks plus one failed
// draw per working CTA) and the CTA that draws k = ntasks - 1 is the last to touch the counter:
// it resets it to zero, so the counter is ready for the next launch without a memset.
// `first` skips the barrier too: callers that stage shared memory before the loop sync first.
__device__ __forceinline__ int next_task(int* counter, int* s_slot, int ntasks, bool first) {
    if (first) return (int)blockIdx.x;
    __syncthreads();
    if (threadIdx.x == 0) {
        const int k = atomicAdd(counter, 1);
        if (k == ntasks - 1) atomicExch(counter, 0);
        *s_slot = (int)gridDim.x + k;
    }
    __syncthreads();
    return *s_slot;
}

// Called by every thread of the CTA after it wrote its partial row: returns true in all
// threads of the CTA that finished the group last (the one that must reduce it).
__device__ __forceinline__ bool group_arrive(int* counters, int group, int nchunk, int* s_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        int prev = atomicAdd(&counters[group], 1);
        int last = (prev == nchunk - 1);
        if (last) counters[group] = 0;  // self-clean for the next launch
        *s_flag = last;
    }
    __syncthreads();
    bool last = *s_flag != 0;
    if (last) __threadfence();
    return last;
}

// SM count of the current device (cached per device)
inline int sm_count(int dev) {
    static int cache[64] = {0};
    if (dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = v > 0 ? v : 148;
    }
    return cache[dev];
}

}  // namespace pgb
