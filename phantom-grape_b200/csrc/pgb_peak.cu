// pgb_peak.cu -- measured throughput ceilings of the two pipes the force kernels run on, for the
// benchmark's roofline (lib/libpgbpeak.so).  Not part of the GRAPE drop-in.
//
//  * FP32 FMA pipe: every thread runs PEAK_CHAINS independent FFMA dependency chains
//    (x = x * a + b), long enough that the launch overhead is negligible; the grid is a whole
//    number of waves of resident CTAs on every SM.  2 flop per FFMA.
//  * MUFU (XU pipe) reciprocal square root: every thread runs PEAK_CHAINS independent chains of
//    rsqrt.approx.ftz.f32 (x = rsqrt(x), which stays in [1, 4) for a start in [1, 4)), the
//    instruction the force kernels use.
//  * The Hermite pair loop's own ceiling: the j-paired inner loop of the force kernel
//    (pgb_g6_kernels.cuh g6_jpair / g6_jquad2, two i per thread, nearest-neighbour tile minimum,
//    FP32 sums folded into FP64 in shared memory every 128 j) over one shared-memory tile staged
//    once, with no j staging, task scheduling or partial rows: what the kernel's arithmetic
//    sustains when nothing else runs.
//  * The accuracy of the rsqrt forms the kernels can be built with (pgb_peak_rsqrt_error).
// Both kernels write one value per thread (so that nothing is optimised away) into a caller
// buffer or a small internal one.  Times are CUDA-event times on the caller's stream.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "pgb_g6_kernels.cuh"

#define PGB_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

constexpr int PEAK_THREADS = 256;
constexpr int PEAK_CHAINS = 8;

__global__ void __launch_bounds__(PEAK_THREADS) ffma_kernel(float* out, int iters, float a, float b) {
    float x[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) x[c] = (float)(threadIdx.x + c) * 1e-3f;
    for (int k = 0; k < iters; k++) {
#pragma unroll
        for (int u = 0; u < 16; u++)
#pragma unroll
            for (int c = 0; c < PEAK_CHAINS; c++) x[c] = __fmaf_rn(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP32 work issued as paired (FFMA2) and scalar (FFMA) instructions in the ratio P : S per
// step, on independent chains: the FMA pipe's throughput for the instruction mixes of the force
// kernels (j-paired Hermite 9 : 18, i-paired 4.5 : 27); 4 flop per FFMA2, 2 per FFMA.
template <int P, int S>
__global__ void __launch_bounds__(PEAK_THREADS) mix_kernel(float* out, int iters, float a, float b) {
    float2 x2[P > 0 ? P : 1];
    float x[S > 0 ? S : 1];
#pragma unroll
    for (int c = 0; c < P; c++) x2[c] = make_float2((float)(threadIdx.x + c) * 1e-3f, (float)c * 1e-3f);
#pragma unroll
    for (int c = 0; c < S; c++) x[c] = (float)(threadIdx.x + 2 * c) * 1e-3f;
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
    for (int k = 0; k < iters; k++) {
#pragma unroll
        for (int u = 0; u < 8; u++) {
#pragma unroll
            for (int c = 0; c < P; c++) x2[c] = __ffma2_rn(x2[c], a2, b2);
#pragma unroll
            for (int c = 0; c < S; c++) x[c] = __fmaf_rn(x[c], a, b);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < P; c++) s += x2[c].x + x2[c].y;
#pragma unroll
    for (int c = 0; c < S; c++) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__global__ void __launch_bounds__(PEAK_THREADS) mufu_kernel(float* out, int iters) {
    float x[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) x[c] = 1.0f + (float)((threadIdx.x + c) & 255) * (1.0f / 128.0f);
    for (int k = 0; k < iters; k++) {
#pragma unroll
        for (int u = 0; u < 16; u++)
#pragma unroll
            for (int c = 0; c < PEAK_CHAINS; c++) x[c] = rsqrt_approx(x[c]);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

constexpr int LOOP_NT = 128;

// Synthetic values in [-1, 1) from a hashed counter (run-time values for every field, so that
// nothing folds at compile time).
__device__ __forceinline__ float hash_unit(unsigned& h) {
    h = h * 1664525u + 1013904223u;
    return (float)(h >> 8) * (1.0f / 8388608.0f) - 1.0f;
}

template <int JP>
__global__ void __launch_bounds__(LOOP_NT) g6_loop_kernel(double* out, int passes, float eps2) {
    __shared__ pgb::G6TileSoA<LOOP_NT> tile;
    __shared__ double Ssh[14 * LOOP_NT];
    const int t = threadIdx.x;
    unsigned h = (blockIdx.x * 977u + t * 7919u + 1u) * 2654435761u;
    tile.xh[t] = hash_unit(h); tile.yh[t] = hash_unit(h); tile.zh[t] = hash_unit(h);
    tile.xl[t] = hash_unit(h) * 1e-8f; tile.yl[t] = hash_unit(h) * 1e-8f; tile.zl[t] = hash_unit(h) * 1e-8f;
    tile.m[t] = 1.0f / 65536; tile.vx[t] = hash_unit(h); tile.vy[t] = hash_unit(h); tile.vz[t] = hash_unit(h);
    tile.id[t] = t;
    pgb::G6IPair IP[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float x = hash_unit(h), y = hash_unit(h), z = hash_unit(h);
        const float lx = hash_unit(h) * 1e-8f, ly = hash_unit(h) * 1e-8f, lz = hash_unit(h) * 1e-8f;
        IP[k].nxh = make_float2(-x, -x); IP[k].nyh = make_float2(-y, -y); IP[k].nzh = make_float2(-z, -z);
        IP[k].nxl = make_float2(-lx, -lx); IP[k].nyl = make_float2(-ly, -ly); IP[k].nzl = make_float2(-lz, -lz);
        IP[k].vx = hash_unit(h); IP[k].vy = hash_unit(h); IP[k].vz = hash_unit(h);
        IP[k].id = -1;
    }
    for (int c = 0; c < 14; c++) Ssh[c * LOOP_NT + t] = 0.0;
    float tmin[2] = {pgb::G6_KEY0, pgb::G6_KEY0};
    __syncthreads();
    for (int p = 0; p < passes; p++) {
        pgb::G6Acc2 a[2];
        const float2 z2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 2; k++) a[k] = pgb::G6Acc2{z2, z2, z2, z2, z2, z2, {0.f, 0.f}};
#pragma unroll 1
        for (int j = 0; j < LOOP_NT; j += 4) {
            const float4 XH = *reinterpret_cast<const float4*>(&tile.xh[j]);
            const float4 YH = *reinterpret_cast<const float4*>(&tile.yh[j]);
            const float4 ZH = *reinterpret_cast<const float4*>(&tile.zh[j]);
            const float4 XL = *reinterpret_cast<const float4*>(&tile.xl[j]);
            const float4 YL = *reinterpret_cast<const float4*>(&tile.yl[j]);
            const float4 ZL = *reinterpret_cast<const float4*>(&tile.zl[j]);
            const float4 M = *reinterpret_cast<const float4*>(&tile.m[j]);
            const float4 VX = *reinterpret_cast<const float4*>(&tile.vx[j]);
            const float4 VY = *reinterpret_cast<const float4*>(&tile.vy[j]);
            const float4 VZ = *reinterpret_cast<const float4*>(&tile.vz[j]);
            const int4 ID = make_int4(0, 0, 0, 0);
            if constexpr (JP == 2) {
                pgb::g6_jquad2<true, false>(XH, YH, ZH, XL, YL, ZL, M, VX, VY, VZ, ID, IP, eps2, a, tmin);
            } else {
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    pgb::g6_jpair<true, false>(make_float2(XH.x, XH.y), make_float2(YH.x, YH.y), make_float2(ZH.x, ZH.y),
                                               make_float2(XL.x, XL.y), make_float2(YL.x, YL.y), make_float2(ZL.x, ZL.y),
                                               make_float2(M.x, M.y), make_float2(VX.x, VX.y), make_float2(VY.x, VY.y),
                                               make_float2(VZ.x, VZ.y), make_int2(ID.x, ID.y), IP[k], eps2, a[k], tmin[k]);
                    pgb::g6_jpair<true, false>(make_float2(XH.z, XH.w), make_float2(YH.z, YH.w), make_float2(ZH.z, ZH.w),
                                               make_float2(XL.z, XL.w), make_float2(YL.z, YL.w), make_float2(ZL.z, ZL.w),
                                               make_float2(M.z, M.w), make_float2(VX.z, VX.w), make_float2(VY.z, VY.w),
                                               make_float2(VZ.z, VZ.w), make_int2(ID.z, ID.w), IP[k], eps2, a[k], tmin[k]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const float2* v = &a[k].ax;
#pragma unroll
            for (int c = 0; c < 6; c++) {
                double& d = Ssh[(k * 7 + c) * LOOP_NT + t];
                d = d + (double)v[c].x + (double)v[c].y;
            }
            double& d = Ssh[(k * 7 + 6) * LOOP_NT + t];
            d = d + (double)a[k].pot[0] + (double)a[k].pot[1];
        }
    }
    double s = (double)tmin[0] + (double)tmin[1];
    for (int c = 0; c < 14; c++) s += Ssh[c * LOOP_NT + t];
    out[blockIdx.x * LOOP_NT + t] = s;
}

// Runs kern `reps` times after one warm-up launch and returns the best launch time (ms), or a
// negative value on a CUDA error.
template <typename L>
float best_ms(L launch, int reps, cudaStream_t s) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -1.f;
    launch();
    float best = 1e30f;
    for (int r = 0; r < reps; r++) {
        cudaEventRecord(e0, s);
        launch();
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            best = -1.f;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaGetLastError() != cudaSuccess) return -1.f;
    return best;
}

int grid_blocks(const void* kern) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PEAK_THREADS, 0);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

}  // namespace

// FP32 FFMA throughput of the current device: *tflops = flops / best launch time (2 flop per
// FFMA), *ms = that time, *blocks = the grid (resident CTAs x SMs).  iters x 16 x 8 FFMA per
// thread.  Returns 0, or -1 on a CUDA error.
PGB_EXPORT int pgb_peak_fp32(int iters, void* stream, double* tflops, double* ms, int* blocks) {
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = grid_blocks((const void*)ffma_kernel);
    float* out = nullptr;
    if (cudaMalloc(&out, (size_t)grid * PEAK_THREADS * sizeof(float)) != cudaSuccess) return -1;
    float t = best_ms([&] { ffma_kernel<<<grid, PEAK_THREADS, 0, s>>>(out, iters, 0.999f, 1e-3f); }, 5, s);
    cudaFree(out);
    if (t <= 0.f) return -1;
    const double flops = 2.0 * grid * PEAK_THREADS * (double)iters * 16 * PEAK_CHAINS;
    if (tflops) *tflops = flops / (t * 1e-3) / 1e12;
    if (ms) *ms = t;
    if (blocks) *blocks = grid;
    return 0;
}

// MUFU rsqrt.approx.ftz.f32 throughput of the current device: *gops = rsqrt per second / 1e9.
PGB_EXPORT int pgb_peak_mufu(int iters, void* stream, double* gops, double* ms, int* blocks) {
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = grid_blocks((const void*)mufu_kernel);
    float* out = nullptr;
    if (cudaMalloc(&out, (size_t)grid * PEAK_THREADS * sizeof(float)) != cudaSuccess) return -1;
    float t = best_ms([&] { mufu_kernel<<<grid, PEAK_THREADS, 0, s>>>(out, iters); }, 5, s);
    cudaFree(out);
    if (t <= 0.f) return -1;
    const double ops = (double)grid * PEAK_THREADS * (double)iters * 16 * PEAK_CHAINS;
    if (gops) *gops = ops / (t * 1e-3) / 1e9;
    if (ms) *ms = t;
    if (blocks) *blocks = grid;
    return 0;
}

// FP32 throughput (TFLOP/s) of a paired : scalar instruction mix, kind 0: paired only (8 FFMA2
// chains), 1: 4 FFMA2 : 8 FFMA (the j-paired Hermite form's 1 : 2), 2: 2 FFMA2 : 12 FFMA (the
// i-paired form's 1 : 6).
PGB_EXPORT int pgb_peak_fp32_mix(int kind, int iters, void* stream, double* tflops, double* ms) {
    cudaStream_t s = (cudaStream_t)stream;
    const void* fn = kind == 0 ? (const void*)mix_kernel<8, 0> : kind == 1 ? (const void*)mix_kernel<4, 8>
                                                                            : (const void*)mix_kernel<2, 12>;
    const int grid = grid_blocks(fn);
    float* out = nullptr;
    if (cudaMalloc(&out, (size_t)grid * PEAK_THREADS * sizeof(float)) != cudaSuccess) return -1;
    float t = best_ms(
        [&] {
            if (kind == 0) mix_kernel<8, 0><<<grid, PEAK_THREADS, 0, s>>>(out, iters, 0.999f, 1e-3f);
            else if (kind == 1) mix_kernel<4, 8><<<grid, PEAK_THREADS, 0, s>>>(out, iters, 0.999f, 1e-3f);
            else mix_kernel<2, 12><<<grid, PEAK_THREADS, 0, s>>>(out, iters, 0.999f, 1e-3f);
        },
        5, s);
    cudaFree(out);
    if (t <= 0.f) return -1;
    const int P = kind == 0 ? 8 : kind == 1 ? 4 : 2, S = kind == 0 ? 0 : kind == 1 ? 8 : 12;
    const double flops = (double)grid * PEAK_THREADS * (double)iters * 8 * (4.0 * P + 2.0 * S);
    if (tflops) *tflops = flops / (t * 1e-3) / 1e12;
    if (ms) *ms = t;
    return 0;
}

// Pair rate of the Hermite force kernel's j-paired inner loop on a resident tile (see the top of
// the file): form 1 = g6_jpair (the autotuner's 128 x 2 j-paired configuration), 2 = g6_jquad2
// (stage-ordered).  `passes` sweeps of the 128-record tile per CTA, the grid a whole wave of
// resident CTAs.  *gpairs = pairs / best launch time / 1e9, *regs = registers per thread.
PGB_EXPORT int pgb_peak_g6_loop(int form, int passes, void* stream, double* gpairs, double* ms, int* regs) {
    cudaStream_t s = (cudaStream_t)stream;
    const void* fn = form == 2 ? (const void*)g6_loop_kernel<2> : (const void*)g6_loop_kernel<1>;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, LOOP_NT, 0);
    if (per_sm < 1) per_sm = 1;
    const int grid = sms * per_sm;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return -1;
    double* out = nullptr;
    if (cudaMalloc(&out, (size_t)grid * LOOP_NT * sizeof(double)) != cudaSuccess) return -1;
    float t = best_ms(
        [&] {
            if (form == 2) g6_loop_kernel<2><<<grid, LOOP_NT, 0, s>>>(out, passes, 1e-8f);
            else g6_loop_kernel<1><<<grid, LOOP_NT, 0, s>>>(out, passes, 1e-8f);
        },
        5, s);
    cudaFree(out);
    if (t <= 0.f) return -1;
    const double pairs = (double)grid * LOOP_NT * 2 * LOOP_NT * passes;
    if (gpairs) *gpairs = pairs / (t * 1e-3) / 1e9;
    if (ms) *ms = t;
    if (regs) *regs = fa.numRegs;
    return 0;
}

// The floor of a small call: `n` launches of an empty kernel (`grid` CTAs of 128 threads) on the
// caller's stream, each waited for before the next -- kind 0: cudaStreamSynchronize; kind 1: the
// kernel sets a flag in mapped host memory (after a system-scope fence) that the host polls, as
// the drop-in API's small calls do.  *us = microseconds per launch (host clock), after 100
// untimed launches.
// Accuracy of the two forms of the scale q = -2/r from the MUFU estimate y = rsqrt.approx(r2)
// (pgb_common.cuh): q = -2 y, the default, and the reference's one Newton step
// q = y (r2 y^2 - 3), each against -2/sqrt(r2) in FP64, for every float r2 in [1, 4) -- two
// binades, one period of the estimate's relative error.  mx[f]: the largest |relative error| of
// form f (the bits of a non-negative double, which order as integers), ss[f]: the sum of squares.
constexpr unsigned RSQ_N = 1u << 24;   // the floats in [1, 4)

__global__ void __launch_bounds__(PEAK_THREADS) rsqrt_err_kernel(unsigned long long* mx, double* ss) {
    double m0 = 0.0, m1 = 0.0, s0 = 0.0, s1 = 0.0;
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < RSQ_N; k += gridDim.x * blockDim.x) {
        const float r2 = __uint_as_float(0x3f800000u + k);
        const float y = pgb::mufu_rsqrt(r2);
        const double ref = -2.0 / sqrt((double)r2);
        const double e0 = fabs(((double)pgb::minus2_mufu(y) - ref) / ref);
        const double e1 = fabs(((double)pgb::minus2_newton(r2, y) - ref) / ref);
        m0 = fmax(m0, e0);
        m1 = fmax(m1, e1);
        s0 += e0 * e0;
        s1 += e1 * e1;
    }
    for (int o = 16; o > 0; o >>= 1) {
        m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&mx[0], (unsigned long long)__double_as_longlong(m0));
        atomicMax(&mx[1], (unsigned long long)__double_as_longlong(m1));
        atomicAdd(&ss[0], s0);
        atomicAdd(&ss[1], s1);
    }
}

__global__ void floor_kernel(volatile unsigned* done, unsigned seq) {
    __syncthreads();
    if (done && threadIdx.x == 0 && blockIdx.x == 0) {
        __threadfence_system();
        done[0] = seq;
    }
}

// max_rel[f], rms_rel[f]: the relative error of q = -2/r over every float r2 in [1, 4), form
// f = 0: -2 y (the default build), f = 1: one Newton step (the lib*_newton.so builds).
PGB_EXPORT int pgb_peak_rsqrt_error(void* stream, double* max_rel, double* rms_rel) {
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long* mx = nullptr;
    double* ss = nullptr;
    if (cudaMalloc(&mx, 2 * sizeof(unsigned long long)) != cudaSuccess) return -1;
    if (cudaMalloc(&ss, 2 * sizeof(double)) != cudaSuccess) {
        cudaFree(mx);
        return -1;
    }
    cudaMemsetAsync(mx, 0, 2 * sizeof(unsigned long long), s);
    cudaMemsetAsync(ss, 0, 2 * sizeof(double), s);
    rsqrt_err_kernel<<<4 * 148, PEAK_THREADS, 0, s>>>(mx, ss);
    unsigned long long hm[2] = {0, 0};
    double hs[2] = {0, 0};
    cudaMemcpyAsync(hm, mx, sizeof hm, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hs, ss, sizeof hs, cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(mx);
    cudaFree(ss);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return -1;
    for (int f = 0; f < 2; f++) {
        double m;
        std::memcpy(&m, &hm[f], sizeof m);
        if (max_rel) max_rel[f] = m;
        if (rms_rel) rms_rel[f] = std::sqrt(hs[f] / RSQ_N);
    }
    return 0;
}

PGB_EXPORT int pgb_peak_launch_floor(int kind, int grid, int n, void* stream, double* us) {
    cudaStream_t s = (cudaStream_t)stream;
    unsigned* hflag = nullptr;
    unsigned* dflag = nullptr;
    if (kind == 1) {
        if (cudaHostAlloc((void**)&hflag, 64, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) return -1;
        if (cudaHostGetDevicePointer((void**)&dflag, hflag, 0) != cudaSuccess) return -1;
        hflag[0] = 0;
    }
    auto one = [&](unsigned seq) {
        if (kind == 1) {
            floor_kernel<<<grid, 128, 0, s>>>(dflag, seq);
            // bounded: a launch that never signals ends the measurement with an error
            for (long it = 0; ((volatile unsigned*)hflag)[0] != seq; it++)
                if (it > (1L << 30)) return false;
        } else {
            floor_kernel<<<grid, 128, 0, s>>>(nullptr, seq);
            if (cudaStreamSynchronize(s) != cudaSuccess) return false;
        }
        return true;
    };
    unsigned seq = 1;
    bool ok = true;
    for (int k = 0; k < 100 && ok; k++) ok = one(seq++);
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < n && ok; k++) ok = one(seq++);
    const auto t1 = std::chrono::steady_clock::now();
    cudaStreamSynchronize(s);
    if (hflag) cudaFreeHost(hflag);
    if (!ok || cudaGetLastError() != cudaSuccess) return -1;
    if (us) *us = std::chrono::duration<double, std::micro>(t1 - t0).count() / n;
    return 0;
}
