// Arithmetic-throughput probes: the compute ceilings of the direct sums measured
// on the device itself (FP32 FMA scalar and packed, MUFU reciprocal square root,
// FP64 FMA, FP64 tensor-core MMA, FP32 -> bf16x2 conversion). Every thread runs kChains independent dependency
// chains of one operation for `iters` steps over a grid of several CTAs per SM, so
// the issue and pipe rates, not latencies, set the time. The results are written
// to a scratch buffer so the compiler keeps every chain.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "solver.h"

namespace bie {
namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;
constexpr int kCtasPerSm = 8;

__global__ void __launch_bounds__(kThreads) k_probe_ffma(float* out, int iters, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3f + c;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_probe_ffma2(float* out, int iters, float a, float b) {
    uint64_t x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = pk2(threadIdx.x * 1e-3f + c, c * 0.5f);
    const uint64_t a2 = pk2(a, a), b2 = pk2(b, b);
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma2(x[c], a2, b2);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
        const float2 v = upk2(x[c]);
        s += v.x + v.y;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_probe_mufu(float* out, int iters, float a, float) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = a + threadIdx.x * 1e-3f + c;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = rsqrt_approx(x[c]);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_probe_dfma(float* out, int iters, float a, float b) {
    double x[kChains];
    const double ad = a, bd = b;
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3 + c;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], ad, bd);
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = (float)s;
}

__global__ void __launch_bounds__(kThreads) k_probe_dmma(float* out, int iters, float a, float b) {
    double d[kChains][2];
#pragma unroll
    for (int c = 0; c < kChains; ++c) d[c][0] = d[c][1] = 0.0;
    const double av = a * (1.0 + threadIdx.x * 1e-6), bv = b;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                         : "+d"(d[c][0]), "+d"(d[c][1])
                         : "d"(av), "d"(bv));
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += d[c][0] + d[c][1];
    out[blockIdx.x * blockDim.x + threadIdx.x] = (float)s;
}

// FP64 MMA and FP64 FMA at once: even warps run the MMA chains of k_probe_dmma, odd
// warps the FMA chains of k_probe_dfma (iters_fma steps), to see whether the two share
// throughput.
__global__ void __launch_bounds__(kThreads) k_probe_dmma_dfma(float* out, int iters, int iters_fma, float a,
                                                              float b) {
    double s = 0.0;
    if (((threadIdx.x >> 5) & 1) == 0) {
        double d[kChains][2];
#pragma unroll
        for (int c = 0; c < kChains; ++c) d[c][0] = d[c][1] = 0.0;
        const double av = a * (1.0 + threadIdx.x * 1e-6), bv = b;
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int c = 0; c < kChains; ++c)
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                             : "+d"(d[c][0]), "+d"(d[c][1])
                             : "d"(av), "d"(bv));
#pragma unroll
        for (int c = 0; c < kChains; ++c) s += d[c][0] + d[c][1];
    } else {
        double x[kChains];
        const double ad = a, bd = b;
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3 + c;
        for (int it = 0; it < iters_fma; ++it)
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], ad, bd);
#pragma unroll
        for (int c = 0; c < kChains; ++c) s += x[c];
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = (float)s;
}

// FP32 pair -> packed bf16x2 conversion (round to nearest), the split step of the
// tensor-core direct sum; the rounded pair is fed back as the next input.
__global__ void __launch_bounds__(kThreads) k_probe_cvt_bf16x2(float* out, int iters, float a, float) {
    uint32_t w[kChains];
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = a + threadIdx.x * 1e-3f + c;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(w[c]) : "f"(x[c]), "f"(x[c]));
            x[c] = __uint_as_float(w[c]);  // the packed word read as FP32: a dependent input
        }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Latency of dependent operations: one warp runs a single chain of `iters` FP64 MMAs
// (lat_op 0) or FP64 FMAs (lat_op 1) and records the SM cycles it took.
__global__ void k_probe_latency(long long* cycles, int iters, int lat_op, double a, double b) {
    double d0 = 0.0, d1 = 0.0, x = threadIdx.x * 1e-3;
    const long long t0 = clock64();
    if (lat_op == 0) {
        for (int it = 0; it < iters; ++it)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                         : "+d"(d0), "+d"(d1)
                         : "d"(a), "d"(b));
    } else {
        for (int it = 0; it < iters; ++it) x = fma(x, a, b);
    }
    const long long t1 = clock64();
    if (threadIdx.x == 0) cycles[0] = t1 - t0;
    if (d0 + d1 + x == -1.0) cycles[1] = 1;  // keeps the chains
}

}  // namespace

void peak_probe(int device, int which, double* per_second, double* ms_out) {
    if (which < 0 || which > 8) throw Error(BIE_EINVAL, "peak_probe: which must be 0 .. 8");
    int prev = 0;
    BIE_CK(cudaGetDevice(&prev));
    BIE_CK(cudaSetDevice(device));
    int sms = 0;
    BIE_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int ctas = sms * kCtasPerSm;
    float* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&] {
        if (out) cudaFree(out);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaSetDevice(prev);
    };
    try {
        BIE_CK(cudaMalloc(&out, sizeof(float) * (size_t)ctas * kThreads));
        BIE_CK(cudaEventCreate(&e0));
        BIE_CK(cudaEventCreate(&e1));
        // steps per thread: about 10 ms per probe at the expected rates
        const int iters = which == 4 ? 2048 : (which == 3 ? 8192 : (which == 2 || which == 5 ? 16384 : 65536));
        if (which == 8) {
            // half the warps on each: the same per-warp work as probes 4 and 3, so with
            // separate pipes the launch takes about as long as the slower half alone
            const int it4 = 2048 / 2, it3 = 8192 / 2;
            auto mixed = [&] {
                k_probe_dmma_dfma<<<ctas, kThreads>>>(out, it4, it3, 0.999f, 1e-3f);
                BIE_CK(cudaGetLastError());
            };
            mixed();
            BIE_CK(cudaEventRecord(e0));
            mixed();
            BIE_CK(cudaEventRecord(e1));
            BIE_CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            BIE_CK(cudaEventElapsedTime(&ms, e0, e1));
            const double half = (double)ctas * kThreads / 2.0;
            // reported: MMA flop/s of the even warps (the FMA lane rate follows from ms)
            *per_second = half / 32.0 * kChains * (double)it4 * 512.0 / (ms * 1e-3);
            *ms_out = ms;
            cleanup();
            return;
        }
        if (which >= 6) {
            // dependent-chain latency in SM cycles per operation (one warp)
            const int n = 4096;
            long long* cyc = reinterpret_cast<long long*>(out);
            k_probe_latency<<<1, 32>>>(cyc, n, which - 6, 0.999, 1e-3);
            BIE_CK(cudaGetLastError());
            k_probe_latency<<<1, 32>>>(cyc, n, which - 6, 0.999, 1e-3);
            BIE_CK(cudaGetLastError());
            long long c = 0;
            BIE_CK(cudaMemcpy(&c, cyc, sizeof(c), cudaMemcpyDeviceToHost));
            *per_second = (double)c / n;
            *ms_out = 0.0;
            cleanup();
            return;
        }
        auto launch = [&] {
            switch (which) {
                case 0: k_probe_ffma<<<ctas, kThreads>>>(out, iters, 0.999f, 1e-3f); break;
                case 1: k_probe_ffma2<<<ctas, kThreads>>>(out, iters, 0.999f, 1e-3f); break;
                case 2: k_probe_mufu<<<ctas, kThreads>>>(out, iters, 1.5f, 0.f); break;
                case 3: k_probe_dfma<<<ctas, kThreads>>>(out, iters, 0.999f, 1e-3f); break;
                case 5: k_probe_cvt_bf16x2<<<ctas, kThreads>>>(out, iters, 1.5f, 0.f); break;
                default: k_probe_dmma<<<ctas, kThreads>>>(out, iters, 0.999f, 1e-3f); break;
            }
            BIE_CK(cudaGetLastError());
        };
        launch();  // warm-up
        BIE_CK(cudaEventRecord(e0));
        launch();
        BIE_CK(cudaEventRecord(e1));
        BIE_CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        BIE_CK(cudaEventElapsedTime(&ms, e0, e1));
        const double threads = (double)ctas * kThreads;
        double ops = threads * kChains * (double)iters;  // lane operations
        if (which == 1) ops *= 2.0;                       // two FMAs per packed lane operation
        if (which == 4) ops = threads / 32.0 * kChains * (double)iters * 512.0;  // flops of m8n8k4
        *per_second = ops / (ms * 1e-3);
        *ms_out = ms;
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
}

}  // namespace bie
