// rt_peak.cu — SIMT arithmetic peaks of the device, measured by a project microbenchmark.
//
// The finest-level operator is matrix free: per node it moves ~70 B and issues ~1000
// thread-instructions, so its bound is the issue rate of the CUDA cores, not HBM.  These
// kernels measure that ceiling on the running device: every thread carries 16 independent
// fused multiply-add chains (enough to hide the FMA pipe latency), one block per
// scheduler slot over a grid of 8 blocks per SM.
//   kind 0: FP32 FFMA          (2 flop per lane-instruction)
//   kind 1: FP32 packed FFMA2  (4 flop per lane-instruction, __ffma2_rn on float2)
//   kind 2: FP64 DFMA          (2 flop per lane-instruction)
#include <cuda_runtime.h>

#include "rt_internal.h"

namespace {

constexpr int PK_CHAINS = 16;
constexpr int PK_BS = 256;

template <int KIND>
__global__ void __launch_bounds__(PK_BS) k_simt_peak(int iters, float seed, double* __restrict__ out) {
    const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (KIND == 0) {
        float a[PK_CHAINS];
        const float b = 0.999f + 1e-6f * seed, c = 1e-3f * seed;
#pragma unroll
        for (int i = 0; i < PK_CHAINS; i++) a[i] = seed + i;
        for (int it = 0; it < iters; it++)
#pragma unroll
            for (int i = 0; i < PK_CHAINS; i++) a[i] = __fmaf_rn(a[i], b, c);
        float s = 0.f;
#pragma unroll
        for (int i = 0; i < PK_CHAINS; i++) s += a[i];
        out[tid] = s;
    } else if (KIND == 1) {
        float2 a[PK_CHAINS];
        const float2 b = make_float2(0.999f + 1e-6f * seed, 0.998f), c = make_float2(1e-3f * seed, 2e-3f);
#pragma unroll
        for (int i = 0; i < PK_CHAINS; i++) a[i] = make_float2(seed + i, seed - i);
        for (int it = 0; it < iters; it++)
#pragma unroll
            for (int i = 0; i < PK_CHAINS; i++) a[i] = __ffma2_rn(a[i], b, c);
        float s = 0.f;
#pragma unroll
        for (int i = 0; i < PK_CHAINS; i++) s += a[i].x + a[i].y;
        out[tid] = s;
    } else {
        double a[PK_CHAINS];
        const double b = 0.999 + 1e-9 * seed, c = 1e-3 * seed;
#pragma unroll
        for (int i = 0; i < PK_CHAINS; i++) a[i] = seed + i;
        for (int it = 0; it < iters; it++)
#pragma unroll
            for (int i = 0; i < PK_CHAINS; i++) a[i] = __fma_rn(a[i], b, c);
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < PK_CHAINS; i++) s += a[i];
        out[tid] = s;
    }
}

}  // namespace

// flop/s of kind (0 FP32 FFMA, 1 FP32 FFMA2, 2 FP64 DFMA): best of reps launches, each about a
// millisecond of device time, CUDA events on the context stream
extern "C" int rt_bench_simt_peak(rt_ctx* c, int kind, int reps, double* tflops) {
    if (!c || kind < 0 || kind > 2 || reps < 1 || !tflops) return RT_EINVAL;
    RT_CUDA(c, cudaSetDevice(c->device));
    const int blocks = c->sm_count * 8;
    const long nthreads = (long)blocks * PK_BS;
    const int iters = kind == 2 ? 2048 : 4096;
    double* out = nullptr;
    RT_CUDA(c, cudaMallocAsync(&out, sizeof(double) * nthreads, c->stream));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    int st = RT_OK;
    for (int r = 0; r <= reps && st == RT_OK; r++) {  // the first launch is a warm-up
        cudaEventRecord(a, c->stream);
        st = rt_launch(c, "simt_peak", [&] {
            switch (kind) {
                case 0: k_simt_peak<0><<<blocks, PK_BS, 0, c->stream>>>(iters, 1.0f + r, out); break;
                case 1: k_simt_peak<1><<<blocks, PK_BS, 0, c->stream>>>(iters, 1.0f + r, out); break;
                default: k_simt_peak<2><<<blocks, PK_BS, 0, c->stream>>>(iters, 1.0f + r, out); break;
            }
        });
        cudaEventRecord(b, c->stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (r > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFreeAsync(out, c->stream);
    RT_CHECK(st);
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    const double flop_per_instr = kind == 1 ? 4.0 : 2.0;
    *tflops = (double)nthreads * iters * PK_CHAINS * flop_per_instr / (best * 1e-3) * 1e-12;
    return RT_OK;
}
