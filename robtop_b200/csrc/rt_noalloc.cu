// rt_noalloc.cu — compliance f.u of caller-owned device vectors without any
// device allocation.
//
// Some callers cannot call cudaMalloc: a host application that hands all
// device memory to its own pool at start-up (so a foreign cudaMalloc fails or
// fragments it), or one that forbids allocation once its time-stepping loop
// runs (cudaMalloc may synchronise the device and stall its other streams).
// rt_compliance needs a hierarchy, and building one allocates; this entry
// point takes the two vectors and the output from the caller and keeps its
// only scratch (the per-block partial sums of the reduction) in a file-scope
// device array of fixed size.
//
// Properties of the scratch array:
//  * RT_NOALLOC_MAX_PARTIALS doubles (512 KiB); every GPU that loads the
//    library holds it until the process exits;
//  * each call writes every slot it reads, so nothing needs clearing, but all
//    calls share the one array: calls that overlap on the GPU (on different
//    streams, or from several host threads without ordering) race;
//  * the device address of the array is looked up once per device, on the
//    first call made while that device is current.  That first call should be
//    made before any stream capture begins.  The address belongs to the
//    device's context, so it is cached together with that context's unique id
//    (cuCtxGetId): after cudaDeviceReset the next call sees a new context id
//    and looks the address up again instead of launching with a stale one;
//  * errors left pending by earlier, unrelated work of the caller are not
//    consumed: the launches are checked with cudaPeekAtLastError before and
//    after, so a sticky error that was already there is reported as RT_ECUDA
//    without being cleared.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "rt_internal.h"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_PER_THREAD = 16;
constexpr long long NA_CHUNK = (long long)NA_THREADS * NA_PER_THREAD;  // elements per partial sum
constexpr int NA_MAX_PARTIALS = RT_NOALLOC_MAX_PARTIALS;
constexpr int NA_MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_partials[NA_MAX_PARTIALS];

std::mutex g_setup_mutex;
double* g_partials_addr[NA_MAX_DEVICES] = {nullptr};
unsigned long long g_partials_ctx[NA_MAX_DEVICES] = {0};  // context id the cached address belongs to

// unique id of the calling thread's current context (0 if none or unknown), through the
// driver entry points the runtime exposes, so the library needs no link against libcuda
unsigned long long current_context_id() {
    using get_current_t = CUresult (*)(CUcontext*);
    using get_id_t = CUresult (*)(CUcontext, unsigned long long*);
    static get_current_t get_current = nullptr;
    static get_id_t get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {  // called with g_setup_mutex held
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess && a)
            get_current = (get_current_t)a;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess && b)
            get_id = (get_id_t)b;
        resolved = true;
    }
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// block b sums a[i] * b[i] over its fixed chunk [b*CHUNK, (b+1)*CHUNK): the
// summation order depends only on n, so repeated calls give identical results
__global__ void __launch_bounds__(NA_THREADS) k_dot_chunks(long long n, const double* __restrict__ a,
                                                           const double* __restrict__ b,
                                                           double* __restrict__ partials) {
    __shared__ double sh[NA_THREADS / 32];
    const long long base = (long long)blockIdx.x * NA_CHUNK;
    double s = 0;
#pragma unroll
    for (int k = 0; k < NA_PER_THREAD; k++) {
        const long long i = base + (long long)k * NA_THREADS + threadIdx.x;
        if (i < n) s += a[i] * b[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < NA_THREADS / 32; w++) t += sh[w];
        partials[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(NA_THREADS) k_sum_partials(int np, const double* __restrict__ partials,
                                                             double* __restrict__ out) {
    __shared__ double sh[NA_THREADS];
    double s = 0;
    for (int i = threadIdx.x; i < np; i += NA_THREADS) s += partials[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = NA_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

}  // namespace

extern "C" int rt_compliance_noalloc(const double* f_dev, const double* u_dev, long long n, double* out_dev,
                                     void* cuda_stream) {
    if (!out_dev || n < 0 || (n > 0 && (!f_dev || !u_dev))) return RT_EINVAL;
    if (n > RT_NOALLOC_MAX_N) {
        fprintf(stderr,
                "rt_compliance_noalloc: n = %lld exceeds the maximum of %lld elements "
                "(%d partial sums of %lld elements each); use rt_compliance instead\n",
                n, (long long)RT_NOALLOC_MAX_N, NA_MAX_PARTIALS, NA_CHUNK);
        return RT_EINVAL;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return RT_ECUDA;
    double* partials = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mutex);
        const unsigned long long id = current_context_id();
        if (g_partials_addr[dev] == nullptr || id == 0 || id != g_partials_ctx[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
            if (e != cudaSuccess) {
                fprintf(stderr, "rt_compliance_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
                g_partials_addr[dev] = nullptr;
                return RT_ECUDA;
            }
            g_partials_addr[dev] = (double*)p;
            // the lookup made the device's context current if it was not yet
            g_partials_ctx[dev] = id ? id : current_context_id();
        }
        partials = g_partials_addr[dev];
    }
    // an error the caller left pending is theirs: report it, leave it in place, launch nothing
    if (cudaPeekAtLastError() != cudaSuccess) return RT_ECUDA;
    cudaStream_t s = (cudaStream_t)cuda_stream;
    const int np = (int)((n + NA_CHUNK - 1) / NA_CHUNK);
    if (np > 0) k_dot_chunks<<<np, NA_THREADS, 0, s>>>(n, f_dev, u_dev, partials);
    k_sum_partials<<<1, NA_THREADS, 0, s>>>(np, partials, out_dev);
    return cudaPeekAtLastError() == cudaSuccess ? RT_OK : RT_ECUDA;
}
