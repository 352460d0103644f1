// rt_unet_kernels.cu — kernels of the learned preconditioner (3D U-Net, BF16 activations,
// FP32 accumulation).  There is no reference counterpart; the network is specified by
// its channel plan (16/32/48/64, 3x3x3 convolutions, four levels).
//
// Activations are channels-last [voxel][C] (x fastest over voxels), C a multiple of 16,
// with a row stride so that an encoder output can live inside its decoder concat buffer.
//
// k_conv3_tc: 3x3x3 convolution (zero padding 1) as an implicit GEMM on the 5th-gen
// tensor cores: D[128 voxels x Cout] in TMEM += A[128 x Cin] * B[Cout x Cin]^T for each
// of the 27 taps; A rows are the tap-shifted input voxels, gathered into shared memory
// in the K-major no-swizzle core-matrix layout, B the tap's weights; one thread issues
// tcgen05.mma, two shared-memory stages overlap the next tap's gather with the MMAs.
// The same kernel computes the input gradient with the tap-flipped, transposed weights.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "rt_internal.h"
#include "rt_tc.cuh"
#include "rt_unet.h"

namespace rtu {

constexpr int CONV_TM = 128;
constexpr int CONV_THREADS = 128;

__global__ void __launch_bounds__(CONV_THREADS) k_conv3_tc(ConvArgs a) {
    extern __shared__ __align__(128) uint8_t sm[];
    const int cin = a.cin, cout = a.cout;
    const uint32_t a_bytes = CONV_TM * cin * 2, b_bytes = cout * cin * 2;
    uint8_t* sA[2] = {sm, sm + a_bytes};
    uint8_t* sB[2] = {sm + 2 * a_bytes, sm + 2 * a_bytes + b_bytes};
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * a_bytes + 2 * b_bytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5;
    const long V = (long)a.X * a.Y * a.Z;
    const long m = (long)blockIdx.x * CONV_TM + tid;  // this thread's A row / TMEM lane / output voxel
    const uint32_t ncols = rttc::tmem_cols(cout);
    if (tid == 0) {
        rttc::mbar_init(&bar[0], 1);
        rttc::mbar_init(&bar[1], 1);
        rttc::fence_mbar_init();
    }
    if (warp == 0) rttc::tmem_alloc(tslot, ncols);
    rttc::tc_fence_before();
    __syncthreads();
    rttc::tc_fence_after();
    const uint32_t tmem = *tslot;
    int x = 0, y = 0, z = 0;
    const bool mv = m < V;
    if (mv) {
        x = (int)(m % a.X);
        y = (int)((m / a.X) % a.Y);
        z = (int)(m / ((long)a.X * a.Y));
    }
    const int kch = cin / 8;  // 16-byte chunks of a row
    const uint32_t lboA = (CONV_TM / 8) * 128, lboB = (uint32_t)(cout / 8) * 128;
    const uint32_t idesc = rttc::idesc_bf16(CONV_TM, cout, 0, 0);
    int last = -1;  // last tap whose MMAs were committed
    bool ok = true;
    for (int t = 0; t < 27; t++) {
        const int b = t & 1;
        if (t >= 2) {
            const bool w = rttc::mbar_wait(&bar[b], ((t - 2) >> 1) & 1);
            if (!__syncthreads_and(w)) {  // the MMAs reading this stage never finished
                ok = false;
                break;
            }
        }
        const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
        const int xn = x + dx, yn = y + dy, zn = z + dz;
        const bool inb = mv && xn >= 0 && xn < a.X && yn >= 0 && yn < a.Y && zn >= 0 && zn < a.Z;
        const uint4* src = reinterpret_cast<const uint4*>(
            a.in + (inb ? ((long)xn + (long)a.X * (yn + (long)a.Y * zn)) * a.in_stride : 0));
        uint8_t* dA = sA[b] + (tid >> 3) * 128 + (tid & 7) * 16;
        for (int j = 0; j < kch; j++) {
            const uint4 v = inb ? __ldg(src + j) : make_uint4(0u, 0u, 0u, 0u);
            *reinterpret_cast<uint4*>(dA + j * lboA) = v;
        }
        for (int idx = tid; idx < cout * kch; idx += CONV_THREADS) {
            const int n = idx / kch, j = idx - n * kch;
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(a.w + ((long)n * 27 + t) * cin) + j);
            *reinterpret_cast<uint4*>(sB[b] + j * lboB + (n >> 3) * 128 + (n & 7) * 16) = v;
        }
        rttc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            rttc::tc_fence_after();
            const uint32_t a0 = rttc::smem_u32(sA[b]), b0 = rttc::smem_u32(sB[b]);
            for (int kk = 0; kk < cin / 16; kk++) {
                const uint64_t ad = rttc::sdesc(a0 + 2 * kk * lboA, lboA, 128);
                const uint64_t bd = rttc::sdesc(b0 + 2 * kk * lboB, lboB, 128);
                rttc::mma_bf16(tmem, ad, bd, idesc, (t > 0 || kk > 0) ? 1u : 0u);
            }
            rttc::mma_commit(&bar[b]);
        }
        last = t;
    }
    // all MMAs done (the last commit covers every earlier MMA of the issuing thread)
    bool done = true;
    if (last >= 0) done = rttc::mbar_wait(&bar[last & 1], (last >> 1) & 1);
    done = __syncthreads_and(done) != 0;
    if (!ok || !done) {
        if (tid == 0 && a.err) atomicExch(a.err, 1);
    } else {
        rttc::tc_fence_after();
        for (int c0 = 0; c0 < cout; c0 += 16) {
            float v[16];
            rttc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (mv) {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    float s = v[i] + (a.bias ? a.bias[c0 + i] : 0.f);
                    v[i] = a.relu ? fmaxf(s, 0.f) : s;
                }
                if (a.out_f32) {
                    float4* o = reinterpret_cast<float4*>(reinterpret_cast<float*>(a.out) + m * a.out_stride + c0);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        float4 val = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                        if (a.accumulate) {
                            const float4 old = o[q];
                            val.x += old.x; val.y += old.y; val.z += old.z; val.w += old.w;
                        }
                        o[q] = val;
                    }
                } else {
                    __align__(16) __nv_bfloat162 pk[8];
#pragma unroll
                    for (int q = 0; q < 8; q++) pk[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                    uint4* o = reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(a.out) + m * a.out_stride + c0);
                    o[0] = *reinterpret_cast<const uint4*>(&pk[0]);
                    o[1] = *reinterpret_cast<const uint4*>(&pk[4]);
                }
            }
        }
    }
    rttc::tc_fence_before();
    __syncthreads();
    if (warp == 0) rttc::tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// k_conv3_halo: the same convolution with the input read once per CTA.  A CTA owns an
// 8 x 16 voxel patch over P consecutive z-planes; the patch's (P+2) x 18 x 10 halo is copied
// into shared memory as [16-byte channel chunk][plane][y][x], which is the no-swizzle K-major
// core-matrix layout of every tap's A operand at once: row m = x + 8 y of the patch is 16 B
// after row m-1 within a patch row (8-row core matrix) and 160 B (one halo row) further per
// patch row (SBO), the next channel chunk is one chunk plane further (LBO), and a tap
// (dx, dy, dz) only moves the descriptor's start address.  Taps run outer: a tap's weights
// are loaded once (two stages) and applied to all P planes, whose accumulators sit side by
// side in TMEM (P x Cout columns).
// ---------------------------------------------------------------------------
constexpr int HALO_X = 10, HALO_Y = 18, HALO_V = HALO_X * HALO_Y;

__global__ void __launch_bounds__(CONV_THREADS) k_conv3_halo(ConvArgs a, int P, int G) {
    extern __shared__ __align__(128) uint8_t sm[];
    const int cin = a.cin, cout = a.cout, kch = cin / 8, npl = P + 2;
    const int ngroups = 27 / G, nstage = ngroups > 1 ? 2 : 1;
    const uint32_t plane_b = HALO_V * 16;           // one plane of one channel chunk
    const uint32_t lboA = (uint32_t)npl * plane_b;  // channel-chunk stride
    const uint32_t halo_bytes = (uint32_t)kch * lboA;
    const uint32_t wtap = (uint32_t)cout * cin * 2;  // one tap's weights
    const uint32_t wstage = (uint32_t)G * wtap;      // one stage: G taps
    uint8_t* sH = sm;
    uint8_t* sW[2] = {sm + halo_bytes, sm + halo_bytes + (nstage > 1 ? wstage : 0)};
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + halo_bytes + nstage * wstage);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int x0 = blockIdx.x * 8, y0 = blockIdx.y * 16, z0 = blockIdx.z * P;
    const uint32_t ncols = rttc::tmem_cols(P * cout);
    if (tid == 0) {
        rttc::mbar_init(&bar[0], 1);
        rttc::mbar_init(&bar[1], 1);
        rttc::fence_mbar_init();
    }
    if (warp == 0) rttc::tmem_alloc(tslot, ncols);
    // halo planes z0-1 .. z0+P (zero outside the box): one (plane, halo voxel) pair per thread
    // and step (constant divisors), its channel chunks in an inner loop
    const int npairs = npl * HALO_V;
    for (int pr = tid; pr < npairs; pr += CONV_THREADS) {
        const int pl = pr / HALO_V, hv = pr - pl * HALO_V;
        const int hy = hv / HALO_X, hx = hv - hy * HALO_X;
        const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + pl;
        const bool inb = gx >= 0 && gx < a.X && gy >= 0 && gy < a.Y && gz >= 0 && gz < a.Z;
        const __nv_bfloat16* src = inb ? a.in + ((long)gx + (long)a.X * (gy + (long)a.Y * gz)) * a.in_stride : a.in;
        uint8_t* dst = sH + pl * plane_b + hv * 16;
        for (int j = 0; j < kch; j++) rttc::cp_async16(dst + j * lboA, src + (inb ? j * 8 : 0), inb ? 16u : 0u);
    }
    // the weights of taps [g G, (g+1) G), each in the K-major layout [chunk][out-channel group][8 rows][16 B]
    const uint32_t lboB = (uint32_t)(cout / 8) * 128;
    auto load_w = [&](int g, uint8_t* dst) {
        const int n_all = G * cout * kch;
        for (int idx = tid; idx < n_all; idx += CONV_THREADS) {
            const int tt = idx / (cout * kch), r = idx - tt * (cout * kch);
            const int n = r / kch, j = r - n * kch;
            rttc::cp_async16(dst + tt * wtap + j * lboB + (n >> 3) * 128 + (n & 7) * 16,
                             a.w + ((long)n * 27 + g * G + tt) * cin + j * 8, 16u);
        }
    };
    load_w(0, sW[0]);
    rttc::cp_async_commit();
    rttc::cp_async_wait_all();
    rttc::fence_async_smem();
    rttc::tc_fence_before();
    __syncthreads();
    rttc::tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = rttc::idesc_bf16(CONV_TM, cout, 0, 0);
    const uint32_t h0 = rttc::smem_u32(sH);
    bool ok = true;
    int last = -1;
    for (int g = 0; g < ngroups; g++) {
        const int b = g & 1;
        if (tid == 0) {
            rttc::tc_fence_after();
            // a descriptor's start field is (address >> 4): moving the operand is an integer add
            const uint64_t ad0 = rttc::sdesc(h0, lboA, HALO_X * 16);
            const uint64_t bd0 = rttc::sdesc(rttc::smem_u32(sW[b]), lboB, 128);
            const uint32_t a_kk = (2 * lboA) >> 4, b_kk = (2 * lboB) >> 4, a_pl = plane_b >> 4;
            const int nk = cin / 16;
            for (int tt = 0; tt < G; tt++) {
                const int t = g * G + tt;
                const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
                const uint64_t at = ad0 + (((uint32_t)(1 + dz) * plane_b + (uint32_t)((1 + dy) * HALO_X + 1 + dx) * 16) >> 4);
                const uint64_t bt = bd0 + ((uint32_t)tt * wtap >> 4);
                const uint32_t acc0 = t > 0 ? 1u : 0u;
                for (int p = 0; p < P; p++) {
                    const uint64_t ap = at + (uint64_t)p * a_pl;
                    const uint32_t dcol = tmem + (uint32_t)(p * cout);
                    for (int kk = 0; kk < nk; kk++)
                        rttc::mma_bf16(dcol, ap + (uint64_t)kk * a_kk, bt + (uint64_t)kk * b_kk, idesc,
                                       (acc0 | (uint32_t)kk) ? 1u : 0u);
                }
            }
            rttc::mma_commit(&bar[b]);
        }
        last = g;
        if (g + 1 < ngroups) {
            // the other stage was read by group g-1's MMAs
            if (g >= 1) {
                const bool w = rttc::mbar_wait(&bar[b ^ 1], ((g - 1) >> 1) & 1);
                if (!__syncthreads_and(w)) {
                    ok = false;
                    break;
                }
            }
            load_w(g + 1, sW[b ^ 1]);
            rttc::cp_async_commit();
            rttc::cp_async_wait_all();
            rttc::fence_async_smem();
            __syncthreads();
        }
    }
    bool done = rttc::mbar_wait(&bar[last & 1], (last >> 1) & 1);
    done = __syncthreads_and(done) != 0;
    if (!ok || !done) {
        if (tid == 0 && a.err) atomicExch(a.err, 1);
    } else {
        rttc::tc_fence_after();
        const int x = x0 + (tid & 7), y = y0 + (tid >> 3);
        for (int p = 0; p < P; p++) {
            const int z = z0 + p;
            const bool mv = x < a.X && y < a.Y && z < a.Z;
            const long m = (long)x + (long)a.X * (y + (long)a.Y * z);
            for (int c0 = 0; c0 < cout; c0 += 16) {
                float v[16];
                rttc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(p * cout + c0), v);
                if (!mv) continue;
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const float s = v[i] + (a.bias ? a.bias[c0 + i] : 0.f);
                    v[i] = a.relu ? fmaxf(s, 0.f) : s;
                }
                if (a.out_f32) {
                    float4* o = reinterpret_cast<float4*>(reinterpret_cast<float*>(a.out) + m * a.out_stride + c0);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        float4 val = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                        if (a.accumulate) {
                            const float4 old = o[q];
                            val.x += old.x; val.y += old.y; val.z += old.z; val.w += old.w;
                        }
                        o[q] = val;
                    }
                } else {
                    __align__(16) __nv_bfloat162 pk[8];
#pragma unroll
                    for (int q = 0; q < 8; q++) pk[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                    uint4* o = reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(a.out) + m * a.out_stride + c0);
                    o[0] = *reinterpret_cast<const uint4*>(&pk[0]);
                    o[1] = *reinterpret_cast<const uint4*>(&pk[4]);
                }
            }
        }
    }
    rttc::tc_fence_before();
    __syncthreads();
    if (warp == 0) rttc::tmem_dealloc(tmem, ncols);
}

// planes per CTA (P), taps per weight stage (G) and shared memory of k_conv3_halo: the largest
// P, then the largest G, whose halo and weight stages fit in 200 KB; P = 0 if nothing fits
static int halo_plan(int cin, int cout, int* G, size_t* smem) {
    static const int gs[4] = {27, 9, 3, 1};
    // first pass: plans that leave two CTAs per SM (one loads its halo while the other multiplies);
    // second pass: anything within 200 KB
    const size_t budgets[2] = {233472 / 2 - 1024, 200 * 1024};
    for (int pass = 0; pass < 2; pass++) {
        for (int P = 8; P >= 1; P /= 2) {
            if (P * cout > 512 || (pass == 0 && 2 * rttc::tmem_cols(P * cout) > 512)) continue;
            for (int gi = 0; gi < 4; gi++) {
                const int nst = gs[gi] == 27 ? 1 : 2;
                const size_t need =
                    (size_t)(P + 2) * HALO_V * cin * 2 + (size_t)nst * gs[gi] * cout * cin * 2 + 32;
                if (need > budgets[pass]) continue;
                const size_t maxc = 512 / rttc::tmem_cols(P * cout);
                const size_t floor_b = 233472 / (maxc + 1);
                *smem = need > floor_b ? need : floor_b;
                *G = gs[gi];
                return P;
            }
        }
    }
    return 0;
}

static int g_conv_variant = 1;  // 1: halo tile (default), 0: per-tap gather

size_t conv3_smem_bytes(int cin, int cout) {
    const size_t need = 2 * (size_t)CONV_TM * cin * 2 + 2 * (size_t)cout * cin * 2 + 32;
    // keep the CTAs an SM can hold within its 512 TMEM columns: more than 512 / ncols of
    // them must not fit in the 228 KB of shared memory
    const size_t maxc = 512 / rttc::tmem_cols(cout);
    const size_t floor_b = 233472 / (maxc + 1);
    return need > floor_b ? need : floor_b;
}

int conv3_init(rt_ctx* c) {
    cudaError_t e = cudaFuncSetAttribute(k_conv3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_conv3_halo, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return rt_fail(c, RT_ECUDA, "conv3 smem attribute: %s", cudaGetErrorString(e));
    return RT_OK;
}

void conv3_set_variant(int v) { g_conv_variant = v ? 1 : 0; }

int conv3(rt_ctx* c, const ConvArgs& a) {
    if (a.cin % 16 || a.cout % 16 || a.cin < 16 || a.cout < 16 || a.cin > 128 || a.cout > 128 || a.in_stride % 8 ||
        a.out_stride % (a.out_f32 ? 4 : 8))
        return rt_fail(c, RT_EINVAL, "conv3: channel counts must be multiples of 16 in [16, 128] (got %d -> %d)",
                       a.cin, a.cout);
    size_t hsmem = 0;
    int G = 1;
    const int P = g_conv_variant ? halo_plan(a.cin, a.cout, &G, &hsmem) : 0;
    if (P > 0) {
        const dim3 grid((unsigned)((a.X + 7) / 8), (unsigned)((a.Y + 15) / 16), (unsigned)((a.Z + P - 1) / P));
        return rt_launch(c, "unet_conv3_halo",
                         [&] { k_conv3_halo<<<grid, CONV_THREADS, hsmem, c->stream>>>(a, P, G); });
    }
    const long V = (long)a.X * a.Y * a.Z;
    const unsigned blocks = (unsigned)((V + CONV_TM - 1) / CONV_TM);
    const size_t smem = conv3_smem_bytes(a.cin, a.cout);
    return rt_launch(c, "unet_conv3_tc", [&] { k_conv3_tc<<<blocks, CONV_THREADS, smem, c->stream>>>(a); });
}

}  // namespace rtu

// ---------------------------------------------------------------------------
// element-wise and reduction kernels of the network (channels-last, x fastest)
// ---------------------------------------------------------------------------
namespace rtu {

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// 2x2x2 average pooling: coarse (X/2 rounded up) box; children outside the fine box are skipped
__global__ void k_pool2(const __nv_bfloat16* __restrict__ in, int in_stride, int C, int X, int Y, int Z,
                        __nv_bfloat16* __restrict__ out, int out_stride) {
    const int Xc = (X + 1) / 2, Yc = (Y + 1) / 2, Zc = (Z + 1) / 2;
    const long n = (long)Xc * Yc * Zc * C;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long v = i / C;
        const int x = (int)(v % Xc), y = (int)((v / Xc) % Yc), z = (int)(v / ((long)Xc * Yc));
        float s = 0.f;
        int cnt = 0;
        for (int d = 0; d < 8; d++) {
            const int xf = 2 * x + (d & 1), yf = 2 * y + ((d >> 1) & 1), zf = 2 * z + (d >> 2);
            if (xf < X && yf < Y && zf < Z) {
                s += bf(in[((long)xf + (long)X * (yf + (long)Y * zf)) * in_stride + c]);
                cnt++;
            }
        }
        out[v * out_stride + c] = __float2bfloat16(s / (float)cnt);
    }
}

// gradient of k_pool2: each fine voxel receives its parent's gradient / (children of the parent)
__global__ void k_pool2_bwd(const float* __restrict__ gout, int C, int X, int Y, int Z, float* __restrict__ gin,
                            int gin_stride) {
    const int Xc = (X + 1) / 2, Yc = (Y + 1) / 2;
    const long n = (long)X * Y * Z * C;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long v = i / C;
        const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long)X * Y));
        const int xc = x / 2, yc = y / 2, zc = z / 2;
        const int cnt = (2 * xc + 1 < X ? 2 : 1) * (2 * yc + 1 < Y ? 2 : 1) * (2 * zc + 1 < Z ? 2 : 1);
        gin[v * gin_stride + c] += gout[((long)xc + (long)Xc * (yc + (long)Yc * zc)) * C + c] / (float)cnt;
    }
}

// nearest-neighbour 2x upsampling of a coarse box into the fine box X x Y x Z
__global__ void k_up2(const __nv_bfloat16* __restrict__ in, int C, int X, int Y, int Z, __nv_bfloat16* __restrict__ out,
                      int out_stride) {
    const int Xc = (X + 1) / 2, Yc = (Y + 1) / 2;
    const long n = (long)X * Y * Z * C;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long v = i / C;
        const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long)X * Y));
        out[v * out_stride + c] = in[((long)(x / 2) + (long)Xc * (y / 2 + (long)Yc * (z / 2))) * C + c];
    }
}

// gradient of k_up2: a coarse voxel sums its children's gradients
__global__ void k_up2_bwd(const float* __restrict__ gout, int gout_stride, int C, int X, int Y, int Z,
                          float* __restrict__ gin) {
    const int Xc = (X + 1) / 2, Yc = (Y + 1) / 2, Zc = (Z + 1) / 2;
    const long n = (long)Xc * Yc * Zc * C;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long v = i / C;
        const int x = (int)(v % Xc), y = (int)((v / Xc) % Yc), z = (int)(v / ((long)Xc * Yc));
        float s = 0.f;
        for (int d = 0; d < 8; d++) {
            const int xf = 2 * x + (d & 1), yf = 2 * y + ((d >> 1) & 1), zf = 2 * z + (d >> 2);
            if (xf < X && yf < Y && zf < Z) s += gout[((long)xf + (long)X * (yf + (long)Y * zf)) * gout_stride + c];
        }
        gin[v * C + c] = s;
    }
}

// gradient through ReLU into bf16 (the tensor-core operand) and the bias gradient partials
__global__ void k_relu_bwd(const float* __restrict__ g, int g_stride, const __nv_bfloat16* __restrict__ y,
                           int y_stride, int C, long V, int relu, __nv_bfloat16* __restrict__ gpre) {
    const long n = V * C;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long v = i / C;
        const float gv = g[v * g_stride + c];
        gpre[i] = __float2bfloat16(!relu || bf(y[v * y_stride + c]) > 0.f ? gv : 0.f);
    }
}

// 1x1x1 head: out[v][k] = hb[k] + sum_c hw[k][c] in[v][c], k < 3 (FP32 output)
__global__ void k_head(const __nv_bfloat16* __restrict__ in, int C, long V, const float* __restrict__ hw,
                       const float* __restrict__ hb, float* __restrict__ out) {
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x) {
        float a0 = hb[0], a1 = hb[1], a2 = hb[2];
        for (int c = 0; c < C; c++) {
            const float x = bf(in[v * C + c]);
            a0 += hw[c] * x;
            a1 += hw[C + c] * x;
            a2 += hw[2 * C + c] * x;
        }
        out[3 * v] = a0;
        out[3 * v + 1] = a1;
        out[3 * v + 2] = a2;
    }
}

// head backward: gin[v][c] = sum_k hw[k][c] gout[v][k]; block partials of dhw, dhb
__global__ void k_head_bwd(const __nv_bfloat16* __restrict__ in, int C, long V, const float* __restrict__ hw,
                           const float* __restrict__ gout, float* __restrict__ gin, float* __restrict__ dhw,
                           float* __restrict__ dhb) {
    __shared__ float sw[3 * 64 + 3];
    for (int i = threadIdx.x; i < 3 * C + 3; i += blockDim.x) sw[i] = 0.f;
    __syncthreads();
    float lw[3 * 16], lb[3] = {0.f, 0.f, 0.f};  // C <= 16
    for (int i = 0; i < 3 * C; i++) lw[i] = 0.f;
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x) {
        const float g0 = gout[3 * v], g1 = gout[3 * v + 1], g2 = gout[3 * v + 2];
        lb[0] += g0; lb[1] += g1; lb[2] += g2;
        for (int c = 0; c < C; c++) {
            const float x = bf(in[v * C + c]);
            gin[v * C + c] = hw[c] * g0 + hw[C + c] * g1 + hw[2 * C + c] * g2;
            lw[c] += g0 * x;
            lw[C + c] += g1 * x;
            lw[2 * C + c] += g2 * x;
        }
    }
    for (int i = 0; i < 3 * C; i++) atomicAdd(&sw[i], lw[i]);
    for (int k = 0; k < 3; k++) atomicAdd(&sw[3 * C + k], lb[k]);
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * C; i += blockDim.x) atomicAdd(&dhw[i], sw[i]);
    for (int k = threadIdx.x; k < 3; k += blockDim.x) atomicAdd(&dhb[k], sw[3 * C + k]);
}

// mean squared error over V x 3 outputs: gout = 2 (out - tgt) / (3V), loss partials
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ tgt, long n, float* __restrict__ gout,
                      double* __restrict__ loss) {
    __shared__ double sh[256];
    double s = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float d = out[i] - tgt[i];
        gout[i] = 2.f * d / (float)n;
        s += (double)d * d;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, sh[0] / (double)n);
}

// dB[n] += sum_v gpre[v][n]  (block partial sums, one atomic per block and channel)
__global__ void k_bias_grad(const __nv_bfloat16* __restrict__ gpre, int C, long V, float* __restrict__ db) {
    __shared__ float sh[128];
    for (int c = threadIdx.x; c < C; c += blockDim.x) sh[c] = 0.f;
    __syncthreads();
    const int c = threadIdx.x % C;
    const int rows_per_pass = blockDim.x / C;
    const int r0 = threadIdx.x / C;
    float s = 0.f;
    if (r0 < rows_per_pass)
        for (long v = blockIdx.x * (long)rows_per_pass + r0; v < V; v += (long)gridDim.x * rows_per_pass)
            s += bf(gpre[v * C + c]);
    if (r0 < rows_per_pass) atomicAdd(&sh[c], s);
    __syncthreads();
    for (int q = threadIdx.x; q < C; q += blockDim.x) atomicAdd(&db[q], sh[q]);
}

// dW[n][tap][c] += sum_v gpre[v][n] * in[v + off(tap)][c]: thread per (n, tap, c) over a voxel chunk
__global__ void k_conv3_dw(const __nv_bfloat16* __restrict__ in, int in_stride, int cin,
                           const __nv_bfloat16* __restrict__ gpre, int cout, int X, int Y, int Z, long chunk,
                           float* __restrict__ dw) {
    const long nw = (long)cout * 27 * cin;
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= nw) return;
    const int c = (int)(idx % cin);
    const int tap = (int)((idx / cin) % 27);
    const int n = (int)(idx / (27L * cin));
    const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
    const long V = (long)X * Y * Z;
    const long v0 = blockIdx.y * chunk, v1 = min(V, v0 + chunk);
    float s = 0.f;
    for (long v = v0; v < v1; v++) {
        const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long)X * Y));
        const int xn = x + dx, yn = y + dy, zn = z + dz;
        if (xn < 0 || xn >= X || yn < 0 || yn >= Y || zn < 0 || zn >= Z) continue;
        const float gv = bf(gpre[v * cout + n]);
        if (gv != 0.f) s += gv * bf(in[((long)xn + (long)X * (yn + (long)Y * zn)) * in_stride + c]);
    }
    atomicAdd(&dw[idx], s);
}

// bf16 weights for the forward pass and tap-flipped transposed weights for the input gradient:
// wt[c][26 - tap][n] = w[n][tap][c]
__global__ void k_weights_bf16(const float* __restrict__ w, int cin, int cout, __nv_bfloat16* __restrict__ w16,
                               __nv_bfloat16* __restrict__ w16t) {
    const long n_all = (long)cout * 27 * cin;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n_all; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i % cin), tap = (int)((i / cin) % 27), n = (int)(i / (27L * cin));
        const __nv_bfloat16 v = __float2bfloat16(w[i]);
        w16[i] = v;
        w16t[((long)c * 27 + (26 - tap)) * cout + n] = v;
    }
}

// Adam (decoupled scale-free form): m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2, p -= lr mhat / (sqrt(vhat) + eps)
__global__ void k_adam(long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float c1, float c2, float eps) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

}  // namespace rtu
