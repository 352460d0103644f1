// rt_coarse.cu — assembled-stencil levels, grid transfers and Galerkin assembly.
//
// Restates:
//   update_residual_kernel_1               grid/Grid.cu:1350-1448
//   gs_relax_kernel                        grid/Grid.cu:678-790
//   restrict_residual{,_nondyadic}_kernel  grid/Grid.cu:1680-1794
//   prolongate_correction{,_nondyadic}_kernel grid/Grid.cu:1818-1895
//   restrict_stencil_nondyadic_OTFA_{NS,WS}_kernel grid/Grid.cu:296-506
//   restrict_stencil_dyadic_kernel         grid/Grid.cu:120-177
// Stencils are [27*9][nv]: entry (k*9 + 3*row + col)*nv + v couples node v to
// neighbour v + d(k), d(k) = (k%3-1, k/3%3-1, k/9-1) — the reference's
// GraftArray<double,27,9> layout over a dense node box.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "rt_internal.h"
#include "rt_tc.cuh"

namespace {

constexpr int ST_BS = 256;

unsigned grid_for(rt_ctx* c, long n, int bs) {
    long b = rt_blocks(n, bs);
    long cap = (long)c->sm_count * 16;
    return (unsigned)(b < cap ? b : cap);
}

// ---------------------------------------------------------------------------
// Stencil storage.  The assembled FP64 operator is row-major, row j = 9 k + 3 r + c
// (neighbour k, block row r, column c) of all nodes: [243][nv].  The FP32 and BF16
// copies the smoothers read are blocked by 32 nodes, [nv/32][RS][32]: the rows of 32
// neighbouring nodes form one contiguous run (31 KB in FP32), so the loads of a warp
// stay in one or two DRAM pages and TLB entries instead of touching 243 rows nv apart.
// The BF16 copy has 9 more rows (RS = 252): the centre block is stored as hi + lo
// BF16 pairs, and is shifted by the rounding error of the 26 off-centre blocks, so
// the row sums of every 3x3 block row (the operator applied to the three rigid
// translations) equal the FP64 operator's to ~2^-17 instead of ~2^-9.
// ---------------------------------------------------------------------------
template <typename S>
struct StAddr {
    static constexpr bool BLK = sizeof(S) < 8;
    static constexpr int RS = sizeof(S) == 2 ? 252 : 243;
    __device__ __forceinline__ static long base(long v) { return BLK ? (v >> 5) * (RS * 32L) + (v & 31) : v; }
    __device__ __forceinline__ static long stride(long nv) { return BLK ? 32 : nv; }
};

// a stencil entry in the compute type: FP64 / FP32 as stored, BF16 bit patterns widened exactly
template <typename T>
__device__ __forceinline__ T st_val(const T* p) { return *p; }
__device__ __forceinline__ float st_val(const uint16_t* p) { return __uint_as_float((uint32_t)*p << 16); }

// entry (block row r, column c) of the centre block; sb = st + StAddr::base(v)
template <typename T, typename S>
__device__ __forceinline__ T st_centre(const S* sb, long rs, int rc) {
    T x = (T)st_val(sb + (117 + rc) * rs);
    if (sizeof(S) == 2) x += (T)st_val(sb + (243 + rc) * rs);
    return x;
}

// sum over the 27 neighbours of A_vk u_k (SKIPSELF: without the centre block)
template <typename T, typename S, bool SKIPSELF>
__device__ __forceinline__ void st_node_sum(int x, int y, int z, int vx, int vy, int vz, long nv,
                                            const S* __restrict__ st, const T* __restrict__ u, long v, T Au[3]) {
    Au[0] = Au[1] = Au[2] = T(0);
    const long rs = StAddr<S>::stride(nv);
    const S* sb = st + StAddr<S>::base(v);
#pragma unroll
    for (int k = 0; k < 27; k++) {
        if (SKIPSELF && k == 13) continue;
        const int jx = x + k % 3 - 1, jy = y + (k / 3) % 3 - 1, jz = z + k / 9 - 1;
        if (jx < 0 || jy < 0 || jz < 0 || jx >= vx || jy >= vy || jz >= vz) continue;
        const long nj = jx + (long)vx * (jy + (long)vy * jz);
        const T u0 = u[nj], u1 = u[nv + nj], u2 = u[2 * nv + nj];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            T a0, a1, a2;
            if (k == 13) {
                a0 = st_centre<T>(sb, rs, 3 * r); a1 = st_centre<T>(sb, rs, 3 * r + 1); a2 = st_centre<T>(sb, rs, 3 * r + 2);
            } else {
                const S* s = sb + (long)(k * 9 + 3 * r) * rs;
                a0 = (T)st_val(s); a1 = (T)st_val(s + rs); a2 = (T)st_val(s + 2 * rs);
            }
            Au[r] += a0 * u0 + a1 * u1 + a2 * u2;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(ST_BS) k_st_gs(int nx, int ny, int nz, int color, bool backward,
                                                  const uint8_t* __restrict__ vact, const T* __restrict__ st,
                                                  T* __restrict__ u, const T* __restrict__ f) {
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long rs = StAddr<T>::stride(nv);
    const int px = color & 1, py = (color >> 1) & 1, pz = (color >> 2) & 1;
    const int cx = (vx - px + 1) / 2, cy = (vy - py + 1) / 2, cz = (vz - pz + 1) / 2;
    const long nc = (long)cx * cy * cz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nc; t += (long)gridDim.x * blockDim.x) {
        const int x = px + 2 * (int)(t % cx), y = py + 2 * (int)((t / cx) % cy), z = pz + 2 * (int)(t / ((long)cx * cy));
        const long v = x + (long)vx * (y + (long)vy * z);
        if (!vact[v]) continue;
        T Au[3];
        st_node_sum<T, T, true>(x, y, z, vx, vy, vz, nv, st, u, v, Au);
        T S[9];
        const T* sb = st + StAddr<T>::base(v);
#pragma unroll
        for (int i = 0; i < 9; i++) S[i] = st_centre<T>(sb, rs, i);
        const T F[3] = {f[v], f[nv + v], f[2 * nv + v]};
        T uu[3] = {u[v], u[nv + v], u[2 * nv + v]};
        if (!backward) {
            uu[0] = (F[0] - S[1] * uu[1] - S[2] * uu[2] - Au[0]) / S[0];
            uu[1] = (F[1] - S[3] * uu[0] - S[5] * uu[2] - Au[1]) / S[4];
            uu[2] = (F[2] - S[6] * uu[0] - S[7] * uu[1] - Au[2]) / S[8];
        } else {
            uu[2] = (F[2] - S[6] * uu[0] - S[7] * uu[1] - Au[2]) / S[8];
            uu[1] = (F[1] - S[3] * uu[0] - S[5] * uu[2] - Au[1]) / S[4];
            uu[0] = (F[0] - S[1] * uu[1] - S[2] * uu[2] - Au[0]) / S[0];
        }
        u[v] = uu[0]; u[nv + v] = uu[1]; u[2 * nv + v] = uu[2];
    }
}

// ---------------------------------------------------------------------------
// Lane-split stencil kernels: 4 lanes per node, lane q sums neighbours
// k = q, q+4, ..., then the three row sums are combined with shuffles.  Coarse
// levels are small (the first coarse level of 128x128x64 has 18.5k nodes), so
// a thread per node leaves most of the GPU idle on long dependent load chains.
// MODE 0: r = f - A u;  MODE 2: Jacobi;  MODE 3: Chebyshev step.
// ---------------------------------------------------------------------------
template <typename T, int MODE, typename S = T>
__global__ void __launch_bounds__(ST_BS, sizeof(T) == 8 ? 1 : 3) k_st_split4(int nx, int ny, int nz, const uint8_t* __restrict__ vact,
                                                      const S* __restrict__ st, const T* __restrict__ u,
                                                      const T* __restrict__ f, T* __restrict__ out,
                                                      T* __restrict__ d, T omega, const double* __restrict__ coef,
                                                      int kstep) {
    T ca = T(0), cb = T(0);
    if (MODE == 3) {
        const double a_ = coef[2 * kstep], b_ = coef[2 * kstep + 1];
        ca = (T)a_;
        cb = (T)b_;
    }
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long rs = StAddr<S>::stride(nv);
    const int q = threadIdx.x & 3;
    const long ngroups = (long)gridDim.x * (blockDim.x >> 2);
    // every lane runs the same number of trips (the shuffles below use the full mask)
    const long vend = ((nv + ngroups - 1) / ngroups) * ngroups;
    for (long v = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 2; v < vend; v += ngroups) {
        const bool inb = v < nv;
        const bool act = inb && vact[v];
        const S* sb = st + StAddr<S>::base(inb ? v : 0);
        T Au[3] = {T(0), T(0), T(0)};
        if (act) {
            const int x = (int)(v % vx), y = (int)((v / vx) % vy), z = (int)(v / ((long)vx * vy));
#pragma unroll
            for (int kk = 0; kk < 7; kk++) {
                const int k = q + 4 * kk;
                if (k >= 27) break;
                const int jx = x + k % 3 - 1, jy = y + (k / 3) % 3 - 1, jz = z + k / 9 - 1;
                if (jx < 0 || jy < 0 || jz < 0 || jx >= vx || jy >= vy || jz >= vz) continue;
                const long nj = jx + (long)vx * (jy + (long)vy * jz);
                const T u0 = u[nj], u1 = u[nv + nj], u2 = u[2 * nv + nj];
                const S* s = sb + (long)(k * 9) * rs;
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    T a0 = (T)st_val(s + (3 * r) * rs), a1 = (T)st_val(s + (3 * r + 1) * rs),
                      a2 = (T)st_val(s + (3 * r + 2) * rs);
                    if (sizeof(S) == 2 && k == 13) {  // low parts of the BF16 centre block
                        a0 += (T)st_val(sb + (243 + 3 * r) * rs);
                        a1 += (T)st_val(sb + (243 + 3 * r + 1) * rs);
                        a2 += (T)st_val(sb + (243 + 3 * r + 2) * rs);
                    }
                    Au[r] += a0 * u0 + a1 * u1 + a2 * u2;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 3; r++) {
            Au[r] += __shfl_xor_sync(0xffffffffu, Au[r], 1);
            Au[r] += __shfl_xor_sync(0xffffffffu, Au[r], 2);
        }
        if (!inb || q == 3) continue;
        // lane q (0..2) owns component q
        const long oq = (long)q * nv + v;
        if (MODE == 0) {
            out[oq] = act ? f[oq] - Au[q] : T(0);
            continue;
        }
        T res = T(0), dn = T(0);
        if (act) {
            T S9[9];
#pragma unroll
            for (int i = 0; i < 9; i++) S9[i] = st_centre<T>(sb, rs, i);
            const T a0 = S9[0], b0 = S9[1], c0 = S9[2], d0 = S9[3], e0 = S9[4], f0 = S9[5], g0 = S9[6], h0 = S9[7],
                    k0 = S9[8];
            const T A = e0 * k0 - f0 * h0, B = -(d0 * k0 - f0 * g0), Cc = d0 * h0 - e0 * g0;
            const T id = T(1) / (a0 * A + b0 * B + c0 * Cc);
            // row q of the inverse (adjugate / determinant)
            const T i0 = q == 0 ? A : (q == 1 ? B : Cc);
            const T i1 = q == 0 ? -(b0 * k0 - c0 * h0) : (q == 1 ? (a0 * k0 - c0 * g0) : -(a0 * h0 - b0 * g0));
            const T i2 = q == 0 ? (b0 * f0 - c0 * e0) : (q == 1 ? -(a0 * f0 - c0 * d0) : (a0 * e0 - b0 * d0));
            const T r0 = f[v] - Au[0], r1 = f[nv + v] - Au[1], r2 = f[2 * nv + v] - Au[2];
            const T zq = (i0 * id) * r0 + (i1 * id) * r1 + (i2 * id) * r2;
            if (MODE == 2) {
                res = u[oq] + omega * zq;
            } else {
                dn = (kstep == 0 ? T(0) : ca * d[oq]) + cb * zq;
                res = u[oq] + dn;
            }
        }
        out[oq] = res;
        if (MODE == 3) d[oq] = dn;
    }
}

// ---------------------------------------------------------------------------
// Fused Chebyshev sweeps of a small stencil level: all nsteps steps in one cooperative
// launch, the steps separated by a grid barrier instead of a kernel boundary.  The coarse
// levels below the first are a few thousand nodes: a separate launch per step spends most
// of its time in launch, ramp-up and drain, not in the 243-entry rows.  Same arithmetic and
// thread layout as k_st_split4 (MODE 3); u is ping-ponged with tmp (u -> tmp -> u ...), so
// after an odd step count a last barrier lets every thread copy its own entries back to u.
// Values written by other blocks in the previous step are read through L2 (ld.global.cg):
// L1 is not coherent across SMs.  The barrier is bounded: a block whose wait runs out sets
// the error slot, poisons u[0] with NaN (the solve then stops on its NaN check) and returns.
// ---------------------------------------------------------------------------
// the polls of a wait come from the context (rt_ctx_set_wait_limit; default 1 << 22, a few hundred
// ns each at most)

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// grid-wide barrier: bar[0] counts arrivals, bar[1] is the generation; gen is thread 0's copy
__device__ __forceinline__ bool coop_grid_sync(unsigned* bar, unsigned& gen, int* s_ok, long spin_limit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        bool ok = true;
        __threadfence();
        const unsigned prev = atomicAdd(bar, 1u);
        if (prev == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicExch(bar + 1, gen + 1);
        } else {
            long it = 0;
            while (ld_acquire_u32(bar + 1) == gen) {
                if (++it > spin_limit) {
                    ok = false;
                    break;
                }
            }
        }
        __threadfence();
        gen++;
        *s_ok = ok ? 1 : 0;
    }
    __syncthreads();
    return *s_ok != 0;
}

template <typename S>
__global__ void __launch_bounds__(ST_BS, 3) k_st_cheby_coop(int nx, int ny, int nz, const uint8_t* __restrict__ vact,
                                                             const S* __restrict__ st, float* u,
                                                             const float* __restrict__ f, float* tmp, float* d,
                                                             const double* __restrict__ coef, int nsteps,
                                                             unsigned* bar, double* err, long spin_limit) {
    __shared__ int s_ok;
    unsigned gen = 0;
    if (threadIdx.x == 0) gen = ld_acquire_u32(bar + 1);
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long rs = StAddr<S>::stride(nv);
    const int q = threadIdx.x & 3;
    const long ngroups = (long)gridDim.x * (blockDim.x >> 2);
    const long vend = ((nv + ngroups - 1) / ngroups) * ngroups;
    const long v0 = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 2;
    for (int s = 0; s < nsteps; s++) {
        const float* src = (s & 1) ? tmp : u;
        float* dst = (s & 1) ? u : tmp;
        const float ca = (float)coef[2 * s], cb = (float)coef[2 * s + 1];
        for (long v = v0; v < vend; v += ngroups) {
            const bool inb = v < nv;
            const bool act = inb && vact[v];
            const S* sb = st + StAddr<S>::base(inb ? v : 0);
            float Au[3] = {0.f, 0.f, 0.f};
            if (act) {
                const int x = (int)(v % vx), y = (int)((v / vx) % vy), z = (int)(v / ((long)vx * vy));
#pragma unroll
                for (int kk = 0; kk < 7; kk++) {
                    const int k = q + 4 * kk;
                    if (k >= 27) break;
                    const int jx = x + k % 3 - 1, jy = y + (k / 3) % 3 - 1, jz = z + k / 9 - 1;
                    if (jx < 0 || jy < 0 || jz < 0 || jx >= vx || jy >= vy || jz >= vz) continue;
                    const long nj = jx + (long)vx * (jy + (long)vy * jz);
                    const float u0 = __ldcg(src + nj), u1 = __ldcg(src + nv + nj), u2 = __ldcg(src + 2 * nv + nj);
                    const S* sk = sb + (long)(k * 9) * rs;
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        float a0 = st_val(sk + (3 * r) * rs), a1 = st_val(sk + (3 * r + 1) * rs),
                              a2 = st_val(sk + (3 * r + 2) * rs);
                        if (sizeof(S) == 2 && k == 13) {  // low parts of the BF16 centre block
                            a0 += st_val(sb + (243 + 3 * r) * rs);
                            a1 += st_val(sb + (243 + 3 * r + 1) * rs);
                            a2 += st_val(sb + (243 + 3 * r + 2) * rs);
                        }
                        Au[r] += a0 * u0 + a1 * u1 + a2 * u2;
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < 3; r++) {
                Au[r] += __shfl_xor_sync(0xffffffffu, Au[r], 1);
                Au[r] += __shfl_xor_sync(0xffffffffu, Au[r], 2);
            }
            if (!inb || q == 3) continue;
            const long oq = (long)q * nv + v;
            float res = 0.f, dn = 0.f;
            if (act) {
                float S9[9];
#pragma unroll
                for (int i = 0; i < 9; i++) S9[i] = st_centre<float>(sb, rs, i);
                const float a0 = S9[0], b0 = S9[1], c0 = S9[2], d0 = S9[3], e0 = S9[4], f0 = S9[5], g0 = S9[6],
                            h0 = S9[7], k0 = S9[8];
                const float A = e0 * k0 - f0 * h0, B = -(d0 * k0 - f0 * g0), Cc = d0 * h0 - e0 * g0;
                const float id = 1.f / (a0 * A + b0 * B + c0 * Cc);
                const float i0 = q == 0 ? A : (q == 1 ? B : Cc);
                const float i1 = q == 0 ? -(b0 * k0 - c0 * h0) : (q == 1 ? (a0 * k0 - c0 * g0) : -(a0 * h0 - b0 * g0));
                const float i2 = q == 0 ? (b0 * f0 - c0 * e0) : (q == 1 ? -(a0 * f0 - c0 * d0) : (a0 * e0 - b0 * d0));
                const float r0 = f[v] - Au[0], r1 = f[nv + v] - Au[1], r2 = f[2 * nv + v] - Au[2];
                const float zq = (i0 * id) * r0 + (i1 * id) * r1 + (i2 * id) * r2;
                dn = (s == 0 ? 0.f : ca * d[oq]) + cb * zq;
                res = __ldcg(src + oq) + dn;
            }
            dst[oq] = res;
            d[oq] = dn;
        }
        if (s + 1 < nsteps || (nsteps & 1)) {
            if (!coop_grid_sync(bar, gen, &s_ok, spin_limit)) {
                if (threadIdx.x == 0) {
                    *err = 2.0;
                    u[0] = __int_as_float(0x7fc00000);
                }
                return;
            }
        }
    }
    if (nsteps & 1) {  // the last step wrote tmp: every thread copies back the entries it wrote
        for (long v = v0; v < nv; v += ngroups)
            if (q < 3) u[(long)q * nv + v] = __ldcg(tmp + (long)q * nv + v);
    }
}

// Resident form of the fused sweeps, for levels whose 4-lane groups all fit on the device at
// once (one group per node, 64 nodes per block): the stencil rows each lane multiplies are
// read once into shared memory (63 x 256 floats, entries outside the box or of inactive
// nodes zeroed so the step has no bounds branches), the inverse diagonal row, f and the
// Chebyshev direction stay in registers, and a step moves only the neighbours' u through L2.
constexpr int RES_ROWS = 63;  // 7 neighbours x 9 entries per lane
constexpr size_t RES_SMEM = (size_t)RES_ROWS * ST_BS * sizeof(float);

template <typename S>
__global__ void __launch_bounds__(ST_BS, 3) k_st_cheby_res(int nx, int ny, int nz, const uint8_t* __restrict__ vact,
                                                            const S* __restrict__ st, float* u,
                                                            const float* __restrict__ f, float* tmp, float* d,
                                                            const double* __restrict__ coef, int nsteps,
                                                            unsigned* bar, double* err, long spin_limit) {
    extern __shared__ float srow[];  // [RES_ROWS][ST_BS]
    __shared__ int s_ok;
    unsigned gen = 0;
    if (threadIdx.x == 0) gen = ld_acquire_u32(bar + 1);
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long rs = StAddr<S>::stride(nv);
    const int tid = threadIdx.x, q = tid & 3;
    const long v = (blockIdx.x * (long)blockDim.x + tid) >> 2;
    const bool inb = v < nv;
    const bool act = inb && vact[v];
    const S* sb = st + StAddr<S>::base(inb ? v : 0);
    const int x = inb ? (int)(v % vx) : 0, y = inb ? (int)((v / vx) % vy) : 0,
              z = inb ? (int)(v / ((long)vx * vy)) : 0;
    long nj[7];
#pragma unroll
    for (int kk = 0; kk < 7; kk++) {
        const int k = q + 4 * kk;
        const int jx = x + k % 3 - 1, jy = y + (k / 3) % 3 - 1, jz = z + k / 9 - 1;
        const bool ok = act && k < 27 && jx >= 0 && jy >= 0 && jz >= 0 && jx < vx && jy < vy && jz < vz;
        nj[kk] = ok ? jx + (long)vx * (jy + (long)vy * jz) : (inb ? v : 0);
        const S* sk = sb + (long)(k * 9) * rs;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            float a = 0.f;
            if (ok) {
                a = st_val(sk + e * rs);
                if (sizeof(S) == 2 && k == 13) a += st_val(sb + (243 + e) * rs);  // BF16 centre low part
            }
            srow[(kk * 9 + e) * ST_BS + tid] = a;
        }
    }
    // row q of the inverse centre block (scaled by 1 / det), f of the node, the direction d
    float i0 = 0.f, i1 = 0.f, i2 = 0.f, f0 = 0.f, f1 = 0.f, f2 = 0.f, dq = 0.f;
    if (act && q < 3) {
        float S9[9];
#pragma unroll
        for (int i = 0; i < 9; i++) S9[i] = st_centre<float>(sb, rs, i);
        const float a0 = S9[0], b0 = S9[1], c0 = S9[2], d0 = S9[3], e0 = S9[4], g0f = S9[5], g0 = S9[6], h0 = S9[7],
                    k0 = S9[8];
        const float A = e0 * k0 - g0f * h0, B = -(d0 * k0 - g0f * g0), Cc = d0 * h0 - e0 * g0;
        const float id = 1.f / (a0 * A + b0 * B + c0 * Cc);
        i0 = (q == 0 ? A : (q == 1 ? B : Cc)) * id;
        i1 = (q == 0 ? -(b0 * k0 - c0 * h0) : (q == 1 ? (a0 * k0 - c0 * g0) : -(a0 * h0 - b0 * g0))) * id;
        i2 = (q == 0 ? (b0 * g0f - c0 * e0) : (q == 1 ? -(a0 * g0f - c0 * d0) : (a0 * e0 - b0 * d0))) * id;
        f0 = f[v];
        f1 = f[nv + v];
        f2 = f[2 * nv + v];
    }
    __syncthreads();
    const long oq = (long)(q < 3 ? q : 0) * nv + (inb ? v : 0);
    for (int s = 0; s < nsteps; s++) {
        const float* src = (s & 1) ? tmp : u;
        float* dst = (s & 1) ? u : tmp;
        float Au[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int kk = 0; kk < 7; kk++) {
            if (q + 4 * kk >= 27) break;
            const float u0 = __ldcg(src + nj[kk]), u1 = __ldcg(src + nv + nj[kk]), u2 = __ldcg(src + 2 * nv + nj[kk]);
#pragma unroll
            for (int r = 0; r < 3; r++)
                Au[r] += srow[(kk * 9 + 3 * r) * ST_BS + tid] * u0 + srow[(kk * 9 + 3 * r + 1) * ST_BS + tid] * u1 +
                         srow[(kk * 9 + 3 * r + 2) * ST_BS + tid] * u2;
        }
#pragma unroll
        for (int r = 0; r < 3; r++) {
            Au[r] += __shfl_xor_sync(0xffffffffu, Au[r], 1);
            Au[r] += __shfl_xor_sync(0xffffffffu, Au[r], 2);
        }
        if (inb && q < 3) {
            float res = 0.f, dn = 0.f;
            if (act) {
                const float zq = i0 * (f0 - Au[0]) + i1 * (f1 - Au[1]) + i2 * (f2 - Au[2]);
                dn = (s == 0 ? 0.f : (float)coef[2 * s] * dq) + (float)coef[2 * s + 1] * zq;
                res = __ldcg(src + oq) + dn;
            }
            dst[oq] = res;
            dq = dn;
        }
        if (s + 1 < nsteps || (nsteps & 1)) {
            if (!coop_grid_sync(bar, gen, &s_ok, spin_limit)) {
                if (threadIdx.x == 0) {
                    *err = 2.0;
                    u[0] = __int_as_float(0x7fc00000);
                }
                return;
            }
        }
    }
    if (inb && q < 3) {
        d[oq] = dq;
        if (nsteps & 1) u[oq] = __ldcg(tmp + oq);
    }
}

// ---------------------------------------------------------------------------
// Stencil kernel over the blocked FP32 / BF16 copies: the 31 KB (FP32) / 16 KB (BF16)
// stencil run of a 32-node block is fetched with one bulk asynchronous copy
// (cp.async.bulk, completion counted on an mbarrier) into a ring of NST shared-memory
// stages, so the stencil stream needs no registers in flight and the copies of the
// next blocks overlap the arithmetic of this one.  A CTA of 8 warps walks its blocks
// (blockIdx.x, + gridDim.x, ...): warp w sums the neighbours k = w, w+8, ... of the
// block's 32 nodes (lane = node, conflict-free stage reads), the eight partial sums
// meet in shared memory, and warps 0..2 finish component q = warp of every node.
// Every mbarrier wait is bounded: on a timeout the CTA waits (bounded) for its copies
// still in flight, writes NaN to the outputs it did not produce and sets the level's
// error slot, so the solve stops with an error instead of hanging.
// ---------------------------------------------------------------------------
constexpr int SB_BS = 256;
constexpr int SB_WARPS = SB_BS / 32;

template <typename S>
__host__ __device__ constexpr int sb_stages() { return sizeof(S) == 2 ? 4 : 3; }
template <typename T, typename S>
constexpr size_t sb_smem() {
    return 128 + (size_t)sb_stages<S>() * StAddr<S>::RS * 32 * sizeof(S) + SB_WARPS * 3 * 32 * sizeof(T);
}
template <typename S>
constexpr int sb_ctas_per_sm() { return sizeof(S) == 2 ? 3 : 2; }

template <typename T, int MODE, typename S>
__global__ void __launch_bounds__(SB_BS) k_st_bulk(int nx, int ny, int nz, const uint8_t* __restrict__ vact,
                                                    const S* __restrict__ st, const T* __restrict__ u,
                                                    const T* __restrict__ f, T* __restrict__ out, T* __restrict__ d,
                                                    T omega, const double* __restrict__ coef, int kstep,
                                                    double* __restrict__ errslot) {
    constexpr int RS = StAddr<S>::RS, NST = sb_stages<S>();
    constexpr uint32_t BLK_BYTES = RS * 32 * sizeof(S);
    constexpr long BLK_ELEMS = RS * 32;
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
    S* stg = reinterpret_cast<S*>(sm + 128);
    T* red = reinterpret_cast<T*>(sm + 128 + NST * BLK_BYTES);
    T ca = T(0), cb = T(0);
    if (MODE == 3) {
        const double a_ = coef[2 * kstep], b_ = coef[2 * kstep + 1];
        ca = (T)a_;
        cb = (T)b_;
    }
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long nblk = (nv + 31) / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long nmine = (long)blockIdx.x < nblk ? (nblk - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    if (tid == 0) {
        for (int s = 0; s < NST; s++) rttc::mbar_init(&bar[s], 1);
        rttc::fence_mbar_init();
    }
    __syncthreads();
    // thread 0: the stencil run of this CTA's i-th block into stage i % NST
    auto issue = [&](long i) {
        const long b = blockIdx.x + i * (long)gridDim.x;
        uint64_t* br = &bar[i % NST];
        rttc::mbar_expect_tx(br, BLK_BYTES);
        rttc::bulk_g2s(stg + (i % NST) * BLK_ELEMS, st + b * BLK_ELEMS, BLK_BYTES, br);
    };
    if (tid == 0)
        for (long i = 0; i < NST - 1 && i < nmine; i++) issue(i);
    long i = 0, issued = nmine < NST - 1 ? nmine : NST - 1;
    bool ok = true;
    for (; i < nmine; i++) {
        // block i + NST - 1 goes into the stage block i - 1 used (released by the barrier ending iteration i - 1)
        if (issued < nmine) {
            if (tid == 0) issue(issued);
            issued++;
        }
        const int s = (int)(i % NST);
        const bool w = rttc::mbar_wait(&bar[s], (uint32_t)((i / NST) & 1));
        if (!__syncthreads_and(w)) {
            ok = false;
            break;
        }
        const S* sb = stg + s * BLK_ELEMS + lane;  // row j of this lane's node at sb[32 j]
        const long v = (blockIdx.x + i * (long)gridDim.x) * 32 + lane;
        const bool inb = v < nv;
        const bool act = inb && vact[v];
        T Au[3] = {T(0), T(0), T(0)};
        if (act) {
            const int x = (int)(v % vx), y = (int)((v / vx) % vy), z = (int)(v / ((long)vx * vy));
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const int k = warp + SB_WARPS * kk;
                if (k >= 27) break;
                const int jx = x + k % 3 - 1, jy = y + (k / 3) % 3 - 1, jz = z + k / 9 - 1;
                if (jx < 0 || jy < 0 || jz < 0 || jx >= vx || jy >= vy || jz >= vz) continue;
                const long nj = jx + (long)vx * (jy + (long)vy * jz);
                const T u0 = u[nj], u1 = u[nv + nj], u2 = u[2 * nv + nj];
                const S* sk = sb + k * 9 * 32;
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    T a0 = (T)st_val(sk + (3 * r) * 32), a1 = (T)st_val(sk + (3 * r + 1) * 32),
                      a2 = (T)st_val(sk + (3 * r + 2) * 32);
                    if (sizeof(S) == 2 && k == 13) {
                        a0 += (T)st_val(sb + (243 + 3 * r) * 32);
                        a1 += (T)st_val(sb + (243 + 3 * r + 1) * 32);
                        a2 += (T)st_val(sb + (243 + 3 * r + 2) * 32);
                    }
                    Au[r] += a0 * u0 + a1 * u1 + a2 * u2;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 3; r++) red[(warp * 3 + r) * 32 + lane] = Au[r];
        __syncthreads();
        if (warp < 3 && inb) {
            const int q = warp;
            T A3[3];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                A3[r] = red[r * 32 + lane];
#pragma unroll
                for (int w2 = 1; w2 < SB_WARPS; w2++) A3[r] += red[(3 * w2 + r) * 32 + lane];
            }
            const long oq = (long)q * nv + v;
            const T Aq = q == 0 ? A3[0] : (q == 1 ? A3[1] : A3[2]);
            if (MODE == 0) {
                out[oq] = act ? f[oq] - Aq : T(0);
            } else {
                T res = T(0), dn = T(0);
                if (act) {
                    T S9[9];
#pragma unroll
                    for (int e = 0; e < 9; e++) S9[e] = st_centre<T>(sb, 32, e);
                    const T a0 = S9[0], b0 = S9[1], c0 = S9[2], d0 = S9[3], e0 = S9[4], f0 = S9[5], g0 = S9[6],
                            h0 = S9[7], k0 = S9[8];
                    const T A = e0 * k0 - f0 * h0, B = -(d0 * k0 - f0 * g0), Cc = d0 * h0 - e0 * g0;
                    const T id = T(1) / (a0 * A + b0 * B + c0 * Cc);
                    const T i0 = q == 0 ? A : (q == 1 ? B : Cc);
                    const T i1 = q == 0 ? -(b0 * k0 - c0 * h0) : (q == 1 ? (a0 * k0 - c0 * g0) : -(a0 * h0 - b0 * g0));
                    const T i2 = q == 0 ? (b0 * f0 - c0 * e0) : (q == 1 ? -(a0 * f0 - c0 * d0) : (a0 * e0 - b0 * d0));
                    const T r0 = f[v] - A3[0], r1 = f[nv + v] - A3[1], r2 = f[2 * nv + v] - A3[2];
                    const T zq = (i0 * id) * r0 + (i1 * id) * r1 + (i2 * id) * r2;
                    if (MODE == 2) {
                        res = u[oq] + omega * zq;
                    } else {
                        dn = (kstep == 0 ? T(0) : ca * d[oq]) + cb * zq;
                        res = u[oq] + dn;
                    }
                }
                out[oq] = res;
                if (MODE == 3) d[oq] = dn;
            }
        }
        __syncthreads();  // the reduction buffer and stage s are free again
    }
    if (!ok) {
        for (long j = i; j < issued; j++) rttc::mbar_wait(&bar[j % NST], (uint32_t)((j / NST) & 1));
        if (tid == 0) errslot[0] = 1.0;
        for (long j = i; j < nmine; j++)
            for (int t = tid; t < 96; t += SB_BS) {
                const long v = (blockIdx.x + j * (long)gridDim.x) * 32 + (t & 31);
                if (v < nv) out[(long)(t >> 5) * nv + v] = T(NAN);
            }
    }
}

// smoother copies of level stencils (layout above); one thread per (node, row group)
__global__ void k_st_to_f32(long nv, long nvpad, const double* __restrict__ st, float* __restrict__ out) {
    const long n = nvpad * 243;
    for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n; o += (long)gridDim.x * blockDim.x) {
        const long blk = o / (243 * 32);
        const int j = (int)((o / 32) % 243), l = (int)(o & 31);
        const long v = blk * 32 + l;
        out[o] = v < nv ? (float)st[(long)j * nv + v] : 0.f;
    }
}

__device__ __forceinline__ uint16_t bf16_bits(double x) { return __bfloat16_as_ushort(__double2bfloat16(x)); }

// thread per (node, centre entry rc): the 26 off-centre entries of column rc are rounded, the
// centre entry takes their summed rounding error, stored as hi + lo
__global__ void k_st_to_bf16(long nv, long nvpad, const double* __restrict__ st, uint16_t* __restrict__ out) {
    const long n = nvpad * 9;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const long v = t % nvpad;
        const int rc = (int)(t / nvpad);
        uint16_t* ob = out + (v >> 5) * (252 * 32L) + (v & 31);
        if (v >= nv) {
            for (int k = 0; k < 27; k++) ob[(k * 9 + rc) * 32] = 0;
            ob[(243 + rc) * 32] = 0;
            continue;
        }
        double err = 0;
        for (int k = 0; k < 27; k++) {
            if (k == 13) continue;
            const double x = st[(long)(k * 9 + rc) * nv + v];
            const uint16_t b = bf16_bits(x);
            ob[(k * 9 + rc) * 32] = b;
            err += x - (double)__uint_as_float((uint32_t)b << 16);
        }
        const double c = st[(long)(117 + rc) * nv + v] + err;
        const uint16_t hi = bf16_bits(c);
        ob[(117 + rc) * 32] = hi;
        ob[(243 + rc) * 32] = bf16_bits(c - (double)__uint_as_float((uint32_t)hi << 16));
    }
}

// ratio-4 restriction, 8 lanes per coarse node: lane t sums the fine plane dz = t - 3
template <typename T>
__global__ void __launch_bounds__(ST_BS) k_restrict4_split8(int fnx, int fny, int fnz, int cnx, int cny, int cnz,
                                                            const uint8_t* __restrict__ cvact,
                                                            const T* __restrict__ rf, T* __restrict__ fc) {
    constexpr int R = 4;
    const int fvx = fnx + 1, fvy = fny + 1, fvz = fnz + 1;
    const int cvx = cnx + 1, cvy = cny + 1, cvz = cnz + 1;
    const long nvf = (long)fvx * fvy * fvz, nvc = (long)cvx * cvy * cvz;
    const int t = threadIdx.x & 7;
    const long ngroups = (long)gridDim.x * (blockDim.x >> 3);
    const long vend = ((nvc + ngroups - 1) / ngroups) * ngroups;
    for (long vc = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 3; vc < vend; vc += ngroups) {
        T s[3] = {T(0), T(0), T(0)};
        const bool inb = vc < nvc;
        if (inb && t < 7 && cvact[vc]) {
            const int X = (int)(vc % cvx), Y = (int)((vc / cvx) % cvy), Z = (int)(vc / ((long)cvx * cvy));
            const int dz = t - 3;
            const int z = R * Z + dz;
            if (z >= 0 && z < fvz) {
                const T wz = T(R - abs(dz));
                for (int dy = -(R - 1); dy <= R - 1; dy++) {
                    const int y = R * Y + dy;
                    if (y < 0 || y >= fvy) continue;
                    const T wyz = wz * T(R - abs(dy));
#pragma unroll
                    for (int dx = -(R - 1); dx <= R - 1; dx++) {
                        const int x = R * X + dx;
                        if (x < 0 || x >= fvx) continue;
                        const long vf = x + (long)fvx * (y + (long)fvy * z);
                        const T wgt = wyz * T(R - abs(dx)) * (T(1) / T(R * R * R));
                        s[0] += wgt * rf[vf];
                        s[1] += wgt * rf[nvf + vf];
                        s[2] += wgt * rf[2 * nvf + vf];
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            s[c] += __shfl_xor_sync(0xffffffffu, s[c], 1);
            s[c] += __shfl_xor_sync(0xffffffffu, s[c], 2);
            s[c] += __shfl_xor_sync(0xffffffffu, s[c], 4);
        }
        if (inb && t < 3) fc[(long)t * nvc + vc] = s[t];
    }
}


// f_c(X) = sum_{|d| < r} prod (r - |d|)/r * r_f(rX + d)
template <typename T, int R>
__global__ void __launch_bounds__(ST_BS) k_restrict(int fnx, int fny, int fnz, int cnx, int cny, int cnz,
                                                     const uint8_t* __restrict__ cvact, const T* __restrict__ rf,
                                                     T* __restrict__ fc) {
    const int fvx = fnx + 1, fvy = fny + 1, fvz = fnz + 1;
    const int cvx = cnx + 1, cvy = cny + 1, cvz = cnz + 1;
    const long nvf = (long)fvx * fvy * fvz, nvc = (long)cvx * cvy * cvz;
    for (long vc = blockIdx.x * (long)blockDim.x + threadIdx.x; vc < nvc; vc += (long)gridDim.x * blockDim.x) {
        const int X = (int)(vc % cvx), Y = (int)((vc / cvx) % cvy), Z = (int)(vc / ((long)cvx * cvy));
        T s[3] = {T(0), T(0), T(0)};
        if (cvact[vc]) {
            for (int dz = -(R - 1); dz <= R - 1; dz++) {
                const int z = R * Z + dz;
                if (z < 0 || z >= fvz) continue;
                const T wz = T(R - abs(dz));
                for (int dy = -(R - 1); dy <= R - 1; dy++) {
                    const int y = R * Y + dy;
                    if (y < 0 || y >= fvy) continue;
                    const T wyz = wz * T(R - abs(dy));
#pragma unroll
                    for (int dx = -(R - 1); dx <= R - 1; dx++) {
                        const int x = R * X + dx;
                        if (x < 0 || x >= fvx) continue;
                        const long vf = x + (long)fvx * (y + (long)fvy * z);
                        const T wgt = wyz * T(R - abs(dx)) * (T(1) / T(R * R * R));
                        s[0] += wgt * rf[vf];
                        s[1] += wgt * rf[nvf + vf];
                        s[2] += wgt * rf[2 * nvf + vf];
                    }
                }
            }
        }
        fc[vc] = s[0]; fc[nvc + vc] = s[1]; fc[2 * nvc + vc] = s[2];
    }
}

// u_f(x) += sum over the 8 corners of the coarse cell containing x of trilinear weights * u_c
template <typename T, int R>
__global__ void __launch_bounds__(ST_BS) k_prolong(int fnx, int fny, int fnz, int cnx, int cny, int cnz,
                                                    const uint8_t* __restrict__ fvact, const T* __restrict__ uc,
                                                    T* __restrict__ uf) {
    const int fvx = fnx + 1, fvy = fny + 1, fvz = fnz + 1;
    const int cvx = cnx + 1, cvy = cny + 1, cvz = cnz + 1;
    const long nvf = (long)fvx * fvy * fvz, nvc = (long)cvx * cvy * cvz;
    for (long vf = blockIdx.x * (long)blockDim.x + threadIdx.x; vf < nvf; vf += (long)gridDim.x * blockDim.x) {
        // every load depends on the indices only: the activity flag, the fine values and the
        // coarse corners are all in flight at once, and the flag decides only the store
        const bool act = fvact[vf];
        const int x = (int)(vf % fvx), y = (int)((vf / fvx) % fvy), z = (int)(vf / ((long)fvx * fvy));
        const int X0 = x / R, Y0 = y / R, Z0 = z / R;
        const int ox = x - R * X0, oy = y - R * Y0, oz = z - R * Z0;
        const T f0 = uf[vf], f1 = uf[nvf + vf], f2 = uf[2 * nvf + vf];
        T s[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int a = i & 1, b = (i >> 1) & 1, c = i >> 2;
            const int wx = a ? ox : R - ox, wy = b ? oy : R - oy, wz = c ? oz : R - oz;
            if (wx == 0 || wy == 0 || wz == 0) continue;  // also keeps the corner inside the coarse box
            const long vc = (X0 + a) + (long)cvx * ((Y0 + b) + (long)cvy * (Z0 + c));
            const T wgt = T(wx * wy * wz) * (T(1) / T(R * R * R));
            s[0] += wgt * uc[vc];
            s[1] += wgt * uc[nvc + vc];
            s[2] += wgt * uc[2 * nvc + vc];
        }
        if (act) {
            uf[vf] = f0 + s[0];
            uf[nvf + vf] = f1 + s[1];
            uf[2 * nvf + vf] = f2 + s[2];
        }
    }
}

// ---------------------------------------------------------------------------
// Galerkin assembly of the first coarse level directly from the elements:
// for every coarse cell M = sum_e rho_e^p Q_pos(e), Q_pos = P_pos^T KE P_pos,
// then M's 3x3 blocks are added into the 8 corner nodes' stencils.  Cells are
// processed in 8 parity colours so no two cells of one launch share a node
// (deterministic, no atomics).  Elements touching a fixed node take the
// Dirichlet form of grid/Grid.cu:465-490 and are computed explicitly.
// ---------------------------------------------------------------------------
constexpr int GAL_CELLS = 8;
constexpr int GAL_BS = 288;  // 2 entries of the 576-entry cell matrix per thread

__device__ __forceinline__ double interp_w(int off, int corner, int R) {
    return (double)(R - abs(off - R * corner)) / (double)R;
}

template <int R>
__global__ void __launch_bounds__(GAL_BS) k_galerkin_cells(int fnx, int fny, int fnz, int cnx, int cny, int cnz,
                                                           int color, const uint8_t* __restrict__ ceact,
                                                           const float* __restrict__ w,
                                                           const uint8_t* __restrict__ vfix,
                                                           const double* __restrict__ Q, const double* __restrict__ KEg,
                                                           double* __restrict__ st) {
    constexpr int NP = R * R * R;
    __shared__ double sw[GAL_CELLS][NP];
    __shared__ int scell[GAL_CELLS];
    __shared__ int sfixed[GAL_CELLS];
    const int fvx = fnx + 1, fvy = fny + 1;
    const int cvx = cnx + 1, cvy = cny + 1, cvz = cnz + 1;
    const long nvc = (long)cvx * cvy * cvz;
    const int px = color & 1, py = (color >> 1) & 1, pz = (color >> 2) & 1;
    const int ccx = (cnx - px + 1) / 2, ccy = (cny - py + 1) / 2, ccz = (cnz - pz + 1) / 2;
    const long ncells = (long)ccx * ccy * ccz;
    const long ngroups = (ncells + GAL_CELLS - 1) / GAL_CELLS;
    for (long g = blockIdx.x; g < ngroups; g += gridDim.x) {
        __syncthreads();
        if (threadIdx.x < GAL_CELLS) {
            long t = g * GAL_CELLS + threadIdx.x;
            int cid = -1;
            if (t < ncells) {
                int X = px + 2 * (int)(t % ccx), Y = py + 2 * (int)((t / ccx) % ccy), Z = pz + 2 * (int)(t / ((long)ccx * ccy));
                if (ceact[X + (long)cnx * (Y + (long)cny * Z)]) cid = X + cnx * (Y + cny * Z);
            }
            scell[threadIdx.x] = cid;
            sfixed[threadIdx.x] = 0;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < GAL_CELLS * NP; i += blockDim.x) {
            const int c = i / NP, pos = i % NP;
            double wv = 0;
            const int cid = scell[c];
            if (cid >= 0) {
                const int X = cid % cnx, Y = (cid / cnx) % cny, Z = cid / (cnx * cny);
                const int a = pos % R, b = (pos / R) % R, cc = pos / (R * R);
                const int ex = R * X + a, ey = R * Y + b, ez = R * Z + cc;
                if (ex < fnx && ey < fny && ez < fnz) {
                    wv = w[ex + (long)fnx * (ey + (long)fny * ez)];
                    if (vfix != nullptr && wv != 0) {
                        bool fx = false;
                        for (int j = 0; j < 8; j++)
                            fx |= vfix[(ex + (j & 1)) + (long)fvx * ((ey + ((j >> 1) & 1)) + (long)fvy * (ez + (j >> 2)))] != 0;
                        if (fx) { sfixed[c] = 1; wv = -1.0 - wv; }  // marker: handled explicitly below
                    }
                }
            }
            sw[c][pos] = wv;
        }
        __syncthreads();
        // dense part: M[c][t] = sum_pos w[c][pos] Q[pos][t] over non-fixed elements
        double acc[GAL_CELLS][2];
#pragma unroll
        for (int c = 0; c < GAL_CELLS; c++) acc[c][0] = acc[c][1] = 0;
        const int t0 = threadIdx.x, t1 = threadIdx.x + GAL_BS;
        for (int pos = 0; pos < NP; pos++) {
            const double q0 = Q[(long)pos * 576 + t0], q1 = Q[(long)pos * 576 + t1];
#pragma unroll
            for (int c = 0; c < GAL_CELLS; c++) {
                const double wv = sw[c][pos] > 0 ? sw[c][pos] : 0.0;
                acc[c][0] += wv * q0;
                acc[c][1] += wv * q1;
            }
        }
        // elements with fixed nodes: rows/cols dropped, 1e6 * P^T P diagonal
        for (int c = 0; c < GAL_CELLS; c++) {
            if (!sfixed[c]) continue;
            const int cid = scell[c];
            const int X = cid % cnx, Y = (cid / cnx) % cny, Z = cid / (cnx * cny);
            for (int pos = 0; pos < NP; pos++) {
                const double wm = sw[c][pos];
                if (wm >= 0) continue;
                const double pen = -1.0 - wm;
                const int a = pos % R, b = (pos / R) % R, cc = pos / (R * R);
                const int ex = R * X + a, ey = R * Y + b, ez = R * Z + cc;
#pragma unroll
                for (int half = 0; half < 2; half++) {
                    const int t = half ? t1 : t0;
                    const int mrow = t / 24, ncol = t % 24;
                    const int m = mrow / 3, row = mrow % 3, n = ncol / 3, col = ncol % 3;
                    double s = 0;
                    for (int j = 0; j < 8; j++) {
                        const int oj[3] = {a + (j & 1), b + ((j >> 1) & 1), cc + (j >> 2)};
                        const double pj = interp_w(oj[0], m & 1, R) * interp_w(oj[1], (m >> 1) & 1, R) *
                                          interp_w(oj[2], m >> 2, R);
                        if (pj == 0) continue;
                        const bool fj = vfix[(ex + (j & 1)) + (long)fvx * ((ey + ((j >> 1) & 1)) + (long)fvy * (ez + (j >> 2)))];
                        for (int k = 0; k < 8; k++) {
                            const int ok[3] = {a + (k & 1), b + ((k >> 1) & 1), cc + (k >> 2)};
                            const double pk = interp_w(ok[0], n & 1, R) * interp_w(ok[1], (n >> 1) & 1, R) *
                                              interp_w(ok[2], n >> 2, R);
                            if (pk == 0) continue;
                            const bool fk = vfix[(ex + (k & 1)) + (long)fvx * ((ey + ((k >> 1) & 1)) + (long)fvy * (ez + (k >> 2)))];
                            double kk;
                            if (fj || fk) kk = (j == k && row == col) ? 1e6 : 0.0;
                            else kk = pen * KEg[(3 * j + row) * 24 + 3 * k + col];
                            s += pj * kk * pk;
                        }
                    }
                    acc[c][half] += s;
                }
            }
        }
        // scatter: entry t = (3m+row)*24 + 3n+col -> node corner m, neighbour k(n-m)
#pragma unroll
        for (int c = 0; c < GAL_CELLS; c++) {
            const int cid = scell[c];
            if (cid < 0) continue;
            const int X = cid % cnx, Y = (cid / cnx) % cny, Z = cid / (cnx * cny);
#pragma unroll
            for (int half = 0; half < 2; half++) {
                const int t = half ? t1 : t0;
                const int mrow = t / 24, ncol = t % 24;
                const int m = mrow / 3, row = mrow % 3, n = ncol / 3, col = ncol % 3;
                const int dx = (n & 1) - (m & 1), dy = ((n >> 1) & 1) - ((m >> 1) & 1), dz = (n >> 2) - (m >> 2);
                const int k = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
                const long vc = (X + (m & 1)) + (long)cvx * ((Y + ((m >> 1) & 1)) + (long)cvy * (Z + (m >> 2)));
                st[(long)(k * 9 + row * 3 + col) * nvc + vc] += acc[c][half];
            }
        }
    }
}

// A_c = P^T A_f P for a dyadic (ratio 2) level from the finer stencil
__global__ void __launch_bounds__(ST_BS) k_galerkin_dyadic(int fnx, int fny, int fnz, int cnx, int cny, int cnz,
                                                           const uint8_t* __restrict__ fvact,
                                                           const uint8_t* __restrict__ cvact,
                                                           const double* __restrict__ stf, double* __restrict__ stc) {
    const int fvx = fnx + 1, fvy = fny + 1, fvz = fnz + 1;
    const int cvx = cnx + 1, cvy = cny + 1, cvz = cnz + 1;
    const long nvf = (long)fvx * fvy * fvz, nvc = (long)cvx * cvy * cvz;
    const double wtab[4] = {1.0, 0.5, 0.25, 0.125};
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nvc * 9; t += (long)gridDim.x * blockDim.x) {
        const long vc = t % nvc;
        const int rc = (int)(t / nvc);
        const int X = (int)(vc % cvx), Y = (int)((vc / cvx) % cvy), Z = (int)(vc / ((long)cvx * cvy));
        double acc[27];
#pragma unroll
        for (int s = 0; s < 27; s++) acc[s] = 0;
        if (cvact[vc]) {
            for (int i = 0; i < 27; i++) {
                const int dx = i % 3 - 1, dy = (i / 3) % 3 - 1, dz = i / 9 - 1;
                const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                if (x < 0 || y < 0 || z < 0 || x >= fvx || y >= fvy || z >= fvz) continue;
                const long vn = x + (long)fvx * (y + (long)fvy * z);
                if (!fvact[vn]) continue;
                const double wi = wtab[abs(dx) + abs(dy) + abs(dz)];
                for (int j = 0; j < 27; j++) {
                    const int mx = x + j % 3 - 1, my = y + (j / 3) % 3 - 1, mz = z + j / 9 - 1;
                    if (mx < 0 || my < 0 || mz < 0 || mx >= fvx || my >= fvy || mz >= fvz) continue;
                    const double kij = stf[(long)(j * 9 + rc) * nvf + vn] * wi;
                    if (kij == 0) continue;
#pragma unroll
                    for (int s = 0; s < 27; s++) {
                        const int ax = abs(2 * (X + s % 3 - 1) - mx), ay = abs(2 * (Y + (s / 3) % 3 - 1) - my),
                                  az = abs(2 * (Z + s / 9 - 1) - mz);
                        if (ax >= 2 || ay >= 2 || az >= 2) continue;
                        acc[s] += wtab[ax + ay + az] * kij;
                    }
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 27; s++) stc[(long)(s * 9 + rc) * nvc + vc] = acc[s];
    }
}

__global__ void k_d2f(long n, const double* __restrict__ a, float* __restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (float)a[i];
}


}  // namespace

namespace rtk {

// stencil kernels on level 1 (the ratio-4 level, by far the largest) report under their own
// name, so a profile separates them from the small levels below
#define LVL_NAME(lvl, f64, base) \
    ((lvl) == 1 ? ((f64) ? base "_f64_l1" : base "_f32_l1") : ((f64) ? base "_f64" : base "_f32"))

template <typename T>
static const T* stp(rt_level& L);
template <>
const double* stp<double>(rt_level& L) { return L.st; }
template <>
const float* stp<float>(rt_level& L) { return L.st32; }

// the FP32 level kernels: bulk-copy stencil kernel over the blocked FP32 (or BF16) copy
template <int MODE, typename S>
static int launch_bulk(rt_hier* h, int lvl, const char* name, const S* st, const float* u, const float* f, float* out,
                       float* d, double omega, const double* coef, int kstep) {
    rt_level& L = h->L[lvl];
    const long nblk = (L.nv + 31) / 32;
    const long cap = (long)h->ctx->sm_count * sb_ctas_per_sm<S>();
    const unsigned grid = (unsigned)(nblk < cap ? nblk : cap);
    return rt_launch(h->ctx, name, [&] {
        k_st_bulk<float, MODE, S><<<grid, SB_BS, sb_smem<float, S>(), h->ctx->stream>>>(
            L.nx, L.ny, L.nz, L.vact, st, u, f, out, d, (float)omega, coef, kstep, h->scal + RT_SCAL_ERR);
    });
}

// the lane-split kernel on an FP32 / BF16 blocked copy
template <int MODE, typename S>
static int launch_split(rt_hier* h, int lvl, const char* name, const S* st, const float* u, const float* f, float* out,
                        float* d, double omega, const double* coef, int kstep) {
    rt_level& L = h->L[lvl];
    return rt_launch(h->ctx, name, [&] {
        k_st_split4<float, MODE, S><<<grid_for(h->ctx, 4 * L.nv, ST_BS), ST_BS, 0, h->ctx->stream>>>(
            L.nx, L.ny, L.nz, L.vact, st, u, f, out, d, (float)omega, coef, kstep);
    });
}

template <int MODE, typename S>
static int launch_f32(rt_hier* h, int lvl, const char* name, const S* st, const float* u, const float* f, float* out,
                      float* d, double omega, const double* coef, int kstep) {
    if (h->st_variant[sizeof(S) == 2 ? 1 : 0] == 1)
        return launch_bulk<MODE, S>(h, lvl, name, st, u, f, out, d, omega, coef, kstep);
    return launch_split<MODE, S>(h, lvl, name, st, u, f, out, d, omega, coef, kstep);
}

template <typename T>
int st_residual(rt_hier* h, int lvl, const T* u, const T* f, T* r) {
    rt_level& L = h->L[lvl];
    if constexpr (sizeof(T) == 4)
        return launch_f32<0, float>(h, lvl, LVL_NAME(lvl, false, "st_residual"), L.st32, u, f, r, nullptr, 0.0,
                                    nullptr, 0);
    return rt_launch(h->ctx, LVL_NAME(lvl, true, "st_residual"), [&] {
        k_st_split4<T, 0><<<grid_for(h->ctx, 4 * L.nv, ST_BS), ST_BS, 0, h->ctx->stream>>>(
            L.nx, L.ny, L.nz, L.vact, stp<T>(L), u, f, r, nullptr, T(0), nullptr, 0);
    });
}

template <typename T>
int st_gs(rt_hier* h, int lvl, T* u, const T* f, bool backward) {
    rt_level& L = h->L[lvl];
    for (int cc = 0; cc < 8; cc++) {
        int col = backward ? 7 - cc : cc;
        long ncol = (long)((L.vx - (col & 1) + 1) / 2) * ((L.vy - ((col >> 1) & 1) + 1) / 2) *
                    ((L.vz - ((col >> 2) & 1) + 1) / 2);
        RT_CHECK(rt_launch(h->ctx, LVL_NAME(lvl, sizeof(T) == 8, "st_gs"), [&] {
            k_st_gs<T><<<grid_for(h->ctx, ncol, ST_BS), ST_BS, 0, h->ctx->stream>>>(L.nx, L.ny, L.nz, col, backward,
                                                                                    L.vact, stp<T>(L), u, f);
        }));
    }
    return RT_OK;
}

// the FP32 smoother reads the BF16 stencil copy when rt_params.coarse_bf16 is set
template <typename T>
static bool use_bf16(rt_hier* h, rt_level& L) {
    return sizeof(T) == 4 && h->P.coarse_bf16 && L.st16;
}

template <typename T>
int st_jacobi(rt_hier* h, int lvl, const T* u, const T* f, T* unew, double omega) {
    rt_level& L = h->L[lvl];
    if constexpr (sizeof(T) == 4) {
        if (use_bf16<T>(h, L))
            return launch_f32<2, uint16_t>(h, lvl, lvl == 1 ? "st_jacobi_bf16_l1" : "st_jacobi_bf16", L.st16, u, f,
                                           unew, nullptr, omega, nullptr, 0);
        return launch_f32<2, float>(h, lvl, LVL_NAME(lvl, false, "st_jacobi"), L.st32, u, f, unew, nullptr, omega,
                                    nullptr, 0);
    }
    return rt_launch(h->ctx, LVL_NAME(lvl, true, "st_jacobi"), [&] {
        k_st_split4<T, 2><<<grid_for(h->ctx, 4 * L.nv, ST_BS), ST_BS, 0, h->ctx->stream>>>(
            L.nx, L.ny, L.nz, L.vact, stp<T>(L), u, f, unew, nullptr, (T)omega, nullptr, 0);
    });
}

template <typename T>
int st_cheby(rt_hier* h, int lvl, const T* u, const T* f, T* unew, T* d, const double* coef, int kstep) {
    rt_level& L = h->L[lvl];
    if constexpr (sizeof(T) == 4) {
        if (use_bf16<T>(h, L))
            return launch_f32<3, uint16_t>(h, lvl, lvl == 1 ? "st_cheby_bf16_l1" : "st_cheby_bf16", L.st16, u, f,
                                           unew, d, 0.0, coef, kstep);
        return launch_f32<3, float>(h, lvl, LVL_NAME(lvl, false, "st_cheby"), L.st32, u, f, unew, d, 0.0, coef,
                                    kstep);
    }
    return rt_launch(h->ctx, LVL_NAME(lvl, true, "st_cheby"), [&] {
        k_st_split4<T, 3><<<grid_for(h->ctx, 4 * L.nv, ST_BS), ST_BS, 0, h->ctx->stream>>>(
            L.nx, L.ny, L.nz, L.vact, stp<T>(L), u, f, unew, d, T(0), coef, kstep);
    });
}
// co-resident blocks per SM of the fused kernels (queried once per context): the streaming form
// in coop_blocks_per_sm, the resident form (RES_SMEM of shared memory per block) in res_blocks_per_sm
static int coop_blocks(rt_hier* h, bool resident = false) {
    rt_ctx* c = h->ctx;
    if (c->coop_blocks_per_sm < 0) {
        int coop = 0, nb = 0, nr = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
        if (coop) {
            int a = 0, b = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_st_cheby_coop<float>, ST_BS, 0) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_st_cheby_coop<uint16_t>, ST_BS, 0) == cudaSuccess)
                nb = a < b ? a : b;
            a = b = 0;
            if (cudaFuncSetAttribute(k_st_cheby_res<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RES_SMEM) ==
                    cudaSuccess &&
                cudaFuncSetAttribute(k_st_cheby_res<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)RES_SMEM) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_st_cheby_res<float>, ST_BS, RES_SMEM) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_st_cheby_res<uint16_t>, ST_BS, RES_SMEM) ==
                    cudaSuccess)
                nr = a < b ? a : b;
        }
        cudaGetLastError();
        c->coop_blocks_per_sm = nb;
        c->res_blocks_per_sm = nr;
    }
    return resident ? c->res_blocks_per_sm : c->coop_blocks_per_sm;
}

bool st_cheby_fused_ok(rt_hier* h) { return coop_blocks(h) > 0; }

int st_cheby_fused(rt_hier* h, int lvl, float* u, const float* f, float* tmp, float* d, const double* coef,
                   int nsteps) {
    rt_level& L = h->L[lvl];
    const int nb = coop_blocks(h);
    if (nb <= 0) return rt_fail(h->ctx, RT_ECUDA, "the device cannot run the fused Chebyshev sweeps");
    if (nsteps < 1 || nsteps > RT_CHEBY_MAXK) return rt_fail(h->ctx, RT_EINVAL, "fused Chebyshev: 1..16 steps");
    // one 4-lane group per node: the resident form when all groups fit on the device at once,
    // else the streaming form over a node loop
    const long want = rt_blocks(4 * L.nv, ST_BS);
    const long cap = (long)nb * h->ctx->sm_count;
    const bool resident = !((h->cheby_stream >> lvl) & 1u) && want <= (long)coop_blocks(h, true) * h->ctx->sm_count;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(resident ? want : (want < cap ? want : cap)));
    cfg.blockDim = dim3(ST_BS);
    cfg.dynamicSmemBytes = resident ? RES_SMEM : 0;
    cfg.stream = h->ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    unsigned* bar = reinterpret_cast<unsigned*>(h->scal + RT_SCAL_GBAR + lvl);
    double* err = h->scal + RT_SCAL_ERR;
    const long spin = (long)h->ctx->wait_limit;
    const bool bf = use_bf16<float>(h, L);
    cudaError_t e = cudaSuccess;
    RT_CHECK(rt_launch(h->ctx, bf ? (lvl == 1 ? "st_cheby_fused_bf16_l1" : "st_cheby_fused_bf16")
                                  : LVL_NAME(lvl, false, "st_cheby_fused"),
                       [&] {
                           if (resident && bf)
                               e = cudaLaunchKernelEx(&cfg, k_st_cheby_res<uint16_t>, L.nx, L.ny, L.nz,
                                                      (const uint8_t*)L.vact, (const uint16_t*)L.st16, u, f, tmp, d,
                                                      coef, nsteps, bar, err, spin);
                           else if (resident)
                               e = cudaLaunchKernelEx(&cfg, k_st_cheby_res<float>, L.nx, L.ny, L.nz,
                                                      (const uint8_t*)L.vact, (const float*)L.st32, u, f, tmp, d,
                                                      coef, nsteps, bar, err, spin);
                           else if (bf)
                               e = cudaLaunchKernelEx(&cfg, k_st_cheby_coop<uint16_t>, L.nx, L.ny, L.nz,
                                                      (const uint8_t*)L.vact, (const uint16_t*)L.st16, u, f, tmp, d,
                                                      coef, nsteps, bar, err, spin);
                           else
                               e = cudaLaunchKernelEx(&cfg, k_st_cheby_coop<float>, L.nx, L.ny, L.nz,
                                                      (const uint8_t*)L.vact, (const float*)L.st32, u, f, tmp, d,
                                                      coef, nsteps, bar, err, spin);
                       }));
    if (e != cudaSuccess)
        return rt_fail(h->ctx, RT_ECUDA, "fused Chebyshev launch failed: %s", cudaGetErrorString(e));
    return RT_OK;
}

template int st_cheby<double>(rt_hier*, int, const double*, const double*, double*, double*, const double*, int);
template int st_cheby<float>(rt_hier*, int, const float*, const float*, float*, float*, const double*, int);

template <typename T>
int restrict_(rt_hier* h, int lvl, const T* rf, T* fc) {
    rt_level& F = h->L[lvl - 1];
    rt_level& Cc = h->L[lvl];
    return rt_launch(h->ctx, sizeof(T) == 8 ? "restrict_f64" : "restrict_f32", [&] {
        unsigned g = grid_for(h->ctx, Cc.nv, ST_BS);
        if (Cc.ratio == 4)
            k_restrict4_split8<T><<<grid_for(h->ctx, 8 * Cc.nv, ST_BS), ST_BS, 0, h->ctx->stream>>>(
                F.nx, F.ny, F.nz, Cc.nx, Cc.ny, Cc.nz, Cc.vact, rf, fc);
        else
            k_restrict<T, 2><<<g, ST_BS, 0, h->ctx->stream>>>(F.nx, F.ny, F.nz, Cc.nx, Cc.ny, Cc.nz, Cc.vact, rf, fc);
    });
}

template <typename T>
int prolong_add(rt_hier* h, int lvl, const T* uc, T* uf) {
    rt_level& F = h->L[lvl];
    rt_level& Cc = h->L[lvl + 1];
    return rt_launch(h->ctx, sizeof(T) == 8 ? "prolong_f64" : "prolong_f32", [&] {
        unsigned g = grid_for(h->ctx, F.nv, ST_BS);
        if (Cc.ratio == 4)
            k_prolong<T, 4><<<g, ST_BS, 0, h->ctx->stream>>>(F.nx, F.ny, F.nz, Cc.nx, Cc.ny, Cc.nz, F.vact, uc, uf);
        else
            k_prolong<T, 2><<<g, ST_BS, 0, h->ctx->stream>>>(F.nx, F.ny, F.nz, Cc.nx, Cc.ny, Cc.nz, F.vact, uc, uf);
    });
}

// Q_pos = P_pos^T KE P_pos for every element position in a coarse cell
static int build_Q(rt_hier* h, int R, double** Qdev) {
    const int NP = R * R * R;
    std::vector<double> Qh((size_t)NP * 576);
    for (int pos = 0; pos < NP; pos++) {
        int a = pos % R, b = (pos / R) % R, c = pos / (R * R);
        double P[8][8];
        for (int j = 0; j < 8; j++) {
            int o[3] = {a + (j & 1), b + ((j >> 1) & 1), c + (j >> 2)};
            for (int m = 0; m < 8; m++) {
                int mm[3] = {m & 1, (m >> 1) & 1, m >> 2};
                double wv = 1;
                for (int t = 0; t < 3; t++) wv *= (double)(R - abs(o[t] - R * mm[t])) / R;
                P[j][m] = wv;
            }
        }
        for (int m = 0; m < 8; m++)
            for (int row = 0; row < 3; row++)
                for (int n = 0; n < 8; n++)
                    for (int col = 0; col < 3; col++) {
                        double s = 0;
                        for (int j = 0; j < 8; j++) {
                            if (P[j][m] == 0) continue;
                            for (int k = 0; k < 8; k++)
                                s += P[j][m] * h->KE[(3 * j + row) * 24 + 3 * k + col] * P[k][n];
                        }
                        Qh[(size_t)pos * 576 + (3 * m + row) * 24 + 3 * n + col] = s;
                    }
    }
    RT_CUDA(h->ctx, cudaMalloc(Qdev, sizeof(double) * Qh.size()));
    RT_CUDA(h->ctx, cudaMemcpyAsync(*Qdev, Qh.data(), sizeof(double) * Qh.size(), cudaMemcpyHostToDevice,
                                    h->ctx->stream));
    return RT_OK;
}

int galerkin_from_elements(rt_hier* h) {
    rt_level& F = h->L[0];
    rt_level& Cc = h->L[1];
    const int R = Cc.ratio;
    if (h->Qgal == nullptr || h->Qgal_ratio != R) {
        if (h->Qgal) cudaFree(h->Qgal);
        h->Qgal = nullptr;
        RT_CHECK(build_Q(h, R, &h->Qgal));
        h->Qgal_ratio = R;
    }
    const double* Q = h->Qgal;
    RT_CUDA(h->ctx, cudaMemsetAsync(Cc.st, 0, sizeof(double) * 243 * Cc.nv, h->ctx->stream));
    for (int color = 0; color < 8; color++) {
        long ccells = (long)((Cc.nx - (color & 1) + 1) / 2) * ((Cc.ny - ((color >> 1) & 1) + 1) / 2) *
                      ((Cc.nz - (color >> 2) + 1) / 2);
        long groups = (ccells + GAL_CELLS - 1) / GAL_CELLS;
        if (groups == 0) continue;
        unsigned g = (unsigned)(groups < (long)h->ctx->sm_count * 8 ? groups : (long)h->ctx->sm_count * 8);
        RT_CHECK(rt_launch(h->ctx, "galerkin_cells", [&] {
            const uint8_t* vf = h->has_support ? h->vfix : nullptr;
            if (R == 4)
                k_galerkin_cells<4><<<g, GAL_BS, 0, h->ctx->stream>>>(F.nx, F.ny, F.nz, Cc.nx, Cc.ny, Cc.nz, color,
                                                                      Cc.eact, h->w, vf, Q, h->KE_dev, Cc.st);
            else
                k_galerkin_cells<2><<<g, GAL_BS, 0, h->ctx->stream>>>(F.nx, F.ny, F.nz, Cc.nx, Cc.ny, Cc.nz, color,
                                                                      Cc.eact, h->w, vf, Q, h->KE_dev, Cc.st);
        }));
    }
    return RT_OK;
}

int galerkin_from_stencil(rt_hier* h, int lvl) {
    rt_level& F = h->L[lvl - 1];
    rt_level& Cc = h->L[lvl];
    return rt_launch(h->ctx, "galerkin_dyadic", [&] {
        k_galerkin_dyadic<<<grid_for(h->ctx, Cc.nv * 9, ST_BS), ST_BS, 0, h->ctx->stream>>>(
            F.nx, F.ny, F.nz, Cc.nx, Cc.ny, Cc.nz, F.vact, Cc.vact, F.st, Cc.st);
    });
}

int d2f(rt_hier* h, long n, const double* a, float* b) {
    return rt_launch(h->ctx, "d2f", [&] { k_d2f<<<grid_for(h->ctx, n, 256), 256, 0, h->ctx->stream>>>(n, a, b); });
}

// dynamic shared-memory limits of the bulk-copy stencil kernels, set once per device
int init_stencil_kernels(rt_ctx* c) {
    cudaError_t e[5] = {
        cudaFuncSetAttribute(k_st_bulk<float, 0, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sb_smem<float, float>()),
        cudaFuncSetAttribute(k_st_bulk<float, 2, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sb_smem<float, float>()),
        cudaFuncSetAttribute(k_st_bulk<float, 3, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sb_smem<float, float>()),
        cudaFuncSetAttribute(k_st_bulk<float, 2, uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sb_smem<float, uint16_t>()),
        cudaFuncSetAttribute(k_st_bulk<float, 3, uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sb_smem<float, uint16_t>())};
    for (cudaError_t x : e)
        if (x != cudaSuccess) return rt_fail(c, RT_ECUDA, "stencil kernel attributes: %s", cudaGetErrorString(x));
    return RT_OK;
}

// the FP32 (and, with rt_params.coarse_bf16, BF16) smoother copies of level lvl's stencils
int stencil_copies(rt_hier* h, int lvl) {
    rt_level& L = h->L[lvl];
    const long nvpad = (L.nv + 31) / 32 * 32;
    RT_CHECK(rt_launch(h->ctx, "stencil_f32", [&] {
        k_st_to_f32<<<grid_for(h->ctx, nvpad * 243, 256), 256, 0, h->ctx->stream>>>(L.nv, nvpad, L.st, L.st32);
    }));
    if (!h->P.coarse_bf16) return RT_OK;
    return rt_launch(h->ctx, "stencil_bf16", [&] {
        k_st_to_bf16<<<grid_for(h->ctx, nvpad * 9, 256), 256, 0, h->ctx->stream>>>(L.nv, nvpad, L.st, L.st16);
    });
}

template int st_residual<double>(rt_hier*, int, const double*, const double*, double*);
template int st_residual<float>(rt_hier*, int, const float*, const float*, float*);
template int st_gs<double>(rt_hier*, int, double*, const double*, bool);
template int st_gs<float>(rt_hier*, int, float*, const float*, bool);
template int st_jacobi<double>(rt_hier*, int, const double*, const double*, double*, double);
template int st_jacobi<float>(rt_hier*, int, const float*, const float*, float*, double);
template int restrict_<double>(rt_hier*, int, const double*, double*);
template int restrict_<float>(rt_hier*, int, const float*, float*);
template int prolong_add<double>(rt_hier*, int, const double*, double*);
template int prolong_add<float>(rt_hier*, int, const float*, float*);

}  // namespace rtk
