// rt_misc.cu — reductions, vector updates, load projection, filter, OC and
// occupancy set-up kernels.
//
// Restates:
//   block_dot/norm kernels, dot/norm, parallel_sum_d, parallel_maxabs   culib/lib.cuh:521-1137
//     (here: single-pass deterministic block partials + one fixed-order final
//      sum, result left on the device)
//   forceProject / getForceSupport / setForceSupport   optimization/projection.cu:165-369
//   displacementProject                                 optimization/projection.cpp:374-392
//   filterSensitivity_kernel                            grid/Grid.cu:2323-2409
//   trySensMultiplier_kernel                            optimization/optimization.cu:136-162
//   cubeGridSetSolidVertices_kernel / setSolidElementFromFineGrid_kernel  grid/Grid.cu:2555-2632
//   mark_surface_nodes_kernel                           grid/Grid.cu:2005-2039
#include <cuda_runtime.h>

#include "rt_internal.h"

namespace {

constexpr int RB = 256;  // reduction block size
constexpr int XR_U = 4;  // grid strides per trip in the fused update + reduction kernels

unsigned gridN(rt_ctx* c, long n, int bs = 256) {
    long b = rt_blocks(n, bs);
    long cap = (long)c->sm_count * 16;
    return (unsigned)(b < 1 ? 1 : (b < cap ? b : cap));
}

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* __restrict__ partials) {
    __shared__ double sh[NV][RB / 32];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double x = threadIdx.x < RB / 32 ? sh[k][threadIdx.x] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (threadIdx.x == 0) partials[blockIdx.x * NV + k] = x;
        }
    }
}

// sum NV interleaved partial arrays in a fixed order (deterministic)
template <int NV>
__global__ void k_final_sum(int nblocks, const double* __restrict__ partials, double* __restrict__ out) {
    __shared__ double sh[NV][32];
    for (int k = 0; k < NV; k++) {
        double x = 0;
        for (int b = threadIdx.x; b < nblocks; b += 32) x += partials[b * NV + k];
        sh[k][threadIdx.x] = x;
    }
    __syncwarp();
    if (threadIdx.x < NV) {
        double s = 0;
        for (int i = 0; i < 32; i++) s += sh[threadIdx.x][i];
        out[threadIdx.x] = s;
    }
}

__global__ void __launch_bounds__(RB) k_dot(long n, const double* __restrict__ a, const double* __restrict__ b,
                                            double* __restrict__ partials) {
    double v[1] = {0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[0] += a[i] * b[i];
    block_reduce_store<1>(v, partials);
}

// (a.b, a.c) in one pass
__global__ void __launch_bounds__(RB) k_dot2(long n, const double* __restrict__ a, const double* __restrict__ b,
                                             const double* __restrict__ c, double* __restrict__ partials) {
    double v[2] = {0, 0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double x = a[i];
        v[0] += x * b[i];
        v[1] += x * c[i];
    }
    block_reduce_store<2>(v, partials);
}

__global__ void k_axpy(long n, double a, const double* __restrict__ x, double* __restrict__ y) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) y[i] += a * x[i];
}

__global__ void k_f2d(long n, const float* __restrict__ a, double* __restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (double)a[i];
}

// b = float(a / s), s = sqrt(s_dev[0]) (scales the FP32 right-hand side to unit norm)
__global__ void k_d2f_scaled(long n, const double* __restrict__ a, float* __restrict__ b, const double* __restrict__ s) {
    const double inv = 1.0 / sqrt(fmax(s[0], 1e-300));
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (float)(a[i] * inv);
}
__global__ void k_f2d_scaled(long n, const float* __restrict__ a, double* __restrict__ b, const double* __restrict__ s) {
    const double sc = sqrt(fmax(s[0], 1e-300));
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] = (double)a[i] * sc;
}

// b += a * sqrt(s) (a coarse correction computed on a right-hand side scaled by 1 / sqrt(s))
__global__ void k_f2d_scaled_add(long n, const float* __restrict__ a, double* __restrict__ b,
                                 const double* __restrict__ s) {
    const double sc = sqrt(fmax(s[0], 1e-300));
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        b[i] += (double)a[i] * sc;
}

// x += alpha p, r -= alpha q, rold = r(before);  alpha = num / den read on the device
__global__ void k_pcg_xr(long n, const double* __restrict__ num, const double* __restrict__ den, double* __restrict__ x,
                         double* __restrict__ r, const double* __restrict__ p, const double* __restrict__ q,
                         double* __restrict__ rold) {
    const double alpha = den[0] != 0.0 ? num[0] / den[0] : 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double ri = r[i];
        rold[i] = ri;
        x[i] += alpha * p[i];
        r[i] = ri - alpha * q[i];
    }
}

// k_pcg_xr and r.r of the updated r in the same pass (partials as k_dot's: same grid, same order)
// r32 (optional): the new residual scaled by 1 / sqrt(rr_old) and rounded to FP32, the right-hand
// side of the next FP32 V-cycle; rr_old (the r.r before this update) is kept in scale_out
__global__ void __launch_bounds__(RB) k_pcg_xr_rr(long n, const double* __restrict__ num, const double* __restrict__ den,
                                                  double* __restrict__ x, double* __restrict__ r,
                                                  const double* __restrict__ p, const double* __restrict__ q,
                                                  double* __restrict__ rold, double* __restrict__ partials,
                                                  float* __restrict__ r32, const double* __restrict__ rr_old,
                                                  double* __restrict__ scale_out) {
    const double alpha = den[0] != 0.0 ? num[0] / den[0] : 0.0;
    const double inv = r32 ? 1.0 / sqrt(fmax(rr_old[0], 1e-300)) : 0.0;
    if (r32 && blockIdx.x == 0 && threadIdx.x == 0) scale_out[0] = rr_old[0];
    double v[1] = {0};
    // the reduction grid is small (2 blocks per SM): XR_U grid strides per trip keep enough loads in
    // flight; the sum still runs over each thread's elements in stride order, as in k_dot
    const long st = (long)gridDim.x * blockDim.x;
    for (long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x; i0 < n; i0 += XR_U * st) {
        double ri[XR_U], pi[XR_U], qi[XR_U], xi[XR_U];
#pragma unroll
        for (int k = 0; k < XR_U; k++) {
            const long i = i0 + k * st;
            if (i < n) { ri[k] = r[i]; pi[k] = p[i]; qi[k] = q[i]; xi[k] = x[i]; }
        }
#pragma unroll
        for (int k = 0; k < XR_U; k++) {
            const long i = i0 + k * st;
            if (i >= n) break;
            rold[i] = ri[k];
            x[i] = xi[k] + alpha * pi[k];
            const double rn = ri[k] - alpha * qi[k];
            r[i] = rn;
            if (r32) r32[i] = (float)(rn * inv);
            v[0] += rn * rn;
        }
    }
    block_reduce_store<1>(v, partials);
}

// z = a * sqrt(s) widened to FP64, with (z.r, z.rold) in the same pass (partials as k_dot2's)
__global__ void __launch_bounds__(RB) k_f2d_scaled_dot2(long n, const float* __restrict__ a, double* __restrict__ z,
                                                        const double* __restrict__ s, const double* __restrict__ r,
                                                        const double* __restrict__ rold,
                                                        double* __restrict__ partials) {
    const double sc = sqrt(fmax(s[0], 1e-300));
    double v[2] = {0, 0};
    const long st = (long)gridDim.x * blockDim.x;
    for (long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x; i0 < n; i0 += XR_U * st) {
        float ai[XR_U];
        double ri[XR_U], oi[XR_U];
#pragma unroll
        for (int k = 0; k < XR_U; k++) {
            const long i = i0 + k * st;
            if (i < n) { ai[k] = a[i]; ri[k] = r[i]; oi[k] = rold[i]; }
        }
#pragma unroll
        for (int k = 0; k < XR_U; k++) {
            const long i = i0 + k * st;
            if (i >= n) break;
            const double x = (double)ai[k] * sc;
            z[i] = x;
            v[0] += x * ri[k];
            v[1] += x * oi[k];
        }
    }
    block_reduce_store<2>(v, partials);
}

// ---- FP32 Krylov vectors (FP64 accumulation of every dot product) ----------------------
__global__ void __launch_bounds__(RB) k_dot32(long n, const float* __restrict__ a, const float* __restrict__ b,
                                              double* __restrict__ partials) {
    double v[1] = {0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        v[0] += (double)a[i] * (double)b[i];
    block_reduce_store<1>(v, partials);
}

__global__ void __launch_bounds__(RB) k_dot32_2(long n, const float* __restrict__ a, const float* __restrict__ b,
                                                const float* __restrict__ c, double* __restrict__ partials) {
    double v[2] = {0, 0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double x = a[i];
        v[0] += x * (double)b[i];
        v[1] += x * (double)c[i];
    }
    block_reduce_store<2>(v, partials);
}

// p = z + beta p (flexible beta as k_pcg_p_it), FP32 vectors
__global__ void k_pcg32_p(long n, const double* __restrict__ s, const double* __restrict__ it, float* __restrict__ p,
                          const float* __restrict__ z) {
    const bool first = it[0] == 0.0;
    const double den = s[2];
    const float beta = (first || den == 0.0) ? 0.f : (float)((s[0] - s[1]) / den);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = first ? z[i] : z[i] + beta * p[i];
}

// d += alpha p, rold = r, r -= alpha q, r.r (FP64 sum) with alpha = num / den
__global__ void __launch_bounds__(RB) k_pcg32_xr_rr(long n, const double* __restrict__ num, const double* __restrict__ den,
                                                    float* __restrict__ d, float* __restrict__ r,
                                                    const float* __restrict__ p, const float* __restrict__ q,
                                                    float* __restrict__ rold, double* __restrict__ partials) {
    const float alpha = den[0] != 0.0 ? (float)(num[0] / den[0]) : 0.f;
    double v[1] = {0};
    const long st = (long)gridDim.x * blockDim.x;
    for (long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x; i0 < n; i0 += XR_U * st) {
        float ri[XR_U], pi[XR_U], qi[XR_U], di[XR_U];
#pragma unroll
        for (int k = 0; k < XR_U; k++) {
            const long i = i0 + k * st;
            if (i < n) { ri[k] = r[i]; pi[k] = p[i]; qi[k] = q[i]; di[k] = d[i]; }
        }
#pragma unroll
        for (int k = 0; k < XR_U; k++) {
            const long i = i0 + k * st;
            if (i >= n) break;
            rold[i] = ri[k];
            d[i] = di[k] + alpha * pi[k];
            const float rn = ri[k] - alpha * qi[k];
            r[i] = rn;
            v[0] += (double)rn * (double)rn;
        }
    }
    block_reduce_store<1>(v, partials);
}

// x += sqrt(s) d (the FP32 correction of a refinement step, scaled back to the FP64 residual)
__global__ void k_axpy_f32_scaled(long n, double* __restrict__ x, const float* __restrict__ d,
                                  const double* __restrict__ s) {
    const double sc = sqrt(fmax(s[0], 0.0));
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        x[i] += sc * (double)d[i];
}

// p = z + beta p with flexible beta = (r.z - rold.z) / rz_old; scalars: s[0]=r.z, s[1]=rold.z, den=rz_old
__global__ void k_pcg_p(long n, const double* __restrict__ s, const double* __restrict__ den, double* __restrict__ p,
                        const double* __restrict__ z, int first) {
    const double beta = first ? 0.0 : (s[0] - s[1]) / den[0];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = first ? z[i] : z[i] + beta * p[i];
}

__global__ void k_scale(long n, double* __restrict__ x, const double* __restrict__ s, int inv_sqrt) {
    const double sc = inv_sqrt ? 1.0 / sqrt(s[0]) : s[0];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] *= sc;
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__global__ void k_rng(uint64_t seed, long n, double* __restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        uint64_t hsh = splitmix64(seed * 0x632BE59BD9B4E019ull + (uint64_t)i);
        out[i] = (double)(hsh >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
}

// gather load-node values into an AoS [3*nload] vector; optionally keep only the normal component
__global__ void k_gather_load(int nload, long nv, const int* __restrict__ nodes, const double* __restrict__ f,
                              const double* __restrict__ normal, int constrain, double* __restrict__ fs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nload; i += gridDim.x * blockDim.x) {
        const long v = nodes[i];
        double a = f[v], b = f[nv + v], c = f[2 * nv + v];
        if (constrain) {
            const double n0 = normal[3 * i], n1 = normal[3 * i + 1], n2 = normal[3 * i + 2];
            const double d = a * n0 + b * n1 + c * n2;
            a = d * n0; b = d * n1; c = d * n2;
        }
        fs[3 * i] = a; fs[3 * i + 1] = b; fs[3 * i + 2] = c;
    }
}
__global__ void k_scatter_load(int nload, long nv, const int* __restrict__ nodes, const double* __restrict__ fs,
                               double* __restrict__ f) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nload; i += gridDim.x * blockDim.x) {
        const long v = nodes[i];
        f[v] = fs[3 * i]; f[nv + v] = fs[3 * i + 1]; f[2 * nv + v] = fs[3 * i + 2];
    }
}
// fs -= sum_k (Rd_k . fs) Rd_k with the dots precomputed in w[0..nrig)
__global__ void k_sub_modes(long n, int nrig, const double* __restrict__ Rd, const double* __restrict__ w,
                            double* __restrict__ fs) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double s = fs[i];
        for (int k = 0; k < nrig; k++) s -= w[k] * Rd[k * n + i];
        fs[i] = s;
    }
}
// six dots against the rigid modes in one pass
__global__ void __launch_bounds__(RB) k_dot6(long n, int nrig, const double* __restrict__ Rd,
                                             const double* __restrict__ x, double* __restrict__ partials) {
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double xi = x[i];
#pragma unroll
        for (int k = 0; k < 6; k++)
            if (k < nrig) v[k] += Rd[k * n + i] * xi;
    }
    block_reduce_store<6>(v, partials);
}

// largest eigenvalue of the symmetric tridiagonal (alpha, beta) by Sturm-count bisection
__global__ void k_tridiag_max(int k, const double* __restrict__ alpha, const double* __restrict__ beta,
                              double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double lo = alpha[0], hi = alpha[0];
    for (int i = 0; i < k; i++) {
        const double r = (i > 0 ? fabs(beta[i - 1]) : 0) + (i < k - 1 ? fabs(beta[i]) : 0);
        lo = fmin(lo, alpha[i] - r);
        hi = fmax(hi, alpha[i] + r);
    }
    for (int it = 0; it < 200; it++) {
        const double mid = 0.5 * (lo + hi);
        if (mid == lo || mid == hi) break;
        int cnt = 0;
        double d = 1;
        for (int i = 0; i < k; i++) {
            const double b2 = i > 0 ? beta[i - 1] * beta[i - 1] : 0;
            d = alpha[i] - mid - (i > 0 ? b2 / d : 0);
            if (d == 0) d = -1e-300;
            if (d < 0) cnt++;
        }
        if (cnt == k) hi = mid; else lo = mid;
    }
    out[0] = 0.5 * (lo + hi);
}

// normalised radial sensitivity filter, one thread per element
__global__ void k_filter(int nx, int ny, int nz, const uint8_t* __restrict__ eact, float radius,
                         const float* __restrict__ sens, float* __restrict__ out) {
    const long ne = (long)nx * ny * nz;
    const float R2 = radius * radius;
    const int Rl = (int)(radius + 0.5f);
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ne; e += (long)gridDim.x * blockDim.x) {
        if (!eact[e]) { out[e] = 0.f; continue; }
        const int x = (int)(e % nx), y = (int)((e / nx) % ny), z = (int)(e / ((long)nx * ny));
        float wsum = 0;
        double gsum = 0;
        for (int dx = -Rl; dx <= Rl; dx++) {
            const int X = x + dx;
            if (X < 0 || X >= nx) continue;
            for (int dy = -Rl; dy <= Rl; dy++) {
                const int Y = y + dy;
                if (Y < 0 || Y >= ny) continue;
                for (int dz = -Rl; dz <= Rl; dz++) {
                    const int Z = z + dz;
                    if (Z < 0 || Z >= nz) continue;
                    const float r2 = (float)(dx * dx + dy * dy + dz * dz);
                    if (r2 > R2) continue;
                    const long n = X + (long)nx * (Y + (long)ny * Z);
                    if (!eact[n]) continue;
                    const float t = sqrtf(r2 / R2);
                    const float t2 = t * t;
                    const float wv = 1 - 6 * t2 + 8 * t2 * t - 3 * t2 * t2;
                    gsum += wv * sens[n];
                    wsum += wv;
                }
            }
        }
        out[e] = (float)(gsum / wsum);
    }
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// OC trial update + FP64 volume partial sums
__global__ void __launch_bounds__(RB) k_oc_try(long ne, const uint8_t* __restrict__ eact,
                                               const uint8_t* __restrict__ eshell, const float* __restrict__ rho,
                                               const float* __restrict__ sens, float thr, float step, float damp,
                                               float rhomin, float* __restrict__ out, double* __restrict__ partials) {
    double v[1] = {0};
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ne; e += (long)gridDim.x * blockDim.x) {
        float rn = 0.f;
        if (eact[e]) {
            float g = sens[e];
            if (g > 0) g = 0;
            g = fabsf(g);
            const float ro = rho[e];
            rn = ro * powf(g / thr, damp);
            rn = clampf(rn, ro - step, ro + step);
            rn = clampf(rn, rhomin, 1.f);
            if (eshell != nullptr && eshell[e]) rn = 1.f;
            v[0] += (double)rn;
        }
        out[e] = rn;
    }
    block_reduce_store<1>(v, partials);
}

__global__ void __launch_bounds__(RB) k_maxabs(long ne, const uint8_t* __restrict__ eact, const float* __restrict__ s,
                                               double* __restrict__ partials) {
    double m = 0;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ne; e += (long)gridDim.x * blockDim.x)
        if (eact[e]) m = fmax(m, (double)fabsf(s[e]));
    __shared__ double sh[RB];
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int o = RB / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}
__global__ void k_final_max(int nblocks, const double* __restrict__ partials, double* __restrict__ out) {
    if (threadIdx.x == 0) {
        double m = 0;
        for (int b = 0; b < nblocks; b++) m = fmax(m, partials[b]);
        out[0] = m;
    }
}

__global__ void __launch_bounds__(RB) k_count_u8(long n, const uint8_t* __restrict__ a, double* __restrict__ partials) {
    double v[1] = {0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[0] += a[i] ? 1.0 : 0.0;
    block_reduce_store<1>(v, partials);
}

__global__ void k_node_active(int nx, int ny, int nz, const uint8_t* __restrict__ eact, uint8_t* __restrict__ vact) {
    const int vx = nx + 1, vy = ny + 1;
    const long nv = (long)vx * vy * (nz + 1);
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < nv; v += (long)gridDim.x * blockDim.x) {
        const int x = (int)(v % vx), y = (int)((v / vx) % vy), z = (int)(v / ((long)vx * vy));
        uint8_t a = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int ex = x + (i & 1) - 1, ey = y + ((i >> 1) & 1) - 1, ez = z + (i >> 2) - 1;
            if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
            a |= eact[ex + (long)nx * (ey + (long)ny * ez)];
        }
        vact[v] = a ? 1 : 0;
    }
}

__global__ void k_coarsen(int nx, int ny, int nz, int ratio, const uint8_t* __restrict__ ef, uint8_t* __restrict__ ec) {
    const int cx = (nx + ratio - 1) / ratio, cy = (ny + ratio - 1) / ratio, cz = (nz + ratio - 1) / ratio;
    const long nc = (long)cx * cy * cz;
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < nc; c += (long)gridDim.x * blockDim.x) {
        const int X = (int)(c % cx), Y = (int)((c / cx) % cy), Z = (int)(c / ((long)cx * cy));
        uint8_t a = 0;
        for (int k = 0; k < ratio && !a; k++)
            for (int j = 0; j < ratio && !a; j++)
                for (int i = 0; i < ratio && !a; i++) {
                    const int x = X * ratio + i, y = Y * ratio + j, z = Z * ratio + k;
                    if (x < nx && y < ny && z < nz) a |= ef[x + (long)nx * (y + (long)ny * z)];
                }
        ec[c] = a ? 1 : 0;
    }
}

__global__ void k_surface(int nx, int ny, int nz, const uint8_t* __restrict__ eact, uint8_t* __restrict__ surf) {
    const int vx = nx + 1, vy = ny + 1;
    const long nv = (long)vx * vy * (nz + 1);
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < nv; v += (long)gridDim.x * blockDim.x) {
        const int x = (int)(v % vx), y = (int)((v / vx) % vy), z = (int)(v / ((long)vx * vy));
        bool s[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int ex = x + (i & 1) - 1, ey = y + ((i >> 1) & 1) - 1, ez = z + (i >> 2) - 1;
            s[i] = (ex >= 0 && ey >= 0 && ez >= 0 && ex < nx && ey < ny && ez < nz) &&
                   eact[ex + (long)nx * (ey + (long)ny * ez)];
        }
        bool ax = false, ay = false, az = false;
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 2; j++) {
                // s index = a + 2b + 4c for element offsets (a, b, c) in {0,1}
                ax |= s[0 + 2 * i + 4 * j] && s[1 + 2 * i + 4 * j];
                ay |= s[i + 0 + 4 * j] && s[i + 2 + 4 * j];
                az |= s[i + 2 * j + 0] && s[i + 2 * j + 4];
            }
        surf[v] = (!ax || !ay || !az) ? 1 : 0;
    }
}

__device__ __forceinline__ bool rbit(const uint32_t* b, long id) { return (b[id >> 5] >> (id & 31)) & 1u; }

// one thread per 32-vertex word: no atomics needed
__global__ void k_cube_vbits(int R, const uint32_t* __restrict__ eb, uint32_t* __restrict__ vb) {
    const int V = R + 1;
    const long nvb = (long)V * V * V;
    const long nw = (nvb + 31) / 32;
    for (long wd = blockIdx.x * (long)blockDim.x + threadIdx.x; wd < nw; wd += (long)gridDim.x * blockDim.x) {
        uint32_t word = 0;
        for (int b = 0; b < 32; b++) {
            const long t = wd * 32 + b;
            if (t >= nvb) break;
            const int x = (int)(t % V), y = (int)((t / V) % V), z = (int)(t / ((long)V * V));
            bool a = false;
            for (int i = 0; i < 8 && !a; i++) {
                const int ex = x + (i & 1) - 1, ey = y + ((i >> 1) & 1) - 1, ez = z + (i >> 2) - 1;
                if (ex < 0 || ey < 0 || ez < 0 || ex >= R || ey >= R || ez >= R) continue;
                a = rbit(eb, ex + (long)R * (ey + (long)R * ez));
            }
            if (a) word |= 1u << b;
        }
        vb[wd] = word;
    }
}

__global__ void k_cube_coarsen(int Rf, const uint32_t* __restrict__ ef, uint32_t* __restrict__ ec) {
    const int Rc = Rf >> 1;
    const long nc = (long)Rc * Rc * Rc;
    const long nw = (nc + 31) / 32;
    for (long wd = blockIdx.x * (long)blockDim.x + threadIdx.x; wd < nw; wd += (long)gridDim.x * blockDim.x) {
        uint32_t word = 0;
        for (int b = 0; b < 32; b++) {
            const long t = wd * 32 + b;
            if (t >= nc) break;
            const int X = (int)(t % Rc), Y = (int)((t / Rc) % Rc), Z = (int)(t / ((long)Rc * Rc));
            bool a = false;
            for (int i = 0; i < 8 && !a; i++) {
                const int x = 2 * X + (i & 1), y = 2 * Y + ((i >> 1) & 1), z = 2 * Z + (i >> 2);
                a = rbit(ef, x + (long)Rf * (y + (long)Rf * z));
            }
            if (a) word |= 1u << b;
        }
        ec[wd] = word;
    }
}

// raw rigid-body modes over active nodes: 3 translations, 3 rotations (columns of [p]x)
__global__ void k_rigid_raw(int vx, int vy, long nv, const uint8_t* __restrict__ vact, double* __restrict__ Ru) {
    const long n = 3 * nv;
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < nv; v += (long)gridDim.x * blockDim.x) {
        const double a = vact[v] ? 1.0 : 0.0;
        const double px = (double)(v % vx), py = (double)((v / vx) % vy), pz = (double)(v / ((long)vx * vy));
        const double ph[3][3] = {{0, -pz, py}, {pz, 0, -px}, {-py, px, 0}};
        for (int t = 0; t < 3; t++)
            for (int c = 0; c < 3; c++) Ru[(long)t * n + c * nv + v] = (t == c) ? a : 0.0;
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++) Ru[(long)(3 + k) * n + c * nv + v] = a * ph[c][k];
    }
}

__global__ void k_axpy_dev(long n, const double* __restrict__ coef, double sign, const double* __restrict__ x,
                           double* __restrict__ y) {
    const double a = sign * coef[0];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) y[i] += a * x[i];
}

__global__ void k_mask_copy(long n, long nv, const uint8_t* __restrict__ vact, const double* __restrict__ src,
                            double* __restrict__ dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = vact[i % nv] ? src[i] : 0.0;
}

}  // namespace

namespace rtk {

static int final_sum(rt_hier* h, int nv_, double* out) {
    return rt_launch(h->ctx, "reduce_final", [&] {
        switch (nv_) {
            case 1: k_final_sum<1><<<1, 32, 0, h->ctx->stream>>>(RT_RED_BLOCKS, h->partials, out); break;
            case 2: k_final_sum<2><<<1, 32, 0, h->ctx->stream>>>(RT_RED_BLOCKS, h->partials, out); break;
            default: k_final_sum<6><<<1, 32, 0, h->ctx->stream>>>(RT_RED_BLOCKS, h->partials, out); break;
        }
    });
}

int dot(rt_hier* h, long n, const double* a, const double* b, double* out) {
    RT_CHECK(rt_launch(h->ctx, "dot", [&] { k_dot<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, a, b, h->partials); }));
    return final_sum(h, 1, out);
}

int dot2(rt_hier* h, long n, const double* a, const double* b, const double* c, double* out) {
    RT_CHECK(rt_launch(h->ctx, "dot2", [&] { k_dot2<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, a, b, c, h->partials); }));
    return final_sum(h, 2, out);
}

int axpy(rt_hier* h, long n, double a, const double* x, double* y) {
    return rt_launch(h->ctx, "axpy", [&] { k_axpy<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, a, x, y); });
}

int f2d(rt_hier* h, long n, const float* a, double* b) {
    return rt_launch(h->ctx, "f2d", [&] { k_f2d<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, a, b); });
}

int d2f_scaled(rt_hier* h, long n, const double* a, float* b, const double* s) {
    return rt_launch(h->ctx, "d2f_scaled", [&] { k_d2f_scaled<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, a, b, s); });
}

int f2d_scaled(rt_hier* h, long n, const float* a, double* b, const double* s) {
    return rt_launch(h->ctx, "f2d_scaled", [&] { k_f2d_scaled<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, a, b, s); });
}

int f2d_scaled_add(rt_hier* h, long n, const float* a, double* b, const double* s) {
    return rt_launch(h->ctx, "f2d_scaled_add",
                     [&] { k_f2d_scaled_add<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, a, b, s); });
}

int pcg_update_xr(rt_hier* h, long n, const double* num, const double* den, double* x, double* r, const double* p,
                  const double* q, double* rold) {
    return rt_launch(h->ctx, "pcg_update_xr",
                     [&] { k_pcg_xr<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, num, den, x, r, p, q, rold); });
}

int pcg_update_xr_rr(rt_hier* h, long n, const double* num, const double* den, double* x, double* r, const double* p,
                     const double* q, double* rold, double* rr_out, float* r32, double* scale_out) {
    RT_CHECK(rt_launch(h->ctx, "pcg_update_xr", [&] {
        k_pcg_xr_rr<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, num, den, x, r, p, q, rold, h->partials, r32, rr_out,
                                                               scale_out);
    }));
    return final_sum(h, 1, rr_out);
}

int f2d_scaled_dot2(rt_hier* h, long n, const float* a, double* z, const double* s, const double* r,
                    const double* rold, double* out) {
    RT_CHECK(rt_launch(h->ctx, "f2d_scaled", [&] {
        k_f2d_scaled_dot2<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, a, z, s, r, rold, h->partials);
    }));
    return final_sum(h, 2, out);
}

int dot32(rt_hier* h, long n, const float* a, const float* b, double* out) {
    RT_CHECK(rt_launch(h->ctx, "dot32", [&] { k_dot32<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, a, b, h->partials); }));
    return final_sum(h, 1, out);
}

int dot32_2(rt_hier* h, long n, const float* a, const float* b, const float* c, double* out) {
    RT_CHECK(rt_launch(h->ctx, "dot32_2", [&] {
        k_dot32_2<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, a, b, c, h->partials);
    }));
    return final_sum(h, 2, out);
}

int pcg32_update_p(rt_hier* h, long n, const double* s, const double* it, float* p, const float* z) {
    return rt_launch(h->ctx, "pcg32_update_p",
                     [&] { k_pcg32_p<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, s, it, p, z); });
}

int pcg32_update_xr_rr(rt_hier* h, long n, const double* num, const double* den, float* d, float* r, const float* p,
                       const float* q, float* rold, double* rr_out) {
    RT_CHECK(rt_launch(h->ctx, "pcg32_update_xr", [&] {
        k_pcg32_xr_rr<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, num, den, d, r, p, q, rold, h->partials);
    }));
    return final_sum(h, 1, rr_out);
}

int axpy_f32_scaled(rt_hier* h, long n, double* x, const float* d, const double* s) {
    return rt_launch(h->ctx, "axpy_f32",
                     [&] { k_axpy_f32_scaled<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, x, d, s); });
}

int pcg_update_p(rt_hier* h, long n, const double* s, const double* den, double* p, const double* z, bool first) {
    return rt_launch(h->ctx, "pcg_update_p",
                     [&] { k_pcg_p<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, s, den, p, z, first ? 1 : 0); });
}

int scale(rt_hier* h, long n, double* x, const double* s, bool inv_sqrt) {
    return rt_launch(h->ctx, "scale", [&] { k_scale<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, x, s, inv_sqrt ? 1 : 0); });
}

int mask_copy(rt_hier* h, long n, const double* src, double* dst) {
    rt_level& L = h->L[0];
    return rt_launch(h->ctx, "mask_copy",
                     [&] { k_mask_copy<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, L.nv, L.vact, src, dst); });
}

int rng_uniform(rt_hier* h, uint64_t seed, long n, double* out) {
    return rt_launch(h->ctx, "rng_uniform", [&] { k_rng<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(seed, n, out); });
}

int gather_load(rt_hier* h, const double* f, double* fs) {
    if (h->nload == 0) return RT_OK;
    return rt_launch(h->ctx, "gather_load", [&] {
        k_gather_load<<<gridN(h->ctx, h->nload), 256, 0, h->ctx->stream>>>(h->nload, h->L[0].nv, h->load_nodes, f,
                                                                          h->load_normal, 0, fs);
    });
}

int scatter_load(rt_hier* h, const double* fs, double* f) {
    if (h->nload == 0) return RT_OK;
    return rt_launch(h->ctx, "scatter_load", [&] {
        k_scatter_load<<<gridN(h->ctx, h->nload), 256, 0, h->ctx->stream>>>(h->nload, h->L[0].nv, h->load_nodes, fs, f);
    });
}

// forceProject: gather -> (normal part) -> minus rigid part -> zero f -> scatter
int project_load(rt_hier* h, double* f) {
    rt_level& L = h->L[0];
    const int constrain = (h->P.mode == RT_MODE_NSCF || h->P.mode == RT_MODE_WSCF) ? 1 : 0;
    const long n = 3L * h->nload;
    if (h->nload > 0)
        RT_CHECK(rt_launch(h->ctx, "gather_load", [&] {
            k_gather_load<<<gridN(h->ctx, h->nload), 256, 0, h->ctx->stream>>>(h->nload, L.nv, h->load_nodes, f,
                                                                              h->load_normal, constrain, h->fs);
        }));
    if (h->nrig > 0 && n > 0) {
        RT_CHECK(rt_launch(h->ctx, "dot6", [&] {
            k_dot6<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, h->nrig, h->Rd, h->fs, h->partials);
        }));
        RT_CHECK(final_sum(h, 6, h->scal + 40));
        RT_CHECK(rt_launch(h->ctx, "sub_modes", [&] {
            k_sub_modes<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, h->nrig, h->Rd, h->scal + 40, h->fs);
        }));
    }
    RT_CUDA(h->ctx, cudaMemsetAsync(f, 0, sizeof(double) * 3 * L.nv, h->ctx->stream));
    return scatter_load(h, h->fs, f);
}

int displacement_project(rt_hier* h, double* u) {
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    RT_CHECK(rt_launch(h->ctx, "dot6", [&] { k_dot6<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(n, 6, h->Ru, u, h->partials); }));
    RT_CHECK(final_sum(h, 6, h->scal + 40));
    return rt_launch(h->ctx, "sub_modes",
                     [&] { k_sub_modes<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, 6, h->Ru, h->scal + 40, u); });
}

// setNodes (optimization/projection.cpp:46-127): orthonormal rigid modes over all active nodes
int rigid_nodes(rt_hier* h) {
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    if (h->Ru == nullptr && cudaMalloc(&h->Ru, sizeof(double) * 6 * n) != cudaSuccess) {
        cudaGetLastError();
        return rt_fail(h->ctx, RT_ENOMEM, "rigid modes: allocation failed");
    }
    RT_CHECK(rt_launch(h->ctx, "rigid_raw", [&] {
        k_rigid_raw<<<gridN(h->ctx, L.nv), 256, 0, h->ctx->stream>>>(L.vx, L.vy, L.nv, L.vact, h->Ru);
    }));
    for (int a = 0; a < 6; a++) {
        double* ra = h->Ru + a * n;
        for (int b = 0; b < a; b++) {
            RT_CHECK(dot(h, n, ra, h->Ru + b * n, h->scal + 70));
            RT_CHECK(rt_launch(h->ctx, "axpy_dev", [&] {
                k_axpy_dev<<<gridN(h->ctx, n), 256, 0, h->ctx->stream>>>(n, h->scal + 70, -1.0, h->Ru + b * n, ra);
            }));
        }
        RT_CHECK(dot(h, n, ra, ra, h->scal + 71));
        RT_CHECK(scale(h, n, ra, h->scal + 71, true));
    }
    return RT_OK;
}

int tridiag_max_eig(rt_hier* h, int k, const double* a, const double* b, double* out) {
    return rt_launch(h->ctx, "tridiag_max", [&] { k_tridiag_max<<<1, 32, 0, h->ctx->stream>>>(k, a, b, out); });
}

int filter(rt_hier* h, float radius) {
    rt_level& L = h->L[0];
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->ftmp, h->sens, sizeof(float) * L.ne, cudaMemcpyDeviceToDevice, h->ctx->stream));
    return rt_launch(h->ctx, "filter", [&] {
        k_filter<<<gridN(h->ctx, L.ne), 256, 0, h->ctx->stream>>>(L.nx, L.ny, L.nz, L.eact, radius, h->ftmp, h->sens);
    });
}

int oc_try(rt_hier* h, float thr, float* out, double* vol_dev) {
    rt_level& L = h->L[0];
    RT_CHECK(rt_launch(h->ctx, "oc_try", [&] {
        k_oc_try<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(L.ne, L.eact, h->eshell, h->rho, h->sens, thr,
                                                           h->P.design_step, h->P.damp_ratio, h->P.min_rho, out,
                                                           h->partials);
    }));
    return final_sum(h, 1, vol_dev);
}

int oc_maxabs(rt_hier* h, float*) {
    rt_level& L = h->L[0];
    RT_CHECK(rt_launch(h->ctx, "maxabs", [&] {
        k_maxabs<<<RT_RED_BLOCKS, RB, 0, h->ctx->stream>>>(L.ne, L.eact, h->sens, h->partials);
    }));
    return rt_launch(h->ctx, "reduce_final_max",
                     [&] { k_final_max<<<1, 32, 0, h->ctx->stream>>>(RT_RED_BLOCKS, h->partials, h->scal + 50); });
}

int count_u8(rt_ctx* c, long n, const uint8_t* a, double* out) {
    double* part = nullptr;
    RT_CUDA(c, cudaMallocAsync(&part, sizeof(double) * RT_RED_BLOCKS, c->stream));
    RT_CHECK(rt_launch(c, "count_u8", [&] { k_count_u8<<<RT_RED_BLOCKS, RB, 0, c->stream>>>(n, a, part); }));
    RT_CHECK(rt_launch(c, "reduce_final", [&] { k_final_sum<1><<<1, 32, 0, c->stream>>>(RT_RED_BLOCKS, part, out); }));
    RT_CUDA(c, cudaFreeAsync(part, c->stream));
    return RT_OK;
}

int node_active(rt_ctx* c, int nx, int ny, int nz, const uint8_t* eact, uint8_t* vact) {
    long nv = (long)(nx + 1) * (ny + 1) * (nz + 1);
    return rt_launch(c, "node_active", [&] { k_node_active<<<gridN(c, nv), 256, 0, c->stream>>>(nx, ny, nz, eact, vact); });
}

int coarsen_elements(rt_ctx* c, int nx, int ny, int nz, int ratio, const uint8_t* ef, uint8_t* ec) {
    long nc = (long)((nx + ratio - 1) / ratio) * ((ny + ratio - 1) / ratio) * ((nz + ratio - 1) / ratio);
    return rt_launch(c, "coarsen_elements",
                     [&] { k_coarsen<<<gridN(c, nc), 256, 0, c->stream>>>(nx, ny, nz, ratio, ef, ec); });
}

int surface_nodes(rt_hier* h, uint8_t* surf) {
    rt_level& L = h->L[0];
    return rt_launch(h->ctx, "surface_nodes",
                     [&] { k_surface<<<gridN(h->ctx, L.nv), 256, 0, h->ctx->stream>>>(L.nx, L.ny, L.nz, L.eact, surf); });
}

int cube_vbits(rt_ctx* c, int R, const uint32_t* eb, uint32_t* vb) {
    long nw = ((long)(R + 1) * (R + 1) * (R + 1) + 31) / 32;
    return rt_launch(c, "cube_vbits", [&] { k_cube_vbits<<<gridN(c, nw), 256, 0, c->stream>>>(R, eb, vb); });
}

int cube_coarsen(rt_ctx* c, int R, const uint32_t* ef, uint32_t* ec) {
    long nw = ((long)(R / 2) * (R / 2) * (R / 2) + 31) / 32;
    return rt_launch(c, "cube_coarsen", [&] { k_cube_coarsen<<<gridN(c, nw), 256, 0, c->stream>>>(R, ef, ec); });
}

}  // namespace rtk
