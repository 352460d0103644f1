// rt_fine.cu — finest-level matrix-free hex8 operator on the dense node box.
//
// Restates (on a dense x-fastest box instead of GS-ordered index tables):
//   update_residual_OTFA_{NS,WS}_kernel  grid/Grid.cu:1450-1557
//   applyK_OTFA_kernel                   grid/Grid.cu:2439-2517
//   gs_relax_OTFA_{NS,WS}_kernel         grid/Grid.cu:792-1066
//   computeSensitivity_kernel            optimization/optimization.cu:44-107
// Node v gathers rho_e^p * KE[(7-i) block row] * u_e over its 8 incident
// elements i (element offset (i%2-1, i/2%2-1, i/4-1)); with supports, fixed
// neighbours contribute u = 0 and fixed rows are identity (applyK), zero
// (residual) or n_e * I (GS).
#include <cuda_runtime.h>

#include "rt_internal.h"

namespace {

constexpr int FINE_BS = 256;

template <typename T>
__device__ __forceinline__ void load_KE(T* sKE, const T* __restrict__ KEg) {
    for (int i = threadIdx.x; i < 576; i += blockDim.x) sKE[i] = KEg[i];
    __syncthreads();
}

// Sum over incident elements.  SELF: 0 = include own column block,
// 1 = skip it and accumulate the diagonal block into S (GS / Jacobi form).
template <typename T, bool WS, bool DIAG, bool SKIPSELF>
__device__ __forceinline__ void fine_node_sum(int x, int y, int z, int vx, int vy, int nx, int ny, int nz, long nv,
                                              const float* __restrict__ w, const uint8_t* __restrict__ vfix,
                                              const T* __restrict__ u, const T* __restrict__ sKE, T KU[3], T S[9],
                                              int& ne) {
    KU[0] = KU[1] = KU[2] = T(0);
    if (DIAG)
#pragma unroll
        for (int i = 0; i < 9; i++) S[i] = T(0);
    ne = 0;
#pragma unroll 1
    for (int i = 0; i < 8; i++) {
        const int ex = x + (i & 1) - 1, ey = y + ((i >> 1) & 1) - 1, ez = z + (i >> 2) - 1;
        if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
        const long e = ex + (long)nx * (ey + (long)ny * ez);
        const float we = w[e];
        if (we == 0.f) continue;
        ne++;
        const int vi = 7 - i;
        if (DIAG) {
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) S[a * 3 + b] += T(we) * sKE[(vi * 3 + a) * 24 + vi * 3 + b];
        }
        T acc[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int vj = 0; vj < 8; vj++) {
            const long nj = (long)(ex + (vj & 1)) + (long)vx * ((ey + ((vj >> 1) & 1)) + (long)vy * (ez + (vj >> 2)));
            if (SKIPSELF && vj == vi) continue;
            if (WS && vfix[nj]) continue;
            const T u0 = u[nj], u1 = u[nv + nj], u2 = u[2 * nv + nj];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const T* kr = sKE + (vi * 3 + r) * 24 + vj * 3;
                acc[r] += kr[0] * u0 + kr[1] * u1 + kr[2] * u2;
            }
        }
#pragma unroll
        for (int r = 0; r < 3; r++) KU[r] += T(we) * acc[r];
    }
}

// MODE 0: r = f - K u (fixed rows: K u = 0); MODE 1: out = K u (fixed rows: u)
template <typename T>
__device__ __forceinline__ void block_gs(const T S[9], const T F[3], const T KU[3], T uu[3], bool backward) {
    if (!backward) {
        uu[0] = (F[0] - S[1] * uu[1] - S[2] * uu[2] - KU[0]) / S[0];
        uu[1] = (F[1] - S[3] * uu[0] - S[5] * uu[2] - KU[1]) / S[4];
        uu[2] = (F[2] - S[6] * uu[0] - S[7] * uu[1] - KU[2]) / S[8];
    } else {
        uu[2] = (F[2] - S[6] * uu[0] - S[7] * uu[1] - KU[2]) / S[8];
        uu[1] = (F[1] - S[3] * uu[0] - S[5] * uu[2] - KU[1]) / S[4];
        uu[0] = (F[0] - S[1] * uu[1] - S[2] * uu[2] - KU[0]) / S[0];
    }
}

// one colour of the 8-colour point-block GS; colour c = x%2 + 2(y%2) + 4(z%2)
template <typename T, bool WS>
__global__ void __launch_bounds__(FINE_BS) k_fine_gs(int nx, int ny, int nz, int color, bool backward,
                                                      const uint8_t* __restrict__ vact, const float* __restrict__ w,
                                                      const uint8_t* __restrict__ vfix, const T* __restrict__ KEg,
                                                      T* __restrict__ u, const T* __restrict__ f) {
    __shared__ T sKE[576];
    load_KE(sKE, KEg);
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const int px = color & 1, py = (color >> 1) & 1, pz = (color >> 2) & 1;
    const int cx = (vx - px + 1) / 2, cy = (vy - py + 1) / 2, cz = (vz - pz + 1) / 2;
    const long nc = (long)cx * cy * cz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nc; t += (long)gridDim.x * blockDim.x) {
        const int x = px + 2 * (int)(t % cx), y = py + 2 * (int)((t / cx) % cy), z = pz + 2 * (int)(t / ((long)cx * cy));
        const long v = x + (long)vx * (y + (long)vy * z);
        if (!vact[v]) continue;
        T KU[3], S[9];
        int ne;
        fine_node_sum<T, WS, true, true>(x, y, z, vx, vy, nx, ny, nz, nv, w, vfix, u, sKE, KU, S, ne);
        if (WS && vfix[v]) {
#pragma unroll
            for (int i = 0; i < 9; i++) S[i] = T(0);
            S[0] = S[4] = S[8] = T(ne);
            KU[0] = KU[1] = KU[2] = T(0);
        }
        T F[3] = {f[v], f[nv + v], f[2 * nv + v]};
        T uu[3] = {u[v], u[nv + v], u[2 * nv + v]};
        block_gs(S, F, KU, uu, backward);
        u[v] = uu[0]; u[nv + v] = uu[1]; u[2 * nv + v] = uu[2];
    }
}

__global__ void k_penalty(long ne, const uint8_t* __restrict__ eact, const float* __restrict__ rho, float p,
                          float* __restrict__ w) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ne; e += (long)gridDim.x * blockDim.x)
        w[e] = eact[e] ? powf(rho[e], p) : 0.f;
}

// element compliance sensitivity s_e = -p rho^(p-1) u_e^T KE u_e, one thread per element
// ELEM_C = false: s_e = -p rho^(p-1) u_e.KE u_e (computeSensitivity_kernel, optimization/optimization.cu:44-107);
// ELEM_C = true: c_e = rho^p u_e.KE u_e (elementCompliance_kernel, grid/Grid.cu:3434-3480)
template <bool ELEM_C>
__global__ void __launch_bounds__(FINE_BS) k_sensitivity(int nx, int ny, int nz, const uint8_t* __restrict__ eact,
                                                          const float* __restrict__ rho, float p,
                                                          const double* __restrict__ KEg, const double* __restrict__ u,
                                                          float* __restrict__ sens) {
    __shared__ double sKE[576];
    load_KE(sKE, KEg);
    const int vx = nx + 1, vy = ny + 1;
    const long nv = (long)vx * vy * (nz + 1);
    const long ne = (long)nx * ny * nz;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ne; e += (long)gridDim.x * blockDim.x) {
        if (!eact[e]) { sens[e] = 0.f; continue; }
        const int x = (int)(e % nx), y = (int)((e / nx) % ny), z = (int)(e / ((long)nx * ny));
        double ue[24];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const long nj = (long)(x + (j & 1)) + (long)vx * ((y + ((j >> 1) & 1)) + (long)vy * (z + (j >> 2)));
            ue[3 * j] = u[nj]; ue[3 * j + 1] = u[nv + nj]; ue[3 * j + 2] = u[2 * nv + nj];
        }
        double s = 0;
#pragma unroll 4
        for (int i = 0; i < 24; i++) {
            double kr = 0;
#pragma unroll
            for (int j = 0; j < 24; j++) kr += sKE[i * 24 + j] * ue[j];
            s += ue[i] * kr;
        }
        if (ELEM_C) {
            sens[e] = (float)(s * (double)powf(rho[e], p));
        } else {
            const double pen = (double)(p * powf(rho[e], p - 1.f));
            sens[e] = (float)(-s * pen);
        }
    }
}

unsigned fine_grid(rt_ctx* c, long n) {
    long b = rt_blocks(n, FINE_BS);
    long cap = (long)c->sm_count * 16;
    return (unsigned)(b < cap ? b : cap);
}

template <typename T>
const T* KEptr(rt_hier* h);
template <>
const double* KEptr<double>(rt_hier* h) { return h->KE_dev; }
template <>
const float* KEptr<float>(rt_hier* h) { return h->KE32_dev; }

}  // namespace

namespace rtk {

int penalty_weights(rt_hier* h) {
    rt_level& L = h->L[0];
    return rt_launch(h->ctx, "penalty_weights", [&] {
        k_penalty<<<fine_grid(h->ctx, L.ne), FINE_BS, 0, h->ctx->stream>>>(L.ne, L.eact, h->rho, h->P.power_penalty,
                                                                          h->w);
    });
}

template <typename T>
int fine_gs(rt_hier* h, T* u, const T* f, bool backward) {
    rt_level& L = h->L[0];
    const char* nm = sizeof(T) == 8 ? "fine_gs_f64" : "fine_gs_f32";
    for (int cc = 0; cc < 8; cc++) {
        int col = backward ? 7 - cc : cc;
        long ncol = (long)((L.vx - (col & 1) + 1) / 2) * ((L.vy - ((col >> 1) & 1) + 1) / 2) *
                    ((L.vz - ((col >> 2) & 1) + 1) / 2);
        RT_CHECK(rt_launch(h->ctx, nm, [&] {
            unsigned g = fine_grid(h->ctx, ncol);
            if (h->has_support)
                k_fine_gs<T, true><<<g, FINE_BS, 0, h->ctx->stream>>>(L.nx, L.ny, L.nz, col, backward, L.vact, h->w,
                                                                      h->vfix, KEptr<T>(h), u, f);
            else
                k_fine_gs<T, false><<<g, FINE_BS, 0, h->ctx->stream>>>(L.nx, L.ny, L.nz, col, backward, L.vact, h->w,
                                                                       h->vfix, KEptr<T>(h), u, f);
        }));
    }
    return RT_OK;
}

int sensitivity(rt_hier* h, const double* u) {
    rt_level& L = h->L[0];
    return rt_launch(h->ctx, "sensitivity", [&] {
        k_sensitivity<false><<<fine_grid(h->ctx, L.ne), FINE_BS, 0, h->ctx->stream>>>(
            L.nx, L.ny, L.nz, L.eact, h->rho, h->P.power_penalty, h->KE_dev, u, h->sens);
    });
}

int element_compliance(rt_hier* h, const double* u, float* out) {
    rt_level& L = h->L[0];
    return rt_launch(h->ctx, "element_compliance", [&] {
        k_sensitivity<true><<<fine_grid(h->ctx, L.ne), FINE_BS, 0, h->ctx->stream>>>(
            L.nx, L.ny, L.nz, L.eact, h->rho, h->P.power_penalty, h->KE_dev, u, out);
    });
}

template int fine_gs<double>(rt_hier*, double*, const double*, bool);
template int fine_gs<float>(rt_hier*, float*, const float*, bool);

}  // namespace rtk
