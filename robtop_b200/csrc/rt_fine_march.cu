// rt_fine_march.cu — finest-level operator as a register-marching element kernel.
//
// Same operators as rt_fine_tile.cu (residual, applyK, damped Jacobi,
// Chebyshev step; grid/Grid.cu:1450-1557, 2439-2517) without shared memory or
// block barriers:
//  * a warp owns a tile of 30 node columns x TY node rows x zchunk node layers;
//    lane l loads node column X0-1+l and evaluates element column X0-1+l;
//  * the x+1 vertex of a lane's element comes from lane l+1 (shfl_down), the
//    contribution of element column c-1 to node column c from lane l-1
//    (shfl_up), so lanes 1..30 own the tile's 30 node columns;
//  * y is marched inside the lane (element rows Y0-1 .. Y0+TY-1) with the
//    partial sums of the next node row carried in registers, z is marched over
//    the chunk with the partial sums of the next node layer carried per row;
//  * Jacobi / Chebyshev read the node's inverted 3x3 diagonal block, prepared
//    once per density by k_fine_dinv.
#include <cuda_runtime.h>

#include "rt_element.cuh"
#include "rt_internal.h"

namespace {

constexpr int MARCH_WARPS = 4;
constexpr int MARCH_BS = 32 * MARCH_WARPS;
constexpr int MARCH_NX = 30;  // node columns owned per warp

// inverse of each node's 3x3 diagonal block sum_e w_e KE(v_e, v_e), 6 unique entries
// (00, 01, 02, 11, 12, 22) as SoA [6][nv]; a fixed node stores I / n_e (its GS and Jacobi
// rule f / n_e), an inactive node zeros.
template <typename T>
__global__ void k_fine_dinv(int nx, int ny, int nz, const uint8_t* __restrict__ vact, const float* __restrict__ w,
                            const uint8_t* __restrict__ vfix, int ws, double a, double b, T* __restrict__ dinv) {
    const int vx = nx + 1, vy = ny + 1;
    const long nv = (long)vx * vy * (nz + 1);
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < nv; v += (long)gridDim.x * blockDim.x) {
        const int x = (int)(v % vx), y = (int)((v / vx) % vy), z = (int)(v / ((long)vx * vy));
        double sw = 0, sxy = 0, sxz = 0, syz = 0;
        int ne = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int dx = i & 1, dy = (i >> 1) & 1, dz = i >> 2;
            const int ex = x - 1 + dx, ey = y - 1 + dy, ez = z - 1 + dz;
            if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
            const double wv = w[ex + (long)nx * (ey + (long)ny * ez)];
            if (wv == 0) continue;
            ne++;
            // the node is vertex (1-dx, 1-dy, 1-dz) of that element; reflection signs +1 for bit 0
            const double sx = dx ? 1.0 : -1.0, sy = dy ? 1.0 : -1.0, sz = dz ? 1.0 : -1.0;
            sw += wv;
            sxy += wv * sx * sy;
            sxz += wv * sx * sz;
            syz += wv * sy * sz;
        }
        double o[6] = {0, 0, 0, 0, 0, 0};
        if (vact[v] && ne > 0) {
            if (ws && vfix[v]) {
                o[0] = o[3] = o[5] = 1.0 / ne;
            } else {
                const double A = a * sw, bxy = b * sxy, bxz = b * sxz, byz = b * syz;
                const double c00 = A * A - byz * byz, c01 = -(bxy * A - byz * bxz), c02 = bxy * byz - A * bxz;
                const double c11 = A * A - bxz * bxz, c12 = -(A * byz - bxy * bxz), c22 = A * A - bxy * bxy;
                const double id = 1.0 / (A * c00 + bxy * c01 + bxz * c02);
                o[0] = c00 * id; o[1] = c01 * id; o[2] = c02 * id; o[3] = c11 * id; o[4] = c12 * id; o[5] = c22 * id;
            }
        }
#pragma unroll
        for (int q = 0; q < 6; q++) dinv[q * nv + v] = (T)o[q];
    }
}

// MODE 0: r = f - K u (fixed rows: r = f)     MODE 1: out = K u (fixed rows: u)
// MODE 2: unew = u + omega D^-1 (f - K u)     MODE 3: Chebyshev step kstep (coefficients a_k, b_k from the level's table, see rt_cheby_coef)
// (fixed nodes in MODE 2/3: unew = f / n_e, d = 0)
// PF: load each layer's output-stage inputs (flags, f, inverted diagonal block, Chebyshev
// direction) at the top of the layer iteration, so that their latency overlaps the element
// arithmetic (more registers: 3 blocks per SM for FP32 instead of 4)
template <typename T, bool WS, int MODE, int TY, bool PF>
__global__ void __launch_bounds__(MARCH_BS, sizeof(T) == 4 ? (PF ? 3 : 4) : 2) k_fine_march(int nx, int ny, int nz, int ntx, int nty, int nch,
                                                          int zchunk, const uint8_t* __restrict__ vact,
                                                          const float* __restrict__ wgt,
                                                          const uint8_t* __restrict__ vfix, const rte::KtVals<T> kt,
                                                          const T* __restrict__ u, const T* __restrict__ f,
                                                          T* __restrict__ out, T omega, T* __restrict__ dvec,
                                                          const double* __restrict__ coef, int kstep,
                                                          const T* __restrict__ dinv) {
    const int lane = threadIdx.x & 31;
    const long wid = (long)blockIdx.x * MARCH_WARPS + (threadIdx.x >> 5);
    if (wid >= (long)ntx * nty * nch) return;  // whole warp leaves together
    T cheb_a = T(0), cheb_b = T(0);
    if (MODE == 3) {
        const double ca = coef[2 * kstep], cb = coef[2 * kstep + 1];
        cheb_a = (T)ca;
        cheb_b = (T)cb;
    }
    const int tx = (int)(wid % ntx), ty = (int)((wid / ntx) % nty), tz = (int)(wid / ((long)ntx * nty));
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long plane = (long)vx * vy;
    const int X0 = tx * MARCH_NX, Y0 = ty * TY, Z0 = tz * zchunk;
    const int Z1 = min(Z0 + zchunk, vz);
    const int cx = X0 - 1 + lane;                            // node column loaded / element column evaluated
    const bool col_ok = cx >= 0 && cx < vx;
    const bool ecol_ok = cx >= 0 && cx < nx;
    const bool own_x = lane >= 1 && lane <= MARCH_NX && col_ok;  // node column cx owned by this lane

    auto load_u = [&](int yy, int zz, T (&dst)[3]) {
        dst[0] = dst[1] = dst[2] = T(0);
        if (col_ok && yy >= 0 && yy < vy && zz >= 0 && zz < vz) {
            const long v = cx + (long)vx * yy + plane * zz;
            if (!(WS && vfix[v])) {
                dst[0] = u[v];
                dst[1] = u[nv + v];
                dst[2] = u[2 * nv + v];
            }
        }
    };

    T ub[TY + 2][3], ut[TY + 2][3];  // node layers ez (bottom) and ez+1 (top), rows Y0-1 .. Y0+TY
    T zc[TY][3];                     // top contributions of element layer ez to node layer ez+1
#pragma unroll
    for (int r = 0; r < TY + 2; r++) load_u(Y0 - 1 + r, Z0 - 1, ub[r]);
#pragma unroll
    for (int r = 0; r < TY; r++) zc[r][0] = zc[r][1] = zc[r][2] = T(0);

    for (int ez = Z0 - 1; ez < Z1; ez++) {
#pragma unroll
        for (int r = 0; r < TY + 2; r++) load_u(Y0 - 1 + r, ez + 1, ut[r]);
        const bool ez_ok = ez >= 0 && ez < nz;
        bool pact[TY], pfix[TY];
        T pf[TY][3], pd[TY][6], pdv[TY][3];
        if (PF) {
#pragma unroll
            for (int ri = 0; ri < TY; ri++) {
                const int ey = Y0 + ri;
                const bool own = own_x && ez >= Z0 && ey < vy;
                const long v = own ? cx + (long)vx * ey + plane * ez : 0;
                pact[ri] = own && vact[v];
                pfix[ri] = WS && pact[ri] && vfix[v];
#pragma unroll
                for (int c = 0; c < 3; c++) pf[ri][c] = (MODE != 1 && pact[ri]) ? f[c * nv + v] : T(0);
#pragma unroll
                for (int q = 0; q < 6; q++) pd[ri][q] = (MODE >= 2 && pact[ri]) ? dinv[q * nv + v] : T(0);
#pragma unroll
                for (int c = 0; c < 3; c++)
                    pdv[ri][c] = (MODE == 3 && pact[ri] && kstep != 0) ? dvec[c * nv + v] : T(0);
            }
        }
        T ycb[3] = {T(0), T(0), T(0)}, yct[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int r = 0; r <= TY; r++) {
            const int ey = Y0 - 1 + r;  // element row; couples node rows r and r+1 of the tile
            float wv = 0.f;
            if (ecol_ok && ez_ok && ey >= 0 && ey < ny) wv = wgt[cx + (long)nx * (ey + (long)ny * ez)];
            T a[24];
#pragma unroll
            for (int by = 0; by < 2; by++)
#pragma unroll
                for (int bz = 0; bz < 2; bz++)
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const T own = bz ? ut[r + by][c] : ub[r + by][c];
                        a[(2 * by + 4 * bz) * 3 + c] = own;
                        a[(1 + 2 * by + 4 * bz) * 3 + c] = __shfl_down_sync(0xffffffffu, own, 1);
                    }
            if (wv != 0.f) {
                rte::element_apply(a, kt, T(wv));
            } else {
#pragma unroll
                for (int q = 0; q < 24; q++) a[q] = T(0);
            }
            // node column cx: vertex bx = 0 of the own element + vertex bx = 1 of element cx-1 (lane-1)
            T cc[2][2][3];
#pragma unroll
            for (int by = 0; by < 2; by++)
#pragma unroll
                for (int bz = 0; bz < 2; bz++)
#pragma unroll
                    for (int c = 0; c < 3; c++)
                        cc[by][bz][c] = a[(2 * by + 4 * bz) * 3 + c] +
                                        __shfl_up_sync(0xffffffffu, a[(1 + 2 * by + 4 * bz) * 3 + c], 1);
            if (r >= 1) {
                const int ri = r - 1;  // owned node row Y0 + ri == ey
                T fin[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    fin[c] = zc[ri][c] + ycb[c] + cc[0][0][c];
                    zc[ri][c] = yct[c] + cc[0][1][c];
                }
                if (own_x && ez >= Z0 && ey < vy) {
                    const long v = cx + (long)vx * ey + plane * ez;
                    const bool act = PF ? pact[ri] : (bool)vact[v];
                    const bool fixed = PF ? pfix[ri] : (WS && act && vfix[v]);
                    auto fv = [&](int c) { return PF ? pf[ri][c] : f[c * nv + v]; };
                    if (MODE == 0) {
#pragma unroll
                        for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? fv(c) : fv(c) - fin[c]) : T(0);
                    } else if (MODE == 1) {
#pragma unroll
                        for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? u[c * nv + v] : fin[c]) : T(0);
                    } else {
                        // u of this (non-fixed) node is ub[r]: node layer ez, node row Y0 - 1 + r == ey
                        T nu[3] = {T(0), T(0), T(0)}, dn[3] = {T(0), T(0), T(0)};
                        if (act) {
                            const T d00 = PF ? pd[ri][0] : dinv[v], d01 = PF ? pd[ri][1] : dinv[nv + v];
                            const T d02 = PF ? pd[ri][2] : dinv[2 * nv + v], d11 = PF ? pd[ri][3] : dinv[3 * nv + v];
                            const T d12 = PF ? pd[ri][4] : dinv[4 * nv + v], d22 = PF ? pd[ri][5] : dinv[5 * nv + v];
                            T rr[3];
#pragma unroll
                            for (int c = 0; c < 3; c++) rr[c] = fixed ? fv(c) : fv(c) - fin[c];
                            const T z0 = d00 * rr[0] + d01 * rr[1] + d02 * rr[2];
                            const T z1 = d01 * rr[0] + d11 * rr[1] + d12 * rr[2];
                            const T z2 = d02 * rr[0] + d12 * rr[1] + d22 * rr[2];
                            const T zz[3] = {z0, z1, z2};
                            if (fixed) {
#pragma unroll
                                for (int c = 0; c < 3; c++) nu[c] = zz[c];
                            } else if (MODE == 2) {
#pragma unroll
                                for (int c = 0; c < 3; c++) nu[c] = ub[r][c] + omega * zz[c];
                            } else {
#pragma unroll
                                for (int c = 0; c < 3; c++) {
                                    dn[c] = (kstep == 0 ? T(0) : cheb_a * (PF ? pdv[ri][c] : dvec[c * nv + v])) +
                                            cheb_b * zz[c];
                                    nu[c] = ub[r][c] + dn[c];
                                }
                            }
                        }
#pragma unroll
                        for (int c = 0; c < 3; c++) out[c * nv + v] = nu[c];
                        if (MODE == 3)
#pragma unroll
                            for (int c = 0; c < 3; c++) dvec[c * nv + v] = dn[c];
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                ycb[c] = cc[1][0][c];
                yct[c] = cc[1][1][c];
            }
        }
#pragma unroll
        for (int r = 0; r < TY + 2; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) ub[r][c] = ut[r][c];
    }
}

template <typename T, bool WS, int MODE, int TY, bool PF>
int launch_march_ty(rt_hier* h, int zc, const T* u, const T* f, T* out, double omega, const char* name, T* dvec,
                    const double* coef, int kstep, const T* dinv) {
    rt_level& L = h->L[0];
    const int ntx = (L.vx + MARCH_NX - 1) / MARCH_NX, nty = (L.vy + TY - 1) / TY, nch = (L.vz + zc - 1) / zc;
    const long nwarps = (long)ntx * nty * nch;
    const unsigned blocks = (unsigned)((nwarps + MARCH_WARPS - 1) / MARCH_WARPS);
    const rte::KtVals<T> kt = rte::make_kt<T>(h);
    return rt_launch(h->ctx, name, [&] {
        k_fine_march<T, WS, MODE, TY, PF><<<blocks, MARCH_BS, 0, h->ctx->stream>>>(
            L.nx, L.ny, L.nz, ntx, nty, nch, zc, L.vact, h->w, h->vfix, kt, u, f, out, (T)omega, dvec, coef, kstep,
            dinv);
    });
}

template <typename T, bool WS, int MODE>
int launch_march(rt_hier* h, const T* u, const T* f, T* out, double omega, const char* name, T* dvec,
                 const double* coef, int kstep) {
    const rt_tile_cfg& tc = h->tune[sizeof(T) == 8 ? 1 : 0][MODE];
    const T* dinv = sizeof(T) == 8 ? (const T*)h->dinv64 : (const T*)h->dinv32;
    if (tc.variant == 2) {
        switch (tc.ty) {
            case 2: return launch_march_ty<T, WS, MODE, 2, true>(h, tc.zchunk, u, f, out, omega, name, dvec, coef, kstep, dinv);
            default: return launch_march_ty<T, WS, MODE, 4, true>(h, tc.zchunk, u, f, out, omega, name, dvec, coef, kstep, dinv);
        }
    }
    switch (tc.ty) {
        case 2: return launch_march_ty<T, WS, MODE, 2, false>(h, tc.zchunk, u, f, out, omega, name, dvec, coef, kstep, dinv);
        case 8: return launch_march_ty<T, WS, MODE, 8, false>(h, tc.zchunk, u, f, out, omega, name, dvec, coef, kstep, dinv);
        default: return launch_march_ty<T, WS, MODE, 4, false>(h, tc.zchunk, u, f, out, omega, name, dvec, coef, kstep, dinv);
    }
}

}  // namespace

namespace rtk {

int fine_dinv(rt_hier* h) {
    rt_level& L = h->L[0];
    const unsigned g = (unsigned)std::min<long>((L.nv + 255) / 256, (long)h->ctx->sm_count * 16);
    const int ws = h->has_support ? 1 : 0;
    RT_CHECK(rt_launch(h->ctx, "fine_dinv_f64", [&] {
        k_fine_dinv<double><<<g, 256, 0, h->ctx->stream>>>(L.nx, L.ny, L.nz, L.vact, h->w, h->vfix, ws, h->KE[0],
                                                           h->KE[1], h->dinv64);
    }));
    return rt_launch(h->ctx, "fine_dinv_f32", [&] {
        k_fine_dinv<float><<<g, 256, 0, h->ctx->stream>>>(L.nx, L.ny, L.nz, L.vact, h->w, h->vfix, ws, h->KE[0],
                                                          h->KE[1], h->dinv32);
    });
}

template <typename T, int MODE>
int fine_march(rt_hier* h, const T* u, const T* f, T* out, double omega, T* dvec, const double* coef, int kstep) {
    static const char* names[2][4] = {{"fine_residual_f32", "fine_applyK_f32", "fine_jacobi_f32", "fine_cheby_f32"},
                                      {"fine_residual_f64", "fine_applyK_f64", "fine_jacobi_f64", "fine_cheby_f64"}};
    const char* nm = names[sizeof(T) == 8 ? 1 : 0][MODE];
    return h->has_support ? launch_march<T, true, MODE>(h, u, f, out, omega, nm, dvec, coef, kstep)
                          : launch_march<T, false, MODE>(h, u, f, out, omega, nm, dvec, coef, kstep);
}

#define RT_INST_MARCH(T)                                                                                       \
    template int fine_march<T, 0>(rt_hier*, const T*, const T*, T*, double, T*, const double*, int);          \
    template int fine_march<T, 1>(rt_hier*, const T*, const T*, T*, double, T*, const double*, int);          \
    template int fine_march<T, 2>(rt_hier*, const T*, const T*, T*, double, T*, const double*, int);          \
    template int fine_march<T, 3>(rt_hier*, const T*, const T*, T*, double, T*, const double*, int);
RT_INST_MARCH(double)
RT_INST_MARCH(float)

}  // namespace rtk
