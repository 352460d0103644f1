// rt_fine_tile.cu — finest-level operator as an element-tile kernel.
//
// Same operator as update_residual_OTFA_{NS,WS}_kernel (grid/Grid.cu:1450-1557),
// applyK_OTFA_kernel (grid/Grid.cu:2439-2517) plus damped point-block Jacobi
// and Chebyshev smoothing steps, computed element by element instead of node
// by node:
//
//  * KE is applied in the Hadamard (+-1 tensor-product) basis of the 8
//    element vertices.  With T = H (x) I3, KE = T Kt T^T / 64 and the 24x24 Kt
//    has 45 non-zeros (independent of E, nu, h), so one element costs two
//    3-stage butterflies per component and 45 FMAs instead of a dense 24x24.
//  * A CTA owns a 32 x TY node tile and marches up through z.  Per element
//    layer the (33 x (TY+1)) elements touching the tile are computed once,
//    their 24 outputs go to shared memory, and every node gathers its 8
//    contributions (4 from the layer below, 4 from the layer above) — no
//    atomics, each element is evaluated once per tile.
//  * The loop is software-pipelined: while layer ez is computed, the u values
//    of node layer ez+2, the weights of element layer ez+1 and the node-phase
//    inputs (f, own u, flags) are already in flight into registers.
//  * Fixed (support) nodes are stored as zero in the shared u tile, so the WS
//    rule of the reference falls out of the data.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <unordered_map>

#include "rt_element.cuh"
#include "rt_internal.h"
#include "rt_tc.cuh"

namespace {

// tile of 32 x TY nodes (TY = 2, 4 or 8; rt_autotune chooses)
template <int TY_>
struct Tile {
    static constexpr int TX = 32, TY = TY_;
    static constexpr int EXT = TX + 1, EYT = TY + 1;  // element tile (one halo element below in x and y)
    static constexpr int UXT = TX + 2, UYT = TY + 2;  // node halo tile
    static constexpr int NE_T = EXT * EYT;            // elements per layer (165 for TY = 4)
    static constexpr int NU_T = UXT * UYT;            // halo nodes per layer (204 for TY = 4)
    static constexpr int BS = ((NE_T > TX * TY ? NE_T : TX * TY) + 31) / 32 * 32;  // threads (192 for TY = 4)
    static constexpr int U_PER_T = (NU_T + BS - 1) / BS;                            // halo nodes per thread
};

template <typename T, int TY_>
struct TileSmem {
    T u[2][3][Tile<TY_>::NU_T];   // node layers ez, ez+1 (slot layer & 1)
    T e[24][Tile<TY_>::NE_T];     // element outputs of the current layer
    float w[3][Tile<TY_>::NE_T];  // element weights of layers ez-1, ez, ez+1 (slot (layer+3)%3)
};

// blocks per SM the register budget is sized for
template <typename T, int TY_>
constexpr int tile_min_blocks() {
    return sizeof(T) == 8 ? (TY_ == 2 ? 3 : TY_ == 4 ? 2 : 1) : (TY_ == 2 ? 8 : TY_ == 4 ? 5 : 2);
}

// smoothing update of one node (MODE 2: damped block Jacobi, MODE 3: Chebyshev step) from its
// accumulated K u (acc), f, u and the Chebyshev direction; wz0 / wz1 are the element-weight rows of the
// element layers below / above the node, el the row index of its (-x, -y) element.  The 3x3 diagonal
// block of K at the node is sum_e w_e KE_vv, KE_vv = a I + b (s s^T - I) with s the node's vertex signs.
template <typename T, int MODE, int EXT>
__device__ __forceinline__ void node_smooth(const rte::KtVals<T>& kt, const float* wz0, const float* wz1, int el,
                                            const T (&acc)[3], const T (&fv)[3], const T (&uo)[3],
                                            const T (&dv)[3], bool act, bool fixed, T omega, T cheb_a, T cheb_b,
                                            int kstep, T (&nu)[3], T (&dn)[3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) nu[c] = dn[c] = T(0);
    if (!act) return;
    T sw = T(0), sxy = T(0), sxz = T(0), syz = T(0);
    int ne = 0;
#pragma unroll
    for (int dz = 0; dz < 2; dz++)
#pragma unroll
        for (int dy = 0; dy < 2; dy++)
#pragma unroll
            for (int dx = 0; dx < 2; dx++) {
                const float wv = (dz ? wz1 : wz0)[el + dy * EXT + dx];
                if (wv != 0.f) ne++;
                // node's vertex bits in that element: (1-dx, 1-dy, 1-dz)
                const T sx = dx ? T(1) : T(-1), sy = dy ? T(1) : T(-1), sz = dz ? T(1) : T(-1);
                sw += T(wv);
                sxy += T(wv) * sx * sy;
                sxz += T(wv) * sx * sz;
                syz += T(wv) * sy * sz;
            }
    if (fixed) {
#pragma unroll
        for (int c = 0; c < 3; c++) nu[c] = fv[c] / T(ne);
        return;
    }
    const T A = kt.diag_a * sw, bxy = kt.diag_b * sxy, bxz = kt.diag_b * sxz, byz = kt.diag_b * syz;
    // inverse of [[A,bxy,bxz],[bxy,A,byz],[bxz,byz,A]]
    const T c00 = A * A - byz * byz, c01 = -(bxy * A - byz * bxz), c02 = bxy * byz - A * bxz;
    const T c11 = A * A - bxz * bxz, c12 = -(A * byz - bxy * bxz), c22 = A * A - bxy * bxy;
    // FP32: the reciprocal by the fast-division intrinsic (2 ulp; the block's determinant is far
    // inside its range); FP64: IEEE division
    const T det = A * c00 + bxy * c01 + bxz * c02;
    T id;
    if constexpr (sizeof(T) == 4)
        id = __fdividef(1.0f, det);
    else
        id = T(1) / det;
    T rr[3];
#pragma unroll
    for (int c = 0; c < 3; c++) rr[c] = fv[c] - acc[c];
    T zz[3];
    zz[0] = id * (c00 * rr[0] + c01 * rr[1] + c02 * rr[2]);
    zz[1] = id * (c01 * rr[0] + c11 * rr[1] + c12 * rr[2]);
    zz[2] = id * (c02 * rr[0] + c12 * rr[1] + c22 * rr[2]);
    if (MODE == 2) {
#pragma unroll
        for (int c = 0; c < 3; c++) nu[c] = uo[c] + omega * zz[c];
    } else {
        // Chebyshev step: d = ca d + cb D^-1 r, u += d
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dn[c] = (kstep == 0 ? T(0) : cheb_a * dv[c]) + cheb_b * zz[c];
            nu[c] = uo[c] + dn[c];
        }
    }
}

// MODE 0: r = f - K u (fixed rows: r = f)     MODE 1: out = K u (fixed rows: u)
// MODE 2: unew = u + omega D^-1 (f - K u) (fixed: f / n_e)
// MODE 3: Chebyshev step kstep: d = a_k d + b_k D^-1 (f - K u), unew = u + d (fixed: f / n_e)
template <typename T, bool WS, int MODE, int TY_>
__global__ void __launch_bounds__(Tile<TY_>::BS, tile_min_blocks<T, TY_>()) k_fine_tile(int nx, int ny, int nz, int zchunk,
                                                        const uint8_t* __restrict__ vact,
                                                        const float* __restrict__ wgt,
                                                        const uint8_t* __restrict__ vfix, const rte::KtVals<T> kt,
                                                        const T* __restrict__ u, const T* __restrict__ f,
                                                        T* __restrict__ out, T omega, T* __restrict__ dvec,
                                                        const double* __restrict__ coef, int kstep) {
    using TS = Tile<TY_>;
    constexpr int TX = TS::TX, TY = TS::TY, EXT = TS::EXT, UXT = TS::UXT, NE_T = TS::NE_T, NU_T = TS::NU_T;
    constexpr int TILE_BS = TS::BS, U_PER_T = TS::U_PER_T;
    extern __shared__ __align__(16) unsigned char smraw[];
    TileSmem<T, TY_>& S = *reinterpret_cast<TileSmem<T, TY_>*>(smraw);
    T cheb_a = T(0), cheb_b = T(0);
    if (MODE == 3) {
        const double ca = coef[2 * kstep], cb = coef[2 * kstep + 1];
        cheb_a = (T)ca;
        cheb_b = (T)cb;
    }
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long plane = (long)vx * vy;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * zchunk;
    const int ze = min(zb + zchunk, vz);
    const int tid = threadIdx.x;
    // node owned by this thread
    const int nxl = tid % TX, nyl = tid / TX;
    const int nxg = x0 + nxl, nyg = y0 + nyl;
    const bool node_thread = tid < TX * TY && nxg < vx && nyg < vy;
    const long vxy = node_thread ? nxg + (long)vx * nyg : 0;
    // element owned by this thread
    const int exl = tid % EXT, eyl = tid / EXT;
    const int exg = x0 - 1 + exl, eyg = y0 - 1 + eyl;
    const bool elem_xy = tid < NE_T && exg >= 0 && eyg >= 0 && exg < nx && eyg < ny;
    const long exy = elem_xy ? exg + (long)nx * eyg : 0;
    // halo nodes this thread loads (columns of the 34 x (TY+2) tile)
    long hxy[U_PER_T];
    bool hok[U_PER_T];
#pragma unroll
    for (int j = 0; j < U_PER_T; j++) {
        const int i = tid + j * TILE_BS;
        const int xx = x0 - 1 + i % UXT, yy = y0 - 1 + i / UXT;
        hok[j] = i < NU_T && xx >= 0 && yy >= 0 && xx < vx && yy < vy;
        hxy[j] = hok[j] ? xx + (long)vx * yy : 0;
    }

    // register stage for one node layer of the halo tile + one element layer of weights
    T pu[U_PER_T][3];
    float pw = 0.f;
    auto fetch_layer = [&](int L) {
#pragma unroll
        for (int j = 0; j < U_PER_T; j++) {
            T a = T(0), b = T(0), c = T(0);
            if (hok[j] && L >= 0 && L < vz) {
                const long v = hxy[j] + plane * L;
                if (!(WS && vfix[v])) {
                    a = u[v];
                    b = u[nv + v];
                    c = u[2 * nv + v];
                }
            }
            pu[j][0] = a;
            pu[j][1] = b;
            pu[j][2] = c;
        }
    };
    auto stash_layer = [&](int L) {
        T* dst = &S.u[L & 1][0][0];
#pragma unroll
        for (int j = 0; j < U_PER_T; j++) {
            const int i = tid + j * TILE_BS;
            if (i < NU_T) {
                dst[i] = pu[j][0];
                dst[NU_T + i] = pu[j][1];
                dst[2 * NU_T + i] = pu[j][2];
            }
        }
    };
    auto fetch_w = [&](int ez) {
        pw = (elem_xy && ez >= 0 && ez < nz) ? wgt[exy + (long)nx * ny * ez] : 0.f;
    };
    auto stash_w = [&](int ez) {
        if (tid < NE_T) S.w[(ez + 3) % 3][tid] = pw;
    };

    // prologue: node layer zb-1 and element weights of layer zb-1 into shared memory,
    // node layer zb in registers
    fetch_layer(zb - 1);
    fetch_w(zb - 1);
    stash_layer(zb - 1);
    stash_w(zb - 1);
    fetch_layer(zb);
    fetch_w(zb);

    T acc[3] = {T(0), T(0), T(0)};
    for (int ez = zb - 1; ez < ze; ez++) {
        // registers hold node layer ez+1 and the weights of element layer ez+1.  The u slot of
        // layer ez+1 was last read by the element phase of iteration ez-1 (behind its second
        // barrier); the weight slot (ez+1)%3 held layer ez-2, read by the node phase of
        // iteration ez-1, so it is only written after the barrier below.
        stash_layer(ez + 1);
        __syncthreads();
        if (ez + 1 < ze) stash_w(ez + 1);
        // start the loads for the next iteration and for this iteration's node phase
        if (ez + 2 <= ze) {
            fetch_layer(ez + 2);
            fetch_w(ez + 2);
        }
        const bool out_layer = ez >= zb;
        T fv[3] = {T(0), T(0), T(0)}, uo[3] = {T(0), T(0), T(0)}, dv[3] = {T(0), T(0), T(0)};
        bool act = false, fixed = false;
        long vout = 0;
        if (node_thread && out_layer) {
            vout = vxy + plane * ez;
            act = vact[vout];
            fixed = WS && act && vfix[vout];
            if (MODE != 1)
#pragma unroll
                for (int c = 0; c < 3; c++) fv[c] = f[c * nv + vout];
            if (MODE >= 1)
#pragma unroll
                for (int c = 0; c < 3; c++) uo[c] = u[c * nv + vout];
            if (MODE == 3 && kstep > 0)
#pragma unroll
                for (int c = 0; c < 3; c++) dv[c] = dvec[c * nv + vout];
        }
        // ---- element phase (element layer ez couples node layers ez and ez+1)
        if (tid < NE_T) {
            T a[24];
            const float wv = S.w[(ez + 3) % 3][tid];
            if (wv != 0.f) {
                const T* lo = &S.u[ez & 1][0][0];
                const T* hi = &S.u[(ez + 1) & 1][0][0];
#pragma unroll
                for (int vtx = 0; vtx < 8; vtx++) {
                    const T* src = (vtx & 4) ? hi : lo;
                    const int idx = (eyl + ((vtx >> 1) & 1)) * UXT + exl + (vtx & 1);
                    a[3 * vtx] = src[idx];
                    a[3 * vtx + 1] = src[NU_T + idx];
                    a[3 * vtx + 2] = src[2 * NU_T + idx];
                }
                rte::element_apply(a, kt, T(wv));
            } else {
#pragma unroll
                for (int q = 0; q < 24; q++) a[q] = T(0);
            }
#pragma unroll
            for (int q = 0; q < 24; q++) S.e[q][tid] = a[q];
        }
        __syncthreads();
        // ---- node phase
        if (node_thread) {
            if (out_layer) {
                // node layer ez: bottom vertices (bit z = 0) of element layer ez
#pragma unroll
                for (int dy = 0; dy < 2; dy++)
#pragma unroll
                    for (int dx = 0; dx < 2; dx++) {
                        const int el = (nyl + dy) * EXT + nxl + dx;
                        const int vtx = (1 - dx) + 2 * (1 - dy);
#pragma unroll
                        for (int c = 0; c < 3; c++) acc[c] += S.e[3 * vtx + c][el];
                    }
                const long v = vout;
                if (MODE == 0) {
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? fv[c] : fv[c] - acc[c]) : T(0);
                } else if (MODE == 1) {
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? uo[c] : acc[c]) : T(0);
                } else {
                    T nu[3], dn[3];
                    node_smooth<T, MODE, EXT>(kt, S.w[(ez + 2) % 3], S.w[ez % 3], nyl * EXT + nxl, acc, fv, uo, dv, act,
                                         fixed, omega, cheb_a, cheb_b, kstep, nu, dn);
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = nu[c];
                    if (MODE == 3)
#pragma unroll
                        for (int c = 0; c < 3; c++) dvec[c * nv + v] = dn[c];
                }
            }
            // start node layer ez+1 with the top vertices (bit z = 1) of element layer ez
#pragma unroll
            for (int c = 0; c < 3; c++) acc[c] = T(0);
#pragma unroll
            for (int dy = 0; dy < 2; dy++)
#pragma unroll
                for (int dx = 0; dx < 2; dx++) {
                    const int el = (nyl + dy) * EXT + nxl + dx;
                    const int vtx = (1 - dx) + 2 * (1 - dy) + 4;
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[c] += S.e[3 * vtx + c][el];
                }
        }
    }
}


// ---------------------------------------------------------------------------
// software-pipelined tile kernel: one barrier per element layer instead of two.
// Iteration t computes element layer t+1 (into one of two element-output buffers)
// while the node phase of node layer t reads element layer t from the other, so
// the element and node work of neighbouring layers share one barrier interval.
// Node layers live in a ring of 3 shared slots (layer t+3 is stored at the top of
// iteration t, into the slot of layer t, whose last readers ran before the
// previous barrier), element weights in a ring of 4 (layers t-1 .. t+2).
// ---------------------------------------------------------------------------
template <typename T, int TY_>
struct PipeSmem {
    T u[3][3][Tile<TY_>::NU_T];   // node layer L in slot (L + 3) % 3
    T e[2][24][Tile<TY_>::NE_T];  // element layer L in slot (L + 2) & 1
    float w[4][Tile<TY_>::NE_T];  // element layer L in slot (L + 4) & 3
};

template <typename T, int TY_>
constexpr int pipe_min_blocks() {
    return sizeof(T) == 8 ? (TY_ == 2 ? 3 : TY_ == 4 ? 2 : 1) : (TY_ == 2 ? 8 : TY_ == 4 ? 5 : 3);
}

template <typename T, bool WS, int MODE, int TY_>
__global__ void __launch_bounds__(Tile<TY_>::BS, pipe_min_blocks<T, TY_>()) k_fine_pipe(int nx, int ny, int nz, int zchunk,
                                                        const uint8_t* __restrict__ vact,
                                                        const float* __restrict__ wgt,
                                                        const uint8_t* __restrict__ vfix, const rte::KtVals<T> kt,
                                                        const T* __restrict__ u, const T* __restrict__ f,
                                                        T* __restrict__ out, T omega, T* __restrict__ dvec,
                                                        const double* __restrict__ coef, int kstep) {
    using TS = Tile<TY_>;
    constexpr int TX = TS::TX, TY = TS::TY, EXT = TS::EXT, UXT = TS::UXT, NE_T = TS::NE_T, NU_T = TS::NU_T;
    constexpr int TILE_BS = TS::BS, U_PER_T = TS::U_PER_T;
    extern __shared__ __align__(16) unsigned char smraw[];
    PipeSmem<T, TY_>& S = *reinterpret_cast<PipeSmem<T, TY_>*>(smraw);
    T cheb_a = T(0), cheb_b = T(0);
    if (MODE == 3) {
        const double ca = coef[2 * kstep], cb = coef[2 * kstep + 1];
        cheb_a = (T)ca;
        cheb_b = (T)cb;
    }
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long plane = (long)vx * vy;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * zchunk;
    const int ze = min(zb + zchunk, vz);
    const int tid = threadIdx.x;
    const int nxl = tid % TX, nyl = tid / TX;
    const int nxg = x0 + nxl, nyg = y0 + nyl;
    const bool node_thread = tid < TX * TY && nxg < vx && nyg < vy;
    const long vxy = node_thread ? nxg + (long)vx * nyg : 0;
    const int exl = tid % EXT, eyl = tid / EXT;
    const int exg = x0 - 1 + exl, eyg = y0 - 1 + eyl;
    const bool elem_xy = tid < NE_T && exg >= 0 && eyg >= 0 && exg < nx && eyg < ny;
    const long exy = elem_xy ? exg + (long)nx * eyg : 0;
    long hxy[U_PER_T];
    bool hok[U_PER_T];
#pragma unroll
    for (int j = 0; j < U_PER_T; j++) {
        const int i = tid + j * TILE_BS;
        const int xx = x0 - 1 + i % UXT, yy = y0 - 1 + i / UXT;
        hok[j] = i < NU_T && xx >= 0 && yy >= 0 && xx < vx && yy < vy;
        hxy[j] = hok[j] ? xx + (long)vx * yy : 0;
    }

    T pu[U_PER_T][3];
    float pw = 0.f;
    auto fetch_layer = [&](int L) {
#pragma unroll
        for (int j = 0; j < U_PER_T; j++) {
            T a = T(0), b = T(0), c = T(0);
            if (hok[j] && L >= 0 && L < vz) {
                const long v = hxy[j] + plane * L;
                if (!(WS && vfix[v])) {
                    a = u[v];
                    b = u[nv + v];
                    c = u[2 * nv + v];
                }
            }
            pu[j][0] = a;
            pu[j][1] = b;
            pu[j][2] = c;
        }
    };
    auto stash_layer = [&](int L) {
        T* dst = &S.u[(L + 3) % 3][0][0];
#pragma unroll
        for (int j = 0; j < U_PER_T; j++) {
            const int i = tid + j * TILE_BS;
            if (i < NU_T) {
                dst[i] = pu[j][0];
                dst[NU_T + i] = pu[j][1];
                dst[2 * NU_T + i] = pu[j][2];
            }
        }
    };
    auto fetch_w = [&](int ez) {
        pw = (elem_xy && ez >= 0 && ez < nz) ? wgt[exy + (long)nx * ny * ez] : 0.f;
    };
    auto stash_w = [&](int ez) {
        if (tid < NE_T) S.w[(ez + 4) & 3][tid] = pw;
    };
    // element layer e (couples node layers e and e+1) into its output slot
    auto element_phase = [&](int e) {
        if (tid >= NE_T) return;
        T a[24];
        const float wv = S.w[(e + 4) & 3][tid];
        if (wv != 0.f) {
            const T* lo = &S.u[(e + 3) % 3][0][0];
            const T* hi = &S.u[(e + 4) % 3][0][0];
#pragma unroll
            for (int vtx = 0; vtx < 8; vtx++) {
                const T* src = (vtx & 4) ? hi : lo;
                const int idx = (eyl + ((vtx >> 1) & 1)) * UXT + exl + (vtx & 1);
                a[3 * vtx] = src[idx];
                a[3 * vtx + 1] = src[NU_T + idx];
                a[3 * vtx + 2] = src[2 * NU_T + idx];
            }
            rte::element_apply(a, kt, T(wv));
        } else {
#pragma unroll
            for (int q = 0; q < 24; q++) a[q] = T(0);
        }
        T* dst = &S.e[(e + 2) & 1][0][0];
#pragma unroll
        for (int q = 0; q < 24; q++) dst[q * NE_T + tid] = a[q];
    };

    // prologue: node layers zb-1 .. zb+1 and weights of element layers zb-1, zb in shared
    // memory, element layer zb-1 computed; registers then hold node layer zb+2 and the
    // weights of element layer zb+1
    fetch_layer(zb - 1);
    stash_layer(zb - 1);
    fetch_layer(zb);
    stash_layer(zb);
    fetch_layer(zb + 1);
    stash_layer(zb + 1);
    fetch_w(zb - 1);
    stash_w(zb - 1);
    fetch_w(zb);
    stash_w(zb);
    __syncthreads();
    element_phase(zb - 1);
    fetch_layer(zb + 2);
    fetch_w(zb + 1);
    __syncthreads();

    T acc[3] = {T(0), T(0), T(0)};
    for (int t = zb - 1; t < ze; t++) {
        if (t + 3 <= ze) stash_layer(t + 3);
        if (t + 2 < ze) stash_w(t + 2);
        if (t + 4 <= ze) fetch_layer(t + 4);
        if (t + 3 < ze) fetch_w(t + 3);
        const bool out_layer = t >= zb;
        T fv[3] = {T(0), T(0), T(0)}, uo[3] = {T(0), T(0), T(0)}, dv[3] = {T(0), T(0), T(0)};
        bool act = false, fixed = false;
        long vout = 0;
        if (node_thread && out_layer) {
            vout = vxy + plane * t;
            act = vact[vout];
            fixed = WS && act && vfix[vout];
            if (MODE != 1)
#pragma unroll
                for (int c = 0; c < 3; c++) fv[c] = f[c * nv + vout];
            if (MODE >= 1)
#pragma unroll
                for (int c = 0; c < 3; c++) uo[c] = u[c * nv + vout];
            if (MODE == 3 && kstep > 0)
#pragma unroll
                for (int c = 0; c < 3; c++) dv[c] = dvec[c * nv + vout];
        }
        if (t + 1 < ze) element_phase(t + 1);
        if (node_thread) {
            const T* E = &S.e[(t + 2) & 1][0][0];
            if (out_layer) {
                // node layer t: bottom vertices (bit z = 0) of element layer t
#pragma unroll
                for (int dy = 0; dy < 2; dy++)
#pragma unroll
                    for (int dx = 0; dx < 2; dx++) {
                        const int el = (nyl + dy) * EXT + nxl + dx;
                        const int vtx = (1 - dx) + 2 * (1 - dy);
#pragma unroll
                        for (int c = 0; c < 3; c++) acc[c] += E[(3 * vtx + c) * NE_T + el];
                    }
                const long v = vout;
                if (MODE == 0) {
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? fv[c] : fv[c] - acc[c]) : T(0);
                } else if (MODE == 1) {
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? uo[c] : acc[c]) : T(0);
                } else {
                    T nu[3], dn[3];
                    node_smooth<T, MODE, EXT>(kt, S.w[(t + 3) & 3], S.w[(t + 4) & 3], nyl * EXT + nxl, acc, fv, uo,
                                              dv, act, fixed, omega, cheb_a, cheb_b, kstep, nu, dn);
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = nu[c];
                    if (MODE == 3)
#pragma unroll
                        for (int c = 0; c < 3; c++) dvec[c * nv + v] = dn[c];
                }
            }
            // start node layer t+1 with the top vertices (bit z = 1) of element layer t
#pragma unroll
            for (int c = 0; c < 3; c++) acc[c] = T(0);
#pragma unroll
            for (int dy = 0; dy < 2; dy++)
#pragma unroll
                for (int dx = 0; dx < 2; dx++) {
                    const int el = (nyl + dy) * EXT + nxl + dx;
                    const int vtx = (1 - dx) + 2 * (1 - dy) + 4;
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[c] += E[(3 * vtx + c) * NE_T + el];
                }
        }
        __syncthreads();
    }
}


// ---------------------------------------------------------------------------
// FP32 pipelined tile kernel with element pairs: a thread applies KE to two x-neighbour
// elements at once in packed FP32 pairs (FADD2 / FFMA2 / FMUL2), loading each pair of
// vertex values with one 64-bit shared load.  The node layers are kept twice in shared
// memory, as is and shifted by one node in x, so that both the (x, x+1) and the
// (x+1, x+2) vertex pairs of an element pair are aligned 64-bit words.  Element rows
// hold 34 slots (17 pairs; the 34th element is a zero-weight pad).  Otherwise the
// schedule is k_fine_pipe's: element layer t+1 and node layer t per barrier interval.
// ---------------------------------------------------------------------------
template <int TY_>
struct PTile {
    static constexpr int TX = 32, TY = TY_;
    static constexpr int EXP = 34, NEP = 17, EYT = TY + 1;  // element row pitch, pairs per row
    static constexpr int NE2 = EXP * EYT;                   // element slots per layer
    static constexpr int NPAIR = NEP * EYT;                 // element-pair threads
    static constexpr int UXR = 34, UXP = 36, UYT = TY + 2;  // halo nodes per row, row pitch (zero pad)
    static constexpr int NU_T = UXR * UYT;                  // halo nodes per layer
    static constexpr int NU2 = UXP * UYT;                   // shared slots per layer and component
    static constexpr int BS = ((NPAIR > TX * TY ? NPAIR : TX * TY) + 31) / 32 * 32;
    static constexpr int U_PER_T = (NU_T + BS - 1) / BS;
};

template <int TY_>
struct PairSmem {
    float u[3][2][3][PTile<TY_>::NU2];  // node layer L in slot (L + 3) % 3; copy 1 = shifted by one node in x
    float e[2][24][PTile<TY_>::NE2];    // element layer L in slot (L + 2) & 1
    float w[4][PTile<TY_>::NE2];        // element layer L in slot (L + 4) & 3
};

template <int TY_>
constexpr int pair_min_blocks() { return TY_ == 2 ? 7 : TY_ == 4 ? 4 : 2; }

template <bool WS, int MODE, int TY_>
__global__ void __launch_bounds__(PTile<TY_>::BS, pair_min_blocks<TY_>()) k_fine_pair(int nx, int ny, int nz, int zchunk,
                                                        const uint8_t* __restrict__ vact,
                                                        const float* __restrict__ wgt,
                                                        const uint8_t* __restrict__ vfix, const rte::KtVals<float> kt,
                                                        const float* __restrict__ u, const float* __restrict__ f,
                                                        float* __restrict__ out, float omega, float* __restrict__ dvec,
                                                        const double* __restrict__ coef, int kstep) {
    using T = float;
    using TS = PTile<TY_>;
    constexpr int TX = TS::TX, TY = TS::TY, EXP = TS::EXP, NEP = TS::NEP, NE2 = TS::NE2, NPAIR = TS::NPAIR;
    constexpr int UXR = TS::UXR, UXP = TS::UXP, NU_T = TS::NU_T, NU2 = TS::NU2, TILE_BS = TS::BS,
                  U_PER_T = TS::U_PER_T;
    extern __shared__ __align__(16) unsigned char smraw[];
    PairSmem<TY_>& S = *reinterpret_cast<PairSmem<TY_>*>(smraw);
    T cheb_a = T(0), cheb_b = T(0);
    if (MODE == 3) {
        const double ca = coef[2 * kstep], cb = coef[2 * kstep + 1];
        cheb_a = (T)ca;
        cheb_b = (T)cb;
    }
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long plane = (long)vx * vy;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * zchunk;
    const int ze = min(zb + zchunk, vz);
    const int tid = threadIdx.x;
    const int nxl = tid % TX, nyl = tid / TX;
    const int nxg = x0 + nxl, nyg = y0 + nyl;
    const bool node_thread = tid < TX * TY && nxg < vx && nyg < vy;
    const long vxy = node_thread ? nxg + (long)vx * nyg : 0;
    // element pair of this thread: elements 2m, 2m+1 of element row prow (tile coordinates)
    const int pm = tid % NEP, prow = tid / NEP;
    const int ex0 = x0 - 1 + 2 * pm, eyg = y0 - 1 + prow;
    const bool pair_thread = tid < NPAIR;
    const bool ey_ok = pair_thread && eyg >= 0 && eyg < ny;
    const bool e0_ok = ey_ok && ex0 >= 0 && ex0 < nx;                       // element 2m
    const bool e1_ok = ey_ok && ex0 + 1 < nx && 2 * pm + 1 <= TX;           // element 2m+1 (2m+1 = 33: pad)
    const long exy0 = e0_ok ? ex0 + (long)nx * eyg : 0;
    long hxy[U_PER_T];
    bool hok[U_PER_T];
#pragma unroll
    for (int j = 0; j < U_PER_T; j++) {
        const int i = tid + j * TILE_BS;
        const int xx = x0 - 1 + i % UXR, yy = y0 - 1 + i / UXR;
        hok[j] = i < NU_T && xx >= 0 && yy >= 0 && xx < vx && yy < vy;
        hxy[j] = hok[j] ? xx + (long)vx * yy : 0;
    }
    // zero the node-layer slots once: the pad columns are read by the pad element
    for (int i = tid; i < 3 * 2 * 3 * NU2; i += TILE_BS) (&S.u[0][0][0][0])[i] = 0.f;

    T pu[U_PER_T][3];
    float2 pw = make_float2(0.f, 0.f);
    auto fetch_layer = [&](int L) {
#pragma unroll
        for (int j = 0; j < U_PER_T; j++) {
            T a = T(0), b = T(0), c = T(0);
            if (hok[j] && L >= 0 && L < vz) {
                const long v = hxy[j] + plane * L;
                if (!(WS && vfix[v])) {
                    a = u[v];
                    b = u[nv + v];
                    c = u[2 * nv + v];
                }
            }
            pu[j][0] = a;
            pu[j][1] = b;
            pu[j][2] = c;
        }
    };
    auto stash_layer = [&](int L) {
        float(*dst)[3][NU2] = S.u[(L + 3) % 3];
#pragma unroll
        for (int j = 0; j < U_PER_T; j++) {
            const int i = tid + j * TILE_BS;
            if (i < NU_T) {
                const int row = i / UXR, col = i % UXR;
                const int o = row * UXP + col;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    dst[0][c][o] = pu[j][c];
                    if (col >= 1) dst[1][c][o - 1] = pu[j][c];
                }
            }
        }
    };
    auto fetch_w = [&](int ez) {
        const bool zok = ez >= 0 && ez < nz;
        const long base = (long)nx * ny * ez;
        pw.x = (e0_ok && zok) ? wgt[exy0 + base] : 0.f;
        pw.y = (e1_ok && zok) ? wgt[ex0 + 1 + (long)nx * eyg + base] : 0.f;
    };
    auto stash_w = [&](int ez) {
        if (pair_thread) *reinterpret_cast<float2*>(&S.w[(ez + 4) & 3][prow * EXP + 2 * pm]) = pw;
    };
    auto element_phase = [&](int e) {
        if (!pair_thread) return;
        const float2 wv = *reinterpret_cast<const float2*>(&S.w[(e + 4) & 3][prow * EXP + 2 * pm]);
        float2 a[24];
        if (wv.x != 0.f || wv.y != 0.f) {
            const float(*lo)[3][NU2] = S.u[(e + 3) % 3];
            const float(*hi)[3][NU2] = S.u[(e + 4) % 3];
#pragma unroll
            for (int vtx = 0; vtx < 8; vtx++) {
                const float(*src)[3][NU2] = (vtx & 4) ? hi : lo;
                const int idx = (prow + ((vtx >> 1) & 1)) * UXP + 2 * pm;
#pragma unroll
                for (int c = 0; c < 3; c++) a[3 * vtx + c] = *reinterpret_cast<const float2*>(&src[vtx & 1][c][idx]);
            }
            rte::element_apply2(a, kt, wv);
        } else {
#pragma unroll
            for (int q = 0; q < 24; q++) a[q] = make_float2(0.f, 0.f);
        }
        float* dst = &S.e[(e + 2) & 1][0][0];
#pragma unroll
        for (int q = 0; q < 24; q++) *reinterpret_cast<float2*>(&dst[q * NE2 + prow * EXP + 2 * pm]) = a[q];
    };

    fetch_layer(zb - 1);
    fetch_w(zb - 1);
    __syncthreads();  // the zeroed slots before the first stores
    stash_layer(zb - 1);
    stash_w(zb - 1);
    fetch_layer(zb);
    stash_layer(zb);
    fetch_layer(zb + 1);
    stash_layer(zb + 1);
    fetch_w(zb);
    stash_w(zb);
    __syncthreads();
    element_phase(zb - 1);
    fetch_layer(zb + 2);
    fetch_w(zb + 1);
    __syncthreads();

    T acc[3] = {T(0), T(0), T(0)};
    for (int t = zb - 1; t < ze; t++) {
        if (t + 3 <= ze) stash_layer(t + 3);
        if (t + 2 < ze) stash_w(t + 2);
        if (t + 4 <= ze) fetch_layer(t + 4);
        if (t + 3 < ze) fetch_w(t + 3);
        const bool out_layer = t >= zb;
        T fv[3] = {T(0), T(0), T(0)}, uo[3] = {T(0), T(0), T(0)}, dv[3] = {T(0), T(0), T(0)};
        bool act = false, fixed = false;
        long vout = 0;
        if (node_thread && out_layer) {
            vout = vxy + plane * t;
            act = vact[vout];
            fixed = WS && act && vfix[vout];
            if (MODE != 1)
#pragma unroll
                for (int c = 0; c < 3; c++) fv[c] = f[c * nv + vout];
            if (MODE >= 1)
#pragma unroll
                for (int c = 0; c < 3; c++) uo[c] = u[c * nv + vout];
            if (MODE == 3 && kstep > 0)
#pragma unroll
                for (int c = 0; c < 3; c++) dv[c] = dvec[c * nv + vout];
        }
        if (t + 1 < ze) element_phase(t + 1);
        if (node_thread) {
            const T* E = &S.e[(t + 2) & 1][0][0];
            if (out_layer) {
#pragma unroll
                for (int dy = 0; dy < 2; dy++)
#pragma unroll
                    for (int dx = 0; dx < 2; dx++) {
                        const int el = (nyl + dy) * EXP + nxl + dx;
                        const int vtx = (1 - dx) + 2 * (1 - dy);
#pragma unroll
                        for (int c = 0; c < 3; c++) acc[c] += E[(3 * vtx + c) * NE2 + el];
                    }
                const long v = vout;
                if (MODE == 0) {
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? fv[c] : fv[c] - acc[c]) : T(0);
                } else if (MODE == 1) {
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? uo[c] : acc[c]) : T(0);
                } else {
                    T nu[3], dn[3];
                    node_smooth<T, MODE, EXP>(kt, S.w[(t + 3) & 3], S.w[(t + 4) & 3], nyl * EXP + nxl, acc, fv, uo,
                                              dv, act, fixed, omega, cheb_a, cheb_b, kstep, nu, dn);
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = nu[c];
                    if (MODE == 3)
#pragma unroll
                        for (int c = 0; c < 3; c++) dvec[c * nv + v] = dn[c];
                }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) acc[c] = T(0);
#pragma unroll
            for (int dy = 0; dy < 2; dy++)
#pragma unroll
                for (int dx = 0; dx < 2; dx++) {
                    const int el = (nyl + dy) * EXP + nxl + dx;
                    const int vtx = (1 - dx) + 2 * (1 - dy) + 4;
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[c] += E[(3 * vtx + c) * NE2 + el];
                }
        }
        __syncthreads();
    }
}


// ---------------------------------------------------------------------------
// variants 6 and 7: the pipelined tile kernel with its node layers staged by the Tensor Memory
// Accelerator.  One thread issues, per node layer, a 4-D tiled bulk tensor copy of the
// (TY+2) x 40 node halo box of all three components (x from the halo's first column X0 - 1
// rounded down to a 16-byte boundary, at most 3 columns earlier) and, with supports, a 3-D copy
// of the 64-wide box of support flags (x rounded down to a multiple of 16), into a ring of 3
// shared slots completed on one mbarrier each.  Layer t + 3 is issued at the top of iteration t,
// into the slot of layer t, whose last reader (element phase t) ran before the previous barrier,
// and waited for at its end, so the copy overlaps that iteration's element and node work (the
// register prefetch of variant 3, without its load instructions).  (A fourth slot, which would
// let the node phase read its own u from shared memory, costs a block per SM at 4 rows and was
// slower.)  Coordinates outside the node box read as zeros (the tile kernel's halo rule).  After a layer's barrier completes, the block
// zeroes the displacements of fixed nodes (the WS rule) before the iteration's block-wide
// barrier.  Every mbarrier wait is bounded: a timed-out wait flags *err = 3, poisons out[0],
// waits (bounded) for the block's copies still in flight and returns.  Applies where the node
// box's x extent is a multiple of 16 (the tensor maps' row pitch must be a multiple of 16 bytes
// for the one-byte flags); the tensor maps cover this GPU's own memory and no copy uses
// multicast.  Variant 6 tiles 32 x TY nodes, variant 7 31 x TY (element rows of 32).
// ---------------------------------------------------------------------------
constexpr int TMA_BX = 40;  // node box x extent (x from the halo's first column rounded down to 4)
constexpr int TMA_FX = 64;  // flag box x extent (x from the same column rounded down to 16)

// tile of the TMA-staged kernel: TXN x TY nodes.  Node threads are laid out one warp per node row
// (lane = x; with TXN = 31 the last lane of each row idles); element threads (TXN+1) x (TY+1).
// TXN = 32 is variant 3's tile; TXN = 31 makes the element tile 32 x (TY+1), whole warps, where
// the 33-wide rows of TXN = 32 leave a last warp with TY+1 of 32 lanes busy.
template <int TY_, int TXN>
struct TTile {
    static constexpr int TX = TXN, TY = TY_;
    static constexpr int EXT = TX + 1, EYT = TY + 1;  // element tile
    static constexpr int UXT = TX + 2, UYT = TY + 2;  // node halo tile
    static constexpr int NE_T = EXT * EYT;
    static constexpr int NU_T = UXT * UYT;
    static constexpr int NODE_T = 32 * TY;
    static constexpr int BS = ((NE_T > NODE_T ? NE_T : NODE_T) + 31) / 32 * 32;
};

template <typename T, int TY_, int TXN>
constexpr int tma_min_blocks() {
    return sizeof(T) == 8 ? (TY_ == 4 ? 2 : 1) : (TY_ == 4 ? 5 : 3);  // TY 6 and 8: 3 (FP32), 1 (FP64)
}

template <typename T, int TY_, int TXN>
struct TmaSmem {
    static constexpr int SLOT = ((3 * (TY_ + 2) * TMA_BX * (int)sizeof(T) + 127) / 128 * 128) / (int)sizeof(T);
    static constexpr int NE_T = TTile<TY_, TXN>::NE_T;
    alignas(128) T u[3][SLOT];                       // node layer j (relative to zb - 1) in slot j % 3: [3][TY+2][40]
    alignas(128) uint8_t fx[3][(TY_ + 2) * TMA_FX];  // support flags of the same layers: [TY+2][64]
    T e[2][24][NE_T];
    float w[4][NE_T];
    uint64_t bar[3];
};

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int c,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(rttc::smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(rttc::smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(rttc::smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(rttc::smem_u32(bar))
        : "memory");
}

template <typename T, bool WS, int MODE, int TY_, int TXN>
__global__ void __launch_bounds__(TTile<TY_, TXN>::BS, tma_min_blocks<T, TY_, TXN>()) k_fine_pipe_tma(
    int nx, int ny, int nz, int zchunk, const uint8_t* __restrict__ vact, const float* __restrict__ wgt,
    const uint8_t* __restrict__ vfix, const rte::KtVals<T> kt, const __grid_constant__ CUtensorMap umap,
    const __grid_constant__ CUtensorMap fmap, const T* __restrict__ u, const T* __restrict__ f, T* __restrict__ out,
    T omega, T* __restrict__ dvec, const double* __restrict__ coef, int kstep, double* err) {
    using TS = TTile<TY_, TXN>;
    constexpr int TX = TS::TX, TY = TS::TY, EXT = TS::EXT, UXT = TS::UXT, NE_T = TS::NE_T, NU_T = TS::NU_T;
    constexpr int TILE_BS = TS::BS, NODE_T = TS::NODE_T;
    constexpr int ROWB = TMA_BX;           // row pitch of a staged component
    constexpr int CP = (TY + 2) * TMA_BX;  // component pitch of a staged layer
    constexpr uint32_t UBYTES = 3u * (TY + 2) * TMA_BX * sizeof(T);
    constexpr uint32_t FBYTES = WS ? (uint32_t)(TY + 2) * TMA_FX : 0u;
    // the copies' shared destinations sit on 128-byte boundaries: the block's dynamic shared
    // memory (sizeof(TmaSmem) + 128 bytes) is rounded up to one
    extern __shared__ __align__(16) unsigned char smraw[];
    TmaSmem<T, TY_, TXN>& S =
        *reinterpret_cast<TmaSmem<T, TY_, TXN>*>(smraw + ((128 - (rttc::smem_u32(smraw) & 127)) & 127));
    T cheb_a = T(0), cheb_b = T(0);
    if (MODE == 3) {
        const double ca = coef[2 * kstep], cb = coef[2 * kstep + 1];
        cheb_a = (T)ca;
        cheb_b = (T)cb;
    }
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long plane = (long)vx * vy;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * zchunk;
    const int ze = min(zb + zchunk, vz);
    const int tid = threadIdx.x;
    const int nxl = tid & 31, nyl = tid >> 5;
    const int nxg = x0 + nxl, nyg = y0 + nyl;
    const bool node_thread = tid < NODE_T && nxl < TX && nxg < vx && nyg < vy;
    const long vxy = node_thread ? nxg + (long)vx * nyg : 0;
    const int exl = tid % EXT, eyl = tid / EXT;
    const int exg = x0 - 1 + exl, eyg = y0 - 1 + eyl;
    const bool elem_xy = tid < NE_T && exg >= 0 && eyg >= 0 && exg < nx && eyg < ny;
    const long exy = elem_xy ? exg + (long)nx * eyg : 0;
    const int zlast = ze;  // node layers zb - 1 .. ze are read
    // the halo's first column x0 - 1, rounded down to the copies' 16-byte boundaries (4 or 2
    // elements of the node vectors, 16 one-byte flags), and its index inside the staged boxes
    const int xs = (x0 - 1) & ~3, xf = (x0 - 1) & ~15;
    const int off = (x0 - 1) - xs, offf = (x0 - 1) - xf;
    // layer L lives in slot (L - zb + 1) % 3, phase parity ((L - zb + 1) / 3) & 1
    auto slot_of = [&](int L) { return (L - zb + 1) % 3; };
    auto parity_of = [&](int L) { return (uint32_t)(((L - zb + 1) / 3) & 1); };
    auto issue_to = [&](int L, int sl) {  // thread 0 only
        rttc::mbar_expect_tx(&S.bar[sl], UBYTES + FBYTES);
        tma_load_4d(&S.u[sl][0], &umap, xs, y0 - 1, L, 0, &S.bar[sl]);
        if (WS) tma_load_3d(&S.fx[sl][0], &fmap, xf, y0 - 1, L, &S.bar[sl]);
    };
    auto issue = [&](int L) { issue_to(L, slot_of(L)); };
    // every thread waits for layer L; false if the wait ran out
    auto wait_layer = [&](int L) -> bool { return rttc::mbar_wait(&S.bar[slot_of(L)], parity_of(L)); };
    // fixed nodes enter the element products as zero
    auto mask_slot = [&](int sl) {
        if (!WS) return;
        for (int i = tid; i < NU_T; i += TILE_BS) {
            const int row = i / UXT, col = i % UXT;
            if (S.fx[sl][row * TMA_FX + col + offf]) {
                T* b = &S.u[sl][row * ROWB + col + off];
                b[0] = T(0);
                b[CP] = T(0);
                b[2 * CP] = T(0);
            }
        }
    };
    auto mask_layer = [&](int L) { mask_slot(slot_of(L)); };
    int issued = zb - 2;  // last layer whose copy was issued (uniform across the block)
    // bounded drain of the copies still in flight, then the error report
    auto give_up = [&](int first_pending) {
        for (int L = first_pending; L <= issued; L++) rttc::mbar_wait(&S.bar[slot_of(L)], parity_of(L));
        if (tid == 0) {
            *err = 3.0;
            out[0] = (T)__int_as_float(0x7fc00000);
        }
    };

    float pw = 0.f;
    auto fetch_w = [&](int ez) {
        pw = (elem_xy && ez >= 0 && ez < nz) ? wgt[exy + (long)nx * ny * ez] : 0.f;
    };
    auto stash_w = [&](int ez) {
        if (tid < NE_T) S.w[(ez + 4) & 3][tid] = pw;
    };
    // element layer e from the node layers in slots slo (layer e) and shi (layer e + 1)
    auto element_phase_s = [&](int e, int slo, int shi) {
        if (tid >= NE_T) return;
        T a[24];
        const float wv = S.w[(e + 4) & 3][tid];
        if (wv != 0.f) {
            const T* lo = &S.u[slo][0];
            const T* hi = &S.u[shi][0];
#pragma unroll
            for (int vtx = 0; vtx < 8; vtx++) {
                const T* src = (vtx & 4) ? hi : lo;
                const int idx = (eyl + ((vtx >> 1) & 1)) * ROWB + exl + (vtx & 1) + off;
                a[3 * vtx] = src[idx];
                a[3 * vtx + 1] = src[CP + idx];
                a[3 * vtx + 2] = src[2 * CP + idx];
            }
            rte::element_apply(a, kt, T(wv));
        } else {
#pragma unroll
            for (int q = 0; q < 24; q++) a[q] = T(0);
        }
        T* dst = &S.e[(e + 2) & 1][0][0];
#pragma unroll
        for (int q = 0; q < 24; q++) dst[q * NE_T + tid] = a[q];
    };
    auto element_phase = [&](int e) { element_phase_s(e, slot_of(e), slot_of(e + 1)); };

    // prologue: barriers, layers zb-1 .. zb+1 copied, waited for and masked, weights of element
    // layers zb-1, zb stashed, element layer zb-1 computed
    if (tid == 0) {
        for (int i = 0; i < 3; i++) rttc::mbar_init(&S.bar[i], 1);
        rttc::fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int L = zb - 1; L <= zb + 1 && L <= zlast; L++) issue(L);
    issued = min(zb + 1, zlast);
    fetch_w(zb - 1);
    stash_w(zb - 1);
    fetch_w(zb);
    stash_w(zb);
    bool ok = true;
    for (int L = zb - 1; L <= zb + 1 && L <= zlast; L++) ok = wait_layer(L) && ok;
    if (__syncthreads_or(!ok)) {
        give_up(zb - 1);
        return;
    }
    for (int L = zb - 1; L <= zb + 1 && L <= zlast; L++) mask_layer(L);
    __syncthreads();
    element_phase(zb - 1);
    fetch_w(zb + 1);
    __syncthreads();

    T acc[3] = {T(0), T(0), T(0)};
    // slots and phase parity carried from iteration to iteration instead of divisions by 3:
    // r3 = slot of layers t and t + 3, (r3 + 1) % 3 of layer t + 1, (r3 + 2) % 3 of layer t + 2;
    // q3 = (t + 3 - zb + 1) / 3, whose low bit is the parity of layer t + 3's phase
    int r3 = 0, q3 = 1;
    for (int t = zb - 1; t < ze; t++) {
        const int s1 = r3 == 2 ? 0 : r3 + 1, s2 = r3 == 0 ? 2 : r3 - 1;
        // the slot of layer t + 3 held layer t, last read by element phase t (previous iteration)
        if (t + 3 <= zlast) {
            if (tid == 0) {
                rttc::fence_async_smem();
                issue_to(t + 3, r3);
            }
            issued = t + 3;
        }
        if (t + 2 < ze) stash_w(t + 2);
        if (t + 3 < ze) fetch_w(t + 3);
        const bool out_layer = t >= zb;
        T fv[3] = {T(0), T(0), T(0)}, uo[3] = {T(0), T(0), T(0)}, dv[3] = {T(0), T(0), T(0)};
        bool act = false, fixed = false;
        long vout = 0;
        if (node_thread && out_layer) {
            vout = vxy + plane * t;
            act = vact[vout];
            fixed = WS && act && vfix[vout];
            if (MODE != 1)
#pragma unroll
                for (int c = 0; c < 3; c++) fv[c] = f[c * nv + vout];
            if (MODE >= 1)
#pragma unroll
                for (int c = 0; c < 3; c++) uo[c] = u[c * nv + vout];
            if (MODE == 3 && kstep > 0)
#pragma unroll
                for (int c = 0; c < 3; c++) dv[c] = dvec[c * nv + vout];
        }
        if (t + 1 < ze) element_phase_s(t + 1, s1, s2);
        if (node_thread) {
            const T* E = &S.e[(t + 2) & 1][0][0];
            if (out_layer) {
#pragma unroll
                for (int dy = 0; dy < 2; dy++)
#pragma unroll
                    for (int dx = 0; dx < 2; dx++) {
                        const int el = (nyl + dy) * EXT + nxl + dx;
                        const int vtx = (1 - dx) + 2 * (1 - dy);
#pragma unroll
                        for (int c = 0; c < 3; c++) acc[c] += E[(3 * vtx + c) * NE_T + el];
                    }
                const long v = vout;
                if (MODE == 0) {
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? fv[c] : fv[c] - acc[c]) : T(0);
                } else if (MODE == 1) {
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = act ? (fixed ? uo[c] : acc[c]) : T(0);
                } else {
                    T nu[3], dn[3];
                    node_smooth<T, MODE, EXT>(kt, S.w[(t + 3) & 3], S.w[(t + 4) & 3], nyl * EXT + nxl, acc, fv, uo,
                                              dv, act, fixed, omega, cheb_a, cheb_b, kstep, nu, dn);
#pragma unroll
                    for (int c = 0; c < 3; c++) out[c * nv + v] = nu[c];
                    if (MODE == 3)
#pragma unroll
                        for (int c = 0; c < 3; c++) dvec[c * nv + v] = dn[c];
                }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) acc[c] = T(0);
#pragma unroll
            for (int dy = 0; dy < 2; dy++)
#pragma unroll
                for (int dx = 0; dx < 2; dx++) {
                    const int el = (nyl + dy) * EXT + nxl + dx;
                    const int vtx = (1 - dx) + 2 * (1 - dy) + 4;
#pragma unroll
                    for (int c = 0; c < 3; c++) acc[c] += E[(3 * vtx + c) * NE_T + el];
                }
        }
        // layer t + 3 (read by element phase t + 2, next iteration) complete and masked; the
        // iteration's barrier publishes the masking
        ok = true;
        if (t + 3 <= zlast) ok = rttc::mbar_wait(&S.bar[r3], (uint32_t)(q3 & 1));
        if (ok && t + 3 <= zlast) mask_slot(r3);
        if (++r3 == 3) {
            r3 = 0;
            q3++;
        }
        if (__syncthreads_or(!ok)) {
            give_up(t + 3);
            return;
        }
    }
}

// tensor maps of the TMA-staged variant: cuTensorMapEncodeTiled through the runtime's driver
// entry point (no link against libcuda); maps cached by (address, element size, box), since the
// Chebyshev steps alternate between a few vectors
using tmap_encode_t = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

tmap_encode_t tmap_encoder() {
    static tmap_encode_t fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<tmap_encode_t>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

struct TmapKey {
    const void* p;
    int esize, vx, vy, vz, rows;
    bool operator==(const TmapKey& o) const {
        return p == o.p && esize == o.esize && vx == o.vx && vy == o.vy && vz == o.vz && rows == o.rows;
    }
};
struct TmapHash {
    size_t operator()(const TmapKey& k) const {
        return std::hash<const void*>()(k.p) ^ ((size_t)k.esize << 1) ^ ((size_t)k.vx << 7) ^ ((size_t)k.rows << 23) ^
               ((size_t)k.vz << 31);
    }
};
std::mutex g_tmap_mutex;
std::unordered_map<TmapKey, CUtensorMap, TmapHash> g_tmaps;

// node vectors [3][vz][vy][vx] (esize 4 or 8) as 4-D boxes {40, rows, 1, 3}; flags [vz][vy][vx] bytes
// (esize 1) as 3-D boxes {64, rows, 1}; false if the encoder refuses (then variant 3 runs)
bool tmap_get(const void* p, int esize, int vx, int vy, int vz, int rows, CUtensorMap* out) {
    const TmapKey key{p, esize, vx, vy, vz, rows};
    std::lock_guard<std::mutex> lk(g_tmap_mutex);
    auto it = g_tmaps.find(key);
    if (it != g_tmaps.end()) {
        *out = it->second;
        return true;
    }
    tmap_encode_t enc = tmap_encoder();
    if (!enc) return false;
    CUtensorMap m;
    memset(&m, 0, sizeof(m));
    CUresult r;
    if (esize == 1) {
        const cuuint64_t dims[3] = {(cuuint64_t)vx, (cuuint64_t)vy, (cuuint64_t)vz};
        const cuuint64_t strides[2] = {(cuuint64_t)vx, (cuuint64_t)vx * vy};
        const cuuint32_t box[3] = {(cuuint32_t)TMA_FX, (cuuint32_t)rows, 1u};
        const cuuint32_t estr[3] = {1u, 1u, 1u};
        r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(p), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        const cuuint64_t nv = (cuuint64_t)vx * vy * vz;
        const cuuint64_t dims[4] = {(cuuint64_t)vx, (cuuint64_t)vy, (cuuint64_t)vz, 3};
        const cuuint64_t strides[3] = {(cuuint64_t)vx * esize, (cuuint64_t)vx * vy * esize, nv * esize};
        const cuuint32_t box[4] = {(cuuint32_t)TMA_BX, (cuuint32_t)rows, 1u, 3u};
        const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
        r = enc(&m, esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                const_cast<void*>(p), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    if (r != CUDA_SUCCESS) return false;
    if (g_tmaps.size() > 256) g_tmaps.clear();
    g_tmaps.emplace(key, m);
    *out = m;
    return true;
}

template <typename T, bool WS, int MODE, int TY_, int TXN>
int launch_tma_ty(rt_hier* h, const T* u, const T* f, T* out, double omega, const char* name, T* dvec,
                  const double* coef, int kstep, bool* done) {
    rt_level& L = h->L[0];
    *done = false;
    CUtensorMap umap, fmap;
    memset(&fmap, 0, sizeof(fmap));
    // the maps' base addresses must sit on 16-byte boundaries
    if ((reinterpret_cast<uintptr_t>(u) & 15) || (WS && (reinterpret_cast<uintptr_t>(h->vfix) & 15))) return RT_OK;
    if (!tmap_get(u, (int)sizeof(T), L.vx, L.vy, L.vz, TY_ + 2, &umap)) return RT_OK;
    if (WS && !tmap_get(h->vfix, 1, L.vx, L.vy, L.vz, TY_ + 2, &fmap)) return RT_OK;
    const int zc = h->tune[sizeof(T) == 8 ? 1 : 0][MODE].zchunk;
    dim3 grid((L.vx + TXN - 1) / TXN, (L.vy + TY_ - 1) / TY_, (L.vz + zc - 1) / zc);
    const rte::KtVals<T> kt = rte::make_kt<T>(h);
    *done = true;
    return rt_launch(h->ctx, name, [&] {
        k_fine_pipe_tma<T, WS, MODE, TY_, TXN>
            <<<grid, TTile<TY_, TXN>::BS, sizeof(TmaSmem<T, TY_, TXN>) + 128, h->ctx->stream>>>(
            L.nx, L.ny, L.nz, zc, L.vact, h->w, h->vfix, kt, umap, fmap, u, f, out, (T)omega, dvec, coef, kstep,
            h->scal + RT_SCAL_ERR);
    });
}

template <typename T, bool WS, int MODE, int TY_, bool PIPE>
int launch_tile_ty(rt_hier* h, const T* u, const T* f, T* out, double omega, const char* name, T* dvec,
                   const double* coef, int kstep) {
    rt_level& L = h->L[0];
    const size_t smem = PIPE ? sizeof(PipeSmem<T, TY_>) : sizeof(TileSmem<T, TY_>);
    const int zc = h->tune[sizeof(T) == 8 ? 1 : 0][MODE].zchunk;
    dim3 grid((L.vx + Tile<TY_>::TX - 1) / Tile<TY_>::TX, (L.vy + TY_ - 1) / TY_, (L.vz + zc - 1) / zc);
    const rte::KtVals<T> kt = rte::make_kt<T>(h);
    return rt_launch(h->ctx, name, [&] {
        if (PIPE)
            k_fine_pipe<T, WS, MODE, TY_><<<grid, Tile<TY_>::BS, smem, h->ctx->stream>>>(
                L.nx, L.ny, L.nz, zc, L.vact, h->w, h->vfix, kt, u, f, out, (T)omega, dvec, coef, kstep);
        else
            k_fine_tile<T, WS, MODE, TY_><<<grid, Tile<TY_>::BS, smem, h->ctx->stream>>>(
                L.nx, L.ny, L.nz, zc, L.vact, h->w, h->vfix, kt, u, f, out, (T)omega, dvec, coef, kstep);
    });
}

template <bool WS, int MODE, int TY_>
int launch_pair_ty(rt_hier* h, const float* u, const float* f, float* out, double omega, const char* name, float* dvec,
                   const double* coef, int kstep) {
    rt_level& L = h->L[0];
    const int zc = h->tune[0][MODE].zchunk;
    dim3 grid((L.vx + 31) / 32, (L.vy + TY_ - 1) / TY_, (L.vz + zc - 1) / zc);
    const rte::KtVals<float> kt = rte::make_kt<float>(h);
    return rt_launch(h->ctx, name, [&] {
        k_fine_pair<WS, MODE, TY_><<<grid, PTile<TY_>::BS, sizeof(PairSmem<TY_>), h->ctx->stream>>>(
            L.nx, L.ny, L.nz, zc, L.vact, h->w, h->vfix, kt, u, f, out, (float)omega, dvec, coef, kstep);
    });
}

// variant 0: two barriers per element layer; 3: software-pipelined, one barrier per layer;
// 4 (FP32): pipelined with element pairs in packed FP32; 5: sum-factorised row marching (rt_fine_sf.cu);
// 6: variant 3 with its node layers staged by TMA (node boxes whose x extent is a multiple of 16);
// 7: variant 6 on 31-node-wide tiles (element rows of 32: whole warps)
template <typename T, bool WS, int MODE>
int launch_tile(rt_hier* h, const T* u, const T* f, T* out, double omega, const char* name, T* dvec = nullptr,
                const double* coef = nullptr, int kstep = 0) {
    const rt_tile_cfg& tn = h->tune[sizeof(T) == 8 ? 1 : 0][MODE];
    if (tn.variant == 5) return rtk::launch_sf<T, WS, MODE>(h, u, f, out, omega, name, dvec, coef, kstep);
    if ((tn.variant == 6 || tn.variant == 7) && h->L[0].vx % 16 == 0) {
        bool done = false;
        int st;
        if (tn.variant == 6)
            st = tn.ty == 4 ? launch_tma_ty<T, WS, MODE, 4, 32>(h, u, f, out, omega, name, dvec, coef, kstep, &done)
                            : launch_tma_ty<T, WS, MODE, 8, 32>(h, u, f, out, omega, name, dvec, coef, kstep, &done);
        else if (tn.ty == 4)
            st = launch_tma_ty<T, WS, MODE, 4, 31>(h, u, f, out, omega, name, dvec, coef, kstep, &done);
        else if (tn.ty == 6)
            st = launch_tma_ty<T, WS, MODE, 6, 31>(h, u, f, out, omega, name, dvec, coef, kstep, &done);
        else
            st = launch_tma_ty<T, WS, MODE, 8, 31>(h, u, f, out, omega, name, dvec, coef, kstep, &done);
        if (done || st != RT_OK) return st;
        // the tensor maps could not be made: the same schedule with per-thread loads
    }
    if (tn.variant == 6 || tn.variant == 7) {
        switch (tn.ty) {
            case 4: return launch_tile_ty<T, WS, MODE, 4, true>(h, u, f, out, omega, name, dvec, coef, kstep);
            default: return launch_tile_ty<T, WS, MODE, 8, true>(h, u, f, out, omega, name, dvec, coef, kstep);
        }
    }
    if constexpr (sizeof(T) == 4) {
        if (tn.variant == 4) {
            switch (tn.ty) {
                case 2: return launch_pair_ty<WS, MODE, 2>(h, u, f, out, omega, name, dvec, coef, kstep);
                case 8: return launch_pair_ty<WS, MODE, 8>(h, u, f, out, omega, name, dvec, coef, kstep);
                default: return launch_pair_ty<WS, MODE, 4>(h, u, f, out, omega, name, dvec, coef, kstep);
            }
        }
    }
    if (tn.variant == 3) {
        switch (tn.ty) {
            case 2: return launch_tile_ty<T, WS, MODE, 2, true>(h, u, f, out, omega, name, dvec, coef, kstep);
            case 8: return launch_tile_ty<T, WS, MODE, 8, true>(h, u, f, out, omega, name, dvec, coef, kstep);
            default: return launch_tile_ty<T, WS, MODE, 4, true>(h, u, f, out, omega, name, dvec, coef, kstep);
        }
    }
    switch (tn.ty) {
        case 2: return launch_tile_ty<T, WS, MODE, 2, false>(h, u, f, out, omega, name, dvec, coef, kstep);
        case 8: return launch_tile_ty<T, WS, MODE, 8, false>(h, u, f, out, omega, name, dvec, coef, kstep);
        default: return launch_tile_ty<T, WS, MODE, 4, false>(h, u, f, out, omega, name, dvec, coef, kstep);
    }
}

template <typename T, bool WS, int MODE, int TY_>
cudaError_t set_attr() {
    cudaError_t e = cudaFuncSetAttribute(k_fine_tile<T, WS, MODE, TY_>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(TileSmem<T, TY_>));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_fine_pipe<T, WS, MODE, TY_>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(PipeSmem<T, TY_>));
}

template <typename T, bool WS, int MODE, int TY_, int TXN>
cudaError_t set_attr_tma() {
    return cudaFuncSetAttribute(k_fine_pipe_tma<T, WS, MODE, TY_, TXN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(TmaSmem<T, TY_, TXN>) + 128);
}

template <typename T, int TY_, int TXN>
cudaError_t set_attrs_tma_x() {
    cudaError_t r[8] = {set_attr_tma<T, false, 0, TY_, TXN>(), set_attr_tma<T, false, 1, TY_, TXN>(),
                        set_attr_tma<T, false, 2, TY_, TXN>(), set_attr_tma<T, false, 3, TY_, TXN>(),
                        set_attr_tma<T, true, 0, TY_, TXN>(),  set_attr_tma<T, true, 1, TY_, TXN>(),
                        set_attr_tma<T, true, 2, TY_, TXN>(),  set_attr_tma<T, true, 3, TY_, TXN>()};
    for (auto x : r)
        if (x != cudaSuccess) return x;
    return cudaSuccess;
}

template <typename T, int TY_>
cudaError_t set_attrs_tma() {
    const cudaError_t a = set_attrs_tma_x<T, TY_, 32>();
    const cudaError_t b = a != cudaSuccess ? a : set_attrs_tma_x<T, TY_, 31>();
    return b != cudaSuccess || TY_ != 4 ? b : set_attrs_tma_x<T, 6, 31>();  // 6 rows: 31-wide tiles only
}

template <bool WS, int MODE, int TY_>
cudaError_t set_attr_pair() {
    return cudaFuncSetAttribute(k_fine_pair<WS, MODE, TY_>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(PairSmem<TY_>));
}

template <int TY_>
cudaError_t set_attrs_pair() {
    cudaError_t e = cudaSuccess;
    cudaError_t r[8] = {set_attr_pair<false, 0, TY_>(), set_attr_pair<false, 1, TY_>(), set_attr_pair<false, 2, TY_>(),
                        set_attr_pair<false, 3, TY_>(), set_attr_pair<true, 0, TY_>(),  set_attr_pair<true, 1, TY_>(),
                        set_attr_pair<true, 2, TY_>(),  set_attr_pair<true, 3, TY_>()};
    for (auto x : r)
        if (x != cudaSuccess) e = x;
    return e;
}

template <typename T, int TY_>
cudaError_t set_attrs_T() {
    cudaError_t e = cudaSuccess;
    cudaError_t r[8] = {set_attr<T, false, 0, TY_>(), set_attr<T, false, 1, TY_>(), set_attr<T, false, 2, TY_>(),
                        set_attr<T, false, 3, TY_>(), set_attr<T, true, 0, TY_>(),  set_attr<T, true, 1, TY_>(),
                        set_attr<T, true, 2, TY_>(),  set_attr<T, true, 3, TY_>()};
    for (auto x : r)
        if (x != cudaSuccess) e = x;
    return e;
}

}  // namespace

namespace rtk {

// dynamic shared-memory limits of every tile-kernel variant, set once per device
// (before any stream capture can include a launch)
int init_tile_kernels(rt_ctx* c) {
    cudaError_t es[13] = {set_attrs_T<double, 2>(),   set_attrs_T<double, 4>(),   set_attrs_T<double, 8>(),
                          set_attrs_T<float, 2>(),    set_attrs_T<float, 4>(),    set_attrs_T<float, 8>(),
                          set_attrs_pair<2>(),        set_attrs_pair<4>(),        set_attrs_pair<8>(),
                          set_attrs_tma<float, 4>(),  set_attrs_tma<float, 8>(),  set_attrs_tma<double, 4>(),
                          set_attrs_tma<double, 8>()};
    for (cudaError_t e : es)
        if (e != cudaSuccess) return rt_fail(c, RT_ECUDA, "tile kernel attributes: %s", cudaGetErrorString(e));
    return RT_OK;
}

// default launch shape (rt_autotune refines it): enough z-chunks for ~4 tiles per SM
int tile_zchunk_default(rt_ctx* c, int vx, int vy, int vz) {
    const long tiles = (long)((vx + 29) / 30) * ((vy + 3) / 4);
    const long target = (long)c->sm_count * 16;  // marching kernel: 4 warps per CTA, ~16 warps per SM
    long chunks = (target + tiles - 1) / tiles;
    if (chunks < 1) chunks = 1;
    int zc = (int)((vz + chunks - 1) / chunks);
    return zc < 8 ? 8 : zc;
}

template <typename T>
static bool use_march(rt_hier* h, int mode) {
    const int v = h->tune[sizeof(T) == 8 ? 1 : 0][mode].variant;
    return v == 1 || v == 2;  // 1: marching, 2: marching with prefetch (0, 3, 4: tile kernels)
}

template <typename T>
int fine_residual(rt_hier* h, const T* u, const T* f, T* r) {
    if (use_march<T>(h, 0)) return fine_march<T, 0>(h, u, f, r, 0.0, nullptr, nullptr, 0);
    const char* nm = sizeof(T) == 8 ? "fine_residual_f64" : "fine_residual_f32";
    return h->has_support ? launch_tile<T, true, 0>(h, u, f, r, 0.0, nm) : launch_tile<T, false, 0>(h, u, f, r, 0.0, nm);
}

template <typename T>
int fine_applyK(rt_hier* h, const T* u, T* out) {
    if (use_march<T>(h, 1)) return fine_march<T, 1>(h, u, nullptr, out, 0.0, nullptr, nullptr, 0);
    const char* nm = sizeof(T) == 8 ? "fine_applyK_f64" : "fine_applyK_f32";
    return h->has_support ? launch_tile<T, true, 1>(h, u, nullptr, out, 0.0, nm)
                          : launch_tile<T, false, 1>(h, u, nullptr, out, 0.0, nm);
}

template <typename T>
int fine_jacobi(rt_hier* h, const T* u, const T* f, T* unew, double omega) {
    if (use_march<T>(h, 2)) return fine_march<T, 2>(h, u, f, unew, omega, nullptr, nullptr, 0);
    const char* nm = sizeof(T) == 8 ? "fine_jacobi_f64" : "fine_jacobi_f32";
    return h->has_support ? launch_tile<T, true, 2>(h, u, f, unew, omega, nm)
                          : launch_tile<T, false, 2>(h, u, f, unew, omega, nm);
}

template <typename T>
int fine_cheby(rt_hier* h, const T* u, const T* f, T* unew, T* d, const double* coef, int kstep) {
    if (use_march<T>(h, 3)) return fine_march<T, 3>(h, u, f, unew, 0.0, d, coef, kstep);
    const char* nm = sizeof(T) == 8 ? "fine_cheby_f64" : "fine_cheby_f32";
    return h->has_support ? launch_tile<T, true, 3>(h, u, f, unew, 0.0, nm, d, coef, kstep)
                          : launch_tile<T, false, 3>(h, u, f, unew, 0.0, nm, d, coef, kstep);
}

template int fine_cheby<double>(rt_hier*, const double*, const double*, double*, double*, const double*, int);
template int fine_cheby<float>(rt_hier*, const float*, const float*, float*, float*, const double*, int);
template int fine_residual<double>(rt_hier*, const double*, const double*, double*);
template int fine_residual<float>(rt_hier*, const float*, const float*, float*);
template int fine_applyK<double>(rt_hier*, const double*, double*);
template int fine_applyK<float>(rt_hier*, const float*, float*);
template int fine_jacobi<double>(rt_hier*, const double*, const double*, double*, double);
template int fine_jacobi<float>(rt_hier*, const float*, const float*, float*, double);

}  // namespace rtk
