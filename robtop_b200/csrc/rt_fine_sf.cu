// rt_fine_sf.cu — finest-level operator by sum factorisation over the element grid.
//
// Same operators as rt_fine_tile.cu (residual, applyK, damped block Jacobi, Chebyshev step;
// grid/Grid.cu:1450-1557, 2439-2517), with the Hadamard transform of the element vectors
// factorised along the grid instead of being evaluated per element:
//
//  * the 8-vertex Hadamard transform H = Hx (x) Hy (x) Hz of an element's displacements is
//    done one axis at a time, and each partial result is shared by every element that needs
//    it: the x stage (sum and difference along an x edge) serves the 4 elements around that
//    edge, the y stage (over an xy face) the 2 elements on either side of the face, and only
//    the z stage is per element.  The inverse transform of the element outputs is factorised
//    the same way, with the contributions of neighbouring elements added between its stages
//    (a face sums the outputs of the element below and above it before its y stage, an x edge
//    those of the two faces next to it before its x stage), so the scatter to the nodes costs
//    no extra adds.  Per element this is 36 + 21 butterflies and adds forward and back instead
//    of 144, next to the 45 products with Kt (KE = T Kt T^T / 64, see rt_element.cuh).
//  * A CTA is TY + 2 warps.  Warp w holds node row Y0 - 1 + w and evaluates element row
//    Y0 - 1 + w; lane l holds node column X0 - 1 + l and the x edge to column X0 + l.  The x
//    stages of neighbouring columns meet through warp shuffles, the y stages of neighbouring
//    rows through shared memory (the forward x-edge data go down one warp, the inverse face
//    data and the weight sums of the diagonal blocks go up one warp).  Lanes 1..30 of warps
//    1..TY produce nodes, so a CTA writes a 30 x TY node tile; warp TY + 1 only supplies the
//    x-edge data of the row above the tile.
//  * The CTA marches up through a z chunk.  Iteration t evaluates element layer t and
//    finishes node layer t - 1 (whose inverse y data crossed the barrier of iteration t), so
//    there is one barrier per layer, with the shared buffers alternating between iterations.
//  * The diagonal 3x3 block of a node, sum_e w_e KE_vv = a sum_e w_e I + b (sum_e w_e s s^T - I),
//    needs four signed sums of the 8 surrounding weights; they are factorised the same way
//    (x pairs by shuffle, y pairs through shared memory, z pairs in registers).
//  * Fixed (support) nodes enter the element products as zero, which is the reference's WS rule
//    (couplings to fixed nodes dropped); their output rows follow the tile kernel's rules.
#include <cuda_runtime.h>

#include "rt_element.cuh"
#include "rt_internal.h"

namespace {

constexpr int SF_TX = 30;  // node columns a CTA produces (lanes 1..30)

template <typename T, int TY>
struct SfSmem {
    T e[2][6][TY + 2][32];       // forward x-edge data of each warp's node row: (sum, diff) x 3 components
    T q[2][6][TY + 2][32];       // inverse y-stage output of element row j toward node row j + 1
    T wq[2][2][TY + 2][32];      // x-pair sum and difference of the element weights of row j
};

template <typename T, int TY>
constexpr int sf_min_blocks() {
    return sizeof(T) == 8 ? (TY <= 4 ? 2 : 1) : (TY <= 4 ? 3 : (TY <= 8 ? 2 : 1));
}

template <typename T>
__device__ __forceinline__ T sf_rcp(T x) {
    if constexpr (sizeof(T) == 4) return __frcp_rn(x);
    else return T(1) / x;
}

// g = w * Kt h (rows 0..2 of Kt, the rigid translations, are empty; the rows are sorted, so the
// first product of a row initialises it)
template <typename T>
__device__ __forceinline__ void sf_kt(const rte::KtVals<T>& kt, const T (&h)[24], T w, T (&g)[24]) {
#pragma unroll
    for (int k = 0; k < 45; k++) {
        if (k == 0 || rte::KT_R[k - 1] != rte::KT_R[k]) g[rte::KT_R[k]] = kt.v[k] * h[rte::KT_C[k]];
        else g[rte::KT_R[k]] += kt.v[k] * h[rte::KT_C[k]];
    }
#pragma unroll
    for (int i = 0; i < 3; i++) g[i] = T(0);
#pragma unroll
    for (int i = 3; i < 24; i++) g[i] *= w;
}

// MODE 0: r = f - K u (fixed rows: r = f)     MODE 1: out = K u (fixed rows: u)
// MODE 2: unew = u + omega D^-1 (f - K u)     MODE 3: Chebyshev step kstep: d = a_k d + b_k D^-1 (f - K u), unew = u + d
// (fixed nodes in MODE 2/3: unew = f / n_e, d = 0; inactive nodes: 0)
template <typename T, bool WS, int MODE, int TY>
__global__ void __launch_bounds__((TY + 2) * 32, sf_min_blocks<T, TY>())
    k_fine_sf(int nx, int ny, int nz, int zchunk, const uint8_t* __restrict__ vact, const float* __restrict__ wgt,
              const uint8_t* __restrict__ vfix, const rte::KtVals<T> kt, const T* __restrict__ u,
              const T* __restrict__ f, T* __restrict__ out, T omega, T* __restrict__ dvec,
              const double* __restrict__ coef, int kstep) {
    extern __shared__ __align__(16) unsigned char smraw[];
    SfSmem<T, TY>& S = *reinterpret_cast<SfSmem<T, TY>*>(smraw);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T cheb_a = T(0), cheb_b = T(0);
    if (MODE == 3) {
        const double ca = coef[2 * kstep], cb = coef[2 * kstep + 1];
        cheb_a = (T)ca;
        cheb_b = (T)cb;
    }
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    const long nv = (long)vx * vy * vz;
    const long plane = (long)vx * vy;
    const long eplane = (long)nx * ny;
    const int X0 = blockIdx.x * SF_TX, Y0 = blockIdx.y * TY;
    const int Z0 = blockIdx.z * zchunk, Z1 = min(Z0 + zchunk, vz);
    const int ci = X0 - 1 + lane;  // node column of the lane; element column of its x edge
    const int rj = Y0 - 1 + w;     // node row of the warp; element row it evaluates
    const bool node_ok = ci >= 0 && ci < vx && rj >= 0 && rj < vy;
    const bool elem_ok = ci >= 0 && ci < nx && rj >= 0 && rj < ny;
    const bool elem_warp = w <= TY;  // warp TY + 1 only supplies x-edge data
    const bool out_node = lane >= 1 && lane <= SF_TX && w >= 1 && w <= TY && node_ok;
    const long nxy = node_ok ? ci + (long)vx * rj : 0;
    const long exy = elem_ok ? ci + (long)nx * rj : 0;

    // displacement of the lane's node at layer L as the elements see it (fixed nodes: 0)
    auto load_u = [&](int L, T (&el)[3]) {
        el[0] = el[1] = el[2] = T(0);
        if (node_ok && L >= 0 && L < vz) {
            const long v = nxy + plane * L;
            if (!(WS && vfix[v])) {
                el[0] = u[v];
                el[1] = u[nv + v];
                el[2] = u[2 * nv + v];
            }
        }
    };
    auto load_w = [&](int t) -> float { return (elem_ok && t >= 0 && t < nz) ? wgt[exy + eplane * t] : 0.f; };
    // x stage: (u_i + u_{i+1}, u_i - u_{i+1}) per component; lane 31's edge is never used
    auto x_stage = [&](const T (&el)[3], T (&E)[6]) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T nb = __shfl_down_sync(0xffffffffu, el[c], 1);
            E[c] = el[c] + nb;
            E[3 + c] = el[c] - nb;
        }
    };
    // y stage over the face between node rows j (own) and j + 1: index 3 (mx + 2 my) + c
    auto y_stage = [&](const T (&E)[6], const T (&En)[6], T (&F)[12]) {
#pragma unroll
        for (int q = 0; q < 6; q++) {
            F[q] = E[q] + En[q];
            F[6 + q] = E[q] - En[q];
        }
    };

    // ---- prologue: forward face data of node layer Z0 - 1
    T Flo[12];
    {
        T el[3], E[6], En[6];
        load_u(Z0 - 1, el);
        x_stage(el, E);
#pragma unroll
        for (int q = 0; q < 6; q++) S.e[0][q][w][lane] = E[q];
        __syncthreads();
        if (elem_warp) {
#pragma unroll
            for (int q = 0; q < 6; q++) En[q] = S.e[0][q][w + 1][lane];
            y_stage(E, En, Flo);
        } else {
#pragma unroll
            for (int q = 0; q < 12; q++) Flo[q] = T(0);
        }
    }
    T Gtop[12];  // inverse z output of element layer t - 1 toward node layer t
#pragma unroll
    for (int q = 0; q < 12; q++) Gtop[q] = T(0);
    T Y0p[6], Y1p[6];  // inverse y output of the last face: own row, row above
#pragma unroll
    for (int q = 0; q < 6; q++) Y0p[q] = Y1p[q] = T(0);
    T Qm1[4] = {T(0), T(0), T(0), T(0)}, Qm2[4] = {T(0), T(0), T(0), T(0)};  // (A, Bxy, Ay, Bx) of layers t-1, t-2
    T un[3];  // element-side displacement of node layer t + 1
    load_u(Z0, un);
    float wt = load_w(Z0 - 1);  // weight of element layer t

    for (int t = Z0 - 1; t <= Z1; t++) {
        const int buf = (t - Z0 + 2) & 1;
        const bool body = t < Z1;  // t == Z1: only node layer Z1 - 1 is finished
        T E[6];
        T wa = T(0), wb = T(0);
        if (body) {
            x_stage(un, E);
            const float wl = __shfl_up_sync(0xffffffffu, wt, 1);
            wa = T(wt) + T(wl);  // element i (x sign +1 for node i) and element i - 1 (sign -1)
            wb = T(wt) - T(wl);
#pragma unroll
            for (int q = 0; q < 6; q++) S.e[buf][q][w][lane] = E[q];
            S.wq[buf][0][w][lane] = wa;
            S.wq[buf][1][w][lane] = wb;
        }
#pragma unroll
        for (int q = 0; q < 6; q++) S.q[buf][q][w][lane] = Y1p[q];
        // loads in flight across the barrier and the element phase: node layer t + 2 and the weight
        // of element layer t + 1 for the next iteration, the node-phase inputs of layer t - 1
        T un2[3] = {T(0), T(0), T(0)};
        float wt2 = 0.f;
        if (body) {
            if (t + 2 <= Z1) load_u(t + 2, un2);
            wt2 = load_w(t + 1);
        }
        const bool fin = out_node && t - 1 >= Z0;  // this lane finishes node layer t - 1
        T pf[3] = {T(0), T(0), T(0)}, pd[3] = {T(0), T(0), T(0)}, pu[3] = {T(0), T(0), T(0)};
        bool pact = false, pfix = false;
        if (fin) {
            const long v = nxy + plane * (t - 1);
            pact = vact[v] != 0;
            pfix = WS && pact && vfix[v];
            if (pact) {
                if (MODE != 1)
#pragma unroll
                    for (int c = 0; c < 3; c++) pf[c] = f[c * nv + v];
                if (MODE >= 1)
#pragma unroll
                    for (int c = 0; c < 3; c++) pu[c] = u[c * nv + v];
                if (MODE == 3 && kstep > 0)
#pragma unroll
                    for (int c = 0; c < 3; c++) pd[c] = dvec[c * nv + v];
            }
        }
        __syncthreads();
        // ---- node phase, first part: the x-edge data of node layer t - 1 (own element row's face
        // t - 1 output plus the row below's), and the weight sums of element layer t
        T X[6];
        T Q[4] = {T(0), T(0), T(0), T(0)};
        const bool node_warp = w >= 1 && w <= TY;
        if (node_warp) {
#pragma unroll
            for (int q = 0; q < 6; q++) X[q] = Y0p[q] + S.q[buf][q][w - 1][lane];
            if (body) {
                const T wa_b = S.wq[buf][0][w - 1][lane], wb_b = S.wq[buf][1][w - 1][lane];
                // element rows j (y sign +1 for node row j) and j - 1 (sign -1)
                Q[0] = wa + wa_b;  // sum w
                Q[1] = wb - wb_b;  // sum w sx sy
                Q[2] = wa - wa_b;  // sum w sy
                Q[3] = wb + wb_b;  // sum w sx
            }
        }
        // ---- element phase: element layer t (node layers t and t + 1)
        if (body && elem_warp) {
            T En[6], Fhi[12];
#pragma unroll
            for (int q = 0; q < 6; q++) En[q] = S.e[buf][q][w + 1][lane];
            y_stage(E, En, Fhi);
            T h[24], g[24];
#pragma unroll
            for (int q = 0; q < 12; q++) {
                h[q] = Flo[q] + Fhi[q];       // z mode 0
                h[12 + q] = Flo[q] - Fhi[q];  // z mode 1
            }
            sf_kt(kt, h, T(wt), g);
            T Ft[12];
#pragma unroll
            for (int q = 0; q < 12; q++) {
                const T g0 = g[q], g1 = g[12 + q];
                Ft[q] = Gtop[q] + (g0 + g1);  // face t: element t - 1 from above, element t from below
                Gtop[q] = g0 - g1;            // toward face t + 1
                Flo[q] = Fhi[q];
            }
#pragma unroll
            for (int q = 0; q < 6; q++) {
                Y0p[q] = Ft[q] + Ft[6 + q];
                Y1p[q] = Ft[q] - Ft[6 + q];
            }
        }
        // ---- node phase, second part: inverse x stage and the update of node layer t - 1
        if (node_warp) {
            T Dm[3];
#pragma unroll
            for (int c = 0; c < 3; c++) Dm[c] = __shfl_up_sync(0xffffffffu, X[c] - X[3 + c], 1);
            if (fin) {
                const long v = nxy + plane * (t - 1);
                T acc[3];
#pragma unroll
                for (int c = 0; c < 3; c++) acc[c] = X[c] + X[3 + c] + Dm[c];
                T o[3] = {T(0), T(0), T(0)}, dn[3] = {T(0), T(0), T(0)};
                if (pact) {
                    if (MODE == 0) {
#pragma unroll
                        for (int c = 0; c < 3; c++) o[c] = pfix ? pf[c] : pf[c] - acc[c];
                    } else if (MODE == 1) {
#pragma unroll
                        for (int c = 0; c < 3; c++) o[c] = pfix ? pu[c] : acc[c];
                    } else if (pfix) {
                        // f / n_e over the elements around the node with non-zero weight
                        const int z = t - 1;
                        int ne = 0;
#pragma unroll
                        for (int i8 = 0; i8 < 8; i8++) {
                            const int ex = ci - 1 + (i8 & 1), ey = rj - 1 + ((i8 >> 1) & 1), ez = z - 1 + (i8 >> 2);
                            if (ex >= 0 && ey >= 0 && ez >= 0 && ex < nx && ey < ny && ez < nz &&
                                wgt[ex + (long)nx * ey + eplane * ez] != 0.f)
                                ne++;
                        }
#pragma unroll
                        for (int c = 0; c < 3; c++) o[c] = pf[c] / T(ne > 0 ? ne : 1);
                    } else {
                        // node layer t - 1 sits between element layers t - 2 (z sign -1) and t - 1 (+1)
                        const T sw = Qm1[0] + Qm2[0], sxy = Qm1[1] + Qm2[1];
                        const T sxz = Qm1[3] - Qm2[3], syz = Qm1[2] - Qm2[2];
                        const T A = kt.diag_a * sw, bxy = kt.diag_b * sxy, bxz = kt.diag_b * sxz,
                                byz = kt.diag_b * syz;
                        const T c00 = A * A - byz * byz, c01 = -(bxy * A - byz * bxz), c02 = bxy * byz - A * bxz;
                        const T c11 = A * A - bxz * bxz, c12 = -(A * byz - bxy * bxz), c22 = A * A - bxy * bxy;
                        const T id = sf_rcp(A * c00 + bxy * c01 + bxz * c02);
                        T rr[3];
#pragma unroll
                        for (int c = 0; c < 3; c++) rr[c] = pf[c] - acc[c];
                        T zz[3];
                        zz[0] = id * (c00 * rr[0] + c01 * rr[1] + c02 * rr[2]);
                        zz[1] = id * (c01 * rr[0] + c11 * rr[1] + c12 * rr[2]);
                        zz[2] = id * (c02 * rr[0] + c12 * rr[1] + c22 * rr[2]);
                        if (MODE == 2) {
#pragma unroll
                            for (int c = 0; c < 3; c++) o[c] = pu[c] + omega * zz[c];
                        } else {
#pragma unroll
                            for (int c = 0; c < 3; c++) {
                                dn[c] = (kstep == 0 ? T(0) : cheb_a * pd[c]) + cheb_b * zz[c];
                                o[c] = pu[c] + dn[c];
                            }
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; c++) out[c * nv + v] = o[c];
                if (MODE == 3)
#pragma unroll
                    for (int c = 0; c < 3; c++) dvec[c * nv + v] = dn[c];
            }
        }
        if (!body) break;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            Qm2[q] = Qm1[q];
            Qm1[q] = Q[q];
        }
#pragma unroll
        for (int c = 0; c < 3; c++) un[c] = un2[c];
        wt = wt2;
    }
}

template <typename T, bool WS, int MODE, int TY>
int launch_sf_ty(rt_hier* h, const T* u, const T* f, T* out, double omega, const char* name, T* dvec,
                 const double* coef, int kstep) {
    rt_level& L = h->L[0];
    const int zc = h->tune[sizeof(T) == 8 ? 1 : 0][MODE].zchunk;
    dim3 grid((L.vx + SF_TX - 1) / SF_TX, (L.vy + TY - 1) / TY, (L.vz + zc - 1) / zc);
    const rte::KtVals<T> kt = rte::make_kt<T>(h);
    return rt_launch(h->ctx, name, [&] {
        k_fine_sf<T, WS, MODE, TY><<<grid, (TY + 2) * 32, sizeof(SfSmem<T, TY>), h->ctx->stream>>>(
            L.nx, L.ny, L.nz, zc, L.vact, h->w, h->vfix, kt, u, f, out, (T)omega, dvec, coef, kstep);
    });
}

template <typename T, bool WS, int MODE, int TY>
cudaError_t sf_attr() {
    return cudaFuncSetAttribute(k_fine_sf<T, WS, MODE, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(SfSmem<T, TY>));
}

template <typename T, int TY>
cudaError_t sf_attrs() {
    cudaError_t r[8] = {sf_attr<T, false, 0, TY>(), sf_attr<T, false, 1, TY>(), sf_attr<T, false, 2, TY>(),
                        sf_attr<T, false, 3, TY>(), sf_attr<T, true, 0, TY>(),  sf_attr<T, true, 1, TY>(),
                        sf_attr<T, true, 2, TY>(),  sf_attr<T, true, 3, TY>()};
    for (auto x : r)
        if (x != cudaSuccess) return x;
    return cudaSuccess;
}

}  // namespace

namespace rtk {

int init_sf_kernels(rt_ctx* c) {
    cudaError_t es[6] = {sf_attrs<double, 4>(), sf_attrs<double, 8>(), sf_attrs<double, 16>(),
                         sf_attrs<float, 4>(),  sf_attrs<float, 8>(),  sf_attrs<float, 16>()};
    for (cudaError_t e : es)
        if (e != cudaSuccess) return rt_fail(c, RT_ECUDA, "sum-factorised kernel attributes: %s", cudaGetErrorString(e));
    return RT_OK;
}

// variant 5 of the finest-level kernels; ty = node rows of the CTA's tile (4, 8 or 16)
template <typename T, bool WS, int MODE>
int launch_sf(rt_hier* h, const T* u, const T* f, T* out, double omega, const char* name, T* dvec, const double* coef,
              int kstep) {
    switch (h->tune[sizeof(T) == 8 ? 1 : 0][MODE].ty) {
        case 4: return launch_sf_ty<T, WS, MODE, 4>(h, u, f, out, omega, name, dvec, coef, kstep);
        case 16: return launch_sf_ty<T, WS, MODE, 16>(h, u, f, out, omega, name, dvec, coef, kstep);
        default: return launch_sf_ty<T, WS, MODE, 8>(h, u, f, out, omega, name, dvec, coef, kstep);
    }
}

#define RT_SF_INST(T, WS, MODE)                                                                                   \
    template int launch_sf<T, WS, MODE>(rt_hier*, const T*, const T*, T*, double, const char*, T*, const double*, \
                                        int);
RT_SF_INST(float, false, 0)
RT_SF_INST(float, false, 1)
RT_SF_INST(float, false, 2)
RT_SF_INST(float, false, 3)
RT_SF_INST(float, true, 0)
RT_SF_INST(float, true, 1)
RT_SF_INST(float, true, 2)
RT_SF_INST(float, true, 3)
RT_SF_INST(double, false, 0)
RT_SF_INST(double, false, 1)
RT_SF_INST(double, false, 2)
RT_SF_INST(double, false, 3)
RT_SF_INST(double, true, 0)
RT_SF_INST(double, true, 1)
RT_SF_INST(double, true, 2)
RT_SF_INST(double, true, 3)
#undef RT_SF_INST

}  // namespace rtk
