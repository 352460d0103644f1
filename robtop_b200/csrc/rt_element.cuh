// rt_element.cuh — the hex8 element operator in the Hadamard basis of its vertices.
//
// With T = H (x) I3 (H the 8x8 Sylvester-Hadamard over the vertex bits x, y, z),
// KE = T Kt T^T / 64 and the 24x24 Kt has 45 non-zeros whose positions do not
// depend on E, nu or h.  Applying rho^p KE to an element costs two 3-stage
// butterflies per displacement component, 45 FMAs and 21 scalings.
#pragma once
#include "rt_internal.h"

namespace rte {

// sparsity pattern of Kt (rows/cols index 3*mode + comp)
__device__ constexpr int KT_R[45] = {3, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 11, 12, 12,
                                     13, 13, 14, 14, 14, 15, 15, 16, 16, 16, 17, 17, 18, 18, 18, 19, 19, 20, 20, 21,
                                     22, 23};
__device__ constexpr int KT_C[45] = {3, 7, 14, 4, 6, 5, 12, 4, 6, 3, 7, 14, 8, 13, 9, 20, 10, 17, 11, 16, 18, 5, 12,
                                     8, 13, 3, 7, 14, 15, 19, 11, 16, 18, 10, 17, 11, 16, 18, 15, 19, 9, 20, 21, 22,
                                     23};

template <typename T>
struct KtVals {
    T v[45];
    T diag_a, diag_b;  // KE diagonal block of any vertex: a I + b (s s^T - I), s = vertex reflection signs
};

// 8-point Sylvester-Hadamard over the vertex bits (x, y, z) of one component
template <typename T>
__device__ __forceinline__ void hadamard8(T* a, int c) {
#pragma unroll
    for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
        for (int i = 0; i < 8; i++)
            if (!(i & bit)) {
                const T p = a[3 * i + c], q = a[3 * (i | bit) + c];
                a[3 * i + c] = p + q;
                a[3 * (i | bit) + c] = p - q;
            }
}

// a <- w * KE * a, a indexed 3*vertex + comp, vertex = bx + 2 by + 4 bz
template <typename T>
__device__ __forceinline__ void element_apply(T* a, const KtVals<T>& kt, T w) {
#pragma unroll
    for (int c = 0; c < 3; c++) hadamard8(a, c);
    T z[24];
#pragma unroll
    for (int i = 0; i < 24; i++) z[i] = T(0);
#pragma unroll
    for (int k = 0; k < 45; k++) z[KT_R[k]] += kt.v[k] * a[KT_C[k]];
#pragma unroll
    for (int i = 0; i < 24; i++) a[i] = w * z[i];
#pragma unroll
    for (int c = 0; c < 3; c++) hadamard8(a, c);
}

template <typename T>
KtVals<T> make_kt(const rt_hier* h) {
    static const int R[45] = {3, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 11, 12, 12,
                              13, 13, 14, 14, 14, 15, 15, 16, 16, 16, 17, 17, 18, 18, 18, 19, 19, 20, 20, 21,
                              22, 23};
    static const int Cc[45] = {3, 7, 14, 4, 6, 5, 12, 4, 6, 3, 7, 14, 8, 13, 9, 20, 10, 17, 11, 16, 18, 5, 12,
                               8, 13, 3, 7, 14, 15, 19, 11, 16, 18, 10, 17, 11, 16, 18, 15, 19, 9, 20, 21, 22,
                               23};
    KtVals<T> k;
    for (int q = 0; q < 45; q++) {
        const int m = R[q] / 3, c = R[q] % 3, n = Cc[q] / 3, d = Cc[q] % 3;
        double s = 0;
        for (int i = 0; i < 8; i++)
            for (int j = 0; j < 8; j++) {
                const double hmi = (__builtin_popcount(m & i) & 1) ? -1.0 : 1.0;
                const double hnj = (__builtin_popcount(n & j) & 1) ? -1.0 : 1.0;
                s += hmi * h->KE[(3 * i + c) * 24 + 3 * j + d] * hnj;
            }
        k.v[q] = (T)(s / 64.0);
    }
    k.diag_a = (T)h->KE[0];
    k.diag_b = (T)h->KE[1];
    return k;
}

}  // namespace rte

namespace rte {

// two elements at once in packed FP32 pairs (the .x / .y lanes are independent elements):
// the same butterflies and 45 Kt products as element_apply<float>, as FADD2 / FFMA2 / FMUL2
__device__ __forceinline__ float2 sub2(float2 p, float2 q) { return __ffma2_rn(q, make_float2(-1.f, -1.f), p); }

__device__ __forceinline__ void hadamard8x2(float2* a, int c) {
#pragma unroll
    for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
        for (int i = 0; i < 8; i++)
            if (!(i & bit)) {
                const float2 p = a[3 * i + c], q = a[3 * (i | bit) + c];
                a[3 * i + c] = __fadd2_rn(p, q);
                a[3 * (i | bit) + c] = sub2(p, q);
            }
}

// a <- w * KE * a for two elements (w.x, w.y their weights)
__device__ __forceinline__ void element_apply2(float2* a, const KtVals<float>& kt, float2 w) {
#pragma unroll
    for (int c = 0; c < 3; c++) hadamard8x2(a, c);
    float2 z[24];
    // Kt's rows are sorted: the first product of a row initialises it
#pragma unroll
    for (int k = 0; k < 45; k++) {
        const float2 kv = make_float2(kt.v[k], kt.v[k]);
        if (k == 0 || KT_R[k - 1] != KT_R[k]) z[KT_R[k]] = __fmul2_rn(kv, a[KT_C[k]]);
        else z[KT_R[k]] = __ffma2_rn(kv, a[KT_C[k]], z[KT_R[k]]);
    }
    // rows 0..2 (the rigid translations) of Kt are empty
#pragma unroll
    for (int i = 0; i < 3; i++) a[i] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 3; i < 24; i++) a[i] = __fmul2_rn(w, z[i]);
#pragma unroll
    for (int c = 0; c < 3; c++) hadamard8x2(a, c);
}

}  // namespace rte
