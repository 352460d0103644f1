// rt_unet.cu — C ABI of the learned preconditioner: its building-block convolution and
// (below) the U-Net object.  No reference counterpart.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "rt_internal.h"
#include "rt_unet.h"

extern "C" int rt_unet_conv3(rt_ctx* c, const void* in, int in_stride, int cin, const void* w, const float* bias,
                             int cout, void* out, int out_stride, int out_f32, int relu, int accumulate, int X, int Y,
                             int Z) {
    if (!c || !in || !w || !out || X <= 0 || Y <= 0 || Z <= 0) return RT_EINVAL;
    if (accumulate && !out_f32) return rt_fail(c, RT_EINVAL, "conv3: accumulate needs a float output");
    RT_CUDA(c, cudaSetDevice(c->device));
    static bool inited[64] = {false};
    if (!inited[c->device & 63]) {
        RT_CHECK(rtu::conv3_init(c));
        inited[c->device & 63] = true;
    }
    int* err = nullptr;
    RT_CUDA(c, cudaMallocAsync(&err, sizeof(int), c->stream));
    RT_CUDA(c, cudaMemsetAsync(err, 0, sizeof(int), c->stream));
    rtu::ConvArgs a;
    a.in = static_cast<const __nv_bfloat16*>(in);
    a.in_stride = in_stride;
    a.cin = cin;
    a.w = static_cast<const __nv_bfloat16*>(w);
    a.bias = bias;
    a.cout = cout;
    a.out = out;
    a.out_stride = out_stride;
    a.out_f32 = out_f32;
    a.relu = relu;
    a.accumulate = accumulate;
    a.X = X;
    a.Y = Y;
    a.Z = Z;
    a.err = err;
    int s = rtu::conv3(c, a);
    int herr = 0;
    cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(err, c->stream);
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    if (s != RT_OK) return s;
    if (e != cudaSuccess) return rt_fail(c, RT_ECUDA, "conv3: %s", cudaGetErrorString(e));
    if (herr) return rt_fail(c, RT_ETIMEOUT, "conv3: tensor-core wait timed out");
    return RT_OK;
}

extern "C" int rt_unet_set_conv_variant(int variant) {
    if (variant < 0 || variant > 1) return RT_EINVAL;
    rtu::conv3_set_variant(variant);
    return RT_OK;
}

// ---------------------------------------------------------------------------
// the U-Net: 4 levels, 16/32/48/64 channels, two 3x3x3 convolutions (+ReLU) per level and
// side, 2x2x2 average pooling, nearest upsampling with skip concatenation, 1x1x1 head
// to 3 channels.  Input: 16 channels (log density, 3 scaled residual components, the
// support flag, 3 scaled components of the V-cycle's output for that residual, zeros).
// ---------------------------------------------------------------------------
namespace {

struct Layer {
    int cin, cout;
    long woff, boff;  // offsets of [cout][27][cin] weights and [cout] bias in the FP32 parameters
    long w16off;      // offset in the bf16 weight copies
};

// the 14 convolutions in forward order (see unet_forward)
constexpr int N_LAYERS = 14;
constexpr int PLAN[N_LAYERS][2] = {{16, 16}, {16, 16}, {16, 32}, {32, 32}, {32, 48}, {48, 48}, {48, 64},
                                   {64, 64}, {112, 48}, {48, 48}, {80, 32}, {32, 32}, {48, 16}, {16, 16}};
constexpr int HEAD_C = 16;

template <typename T>
int ualloc(rt_ctx* c, T** p, size_t n) {
    if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
        cudaGetLastError();
        return rt_fail(c, RT_ENOMEM, "U-Net: cudaMalloc of %zu bytes failed", sizeof(T) * n);
    }
    return RT_OK;
}

}  // namespace

struct rt_unet {
    rt_ctx* ctx = nullptr;
    int X[4], Y[4], Z[4];
    long V[4];
    Layer L[N_LAYERS];
    long nparam = 0, nw16 = 0, head_w = 0, head_b = 0;
    float *P = nullptr, *G = nullptr, *M = nullptr, *Vv = nullptr;
    __nv_bfloat16 *W16 = nullptr, *W16t = nullptr;
    bool w16_dirty = true;
    int adam_t = 0;
    // activations (bf16, channels-last)
    __nv_bfloat16 *in0 = nullptr, *a0 = nullptr, *cat0 = nullptr, *p1 = nullptr, *a1 = nullptr, *cat1 = nullptr,
                  *p2 = nullptr, *a2 = nullptr, *cat2 = nullptr, *p3 = nullptr, *a3 = nullptr, *b3 = nullptr,
                  *d2a = nullptr, *d2 = nullptr, *d1a = nullptr, *d1 = nullptr, *d0a = nullptr, *d0 = nullptr;
    float* out = nullptr;  // [V0][3]
    // training buffers (allocated on the first backward)
    float *g_out = nullptr, *g_d0 = nullptr, *g_x = nullptr, *g_cat0 = nullptr, *g_cat1 = nullptr, *g_cat2 = nullptr,
          *g_y = nullptr, *g_p = nullptr;
    __nv_bfloat16* gpre = nullptr;
    double* dloss = nullptr;
    int* err = nullptr;
    double oscale = 0.0;  // network output unit: rms of the scaled training targets (0 until the first harvest)
    double* dscal = nullptr;  // [4] device scratch: target sum of squares, active count
};

static void unet_free(rt_unet* u) {
    if (!u) return;
    void* ptrs[] = {u->P, u->G, u->M, u->Vv, u->W16, u->W16t, u->in0, u->a0, u->cat0, u->p1, u->a1, u->cat1,
                    u->p2, u->a2, u->cat2, u->p3, u->a3, u->b3, u->d2a, u->d2, u->d1a, u->d1, u->d0a, u->d0,
                    u->out, u->g_out, u->g_d0, u->g_x, u->g_cat0, u->g_cat1, u->g_cat2, u->g_y, u->g_p, u->gpre,
                    u->dloss, u->err, u->dscal};
    for (void* p : ptrs) cudaFree(p);
    rt_ctx* c = u->ctx;
    delete u;
    rt_ctx_release(c);
}

static unsigned ew_blocks(rt_ctx* c, long n) {
    return (unsigned)std::min<long>((n + 255) / 256, (long)c->sm_count * 16);
}

static int unet_conv(rt_unet* u, int li, int lvl, const __nv_bfloat16* in, int in_stride, void* out, int out_stride,
                     int relu) {
    const Layer& l = u->L[li];
    rtu::ConvArgs a;
    a.in = in;
    a.in_stride = in_stride;
    a.cin = l.cin;
    a.w = u->W16 + l.w16off;
    a.bias = u->P + l.boff;
    a.cout = l.cout;
    a.out = out;
    a.out_stride = out_stride;
    a.relu = relu;
    a.X = u->X[lvl];
    a.Y = u->Y[lvl];
    a.Z = u->Z[lvl];
    a.err = u->err;
    return rtu::conv3(u->ctx, a);
}

static int unet_refresh_w16(rt_unet* u) {
    if (!u->w16_dirty) return RT_OK;
    rt_ctx* c = u->ctx;
    for (int i = 0; i < N_LAYERS; i++) {
        const Layer& l = u->L[i];
        RT_CHECK(rt_launch(c, "unet_weights_bf16", [&] {
            rtu::k_weights_bf16<<<ew_blocks(c, 27L * l.cin * l.cout), 256, 0, c->stream>>>(
                u->P + l.woff, l.cin, l.cout, u->W16 + l.w16off, u->W16t + l.w16off);
        }));
    }
    u->w16_dirty = false;
    return RT_OK;
}

static int unet_pool(rt_unet* u, int lvl_fine, const __nv_bfloat16* in, int in_stride, int C, __nv_bfloat16* out) {
    rt_ctx* c = u->ctx;
    const long n = u->V[lvl_fine + 1] * C;
    return rt_launch(c, "unet_pool", [&] {
        rtu::k_pool2<<<ew_blocks(c, n), 256, 0, c->stream>>>(in, in_stride, C, u->X[lvl_fine], u->Y[lvl_fine],
                                                             u->Z[lvl_fine], out, C);
    });
}

static int unet_up(rt_unet* u, int lvl_fine, const __nv_bfloat16* in, int C, __nv_bfloat16* out, int out_stride) {
    rt_ctx* c = u->ctx;
    const long n = u->V[lvl_fine] * C;
    return rt_launch(c, "unet_up", [&] {
        rtu::k_up2<<<ew_blocks(c, n), 256, 0, c->stream>>>(in, C, u->X[lvl_fine], u->Y[lvl_fine], u->Z[lvl_fine], out,
                                                           out_stride);
    });
}

// forward pass from u->in0 to u->out
static int unet_forward(rt_unet* u) {
    rt_ctx* c = u->ctx;
    RT_CHECK(unet_refresh_w16(u));
    RT_CHECK(unet_conv(u, 0, 0, u->in0, 16, u->a0, 16, 1));
    RT_CHECK(unet_conv(u, 1, 0, u->a0, 16, u->cat0 + 32, 48, 1));
    RT_CHECK(unet_pool(u, 0, u->cat0 + 32, 48, 16, u->p1));
    RT_CHECK(unet_conv(u, 2, 1, u->p1, 16, u->a1, 32, 1));
    RT_CHECK(unet_conv(u, 3, 1, u->a1, 32, u->cat1 + 48, 80, 1));
    RT_CHECK(unet_pool(u, 1, u->cat1 + 48, 80, 32, u->p2));
    RT_CHECK(unet_conv(u, 4, 2, u->p2, 32, u->a2, 48, 1));
    RT_CHECK(unet_conv(u, 5, 2, u->a2, 48, u->cat2 + 64, 112, 1));
    RT_CHECK(unet_pool(u, 2, u->cat2 + 64, 112, 48, u->p3));
    RT_CHECK(unet_conv(u, 6, 3, u->p3, 48, u->a3, 64, 1));
    RT_CHECK(unet_conv(u, 7, 3, u->a3, 64, u->b3, 64, 1));
    RT_CHECK(unet_up(u, 2, u->b3, 64, u->cat2, 112));
    RT_CHECK(unet_conv(u, 8, 2, u->cat2, 112, u->d2a, 48, 1));
    RT_CHECK(unet_conv(u, 9, 2, u->d2a, 48, u->d2, 48, 1));
    RT_CHECK(unet_up(u, 1, u->d2, 48, u->cat1, 80));
    RT_CHECK(unet_conv(u, 10, 1, u->cat1, 80, u->d1a, 32, 1));
    RT_CHECK(unet_conv(u, 11, 1, u->d1a, 32, u->d1, 32, 1));
    RT_CHECK(unet_up(u, 0, u->d1, 32, u->cat0, 48));
    RT_CHECK(unet_conv(u, 12, 0, u->cat0, 48, u->d0a, 16, 1));
    RT_CHECK(unet_conv(u, 13, 0, u->d0a, 16, u->d0, 16, 1));
    return rt_launch(c, "unet_head", [&] {
        rtu::k_head<<<ew_blocks(c, u->V[0]), 256, 0, c->stream>>>(u->d0, HEAD_C, u->V[0], u->P + u->head_w,
                                                                  u->P + u->head_b, u->out);
    });
}

static int unet_alloc_train(rt_unet* u) {
    if (u->g_out) return RT_OK;
    rt_ctx* c = u->ctx;
    const long V0 = u->V[0], V1 = u->V[1];
    RT_CHECK(ualloc(c, &u->g_out, 3 * V0));
    RT_CHECK(ualloc(c, &u->g_d0, 16 * V0));
    RT_CHECK(ualloc(c, &u->g_x, 64 * std::max(V0 / 4 + 1, V1)));  // largest single-layer gradient below level 0
    RT_CHECK(ualloc(c, &u->g_cat0, 48 * V0));
    RT_CHECK(ualloc(c, &u->g_cat1, 80 * V1));
    RT_CHECK(ualloc(c, &u->g_cat2, 112 * u->V[2]));
    RT_CHECK(ualloc(c, &u->g_y, 16 * V0 > 64 * V1 ? 16 * V0 : 64 * V1));
    RT_CHECK(ualloc(c, &u->g_p, 48 * V1));
    RT_CHECK(ualloc(c, &u->gpre, 112 * V0));
    RT_CHECK(ualloc(c, &u->dloss, 1));
    return RT_OK;
}

// backward of one convolution: gradient g (FP32, stride gs) of its ReLU output y -> dW, dB and,
// when gin is given, the FP32 input gradient [V][cin] (written, not accumulated)
static int unet_conv_bwd(rt_unet* u, int li, int lvl, const __nv_bfloat16* in, int in_stride,
                         const __nv_bfloat16* y, int y_stride, const float* g, int gs, float* gin, int relu = 1) {
    rt_ctx* c = u->ctx;
    const Layer& l = u->L[li];
    const long V = u->V[lvl];
    RT_CHECK(rt_launch(c, "unet_relu_bwd", [&] {
        rtu::k_relu_bwd<<<ew_blocks(c, V * l.cout), 256, 0, c->stream>>>(g, gs, y, y_stride, l.cout, V, relu, u->gpre);
    }));
    RT_CHECK(rt_launch(c, "unet_bias_grad", [&] {
        rtu::k_bias_grad<<<(unsigned)std::min<long>((V + 63) / 64, 1024), 256, 0, c->stream>>>(u->gpre, l.cout, V,
                                                                                               u->G + l.boff);
    }));
    const long nw = 27L * l.cin * l.cout;
    const long chunk = 4096;
    const dim3 gdw((unsigned)((nw + 255) / 256), (unsigned)((V + chunk - 1) / chunk));
    RT_CHECK(rt_launch(c, "unet_conv3_dw", [&] {
        rtu::k_conv3_dw<<<gdw, 256, 0, c->stream>>>(in, in_stride, l.cin, u->gpre, l.cout, u->X[lvl], u->Y[lvl],
                                                    u->Z[lvl], chunk, u->G + l.woff);
    }));
    if (!gin) return RT_OK;
    rtu::ConvArgs a;
    a.in = u->gpre;
    a.in_stride = l.cout;
    a.cin = l.cout;
    a.w = u->W16t + l.w16off;
    a.cout = l.cin;
    a.out = gin;
    a.out_stride = l.cin;
    a.out_f32 = 1;
    a.X = u->X[lvl];
    a.Y = u->Y[lvl];
    a.Z = u->Z[lvl];
    a.err = u->err;
    return rtu::conv3(c, a);
}

// loss and gradients for target tgt [V0][3] (u->out from the forward pass); G accumulates
static int unet_backward(rt_unet* u, const float* tgt) {
    rt_ctx* c = u->ctx;
    RT_CHECK(unet_alloc_train(u));
    const long V0 = u->V[0], V1 = u->V[1], V2 = u->V[2], V3 = u->V[3];
    RT_CHECK(rt_launch(c, "unet_mse", [&] {
        rtu::k_mse<<<ew_blocks(c, 3 * V0), 256, 0, c->stream>>>(u->out, tgt, 3 * V0, u->g_out, u->dloss);
    }));
    RT_CHECK(rt_launch(c, "unet_head_bwd", [&] {
        rtu::k_head_bwd<<<(unsigned)std::min<long>((V0 + 255) / 256, 512), 256, 0, c->stream>>>(
            u->d0, HEAD_C, V0, u->P + u->head_w, u->g_out, u->g_d0, u->G + u->head_w, u->G + u->head_b);
    }));
    // level 0 decoder
    RT_CHECK(unet_conv_bwd(u, 13, 0, u->d0a, 16, u->d0, 16, u->g_d0, 16, u->g_y));
    RT_CHECK(unet_conv_bwd(u, 12, 0, u->cat0, 48, u->d0a, 16, u->g_y, 16, u->g_cat0));
    RT_CHECK(rt_launch(c, "unet_up_bwd", [&] {
        rtu::k_up2_bwd<<<ew_blocks(c, V1 * 32), 256, 0, c->stream>>>(u->g_cat0, 48, 32, u->X[0], u->Y[0], u->Z[0],
                                                                      u->g_x);
    }));
    // level 1 decoder (g_x = gradient of d1)
    RT_CHECK(unet_conv_bwd(u, 11, 1, u->d1a, 32, u->d1, 32, u->g_x, 32, u->g_y));
    RT_CHECK(unet_conv_bwd(u, 10, 1, u->cat1, 80, u->d1a, 32, u->g_y, 32, u->g_cat1));
    RT_CHECK(rt_launch(c, "unet_up_bwd", [&] {
        rtu::k_up2_bwd<<<ew_blocks(c, V2 * 48), 256, 0, c->stream>>>(u->g_cat1, 80, 48, u->X[1], u->Y[1], u->Z[1],
                                                                      u->g_x);
    }));
    // level 2 decoder (g_x = gradient of d2)
    RT_CHECK(unet_conv_bwd(u, 9, 2, u->d2a, 48, u->d2, 48, u->g_x, 48, u->g_y));
    RT_CHECK(unet_conv_bwd(u, 8, 2, u->cat2, 112, u->d2a, 48, u->g_y, 48, u->g_cat2));
    RT_CHECK(rt_launch(c, "unet_up_bwd", [&] {
        rtu::k_up2_bwd<<<ew_blocks(c, V3 * 64), 256, 0, c->stream>>>(u->g_cat2, 112, 64, u->X[2], u->Y[2], u->Z[2],
                                                                      u->g_x);
    }));
    // bottleneck (g_x = gradient of b3)
    RT_CHECK(unet_conv_bwd(u, 7, 3, u->a3, 64, u->b3, 64, u->g_x, 64, u->g_y));
    RT_CHECK(unet_conv_bwd(u, 6, 3, u->p3, 48, u->a3, 64, u->g_y, 64, u->g_p));
    RT_CHECK(rt_launch(c, "unet_pool_bwd", [&] {
        rtu::k_pool2_bwd<<<ew_blocks(c, V2 * 48), 256, 0, c->stream>>>(u->g_p, 48, u->X[2], u->Y[2], u->Z[2],
                                                                        u->g_cat2 + 64, 112);
    }));
    // level 2 encoder: skip gradient in g_cat2[:, 64:112]
    RT_CHECK(unet_conv_bwd(u, 5, 2, u->a2, 48, u->cat2 + 64, 112, u->g_cat2 + 64, 112, u->g_y));
    RT_CHECK(unet_conv_bwd(u, 4, 2, u->p2, 32, u->a2, 48, u->g_y, 48, u->g_p));
    RT_CHECK(rt_launch(c, "unet_pool_bwd", [&] {
        rtu::k_pool2_bwd<<<ew_blocks(c, V1 * 32), 256, 0, c->stream>>>(u->g_p, 32, u->X[1], u->Y[1], u->Z[1],
                                                                        u->g_cat1 + 48, 80);
    }));
    // level 1 encoder
    RT_CHECK(unet_conv_bwd(u, 3, 1, u->a1, 32, u->cat1 + 48, 80, u->g_cat1 + 48, 80, u->g_y));
    RT_CHECK(unet_conv_bwd(u, 2, 1, u->p1, 16, u->a1, 32, u->g_y, 32, u->g_p));
    RT_CHECK(rt_launch(c, "unet_pool_bwd", [&] {
        rtu::k_pool2_bwd<<<ew_blocks(c, V0 * 16), 256, 0, c->stream>>>(u->g_p, 16, u->X[0], u->Y[0], u->Z[0],
                                                                        u->g_cat0 + 32, 48);
    }));
    // level 0 encoder
    RT_CHECK(unet_conv_bwd(u, 1, 0, u->a0, 16, u->cat0 + 32, 48, u->g_cat0 + 32, 48, u->g_y));
    return unet_conv_bwd(u, 0, 0, u->in0, 16, u->a0, 16, u->g_y, 16, nullptr);
}

// deterministic initialisation: He-normal weights from a seeded counter hash, zero biases
static void unet_init_params(rt_unet* u, uint64_t seed, std::vector<float>& host) {
    host.assign(u->nparam, 0.f);
    auto uni = [&](uint64_t i) {
        uint64_t z = seed + 0x9e3779b97f4a7c15ull * (i + 1);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    for (int li = 0; li < N_LAYERS; li++) {
        const Layer& l = u->L[li];
        const double sd = std::sqrt(2.0 / (27.0 * l.cin));
        for (long i = 0; i < 27L * l.cin * l.cout; i++) {
            // Box-Muller from two uniforms
            const double a = uni(2 * (l.woff + i)), b = uni(2 * (l.woff + i) + 1);
            host[l.woff + i] = (float)(sd * std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b));
        }
    }
    const double sd = std::sqrt(1.0 / HEAD_C);
    for (long i = 0; i < 3 * HEAD_C; i++) {
        const double a = uni(2 * (u->head_w + i)), b = uni(2 * (u->head_w + i) + 1);
        host[u->head_w + i] = (float)(sd * std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b));
    }
}

extern "C" int rt_unet_create(rt_ctx* c, int X, int Y, int Z, uint64_t seed, rt_unet** out) {
    if (!c || !out || X < 8 || Y < 8 || Z < 8) return RT_EINVAL;
    *out = nullptr;
    RT_CUDA(c, cudaSetDevice(c->device));
    static bool inited[64] = {false};
    if (!inited[c->device & 63]) {
        RT_CHECK(rtu::conv3_init(c));
        inited[c->device & 63] = true;
    }
    rt_unet* u = new rt_unet();
    u->ctx = c;
    rt_ctx_retain(c);
    u->X[0] = X; u->Y[0] = Y; u->Z[0] = Z;
    for (int l = 1; l < 4; l++) {
        u->X[l] = (u->X[l - 1] + 1) / 2;
        u->Y[l] = (u->Y[l - 1] + 1) / 2;
        u->Z[l] = (u->Z[l - 1] + 1) / 2;
    }
    for (int l = 0; l < 4; l++) u->V[l] = (long)u->X[l] * u->Y[l] * u->Z[l];
    long off = 0, off16 = 0;
    for (int i = 0; i < N_LAYERS; i++) {
        Layer& l = u->L[i];
        l.cin = PLAN[i][0];
        l.cout = PLAN[i][1];
        l.woff = off;
        off += 27L * l.cin * l.cout;
        l.boff = off;
        off += l.cout;
        l.w16off = off16;
        off16 += 27L * l.cin * l.cout;
    }
    u->head_w = off;
    off += 3 * HEAD_C;
    u->head_b = off;
    off += 3;
    u->nparam = off;
    u->nw16 = off16;
    const long V0 = u->V[0], V1 = u->V[1], V2 = u->V[2], V3 = u->V[3];
    int s = RT_OK;
    auto A = [&](int st) { if (s == RT_OK) s = st; };
    A(ualloc(c, &u->P, u->nparam)); A(ualloc(c, &u->G, u->nparam)); A(ualloc(c, &u->M, u->nparam));
    A(ualloc(c, &u->Vv, u->nparam)); A(ualloc(c, &u->W16, u->nw16)); A(ualloc(c, &u->W16t, u->nw16));
    A(ualloc(c, &u->in0, 16 * V0)); A(ualloc(c, &u->a0, 16 * V0)); A(ualloc(c, &u->cat0, 48 * V0));
    A(ualloc(c, &u->p1, 16 * V1)); A(ualloc(c, &u->a1, 32 * V1)); A(ualloc(c, &u->cat1, 80 * V1));
    A(ualloc(c, &u->p2, 32 * V2)); A(ualloc(c, &u->a2, 48 * V2)); A(ualloc(c, &u->cat2, 112 * V2));
    A(ualloc(c, &u->p3, 48 * V3)); A(ualloc(c, &u->a3, 64 * V3)); A(ualloc(c, &u->b3, 64 * V3));
    A(ualloc(c, &u->d2a, 48 * V2)); A(ualloc(c, &u->d2, 48 * V2)); A(ualloc(c, &u->d1a, 32 * V1));
    A(ualloc(c, &u->d1, 32 * V1)); A(ualloc(c, &u->d0a, 16 * V0)); A(ualloc(c, &u->d0, 16 * V0));
    A(ualloc(c, &u->out, 3 * V0)); A(ualloc(c, &u->err, 1)); A(ualloc(c, &u->dscal, 4));
    if (s != RT_OK) {
        unet_free(u);
        return s;
    }
    std::vector<float> host;
    unet_init_params(u, seed, host);
    RT_CUDA(c, cudaMemcpyAsync(u->P, host.data(), sizeof(float) * u->nparam, cudaMemcpyHostToDevice, c->stream));
    RT_CUDA(c, cudaMemsetAsync(u->M, 0, sizeof(float) * u->nparam, c->stream));
    RT_CUDA(c, cudaMemsetAsync(u->Vv, 0, sizeof(float) * u->nparam, c->stream));
    RT_CUDA(c, cudaMemsetAsync(u->err, 0, sizeof(int), c->stream));
    RT_CUDA(c, cudaMemsetAsync(u->in0, 0, sizeof(__nv_bfloat16) * 16 * V0, c->stream));
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    *out = u;
    return RT_OK;
}

extern "C" void rt_unet_destroy(rt_unet* u) {
    if (!u) return;
    cudaSetDevice(u->ctx->device);
    cudaStreamSynchronize(u->ctx->stream);
    unet_free(u);
}

extern "C" long long rt_unet_n_params(rt_unet* u) { return u ? u->nparam : 0; }

extern "C" int rt_unet_get_params(rt_unet* u, float* host) {
    if (!u || !host) return RT_EINVAL;
    RT_CUDA(u->ctx, cudaMemcpyAsync(host, u->P, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost, u->ctx->stream));
    RT_CUDA(u->ctx, cudaStreamSynchronize(u->ctx->stream));
    return RT_OK;
}

extern "C" int rt_unet_set_params(rt_unet* u, const float* host) {
    if (!u || !host) return RT_EINVAL;
    RT_CUDA(u->ctx, cudaMemcpyAsync(u->P, host, sizeof(float) * u->nparam, cudaMemcpyHostToDevice, u->ctx->stream));
    RT_CUDA(u->ctx, cudaStreamSynchronize(u->ctx->stream));
    u->w16_dirty = true;
    return RT_OK;
}

static int unet_check_err(rt_unet* u) {
    int herr = 0;
    RT_CUDA(u->ctx, cudaMemcpyAsync(&herr, u->err, sizeof(int), cudaMemcpyDeviceToHost, u->ctx->stream));
    RT_CUDA(u->ctx, cudaStreamSynchronize(u->ctx->stream));
    if (herr) return rt_fail(u->ctx, RT_ETIMEOUT, "U-Net: tensor-core wait timed out");
    return RT_OK;
}

// in: bf16 [V0][16] device; out: float [V0][3] device (either may be null to use the internal buffers)
extern "C" int rt_unet_forward(rt_unet* u, const void* in, float* out) {
    if (!u) return RT_EINVAL;
    rt_ctx* c = u->ctx;
    RT_CUDA(c, cudaSetDevice(c->device));
    if (in)
        RT_CUDA(c, cudaMemcpyAsync(u->in0, in, sizeof(__nv_bfloat16) * 16 * u->V[0], cudaMemcpyDeviceToDevice,
                                   c->stream));
    RT_CHECK(unet_forward(u));
    if (out) RT_CUDA(c, cudaMemcpyAsync(out, u->out, sizeof(float) * 3 * u->V[0], cudaMemcpyDeviceToDevice, c->stream));
    return unet_check_err(u);
}

// gradients of the mean squared error for one sample (no parameter update); grads_host may be null
extern "C" int rt_unet_gradients(rt_unet* u, const void* in, const float* tgt, double* loss, float* grads_host) {
    if (!u || !in || !tgt) return RT_EINVAL;
    rt_ctx* c = u->ctx;
    RT_CUDA(c, cudaSetDevice(c->device));
    RT_CUDA(c, cudaMemcpyAsync(u->in0, in, sizeof(__nv_bfloat16) * 16 * u->V[0], cudaMemcpyDeviceToDevice, c->stream));
    RT_CHECK(unet_alloc_train(u));
    RT_CUDA(c, cudaMemsetAsync(u->G, 0, sizeof(float) * u->nparam, c->stream));
    RT_CUDA(c, cudaMemsetAsync(u->dloss, 0, sizeof(double), c->stream));
    RT_CHECK(unet_forward(u));
    RT_CHECK(unet_backward(u, tgt));
    if (loss) RT_CUDA(c, cudaMemcpyAsync(loss, u->dloss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (grads_host)
        RT_CUDA(c, cudaMemcpyAsync(grads_host, u->G, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost, c->stream));
    return unet_check_err(u);
}

// one Adam step on a batch of samples (device pointers: in [batch][V0][16] bf16, tgt [batch][V0][3])
extern "C" int rt_unet_train_step(rt_unet* u, int batch, const void* in, const float* tgt, float lr, double* loss) {
    if (!u || !in || !tgt || batch < 1 || lr <= 0) return RT_EINVAL;
    rt_ctx* c = u->ctx;
    RT_CUDA(c, cudaSetDevice(c->device));
    RT_CHECK(unet_alloc_train(u));
    RT_CUDA(c, cudaMemsetAsync(u->G, 0, sizeof(float) * u->nparam, c->stream));
    RT_CUDA(c, cudaMemsetAsync(u->dloss, 0, sizeof(double), c->stream));
    const long V0 = u->V[0];
    for (int b = 0; b < batch; b++) {
        RT_CUDA(c, cudaMemcpyAsync(u->in0, static_cast<const __nv_bfloat16*>(in) + (long)b * 16 * V0,
                                   sizeof(__nv_bfloat16) * 16 * V0, cudaMemcpyDeviceToDevice, c->stream));
        RT_CHECK(unet_forward(u));
        RT_CHECK(unet_backward(u, tgt + (long)b * 3 * V0));
    }
    u->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)u->adam_t), c2 = 1.f - std::pow(b2, (float)u->adam_t);
    // G is the sum of the per-sample gradients; Adam's step does not depend on that scale
    // (only its epsilon does, which is scaled with the batch)
    RT_CHECK(rt_launch(c, "unet_adam", [&] {
        rtu::k_adam<<<ew_blocks(c, u->nparam), 256, 0, c->stream>>>(u->nparam, u->P, u->G, u->M, u->Vv, lr, b1, b2,
                                                                     c1, c2, 1e-8f * (float)batch);
    }));
    u->w16_dirty = true;
    if (loss) {
        RT_CUDA(c, cudaMemcpyAsync(loss, u->dloss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        RT_CUDA(c, cudaStreamSynchronize(c->stream));
        *loss /= batch;
    }
    return unet_check_err(u);
}

// ---------------------------------------------------------------------------
// the network as a preconditioner correction of the solver's finest level
// (node box of level 0; the residual is scaled to unit rms over the active nodes)
// ---------------------------------------------------------------------------
namespace {

// input channels: 0 log10 density feature mapped to [0, 1], 1-3 r * s, 4 support flag, rest 0
__global__ void k_unet_pack(int nx, int ny, int nz, const uint8_t* __restrict__ vact, const uint8_t* __restrict__ vfix,
                            int ws, const float* __restrict__ w, const double* __restrict__ r,
                            const double* __restrict__ rr, const double* __restrict__ zv,
                            const double* __restrict__ zz, double nact, __nv_bfloat16* __restrict__ in) {
    const int vx = nx + 1, vy = ny + 1;
    const long nv = (long)vx * vy * (nz + 1);
    const double s = sqrt(nact / fmax(rr[0], 1e-300));
    const double sz = sqrt(nact / fmax(zz[0], 1e-300));
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < nv; v += (long)gridDim.x * blockDim.x) {
        const int x = (int)(v % vx), y = (int)((v / vx) % vy), z = (int)(v / ((long)vx * vy));
        float feat[16];
#pragma unroll
        for (int c = 0; c < 16; c++) feat[c] = 0.f;
        if (vact[v]) {
            double sw = 0;
            int cnt = 0;
            for (int i = 0; i < 8; i++) {
                const int ex = x - 1 + (i & 1), ey = y - 1 + ((i >> 1) & 1), ez = z - 1 + (i >> 2);
                if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
                const float wv = w[ex + (long)nx * (ey + (long)ny * ez)];
                if (wv > 0.f) { sw += wv; cnt++; }
            }
            const double mw = cnt ? sw / cnt : 1e-9;
            feat[0] = (float)(1.0 + log10(fmax(mw, 1e-9)) / 9.0);
            feat[1] = (float)(r[v] * s);
            feat[2] = (float)(r[nv + v] * s);
            feat[3] = (float)(r[2 * nv + v] * s);
            feat[4] = (ws && vfix[v]) ? 1.f : 0.f;
            feat[5] = (float)(zv[v] * sz);
            feat[6] = (float)(zv[nv + v] * sz);
            feat[7] = (float)(zv[2 * nv + v] * sz);
        }
        uint4* o = reinterpret_cast<uint4*>(in + v * 16);
        __align__(16) __nv_bfloat162 pk[8];
#pragma unroll
        for (int q = 0; q < 8; q++) pk[q] = __floats2bfloat162_rn(feat[2 * q], feat[2 * q + 1]);
        o[0] = *reinterpret_cast<const uint4*>(&pk[0]);
        o[1] = *reinterpret_cast<const uint4*>(&pk[4]);
    }
}

// z += gate * (oscale / sz) * out on active, non-fixed nodes (sz: the inverse rms of the V-cycle's z)
__global__ void k_unet_correct(long nv, const uint8_t* __restrict__ vact, const uint8_t* __restrict__ vfix, int ws,
                               const float* __restrict__ out, const double* __restrict__ zz, double nact,
                               double oscale, const double* __restrict__ gate, double* __restrict__ z) {
    const double g = gate ? gate[0] : 1.0;
    if (g == 0.0) return;
    const double sz = sqrt(nact / fmax(zz[0], 1e-300));
    const double f = g * oscale / sz;
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < nv; v += (long)gridDim.x * blockDim.x) {
        if (!vact[v] || (ws && vfix[v])) continue;
        z[v] += f * out[3 * v];
        z[nv + v] += f * out[3 * v + 1];
        z[2 * nv + v] += f * out[3 * v + 2];
    }
}

// scaled target t = (e - zv) sz on active non-fixed nodes: [V][3] float and its sum of squares
__global__ void k_unet_target(long nv, const uint8_t* __restrict__ vact, const uint8_t* __restrict__ vfix, int ws,
                              const double* __restrict__ e, const double* __restrict__ zv, const double* __restrict__ zz,
                              double nact, float* __restrict__ tgt, double* __restrict__ ss) {
    __shared__ double sh[256];
    const double sz = sqrt(nact / fmax(zz[0], 1e-300));
    double acc = 0;
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < nv; v += (long)gridDim.x * blockDim.x) {
        const bool on = vact[v] && !(ws && vfix[v]);
        for (int c = 0; c < 3; c++) {
            const double t = on ? (e[c * nv + v] - zv[c * nv + v]) * sz : 0.0;
            tgt[3 * v + c] = (float)t;
            acc += t * t;
        }
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(ss, sh[0]);
}

__global__ void k_scale_f32(long n, float* __restrict__ a, double f) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        a[i] = (float)(a[i] * f);
}

}  // namespace

namespace rtu {

bool box_matches(const rt_unet* u, const rt_hier* h) {
    const rt_level& L = h->L[0];
    return u->X[0] == L.vx && u->Y[0] == L.vy && u->Z[0] == L.vz;
}

int pack(rt_unet* u, rt_hier* h, const double* r, const double* rr_dev, const double* zv, const double* zz_dev) {
    rt_ctx* c = h->ctx;
    const rt_level& L = h->L[0];
    const int ws = h->has_support ? 1 : 0;
    return rt_launch(c, "unet_pack", [&] {
        k_unet_pack<<<ew_blocks(c, L.nv), 256, 0, c->stream>>>(L.nx, L.ny, L.nz, L.vact, h->vfix, ws, h->w, r, rr_dev,
                                                               zv, zz_dev, (double)L.n_act_nodes, u->in0);
    });
}

int refresh(rt_unet* u) { return unet_refresh_w16(u); }

// z += N(rho, r, z) correction (forward pass on the packed input), scaled back to solver units
int correct(rt_unet* u, rt_hier* h, const double* r, const double* rr_dev, const double* zz_dev, const double* gate,
            double* z) {
    rt_ctx* c = h->ctx;
    const rt_level& L = h->L[0];
    RT_CHECK(pack(u, h, r, rr_dev, z, zz_dev));
    RT_CHECK(unet_forward(u));
    const int ws = h->has_support ? 1 : 0;
    const double osc = u->oscale > 0 ? u->oscale : 1.0;
    return rt_launch(c, "unet_correct", [&] {
        k_unet_correct<<<ew_blocks(c, L.nv), 256, 0, c->stream>>>(L.nv, L.vact, h->vfix, ws, u->out, zz_dev,
                                                                  (double)L.n_act_nodes, osc, gate, z);
    });
}

// training target from the exact error e and the V-cycle's zv (zv.zv in zz_dev); the first
// call fixes the output unit oscale to the target rms
int target(rt_unet* u, rt_hier* h, const double* e, const double* zv, const double* zz_dev, float* tgt) {
    rt_ctx* c = h->ctx;
    const rt_level& L = h->L[0];
    const int ws = h->has_support ? 1 : 0;
    RT_CUDA(c, cudaMemsetAsync(u->dscal, 0, sizeof(double), c->stream));
    RT_CHECK(rt_launch(c, "unet_target", [&] {
        k_unet_target<<<ew_blocks(c, L.nv), 256, 0, c->stream>>>(L.nv, L.vact, h->vfix, ws, e, zv, zz_dev,
                                                                 (double)L.n_act_nodes, tgt, u->dscal);
    }));
    if (u->oscale <= 0) {
        double ss = 0;
        RT_CUDA(c, cudaMemcpyAsync(&ss, u->dscal, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        RT_CUDA(c, cudaStreamSynchronize(c->stream));
        u->oscale = ss > 0 ? std::sqrt(ss / (3.0 * (double)L.n_act_nodes)) : 1.0;
    }
    const double f = 1.0 / u->oscale;
    return rt_launch(c, "unet_target_scale", [&] {
        k_scale_f32<<<ew_blocks(c, 3 * L.nv), 256, 0, c->stream>>>(3 * L.nv, tgt, f);
    });
}

const void* input(const rt_unet* u) { return u->in0; }
long voxels(const rt_unet* u) { return u->V[0]; }

}  // namespace rtu

extern "C" double rt_unet_output_scale(rt_unet* u) { return u ? u->oscale : 0.0; }

extern "C" int rt_unet_set_output_scale(rt_unet* u, double oscale) {
    if (!u || !(oscale > 0)) return RT_EINVAL;
    u->oscale = oscale;
    return RT_OK;
}
