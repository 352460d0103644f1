// rt_unet.h — internal interface of the learned preconditioner (not part of the ABI).
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include <vector>

#include "rt_internal.h"

namespace rtu {

// one 3x3x3 convolution launch (zero padding 1, stride 1) over an X x Y x Z voxel box
struct ConvArgs {
    const __nv_bfloat16* in = nullptr;  // [V][in_stride], channels [0, cin)
    int in_stride = 0;
    int cin = 0;
    const __nv_bfloat16* w = nullptr;   // [cout][27][cin], tap = (dz+1)*9 + (dy+1)*3 + (dx+1)
    const float* bias = nullptr;        // [cout] or null
    int cout = 0;
    void* out = nullptr;                // [V][out_stride] bf16, or float when out_f32
    int out_stride = 0;
    int out_f32 = 0;
    int relu = 0;
    int accumulate = 0;                 // float output only: out += result
    int X = 0, Y = 0, Z = 0;
    int* err = nullptr;                 // set to 1 if an MMA wait timed out
};

int conv3_init(rt_ctx* c);
int conv3(rt_ctx* c, const ConvArgs& a);
size_t conv3_smem_bytes(int cin, int cout);
void conv3_set_variant(int v);  // 1: halo tile (default), 0: per-tap gather

}  // namespace rtu

namespace rtu {
// element-wise and reduction kernels (rt_unet_kernels.cu)
__global__ void k_pool2(const __nv_bfloat16* in, int in_stride, int C, int X, int Y, int Z, __nv_bfloat16* out,
                        int out_stride);
__global__ void k_pool2_bwd(const float* gout, int C, int X, int Y, int Z, float* gin, int gin_stride);
__global__ void k_up2(const __nv_bfloat16* in, int C, int X, int Y, int Z, __nv_bfloat16* out, int out_stride);
__global__ void k_up2_bwd(const float* gout, int gout_stride, int C, int X, int Y, int Z, float* gin);
__global__ void k_relu_bwd(const float* g, int g_stride, const __nv_bfloat16* y, int y_stride, int C, long V, int relu,
                           __nv_bfloat16* gpre);
__global__ void k_bias_grad(const __nv_bfloat16* gpre, int C, long V, float* db);
__global__ void k_conv3_dw(const __nv_bfloat16* in, int in_stride, int cin, const __nv_bfloat16* gpre, int cout, int X,
                           int Y, int Z, long chunk, float* dw);
__global__ void k_weights_bf16(const float* w, int cin, int cout, __nv_bfloat16* w16, __nv_bfloat16* w16t);
__global__ void k_adam(long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float c1,
                       float c2, float eps);
__global__ void k_head(const __nv_bfloat16* in, int C, long V, const float* hw, const float* hb, float* out);
__global__ void k_head_bwd(const __nv_bfloat16* in, int C, long V, const float* hw, const float* gout, float* gin,
                           float* dhw, float* dhb);
__global__ void k_mse(const float* out, const float* tgt, long n, float* gout, double* loss);
}  // namespace rtu

struct rt_unet;
namespace rtu {
bool box_matches(const rt_unet* u, const rt_hier* h);
// input channels: 0 log density, 1-3 r / rms(r), 4 support flag, 5-7 zv / rms(zv) (zv = the
// V-cycle's output for r); rr_dev = r.r, zz_dev = zv.zv
int pack(rt_unet* u, rt_hier* h, const double* r, const double* rr_dev, const double* zv, const double* zz_dev);
// z += gate * rms(z) * oscale * N(rho, r, z): z holds the V-cycle's output on entry
int correct(rt_unet* u, rt_hier* h, const double* r, const double* rr_dev, const double* zz_dev, const double* gate,
            double* z);
// target (e - zv) / (rms(zv) oscale) from the exact error e and the V-cycle's zv
int target(rt_unet* u, rt_hier* h, const double* e, const double* zv, const double* zz_dev, float* tgt);
// convert the FP32 parameters to the BF16 copies the convolutions read, if they changed
int refresh(rt_unet* u);
const void* input(const rt_unet* u);
long voxels(const rt_unet* u);
}  // namespace rtu
