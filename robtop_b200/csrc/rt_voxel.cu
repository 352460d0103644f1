// rt_voxel.cu — solid voxelisation of a closed triangle mesh on the device.
//
// Same result, bit for bit, as the reference's solid voxeliser
// (voxelizer/voxelize_solid.cu:80-150, voxelizer/cpu_voxelizer.cpp:245-322:
// Schwarz-Seidel rays along +x): for every triangle whose unit normal has
// |n.x| >= 1e-6, every voxel-centre point (y, z) inside its yz projection (edge
// points by the top-left rule) flips the bits of voxels x = 0 .. xmax of its row,
// xmax = int(x_hit / unit.x - 0.5).  The reference flips those xmax + 1 bits one
// atomicXor each; here a triangle toggles ONE event bit at xmax and a second pass
// turns each row's events into solid bits with a suffix XOR along x (a voxel is
// solid iff an odd number of events lie at or beyond it).  XOR commutes, so the
// result does not depend on the order of the triangles.
//
// Arithmetic: every float operation is written with an explicit IEEE single
// round-to-nearest intrinsic, so nothing is contracted into an FMA and each rounds
// once, as in the reference's host build; the (y + 0.5) * unit and x / unit - 0.5
// steps are double, as the reference's double literals make them.
//
// Bit layout of the output: bit id x + y*R + z*R^2, bit (31 - id % 32) of word
// id / 32 (the voxeliser's most-significant-first words); genFromMesh reverses the
// words to the least-significant-first layout of the hierarchy
// (grid/Grid.cpp:184-205, wordReverse_g).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "rt_internal.h"

namespace {

constexpr double VOX_EPS = 0.000001;

struct f2 { float x, y; };

__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)}; }
__device__ __forceinline__ float cross2(f2 a, f2 b) { return __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)); }

__device__ __forceinline__ bool top_left(f2 v0, f2 v1) { return (v1.y < v0.y) || (v1.y == v0.y && v0.x > v1.x); }

// 0 inside, 1..3 on edge v0v1 / v1v2 / v2v0, -1 outside (check_point_triangle)
__device__ __forceinline__ int point_in_tri(f2 v0, f2 v1, f2 v2, f2 p) {
    const f2 PA = sub2(p, v0), PB = sub2(p, v1), PC = sub2(p, v2);
    const float t1 = cross2(PA, PB);
    if (fabs((double)t1) < VOX_EPS && __fmul_rn(PA.x, PB.x) <= 0.f && __fmul_rn(PA.y, PB.y) <= 0.f) return 1;
    const float t2 = cross2(PB, PC);
    if (fabs((double)t2) < VOX_EPS && __fmul_rn(PB.x, PC.x) <= 0.f && __fmul_rn(PB.y, PC.y) <= 0.f) return 2;
    const float t3 = cross2(PC, PA);
    if (fabs((double)t3) < VOX_EPS && __fmul_rn(PC.x, PA.x) <= 0.f && __fmul_rn(PC.y, PA.y) <= 0.f) return 3;
    if (__fmul_rn(t1, t2) > 0.f && __fmul_rn(t1, t3) > 0.f) return 0;
    return -1;
}

// one event bit per covered (y, z) row of each triangle
__global__ void k_vox_events(const float* __restrict__ coords, const int* __restrict__ tris, long ntri, int R,
                             float bminx, float bminy, float bminz, float ux, float uy, float uz,
                             unsigned int* __restrict__ ev) {
    const size_t RR = (size_t)R;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < ntri; t += (long)gridDim.x * blockDim.x) {
        float vx[3], vy[3], vz[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float* p = coords + 3 * (long)tris[3 * t + k];
            vx[k] = __fsub_rn(p[0], bminx);
            vy[k] = __fsub_rn(p[1], bminy);
            vz[k] = __fsub_rn(p[2], bminz);
        }
        const float e0x = __fsub_rn(vx[1], vx[0]), e0y = __fsub_rn(vy[1], vy[0]), e0z = __fsub_rn(vz[1], vz[0]);
        const float e1x = __fsub_rn(vx[2], vx[1]), e1y = __fsub_rn(vy[2], vy[1]), e1z = __fsub_rn(vz[2], vz[1]);
        const float cx = __fsub_rn(__fmul_rn(e0y, e1z), __fmul_rn(e1y, e0z));
        const float cy = __fsub_rn(__fmul_rn(e0z, e1x), __fmul_rn(e1z, e0x));
        const float cz = __fsub_rn(__fmul_rn(e0x, e1y), __fmul_rn(e1x, e0y));
        const float dd = __fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz));
        if (dd == 0.f) continue;  // degenerate triangle
        const float inv = __fdiv_rn(1.f, __fsqrt_rn(dd));
        const float nx = __fmul_rn(cx, inv), ny = __fmul_rn(cy, inv), nz = __fmul_rn(cz, inv);
        if (fabs((double)nx) < VOX_EPS) continue;
        f2 a = {vy[0], vz[0]}, b = {vy[1], vz[1]}, c = {vy[2], vz[2]};
        if (!(cross2(sub2(b, a), sub2(c, a)) > 0.f)) {  // counter-clockwise in the yz plane
            const f2 s = b;
            b = c;
            c = s;
        }
        const float mxy = fmaxf(a.x, fmaxf(b.x, c.x)), mxz = fmaxf(a.y, fmaxf(b.y, c.y));
        const float mny = fminf(a.x, fminf(b.x, c.x)), mnz = fminf(a.y, fminf(b.y, c.y));
        const int y1 = (int)(float)floor((double)__fdiv_rn(mxy, uy) - 0.5);
        const int z1 = (int)(float)floor((double)__fdiv_rn(mxz, uz) - 0.5);
        const int y0 = (int)(float)ceil((double)__fdiv_rn(mny, uy) - 0.5);
        const int z0 = (int)(float)ceil((double)__fdiv_rn(mnz, uz) - 0.5);
        for (int y = y0; y <= y1; y++)
            for (int z = z0; z <= z1; z++) {
                const f2 p = {(float)__dmul_rn((double)y + 0.5, (double)uy), (float)__dmul_rn((double)z + 0.5, (double)uz)};
                const int k = point_in_tri(a, b, c, p);
                if (!((k == 1 && top_left(a, b)) || (k == 2 && top_left(b, c)) || (k == 3 && top_left(c, a)) || k == 0))
                    continue;
                if (y < 0 || z < 0 || y >= R || z >= R) continue;  // outside the box (not reached for hits inside it)
                // x of the hit: -(n.y (p.y' - v0.y) + n.z (p.z' - v0.z)) / n.x + v0.x
                const float hb = __fmul_rn(ny, __fsub_rn(p.x, vy[0]));
                const float hd = __fmul_rn(nz, __fsub_rn(p.y, vz[0]));
                const float xh = __fadd_rn(__fdiv_rn(-__fadd_rn(hb, hd), nx), vx[0]);
                int xmax = (int)((double)__fdiv_rn(xh, ux) - 0.5);
                if (xmax < 0) continue;
                if (xmax >= R) xmax = R - 1;
                const size_t id = (size_t)xmax + (size_t)y * RR + (size_t)z * RR * RR;
                atomicXor(&ev[id >> 5], 1u << (31 - (id & 31)));
            }
    }
}

// events -> solid bits for rows of R >= 32 voxels (W = R / 32 words): a segment of
// S = min(W, 32) lanes per row, 32 / S rows per warp.  Within a word the most significant
// bit is the smallest x, so the XOR of the events at or beyond x is the XOR of bit
// positions 0 .. p; the words beyond (later lanes, later chunks of 32 words) carry their
// parity
__global__ void k_vox_rows(int R, unsigned int* __restrict__ bits) {
    const int W = R >> 5;
    const int S = W < 32 ? W : 32;  // power of two
    const long nrows = (long)R * R;
    const int lane = threadIdx.x & 31, sl = lane & (S - 1);
    const long seg = (blockIdx.x * (long)blockDim.x + threadIdx.x) / S;
    const long nsegs = ((long)gridDim.x * blockDim.x) / S;
    // every lane of a warp runs the same number of trips (the shuffles use the full mask)
    const long trips = (nrows + nsegs - 1) / nsegs;
    for (long tr = 0; tr < trips; tr++) {
        const long row = seg + tr * nsegs;
        const bool ok = row < nrows;
        unsigned int* w = bits + (ok ? row : 0) * W;
        unsigned int carry = 0;
        for (int c0 = ((W - 1) >> 5) << 5; c0 >= 0; c0 -= 32) {
            const int i = c0 + sl;
            const unsigned int e = (ok && i < W) ? w[i] : 0u;
            unsigned int t = e;
            t ^= t << 1;
            t ^= t << 2;
            t ^= t << 4;
            t ^= t << 8;
            t ^= t << 16;
            const unsigned int par = __popc(e) & 1u;
            // inclusive suffix XOR of the parities within the segment
            unsigned int sfx = par;
            for (int d = 1; d < S; d <<= 1) {
                const unsigned int o = __shfl_down_sync(0xffffffffu, sfx, d, S);
                if (sl + d < S) sfx ^= o;
            }
            const unsigned int after = (sfx ^ par) ^ carry;  // exclusive suffix + later chunks
            if (ok && i < W) w[i] = after ? ~t : t;
            carry ^= __shfl_sync(0xffffffffu, sfx, 0, S);
        }
    }
}

// R < 32: rows share words; one thread per row walks its bits
__global__ void k_vox_rows_small(int R, unsigned int* __restrict__ bits) {
    const long nrows = (long)R * R;
    for (long row = blockIdx.x * (long)blockDim.x + threadIdx.x; row < nrows; row += (long)gridDim.x * blockDim.x) {
        unsigned int par = 0;
        for (int x = R - 1; x >= 0; x--) {
            const long id = row * R + x;
            const unsigned int m = 1u << (31 - (id & 31));
            par ^= (bits[id >> 5] & m) ? 1u : 0u;
            // each row's bits belong to this thread only: rows of R < 32 bits never straddle
            // a word boundary (R is a power of two), but several rows share a word
            if (par) atomicOr(&bits[id >> 5], m);
            else atomicAnd(&bits[id >> 5], ~m);
        }
    }
}

__global__ void k_brev(long n, unsigned int* __restrict__ w) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        w[i] = __brev(w[i]);
}

}  // namespace

// the padded cube around the vertices and its resolution: get_point_bb and
// padd2SatifyResolution (voxelizer/voxelize_main.cpp:290-342), unit (voxelizer/util.h:63-68)
static void voxel_box(const float* coords, long nvert, int prefer_reso, int* reso, float bmin[3], float bmax[3],
                      float unit[3]) {
    float lo[3], hi[3];
    for (int j = 0; j < 3; j++) {
        lo[j] = INFINITY;
        hi[j] = -INFINITY;
    }
    for (long i = 0; i < nvert; i++)
        for (int j = 0; j < 3; j++) {
            lo[j] = std::fmin(lo[j], coords[3 * i + j]);
            hi[j] = std::fmax(hi[j], coords[3 * i + j]);
        }
    unsigned int r = 1;
    for (int i = 0; i < 32; i++) {
        if ((unsigned int)prefer_reso < r) break;
        r <<= 1;
    }
    const float len[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    const float max_len = std::fmax(std::fmax(len[0], len[1]), len[2]);
    for (int j = 0; j < 3; j++) {
        const float pad = max_len * (float)r / (float)prefer_reso;
        bmin[j] = lo[j] - (pad - len[j]) / 2;
        bmax[j] = hi[j] + (pad - len[j]) / 2;
        unit[j] = (bmax[j] - bmin[j]) / (float)r;
    }
    *reso = (int)r;
}

static int check_mesh(rt_ctx* c, const float* coords, long nvert, const int* tris, long ntri, int prefer_reso) {
    if (!coords || nvert <= 0 || (ntri > 0 && !tris) || ntri < 0) return rt_fail(c, RT_EINVAL, "empty mesh");
    if (prefer_reso < 1 || prefer_reso > 1023) return rt_fail(c, RT_EINVAL, "prefer_reso must be in [1, 1023]");
    for (long i = 0; i < 3 * nvert; i++)
        if (!std::isfinite(coords[i])) return rt_fail(c, RT_EINVAL, "vertex coordinate %ld is not finite", i / 3);
    for (long i = 0; i < 3 * ntri; i++)
        if (tris[i] < 0 || tris[i] >= nvert) return rt_fail(c, RT_EINVAL, "triangle %ld: vertex index out of range", i / 3);
    return RT_OK;
}

// voxelise into device words (event pass + row pass), optionally reversed to LSB-first
static int voxelize_dev(rt_ctx* c, const float* dcoords, const int* dtris, long ntri, int R, const float bmin[3],
                        const float unit[3], unsigned int* dbits, bool lsb_first) {
    const long nw = ((long)R * R * R + 31) / 32;
    RT_CUDA(c, cudaMemsetAsync(dbits, 0, sizeof(unsigned int) * nw, c->stream));
    if (ntri > 0) {
        const long cap = (long)c->sm_count * 8;
        const long nb = (ntri + 127) / 128;
        RT_CHECK(rt_launch(c, "vox_events", [&] {
            k_vox_events<<<(unsigned)(nb < cap ? nb : cap), 128, 0, c->stream>>>(
                dcoords, dtris, ntri, R, bmin[0], bmin[1], bmin[2], unit[0], unit[1], unit[2], dbits);
        }));
    }
    const long rows = (long)R * R;
    if (R >= 32) {
        const long S = (R >> 5) < 32 ? (R >> 5) : 32;  // lanes per row
        const long cap = (long)c->sm_count * 16;
        const long nb = (rows * S + 255) / 256;
        RT_CHECK(rt_launch(c, "vox_rows", [&] {
            k_vox_rows<<<(unsigned)(nb < cap ? nb : cap), 256, 0, c->stream>>>(R, dbits);
        }));
    } else {
        RT_CHECK(rt_launch(c, "vox_rows", [&] {
            k_vox_rows_small<<<(unsigned)((rows + 127) / 128), 128, 0, c->stream>>>(R, dbits);
        }));
    }
    if (lsb_first)
        RT_CHECK(rt_launch(c, "vox_brev", [&] {
            k_brev<<<(unsigned)((nw + 255) / 256 < 4096 ? (nw + 255) / 256 : 4096), 256, 0, c->stream>>>(nw, dbits);
        }));
    return RT_OK;
}

// upload, voxelise, download (host arrays in and out)
static int voxelize_host(rt_ctx* c, const float* coords, long nvert, const int* tris, long ntri, int prefer_reso,
                         bool lsb_first, std::vector<unsigned int>& out, int* reso, float bmin[3], float bmax[3]) {
    RT_CHECK(check_mesh(c, coords, nvert, tris, ntri, prefer_reso));
    RT_CUDA(c, cudaSetDevice(c->device));
    float unit[3];
    voxel_box(coords, nvert, prefer_reso, reso, bmin, bmax, unit);
    const int R = *reso;
    const long nw = ((long)R * R * R + 31) / 32;
    float* dcoords = nullptr;
    int* dtris = nullptr;
    unsigned int* dbits = nullptr;
    int st = RT_OK;
    if (cudaMalloc(&dcoords, sizeof(float) * 3 * nvert) != cudaSuccess ||
        (ntri > 0 && cudaMalloc(&dtris, sizeof(int) * 3 * ntri) != cudaSuccess) ||
        cudaMalloc(&dbits, sizeof(unsigned int) * nw) != cudaSuccess) {
        st = rt_fail(c, RT_ECUDA, "voxeliser: out of device memory");
    }
    if (st == RT_OK && cudaMemcpyAsync(dcoords, coords, sizeof(float) * 3 * nvert, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        st = rt_fail(c, RT_ECUDA, "voxeliser: upload failed");
    if (st == RT_OK && ntri > 0 &&
        cudaMemcpyAsync(dtris, tris, sizeof(int) * 3 * ntri, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        st = rt_fail(c, RT_ECUDA, "voxeliser: upload failed");
    if (st == RT_OK) st = voxelize_dev(c, dcoords, dtris, ntri, R, bmin, unit, dbits, lsb_first);
    if (st == RT_OK) {
        out.resize(nw);
        if (cudaMemcpyAsync(out.data(), dbits, sizeof(unsigned int) * nw, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            st = rt_fail(c, RT_ECUDA, "voxeliser: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cudaStreamSynchronize(c->stream);
    cudaFree(dcoords);
    cudaFree(dtris);
    cudaFree(dbits);
    return st;
}

extern "C" int rt_voxel_resolution(int prefer_reso) {
    if (prefer_reso < 1 || prefer_reso > 1023) return 0;
    unsigned int r = 1;
    while ((unsigned int)prefer_reso >= r) r <<= 1;
    return (int)r;
}

extern "C" int rt_voxelize_mesh(rt_ctx* c, const float* vcoords, long nvert, const int* tri_ids, long ntri,
                                int prefer_reso, uint32_t* solid_bits, long capacity_words, int out_reso[3],
                                float out_box[6]) {
    if (!c || !solid_bits) return RT_EINVAL;
    const int R = rt_voxel_resolution(prefer_reso);
    if (R == 0) return rt_fail(c, RT_EINVAL, "prefer_reso must be in [1, 1023]");
    const long nw = ((long)R * R * R + 31) / 32;
    if (capacity_words < nw) return rt_fail(c, RT_EINVAL, "solid_bits holds %ld words, %ld needed", capacity_words, nw);
    std::vector<unsigned int> bits;
    int reso = 0;
    float bmin[3], bmax[3];
    RT_CHECK(voxelize_host(c, vcoords, nvert, tri_ids, ntri, prefer_reso, false, bits, &reso, bmin, bmax));
    memcpy(solid_bits, bits.data(), sizeof(uint32_t) * nw);
    if (out_reso)
        for (int j = 0; j < 3; j++) out_reso[j] = reso;
    if (out_box)
        for (int j = 0; j < 3; j++) {
            out_box[j] = bmin[j];
            out_box[3 + j] = bmax[j];
        }
    return RT_OK;
}

extern "C" int rt_hier_create_from_mesh(rt_ctx* c, const rt_params* p, const float* vcoords, long nvert,
                                        const int* tri_ids, long ntri, int prefer_reso, rt_hier** out) {
    if (!c || !p || !out) return RT_EINVAL;
    std::vector<unsigned int> bits;
    int reso = 0;
    float bmin[3], bmax[3];
    RT_CHECK(voxelize_host(c, vcoords, nvert, tri_ids, ntri, prefer_reso, true, bits, &reso, bmin, bmax));
    return rt_hier_create_from_bits(c, p, reso, bits.data(), out);
}

// device-resident voxelisation timed with CUDA events (mesh uploaded once)
extern "C" int rt_bench_voxelize(rt_ctx* c, const float* vcoords, long nvert, const int* tri_ids, long ntri,
                                 int prefer_reso, int reps, double* us_per_call) {
    if (!c || reps < 1) return RT_EINVAL;
    RT_CHECK(check_mesh(c, vcoords, nvert, tri_ids, ntri, prefer_reso));
    RT_CUDA(c, cudaSetDevice(c->device));
    int R;
    float bmin[3], bmax[3], unit[3];
    voxel_box(vcoords, nvert, prefer_reso, &R, bmin, bmax, unit);
    const long nw = ((long)R * R * R + 31) / 32;
    float* dcoords = nullptr;
    int* dtris = nullptr;
    unsigned int* dbits = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    int st = RT_OK;
    if (cudaMalloc(&dcoords, sizeof(float) * 3 * nvert) != cudaSuccess ||
        (ntri > 0 && cudaMalloc(&dtris, sizeof(int) * 3 * ntri) != cudaSuccess) ||
        cudaMalloc(&dbits, sizeof(unsigned int) * nw) != cudaSuccess)
        st = rt_fail(c, RT_ECUDA, "voxeliser: out of device memory");
    if (st == RT_OK) {
        cudaMemcpyAsync(dcoords, vcoords, sizeof(float) * 3 * nvert, cudaMemcpyHostToDevice, c->stream);
        if (ntri > 0) cudaMemcpyAsync(dtris, tri_ids, sizeof(int) * 3 * ntri, cudaMemcpyHostToDevice, c->stream);
        st = voxelize_dev(c, dcoords, dtris, ntri, R, bmin, unit, dbits, false);  // warm-up
    }
    if (st == RT_OK) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, c->stream);
        for (int i = 0; i < reps && st == RT_OK; i++) st = voxelize_dev(c, dcoords, dtris, ntri, R, bmin, unit, dbits, false);
        cudaEventRecord(b, c->stream);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (us_per_call) *us_per_call = ms * 1e3 / reps;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    cudaStreamSynchronize(c->stream);
    cudaFree(dcoords);
    cudaFree(dtris);
    cudaFree(dbits);
    return st;
}
