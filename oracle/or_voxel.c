/* or_voxel.c — CPU oracle of the solid mesh voxeliser (TEST INFRASTRUCTURE ONLY).
 *
 * Restates, in plain C with the reference's float / double arithmetic:
 *  - get_point_bb and padd2SatifyResolution (voxelizer/voxelize_main.cpp:290-342):
 *    tight bounding box of the vertices, resolution rounded up to a power of two
 *    (the first power of two above prefer_reso), the cube of side max_len * R /
 *    prefer_reso centred on the tight box;
 *  - voxinfo's unit length (voxelizer/util.h:63-68): (max - min) / R per axis;
 *  - cpu_voxelize_mesh_solid (voxelizer/cpu_voxelizer.cpp:245-322) with its helpers
 *    checkCCW, TopLeftEdge, check_point_triangle, get_x_coordinate and setBitXor
 *    (:194-243): Schwarz-Seidel solid voxelisation by rays along +x.  For every
 *    triangle whose unit normal has |n.x| >= 1e-6, every voxel-centre point (y, z)
 *    inside its yz projection (edges by the top-left rule) flips the bits of voxels
 *    x = 0 .. xmax of that row, xmax = int(x_hit / unit.x - 0.5).  Bit id
 *    x + y*R + z*R^2, bit (31 - id % 32) of word id / 32 (most significant first).
 *
 * Deviations, stated: a triangle with a zero cross product (degenerate: its normal is
 * NaN in the reference, whose rows then flip an unspecified range) is skipped, and a
 * row with xmax < 0 flips nothing (the GPU reference's signed loop; the CPU reference
 * stores xmax unsigned).  Compiled without FMA contraction (x86-64-v2 has no FMA), so
 * every float operation rounds once, as in the reference's host build.
 */
#include "rt_oracle.h"
#include <math.h>
#include <stdint.h>
#include <string.h>

#define VOX_EPS 0.000001

typedef struct { float x, y; } v2f;
typedef struct { float x, y, z; } v3f;

static v2f v2sub(v2f a, v2f b) { v2f r = {a.x - b.x, a.y - b.y}; return r; }

static int ccw(v2f v0, v2f v1, v2f v2) {
    v2f e0 = v2sub(v1, v0), e1 = v2sub(v2, v0);
    float r = e0.x * e1.y - e1.x * e0.y;
    return r > 0;
}

static int top_left(v2f v0, v2f v1) { return (v1.y < v0.y) || (v1.y == v0.y && v0.x > v1.x); }

/* 0 inside, 1..3 on edge v0v1 / v1v2 / v2v0, -1 outside */
static int point_in_tri(v2f v0, v2f v1, v2f v2, v2f p) {
    v2f PA = v2sub(p, v0), PB = v2sub(p, v1), PC = v2sub(p, v2);
    float t1 = PA.x * PB.y - PA.y * PB.x;
    if (fabs((double)t1) < VOX_EPS && PA.x * PB.x <= 0 && PA.y * PB.y <= 0) return 1;
    float t2 = PB.x * PC.y - PB.y * PC.x;
    if (fabs((double)t2) < VOX_EPS && PB.x * PC.x <= 0 && PB.y * PC.y <= 0) return 2;
    float t3 = PC.x * PA.y - PC.y * PA.x;
    if (fabs((double)t3) < VOX_EPS && PC.x * PA.x <= 0 && PC.y * PA.y <= 0) return 3;
    if (t1 * t2 > 0 && t1 * t3 > 0) return 0;
    return -1;
}

static float x_hit(v3f n, v3f v0, v2f p) {
    float a = p.x - v0.y, c = p.y - v0.z;
    float b = n.y * a, d = n.z * c;
    float e = b + d;
    return -e / n.x + v0.x;
}

void or_voxel_box(const float* coords, long nvert, int prefer_reso, int* reso, float bmin[3], float bmax[3],
                  float unit[3]) {
    float lo[3], hi[3];
    for (int j = 0; j < 3; j++) { lo[j] = INFINITY; hi[j] = -INFINITY; }
    for (long i = 0; i < nvert; i++)
        for (int j = 0; j < 3; j++) {
            float v = coords[3 * i + j];
            lo[j] = fminf(lo[j], v);
            hi[j] = fmaxf(hi[j], v);
        }
    unsigned int r = 1;
    for (int i = 0; i < 32; i++) {
        if ((unsigned int)prefer_reso < r) break;
        r <<= 1;
    }
    float len[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    float max_len = fmaxf(fmaxf(len[0], len[1]), len[2]);
    for (int j = 0; j < 3; j++) {
        float pad = max_len * (float)r / (float)prefer_reso;
        bmin[j] = lo[j] - (pad - len[j]) / 2;
        bmax[j] = hi[j] + (pad - len[j]) / 2;
        unit[j] = (bmax[j] - bmin[j]) / (float)r;
    }
    *reso = (int)r;
}

void or_voxelize_solid(const float* coords, const int* tris, long ntri, int reso, const float bmin[3],
                       const float unit[3], uint32_t* bits) {
    const size_t R = (size_t)reso;
    memset(bits, 0, (R * R * R + 31) / 32 * 4);
    for (long t = 0; t < ntri; t++) {
        v3f v[3];
        for (int k = 0; k < 3; k++) {
            const float* p = coords + 3 * (long)tris[3 * t + k];
            v[k].x = p[0] - bmin[0];
            v[k].y = p[1] - bmin[1];
            v[k].z = p[2] - bmin[2];
        }
        v3f e0 = {v[1].x - v[0].x, v[1].y - v[0].y, v[1].z - v[0].z};
        v3f e1 = {v[2].x - v[1].x, v[2].y - v[1].y, v[2].z - v[1].z};
        v3f c = {e0.y * e1.z - e1.y * e0.z, e0.z * e1.x - e1.z * e0.x, e0.x * e1.y - e1.x * e0.y};
        float dd = c.x * c.x + c.y * c.y;
        dd = dd + c.z * c.z;
        if (dd == 0.f) continue; /* degenerate */
        float inv = 1.f / sqrtf(dd);
        v3f n = {c.x * inv, c.y * inv, c.z * inv};
        if (fabs((double)n.x) < VOX_EPS) continue;
        v2f a = {v[0].y, v[0].z}, b = {v[1].y, v[1].z}, d = {v[2].y, v[2].z};
        if (!ccw(a, b, d)) { v2f s = b; b = d; d = s; }
        float mx = fmaxf(a.x, fmaxf(b.x, d.x)), my = fmaxf(a.y, fmaxf(b.y, d.y));
        float nx_ = fminf(a.x, fminf(b.x, d.x)), ny_ = fminf(a.y, fminf(b.y, d.y));
        int y1 = (int)(float)floor(mx / unit[1] - 0.5), z1 = (int)(float)floor(my / unit[2] - 0.5);
        int y0 = (int)(float)ceil(nx_ / unit[1] - 0.5), z0 = (int)(float)ceil(ny_ / unit[2] - 0.5);
        for (int y = y0; y <= y1; y++)
            for (int z = z0; z <= z1; z++) {
                v2f p = {(float)((y + 0.5) * unit[1]), (float)((z + 0.5) * unit[2])};
                int k = point_in_tri(a, b, d, p);
                if (!((k == 1 && top_left(a, b)) || (k == 2 && top_left(b, d)) || (k == 3 && top_left(d, a)) || k == 0))
                    continue;
                if (y < 0 || z < 0 || y >= reso || z >= reso) continue; /* outside the box */
                int xmax = (int)(x_hit(n, v[0], p) / unit[0] - 0.5);
                if (xmax < 0) continue;
                if (xmax >= reso) xmax = reso - 1; /* stays in its row (hits lie inside the box) */
                for (int x = 0; x <= xmax; x++) {
                    size_t id = (size_t)x + (size_t)y * R + (size_t)z * R * R;
                    bits[id / 32] ^= 1u << (31 - id % 32);
                }
            }
    }
}

/* MSB-first words -> LSB-first words (wordReverse_g, grid/Grid.cu) */
void or_word_reverse(long nwords, uint32_t* w) {
    for (long i = 0; i < nwords; i++) {
        uint32_t x = w[i], r = 0;
        for (int b = 0; b < 32; b++) r |= ((x >> b) & 1u) << (31 - b);
        w[i] = r;
    }
}
