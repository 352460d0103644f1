/*
 * rt_oracle.c — FP64 CPU restatement of robtop's multigrid solver hot path.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE: the checker for the CUDA library and
 * the timed CPU baseline.  Every function names the reference file:line whose
 * behaviour it restates (paths relative to the lavenklau/robtop project root).
 * See rt_oracle.h for the parity status ("parity unpinned": no golden vectors
 * exist in the reference; pinned by its known-answer tests only).
 */
#include "rt_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define NODE(x, y, z, vx, vy) ((long)(x) + (long)(vx) * ((long)(y) + (long)(vy) * (long)(z)))

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* ------------------------------------------------------------------------ */
/* element template matrix: element/templateMatrix.cpp:15-124               */
/* ------------------------------------------------------------------------ */
static void dN(int i, double elen, const double param[3], double dn[3]) {
    int id[3] = {i % 2, i / 2 % 2, i / 4};
    double r[3];
    for (int k = 0; k < 3; k++) r[k] = id[k] ? param[k] : (1 - param[k]);
    for (int k = 0; k < 3; k++)
        dn[k] = (id[k] ? 1.0 / elen : -1.0 / elen) * r[(k + 1) % 3] * r[(k + 2) % 3];
}

void or_template_matrix(double E, double nu, double h, double* KE) {
    double D[6][6];
    memset(D, 0, sizeof(D));
    double s = E / ((1 + nu) * (1 - 2 * nu));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i][j] = s * (i == j ? 1 - nu : nu);
    for (int i = 3; i < 6; i++) D[i][i] = s * (1 - 2 * nu) / 2;
    double p = sqrt(3.0) / 3;
    memset(KE, 0, sizeof(double) * 576);
    for (int g = 0; g < 8; g++) {
        double gp[3] = {((2 * (g % 2) - 1) * p + 1) / 2, ((2 * (g / 2 % 2) - 1) * p + 1) / 2,
                        ((2 * (g / 4) - 1) * p + 1) / 2};
        double gN[8][3];
        for (int k = 0; k < 8; k++) dN(k, h, gp, gN[k]);
        double B[6][24];
        memset(B, 0, sizeof(B));
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 8; b++) B[a][3 * b + a] = gN[b][a];
        for (int b = 0; b < 8; b++) {
            B[3][3 * b + 1] = gN[b][2]; B[3][3 * b + 2] = gN[b][1]; /* yz */
            B[4][3 * b + 0] = gN[b][2]; B[4][3 * b + 2] = gN[b][0]; /* xz */
            B[5][3 * b + 0] = gN[b][1]; B[5][3 * b + 1] = gN[b][0]; /* xy */
        }
        double DB[6][24];
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 24; j++) {
                double acc = 0;
                for (int k = 0; k < 6; k++) acc += D[i][k] * B[k][j];
                DB[i][j] = acc;
            }
        for (int i = 0; i < 24; i++)
            for (int j = 0; j < 24; j++) {
                double acc = 0;
                for (int k = 0; k < 6; k++) acc += B[k][i] * DB[k][j];
                KE[i * 24 + j] += acc;
            }
    }
    double sc = pow(h / 2, 3);
    for (int i = 0; i < 576; i++) KE[i] *= sc;
}

/* ------------------------------------------------------------------------ */
/* occupancy on the cubic bit grid                                          */
/* ------------------------------------------------------------------------ */
static inline int rbit(const uint32_t* b, long id) { return (b[id >> 5] >> (id & 31)) & 1u; }
static inline void sbit(uint32_t* b, long id) { b[id >> 5] |= 1u << (id & 31); }

/* grid/Grid.cu:2555-2583: a vertex is solid iff one of its 8 incident elements is */
void or_cube_vbits(int R, const uint32_t* ebits, uint32_t* vbits) {
    int V = R + 1;
    long nv = (long)V * V * V;
    memset(vbits, 0, sizeof(uint32_t) * ((nv + 31) / 32));
    for (long t = 0; t < nv; t++) {
        int p[3] = {(int)(t % V), (int)(t % ((long)V * V) / V), (int)(t / ((long)V * V))};
        for (int i = 0; i < 8; i++) {
            int e[3] = {p[0] + i % 2 - 1, p[1] + i % 4 / 2 - 1, p[2] + i / 4 - 1};
            if (e[0] < 0 || e[1] < 0 || e[2] < 0 || e[0] >= R || e[1] >= R || e[2] >= R) continue;
            if (rbit(ebits, e[0] + (long)e[1] * R + (long)e[2] * R * R)) { sbit(vbits, t); break; }
        }
    }
}

/* grid/Grid.cu:2612-2632: coarse element solid iff any of its 8 children is */
void or_cube_coarsen(int Rf, const uint32_t* ef, uint32_t* ec) {
    int Rc = Rf >> 1;
    long nc = (long)Rc * Rc * Rc;
    memset(ec, 0, sizeof(uint32_t) * ((nc + 31) / 32));
    long nf = (long)Rf * Rf * Rf;
    for (long t = 0; t < nf; t++) {
        if (!rbit(ef, t)) continue;
        int x = (int)(t % Rf) >> 1, y = (int)(t % ((long)Rf * Rf) / Rf) >> 1, z = (int)(t / ((long)Rf * Rf)) >> 1;
        sbit(ec, x + (long)y * Rc + (long)z * Rc * Rc);
    }
}

long or_bits_total(long nwords, const uint32_t* bits) {
    long s = 0;
    for (long i = 0; i < nwords; i++) s += __builtin_popcount(bits[i]);
    return s;
}

/* BitSAT::operator[] (grid/Grid.h:116-120): number of set bits strictly below id */
void or_bitsat_rank(long nwords, const uint32_t* bits, long nq, const long* q, int* rank) {
    int* sat = (int*)malloc(sizeof(int) * (nwords + 1));
    int acc = 0;
    for (long i = 0; i < nwords; i++) { sat[i] = acc; acc += __builtin_popcount(bits[i]); }
    sat[nwords] = acc;
    for (long i = 0; i < nq; i++) {
        long id = q[i];
        long w = id >> 5;
        int m = (int)(id & 31);
        rank[i] = sat[w] + __builtin_popcount(bits[w] & ((1u << m) - 1u));
    }
    free(sat);
}

/* Grid::compute_gscolor (grid/Grid.cu:548-623) + Grid::enumerate_gs_subset
 * (grid/Grid.cpp:2045-2106): colour = x%2 + 2(y%2) + 4(z%2); each colour set is
 * padded to a multiple of 32; within a colour, active vertices keep bit order. */
void or_gs_maps(int vreso, const uint32_t* vbits, int nv_act, int* vlexi2gs, int* gs_num, int* nv_gs) {
    long nb = (long)vreso * vreso * vreso;
    int* col = (int*)malloc(sizeof(int) * (nv_act > 0 ? nv_act : 1));
    int cnt[8] = {0};
    int k = 0;
    for (long t = 0; t < nb; t++) {
        if (!rbit(vbits, t)) continue;
        int x = (int)(t % vreso), y = (int)(t % ((long)vreso * vreso) / vreso), z = (int)(t / ((long)vreso * vreso));
        int c = x % 2 + (y % 2) * 2 + (z % 2) * 4;
        col[k++] = c;
        cnt[c]++;
    }
    int off[8], tot = 0;
    for (int c = 0; c < 8; c++) {
        int padded = (cnt[c] + 31) / 32 * 32;
        gs_num[c] = padded;
        off[c] = tot;
        tot += padded;
    }
    int acc[8] = {0};
    for (int i = 0; i < k; i++) vlexi2gs[i] = off[col[i]] + acc[col[i]]++;
    *nv_gs = tot;
    free(col);
}

/* ------------------------------------------------------------------------ */
/* dense-box hierarchy helpers                                              */
/* ------------------------------------------------------------------------ */
void or_node_active(int nx, int ny, int nz, const uint8_t* eact, uint8_t* vact) {
    int vx = nx + 1, vy = ny + 1, vz = nz + 1;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                int a = 0;
                for (int i = 0; i < 8 && !a; i++) {
                    int ex = x + i % 2 - 1, ey = y + i / 2 % 2 - 1, ez = z + i / 4 - 1;
                    if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
                    a = eact[ex + (long)nx * (ey + (long)ny * ez)] != 0;
                }
                vact[NODE(x, y, z, vx, vy)] = (uint8_t)a;
            }
}

void or_coarsen_elements(int nx, int ny, int nz, int ratio, const uint8_t* ef, uint8_t* ec) {
    int cx = (nx + ratio - 1) / ratio, cy = (ny + ratio - 1) / ratio, cz = (nz + ratio - 1) / ratio;
    memset(ec, 0, (size_t)cx * cy * cz);
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++)
                if (ef[x + (long)nx * (y + (long)ny * z)])
                    ec[x / ratio + (long)cx * (y / ratio + (long)cy * (z / ratio))] = 1;
}

/* mark_surface_nodes_kernel (grid/Grid.cu:2005-2039): a node is on the surface
 * unless, along every axis, some pair of its incident elements facing each
 * other across the node is solid. */
void or_surface_nodes(int nx, int ny, int nz, const uint8_t* eact, uint8_t* surf) {
    int vx = nx + 1, vy = ny + 1, vz = nz + 1;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                int s[2][2][2];
                for (int i = 0; i < 8; i++) {
                    int ex = x + i % 2 - 1, ey = y + i / 2 % 2 - 1, ez = z + i / 4 - 1;
                    int a = 0;
                    if (ex >= 0 && ey >= 0 && ez >= 0 && ex < nx && ey < ny && ez < nz)
                        a = eact[ex + (long)nx * (ey + (long)ny * ez)] != 0;
                    s[i % 2][i / 2 % 2][i / 4] = a;
                }
                int ax[3] = {0, 0, 0};
                for (int i = 0; i < 2; i++)
                    for (int j = 0; j < 2; j++) {
                        ax[0] |= s[0][i][j] && s[1][i][j];
                        ax[1] |= s[i][0][j] && s[i][1][j];
                        ax[2] |= s[i][j][0] && s[i][j][1];
                    }
                surf[NODE(x, y, z, vx, vy)] = (uint8_t)(!ax[0] || !ax[1] || !ax[2]);
            }
}

/* penalty = powf(rho, p) in single precision, as every reference kernel does it */
void or_penalty_weights(long ne, const uint8_t* eact, const float* rho, float p, double* w) {
    for (long e = 0; e < ne; e++) w[e] = eact[e] ? (double)powf(rho[e], p) : 0.0;
}

/* ------------------------------------------------------------------------ */
/* finest level, matrix free                                                */
/* ------------------------------------------------------------------------ */
/* Sum over the 8 incident elements of rho^p * KE-row-block(vi) * u_e.
 * skip_self: leave out the node's own column block (GS form, grid/Grid.cu:1000).
 * Fixed neighbours contribute u = 0 (grid/Grid.cu:1540-1542). */
static void fine_node_sum(const or_level* L, const double* KE, const double* u, int x, int y, int z, int skip_self,
                          double KU[3], double S[9], int* ne_out) {
    int nx = L->nx, ny = L->ny, nz = L->nz, vx = nx + 1, vy = ny + 1;
    long nv = (long)vx * vy * (nz + 1);
    KU[0] = KU[1] = KU[2] = 0;
    if (S) for (int i = 0; i < 9; i++) S[i] = 0;
    int ne = 0;
    for (int i = 0; i < 8; i++) {
        int ex = x + i % 2 - 1, ey = y + i / 2 % 2 - 1, ez = z + i / 4 - 1;
        if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
        long e = ex + (long)nx * (ey + (long)ny * ez);
        if (!L->eact[e]) continue;
        ne++;
        double pen = L->w[e];
        int vi = 7 - i;
        for (int vj = 0; vj < 8; vj++) {
            int jx = ex + vj % 2, jy = ey + vj / 2 % 2, jz = ez + vj / 4;
            long nj = NODE(jx, jy, jz, vx, vy);
            int self = (jx == x && jy == y && jz == z);
            if (self && S) {
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) S[a * 3 + b] += pen * KE[(vi * 3 + a) * 24 + vj * 3 + b];
            }
            if (self && skip_self) continue;
            if (L->vfix && L->vfix[nj]) continue;
            double uj[3] = {u[nj], u[nv + nj], u[2 * nv + nj]};
            for (int row = 0; row < 3; row++)
                for (int col = 0; col < 3; col++) KU[row] += pen * KE[(row + vi * 3) * 24 + col + vj * 3] * uj[col];
        }
    }
    if (ne_out) *ne_out = ne;
}

/* applyK_OTFA_kernel (grid/Grid.cu:2439-2517): fixed rows return u_i */
void or_fine_applyK(const or_level* L, const double* KE, const double* u, double* out) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                long v = NODE(x, y, z, vx, vy);
                double KU[3] = {0, 0, 0};
                if (L->vact[v]) {
                    if (L->vfix && L->vfix[v]) { KU[0] = u[v]; KU[1] = u[nv + v]; KU[2] = u[2 * nv + v]; }
                    else fine_node_sum(L, KE, u, x, y, z, 0, KU, NULL, NULL);
                }
                out[v] = KU[0]; out[nv + v] = KU[1]; out[2 * nv + v] = KU[2];
            }
}

/* update_residual_OTFA_{NS,WS}_kernel (grid/Grid.cu:1450-1557): fixed rows have KU = 0 */
void or_fine_residual(const or_level* L, const double* KE, const double* u, const double* f, double* r) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                long v = NODE(x, y, z, vx, vy);
                double KU[3] = {0, 0, 0};
                if (L->vact[v] && !(L->vfix && L->vfix[v])) fine_node_sum(L, KE, u, x, y, z, 0, KU, NULL, NULL);
                for (int c = 0; c < 3; c++) r[c * nv + v] = L->vact[v] ? f[c * nv + v] - KU[c] : 0.0;
            }
}

/* point-block update with the in-node sequential x->y->z order of
 * grid/Grid.cu:1043-1048 (backward = z->y->x, the adjoint sweep) */
static inline void block_gs_update(const double S[9], const double F[3], const double KU[3], double u[3], int backward) {
    if (!backward) {
        u[0] = (F[0] - S[1] * u[1] - S[2] * u[2] - KU[0]) / S[0];
        u[1] = (F[1] - S[3] * u[0] - S[5] * u[2] - KU[1]) / S[4];
        u[2] = (F[2] - S[6] * u[0] - S[7] * u[1] - KU[2]) / S[8];
    } else {
        u[2] = (F[2] - S[6] * u[0] - S[7] * u[1] - KU[2]) / S[8];
        u[1] = (F[1] - S[3] * u[0] - S[5] * u[2] - KU[1]) / S[4];
        u[0] = (F[0] - S[1] * u[1] - S[2] * u[2] - KU[0]) / S[0];
    }
}

/* gs_relax_OTFA_{NS,WS}_kernel (grid/Grid.cu:792-1066) over colours 0..7
 * (Grid::gs_relax, grid/Grid.cu:1068-1092); a fixed node gets S = n_e * I, KU = 0 */
void or_fine_gs(const or_level* L, const double* KE, double* u, const double* f, int backward) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
    for (int cc = 0; cc < 8; cc++) {
        int c = backward ? 7 - cc : cc;
        int px = c & 1, py = (c >> 1) & 1, pz = (c >> 2) & 1;
#pragma omp parallel for collapse(2)
        for (int z = pz; z < vz; z += 2)
            for (int y = py; y < vy; y += 2)
                for (int x = px; x < vx; x += 2) {
                    long v = NODE(x, y, z, vx, vy);
                    if (!L->vact[v]) continue;
                    double KU[3], S[9];
                    int ne;
                    fine_node_sum(L, KE, u, x, y, z, 1, KU, S, &ne);
                    if (L->vfix && L->vfix[v]) {
                        for (int i = 0; i < 9; i++) S[i] = 0;
                        S[0] = S[4] = S[8] = ne;
                        KU[0] = KU[1] = KU[2] = 0;
                    }
                    double F[3] = {f[v], f[nv + v], f[2 * nv + v]};
                    double uu[3] = {u[v], u[nv + v], u[2 * nv + v]};
                    block_gs_update(S, F, KU, uu, backward);
                    u[v] = uu[0]; u[nv + v] = uu[1]; u[2 * nv + v] = uu[2];
                }
    }
}

static void inv3(const double S[9], double I[9]) {
    double a = S[0], b = S[1], c = S[2], d = S[3], e = S[4], f = S[5], g = S[6], h = S[7], k = S[8];
    double A = e * k - f * h, B = -(d * k - f * g), C = d * h - e * g;
    double det = a * A + b * B + c * C;
    double id = 1.0 / det;
    I[0] = A * id; I[1] = -(b * k - c * h) * id; I[2] = (b * f - c * e) * id;
    I[3] = B * id; I[4] = (a * k - c * g) * id; I[5] = -(a * f - c * d) * id;
    I[6] = C * id; I[7] = -(a * h - b * g) * id; I[8] = (a * e - b * d) * id;
}

/* damped point-block Jacobi, u += omega * D^-1 (f - K u); fixed nodes are set to f / n_e
 * (the value the reference's GS gives them). Not in the reference: the smoother
 * named by the 64x32x32 cantilever configuration. */
void or_fine_jacobi(const or_level* L, const double* KE, double* u, const double* f, double omega, double* tmp) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                long v = NODE(x, y, z, vx, vy);
                double nu[3] = {0, 0, 0};
                if (L->vact[v]) {
                    double KU[3], S[9];
                    int ne;
                    fine_node_sum(L, KE, u, x, y, z, 0, KU, S, &ne);
                    if (L->vfix && L->vfix[v]) {
                        for (int c = 0; c < 3; c++) nu[c] = f[c * nv + v] / ne;
                    } else {
                        double Si[9], rr[3];
                        inv3(S, Si);
                        for (int c = 0; c < 3; c++) rr[c] = f[c * nv + v] - KU[c];
                        for (int c = 0; c < 3; c++)
                            nu[c] = u[c * nv + v] + omega * (Si[c * 3] * rr[0] + Si[c * 3 + 1] * rr[1] + Si[c * 3 + 2] * rr[2]);
                    }
                }
                for (int c = 0; c < 3; c++) tmp[c * nv + v] = nu[c];
            }
    memcpy(u, tmp, sizeof(double) * 3 * nv);
}

/* ------------------------------------------------------------------------ */
/* assembled-stencil levels                                                 */
/* ------------------------------------------------------------------------ */
static void st_node_sum(const or_level* L, const double* u, int x, int y, int z, int skip_self, double Au[3]) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
    long v = NODE(x, y, z, vx, vy);
    Au[0] = Au[1] = Au[2] = 0;
    for (int k = 0; k < 27; k++) {
        if (skip_self && k == 13) continue;
        int jx = x + k % 3 - 1, jy = y + k / 3 % 3 - 1, jz = z + k / 9 - 1;
        if (jx < 0 || jy < 0 || jz < 0 || jx >= vx || jy >= vy || jz >= vz) continue;
        long nj = NODE(jx, jy, jz, vx, vy);
        if (!L->vact[nj]) continue;
        double uj[3] = {u[nj], u[nv + nj], u[2 * nv + nj]};
        for (int row = 0; row < 3; row++)
            for (int col = 0; col < 3; col++) Au[row] += L->st[(long)(k * 9 + row * 3 + col) * nv + v] * uj[col];
    }
}

void or_st_applyA(const or_level* L, const double* u, double* out) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                long v = NODE(x, y, z, vx, vy);
                double Au[3] = {0, 0, 0};
                if (L->vact[v]) st_node_sum(L, u, x, y, z, 0, Au);
                for (int c = 0; c < 3; c++) out[c * nv + v] = Au[c];
            }
}

/* update_residual_kernel_1 (grid/Grid.cu:1350-1448) */
void or_st_residual(const or_level* L, const double* u, const double* f, double* r) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                long v = NODE(x, y, z, vx, vy);
                double Au[3] = {0, 0, 0};
                if (L->vact[v]) st_node_sum(L, u, x, y, z, 0, Au);
                for (int c = 0; c < 3; c++) r[c * nv + v] = L->vact[v] ? f[c * nv + v] - Au[c] : 0.0;
            }
}

/* gs_relax_kernel (grid/Grid.cu:678-790) over colours 0..7 */
void or_st_gs(const or_level* L, double* u, const double* f, int backward) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
    for (int cc = 0; cc < 8; cc++) {
        int c = backward ? 7 - cc : cc;
        int px = c & 1, py = (c >> 1) & 1, pz = (c >> 2) & 1;
#pragma omp parallel for collapse(2)
        for (int z = pz; z < vz; z += 2)
            for (int y = py; y < vy; y += 2)
                for (int x = px; x < vx; x += 2) {
                    long v = NODE(x, y, z, vx, vy);
                    if (!L->vact[v]) continue;
                    double Au[3], S[9];
                    st_node_sum(L, u, x, y, z, 1, Au);
                    for (int i = 0; i < 9; i++) S[i] = L->st[(long)(13 * 9 + i) * nv + v];
                    double F[3] = {f[v], f[nv + v], f[2 * nv + v]};
                    double uu[3] = {u[v], u[nv + v], u[2 * nv + v]};
                    block_gs_update(S, F, Au, uu, backward);
                    u[v] = uu[0]; u[nv + v] = uu[1]; u[2 * nv + v] = uu[2];
                }
    }
}

void or_st_jacobi(const or_level* L, double* u, const double* f, double omega, double* tmp) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                long v = NODE(x, y, z, vx, vy);
                double nu[3] = {0, 0, 0};
                if (L->vact[v]) {
                    double Au[3], S[9], Si[9], rr[3];
                    st_node_sum(L, u, x, y, z, 0, Au);
                    for (int i = 0; i < 9; i++) S[i] = L->st[(long)(13 * 9 + i) * nv + v];
                    inv3(S, Si);
                    for (int c = 0; c < 3; c++) rr[c] = f[c * nv + v] - Au[c];
                    for (int c = 0; c < 3; c++)
                        nu[c] = u[c * nv + v] + omega * (Si[c * 3] * rr[0] + Si[c * 3 + 1] * rr[1] + Si[c * 3 + 2] * rr[2]);
                }
                for (int c = 0; c < 3; c++) tmp[c * nv + v] = nu[c];
            }
    memcpy(u, tmp, sizeof(double) * 3 * nv);
}

/* ------------------------------------------------------------------------ */
/* Chebyshev smoothing (not in the reference)                               */
/* ------------------------------------------------------------------------ */
void or_cheby_coef(double lmax, int k, double* a, double* b) {
    double hi = 1.1 * lmax, lo = lmax / 30.0;
    double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    double rho = 1.0 / sigma;
    *a = 0.0;
    *b = 1.0 / theta;
    for (int i = 1; i <= k; i++) {
        double rn = 1.0 / (2.0 * sigma - rho);
        *a = rn * rho;
        *b = 2.0 * rn / delta;
        rho = rn;
    }
}

/* d = a_k d + b_k D^-1 (f - K u), unew = u + d; fixed nodes: unew = f / n_e, d = 0 */
void or_fine_cheby(const or_level* L, const double* KE, const double* u, const double* f, double* unew, double* d,
                   int k) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
    double ca, cb;
    or_cheby_coef(L->lmax, k, &ca, &cb);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                long v = NODE(x, y, z, vx, vy);
                double nu[3] = {0, 0, 0}, dn[3] = {0, 0, 0};
                if (L->vact[v]) {
                    double KU[3], S[9];
                    int ne;
                    fine_node_sum(L, KE, u, x, y, z, 0, KU, S, &ne);
                    if (L->vfix && L->vfix[v]) {
                        for (int c = 0; c < 3; c++) nu[c] = f[c * nv + v] / ne;
                    } else {
                        double Si[9], rr[3];
                        inv3(S, Si);
                        for (int c = 0; c < 3; c++) rr[c] = f[c * nv + v] - KU[c];
                        for (int c = 0; c < 3; c++) {
                            double zc = Si[c * 3] * rr[0] + Si[c * 3 + 1] * rr[1] + Si[c * 3 + 2] * rr[2];
                            dn[c] = (k == 0 ? 0.0 : ca * d[c * nv + v]) + cb * zc;
                            nu[c] = u[c * nv + v] + dn[c];
                        }
                    }
                }
                for (int c = 0; c < 3; c++) { unew[c * nv + v] = nu[c]; d[c * nv + v] = dn[c]; }
            }
}

/* ------------------------------------------------------------------------ */
/* transfers: trilinear P with weights prod (r-|d|)/r, restriction = P^T    */
/* restrict_residual{,_nondyadic}_kernel (grid/Grid.cu:1680-1794),          */
/* prolongate_correction{,_nondyadic}_kernel (grid/Grid.cu:1818-1895)        */
/* ------------------------------------------------------------------------ */
void or_restrict(const or_level* fine, const or_level* coarse, const double* rf, double* fc) {
    int r = coarse->ratio;
    int fvx = fine->nx + 1, fvy = fine->ny + 1, fvz = fine->nz + 1;
    int cvx = coarse->nx + 1, cvy = coarse->ny + 1, cvz = coarse->nz + 1;
    long nvf = (long)fvx * fvy * fvz, nvc = (long)cvx * cvy * cvz;
#pragma omp parallel for collapse(2)
    for (int Z = 0; Z < cvz; Z++)
        for (int Y = 0; Y < cvy; Y++)
            for (int X = 0; X < cvx; X++) {
                long vc = NODE(X, Y, Z, cvx, cvy);
                double s[3] = {0, 0, 0};
                if (coarse->vact[vc]) {
                    for (int dz = -(r - 1); dz <= r - 1; dz++) {
                        int z = r * Z + dz;
                        if (z < 0 || z >= fvz) continue;
                        for (int dy = -(r - 1); dy <= r - 1; dy++) {
                            int y = r * Y + dy;
                            if (y < 0 || y >= fvy) continue;
                            for (int dx = -(r - 1); dx <= r - 1; dx++) {
                                int x = r * X + dx;
                                if (x < 0 || x >= fvx) continue;
                                long vf = NODE(x, y, z, fvx, fvy);
                                if (!fine->vact[vf]) continue;
                                double w = (double)((r - abs(dx)) * (r - abs(dy)) * (r - abs(dz))) / (double)(r * r * r);
                                for (int c = 0; c < 3; c++) s[c] += w * rf[c * nvf + vf];
                            }
                        }
                    }
                }
                for (int c = 0; c < 3; c++) fc[c * nvc + vc] = s[c];
            }
}

void or_prolong_add(const or_level* fine, const or_level* coarse, const double* uc, double* uf) {
    int r = coarse->ratio;
    int fvx = fine->nx + 1, fvy = fine->ny + 1, fvz = fine->nz + 1;
    int cvx = coarse->nx + 1, cvy = coarse->ny + 1;
    long nvf = (long)fvx * fvy * fvz, nvc = (long)cvx * cvy * (coarse->nz + 1);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < fvz; z++)
        for (int y = 0; y < fvy; y++)
            for (int x = 0; x < fvx; x++) {
                long vf = NODE(x, y, z, fvx, fvy);
                if (!fine->vact[vf]) continue;
                int X0 = x / r, Y0 = y / r, Z0 = z / r;
                int ox = x - r * X0, oy = y - r * Y0, oz = z - r * Z0;
                double s[3] = {0, 0, 0};
                for (int i = 0; i < 8; i++) {
                    int a = i % 2, b = i / 2 % 2, cc = i / 4;
                    double wx = a ? ox : r - ox, wy = b ? oy : r - oy, wz = cc ? oz : r - oz;
                    if (wx == 0 || wy == 0 || wz == 0) continue;
                    long vc = NODE(X0 + a, Y0 + b, Z0 + cc, cvx, cvy);
                    double w = wx * wy * wz / (double)(r * r * r);
                    for (int c = 0; c < 3; c++) s[c] += w * uc[c * nvc + vc];
                }
                for (int c = 0; c < 3; c++) uf[c * nvf + vf] += s[c];
            }
}

void or_st_cheby(const or_level* L, const double* u, const double* f, double* unew, double* d, int k) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
    double ca, cb;
    or_cheby_coef(L->lmax, k, &ca, &cb);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < vz; z++)
        for (int y = 0; y < vy; y++)
            for (int x = 0; x < vx; x++) {
                long v = NODE(x, y, z, vx, vy);
                double nu[3] = {0, 0, 0}, dn[3] = {0, 0, 0};
                if (L->vact[v]) {
                    double Au[3], S[9], Si[9], rr[3];
                    st_node_sum(L, u, x, y, z, 0, Au);
                    for (int i = 0; i < 9; i++) S[i] = L->st[(long)(13 * 9 + i) * nv + v];
                    inv3(S, Si);
                    for (int c = 0; c < 3; c++) rr[c] = f[c * nv + v] - Au[c];
                    for (int c = 0; c < 3; c++) {
                        double zc = Si[c * 3] * rr[0] + Si[c * 3 + 1] * rr[1] + Si[c * 3 + 2] * rr[2];
                        dn[c] = (k == 0 ? 0.0 : ca * d[c * nv + v]) + cb * zc;
                        nu[c] = u[c * nv + v] + dn[c];
                    }
                }
                for (int c = 0; c < 3; c++) { unew[c * nv + v] = nu[c]; d[c * nv + v] = dn[c]; }
            }
}

/* largest eigenvalue of D^-1 A by power steps (D^-1 A v = v - jacobi(v; f = 0, omega = 1)) */
double or_lambda_max(or_level* L, int is_fine, const double* KE, uint64_t seed, int iters, double* work) {
    /* lambda_max(D^-1 A) by `iters` Lanczos steps in the A inner product, in which M = D^-1 A is
     * self-adjoint (no re-orthogonalisation: only the extreme Ritz value is used).  r = f - A v with
     * f = 0 gives -A v; one Jacobi step from u = 0 (omega = 1) gives D^-1 r = -M v.  Step j, with
     * v_j and r_j = -A v_j:  w = -D^-1 r_j;  alpha_j = r_j . D^-1 r_j;  w -= alpha_j v_j + beta_{j-1} v_{j-1};
     * beta_j = |w|_A;  v_{j+1} = w / beta_j.  Supported rows drop out (r = f = 0 there).
     * work: 6 n doubles */
    long nv = (long)(L->nx + 1) * (L->ny + 1) * (L->nz + 1), n = 3 * nv;
    double *vp = work, *v = work + n, *r = work + 2 * n, *w = work + 3 * n, *r2 = work + 4 * n, *zero = work + 5 * n;
    double alpha[64], beta[64];
    if (iters > 64) iters = 64;
    memset(zero, 0, sizeof(double) * n);
    memset(vp, 0, sizeof(double) * n);
    or_rng_uniform(seed, n, v);
    if (is_fine) or_fine_residual(L, KE, v, zero, r);
    else or_st_residual(L, v, zero, r);
    double an = sqrt(fmax(-or_dot(n, v, r), 1e-300));
    for (long i = 0; i < n; i++) { v[i] /= an; r[i] /= an; }
    int k = 0;
    for (int it = 0; it < iters; it++) {
        memset(w, 0, sizeof(double) * n);
        if (is_fine) or_fine_jacobi(L, KE, w, r, 1.0, L->r);
        else or_st_jacobi(L, w, r, 1.0, L->r);
        const double a = or_dot(n, r, w);
        const double bp = it > 0 ? beta[it - 1] : 0.0;
        for (long i = 0; i < n; i++) w[i] = -w[i] - a * v[i] - bp * vp[i];
        if (is_fine) or_fine_residual(L, KE, w, zero, r2);
        else or_st_residual(L, w, zero, r2);
        const double b = sqrt(fmax(-or_dot(n, w, r2), 1e-300));
        alpha[it] = a;
        beta[it] = b;
        k = it + 1;
        for (long i = 0; i < n; i++) { vp[i] = v[i]; v[i] = w[i] / b; r[i] = r2[i] / b; }
    }
    return or_tridiag_max_eig(k, alpha, beta);
}

/* ------------------------------------------------------------------------ */
/* Galerkin coarse stencils                                                 */
/* ------------------------------------------------------------------------ */
#define DIRICHLET_DIAGONAL_WEIGHT 1e6

/* restrict_stencil_nondyadic_OTFA_{NS,WS}_kernel (grid/Grid.cu:296-506) and
 * restrict_stencil_dyadic_OTFA_kernel (grid/Grid.cu:181-274) restated per
 * coarse cell: A_c = sum_e P_e^T (rho_e^p KE) P_e, where P_e interpolates the
 * 8 corners of the coarse cell to element e's 8 nodes.  With supports, rows and
 * columns of fixed fine nodes are dropped and each (element, fixed node) pair
 * adds DIRICHLET_DIAGONAL_WEIGHT * P^T P on the diagonal (grid/Grid.cu:480-488). */
void or_galerkin_from_elements(const or_level* fine, or_level* coarse, const double* KE, int with_support) {
    int r = coarse->ratio;
    int nx = fine->nx, ny = fine->ny, nz = fine->nz, fvx = nx + 1, fvy = ny + 1;
    int cx = coarse->nx, cy = coarse->ny, cz = coarse->nz, cvx = cx + 1, cvy = cy + 1, cvz = cz + 1;
    long nvc = (long)cvx * cvy * cvz;
    memset(coarse->st, 0, sizeof(double) * 243 * nvc);
    /* cell loop coloured by parity so that no two threads scatter into the same coarse node */
    for (int col = 0; col < 8; col++) {
#pragma omp parallel for collapse(2)
        for (int Z = (col >> 2) & 1; Z < cz; Z += 2)
            for (int Y = (col >> 1) & 1; Y < cy; Y += 2)
                for (int X = col & 1; X < cx; X += 2) {
                    if (!coarse->eact[X + (long)cx * (Y + (long)cy * Z)]) continue;
                    double M[24][24];
                    memset(M, 0, sizeof(M));
                    for (int c = 0; c < r; c++)
                        for (int b = 0; b < r; b++)
                            for (int a = 0; a < r; a++) {
                                int ex = r * X + a, ey = r * Y + b, ez = r * Z + c;
                                if (ex >= nx || ey >= ny || ez >= nz) continue;
                                long e = ex + (long)nx * (ey + (long)ny * ez);
                                if (!fine->eact[e]) continue;
                                double pen = fine->w[e];
                                double P[8][8];
                                int fixed[8];
                                for (int j = 0; j < 8; j++) {
                                    int o[3] = {a + j % 2, b + j / 2 % 2, c + j / 4};
                                    for (int m = 0; m < 8; m++) {
                                        int mm[3] = {m % 2, m / 2 % 2, m / 4};
                                        double w = 1;
                                        for (int t = 0; t < 3; t++) w *= (double)(r - abs(o[t] - r * mm[t])) / r;
                                        P[j][m] = w;
                                    }
                                    fixed[j] = with_support && fine->vfix &&
                                               fine->vfix[NODE(ex + j % 2, ey + j / 2 % 2, ez + j / 4, fvx, fvy)];
                                }
                                /* T = Ktilde_e P  (24 x 24 over (node j,row) x (corner n, col)) */
                                double T[24][24];
                                for (int j = 0; j < 8; j++)
                                    for (int row = 0; row < 3; row++)
                                        for (int n = 0; n < 8; n++)
                                            for (int cl = 0; cl < 3; cl++) {
                                                double acc = 0;
                                                for (int k = 0; k < 8; k++) {
                                                    double kk;
                                                    if (fixed[j] || fixed[k])
                                                        kk = (j == k && row == cl) ? DIRICHLET_DIAGONAL_WEIGHT : 0.0;
                                                    else
                                                        kk = pen * KE[(3 * j + row) * 24 + 3 * k + cl];
                                                    acc += kk * P[k][n];
                                                }
                                                T[3 * j + row][3 * n + cl] = acc;
                                            }
                                for (int m = 0; m < 8; m++)
                                    for (int row = 0; row < 3; row++)
                                        for (int q = 0; q < 24; q++) {
                                            double acc = 0;
                                            for (int j = 0; j < 8; j++) acc += P[j][m] * T[3 * j + row][q];
                                            M[3 * m + row][q] += acc;
                                        }
                            }
                    for (int m = 0; m < 8; m++) {
                        long vc = NODE(X + m % 2, Y + m / 2 % 2, Z + m / 4, cvx, cvy);
                        for (int n = 0; n < 8; n++) {
                            int d[3] = {n % 2 - m % 2, n / 2 % 2 - m / 2 % 2, n / 4 - m / 4};
                            int k = (d[0] + 1) + 3 * (d[1] + 1) + 9 * (d[2] + 1);
                            for (int row = 0; row < 3; row++)
                                for (int cl = 0; cl < 3; cl++)
                                    coarse->st[(long)(k * 9 + row * 3 + cl) * nvc + vc] += M[3 * m + row][3 * n + cl];
                        }
                    }
                }
    }
}

/* restrict_stencil_dyadic_kernel (grid/Grid.cu:120-177): A_c = P^T A_f P with
 * dyadic weights 1, 1/2, 1/4, 1/8 */
void or_galerkin_from_stencil(const or_level* fine, or_level* coarse) {
    int fvx = fine->nx + 1, fvy = fine->ny + 1, fvz = fine->nz + 1;
    int cvx = coarse->nx + 1, cvy = coarse->ny + 1, cvz = coarse->nz + 1;
    long nvf = (long)fvx * fvy * fvz, nvc = (long)cvx * cvy * cvz;
    static const double w[4] = {1.0, 0.5, 0.25, 0.125};
#pragma omp parallel for collapse(2)
    for (int Z = 0; Z < cvz; Z++)
        for (int Y = 0; Y < cvy; Y++)
            for (int X = 0; X < cvx; X++) {
                long vc = NODE(X, Y, Z, cvx, cvy);
                double acc[243];
                memset(acc, 0, sizeof(acc));
                if (coarse->vact[vc]) {
                    for (int i = 0; i < 27; i++) {
                        int dx = i % 3 - 1, dy = i / 3 % 3 - 1, dz = i / 9 - 1;
                        int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
                        if (x < 0 || y < 0 || z < 0 || x >= fvx || y >= fvy || z >= fvz) continue;
                        long vn = NODE(x, y, z, fvx, fvy);
                        if (!fine->vact[vn]) continue;
                        double wi = w[abs(dx) + abs(dy) + abs(dz)];
                        for (int j = 0; j < 27; j++) {
                            int mx = x + j % 3 - 1, my = y + j / 3 % 3 - 1, mz = z + j / 9 - 1;
                            if (mx < 0 || my < 0 || mz < 0 || mx >= fvx || my >= fvy || mz >= fvz) continue;
                            if (!fine->vact[NODE(mx, my, mz, fvx, fvy)]) continue;
                            for (int s = 0; s < 27; s++) {
                                int sx = 2 * (X + s % 3 - 1), sy = 2 * (Y + s / 3 % 3 - 1), sz = 2 * (Z + s / 9 - 1);
                                int ax = abs(sx - mx), ay = abs(sy - my), az = abs(sz - mz);
                                if (ax >= 2 || ay >= 2 || az >= 2) continue;
                                double ws = w[ax + ay + az] * wi;
                                for (int rc = 0; rc < 9; rc++)
                                    acc[s * 9 + rc] += ws * fine->st[(long)(j * 9 + rc) * nvf + vn];
                            }
                        }
                    }
                }
                for (int q = 0; q < 243; q++) coarse->st[(long)q * nvc + vc] = acc[q];
            }
}

/* ------------------------------------------------------------------------ */
/* coarsest level: dense (pseudo-)inverse                                   */
/* Grid::buildCoarsestSystem / Grid::solve_fem_host (grid/Grid.cpp:1884-2043)*/
/* use Eigen::BDCSVD::solve (minimum-norm least squares).  Restated as the   */
/* exact inverse for supported structures and, without supports, as         */
/* (A + a R R^T)^-1 - R R^T / a with R the orthonormal rigid modes, which is */
/* the pseudo-inverse whenever the null space is exactly the rigid modes.    */
/* ------------------------------------------------------------------------ */
static int chol_inverse(int n, double* A) {
    /* in-place lower Cholesky then inverse via L^-T L^-1 */
    for (int j = 0; j < n; j++) {
        double d = A[(long)j * n + j];
        for (int k = 0; k < j; k++) d -= A[(long)j * n + k] * A[(long)j * n + k];
        if (!(d > 0)) return -1;
        d = sqrt(d);
        A[(long)j * n + j] = d;
#pragma omp parallel for
        for (int i = j + 1; i < n; i++) {
            double s = A[(long)i * n + j];
            for (int k = 0; k < j; k++) s -= A[(long)i * n + k] * A[(long)j * n + k];
            A[(long)i * n + j] = s / d;
        }
    }
    /* Linv (lower) */
    double* Li = (double*)calloc((size_t)n * n, sizeof(double));
#pragma omp parallel for
    for (int c = 0; c < n; c++) {
        Li[(long)c * n + c] = 1.0 / A[(long)c * n + c];
        for (int i = c + 1; i < n; i++) {
            double s = 0;
            for (int k = c; k < i; k++) s -= A[(long)i * n + k] * Li[(long)k * n + c];
            Li[(long)i * n + c] = s / A[(long)i * n + i];
        }
    }
    /* Ainv = Li^T Li */
#pragma omp parallel for
    for (int i = 0; i < n; i++)
        for (int j = 0; j <= i; j++) {
            double s = 0;
            for (int k = i; k < n; k++) s += Li[(long)k * n + i] * Li[(long)k * n + j];
            A[(long)i * n + j] = s;
            A[(long)j * n + i] = s;
        }
    free(Li);
    return 0;
}

int or_coarsest_setup(or_level* L, int no_support) {
    int vx = L->nx + 1, vy = L->ny + 1, vz = L->nz + 1;
    long nv = (long)vx * vy * vz;
    int na = 0;
    for (long v = 0; v < nv; v++)
        if (L->vact[v]) L->aidx[na++] = (int)v;
    L->na = na;
    int n = 3 * na;
    int* rowof = (int*)malloc(sizeof(int) * nv);
    for (long v = 0; v < nv; v++) rowof[v] = -1;
    for (int i = 0; i < na; i++) rowof[L->aidx[i]] = i;
    double* A = L->ainv;
    memset(A, 0, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < na; i++) {
        int v = L->aidx[i];
        int x = v % vx, y = v / vx % vy, z = v / (vx * vy);
        for (int k = 0; k < 27; k++) {
            int jx = x + k % 3 - 1, jy = y + k / 3 % 3 - 1, jz = z + k / 9 - 1;
            if (jx < 0 || jy < 0 || jz < 0 || jx >= vx || jy >= vy || jz >= vz) continue;
            int j = rowof[NODE(jx, jy, jz, vx, vy)];
            if (j < 0) continue;
            for (int row = 0; row < 3; row++)
                for (int col = 0; col < 3; col++)
                    A[(long)(3 * i + row) * n + 3 * j + col] = L->st[(long)(k * 9 + row * 3 + col) * nv + v];
        }
    }
    double* R = NULL;
    double alpha = 0;
    if (no_support) {
        R = (double*)calloc((size_t)6 * n, sizeof(double));
        for (int i = 0; i < na; i++) {
            int v = L->aidx[i];
            double p[3] = {v % vx, v / vx % vy, v / (vx * vy)};
            for (int t = 0; t < 3; t++) R[(long)t * n + 3 * i + t] = 1.0;
            /* rotations: column k of [p]x */
            double ph[3][3] = {{0, -p[2], p[1]}, {p[2], 0, -p[0]}, {-p[1], p[0], 0}};
            for (int k = 0; k < 3; k++)
                for (int t = 0; t < 3; t++) R[(long)(3 + k) * n + 3 * i + t] = ph[t][k];
        }
        for (int a = 0; a < 6; a++) {
            for (int b = 0; b < a; b++) {
                double d = 0;
                for (int q = 0; q < n; q++) d += R[(long)a * n + q] * R[(long)b * n + q];
                for (int q = 0; q < n; q++) R[(long)a * n + q] -= d * R[(long)b * n + q];
            }
            double nn = 0;
            for (int q = 0; q < n; q++) nn += R[(long)a * n + q] * R[(long)a * n + q];
            nn = sqrt(nn);
            for (int q = 0; q < n; q++) R[(long)a * n + q] /= nn;
        }
        for (int q = 0; q < n; q++) alpha += A[(long)q * n + q];
        alpha /= n;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double s = 0;
                for (int a = 0; a < 6; a++) s += R[(long)a * n + i] * R[(long)a * n + j];
                A[(long)i * n + j] += alpha * s;
            }
    }
    int rc = chol_inverse(n, A);
    if (no_support && rc == 0) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double s = 0;
                for (int a = 0; a < 6; a++) s += R[(long)a * n + i] * R[(long)a * n + j];
                A[(long)i * n + j] -= s / alpha;
            }
    }
    free(R);
    free(rowof);
    return rc;
}

void or_coarsest_solve(const or_level* L) {
    long nv = (long)(L->nx + 1) * (L->ny + 1) * (L->nz + 1);
    int n = 3 * L->na;
    double* fa = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
    for (int i = 0; i < L->na; i++)
        for (int c = 0; c < 3; c++) fa[3 * i + c] = L->f[c * nv + L->aidx[i]];
    memset(L->u, 0, sizeof(double) * 3 * nv);
#pragma omp parallel for
    for (int i = 0; i < n; i++) {
        double s = 0;
        for (int j = 0; j < n; j++) s += L->ainv[(long)i * n + j] * fa[j];
        L->u[(i % 3) * nv + L->aidx[i / 3]] = s;
    }
    free(fa);
}

/* ------------------------------------------------------------------------ */
/* V-cycle (HierarchyGrid::v_cycle, grid/Grid.cpp:1068-1113)                */
/* ------------------------------------------------------------------------ */
double or_dot(long n, const double* a, const double* b) {
    double s = 0;
#pragma omp parallel for reduction(+ : s)
    for (long i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

static long lvl_nv(const or_level* L) { return (long)(L->nx + 1) * (L->ny + 1) * (L->nz + 1); }

static void smooth(or_level* L, int is_fine, const double* KE, int smoother, int backward, double omega) {
    if (smoother == OR_SMOOTH_CHEBY) {
        /* one step of degree 1 (callers use smooth_n for higher degree) */
        double* tmp = L->r;
        if (is_fine) or_fine_cheby(L, KE, L->u, L->f, tmp, L->d, 0);
        else or_st_cheby(L, L->u, L->f, tmp, L->d, 0);
        memcpy(L->u, tmp, sizeof(double) * 3 * lvl_nv(L));
    } else if (smoother == OR_SMOOTH_JACOBI) {
        double* tmp = L->r; /* r is free scratch while smoothing */
        if (is_fine) or_fine_jacobi(L, KE, L->u, L->f, omega, tmp);
        else or_st_jacobi(L, L->u, L->f, omega, tmp);
    } else {
        if (is_fine) or_fine_gs(L, KE, L->u, L->f, backward);
        else or_st_gs(L, L->u, L->f, backward);
    }
}

static void smooth_n(or_level* L, int is_fine, const double* KE, int smoother, int n, int backward, double omega) {
    if (smoother != OR_SMOOTH_CHEBY) {
        for (int s = 0; s < n; s++) smooth(L, is_fine, KE, smoother, backward, omega);
        return;
    }
    long nn = 3 * lvl_nv(L);
    for (int s = 0; s < n; s++) {
        double* src = (s % 2 == 0) ? L->u : L->r;
        double* dst = (s % 2 == 0) ? L->r : L->u;
        if (is_fine) or_fine_cheby(L, KE, src, L->f, dst, L->d, s);
        else or_st_cheby(L, src, L->f, dst, L->d, s);
    }
    if (n % 2 == 1) memcpy(L->u, L->r, sizeof(double) * nn);
}

double or_vcycle(or_level* lv, int nlev, const double* KE, int smoother, int npre, int npost, double omega,
                 int precond_mode) {
    for (int i = 0; i < nlev; i++) {
        if (i > 0) {
            if (i == 1) or_fine_residual(&lv[0], KE, lv[0].u, lv[0].f, lv[0].r);
            else or_st_residual(&lv[i - 1], lv[i - 1].u, lv[i - 1].f, lv[i - 1].r);
            or_restrict(&lv[i - 1], &lv[i], lv[i - 1].r, lv[i].f);
            memset(lv[i].u, 0, sizeof(double) * 3 * lvl_nv(&lv[i]));
        }
        if (i < nlev - 1) {
            smooth_n(&lv[i], i == 0, KE, smoother, npre, 0, omega);
        } else {
            or_coarsest_solve(&lv[i]);
        }
    }
    for (int i = nlev - 2; i >= 0; i--) {
        or_prolong_add(&lv[i], &lv[i + 1], lv[i + 1].u, lv[i].u);
        smooth_n(&lv[i], i == 0, KE, smoother, npost, smoother == OR_SMOOTH_SGS, omega);
    }
    if (precond_mode) return 0;
    or_fine_residual(&lv[0], KE, lv[0].u, lv[0].f, lv[0].r);
    long n = 3 * lvl_nv(&lv[0]);
    return sqrt(or_dot(n, lv[0].r, lv[0].r)) / sqrt(or_dot(n, lv[0].f, lv[0].f));
}

/* MG-preconditioned flexible CG (not in the reference; the plain FP64 method
 * every form is judged against).  The operator is K with identity rows on
 * fixed nodes (applyK_OTFA_kernel semantics). */
int or_pcg(or_level* lv, int nlev, const double* KE, int smoother, int npre, int npost, double omega, double* x,
           const double* b, double tol, int maxit, double* relres_out, double* work) {
    long nv = lvl_nv(&lv[0]);
    long n = 3 * nv;
    double *r = work, *z = work + n, *p = work + 2 * n, *q = work + 3 * n, *rold = work + 4 * n;
    or_fine_applyK(&lv[0], KE, x, q);
    for (long i = 0; i < n; i++) r[i] = lv[0].vact[i % nv] ? b[i] - q[i] : 0.0;
    double bn = sqrt(or_dot(n, b, b));
    if (bn == 0) bn = 1;
    double rel = sqrt(or_dot(n, r, r)) / bn;
    int it = 0;
    double rz = 0;
    while (rel > tol && it < maxit) {
        memcpy(lv[0].f, r, sizeof(double) * n);
        memset(lv[0].u, 0, sizeof(double) * n);
        or_vcycle(lv, nlev, KE, smoother, npre, npost, omega, 1);
        memcpy(z, lv[0].u, sizeof(double) * n);
        double rz_new = or_dot(n, r, z);
        if (it == 0) {
            memcpy(p, z, sizeof(double) * n);
        } else {
            double num = rz_new - or_dot(n, rold, z); /* flexible (Polak-Ribiere) beta */
            double beta = num / rz;
            for (long i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        }
        rz = rz_new;
        or_fine_applyK(&lv[0], KE, p, q);
        double alpha = rz / or_dot(n, p, q);
        memcpy(rold, r, sizeof(double) * n);
        for (long i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
        rel = sqrt(or_dot(n, r, r)) / bn;
        it++;
    }
    if (relres_out) *relres_out = rel;
    return it;
}

/* ------------------------------------------------------------------------ */
/* worst-case load                                                          */
/* ------------------------------------------------------------------------ */
static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
/* seeded stand-in for curandGenerateUniformDouble(-1,1) (culib/lib.cuh:1312-1348,
 * which the reference seeds with time(nullptr)); element i depends only on (seed, i) */
void or_rng_uniform(uint64_t seed, long n, double* out) {
    for (long i = 0; i < n; i++) {
        uint64_t h = splitmix64(seed * 0x632BE59BD9B4E019ull + (uint64_t)i);
        out[i] = (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
}

/* setLoadNodes (optimization/projection.cpp:129-269): rigid modes on the load
 * set, minus their tangential part when the load direction is constrained,
 * Gram-Schmidt orthonormalised, degenerate modes dropped.  Returns the count. */
int or_rigid_basis(int nload, const double* pos, const double* normal, int constrain_dir, double* Rd) {
    long n = 3L * nload;
    for (int k = 0; k < 6; k++) memset(Rd + k * n, 0, sizeof(double) * n);
    for (int i = 0; i < nload; i++) {
        const double* p = pos + 3 * i;
        double ph[3][3] = {{0, -p[2], p[1]}, {p[2], 0, -p[0]}, {-p[1], p[0], 0}};
        for (int t = 0; t < 3; t++) Rd[t * n + 3 * i + t] = 1.0;
        for (int k = 0; k < 3; k++)
            for (int t = 0; t < 3; t++) Rd[(3 + k) * n + 3 * i + t] = ph[t][k];
    }
    if (constrain_dir) {
        /* R -= N^T N R keeps only the normal component at each node */
        for (int k = 0; k < 6; k++)
            for (int i = 0; i < nload; i++) {
                const double* nn = normal + 3 * i;
                double* v = Rd + k * n + 3 * i;
                double d = v[0] * nn[0] + v[1] * nn[1] + v[2] * nn[2];
                for (int t = 0; t < 3; t++) v[t] = d * nn[t];
            }
    }
    int valid = 0;
    int invalid[6] = {0};
    for (int k = 0; k < 6; k++) {
        double* ck = Rd + k * n;
        double oldres = sqrt(or_dot(n, ck, ck));
        for (int j = 0; j < k; j++) {
            if (invalid[j]) continue;
            double w = or_dot(n, ck, Rd + j * n);
            for (long q = 0; q < n; q++) ck[q] -= w * Rd[j * n + q];
        }
        double res = sqrt(or_dot(n, ck, ck));
        if (res / oldres < 1e-6 || oldres < 1e-6) invalid[k] = 1;
        for (long q = 0; q < n; q++) ck[q] /= res;
    }
    for (int k = 0; k < 6; k++)
        if (!invalid[k]) {
            if (valid != k) memcpy(Rd + valid * n, Rd + k * n, sizeof(double) * n);
            valid++;
        }
    return valid;
}

/* forceProject (optimization/projection.cpp:289-360, projection.cu:165-231):
 * gather the load nodes, remove the tangential component (constrained
 * direction) and/or the rigid component (no supports), zero every other node. */
void or_force_project(long nv, int nload, const int* load_nodes, const double* normal, int constrain_dir, int nrig,
                      const double* Rd, double* f) {
    long n = 3L * nload;
    double* fs = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
    for (int i = 0; i < nload; i++)
        for (int c = 0; c < 3; c++) fs[3 * i + c] = f[c * nv + load_nodes[i]];
    double wr[6];
    for (int k = 0; k < nrig; k++) wr[k] = or_dot(n, Rd + k * n, fs);
    double* out = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
    memcpy(out, fs, sizeof(double) * n);
    if (constrain_dir) {
        for (int i = 0; i < nload; i++) {
            const double* nn = normal + 3 * i;
            double d = fs[3 * i] * nn[0] + fs[3 * i + 1] * nn[1] + fs[3 * i + 2] * nn[2];
            for (int t = 0; t < 3; t++) out[3 * i + t] = d * nn[t];
        }
    }
    for (int k = 0; k < nrig; k++)
        for (long q = 0; q < n; q++) out[q] -= wr[k] * Rd[k * n + q];
    memset(f, 0, sizeof(double) * 3 * nv);
    for (int i = 0; i < nload; i++)
        for (int c = 0; c < 3; c++) f[c * nv + load_nodes[i]] = out[3 * i + c];
    free(fs);
    free(out);
}

/* setNodes (optimization/projection.cpp:46-127): orthonormal rigid modes over all active nodes */
void or_rigid_nodes(const or_level* L, double* Ru) {
    int vx = L->nx + 1, vy = L->ny + 1;
    long nv = lvl_nv(L), n = 3 * nv;
    memset(Ru, 0, sizeof(double) * 6 * n);
    for (long v = 0; v < nv; v++) {
        if (!L->vact[v]) continue;
        double p[3] = {(double)(v % vx), (double)(v / vx % vy), (double)(v / ((long)vx * vy))};
        double ph[3][3] = {{0, -p[2], p[1]}, {p[2], 0, -p[0]}, {-p[1], p[0], 0}};
        for (int t = 0; t < 3; t++) Ru[t * n + t * nv + v] = 1.0;
        for (int k = 0; k < 3; k++)
            for (int t = 0; t < 3; t++) Ru[(3 + k) * n + t * nv + v] = ph[t][k];
    }
    for (int a = 0; a < 6; a++) {
        for (int b = 0; b < a; b++) {
            double d = or_dot(n, Ru + a * n, Ru + b * n);
            for (long q = 0; q < n; q++) Ru[a * n + q] -= d * Ru[b * n + q];
        }
        double nn = sqrt(or_dot(n, Ru + a * n, Ru + a * n));
        for (long q = 0; q < n; q++) Ru[a * n + q] /= nn;
    }
}

/* displacementProject (optimization/projection.cpp:374-392) */
void or_displacement_project(long nv, const double* Ru, double* u) {
    long n = 3 * nv;
    for (int k = 0; k < 6; k++) {
        double s = or_dot(n, u, Ru + k * n);
        for (long q = 0; q < n; q++) u[q] -= s * Ru[k * n + q];
    }
}

/* modifiedPM (optimization/optimization.cpp:123-261): power iteration on
 * P K^-1 P with one warm-started V-cycle (GS 1/1) per step. */
double or_modified_pm(or_level* lv, int nlev, const double* KE, int nload, const int* load_nodes,
                      const double* normal, int constrain_dir, int nrig, const double* Rd, const double* Ru,
                      uint64_t seed, int maxit, int* iters_out, double* fs_old) {
    long nv = lvl_nv(&lv[0]), n = 3 * nv, nl = 3L * nload;
    double* f = lv[0].f;
    or_rng_uniform(seed, n, f);
    or_force_project(nv, nload, load_nodes, normal, constrain_dir, nrig, Rd, f);
    double fn = sqrt(or_dot(n, f, f));
    for (long q = 0; q < n; q++) f[q] /= fn;
    memset(lv[0].u, 0, sizeof(double) * n);
    for (int i = 0; i < nload; i++)
        for (int c = 0; c < 3; c++) fs_old[3 * i + c] = f[c * nv + load_nodes[i]];
    double fch = 1, rel = 1;
    int itn = 0;
    while (itn++ < maxit && (fch > 1e-4 || rel > 1e-2)) {
        rel = or_vcycle(lv, nlev, KE, OR_SMOOTH_GS, 1, 1, 0, 0);
        if (Ru) or_displacement_project(nv, Ru, lv[0].u);
        if (rel > 1e4 || rel != rel) { if (iters_out) *iters_out = -itn; return NAN; }
        memcpy(f, lv[0].u, sizeof(double) * n);
        or_force_project(nv, nload, load_nodes, normal, constrain_dir, nrig, Rd, f);
        fn = sqrt(or_dot(n, f, f));
        for (long q = 0; q < n; q++) f[q] /= fn;
        double num = 0, den = 0;
        for (int i = 0; i < nload; i++)
            for (int c = 0; c < 3; c++) {
                double a = f[c * nv + load_nodes[i]], b = fs_old[3 * i + c];
                num += (a - b) * (a - b);
                den += b * b;
                fs_old[3 * i + c] = a;
            }
        fch = sqrt(num) / sqrt(den);
    }
    if (iters_out) *iters_out = itn - 1;
    (void)nl;
    return or_dot(n, f, lv[0].u);
}

/* largest eigenvalue of the symmetric tridiagonal (alpha, beta) by Sturm bisection */
double or_tridiag_max_eig(int k, const double* alpha, const double* beta) {
    double lo = alpha[0], hi = alpha[0];
    for (int i = 0; i < k; i++) {
        double r = (i > 0 ? fabs(beta[i - 1]) : 0) + (i < k - 1 ? fabs(beta[i]) : 0);
        if (alpha[i] - r < lo) lo = alpha[i] - r;
        if (alpha[i] + r > hi) hi = alpha[i] + r;
    }
    for (int it = 0; it < 200; it++) {
        double mid = 0.5 * (lo + hi);
        if (mid == lo || mid == hi) break;
        /* count eigenvalues < mid */
        int cnt = 0;
        double d = 1;
        for (int i = 0; i < k; i++) {
            double b2 = i > 0 ? beta[i - 1] * beta[i - 1] : 0;
            d = alpha[i] - mid - (i > 0 ? b2 / d : 0);
            if (d == 0) d = -1e-300;
            if (d < 0) cnt++;
        }
        if (cnt == k) hi = mid; else lo = mid;
    }
    return 0.5 * (lo + hi);
}

/* Lanczos on A = P S K^-1 S^T P over the load DOFs, with FP64 full
 * re-orthogonalisation and MG-PCG inner solves.  Not in the reference: the
 * Krylov replacement for the modified power method. */
int or_lanczos(or_level* lv, int nlev, const double* KE, int smoother, int npre, int npost, double omega, int nload,
               const int* load_nodes, const double* normal, int constrain_dir, int nrig, const double* Rd,
               uint64_t seed, int k, double inner_tol, int inner_maxit, double* lambda_out, double* ritz_f,
               double* work) {
    long nv = lvl_nv(&lv[0]), n = 3 * nv, nl = 3L * nload;
    double* Q = work;                      /* (k+1) x nl */
    double* full = work + (long)(k + 1) * nl; /* n */
    double* x = full + n;                  /* n */
    double* pcgw = x + n;                  /* 6n */
    double alpha[64], beta[64];
    /* start vector: seeded uniform, projected, unit norm */
    or_rng_uniform(seed, n, full);
    or_force_project(nv, nload, load_nodes, normal, constrain_dir, nrig, Rd, full);
    for (int i = 0; i < nload; i++)
        for (int c = 0; c < 3; c++) Q[3 * i + c] = full[c * nv + load_nodes[i]];
    double qn = sqrt(or_dot(nl, Q, Q));
    for (long q = 0; q < nl; q++) Q[q] /= qn;
    int steps = 0, total_inner = 0;
    for (int j = 0; j < k; j++) {
        double* qj = Q + (long)j * nl;
        double* w = Q + (long)(j + 1) * nl;
        memset(full, 0, sizeof(double) * n);
        for (int i = 0; i < nload; i++)
            for (int c = 0; c < 3; c++) full[c * nv + load_nodes[i]] = qj[3 * i + c];
        memset(x, 0, sizeof(double) * n);
        double rr;
        total_inner += or_pcg(lv, nlev, KE, smoother, npre, npost, omega, x, full, inner_tol, inner_maxit, &rr, pcgw);
        or_force_project(nv, nload, load_nodes, normal, constrain_dir, nrig, Rd, x);
        for (int i = 0; i < nload; i++)
            for (int c = 0; c < 3; c++) w[3 * i + c] = x[c * nv + load_nodes[i]];
        alpha[j] = or_dot(nl, w, qj);
        for (int pass = 0; pass < 2; pass++)
            for (int i = 0; i <= j; i++) {
                double h = or_dot(nl, w, Q + (long)i * nl);
                for (long q = 0; q < nl; q++) w[q] -= h * Q[(long)i * nl + q];
            }
        beta[j] = sqrt(or_dot(nl, w, w));
        steps = j + 1;
        if (beta[j] < 1e-14 * fabs(alpha[0])) break;
        for (long q = 0; q < nl; q++) w[q] /= beta[j];
    }
    double lam = or_tridiag_max_eig(steps, alpha, beta);
    *lambda_out = lam;
    if (ritz_f) {
        /* Ritz vector: inverse iteration on T - lam I */
        double y[64], ynew[64];
        for (int i = 0; i < steps; i++) y[i] = 1.0;
        for (int it = 0; it < 3; it++) {
            double shift = lam * (1 + 1e-12) + 1e-300;
            /* solve (T - shift I) ynew = y by the Thomas algorithm */
            double cp[64], dp[64];
            for (int i = 0; i < steps; i++) {
                double a = i > 0 ? beta[i - 1] : 0, b = alpha[i] - shift, c = i < steps - 1 ? beta[i] : 0;
                double den = b - (i > 0 ? a * cp[i - 1] : 0);
                cp[i] = c / den;
                dp[i] = (y[i] - (i > 0 ? a * dp[i - 1] : 0)) / den;
            }
            for (int i = steps - 1; i >= 0; i--) ynew[i] = dp[i] - (i < steps - 1 ? cp[i] * ynew[i + 1] : 0);
            double s = 0;
            for (int i = 0; i < steps; i++) s += ynew[i] * ynew[i];
            s = sqrt(s);
            for (int i = 0; i < steps; i++) y[i] = ynew[i] / s;
        }
        memset(ritz_f, 0, sizeof(double) * n);
        for (int i = 0; i < nload; i++)
            for (int c = 0; c < 3; c++) {
                double s = 0;
                for (int j = 0; j < steps; j++) s += y[j] * Q[(long)j * nl + 3 * i + c];
                ritz_f[c * nv + load_nodes[i]] = s;
            }
    }
    return total_inner;
}

/* ------------------------------------------------------------------------ */
/* sensitivity, filter, OC                                                  */
/* ------------------------------------------------------------------------ */
/* computeSensitivity_kernel (optimization/optimization.cu:44-107):
 * s_e = -p rho^(p-1) u_e^T KE u_e (summed per element in FP64, stored FP32) */
void or_sensitivity(int nx, int ny, int nz, const uint8_t* eact, const float* rho, float p, const double* KE,
                    const double* u, float* sens) {
    int vx = nx + 1, vy = ny + 1;
    long nv = (long)vx * vy * (nz + 1);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                long e = x + (long)nx * (y + (long)ny * z);
                if (!eact[e]) { sens[e] = 0; continue; }
                double ue[24];
                for (int j = 0; j < 8; j++) {
                    long nj = NODE(x + j % 2, y + j / 2 % 2, z + j / 4, vx, vy);
                    for (int c = 0; c < 3; c++) ue[3 * j + c] = u[c * nv + nj];
                }
                double pen = (double)(p * powf(rho[e], p - 1));
                double s = 0;
                for (int i = 0; i < 24; i++) {
                    double kr = 0;
                    for (int j = 0; j < 24; j++) kr += KE[i * 24 + j] * ue[j];
                    s -= ue[i] * kr * pen;
                }
                sens[e] = (float)s;
            }
}

/* filterSensitivity_kernel (grid/Grid.cu:2323-2409): normalised radial filter,
 * w(t) = 1 - 6t^2 + 8t^3 - 3t^4, t = sqrt(r^2/R^2), loop radius int(R + 0.5) */
void or_filter(int nx, int ny, int nz, const uint8_t* eact, float radius, const float* sens, float* out) {
    float R2 = radius * radius;
    int Rl = (int)(radius + 0.5f);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                long e = x + (long)nx * (y + (long)ny * z);
                if (!eact[e]) { out[e] = 0; continue; }
                float wsum = 0;
                double gsum = 0;
                for (int dx = -Rl; dx <= Rl; dx++) {
                    int X = x + dx;
                    if (X < 0 || X >= nx) continue;
                    for (int dy = -Rl; dy <= Rl; dy++) {
                        int Y = y + dy;
                        if (Y < 0 || Y >= ny) continue;
                        for (int dz = -Rl; dz <= Rl; dz++) {
                            int Z = z + dz;
                            if (Z < 0 || Z >= nz) continue;
                            float r2 = (float)(dx * dx + dy * dy + dz * dz);
                            if (r2 > R2) continue;
                            long n = X + (long)nx * (Y + (long)ny * Z);
                            if (!eact[n]) continue;
                            float t = sqrtf(r2 / R2);
                            float t2 = t * t;
                            float w = 1 - 6 * t2 + 8 * t2 * t - 3 * t2 * t2;
                            gsum += w * sens[n];
                            wsum += w;
                        }
                    }
                }
                out[e] = (float)(gsum / wsum);
            }
}

static inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* trySensMultiplier_kernel (optimization/optimization.cu:136-162) */
void or_oc_try(long ne, const uint8_t* eact, const uint8_t* eshell, const float* rho, const float* sens, float lambda,
               float step, float damp, float rhomin, float* out) {
#pragma omp parallel for
    for (long e = 0; e < ne; e++) {
        if (!eact[e]) { out[e] = 0; continue; }
        float g = sens[e];
        if (g > 0) g = 0;
        g = fabsf(g);
        float ro = rho[e];
        float rn = ro * powf(g / lambda, damp);
        rn = clampf(rn, ro - step, ro + step);
        rn = clampf(rn, rhomin, 1.f);
        if (eshell && eshell[e]) rn = 1;
        out[e] = rn;
    }
}

/* updateDensities (optimization/optimization.cu:164-226): bisection on the
 * multiplier in [0, max|s|] until |V - Vgoal| <= 1e-4 or 31 trials; the volume
 * is the FP64 sum of the trial densities over n_count slots. */
float or_oc_update(long ne, const uint8_t* eact, const uint8_t* eshell, float* rho, const float* sens, float vgoal,
                   float step, float damp, float rhomin, long n_count, int* iters_out, float* tmp) {
    float gmax = 0;
    for (long e = 0; e < ne; e++)
        if (eact[e] && fabsf(sens[e]) > gmax) gmax = fabsf(sens[e]);
    float lo = 0, hi = gmax, thr = (lo + hi) / 2;
    float V = 2;
    int itn = 0;
    int trials = 0;
    do {
        thr = (lo + hi) / 2;
        or_oc_try(ne, eact, eshell, rho, sens, thr, step, damp, rhomin, tmp);
        double s = 0;
        for (long e = 0; e < ne; e++)
            if (eact[e]) s += tmp[e];
        V = (float)(s / n_count);
        trials++;
        if (V > vgoal) lo = thr;
        else if (V < vgoal) hi = thr;
    } while (fabsf(V - vgoal) > 1e-4f && itn++ < 30);
    or_oc_try(ne, eact, eshell, rho, sens, thr, step, damp, rhomin, rho);
    if (iters_out) *iters_out = trials;
    return thr;
}
