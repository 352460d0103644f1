// C ABI around four of the reference's own CUDA kernels, compiled unchanged from the reference
// sources for sm_100a against the stubs in oracle/ref_stubs/ (grid/Grid.cu is included below as it
// is, optimization/optimization.cu by oracle/ref_opt_kernels.cu):
//
//   applyK_OTFA_kernel            grid/Grid.cu:2439-2517        f = K(rho) u, fixed rows u
//   computeSensitivity_kernel     optimization/optimization.cu:44-107   s_e = -p rho^(p-1) u_e.KE u_e
//   trySensMultiplier_kernel      optimization/optimization.cu:136-162  one OC trial
//   filterSensitivity_kernel      grid/Grid.cu:2323-2409        radial sensitivity filter
//
// The reference keeps its grids in GS-colour order with per-vertex index tables bound to
// __constant__ pointer arrays (Grid::use_grid, grid/Grid.cu:48-75).  This driver builds those
// tables for a dense element box: vertices and elements are numbered in lexicographic order of
// the active ones (the kernels follow the tables, so any numbering gives the same values), the
// 27-neighbour table gV2V has offset x + 3 y + 9 z around the vertex (centre 13 = the vertex), and
// gV2E[e] is the element whose lowest corner sits at offset (e & 1, e >> 1 & 1, e >> 2) - 1.
// The filter's weight function, a lambda inside Grid::filterSensitivity (grid/Grid.cu:2419-2422),
// is restated as a functor; the element bit array is the reference's LSB-first layout over a cube
// of side max(nx, ny, nz) holding the box at its origin.
//
// Test infrastructure only (pins the oracle and the CUDA path to the reference's kernels).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "Grid.cu"

// launches of the optimization/optimization.cu kernels, compiled in their own translation unit
// (oracle/ref_opt_kernels.cu: that file's extern __constant__ declarations cannot follow the
// definitions of this one) and device-linked with this one
void ref_launch_sensitivity(int nv, float* rho, float* sens);
void ref_launch_oc_try(int nv, const float* rho, float* sens, float thres, float step, float damp, float rhomin,
                       float* newrho);

namespace {

struct RefBox {
    int nx, ny, nz, vx, vy, vz;
    long nvb, neb;  // dense box sizes
    std::vector<int> vid, eid;        // dense -> active id (-1: inactive)
    std::vector<long> vdense, edense;  // active id -> dense
};

RefBox make_box(int nx, int ny, int nz, const uint8_t* eact) {
    RefBox b{nx, ny, nz, nx + 1, ny + 1, nz + 1, (long)(nx + 1) * (ny + 1) * (nz + 1), (long)nx * ny * nz, {}, {}, {}, {}};
    b.eid.assign(b.neb, -1);
    for (long e = 0; e < b.neb; e++)
        if (eact[e]) {
            b.eid[e] = (int)b.edense.size();
            b.edense.push_back(e);
        }
    b.vid.assign(b.nvb, -1);
    for (int z = 0; z < b.vz; z++)
        for (int y = 0; y < b.vy; y++)
            for (int x = 0; x < b.vx; x++) {
                bool act = false;
                for (int i = 0; i < 8 && !act; i++) {
                    const int ex = x - 1 + (i & 1), ey = y - 1 + ((i >> 1) & 1), ez = z - 1 + (i >> 2);
                    if (ex >= 0 && ey >= 0 && ez >= 0 && ex < nx && ey < ny && ez < nz &&
                        eact[ex + (long)nx * (ey + (long)ny * ez)])
                        act = true;
                }
                if (act) {
                    const long v = x + (long)b.vx * (y + (long)b.vy * z);
                    b.vid[v] = (int)b.vdense.size();
                    b.vdense.push_back(v);
                }
            }
    return b;
}

template <typename T>
T* upload(const std::vector<T>& h) {
    T* d = nullptr;
    cudaMalloc(&d, sizeof(T) * (h.size() ? h.size() : 1));
    if (!h.empty()) cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    return d;
}

// device tables of the box bound to the reference's __constant__ pointer arrays; freed by release()
struct Tables {
    std::vector<void*> owned;
    int nv = 0;
    void release() {
        for (void* p : owned) cudaFree(p);
        owned.clear();
    }
    template <typename T>
    T* keep(T* p) {
        owned.push_back(p);
        return p;
    }
};

Tables bind(const RefBox& b, const uint8_t* vfix, const uint8_t* eshell, float p, const double* KE) {
    Tables t;
    const int nva = (int)b.vdense.size();
    t.nv = nva;
    int* v2v[27];
    int* v2e[8];
    std::vector<int> h(nva);
    for (int k = 0; k < 27; k++) {
        const int dx = k % 3 - 1, dy = k / 3 % 3 - 1, dz = k / 9 - 1;
        for (int i = 0; i < nva; i++) {
            const long v = b.vdense[i];
            const int x = (int)(v % b.vx), y = (int)(v / b.vx % b.vy), z = (int)(v / ((long)b.vx * b.vy));
            const int X = x + dx, Y = y + dy, Z = z + dz;
            h[i] = (X >= 0 && Y >= 0 && Z >= 0 && X < b.vx && Y < b.vy && Z < b.vz)
                       ? b.vid[X + (long)b.vx * (Y + (long)b.vy * Z)]
                       : -1;
        }
        v2v[k] = t.keep(upload(h));
    }
    for (int e = 0; e < 8; e++) {
        const int dx = (e & 1) - 1, dy = ((e >> 1) & 1) - 1, dz = (e >> 2) - 1;
        for (int i = 0; i < nva; i++) {
            const long v = b.vdense[i];
            const int x = (int)(v % b.vx), y = (int)(v / b.vx % b.vy), z = (int)(v / ((long)b.vx * b.vy));
            const int X = x + dx, Y = y + dy, Z = z + dz;
            h[i] = (X >= 0 && Y >= 0 && Z >= 0 && X < b.nx && Y < b.ny && Z < b.nz)
                       ? b.eid[X + (long)b.nx * (Y + (long)b.ny * Z)]
                       : -1;
        }
        v2e[e] = t.keep(upload(h));
    }
    std::vector<int> vflag(nva, 0), eflag(b.edense.size(), 0);
    if (vfix)
        for (int i = 0; i < nva; i++)
            if (vfix[b.vdense[i]]) vflag[i] |= grid::Grid::Bitmask::mask_supportnodes;
    if (eshell)
        for (size_t i = 0; i < b.edense.size(); i++)
            if (eshell[b.edense[i]]) eflag[i] |= grid::Grid::Bitmask::mask_shellelement;
    int* dvflag = t.keep(upload(vflag));
    int* deflag = t.keep(upload(eflag));
    cudaMemcpyToSymbol(gV2V, v2v, sizeof(v2v));
    cudaMemcpyToSymbol(gV2E, v2e, sizeof(v2e));
    cudaMemcpyToSymbol(gVflag, &dvflag, sizeof(int*));
    cudaMemcpyToSymbol(gEflag, &deflag, sizeof(int*));
    cudaMemcpyToSymbol(power_penalty, &p, sizeof(float));
    if (KE) cudaMemcpyToSymbol(gTemplateMatrix, KE, sizeof(double) * 576);
    return t;
}

// displacement of the dense box [3][nvb] as the reference's [3][nv] active-vertex vectors
void upload_u(const RefBox& b, const double* u, Tables& t, double* dU[3]) {
    const int nva = (int)b.vdense.size();
    std::vector<double> h(nva);
    for (int c = 0; c < 3; c++) {
        for (int i = 0; i < nva; i++) h[i] = u[c * b.nvb + b.vdense[i]];
        dU[c] = t.keep(upload(h));
    }
    cudaMemcpyToSymbol(gU, dU, sizeof(double*) * 3);
}

std::vector<float> element_values(const RefBox& b, const float* dense) {
    std::vector<float> h(b.edense.size());
    for (size_t i = 0; i < b.edense.size(); i++) h[i] = dense[b.edense[i]];
    return h;
}

// Grid::filterSensitivity's weight (grid/Grid.cu:2419-2422)
struct FilterWeight {
    __device__ float operator()(float r) const {
        const float r2 = r * r;
        return 1 - 6 * r2 + 8 * r2 * r - 3 * r2 * r2;
    }
};

unsigned blocks(int n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int finish() { return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 1; }

}  // namespace

extern "C" __attribute__((visibility("default"))) int ref_apply_k(int nx, int ny, int nz, const uint8_t* eact, const uint8_t* vfix, const float* rho, float p,
                           const double* KE, const double* u, double* f_out) {
    RefBox b = make_box(nx, ny, nz, eact);
    Tables t = bind(b, vfix, nullptr, p, KE);
    double* dU[3];
    upload_u(b, u, t, dU);
    double* dF[3];
    for (int c = 0; c < 3; c++) {
        cudaMalloc(&dF[c], sizeof(double) * t.nv);
        t.keep(dF[c]);
    }
    float* drho = t.keep(upload(element_values(b, rho)));
    devArray_t<double*, 3> ulist{dU[0], dU[1], dU[2]};
    devArray_t<double*, 3> flist{dF[0], dF[1], dF[2]};
    applyK_OTFA_kernel<<<blocks(t.nv, 512), 512>>>(t.nv, ulist, flist, drho);
    int st = finish();
    std::vector<double> h(t.nv);
    std::memset(f_out, 0, sizeof(double) * 3 * b.nvb);
    for (int c = 0; c < 3 && st == 0; c++) {
        cudaMemcpy(h.data(), dF[c], sizeof(double) * t.nv, cudaMemcpyDeviceToHost);
        for (int i = 0; i < t.nv; i++) f_out[c * b.nvb + b.vdense[i]] = h[i];
    }
    t.release();
    return st;
}

extern "C" __attribute__((visibility("default"))) int ref_sensitivity(int nx, int ny, int nz, const uint8_t* eact, const float* rho, float p, const double* KE,
                               const double* u, float* sens_out) {
    RefBox b = make_box(nx, ny, nz, eact);
    Tables t = bind(b, nullptr, nullptr, p, KE);
    double* dU[3];
    upload_u(b, u, t, dU);
    float* drho = t.keep(upload(element_values(b, rho)));
    std::vector<float> zero(b.edense.size(), 0.f);
    float* dsens = t.keep(upload(zero));
    ref_launch_sensitivity(t.nv, drho, dsens);
    int st = finish();
    std::vector<float> h(b.edense.size());
    if (st == 0) cudaMemcpy(h.data(), dsens, sizeof(float) * h.size(), cudaMemcpyDeviceToHost);
    std::memset(sens_out, 0, sizeof(float) * b.neb);
    for (size_t i = 0; i < h.size(); i++) sens_out[b.edense[i]] = h[i];
    t.release();
    return st;
}

extern "C" __attribute__((visibility("default"))) int ref_oc_try(int nx, int ny, int nz, const uint8_t* eact, const uint8_t* eshell, const float* rho,
                          const float* sens, float thres, float step, float damp, float rhomin, float* rho_out) {
    RefBox b = make_box(nx, ny, nz, eact);
    Tables t = bind(b, nullptr, eshell, 3.f, nullptr);
    float* drho = t.keep(upload(element_values(b, rho)));
    float* dsens = t.keep(upload(element_values(b, sens)));
    std::vector<float> init(b.edense.size(), -1.f);
    float* dnew = t.keep(upload(init));
    ref_launch_oc_try(t.nv, drho, dsens, thres, step, damp, rhomin, dnew);
    int st = finish();
    std::vector<float> h(b.edense.size());
    if (st == 0) cudaMemcpy(h.data(), dnew, sizeof(float) * h.size(), cudaMemcpyDeviceToHost);
    std::memset(rho_out, 0, sizeof(float) * b.neb);
    for (size_t i = 0; i < h.size(); i++) rho_out[b.edense[i]] = h[i];
    t.release();
    return st;
}

extern "C" __attribute__((visibility("default"))) int ref_filter(int nx, int ny, int nz, const uint8_t* eact, float radius, const float* sens, float* out) {
    RefBox b = make_box(nx, ny, nz, eact);
    const int R = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
    const long nbits = (long)R * R * R;
    const int nword = (int)((nbits + 31) / 32);
    std::vector<unsigned int> bits(nword, 0u);
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++)
                if (eact[x + (long)nx * (y + (long)ny * z)]) {
                    const long id = x + (long)R * (y + (long)R * z);
                    bits[id / 32] |= 1u << (id % 32);
                }
    std::vector<int> sat(nword + 1, 0);
    for (int w = 0; w < nword; w++) sat[w + 1] = sat[w] + __builtin_popcount(bits[w]);
    Tables t;
    unsigned int* dbits = t.keep(upload(bits));
    int* dsat = t.keep(upload(sat));
    // element ids in bit order over the cube = lexicographic order of the box's active elements
    float* dsens = t.keep(upload(element_values(b, sens)));
    std::vector<float> zero(b.edense.size(), 0.f);
    float* ddst = t.keep(upload(zero));
    gBitSAT<unsigned int> esat(dbits, dsat);
    filterSensitivity_kernel<<<blocks(nword, 512), 512>>>(nword, esat, R, dsens, ddst, radius, FilterWeight{},
                                                          (const int*)nullptr);
    int st = finish();
    std::vector<float> h(b.edense.size());
    if (st == 0) cudaMemcpy(h.data(), ddst, sizeof(float) * h.size(), cudaMemcpyDeviceToHost);
    std::memset(out, 0, sizeof(float) * b.neb);
    for (size_t i = 0; i < h.size(); i++) out[b.edense[i]] = h[i];
    t.release();
    return st;
}
