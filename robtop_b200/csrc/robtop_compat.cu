// robtop_compat.cu — the reference's C++ entry points (robtop_compat.h) on the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "robtop_compat.h"
#include "rt_internal.h"

Parameter params;
grid::HierarchyGrid grids;
gpu_manager_t gpu_manager;

// mem/gpu_manager_t.cu: named device buffers, freed with the manager
// a failed runtime call in the shim ends the calling function with the runtime's message
static void ck_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

// The reference's copies are cudaMemcpy / cudaMemset on the legacy default stream, which its
// kernels share, so a copy always sees the kernels launched before it.  This library's kernels
// run on a non-blocking stream per context, which the legacy stream does not wait for: each
// copy first waits for the device, so that a caller reading a buffer the library just wrote
// (or refilling one it is still reading) sees the same order as with the reference.
void gpu_manager_t::upload_buf(void* dst, const void* src, size_t size) {
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(dst, src, size, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("upload_buf failed");
}
void gpu_manager_t::download_buf(void* host_dst, const void* dev_src, size_t n) {
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(host_dst, dev_src, n, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("download_buf failed");
}
void gpu_manager_t::initMem(void* pdata, size_t len, char value) {
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemset(pdata, value, len) != cudaSuccess)
        throw std::runtime_error("initMem failed");
}
void* gpu_manager_t::add_buf(const std::string& name, size_t size, const void* src) {
    void* p = nullptr;
    if (cudaMalloc(&p, size ? size : 1) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("add_buf: cudaMalloc of " + std::to_string(size) + " bytes failed");
    }
    if (src) upload_buf(p, src, size);
    _bufs.push_back(Buf{name, p, size});
    return p;
}
void* gpu_manager_t::add_buf(size_t size, const void* src) {
    return add_buf("anonymous_" + std::to_string(_anonymous++), size, src);
}
void gpu_manager_t::delete_buf(const std::string& name) {
    for (size_t i = 0; i < _bufs.size(); i++)
        if (_bufs[i].name == name) {
            cudaFree(_bufs[i].p);
            _bufs.erase(_bufs.begin() + i);
            return;
        }
}
void gpu_manager_t::delete_buf(void* pbuf) {
    for (size_t i = 0; i < _bufs.size(); i++)
        if (_bufs[i].p == pbuf) {
            cudaFree(_bufs[i].p);
            _bufs.erase(_bufs.begin() + i);
            return;
        }
}
size_t gpu_manager_t::size(void) {
    size_t s = 0;
    for (const Buf& b : _bufs) s += b.size;
    return s;
}
gpu_manager_t::~gpu_manager_t() {
    // at static destruction the runtime may already be gone
    if (cudaFree(nullptr) == cudaSuccess)
        for (const Buf& b : _bufs) cudaFree(b.p);
}

namespace grid {

void HierarchyGrid::check(int status, const char* what) {
    if (status != RT_OK) {
        std::string msg = std::string(what) + ": " + (_ctx ? rt_last_error(_ctx) : "no context") + " (status " +
                          std::to_string(status) + ")";
        throw std::runtime_error(msg);
    }
}

HierarchyGrid::HierarchyGrid(void) {
    rt_params_default(&_params);
    _params.smoother = RT_SMOOTH_GS;  // the reference's V-cycle smoother
}

HierarchyGrid::~HierarchyGrid() {
    for (auto g : _grids) delete g;
    // the process may already be tearing the CUDA runtime down at static destruction;
    // library handles are released only when the runtime is still usable
    if (_h && cudaFree(nullptr) == cudaSuccess) rt_hier_destroy(_h);
    if (_ctx && cudaFree(nullptr) == cudaSuccess) rt_ctx_destroy(_ctx);
}

void HierarchyGrid::setMode(Mode mode) {
    _mode = mode;
    _params.mode = (int)mode;  // same order as rt_mode
    if (_h) check(rt_hier_set_params(_h, &_params), "setMode");
}

void HierarchyGrid::resetAllResidual(void) {
    for (auto g : _grids) g->reset_residual();
}

// HierarchyGrid::genFromMesh(pcoords, facevertices) (grid/Grid.cpp:184-205): solid voxelisation
// on the device, word reverse to least significant bit first, then the bit-grid form
void HierarchyGrid::genFromMesh(const std::vector<float>& pcoords, const std::vector<int>& facevertices) {
    if (!_ctx) check(rt_ctx_create(0, nullptr, &_ctx), "rt_ctx_create");
    const int R = rt_voxel_resolution(_prefer_reso);
    if (R == 0) throw std::runtime_error("genFromMesh: prefer_reso must be in [1, 1023]");
    std::vector<unsigned int> bits(((size_t)R * R * R + 31) / 32);
    int reso[3];
    float box[6];
    check(rt_voxelize_mesh(_ctx, pcoords.data(), (long)pcoords.size() / 3, facevertices.data(),
                           (long)facevertices.size() / 3, _prefer_reso, bits.data(), (long)bits.size(), reso, box),
          "voxelize_mesh");
    for (auto& w : bits) {  // most significant bit first -> least significant bit first
        unsigned int r = 0;
        for (int b = 0; b < 32; b++) r |= ((w >> b) & 1u) << (31 - b);
        w = r;
    }
    genFromMesh(bits, reso);
}

// HierarchyGrid::genFromMesh(solid_bit, out_reso) (grid/Grid.cpp:455-712) plus the
// support / load flags of Grid::computeProjectionMatrix (grid/Grid.cpp:1291-1403)
void HierarchyGrid::genFromMesh(const std::vector<unsigned int>& solid_bit, int out_reso[3]) {
    if (!_ctx) check(rt_ctx_create(0, nullptr, &_ctx), "rt_ctx_create");
    if (_h) {
        rt_hier_destroy(_h);
        _h = nullptr;
        for (auto g : _grids) delete g;
        _grids.clear();
    }
    const int R = out_reso[0];
    if ((long long)solid_bit.size() * 32 < (long long)R * R * R) throw std::runtime_error("genFromMesh: bit array too short");
    check(rt_hier_create_from_bits(_ctx, &_params, R, solid_bit.data(), &_h), "genFromMesh");
    for (int i = 0; i < rt_hier_n_levels(_h); i++) _grids.push_back(new Grid(this, i));
    rt_level_info li;
    check(rt_hier_level_info(_h, 0, &li), "level info");
    const int vx = li.nx + 1, vy = li.ny + 1, vz = li.nz + 1;
    const long nv = (long)vx * vy * vz;
    std::vector<uint8_t> surf(nv), vact(nv), vfix(nv, 0), eact((size_t)li.nx * li.ny * li.nz);
    check(rt_surface_nodes(_h, surf.data()), "surface nodes");
    check(rt_get(_h, RT_FIELD_VACT, 0, RT_LAYOUT_DENSE, vact.data()), "vact");
    check(rt_get(_h, RT_FIELD_EACT, 0, RT_LAYOUT_DENSE, eact.data()), "eact");
    std::vector<double> normals;
    _load_nodes.clear();
    _preload.clear();
    const double eh = _params.element_length;
    for (long v = 0; v < nv; v++) {
        if (!surf[v] || !vact[v]) continue;
        const int x = v % vx, y = (v / vx) % vy, z = v / ((long)vx * vy);
        double pos[3] = {x * eh, y * eh, z * eh};
        if (_inFixedArea && _inFixedArea(pos)) {
            vfix[v] = 1;
            continue;
        }
        if (_inLoadArea && _inLoadArea(pos)) {
            _load_nodes.push_back((int)v);
            // outward normal from the empty incident element slots (stand-in for the
            // CGAL AABB-tree normal of Grid::outwardNormal, grid/Grid.cpp:1405-1423)
            double n[3] = {0, 0, 0};
            for (int i = 0; i < 8; i++) {
                const int ex = x + (i & 1) - 1, ey = y + ((i >> 1) & 1) - 1, ez = z + (i >> 2) - 1;
                const bool inside = ex >= 0 && ey >= 0 && ez >= 0 && ex < li.nx && ey < li.ny && ez < li.nz &&
                                    eact[ex + (size_t)li.nx * (ey + (size_t)li.ny * ez)];
                if (!inside) {
                    n[0] += (i & 1) ? 0.5 : -0.5;
                    n[1] += ((i >> 1) & 1) ? 0.5 : -0.5;
                    n[2] += (i >> 2) ? 0.5 : -0.5;
                }
            }
            double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            if (nn == 0) { n[2] = 1; nn = 1; }
            for (int t = 0; t < 3; t++) normals.push_back(n[t] / nn);
            std::array<double, 3> fl = _loadField ? _loadField(pos) : std::array<double, 3>{0, 0, 0};
            for (int t = 0; t < 3; t++) _preload.push_back(fl[t]);
        }
    }
    check(rt_set_support(_h, vfix.data()), "rt_set_support");
    check(rt_set_load_nodes(_h, (int)_load_nodes.size(), _load_nodes.data(), normals.data()), "rt_set_load_nodes");
    // rt_set_load_nodes keeps the nodes sorted; _load_nodes was built in increasing order already
}

void HierarchyGrid::update_stencil(void) { check(rt_update_stencil(_h), "update_stencil"); }

double HierarchyGrid::v_cycle(int pre_relax, int post_relax) {
    double r = 0;
    check(rt_vcycle(_h, pre_relax, post_relax, &r), "v_cycle");
    return r;
}

Grid::Grid(HierarchyGrid* owner, int layer) : _layer(layer), _H(owner) {
    rt_level_info li;
    owner->check(rt_hier_level_info(owner->hier(), layer, &li), "level info");
    _nv = li.n_nodes;
    _n_active_nodes = li.n_active_nodes;
    _n_active_elements = li.n_active_elements;
    rt_level& L = owner->hier()->L[layer];
    for (int c = 0; c < 3; c++) {
        _U[c] = L.u + c * L.nv;
        _F[c] = L.f + c * L.nv;
        _R[c] = L.r + c * L.nv;
    }
}

void Grid::update_residual(void) { _H->check(rt_update_residual(_H->hier(), _layer), "update_residual"); }
void Grid::gs_relax(int n) { _H->check(rt_smooth(_H->hier(), _layer, RT_SMOOTH_GS, n, 1.0), "gs_relax"); }
void Grid::restrict_residual(void) { _H->check(rt_restrict_residual(_H->hier(), _layer), "restrict_residual"); }
void Grid::prolongate_correction(void) {
    _H->check(rt_prolongate_correction(_H->hier(), _layer), "prolongate_correction");
}
void Grid::solve_fem_host(void) { _H->check(rt_coarsest_solve(_H->hier()), "solve_fem_host"); }

static bool contiguous(double* v[3], long long nv) { return v[1] == v[0] + nv && v[2] == v[0] + 2 * nv; }

void Grid::applyK(double* u[3], double* f[3]) {
    if (_layer != 0) throw std::runtime_error("applyK is defined on the finest level");
    rt_hier* h = _H->hier();
    cudaStream_t s = h->ctx->stream;
    const double* uin = u[0];
    if (!contiguous(u, _nv)) {
        for (int c = 0; c < 3; c++) ck_cuda(cudaMemcpyAsync(h->x + c * _nv, u[c], sizeof(double) * _nv, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync");
        uin = h->x;
    }
    double* out = contiguous(f, _nv) ? f[0] : h->q;
    _H->check(rt_apply_K_dev(h, uin, out), "applyK");
    if (out == h->q)
        for (int c = 0; c < 3; c++) ck_cuda(cudaMemcpyAsync(f[c], h->q + c * _nv, sizeof(double) * _nv, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync");
}

double Grid::compliance(void) {
    if (_layer != 0) return v3_dot(_F, _U);
    double c = 0;
    _H->check(rt_compliance(_H->hier(), &c), "compliance");
    return c;
}

double Grid::relative_residual(void) { return v3_norm(_R) / v3_norm(_F); }
double Grid::residual(void) { return v3_norm(_R); }
void Grid::filterSensitivity(double radii) {
    _H->check(rt_filter_sensitivity(_H->hier(), (float)radii), "filterSensitivity");
}
void Grid::init_rho(double rh0) { _H->check(rt_init_density(_H->hier(), (float)rh0), "init_rho"); }

static uint64_t g_rand_seed = 0x5eed;
void Grid::randForce(void) {
    rt_hier* h = _H->hier();
    _H->check(rtk::rng_uniform(h, g_rand_seed++, 3 * _nv, _F[0]), "randForce");
}

double Grid::unitizeForce(void) {
    const double n = v3_norm(_F);
    v3_scale(_F, 1.0 / n);
    return n;
}

void Grid::reset_displacement(void) {
    for (int c = 0; c < 3; c++) ck_cuda(cudaMemsetAsync(_U[c], 0, sizeof(double) * _nv, _H->hier()->ctx->stream), "cudaMemsetAsync");
}
void Grid::reset_force(void) {
    for (int c = 0; c < 3; c++) ck_cuda(cudaMemsetAsync(_F[c], 0, sizeof(double) * _nv, _H->hier()->ctx->stream), "cudaMemsetAsync");
}
void Grid::reset_residual(void) {
    for (int c = 0; c < 3; c++) ck_cuda(cudaMemsetAsync(_R[c], 0, sizeof(double) * _nv, _H->hier()->ctx->stream), "cudaMemsetAsync");
}
float* Grid::getRho(void) { return _layer == 0 ? _H->hier()->rho : nullptr; }
float* Grid::getSens(void) { return _layer == 0 ? _H->hier()->sens : nullptr; }

double Grid::v3_dot(double* v[3], double* u[3]) {
    rt_hier* h = _H->hier();
    double tot = 0;
    for (int c = 0; c < 3; c++) {
        _H->check(rtk::dot(h, _nv, v[c], u[c], h->scal + 80 + c), "v3_dot");
    }
    ck_cuda(cudaMemcpyAsync(h->ctx->hscal, h->scal + 80, sizeof(double) * 3, cudaMemcpyDeviceToHost, h->ctx->stream), "cudaMemcpyAsync");
    ck_cuda(cudaStreamSynchronize(h->ctx->stream), "cudaStreamSynchronize");
    for (int c = 0; c < 3; c++) tot += h->ctx->hscal[c];
    return tot;
}

double Grid::v3_norm(double* v[3]) { return std::sqrt(v3_dot(v, v)); }

void Grid::v3_copy(double* vsrc[3], double* vdst[3]) {
    for (int c = 0; c < 3; c++)
        ck_cuda(cudaMemcpyAsync(vdst[c], vsrc[c], sizeof(double) * _nv, cudaMemcpyDeviceToDevice, _H->hier()->ctx->stream), "cudaMemcpyAsync");
}

void Grid::v3_scale(double* v[3], double ampl) {
    rt_hier* h = _H->hier();
    ck_cuda(cudaMemcpyAsync(h->scal + 84, &ampl, sizeof(double), cudaMemcpyHostToDevice, h->ctx->stream), "cudaMemcpyAsync");
    for (int c = 0; c < 3; c++) _H->check(rtk::scale(h, _nv, v[c], h->scal + 84, false), "v3_scale");
    ck_cuda(cudaStreamSynchronize(h->ctx->stream), "cudaStreamSynchronize");
}

void Grid::v3_add(double* a[3], double alpha, double* b[3]) { v3_add(1.0, a, alpha, b); }

void Grid::v3_add(double alpha, double* a[3], double beta, double* b[3]) {
    rt_hier* h = _H->hier();
    double ab[2] = {alpha, beta};
    memcpy(h->ctx->hscal + 30, ab, sizeof(ab));
    ck_cuda(cudaMemcpyAsync(h->scal + 86, h->ctx->hscal + 30, sizeof(ab), cudaMemcpyHostToDevice, h->ctx->stream), "cudaMemcpyAsync");
    for (int c = 0; c < 3; c++) {
        _H->check(rtk::scale(h, _nv, a[c], h->scal + 86, false), "v3_add");
        _H->check(rtk::axpy(h, _nv, beta, b[c], a[c]), "v3_add");
    }
    ck_cuda(cudaStreamSynchronize(h->ctx->stream), "cudaStreamSynchronize");
}

void Grid::elementCompliance(double* u[3], float* ce) {
    if (_layer != 0) throw std::runtime_error("elementCompliance is defined on the finest level");
    rt_hier* h = _H->hier();
    const double* uin = u[0];
    if (!contiguous(u, _nv)) {
        for (int c = 0; c < 3; c++)
            ck_cuda(cudaMemcpyAsync(h->x + c * _nv, u[c], sizeof(double) * _nv, cudaMemcpyDeviceToDevice, h->ctx->stream), "cudaMemcpyAsync");
        uin = h->x;
    }
    _H->check(rt_element_compliance(h, uin, ce), "elementCompliance");
}

// the support force arrays of level 0: allocated on first use, again when the load-node count
// changed, zeroed on allocation
void Grid::ensure_support(void) {
    const int nl = (int)_H->loadNodes().size();
    if (_FS[0] && _FS_n == nl) return;
    if (_FS[0]) cudaFree(_FS[0]);
    _FS[0] = _FS[1] = _FS[2] = _FS_new = nullptr;
    double* p = nullptr;
    _H->check(cudaMalloc(&p, sizeof(double) * 6 * (nl > 0 ? nl : 1)) == cudaSuccess ? RT_OK : RT_ENOMEM,
              "support force allocation");
    _H->check(cudaMemset(p, 0, sizeof(double) * 6 * (nl > 0 ? nl : 1)) == cudaSuccess ? RT_OK : RT_ECUDA,
              "support force allocation");
    for (int c = 0; c < 3; c++) _FS[c] = p + c * nl;
    _FS_new = p + 3 * nl;
    _FS_n = nl;
}

Grid::~Grid() {
    if (_FS[0]) cudaFree(_FS[0]);
}

double** Grid::getSupportForce(void) {
    ensure_support();
    return _FS;
}

static double support_diff_norm(grid::HierarchyGrid* H, double* const fs_old[3], const double* fs_new, int nl) {
    rt_hier* h = H->hier();
    std::vector<double> a(3 * (size_t)nl), b(3 * (size_t)nl);
    ck_cuda(cudaMemcpyAsync(b.data(), fs_new, sizeof(double) * 3 * nl, cudaMemcpyDeviceToHost, h->ctx->stream), "cudaMemcpyAsync");
    ck_cuda(cudaMemcpyAsync(a.data(), fs_old[0], sizeof(double) * 3 * nl, cudaMemcpyDeviceToHost, h->ctx->stream), "cudaMemcpyAsync");
    ck_cuda(cudaStreamSynchronize(h->ctx->stream), "cudaStreamSynchronize");
    double s = 0;
    for (size_t i = 0; i < a.size(); i++) s += (a[i] - b[i]) * (a[i] - b[i]);
    return std::sqrt(s);
}

double Grid::supportForceCh(void) { return supportForceCh(_F); }

double Grid::supportForceCh(double* f[3]) {
    ensure_support();
    const int nl = (int)_H->loadNodes().size();
    double* fin[3] = {f[0], f[1], f[2]};
    rt_hier* h = _H->hier();
    const double* src = f[0];
    if (!contiguous(fin, _nv)) {
        for (int c = 0; c < 3; c++)
            ck_cuda(cudaMemcpyAsync(h->x + c * _nv, f[c], sizeof(double) * _nv, cudaMemcpyDeviceToDevice, h->ctx->stream), "cudaMemcpyAsync");
        src = h->x;
    }
    _H->check(rt_get_force_support(h, src, _FS_new), "supportForceCh");
    return support_diff_norm(_H, _FS, _FS_new, nl);
}

double Grid::supportForceNorm(void) {
    ensure_support();
    const int nl = (int)_H->loadNodes().size();
    rt_hier* h = _H->hier();
    std::vector<double> a(3 * (size_t)nl);
    ck_cuda(cudaMemcpyAsync(a.data(), _FS[0], sizeof(double) * 3 * nl, cudaMemcpyDeviceToHost, h->ctx->stream), "cudaMemcpyAsync");
    ck_cuda(cudaStreamSynchronize(h->ctx->stream), "cudaStreamSynchronize");
    double s = 0;
    for (double v : a) s += v * v;
    return std::sqrt(s);
}

// HierarchyGrid::writeDensity / readDensity (grid/Grid.cpp:727-764, 809-839) as raw files
void HierarchyGrid::writeDensity(const std::string& filename) {
    rt_level_info li;
    check(rt_hier_level_info(_h, 0, &li), "level info");
    std::vector<float> rho((size_t)li.nx * li.ny * li.nz);
    check(rt_get(_h, RT_FIELD_RHO, 0, RT_LAYOUT_DENSE, rho.data()), "writeDensity");
    FILE* fp = fopen(filename.c_str(), "wb");
    if (!fp) throw std::runtime_error("writeDensity: cannot open " + filename);
    const int32_t dims[3] = {li.nx, li.ny, li.nz};
    const bool ok = fwrite("RTB200D1", 1, 8, fp) == 8 && fwrite(dims, sizeof(int32_t), 3, fp) == 3 &&
                    fwrite(rho.data(), sizeof(float), rho.size(), fp) == rho.size();
    fclose(fp);
    if (!ok) throw std::runtime_error("writeDensity: short write to " + filename);
}

void HierarchyGrid::readDensity(const std::string& filename) {
    rt_level_info li;
    check(rt_hier_level_info(_h, 0, &li), "level info");
    FILE* fp = fopen(filename.c_str(), "rb");
    if (!fp) throw std::runtime_error("readDensity: cannot open " + filename);
    char magic[8];
    int32_t dims[3];
    std::vector<float> rho((size_t)li.nx * li.ny * li.nz);
    bool ok = fread(magic, 1, 8, fp) == 8 && memcmp(magic, "RTB200D1", 8) == 0 &&
              fread(dims, sizeof(int32_t), 3, fp) == 3 && dims[0] == li.nx && dims[1] == li.ny && dims[2] == li.nz;
    ok = ok && fread(rho.data(), sizeof(float), rho.size(), fp) == rho.size();
    fclose(fp);
    if (!ok) throw std::runtime_error("readDensity: " + filename + " is not a density file of this grid");
    check(rt_put(_h, RT_FIELD_RHO, 0, RT_LAYOUT_DENSE, rho.data()), "readDensity");
}

}  // namespace grid

// ---------------------------------------------------------------------------
// optimization/optimization.h free functions
// ---------------------------------------------------------------------------
static uint64_t g_pm_seed = 1;

void buildGrids(const std::vector<float>& coords, const std::vector<int>& trifaces) {
    grids.set_prefer_reso(params.gridreso);
    grids.set_skip_layer(true);
    grids.genFromMesh(coords, trifaces);
}

void buildGrids(const std::vector<unsigned int>& solid_bit, int reso) {
    grids.set_skip_layer(true);  // buildGrids always skips layer 1 (optimization/optimization.cpp:17)
    int r[3] = {reso, reso, reso};
    grids.genFromMesh(solid_bit, r);
}

void setParameters(float volRatio, float volDecrease, float designStep, float filterRadi, float dampRatio,
                   float powerPenal, float min_density, int gridreso, float youngs_modulu, float poisson_ratio,
                   float /*shell_width*/, bool /*logdensity*/, bool /*logcompliance*/) {
    params.volume_ratio = volRatio;
    params.volume_decrease = volDecrease;
    params.design_step = designStep;
    params.filter_radius = (int)filterRadi;
    params.damp_ratio = dampRatio;
    params.power_penalty = powerPenal;
    params.min_rho = min_density;
    params.gridreso = gridreso;
    params.youngs_modulu = youngs_modulu;
    params.poisson_ratio = poisson_ratio;
    rt_params& p = grids.params();
    p.volume_ratio = volRatio;
    p.design_step = designStep;
    p.filter_radius = (float)params.filter_radius;
    p.damp_ratio = dampRatio;
    p.power_penalty = powerPenal;
    p.min_rho = min_density;
    p.youngs_modulus = youngs_modulu;
    p.poisson_ratio = poisson_ratio;
    if (grids.hier()) grids.check(rt_hier_set_params(grids.hier(), &p), "setParameters");
}

void setWorkMode(const std::string& m) {
    if (m == "nscf") grids.setMode(grid::no_support_constrain_force_direction);
    else if (m == "nsff") grids.setMode(grid::no_support_free_force);
    else if (m == "wscf") grids.setMode(grid::with_support_constrain_force_direction);
    else if (m == "wsff") grids.setMode(grid::with_support_free_force);
    else throw std::invalid_argument("unsupported mode " + m);
}

grid::HierarchyGrid& getGrids(void) { return grids; }

void setBoundaryCondition(std::function<bool(double[3])> fixarea, std::function<bool(double[3])> loadarea,
                          std::function<std::array<double, 3>(double[3])> forcefield) {
    grids._inFixedArea = fixarea;
    grids._inLoadArea = loadarea;
    grids._loadField = forcefield;
}

void uploadTemplateMatrix(void) {
    rt_params& p = grids.params();
    p.youngs_modulus = params.youngs_modulu;
    p.poisson_ratio = params.poisson_ratio;
    p.power_penalty = params.power_penalty;
    grids.check(rt_hier_set_params(grids.hier(), &p), "uploadTemplateMatrix");
}

void initDensities(double rho) { grids[0]->init_rho(rho); }

void update_stencil(void) { grids.update_stencil(); }

// solveFEM (optimization/optimization.cpp:85-91): V-cycles on the force the caller has set
// (TestSuit::testOrdinaryTopopt, utils/test_utils.cpp:589-660, first sets the preloaded field
// with setForceSupport(getPreloadForce(), grids[0]->getForce()))
void solveFEM(void) {
    double rel = 1;
    int it = 0;
    while (rel > 1e-4) {
        rel = grids.v_cycle();
        if (++it > 1000 || !std::isfinite(rel)) throw std::runtime_error("solveFEM did not converge");
    }
}

void remember_worst_case(void);

double modifiedPM(void) {
    double lam = 0;
    rt_solve_info info;
    grids.check(rt_worst_case(grids.hier(), RT_WORST_MODPM, 500, 0.0, g_pm_seed++, &lam, &info), "modifiedPM");
    remember_worst_case();
    return lam;
}

void computeSensitivity(void) { grids.check(rt_sensitivity(grids.hier(), 1), "computeSensitivity"); }

float updateDensities(float Vgoal) {
    float lam = 0;
    int trials = 0;
    grids.check(rt_oc_update(grids.hier(), Vgoal, &lam, &trials), "updateDensities");
    return lam;
}

// the stop test of optimization(): converge_criteria(n_constrain, max_counter, thres)
// (utils/snippet.h:156-213).  The change of a recorded sequence h is
// |h_k + h_{k-1} - h_{k-2} - h_{k-3}| / (h_{k-2} + h_{k-3}) (not a number before four values);
// an update passes when the objective's change is below thres and no constraint's change exceeds
// 1e-3, raising a counter (a failing update lowers it, not below 0); it reports convergence once
// the counter exceeds max_counter.  The change is the floating-point one (the header's
// behaviour under MSVC; under g++ its unqualified abs() truncates the change to an integer).
namespace {
class StopTest {
public:
    StopTest(int n_constrain, int max_counter, double thres)
        : _n(n_constrain), _max(max_counter), _thres(thres), _g(n_constrain) {}
    bool update(double value, const double* constraints) {
        _c.push_back(value);
        for (int i = 0; i < _n; i++) _g[i].push_back(constraints[i]);
        bool ok = change(_c) < _thres;
        for (int i = 0; i < _n && ok; i++)
            if (change(_g[i]) > 1e-3) ok = false;
        _counter = ok ? _counter + 1 : std::max(_counter - 1, 0);
        return _counter > _max;
    }

private:
    static double change(const std::vector<double>& h) {
        const size_t k = h.size();
        if (k < 4) return std::numeric_limits<double>::quiet_NaN();
        return std::fabs(h[k - 1] + h[k - 2] - h[k - 3] - h[k - 4]) / (h[k - 3] + h[k - 4]);
    }
    int _n, _max, _counter = 0;
    double _thres;
    std::vector<double> _c;
    std::vector<std::vector<double>> _g;
};
}  // namespace

// optimization() (optimization/optimization.cpp:583-673) without the file output: the volume
// goal shrinks by volume_decrease each iteration (the constraint value Vc is taken before the
// goal is clamped to volume_ratio), and the loop ends when the stop test converges with the goal
// at the volume ratio; the worst-case compliances and goals are kept (optimizationRecords)
static std::vector<double> g_c_record, g_vol_record;
void optimization(int max_iter) {
    initDensities(params.volume_ratio);
    float Vgoal = params.volume_ratio;
    StopTest stop_check(1, 2, 5e-3);
    g_c_record.clear();
    g_vol_record.clear();
    for (int itn = 1; itn <= max_iter; itn++) {
        Vgoal *= (1 - params.volume_decrease);
        double Vc = Vgoal - params.volume_ratio;
        if (Vgoal < params.volume_ratio) Vgoal = params.volume_ratio;
        update_stencil();
        const double c = modifiedPM();
        g_c_record.push_back(c);
        g_vol_record.push_back(Vgoal);
        if (stop_check.update(c, &Vc) && Vgoal <= params.volume_ratio + 1e-3) break;
        computeSensitivity();
        updateDensities(Vgoal);
    }
}

const std::vector<double>& optimizationRecords(std::vector<double>* volumes) {
    if (volumes) *volumes = g_vol_record;
    return g_c_record;
}

// test_rigid_displacement (optimization/optimization.cpp:697-709)
void test_rigid_displacement(void) {
    grid::Grid* g = grids[0];
    rt_hier* h = grids.hier();
    rt_level& L = h->L[0];
    std::vector<double> u(3 * L.nv);
    std::vector<uint8_t> act(L.nv);
    grids.check(rt_get(h, RT_FIELD_VACT, 0, RT_LAYOUT_DENSE, act.data()), "vact");
    for (int k = 0; k < 6; k++) {
        for (long v = 0; v < L.nv; v++) {
            const double p[3] = {(double)(v % L.vx), (double)((v / L.vx) % L.vy), (double)(v / ((long)L.vx * L.vy))};
            double m[3] = {0, 0, 0};
            if (k < 3) m[k] = 1;
            else {
                const double w[3] = {k == 3 ? 1.0 : 0.0, k == 4 ? 1.0 : 0.0, k == 5 ? 1.0 : 0.0};
                m[0] = w[1] * p[2] - w[2] * p[1];
                m[1] = w[2] * p[0] - w[0] * p[2];
                m[2] = w[0] * p[1] - w[1] * p[0];
            }
            for (int c = 0; c < 3; c++) u[c * L.nv + v] = act[v] ? m[c] : 0.0;
        }
        grids.check(rt_put(h, RT_FIELD_U, 0, RT_LAYOUT_DENSE, u.data()), "rigid u");
        g->reset_force();
        g->update_residual();
        printf("-- u_rigid %d res = %lf\n", k, g->residual());
    }
}

// ---------------------------------------------------------------------------
// optimization/projection.h:16-65
// ---------------------------------------------------------------------------
static double* contiguous_copy(double* const v[3], long long nv, double* scratch) {
    if (v[1] == v[0] + nv && v[2] == v[0] + 2 * nv) return v[0];
    rt_hier* h = grids.hier();
    for (int c = 0; c < 3; c++)
        ck_cuda(cudaMemcpyAsync(scratch + c * nv, v[c], sizeof(double) * nv, cudaMemcpyDeviceToDevice, h->ctx->stream), "cudaMemcpyAsync");
    return scratch;
}

static void copy_back(double* const v[3], long long nv, const double* src) {
    if (src == v[0]) return;
    rt_hier* h = grids.hier();
    for (int c = 0; c < 3; c++)
        ck_cuda(cudaMemcpyAsync(v[c], src + c * nv, sizeof(double) * nv, cudaMemcpyDeviceToDevice, h->ctx->stream), "cudaMemcpyAsync");
}

const std::vector<int>& getLoadNodes(void) { return grids.loadNodes(); }
int n_loadnodes(void) { return (int)grids.loadNodes().size(); }

void forceProject(double* f_dev[3]) {
    const long long nv = grids[0]->n_box_nodes();
    double* f = contiguous_copy(f_dev, nv, grids.hier()->x);
    grids.check(rt_force_project(grids.hier(), f), "forceProject");
    copy_back(f_dev, nv, f);
}

// host support-force vectors (one per component, the load nodes in order): scattered into a
// device vector, projected, gathered back
void forceProject(std::vector<double> fsupport[3]) {
    rt_hier* h = grids.hier();
    const int nl = n_loadnodes();
    for (int c = 0; c < 3; c++)
        if ((int)fsupport[c].size() != nl) throw std::invalid_argument("forceProject: support vectors of the wrong length");
    std::vector<double> soa(3 * (size_t)nl);
    for (int c = 0; c < 3; c++) std::copy(fsupport[c].begin(), fsupport[c].end(), soa.begin() + (size_t)c * nl);
    if (nl == 0) return;
    double* d = h->fs;  // the hierarchy's [3][nload] support-force scratch
    ck_cuda(cudaMemcpyAsync(d, soa.data(), sizeof(double) * 3 * nl, cudaMemcpyHostToDevice, h->ctx->stream), "cudaMemcpyAsync");
    grids.check(rt_set_force_support(h, d, h->x), "forceProject");
    grids.check(rt_force_project(h, h->x), "forceProject");
    grids.check(rt_get_force_support(h, h->x, d), "forceProject");
    ck_cuda(cudaMemcpyAsync(soa.data(), d, sizeof(double) * 3 * nl, cudaMemcpyDeviceToHost, h->ctx->stream), "cudaMemcpyAsync");
    ck_cuda(cudaStreamSynchronize(h->ctx->stream), "cudaStreamSynchronize");
    for (int c = 0; c < 3; c++) std::copy(soa.begin() + (size_t)c * nl, soa.begin() + (size_t)(c + 1) * nl, fsupport[c].begin());
}

void getForceSupport(double const* const f_dev[3], double* fsup[3]) {
    rt_hier* h = grids.hier();
    const long long nv = grids[0]->n_box_nodes();
    const int nl = n_loadnodes();
    double* fv[3] = {const_cast<double*>(f_dev[0]), const_cast<double*>(f_dev[1]), const_cast<double*>(f_dev[2])};
    const double* f = contiguous_copy(fv, nv, h->x);
    const bool soa = fsup[1] == fsup[0] + nl && fsup[2] == fsup[0] + 2 * nl;
    double* dst = soa ? fsup[0] : h->fs;  // h->fs holds 3 * nload doubles
    grids.check(rt_get_force_support(h, f, dst), "getForceSupport");
    if (!soa)
        for (int c = 0; c < 3; c++)
            ck_cuda(cudaMemcpyAsync(fsup[c], dst + (size_t)c * nl, sizeof(double) * nl, cudaMemcpyDeviceToDevice, h->ctx->stream), "cudaMemcpyAsync");
    ck_cuda(cudaStreamSynchronize(h->ctx->stream), "cudaStreamSynchronize");
}

void getForceSupport(double const* const f_dev[3], std::vector<double> fs[3]) {
    rt_hier* h = grids.hier();
    const int nl = n_loadnodes();
    double* p[3] = {h->fs, h->fs + nl, h->fs + 2 * nl};
    getForceSupport(f_dev, p);
    for (int c = 0; c < 3; c++) {
        fs[c].resize(nl);
        ck_cuda(cudaMemcpy(fs[c].data(), p[c], sizeof(double) * nl, cudaMemcpyDeviceToHost), "cudaMemcpy");
    }
}

void setForceSupport(double const* const fsup[3], double* f_dev[3]) {
    rt_hier* h = grids.hier();
    const long long nv = grids[0]->n_box_nodes();
    const int nl = n_loadnodes();
    const double* src = fsup[0];
    if (!(fsup[1] == fsup[0] + nl && fsup[2] == fsup[0] + 2 * nl)) {
        for (int c = 0; c < 3; c++)
            ck_cuda(cudaMemcpyAsync(h->fs + (size_t)c * nl, fsup[c], sizeof(double) * nl, cudaMemcpyDeviceToDevice, h->ctx->stream), "cudaMemcpyAsync");
        src = h->fs;
    }
    const bool contig = f_dev[1] == f_dev[0] + nv && f_dev[2] == f_dev[0] + 2 * nv;
    double* dst = contig ? f_dev[0] : h->x;
    grids.check(rt_set_force_support(h, src, dst), "setForceSupport");
    copy_back(f_dev, nv, dst);
    ck_cuda(cudaStreamSynchronize(h->ctx->stream), "cudaStreamSynchronize");
}

void displacementProject(double* u_dev[3]) {
    const long long nv = grids[0]->n_box_nodes();
    double* u = contiguous_copy(u_dev, nv, grids.hier()->x);
    grids.check(rt_displacement_project(grids.hier(), u), "displacementProject");
    copy_back(u_dev, nv, u);
    ck_cuda(cudaStreamSynchronize(grids.hier()->ctx->stream), "cudaStreamSynchronize");
}

// ---------------------------------------------------------------------------
// remaining optimization/optimization.h entry points
// ---------------------------------------------------------------------------
static std::string g_output_dir = ".";

void setOutpurDir(const std::string& dirname) { g_output_dir = dirname; }
const std::string& getOutputDir(void) { return g_output_dir; }

// inCompleteModiPM (optimization/optimization.cpp:427-472): a random balanced unit load, then up to
// 50 steps of one V-cycle on it, the displacement projected and normalised as the next load, until
// the support force changes by less than fch_thres; returns the compliance f.u
double inCompleteModiPM(double fch_thres) {
    grid::Grid* g = grids[0];
    g->randForce();
    forceProject(g->getForce());
    g->unitizeForce();
    g->reset_displacement();
    getForceSupport(g->getForce(), g->getSupportForce());
    double fch = 1;
    int itn = 0;
    while (itn++ < 50 && fch > fch_thres) {
        grids.v_cycle(1, 1);
        g->v3_copy(g->getDisplacement(), g->getForce());
        forceProject(g->getForce());
        g->unitizeForce();
        fch = g->supportForceCh() / g->supportForceNorm();
        getForceSupport(g->getForce(), g->getSupportForce());
    }
    const double c = g->compliance();
    if (!std::isfinite(c)) throw std::runtime_error("inCompleteModiPM: NaN compliance");
    return c;
}

// MGPSOR (optimization/optimization.cpp:474-535): inCompleteModiPM, then preconditioned
// eigen-iterations x <- x + Vcycle(P x - lambda K x) with lambda = |P x|^2 / x.K x; like the
// reference it returns u.K u for u = x / |P x|, i.e. 1 / lambda
double MGPSOR(void) {
    grid::Grid* g = grids[0];
    inCompleteModiPM();
    rt_hier* h = grids.hier();
    const long long nv = g->n_box_nodes();
    double* xk_mem = nullptr;
    grids.check(cudaMalloc(&xk_mem, sizeof(double) * 3 * nv) == cudaSuccess ? RT_OK : RT_ENOMEM, "MGPSOR");
    double* xk[3] = {xk_mem, xk_mem + nv, xk_mem + 2 * nv};
    double fch = 1, fsnorm = 1;
    int itn = 0;
    while ((itn++ < 200 && fch > 1e-4) || itn < 3) {
        g->v3_copy(g->getDisplacement(), xk);
        g->applyK(g->getDisplacement(), g->getForce());
        const double c = g->v3_dot(g->getDisplacement(), g->getForce());
        forceProject(g->getDisplacement());
        fsnorm = g->v3_norm(g->getDisplacement());
        const double lambda = fsnorm * fsnorm / c;
        g->v3_add(-lambda, g->getForce(), 1, g->getDisplacement());
        g->v3_scale(g->getDisplacement(), 1.0 / g->v3_norm(g->getDisplacement()));
        fch = g->supportForceCh(g->getDisplacement());
        getForceSupport(g->getDisplacement(), g->getSupportForce());
        g->reset_displacement();
        double rel_res = 1;
        int vit = 0;
        while (rel_res > 1e-1 && vit++ < 3) rel_res = grids.v_cycle();
        g->v3_add(g->getDisplacement(), 1, xk);
    }
    cudaFree(xk_mem);
    (void)h;
    g->v3_scale(g->getDisplacement(), 1.0 / fsnorm);
    g->applyK(g->getDisplacement(), g->getForce());
    return g->v3_dot(g->getDisplacement(), g->getForce());
}

// RayleighGradient (optimization/optimization.cpp:385-398): for R(u) = |P u|^2 / u.K u, returns
// (|P u|^2, u.K u) and g <- the gradient -2 P u / u.K u + 2 |P u|^2 K u / (u.K u)^2 (the
// reference's sign convention); leaves K u in the force vector
std::pair<double, double> RayleighGradient(double* u[3], double* g[3]) {
    grid::Grid* G = grids[0];
    G->v3_copy(u, g);
    forceProject(g);
    const double pnorm = G->v3_dot(g, g);
    G->applyK(u, G->getForce());
    const double knorm = G->v3_dot(u, G->getForce());
    G->v3_add(-2.0 / knorm, g, 2.0 * pnorm / (knorm * knorm), G->getForce());
    return {pnorm, knorm};
}

// Pnorm / Knorm (optimization/optimization.cpp:400-425)
double Pnorm(double* u[3]) {
    std::vector<double> fs[3];
    getForceSupport(u, fs);
    forceProject(fs);
    double s = 0;
    for (int c = 0; c < 3; c++)
        for (double v : fs[c]) s += v * v;
    return s;
}

double Knorm(double* u[3]) {
    grid::Grid* G = grids[0];
    G->applyK(u, G->getForce());
    return G->v3_dot(u, G->getForce());
}

// checkAdjointVariable (optimization/optimization.cu:353-402): with the adjoint N^T lambda in the
// displacement vector and the last worst-case pair from modifiedPM (u_w, its compliance mu, and
// f_w = K u_w, which the reference keeps in Fworst), |2 f_w - K (N^T lambda) - 2 mu K f_w| on the
// free nodes must be below 1e-6 (relative to |f_w|); the displacement vector is left unchanged
static std::vector<double> g_uworst, g_fworst;
static double g_mu = 0;

void remember_worst_case(void) {
    rt_hier* h = grids.hier();
    const long long nv = grids[0]->n_box_nodes();
    g_uworst.resize(3 * nv);
    g_fworst.resize(3 * nv);
    std::vector<double> f(3 * nv);
    grids.check(rt_get(h, RT_FIELD_U, 0, RT_LAYOUT_DENSE, g_uworst.data()), "worst-case displacement");
    grids.check(rt_get(h, RT_FIELD_F, 0, RT_LAYOUT_DENSE, f.data()), "worst-case force");
    grids.check(rt_apply_K(h, g_uworst.data(), g_fworst.data()), "K u_worst");
    g_mu = 0;
    for (long long i = 0; i < 3 * nv; i++) g_mu += g_uworst[i] * f[i];
}

bool checkAdjointVariable(void) {
    if (g_fworst.empty()) throw std::runtime_error("checkAdjointVariable: run modifiedPM first");
    rt_hier* h = grids.hier();
    const long long nv = grids[0]->n_box_nodes();
    std::vector<double> adj(3 * nv), kadj(3 * nv), kkf(3 * nv);
    std::vector<uint8_t> fix(nv, 0);
    grids.check(rt_get(h, RT_FIELD_U, 0, RT_LAYOUT_DENSE, adj.data()), "adjoint");
    grids.check(rt_apply_K(h, adj.data(), kadj.data()), "K adjoint");
    grids.check(rt_apply_K(h, g_fworst.data(), kkf.data()), "K f_worst");
    grids.check(rt_get(h, RT_FIELD_VFIX, 0, RT_LAYOUT_DENSE, fix.data()), "supports");
    double r2 = 0, f2 = 0;
    for (long long i = 0; i < 3 * nv; i++) {
        if (fix[i % nv]) continue;  // resetDirchlet: rows of fixed nodes dropped
        const double r = 2 * g_fworst[i] - kadj[i] - 2 * g_mu * kkf[i];
        r2 += r * r;
        f2 += g_fworst[i] * g_fworst[i];
    }
    return std::sqrt(r2) < 1e-6 * std::max(std::sqrt(f2), 1e-300);
}

// selfTest (optimization/optimization.cu:231-328): the reference checks its BitSAT and GraftArray
// containers; here the equivalent checks of this library's structures: the rigid modes are in the
// null space of the finest operator (test_rigid_displacement) and the template matrix is symmetric
void selfTest(void) {
    printf("-- Self testing...\n");
    double ke[576];
    grids.check(rt_template_matrix(grids.hier(), ke), "template matrix");
    double asym = 0;
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) asym = std::max(asym, std::fabs(ke[i * 24 + j] - ke[j * 24 + i]));
    printf("-- template matrix asymmetry %g\n", asym);
    test_rigid_displacement();
}

// getPreloadForce (optimization/projection.cu:387-390): the load field evaluated at the load nodes
// when the grid was built, as device arrays [3][nload] (refreshed on every call)
double** getPreloadForce(void) {
    static double* fl[3] = {nullptr, nullptr, nullptr};
    static size_t cap = 0;
    const int nl = n_loadnodes();
    if ((size_t)nl > cap || !fl[0]) {
        if (fl[0]) gpu_manager.delete_buf(fl[0]);
        fl[0] = (double*)gpu_manager.add_buf("preload force", sizeof(double) * 3 * (nl > 0 ? nl : 1));
        cap = nl;
    }
    for (int c = 0; c < 3; c++) fl[c] = fl[0] + (size_t)c * nl;
    const auto& pl = grids.preloadForce();
    std::vector<double> soa(3 * (size_t)nl);
    for (int i = 0; i < nl; i++)
        for (int c = 0; c < 3; c++) soa[(size_t)c * nl + i] = pl[3 * (size_t)i + c];
    if (nl > 0) gpu_manager_t::upload_buf(fl[0], soa.data(), sizeof(double) * soa.size());
    return fl;
}

// setDensity (utils/test_utils.cpp:1672) and Grid::volumeRatio
void setDensity(const float* rho_dev) {
    grids.check(rt_put_dev(grids.hier(), RT_FIELD_RHO, 0, rho_dev), "setDensity");
}

double volumeRatio(void) {
    rt_hier* h = grids.hier();
    rt_level_info li;
    grids.check(rt_hier_level_info(h, 0, &li), "volumeRatio");
    const size_t ne = (size_t)li.nx * li.ny * li.nz;
    std::vector<float> rho(ne);
    std::vector<uint8_t> act(ne);
    grids.check(rt_get(h, RT_FIELD_RHO, 0, RT_LAYOUT_DENSE, rho.data()), "volumeRatio");
    grids.check(rt_get(h, RT_FIELD_EACT, 0, RT_LAYOUT_DENSE, act.data()), "volumeRatio");
    double s = 0;
    long long na = 0;
    for (size_t e = 0; e < ne; e++)
        if (act[e]) {
            s += rho[e];
            na++;
        }
    return na ? s / (double)na : 0.0;
}

namespace MMA {
namespace {
__global__ void k_d2f(long long n, const double* __restrict__ x, float* __restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = (float)x[i];
}
}  // namespace

mma_t::mma_t(int ndim, int nConstrain, double) : _n(ndim) {
    if (nConstrain != 1) throw std::invalid_argument("mma_t: this implementation takes exactly one constraint");
    if (ndim < 1) throw std::invalid_argument("mma_t: no design variables");
}

mma_t::~mma_t() {
    if (_m) rt_mma_destroy(_m);
    if (_x32 && cudaFree(nullptr) == cudaSuccess) cudaFree(_x32);
}

void mma_t::init(float lower_bound, float upper_bound) {
    if (_m) rt_mma_destroy(_m);
    _m = nullptr;
    grids.check(rt_mma_create(grids.ctx(), _n, nullptr, nullptr, lower_bound, upper_bound, &_m), "mma_t::init");
}

void mma_t::init(const float* lower_bound_host, const float* upper_bound_host) {
    std::vector<double> lo(lower_bound_host, lower_bound_host + _n), hi(upper_bound_host, upper_bound_host + _n);
    if (_m) rt_mma_destroy(_m);
    _m = nullptr;
    grids.check(rt_mma_create(grids.ctx(), _n, lo.data(), hi.data(), 0.0, 0.0, &_m), "mma_t::init");
}

bool mma_t::update(float* dev_df, float** dg, float* dev_g) {
    if (!_m) throw std::runtime_error("mma_t::update: call init first");
    float g = 0;
    ck_cuda(cudaMemcpy(&g, dev_g, sizeof(float), cudaMemcpyDeviceToHost), "mma_t::update");
    int stop = 0;
    grids.check(rt_mma_update(_m, dev_df, dg[0], (double)g, &stop, nullptr, nullptr), "mma_t::update");
    return stop != 0;
}

mma_t::XView mma_t::get_x(void) {
    if (!_m) throw std::runtime_error("mma_t::get_x: call init first");
    if (!_x32) ck_cuda(cudaMalloc(&_x32, sizeof(float) * (size_t)_n), "mma_t::get_x");
    const double* x = nullptr;
    grids.check(rt_mma_x(_m, &x), "mma_t::get_x");
    rt_ctx* c = grids.hier()->ctx;
    const unsigned nb = (unsigned)std::min<long long>((_n + 255) / 256, 1184);
    grids.check(rt_launch(c, "mma_design_f32", [&] { k_d2f<<<nb, 256, 0, c->stream>>>(_n, x, _x32); }), "mma_t::get_x");
    ck_cuda(cudaStreamSynchronize(c->stream), "mma_t::get_x");
    return XView{_x32};
}
}  // namespace MMA

