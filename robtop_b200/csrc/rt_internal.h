// rt_internal.h — internal state of the B200 solver library (not part of the ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/rtb200.h"

#define RT_KERNEL_NAMES_MAX 64

struct rt_kstat {
    std::string name;
    long long launches = 0;
    double ms = 0;
};

struct rt_ctx {
    // references: the caller's handle plus every hierarchy, workspace and network made on the
    // context; rt_ctx_destroy drops the caller's, the last release frees the context
    int refs = 1;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    int sm_count = 148;
    long long launches = 0;
    // polls of a bounded device wait on another block (the grid barrier of the fused sweeps);
    // rt_ctx_set_wait_limit lowers it so a test can make a wait run out
    long long wait_limit = 1LL << 22;
    // a CUDA error already pending when a launch began (reported with that launch)
    cudaError_t pending_err = cudaSuccess;
    // profiling
    bool profile = false;
    // set while a batched graph is captured: its instances run concurrently, so no cooperative
    // (grid-synchronised) launch may be part of it
    bool batch_capture = false;
    int coop_blocks_per_sm = -1;  // co-resident blocks of the fused Chebyshev kernels (-1: not queried)
    int res_blocks_per_sm = 0;
    std::vector<rt_kstat> kstats;
    std::unordered_map<const void*, int> kid_by_name;  // kernel-name literal -> kstats index
    std::vector<cudaEvent_t> ev_pool;
    struct Pending { int kid; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    // host-pinned scalar mailbox
    double* hscal = nullptr;
    // second stream, only ever used as a capture target: the body of a conditional node is
    // captured on it while the context stream's own capture is still open
    cudaStream_t aux_stream = nullptr;
    // instantiated batched-PCG graphs (rt_pcg_batch), newest last
    struct BatchGraph {
        uint64_t key = 0;
        std::vector<uint64_t> uids;  // hierarchies whose buffers the graph references
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        // kernels per instance: prologue + start kernel, and one loop iteration
        std::vector<long> once_kernels, iter_kernels;
    };
    std::vector<BatchGraph> batch_graphs;
};

struct rt_level {
    int nx = 0, ny = 0, nz = 0, vx = 0, vy = 0, vz = 0;
    long nv = 0, ne = 0;
    int ratio = 0;
    long n_act_nodes = 0, n_act_elems = 0;
    uint8_t* vact = nullptr;
    uint8_t* eact = nullptr;
    double *u = nullptr, *f = nullptr, *r = nullptr;
    float *u32 = nullptr, *f32 = nullptr, *r32 = nullptr;
    double* d = nullptr;  // Chebyshev direction
    float* d32 = nullptr;
    double* st = nullptr;   // [243][nv]
    float* st32 = nullptr;     // FP32 smoother copy, 32-node blocks [nv/32][243][32]
    uint16_t* st16 = nullptr;  // BF16 copy [nv/32][252][32] (only once rt_params.coarse_bf16 was set)
    // coarsest level
    int na = 0;
    int* aidx = nullptr;
    double* ainv = nullptr;  // [3na][3na]
    double* dvec = nullptr;  // [3na] gather buffer
};

// launch shape of a finest-level operator kernel (chosen by rt_autotune)
struct rt_tile_cfg {
    int variant = 1;  // 0: shared-memory element tile (rt_fine_tile.cu), 1: register marching (rt_fine_march.cu),
                      // 5: sum-factorised row marching (rt_fine_sf.cu; ty = node rows 4, 8 or 16),
                      // 2: register marching with the output-stage loads issued ahead
    int ty = 4;       // node rows per warp tile (marching kernel: 2, 4 or 8)
    int zchunk = 16;  // node layers per tile
};

struct rt_hier {
    rt_ctx* ctx = nullptr;
    uint64_t uid = 0;            // unique per hierarchy / workspace of the process (graph cache keys)
    // a solve workspace (rt_hier_workspace_create) owns only its solve vectors and scalars;
    // every operator buffer and setting is the parent's, refreshed by ws_sync before each use
    rt_hier* parent = nullptr;
    std::vector<rt_hier*> wspool;  // workspaces this hierarchy made for its own block solves
    rt_params P;
    rt_tile_cfg tune[2][4];          // [FP32, FP64][residual, applyK, jacobi, chebyshev]
    double tune_us[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};  // measured time of the chosen shape
    // stencil-level kernels of the FP32 smoother [FP32 stencils, BF16 stencils]: 0 lane-split
    // (4 lanes per node, loads through L1), 1 bulk-copy (32-node stencil runs staged in shared memory)
    int st_variant[2] = {0, 1};
    double st_us[2][2] = {{0, 0}, {0, 0}};  // [stencil type][variant] level-1 Chebyshev step (rt_autotune)
    // stencil levels whose FP32 Chebyshev sweeps run as one cooperative launch (bit lvl; rt_autotune),
    // with the measured time of a sweep set [level][separate launches, one launch]
    uint32_t cheby_fused = 0;
    uint32_t cheby_stream = 0;  // fused levels held to the streaming form (rt_set_level_fused on = 2)
    double fused_us[15][2] = {};
    double* dinv64 = nullptr;        // [6][nv] inverted diagonal blocks of the finest level
    float* dinv32 = nullptr;
    std::vector<rt_level> L;
    double KE[576];
    double* KE_dev = nullptr;
    float* KE32_dev = nullptr;
    // level-0 design data
    float* rho = nullptr;
    float* w = nullptr;       // powf(rho, p) or 0
    uint8_t* vfix = nullptr;  // support flags
    bool has_support = false;
    float* sens = nullptr;
    float* ftmp = nullptr;    // element scratch (filter copy / OC trial)
    uint8_t* eshell = nullptr;
    // load set
    int nload = 0;
    int* load_nodes = nullptr;
    double* load_normal = nullptr;  // [3*nload]
    double* Rd = nullptr;           // [6][3*nload]
    int nrig = 0;
    double* Ru = nullptr;           // [6][3*nv] rigid modes over active nodes (no-support modes)
    double* fs = nullptr;           // [3*nload] gather buffer
    double* fs_old = nullptr;       // [3*nload]
    // solver work vectors (3*nv doubles each)
    double *x = nullptr, *rr = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *rold = nullptr;
    // Lanczos basis
    double* Q = nullptr;
    int Qcap = 0;
    // reductions
    double* partials = nullptr;  // [RT_RED_BLOCKS * 8]
    // FP32 Krylov vectors of the refinement form (rt_params.krylov_fp32), allocated on first use
    float *p32k = nullptr, *q32k = nullptr, *d32k = nullptr, *ro32k = nullptr;
    cudaGraph_t pcg32_graph = nullptr;
    cudaGraphExec_t pcg32_exec = nullptr;
    uint64_t pcg32_key = 0;
    long pcg32_iter_kernels = 0;  // kernels in one iteration of the captured FP32 loop
    double* scal = nullptr;      // [64] device scalars
    bool stencil_ready = false;
    double* Qgal = nullptr;  // [R^3][576] cell Galerkin blocks P^T KE P (rebuilt when KE changes)
    int Qgal_ratio = 0;
    // MG-PCG loop captured as one CUDA graph (WHILE conditional node)
    bool use_graphs = true;
    cudaGraph_t pcg_graph = nullptr;
    cudaGraphExec_t pcg_exec = nullptr;
    uint64_t pcg_key = 0;
    long pcg_iter_kernels = 0;  // kernels in one iteration of the captured loop (launch accounting)
    // the previously used PCG graph, kept so that two forms can alternate without re-capture (the
    // loop with the learned correction for a design's first solve, without it once the gate
    // judged the network off)
    cudaGraph_t pcg_graph_alt = nullptr;
    cudaGraphExec_t pcg_exec_alt = nullptr;
    uint64_t pcg_key_alt = 0;
    long pcg_iter_kernels_alt = 0;
    uint64_t graph_epoch = 0;  // bumped whenever captured pointers may change
    // learned correction added to the V-cycle inside PCG (rt_hier_set_learned); scal[27] holds the
    // fallback ratio, scal[28] the gate (1 while active), scal[29] the previous iteration's r.r
    struct rt_unet* unet = nullptr;
    double unet_fallback = 1.0;
    // the gate's verdict carries over from solve to solve: once an iteration with the network
    // failed the ratio, the correction stays off until the design (rt_update_stencil) or the
    // network changes.  unet_kernels: kernels of one correction (launch accounting of the IF node
    // that runs it inside the captured loop); unet_applied: corrections run since attach
    bool unet_off = false;
    // bumped whenever the density, the supports, the stencil or the parameters change; the gate's
    // verdict on the learned correction holds while the design it was made on is unchanged
    uint64_t design_epoch = 0;
    uint64_t unet_verdict_epoch = ~0ull;
    int unet_post = 0;  // finest-level smoothing steps applied to z after the correction
    long unet_kernels = 0;
    long long unet_applied = 0;
    long long fallbacks = 0;  // PCG solves that continued with FP64 V-cycles after stalling
};

#define RT_RED_BLOCKS 296
#define RT_PARTIALS (148 * 64)  // block partial sums: up to 64 values from 148 blocks
#define RT_NSCAL 1024           // device scalar slots

void rt_ctx_retain(rt_ctx* c);
void rt_ctx_release(rt_ctx* c);

// error helpers -------------------------------------------------------------
int rt_fail(rt_ctx* c, int code, const char* fmt, ...);
#define RT_CUDA(c, call)                                                                    \
    do {                                                                                    \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess)                                                              \
            return rt_fail((c), RT_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,        \
                           cudaGetErrorString(_e));                                         \
    } while (0)
#define RT_CHECK(x)                     \
    do {                                \
        int _s = (x);                   \
        if (_s != RT_OK) return _s;     \
    } while (0)

// launch accounting ------------------------------------------------------------
int rt_kernel_id(rt_ctx* c, const char* name);
void rt_launch_begin(rt_ctx* c, int kid, cudaEvent_t* a);
int rt_launch_end(rt_ctx* c, int kid, cudaEvent_t a, const char* name);

// every kernel launch of the library goes through here: per-context launch counts
// and, when profiling is on, CUDA events around the launch
template <typename F>
inline int rt_launch(rt_ctx* c, const char* name, F&& f) {
    const int kid = rt_kernel_id(c, name);
    cudaEvent_t a = nullptr;
    rt_launch_begin(c, kid, &a);
    f();
    return rt_launch_end(c, kid, a, name);
}

static inline unsigned rt_blocks(long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// Chebyshev smoother on the interval [lmax / 30, 1.1 lmax] of D^-1 A (lmax from a
// power iteration at stencil set-up).  Step k of the three-term recurrence
//   d_0 = D^-1 r_0 / theta,   d_k = a_k d_{k-1} + b_k D^-1 r_k,   u += d_k
// with theta = (hi+lo)/2, delta = (hi-lo)/2, sigma = theta/delta, rho_0 = 1/sigma,
// rho_k = 1/(2 sigma - rho_{k-1}), a_k = rho_k rho_{k-1}, b_k = 2 rho_k / delta.
#define RT_CHEBY_LO_FRAC (1.0 / 30.0)
#define RT_CHEBY_HI_FRAC 1.1
#define RT_SCAL_ERR 295   // set to 1 by a stencil kernel whose bounded copy wait ran out
#define RT_SCAL_LMAX 300  // device scalar slots holding lmax(D^-1 A) per level
#define RT_SCAL_GBAR 480  // per level: the grid barrier of the fused Chebyshev sweeps (arrivals, generation as 2 x u32)
// (a_k, b_k), k < RT_CHEBY_MAXK, per level at RT_SCAL_CHEB + 2 RT_CHEBY_MAXK lvl (levels 0..14);
// the 16th table serves kernel timing before any stencil exists
#define RT_CHEBY_MAXK 16
#define RT_SCAL_CHEB 512
#define RT_SCAL_CHEB_SPARE (RT_SCAL_CHEB + 2 * RT_CHEBY_MAXK * 15)
#define RT_MAX_LEVELS 15
__host__ __device__ inline void rt_cheby_coef(double lmax, int k, double& a, double& b) {
    const double hi = RT_CHEBY_HI_FRAC * lmax, lo = RT_CHEBY_LO_FRAC * lmax;
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    double rho = 1.0 / sigma;
    a = 0.0;
    b = 1.0 / theta;
    for (int i = 1; i <= k; i++) {
        const double rn = 1.0 / (2.0 * sigma - rho);
        a = rn * rho;
        b = 2.0 * rn / delta;
        rho = rn;
    }
}

// kernels (each returns RT_OK or an error code) -------------------------------
namespace rtk {
// fine level
template <typename T>
int fine_residual(rt_hier* h, const T* u, const T* f, T* r);
template <typename T>
int fine_applyK(rt_hier* h, const T* u, T* out);
template <typename T>
int fine_gs(rt_hier* h, T* u, const T* f, bool backward);
template <typename T>
int fine_jacobi(rt_hier* h, const T* u, const T* f, T* unew, double omega);
template <typename T>
int fine_cheby(rt_hier* h, const T* u, const T* f, T* unew, T* d, const double* coef, int kstep);
template <typename T>
int st_cheby(rt_hier* h, int lvl, const T* u, const T* f, T* unew, T* d, const double* coef, int kstep);
// nsteps FP32 Chebyshev steps of stencil level lvl in one cooperative launch (u -> tmp -> u ...,
// the result in u); false from st_cheby_fused_ok when the device cannot co-schedule the grid
int st_cheby_fused(rt_hier* h, int lvl, float* u, const float* f, float* tmp, float* d, const double* coef, int nsteps);
bool st_cheby_fused_ok(rt_hier* h);
int penalty_weights(rt_hier* h);
int init_tile_kernels(rt_ctx* c);
int init_sf_kernels(rt_ctx* c);
template <typename T, bool WS, int MODE>
int launch_sf(rt_hier* h, const T* u, const T* f, T* out, double omega, const char* name, T* dvec, const double* coef,
              int kstep);
int init_stencil_kernels(rt_ctx* c);
int fine_dinv(rt_hier* h);
template <typename T, int MODE>
int fine_march(rt_hier* h, const T* u, const T* f, T* out, double omega, T* dvec, const double* coef, int kstep);
int tile_zchunk_default(rt_ctx* c, int vx, int vy, int vz);
// stencil levels
template <typename T>
int st_residual(rt_hier* h, int lvl, const T* u, const T* f, T* r);
template <typename T>
int st_gs(rt_hier* h, int lvl, T* u, const T* f, bool backward);
template <typename T>
int st_jacobi(rt_hier* h, int lvl, const T* u, const T* f, T* unew, double omega);
int galerkin_from_elements(rt_hier* h);
int galerkin_from_stencil(rt_hier* h, int lvl);
// transfers
template <typename T>
int restrict_(rt_hier* h, int lvl, const T* rf, T* fc);
template <typename T>
int prolong_add(rt_hier* h, int lvl, const T* uc, T* uf);
// coarsest
int coarsest_setup(rt_hier* h);
template <typename T>
int coarsest_solve(rt_hier* h, const T* f, T* u);
// BLAS-1 / reductions
int dot(rt_hier* h, long n, const double* a, const double* b, double* out_dev);
int dot2(rt_hier* h, long n, const double* a, const double* b, const double* c, double* out_dev);
int axpy(rt_hier* h, long n, double a, const double* x, double* y);
int d2f(rt_hier* h, long n, const double* a, float* b);
int stencil_copies(rt_hier* h, int lvl);
int f2d(rt_hier* h, long n, const float* a, double* b);
int d2f_scaled(rt_hier* h, long n, const double* a, float* b, const double* s_dev);
int f2d_scaled(rt_hier* h, long n, const float* a, double* b, const double* s_dev);
int f2d_scaled_add(rt_hier* h, long n, const float* a, double* b, const double* s_dev);
// fused passes of the PCG iteration: x, r update with r.r; widening of z with (z.r, z.rold)
int pcg_update_xr_rr(rt_hier* h, long n, const double* num, const double* den, double* x, double* r, const double* p,
                     const double* q, double* rold, double* rr_out, float* r32 = nullptr, double* scale_out = nullptr);
int dot32(rt_hier* h, long n, const float* a, const float* b, double* out);
int dot32_2(rt_hier* h, long n, const float* a, const float* b, const float* c, double* out);
int pcg32_update_p(rt_hier* h, long n, const double* s, const double* it, float* p, const float* z);
int pcg32_update_xr_rr(rt_hier* h, long n, const double* num, const double* den, float* d, float* r, const float* p,
                       const float* q, float* rold, double* rr_out);
int axpy_f32_scaled(rt_hier* h, long n, double* x, const float* d, const double* s);
int f2d_scaled_dot2(rt_hier* h, long n, const float* a, double* z, const double* s_dev, const double* r,
                    const double* rold, double* out);
int pcg_update_xr(rt_hier* h, long n, const double* scal_alpha_num, const double* scal_alpha_den, double* x,
                  double* r, const double* p, const double* q, double* rold);
int pcg_update_p(rt_hier* h, long n, const double* s_num, const double* s_den, double* p, const double* z,
                 bool first);
int mask_copy(rt_hier* h, long n, const double* src, double* dst);
// worst case
int rng_uniform(rt_hier* h, uint64_t seed, long n, double* out);
int project_load(rt_hier* h, double* f);
int gather_load(rt_hier* h, const double* f, double* fs);
int scatter_load(rt_hier* h, const double* fs, double* f);
int rigid_basis(rt_hier* h);
int rigid_nodes(rt_hier* h);
int displacement_project(rt_hier* h, double* u);
int scale(rt_hier* h, long n, double* x, const double* s_dev, bool inverse_sqrt);
int tridiag_max_eig(rt_hier* h, int k, const double* alpha_dev, const double* beta_dev, double* out_dev);
// optimisation
int sensitivity(rt_hier* h, const double* u);
int element_compliance(rt_hier* h, const double* u, float* out);
int filter(rt_hier* h, float radius);
int oc_try(rt_hier* h, float thr, float* out, double* vol_dev);
int oc_maxabs(rt_hier* h, float* out_dev);
// setup
int node_active(rt_ctx* c, int nx, int ny, int nz, const uint8_t* eact, uint8_t* vact);
int coarsen_elements(rt_ctx* c, int nx, int ny, int nz, int ratio, const uint8_t* ef, uint8_t* ec);
int surface_nodes(rt_hier* h, uint8_t* surf_dev);
int cube_vbits(rt_ctx* c, int R, const uint32_t* eb, uint32_t* vb);
int cube_coarsen(rt_ctx* c, int R, const uint32_t* ef, uint32_t* ec);
int count_u8(rt_ctx* c, long n, const uint8_t* a, double* out_dev);
}  // namespace rtk
