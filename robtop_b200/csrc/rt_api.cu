// rt_api.cu — C ABI entry points and host orchestration of the solver.
//
// The host side only sequences kernels on the context stream; every
// arithmetic step of the hot path runs on the GPU.  Host work is limited to
// set-up bookkeeping (level plan, index maps, load-set rigid basis) and to
// reading back convergence scalars.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "rt_internal.h"
#include "rt_unet.h"

// ---------------------------------------------------------------------------
// errors, launch accounting
// ---------------------------------------------------------------------------
int rt_fail(rt_ctx* c, int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

int rt_kernel_id(rt_ctx* c, const char* name) {
    auto it = c->kid_by_name.find(name);
    if (it != c->kid_by_name.end()) return it->second;
    int id = -1;
    for (size_t i = 0; i < c->kstats.size(); i++)  // same name from another literal
        if (c->kstats[i].name == name) id = (int)i;
    if (id < 0) {
        rt_kstat k;
        k.name = name;
        c->kstats.push_back(k);
        id = (int)c->kstats.size() - 1;
    }
    c->kid_by_name[name] = id;
    return id;
}

static cudaEvent_t ev_get(rt_ctx* c) {
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

static void profile_drain(rt_ctx* c) {
    for (auto& p : c->pending) {
        float ms = 0;
        cudaEventSynchronize(p.b);
        cudaEventElapsedTime(&ms, p.a, p.b);
        c->kstats[p.kid].ms += ms;
        c->ev_pool.push_back(p.a);
        c->ev_pool.push_back(p.b);
    }
    c->pending.clear();
}

void rt_launch_begin(rt_ctx* c, int kid, cudaEvent_t* a) {
    (void)kid;
    // an error left by an earlier runtime call is reported as such, not as this launch's
    c->pending_err = cudaGetLastError();
    if (c->profile) {
        *a = ev_get(c);
        cudaEventRecord(*a, c->stream);
    }
}

int rt_launch_end(rt_ctx* c, int kid, cudaEvent_t a, const char* name) {
    c->launches++;
    c->kstats[kid].launches++;
    cudaError_t e = cudaGetLastError();
    if (c->profile) {
        cudaEvent_t b = ev_get(c);
        cudaEventRecord(b, c->stream);
        c->pending.push_back({kid, a, b});
        if (c->pending.size() > 4096) profile_drain(c);
    }
    if (c->pending_err != cudaSuccess) {
        const cudaError_t pe = c->pending_err;
        c->pending_err = cudaSuccess;
        return rt_fail(c, RT_ECUDA, "a CUDA error was pending before the launch of %s: %s", name, cudaGetErrorString(pe));
    }
    if (e != cudaSuccess) return rt_fail(c, RT_ECUDA, "launch of %s failed: %s", name, cudaGetErrorString(e));
    return RT_OK;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
extern "C" int rt_ctx_create(int device, void* stream, rt_ctx** out) {
    if (!out) return RT_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RT_ECUDA;
    if (device < 0 || device >= ndev) return RT_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return RT_ECUDA;
    rt_ctx* c = new rt_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return RT_ECUDA;
        }
        c->own_stream = true;
    }
    if (cudaMallocHost(&c->hscal, sizeof(double) * 64) != cudaSuccess) {
        delete c;
        return RT_ECUDA;
    }
    *out = c;
    return RT_OK;
}

void rt_ctx_retain(rt_ctx* c) {
    if (c) c->refs++;
}

static void ctx_free(rt_ctx* c);

void rt_ctx_release(rt_ctx* c) {
    if (c && --c->refs == 0) ctx_free(c);
}

// the caller's reference: the context lives on until its last hierarchy, workspace or network is destroyed
extern "C" void rt_ctx_destroy(rt_ctx* c) { rt_ctx_release(c); }

static void ctx_free(rt_ctx* c) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    profile_drain(c);
    for (auto& bg : c->batch_graphs) {
        if (bg.exec) cudaGraphExecDestroy(bg.exec);
        if (bg.graph) cudaGraphDestroy(bg.graph);
    }
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    if (c->hscal) cudaFreeHost(c->hscal);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    delete c;
}

extern "C" const char* rt_last_error(rt_ctx* c) { return c ? c->err.c_str() : "null context"; }

extern "C" int rt_ctx_set_wait_limit(rt_ctx* c, long long polls) {
    if (!c) return RT_EINVAL;
    c->wait_limit = polls >= 0 ? polls : (1LL << 22);
    return RT_OK;
}

extern "C" int rt_ctx_sync(rt_ctx* c) {
    if (!c) return RT_EINVAL;
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    return RT_OK;
}

extern "C" int rt_profile_enable(rt_ctx* c, int on) {
    if (!c) return RT_EINVAL;
    if (!on) {
        cudaStreamSynchronize(c->stream);
        profile_drain(c);
    }
    c->profile = on != 0;
    return RT_OK;
}

extern "C" int rt_profile_reset(rt_ctx* c) {
    if (!c) return RT_EINVAL;
    cudaStreamSynchronize(c->stream);
    profile_drain(c);
    for (auto& k : c->kstats) { k.launches = 0; k.ms = 0; }
    return RT_OK;
}

extern "C" int rt_profile_query(rt_ctx* c, int idx, char* name, int name_len, long long* launches, double* ms) {
    if (!c) return RT_EINVAL;
    cudaStreamSynchronize(c->stream);
    profile_drain(c);
    if (idx < 0 || idx >= (int)c->kstats.size()) return RT_EINVAL;
    if (name && name_len > 0) {
        strncpy(name, c->kstats[idx].name.c_str(), name_len - 1);
        name[name_len - 1] = 0;
    }
    if (launches) *launches = c->kstats[idx].launches;
    if (ms) *ms = c->kstats[idx].ms;
    return RT_OK;
}

extern "C" long long rt_launch_count(rt_ctx* c) { return c ? c->launches : 0; }

extern "C" void rt_params_default(rt_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->power_penalty = 3.f;
    p->min_rho = 1e-3f;
    p->volume_ratio = 0.4f;
    p->design_step = 0.03f;
    p->damp_ratio = 0.5f;
    p->filter_radius = 2.f;
    p->youngs_modulus = 1e6;
    p->poisson_ratio = 0.4;
    p->element_length = 1.0;
    p->mode = RT_MODE_WSFF;
    p->skip_layer1 = 1;
    p->smoother = RT_SMOOTH_SGS;
    p->pre_sweeps = 1;
    p->post_sweeps = 1;
    p->jacobi_omega = 0.6;
    p->precision = RT_FP64;
    p->coarsest_elements = 400;
    p->cycle_gamma = 1;
    p->coarse_sweeps = 0;
    p->precision_fallback = 100;
    p->coarse_bf16 = 0;
    p->krylov_fp32 = 0;
    p->cycle_gamma_levels = 0;
}

// ---------------------------------------------------------------------------
// element template: element/templateMatrix.cpp:15-124 (host, once per parameter set)
// ---------------------------------------------------------------------------
static void template_matrix(double E, double nu, double h, double* KE) {
    double D[6][6] = {};
    const double s = E / ((1 + nu) * (1 - 2 * nu));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i][j] = s * (i == j ? 1 - nu : nu);
    for (int i = 3; i < 6; i++) D[i][i] = s * (1 - 2 * nu) / 2;
    const double p = std::sqrt(3.0) / 3;
    std::fill(KE, KE + 576, 0.0);
    for (int g = 0; g < 8; g++) {
        const double gp[3] = {((2 * (g % 2) - 1) * p + 1) / 2, ((2 * (g / 2 % 2) - 1) * p + 1) / 2,
                              ((2 * (g / 4) - 1) * p + 1) / 2};
        double gN[8][3];
        for (int k = 0; k < 8; k++) {
            const int id[3] = {k % 2, k / 2 % 2, k / 4};
            double r[3];
            for (int a = 0; a < 3; a++) r[a] = id[a] ? gp[a] : 1 - gp[a];
            for (int a = 0; a < 3; a++) gN[k][a] = (id[a] ? 1.0 / h : -1.0 / h) * r[(a + 1) % 3] * r[(a + 2) % 3];
        }
        double B[6][24] = {};
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 8; b++) B[a][3 * b + a] = gN[b][a];
        for (int b = 0; b < 8; b++) {
            B[3][3 * b + 1] = gN[b][2]; B[3][3 * b + 2] = gN[b][1];
            B[4][3 * b + 0] = gN[b][2]; B[4][3 * b + 2] = gN[b][0];
            B[5][3 * b + 0] = gN[b][1]; B[5][3 * b + 1] = gN[b][0];
        }
        for (int i = 0; i < 24; i++)
            for (int j = 0; j < 24; j++) {
                double acc = 0;
                for (int a = 0; a < 6; a++)
                    for (int b = 0; b < 6; b++) acc += B[a][i] * D[a][b] * B[b][j];
                KE[i * 24 + j] += acc;
            }
    }
    const double sc = std::pow(h / 2, 3);
    for (int i = 0; i < 576; i++) KE[i] *= sc;
}

// ---------------------------------------------------------------------------
// hierarchy
// ---------------------------------------------------------------------------
static uint64_t next_uid() {
    static std::atomic<uint64_t> counter{1};
    return counter.fetch_add(1);
}

template <typename T>
static int dalloc(rt_ctx* c, T** p, size_t n) {
    if (n == 0) n = 1;
    if (cudaMalloc((void**)p, sizeof(T) * n) != cudaSuccess) {
        cudaGetLastError();
        return rt_fail(c, RT_ENOMEM, "cudaMalloc of %zu bytes failed", sizeof(T) * n);
    }
    return RT_OK;
}

// drop the context's batched graphs that reference hierarchy uid (its buffers are going away)
static void purge_batch_graphs(rt_ctx* c, uint64_t uid) {
    auto& v = c->batch_graphs;
    for (size_t i = 0; i < v.size();) {
        if (std::find(v[i].uids.begin(), v[i].uids.end(), uid) != v[i].uids.end()) {
            if (v[i].exec) cudaGraphExecDestroy(v[i].exec);
            if (v[i].graph) cudaGraphDestroy(v[i].graph);
            v.erase(v.begin() + i);
        } else {
            i++;
        }
    }
}

static void free_hier(rt_hier* h);

// a workspace frees only the solve buffers it allocated (rt_hier_workspace_create)
static void free_workspace(rt_hier* w) {
    for (auto& L : w->L) {
        cudaFree(L.u); cudaFree(L.f); cudaFree(L.r); cudaFree(L.u32); cudaFree(L.f32); cudaFree(L.r32);
        cudaFree(L.d); cudaFree(L.d32); cudaFree(L.dvec);
    }
    cudaFree(w->x); cudaFree(w->rr); cudaFree(w->z); cudaFree(w->p); cudaFree(w->q); cudaFree(w->rold);
    cudaFree(w->partials); cudaFree(w->scal);
    if (w->pcg_exec) cudaGraphExecDestroy(w->pcg_exec);
    if (w->pcg_graph) cudaGraphDestroy(w->pcg_graph);
    if (w->pcg_exec_alt) cudaGraphExecDestroy(w->pcg_exec_alt);
    if (w->pcg_graph_alt) cudaGraphDestroy(w->pcg_graph_alt);
    if (w->pcg32_exec) cudaGraphExecDestroy(w->pcg32_exec);
    if (w->pcg32_graph) cudaGraphDestroy(w->pcg32_graph);
    cudaFree(w->p32k); cudaFree(w->q32k); cudaFree(w->d32k); cudaFree(w->ro32k);
    rt_ctx* c = w->ctx;
    delete w;
    rt_ctx_release(c);
}

static void free_hier(rt_hier* h) {
    if (!h) return;
    if (h->ctx) purge_batch_graphs(h->ctx, h->uid);
    for (rt_hier* w : h->wspool) {
        purge_batch_graphs(h->ctx, w->uid);
        free_workspace(w);
    }
    h->wspool.clear();
    if (h->parent) {
        free_workspace(h);
        return;
    }
    for (auto& L : h->L) {
        cudaFree(L.vact); cudaFree(L.eact); cudaFree(L.u); cudaFree(L.f); cudaFree(L.r);
        cudaFree(L.u32); cudaFree(L.f32); cudaFree(L.r32); cudaFree(L.st); cudaFree(L.st32); cudaFree(L.st16);
        cudaFree(L.d); cudaFree(L.d32);
        cudaFree(L.aidx); cudaFree(L.ainv); cudaFree(L.dvec);
    }
    cudaFree(h->KE_dev); cudaFree(h->KE32_dev); cudaFree(h->rho); cudaFree(h->w); cudaFree(h->vfix);
    cudaFree(h->sens); cudaFree(h->ftmp); cudaFree(h->eshell); cudaFree(h->load_nodes); cudaFree(h->load_normal);
    cudaFree(h->Rd); cudaFree(h->Ru); cudaFree(h->fs); cudaFree(h->fs_old); cudaFree(h->x); cudaFree(h->rr);
    cudaFree(h->z); cudaFree(h->p); cudaFree(h->q); cudaFree(h->rold); cudaFree(h->Q); cudaFree(h->partials);
    cudaFree(h->scal); cudaFree(h->Qgal); cudaFree(h->dinv64); cudaFree(h->dinv32);
    if (h->pcg_exec) cudaGraphExecDestroy(h->pcg_exec);
    if (h->pcg_graph) cudaGraphDestroy(h->pcg_graph);
    if (h->pcg_exec_alt) cudaGraphExecDestroy(h->pcg_exec_alt);
    if (h->pcg_graph_alt) cudaGraphDestroy(h->pcg_graph_alt);
    if (h->pcg32_exec) cudaGraphExecDestroy(h->pcg32_exec);
    if (h->pcg32_graph) cudaGraphDestroy(h->pcg32_graph);
    cudaFree(h->p32k); cudaFree(h->q32k); cudaFree(h->d32k); cudaFree(h->ro32k);
    rt_ctx* c = h->ctx;
    delete h;
    rt_ctx_release(c);
}

// refresh a workspace's copy of its parent's operator (buffers, settings, launch shapes)
static void ws_sync(rt_hier* w) {
    const rt_hier* p = w->parent;
    if (!p) return;
    w->P = p->P;
    memcpy(w->tune, p->tune, sizeof(w->tune));
    memcpy(w->tune_us, p->tune_us, sizeof(w->tune_us));
    memcpy(w->st_variant, p->st_variant, sizeof(w->st_variant));
    w->cheby_fused = p->cheby_fused;
    w->cheby_stream = p->cheby_stream;
    w->dinv64 = p->dinv64; w->dinv32 = p->dinv32;
    for (size_t i = 0; i < w->L.size(); i++) {
        rt_level& a = w->L[i];
        const rt_level& b = p->L[i];
        a.vact = b.vact; a.eact = b.eact; a.st = b.st; a.st32 = b.st32; a.st16 = b.st16;
        a.na = b.na; a.aidx = b.aidx; a.ainv = b.ainv;
        a.n_act_nodes = b.n_act_nodes; a.n_act_elems = b.n_act_elems;
    }
    memcpy(w->KE, p->KE, sizeof(w->KE));
    w->KE_dev = p->KE_dev; w->KE32_dev = p->KE32_dev;
    w->rho = p->rho; w->w = p->w; w->vfix = p->vfix; w->has_support = p->has_support;
    w->sens = p->sens; w->ftmp = p->ftmp; w->eshell = p->eshell;
    w->nload = p->nload; w->load_nodes = p->load_nodes; w->load_normal = p->load_normal; w->Rd = p->Rd;
    w->nrig = p->nrig; w->Ru = p->Ru;
    w->stencil_ready = p->stencil_ready;
    w->Qgal = p->Qgal; w->Qgal_ratio = p->Qgal_ratio;
    w->use_graphs = p->use_graphs;
    w->graph_epoch = p->graph_epoch;
    w->unet = nullptr;  // the network's activation buffers cannot be shared by concurrent solves
}

#define RT_NOT_WORKSPACE(h)                                                                                   \
    do {                                                                                                      \
        if ((h)->parent)                                                                                      \
            return rt_fail((h)->ctx, RT_ESTATE, "%s changes or reads the operator's own state: call it on the " \
                                                "parent hierarchy, not on a solve workspace", __func__);      \
    } while (0)

static int upload_KE(rt_hier* h) {
    template_matrix(h->P.youngs_modulus, h->P.poisson_ratio, h->P.element_length, h->KE);
    float ke32[576];
    for (int i = 0; i < 576; i++) ke32[i] = (float)h->KE[i];
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->KE_dev, h->KE, sizeof(double) * 576, cudaMemcpyHostToDevice, h->ctx->stream));
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->KE32_dev, ke32, sizeof(float) * 576, cudaMemcpyHostToDevice, h->ctx->stream));
    RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    if (h->Qgal) { cudaFree(h->Qgal); h->Qgal = nullptr; h->Qgal_ratio = 0; }
    h->graph_epoch++;  // the element operator's Hadamard-domain values are kernel parameters
    return RT_OK;
}

static int build_hier(rt_ctx* c, const rt_params* p, int nx, int ny, int nz, uint8_t* eact_dev, rt_hier** out) {
    rt_hier* h = new rt_hier();
    h->ctx = c;
    rt_ctx_retain(c);
    h->uid = next_uid();
    h->P = *p;
    // RT_GRAPHS=0 runs the PCG loop as individual launches (same kernels; for per-launch profilers)
    if (const char* g = std::getenv("RT_GRAPHS")) h->use_graphs = std::atoi(g) != 0;
    *out = h;  // the caller releases a partially built hierarchy on failure
    // level chain on the device: halve while more than 400 elements are solid (grid/Grid.cpp:488)
    struct Chain { int nx, ny, nz; uint8_t* e; long cnt; };
    std::vector<Chain> chain;
    double* dcnt = nullptr;
    RT_CUDA(c, cudaMalloc(&dcnt, sizeof(double)));
    chain.push_back({nx, ny, nz, eact_dev, 0});
    for (;;) {
        Chain& last = chain.back();
        long ne = (long)last.nx * last.ny * last.nz;
        RT_CHECK(rtk::count_u8(c, ne, last.e, dcnt));
        double hc = 0;
        RT_CUDA(c, cudaMemcpyAsync(&hc, dcnt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        RT_CUDA(c, cudaStreamSynchronize(c->stream));
        last.cnt = (long)hc;
        const long stop = p->coarsest_elements > 0 ? p->coarsest_elements : 400;
        if (last.cnt <= stop || (last.nx <= 1 && last.ny <= 1 && last.nz <= 1)) break;
        Chain nxt{(last.nx + 1) / 2, (last.ny + 1) / 2, (last.nz + 1) / 2, nullptr, 0};
        RT_CHECK(dalloc(c, &nxt.e, (size_t)nxt.nx * nxt.ny * nxt.nz));
        RT_CHECK(rtk::coarsen_elements(c, last.nx, last.ny, last.nz, 2, last.e, nxt.e));
        chain.push_back(nxt);
    }
    cudaFree(dcnt);
    std::vector<int> idx, ratio;
    if (p->skip_layer1 && chain.size() >= 3) {
        idx.push_back(0); ratio.push_back(0);
        idx.push_back(2); ratio.push_back(4);
        for (size_t i = 3; i < chain.size(); i++) { idx.push_back((int)i); ratio.push_back(2); }
    } else {
        for (size_t i = 0; i < chain.size(); i++) { idx.push_back((int)i); ratio.push_back(i ? 2 : 0); }
    }
    if (chain.size() == 1) {
        cudaFree(chain[0].e);
        return rt_fail(c, RT_EINVAL, "grid too small for multigrid (no level above the coarsest-size limit)");
    }
    if (idx.size() > RT_MAX_LEVELS) {
        for (Chain& ch : chain) cudaFree(ch.e);
        return rt_fail(c, RT_EINVAL, "more than 15 multigrid levels");
    }
    for (size_t k = 0; k < idx.size(); k++) {
        Chain& ch = chain[idx[k]];
        rt_level L;
        L.nx = ch.nx; L.ny = ch.ny; L.nz = ch.nz;
        L.vx = L.nx + 1; L.vy = L.ny + 1; L.vz = L.nz + 1;
        L.nv = (long)L.vx * L.vy * L.vz;
        L.ne = (long)L.nx * L.ny * L.nz;
        L.ratio = ratio[k];
        L.n_act_elems = ch.cnt;
        L.eact = ch.e;
        ch.e = nullptr;
        h->L.push_back(L);
    }
    for (auto& ch : chain) if (ch.e) cudaFree(ch.e);
    for (size_t k = 0; k < h->L.size(); k++) {
        rt_level& L = h->L[k];
        if ((double)L.nv * 243.0 >= 2147483647.0 && k > 0) return rt_fail(c, RT_EINVAL, "coarse level too large");
        RT_CHECK(dalloc(c, &L.vact, L.nv));
        RT_CHECK(rtk::node_active(c, L.nx, L.ny, L.nz, L.eact, L.vact));
        RT_CHECK(dalloc(c, &L.u, 3 * L.nv)); RT_CHECK(dalloc(c, &L.f, 3 * L.nv)); RT_CHECK(dalloc(c, &L.r, 3 * L.nv));
        RT_CHECK(dalloc(c, &L.u32, 3 * L.nv)); RT_CHECK(dalloc(c, &L.f32, 3 * L.nv)); RT_CHECK(dalloc(c, &L.r32, 3 * L.nv));
        RT_CHECK(dalloc(c, &L.d, 3 * L.nv)); RT_CHECK(dalloc(c, &L.d32, 3 * L.nv));
        RT_CUDA(c, cudaMemsetAsync(L.u, 0, sizeof(double) * 3 * L.nv, c->stream));
        RT_CUDA(c, cudaMemsetAsync(L.f, 0, sizeof(double) * 3 * L.nv, c->stream));
        RT_CUDA(c, cudaMemsetAsync(L.r, 0, sizeof(double) * 3 * L.nv, c->stream));
        if (k > 0) {
            RT_CHECK(dalloc(c, &L.st, 243 * L.nv));
            RT_CHECK(dalloc(c, &L.st32, 243 * (size_t)((L.nv + 31) / 32 * 32)));
            RT_CUDA(c, cudaMemsetAsync(L.st, 0, sizeof(double) * 243 * L.nv, c->stream));
        }
        std::vector<uint8_t> va(L.nv);
        RT_CUDA(c, cudaMemcpyAsync(va.data(), L.vact, L.nv, cudaMemcpyDeviceToHost, c->stream));
        RT_CUDA(c, cudaStreamSynchronize(c->stream));
        long na = 0;
        for (long v = 0; v < L.nv; v++) na += va[v];
        L.n_act_nodes = na;
        if (k + 1 == h->L.size()) {
            std::vector<int> aidx;
            for (long v = 0; v < L.nv; v++)
                if (va[v]) aidx.push_back((int)v);
            L.na = (int)aidx.size();
            const size_t n = 3 * (size_t)L.na;
            if (n > 12288) return rt_fail(c, RT_EINVAL, "coarsest level too large for the dense solve (%zu DOF)", n);
            RT_CHECK(dalloc(c, &L.aidx, L.na));
            RT_CUDA(c, cudaMemcpyAsync(L.aidx, aidx.data(), sizeof(int) * L.na, cudaMemcpyHostToDevice, c->stream));
            RT_CHECK(dalloc(c, &L.ainv, n * n));
            RT_CHECK(dalloc(c, &L.dvec, n));
            RT_CUDA(c, cudaStreamSynchronize(c->stream));
        }
    }
    rt_level& L0 = h->L[0];
    RT_CHECK(dalloc(c, &h->KE_dev, 576));
    RT_CHECK(dalloc(c, &h->KE32_dev, 576));
    RT_CHECK(dalloc(c, &h->dinv64, 6 * (size_t)L0.nv));
    RT_CHECK(dalloc(c, &h->dinv32, 6 * (size_t)L0.nv));
    {
        const int zc = rtk::tile_zchunk_default(c, L0.vx, L0.vy, L0.vz);
        for (int pr = 0; pr < 2; pr++)
            for (int m = 0; m < 4; m++) h->tune[pr][m] = rt_tile_cfg{1, 4, zc};
    }
    RT_CHECK(dalloc(c, &h->rho, L0.ne));
    RT_CHECK(dalloc(c, &h->w, L0.ne));
    RT_CHECK(dalloc(c, &h->vfix, L0.nv));
    RT_CHECK(dalloc(c, &h->sens, L0.ne));
    RT_CHECK(dalloc(c, &h->ftmp, L0.ne));
    RT_CUDA(c, cudaMemsetAsync(h->vfix, 0, L0.nv, c->stream));
    RT_CUDA(c, cudaMemsetAsync(h->sens, 0, sizeof(float) * L0.ne, c->stream));
    const size_t n3 = 3 * (size_t)L0.nv;
    RT_CHECK(dalloc(c, &h->x, n3)); RT_CHECK(dalloc(c, &h->rr, n3)); RT_CHECK(dalloc(c, &h->z, n3));
    RT_CHECK(dalloc(c, &h->p, n3)); RT_CHECK(dalloc(c, &h->q, n3)); RT_CHECK(dalloc(c, &h->rold, n3));
    RT_CHECK(dalloc(c, &h->partials, RT_PARTIALS));
    RT_CHECK(dalloc(c, &h->scal, RT_NSCAL));
    RT_CUDA(c, cudaMemsetAsync(h->scal, 0, sizeof(double) * RT_NSCAL, c->stream));
    RT_CHECK(upload_KE(h));
    RT_CHECK(rtk::init_tile_kernels(c));
    RT_CHECK(rtk::init_sf_kernels(c));
    RT_CHECK(rtk::init_stencil_kernels(c));
    *out = h;
    return RT_OK;
}

extern "C" int rt_hier_create(rt_ctx* c, const rt_params* p, int nx, int ny, int nz, const uint8_t* eact,
                              rt_hier** out) {
    if (!c || !p || !eact || !out || nx <= 0 || ny <= 0 || nz <= 0) return RT_EINVAL;
    *out = nullptr;
    RT_CUDA(c, cudaSetDevice(c->device));
    uint8_t* e = nullptr;
    const size_t ne = (size_t)nx * ny * nz;
    RT_CHECK(dalloc(c, &e, ne));
    RT_CUDA(c, cudaMemcpyAsync(e, eact, ne, cudaMemcpyHostToDevice, c->stream));
    rt_hier* h = nullptr;
    int s = build_hier(c, p, nx, ny, nz, e, &h);
    if (s != RT_OK) {
        if (h) free_hier(h);
        return s;
    }
    *out = h;
    return RT_OK;
}

// genFromMesh(solid_bit, out_reso) takes a cubic reso^3 bit grid; the dense box is
// the solid's extent from the origin (coarsening stays aligned with the cube's).
extern "C" int rt_hier_create_from_bits(rt_ctx* c, const rt_params* p, int reso, const uint32_t* bits, rt_hier** out) {
    if (!c || !p || !bits || !out || reso <= 0) return RT_EINVAL;
    int mx = 0, my = 0, mz = 0;
    const long nb = (long)reso * reso * reso;
    for (long t = 0; t < nb; t++)
        if ((bits[t >> 5] >> (t & 31)) & 1u) {
            mx = std::max(mx, (int)(t % reso) + 1);
            my = std::max(my, (int)((t / reso) % reso) + 1);
            mz = std::max(mz, (int)(t / ((long)reso * reso)) + 1);
        }
    if (mx == 0) return rt_fail(c, RT_EINVAL, "empty solid");
    std::vector<uint8_t> e((size_t)mx * my * mz, 0);
    for (int z = 0; z < mz; z++)
        for (int y = 0; y < my; y++)
            for (int x = 0; x < mx; x++) {
                long t = x + (long)reso * (y + (long)reso * z);
                e[x + (size_t)mx * (y + (size_t)my * z)] = (bits[t >> 5] >> (t & 31)) & 1u;
            }
    return rt_hier_create(c, p, mx, my, mz, e.data(), out);
}

extern "C" void rt_hier_destroy(rt_hier* h) {
    if (!h) return;
    cudaSetDevice(h->ctx->device);
    cudaStreamSynchronize(h->ctx->stream);
    free_hier(h);
}

extern "C" int rt_hier_n_levels(rt_hier* h) { return h ? (int)h->L.size() : 0; }

extern "C" int rt_hier_level_info(rt_hier* h, int lvl, rt_level_info* out) {
    if (!h || !out || lvl < 0 || lvl >= (int)h->L.size()) return RT_EINVAL;
    rt_level& L = h->L[lvl];
    out->nx = L.nx; out->ny = L.ny; out->nz = L.nz; out->ratio = L.ratio;
    out->n_nodes = L.nv; out->n_active_nodes = L.n_act_nodes; out->n_active_elements = L.n_act_elems;
    return RT_OK;
}

extern "C" int rt_hier_get_params(rt_hier* h, rt_params* p) {
    if (!h || !p) return RT_EINVAL;
    *p = h->P;
    return RT_OK;
}

extern "C" int rt_hier_set_params(rt_hier* h, const rt_params* p) {
    if (!h || !p) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    const bool ke = p->youngs_modulus != h->P.youngs_modulus || p->poisson_ratio != h->P.poisson_ratio ||
                    p->element_length != h->P.element_length;
    if (p->skip_layer1 != h->P.skip_layer1)
        return rt_fail(h->ctx, RT_EINVAL, "skip_layer1 is fixed when the hierarchy is built");
    auto coarsest = [](int v) { return v > 0 ? v : 400; };
    if (coarsest(p->coarsest_elements) != coarsest(h->P.coarsest_elements))
        return rt_fail(h->ctx, RT_EINVAL, "coarsest_elements is fixed when the hierarchy is built");
    if (p->precision < RT_FP64 || p->precision > RT_FP64_FINE) return rt_fail(h->ctx, RT_EINVAL, "unknown precision");
    h->P = *p;
    if (ke) RT_CHECK(upload_KE(h));
    h->stencil_ready = false;
    h->design_epoch++;
    h->graph_epoch++;  // captured graphs bake in the settings and the stencil copies they read
    return RT_OK;
}

extern "C" int rt_template_matrix(rt_hier* h, double* KE) {
    if (!h || !KE) return RT_EINVAL;
    memcpy(KE, h->KE, sizeof(double) * 576);
    return RT_OK;
}

extern "C" int rt_cube_vertex_bits(rt_ctx* c, int reso, const uint32_t* eb, uint32_t* vb) {
    if (!c || !eb || !vb || reso <= 0) return RT_EINVAL;
    const size_t ne = ((size_t)reso * reso * reso + 31) / 32, nv = ((size_t)(reso + 1) * (reso + 1) * (reso + 1) + 31) / 32;
    uint32_t *de = nullptr, *dv = nullptr;
    RT_CHECK(dalloc(c, &de, ne));
    RT_CHECK(dalloc(c, &dv, nv));
    RT_CUDA(c, cudaMemcpyAsync(de, eb, ne * 4, cudaMemcpyHostToDevice, c->stream));
    int s = rtk::cube_vbits(c, reso, de, dv);
    if (s == RT_OK) {
        cudaMemcpyAsync(vb, dv, nv * 4, cudaMemcpyDeviceToHost, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) s = RT_ECUDA;
    }
    cudaFree(de);
    cudaFree(dv);
    return s;
}

extern "C" int rt_cube_coarsen_bits(rt_ctx* c, int reso, const uint32_t* ef, uint32_t* ec) {
    if (!c || !ef || !ec || reso < 2) return RT_EINVAL;
    const int rc = reso / 2;
    const size_t nf = ((size_t)reso * reso * reso + 31) / 32, ncw = ((size_t)rc * rc * rc + 31) / 32;
    uint32_t *df = nullptr, *dc = nullptr;
    RT_CHECK(dalloc(c, &df, nf));
    RT_CHECK(dalloc(c, &dc, ncw));
    RT_CUDA(c, cudaMemcpyAsync(df, ef, nf * 4, cudaMemcpyHostToDevice, c->stream));
    int s = rtk::cube_coarsen(c, reso, df, dc);
    if (s == RT_OK) {
        cudaMemcpyAsync(ec, dc, ncw * 4, cudaMemcpyDeviceToHost, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) s = RT_ECUDA;
    }
    cudaFree(df);
    cudaFree(dc);
    return s;
}

// ---------------------------------------------------------------------------
// boundary conditions
// ---------------------------------------------------------------------------
extern "C" int rt_surface_nodes(rt_hier* h, uint8_t* surf) {
    if (!h || !surf) return RT_EINVAL;
    rt_level& L = h->L[0];
    uint8_t* d = nullptr;
    RT_CHECK(dalloc(h->ctx, &d, L.nv));
    int s = rtk::surface_nodes(h, d);
    if (s == RT_OK) {
        cudaMemcpyAsync(surf, d, L.nv, cudaMemcpyDeviceToHost, h->ctx->stream);
        if (cudaStreamSynchronize(h->ctx->stream) != cudaSuccess) s = RT_ECUDA;
    }
    cudaFree(d);
    return s;
}

extern "C" int rt_set_support(rt_hier* h, const uint8_t* vfix) {
    if (!h || !vfix) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    rt_level& L = h->L[0];
    long cnt = 0;
    for (long v = 0; v < L.nv; v++) cnt += vfix[v] != 0;
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->vfix, vfix, L.nv, cudaMemcpyHostToDevice, h->ctx->stream));
    RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    h->has_support = cnt > 0;
    h->graph_epoch++;  // kernel variants depend on whether supports exist
    h->stencil_ready = false;
    h->design_epoch++;
    return RT_OK;
}

// shell elements (HierarchyGrid::setSolidShellElement, grid/Grid.cpp:67-137 marks them):
// level-0 elements whose density the OC update holds at 1 (optimization/optimization.cu:136-162)
extern "C" int rt_set_shell(rt_hier* h, const uint8_t* eshell) {
    if (!h) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    rt_level& L = h->L[0];
    if (!eshell) {
        cudaFree(h->eshell);
        h->eshell = nullptr;
        return RT_OK;
    }
    if (!h->eshell) RT_CHECK(dalloc(h->ctx, &h->eshell, (size_t)L.ne));
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->eshell, eshell, L.ne, cudaMemcpyHostToDevice, h->ctx->stream));
    RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    return RT_OK;
}

// setLoadNodes (optimization/projection.cpp:129-269): rigid modes on the load set,
// normal part only when the direction is constrained, Gram-Schmidt, degenerate dropped
static int load_rigid_basis(rt_hier* h, const int* nodes, const double* normals) {
    const int nl = h->nload;
    const size_t n = 3 * (size_t)nl;
    rt_level& L = h->L[0];
    const bool constrain = (h->P.mode == RT_MODE_NSCF || h->P.mode == RT_MODE_WSCF);
    const bool no_support = (h->P.mode == RT_MODE_NSCF || h->P.mode == RT_MODE_NSFF);
    h->nrig = 0;
    if (!no_support || nl == 0) return RT_OK;
    std::vector<double> R(6 * n, 0.0);
    for (int i = 0; i < nl; i++) {
        const long v = nodes[i];
        const double pz = (double)(v / ((long)L.vx * L.vy)), py = (double)((v / L.vx) % L.vy), px = (double)(v % L.vx);
        const double ph[3][3] = {{0, -pz, py}, {pz, 0, -px}, {-py, px, 0}};
        for (int t = 0; t < 3; t++) R[t * n + 3 * i + t] = 1.0;
        for (int k = 0; k < 3; k++)
            for (int t = 0; t < 3; t++) R[(3 + k) * n + 3 * i + t] = ph[t][k];
    }
    if (constrain)
        for (int k = 0; k < 6; k++)
            for (int i = 0; i < nl; i++) {
                const double* nn = normals + 3 * i;
                double* vv = &R[k * n + 3 * i];
                const double d = vv[0] * nn[0] + vv[1] * nn[1] + vv[2] * nn[2];
                for (int t = 0; t < 3; t++) vv[t] = d * nn[t];
            }
    bool invalid[6] = {false};
    for (int k = 0; k < 6; k++) {
        double* ck = &R[k * n];
        double old = 0;
        for (size_t q = 0; q < n; q++) old += ck[q] * ck[q];
        old = std::sqrt(old);
        for (int j = 0; j < k; j++) {
            if (invalid[j]) continue;
            double w = 0;
            for (size_t q = 0; q < n; q++) w += ck[q] * R[j * n + q];
            for (size_t q = 0; q < n; q++) ck[q] -= w * R[j * n + q];
        }
        double res = 0;
        for (size_t q = 0; q < n; q++) res += ck[q] * ck[q];
        res = std::sqrt(res);
        if (res / old < 1e-6 || old < 1e-6) invalid[k] = true;
        for (size_t q = 0; q < n; q++) ck[q] /= res;
    }
    std::vector<double> Rv;
    for (int k = 0; k < 6; k++)
        if (!invalid[k]) Rv.insert(Rv.end(), R.begin() + k * n, R.begin() + (k + 1) * n);
    h->nrig = (int)(Rv.size() / std::max<size_t>(n, 1));
    if (h->nrig > 0)
        RT_CUDA(h->ctx, cudaMemcpyAsync(h->Rd, Rv.data(), sizeof(double) * Rv.size(), cudaMemcpyHostToDevice,
                                        h->ctx->stream));
    return RT_OK;
}

extern "C" int rt_set_load_nodes(rt_hier* h, int nload, const int* nodes, const double* normals) {
    if (!h || nload < 0 || (nload > 0 && (!nodes || !normals))) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[0];
    for (int i = 0; i < nload; i++)
        if (nodes[i] < 0 || nodes[i] >= L.nv) return rt_fail(c, RT_EINVAL, "load node %d out of range", nodes[i]);
    // keep load nodes sorted (setLoadNodes sorts them, optimization/projection.cpp:139-143)
    std::vector<int> perm(nload);
    for (int i = 0; i < nload; i++) perm[i] = i;
    std::sort(perm.begin(), perm.end(), [&](int a, int b) { return nodes[a] < nodes[b]; });
    std::vector<int> sn(nload);
    std::vector<double> sN(3 * (size_t)nload);
    for (int i = 0; i < nload; i++) {
        sn[i] = nodes[perm[i]];
        for (int t = 0; t < 3; t++) sN[3 * i + t] = normals[3 * perm[i] + t];
    }
    cudaFree(h->load_nodes); cudaFree(h->load_normal); cudaFree(h->Rd); cudaFree(h->fs); cudaFree(h->fs_old);
    h->load_nodes = nullptr; h->load_normal = nullptr; h->Rd = nullptr; h->fs = nullptr; h->fs_old = nullptr;
    h->nload = nload;
    RT_CHECK(dalloc(c, &h->load_nodes, nload));
    RT_CHECK(dalloc(c, &h->load_normal, 3 * (size_t)nload));
    RT_CHECK(dalloc(c, &h->Rd, 6 * 3 * (size_t)nload));
    RT_CHECK(dalloc(c, &h->fs, 3 * (size_t)nload));
    RT_CHECK(dalloc(c, &h->fs_old, 3 * (size_t)nload));
    if (nload > 0) {
        RT_CUDA(c, cudaMemcpyAsync(h->load_nodes, sn.data(), sizeof(int) * nload, cudaMemcpyHostToDevice, c->stream));
        RT_CUDA(c, cudaMemcpyAsync(h->load_normal, sN.data(), sizeof(double) * 3 * nload, cudaMemcpyHostToDevice,
                                   c->stream));
    }
    RT_CHECK(load_rigid_basis(h, sn.data(), sN.data()));
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    return RT_OK;
}

// ---------------------------------------------------------------------------
// fields
// ---------------------------------------------------------------------------
static int field_ptr(rt_hier* h, int field, int lvl, void** ptr, size_t* bytes) {
    if (lvl < 0 || lvl >= (int)h->L.size()) return RT_EINVAL;
    ws_sync(h);
    rt_level& L = h->L[lvl];
    switch (field) {
        case RT_FIELD_U: *ptr = L.u; *bytes = sizeof(double) * 3 * L.nv; return RT_OK;
        case RT_FIELD_F: *ptr = L.f; *bytes = sizeof(double) * 3 * L.nv; return RT_OK;
        case RT_FIELD_R: *ptr = L.r; *bytes = sizeof(double) * 3 * L.nv; return RT_OK;
        case RT_FIELD_STENCIL:
            if (lvl == 0) return RT_EINVAL;
            *ptr = L.st; *bytes = sizeof(double) * 243 * L.nv; return RT_OK;
        case RT_FIELD_VACT: *ptr = L.vact; *bytes = L.nv; return RT_OK;
        case RT_FIELD_EACT: *ptr = L.eact; *bytes = L.ne; return RT_OK;
        case RT_FIELD_RHO: if (lvl) return RT_EINVAL; *ptr = h->rho; *bytes = sizeof(float) * L.ne; return RT_OK;
        case RT_FIELD_SENS: if (lvl) return RT_EINVAL; *ptr = h->sens; *bytes = sizeof(float) * L.ne; return RT_OK;
        case RT_FIELD_VFIX: if (lvl) return RT_EINVAL; *ptr = h->vfix; *bytes = L.nv; return RT_OK;
        case RT_FIELD_PENALTY: if (lvl) return RT_EINVAL; *ptr = h->w; *bytes = sizeof(float) * L.ne; return RT_OK;
    }
    return RT_EINVAL;
}

// reference GS colour order of a level (grid/Grid.cpp:2045-2106): vertices by colour
// x%2 + 2(y%2) + 4(z%2), bit order within a colour, each colour padded to 32
static void ref_gs_order(int vx, int vy, int vz, const std::vector<uint8_t>& act, std::vector<int>& map, int& ngs,
                         int gs_num[8]) {
    long nv = (long)vx * vy * vz;
    int cnt[8] = {0};
    for (long v = 0; v < nv; v++)
        if (act[v]) {
            int x = v % vx, y = (v / vx) % vy, z = v / ((long)vx * vy);
            cnt[(x & 1) + 2 * (y & 1) + 4 * (z & 1)]++;
        }
    int off[8], tot = 0;
    for (int c = 0; c < 8; c++) {
        gs_num[c] = (cnt[c] + 31) / 32 * 32;
        off[c] = tot;
        tot += gs_num[c];
    }
    map.assign(nv, -1);
    int acc[8] = {0};
    for (long v = 0; v < nv; v++)
        if (act[v]) {
            int x = v % vx, y = (v / vx) % vy, z = v / ((long)vx * vy);
            int c = (x & 1) + 2 * (y & 1) + 4 * (z & 1);
            map[v] = off[c] + acc[c]++;
        }
    ngs = tot;
}

extern "C" int rt_ref_gs_map(rt_hier* h, int lvl, int* vidmap, int* n_gs, int* gs_num) {
    if (!h || lvl < 0 || lvl >= (int)h->L.size()) return RT_EINVAL;
    rt_level& L = h->L[lvl];
    std::vector<uint8_t> act(L.nv);
    RT_CUDA(h->ctx, cudaMemcpyAsync(act.data(), L.vact, L.nv, cudaMemcpyDeviceToHost, h->ctx->stream));
    RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    std::vector<int> map;
    int ngs, gn[8];
    ref_gs_order(L.vx, L.vy, L.vz, act, map, ngs, gn);
    if (vidmap) memcpy(vidmap, map.data(), sizeof(int) * L.nv);
    if (n_gs) *n_gs = ngs;
    if (gs_num) memcpy(gs_num, gn, sizeof(gn));
    return RT_OK;
}

// element GS order (colour of the element position, grid/Grid.cu:583-600)
static void ref_gs_order_elems(int nx, int ny, int nz, const std::vector<uint8_t>& act, std::vector<int>& map, int& ngs) {
    int gn[8];
    // element colour uses the same parity rule as vertices
    long ne = (long)nx * ny * nz;
    int cnt[8] = {0};
    for (long e = 0; e < ne; e++)
        if (act[e]) cnt[(e % nx & 1) + 2 * ((e / nx) % ny & 1) + 4 * ((e / ((long)nx * ny)) & 1)]++;
    int off[8], tot = 0;
    for (int c = 0; c < 8; c++) { gn[c] = (cnt[c] + 31) / 32 * 32; off[c] = tot; tot += gn[c]; }
    map.assign(ne, -1);
    int acc[8] = {0};
    for (long e = 0; e < ne; e++)
        if (act[e]) {
            int c = (e % nx & 1) + 2 * ((e / nx) % ny & 1) + 4 * ((e / ((long)nx * ny)) & 1);
            map[e] = off[c] + acc[c]++;
        }
    ngs = tot;
}

static int convert_layout(rt_hier* h, int field, int lvl, bool to_ref, const void* src, void* dst, size_t bytes) {
    rt_level& L = h->L[lvl];
    const bool elem = field == RT_FIELD_RHO || field == RT_FIELD_SENS;
    std::vector<uint8_t> act(elem ? L.ne : L.nv);
    RT_CUDA(h->ctx, cudaMemcpyAsync(act.data(), elem ? L.eact : L.vact, act.size(), cudaMemcpyDeviceToHost, h->ctx->stream));
    RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    std::vector<int> map;
    int ngs, gn[8];
    if (elem) ref_gs_order_elems(L.nx, L.ny, L.nz, act, map, ngs);
    else ref_gs_order(L.vx, L.vy, L.vz, act, map, ngs, gn);
    if (field == RT_FIELD_U || field == RT_FIELD_F || field == RT_FIELD_R) {
        const double* s = (const double*)src;
        double* d = (double*)dst;
        if (to_ref) {
            std::fill(d, d + 3 * (size_t)ngs, 0.0);
            for (long v = 0; v < L.nv; v++)
                if (map[v] >= 0)
                    for (int c = 0; c < 3; c++) d[(size_t)c * ngs + map[v]] = s[c * L.nv + v];
        } else {
            std::fill(d, d + 3 * L.nv, 0.0);
            for (long v = 0; v < L.nv; v++)
                if (map[v] >= 0)
                    for (int c = 0; c < 3; c++) d[c * L.nv + v] = s[(size_t)c * ngs + map[v]];
        }
        return RT_OK;
    }
    if (elem) {
        const float* s = (const float*)src;
        float* d = (float*)dst;
        if (to_ref) {
            std::fill(d, d + ngs, 0.f);
            for (long e = 0; e < L.ne; e++) if (map[e] >= 0) d[map[e]] = s[e];
        } else {
            std::fill(d, d + L.ne, 0.f);
            for (long e = 0; e < L.ne; e++) if (map[e] >= 0) d[e] = s[map[e]];
        }
        return RT_OK;
    }
    (void)bytes;
    return rt_fail(h->ctx, RT_EINVAL, "field has no reference-order layout");
}

extern "C" int rt_put(rt_hier* h, int field, int lvl, int layout, const void* src) {
    if (!h || !src) return RT_EINVAL;
    if (h->parent && field != RT_FIELD_U && field != RT_FIELD_F && field != RT_FIELD_R)
        return rt_fail(h->ctx, RT_ESTATE, "a solve workspace takes only displacement, force and residual fields");
    void* d;
    size_t bytes;
    RT_CHECK(field_ptr(h, field, lvl, &d, &bytes));
    if (layout == RT_LAYOUT_REF_GS) {
        std::vector<char> tmp(bytes);
        RT_CHECK(convert_layout(h, field, lvl, false, src, tmp.data(), bytes));
        RT_CUDA(h->ctx, cudaMemcpyAsync(d, tmp.data(), bytes, cudaMemcpyHostToDevice, h->ctx->stream));
        RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    } else {
        RT_CUDA(h->ctx, cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, h->ctx->stream));
        RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    }
    if (field == RT_FIELD_RHO || field == RT_FIELD_VFIX || field == RT_FIELD_STENCIL) {
        h->stencil_ready = false;
        h->design_epoch++;
    }
    return RT_OK;
}

extern "C" int rt_get(rt_hier* h, int field, int lvl, int layout, void* dst) {
    if (!h || !dst) return RT_EINVAL;
    void* d;
    size_t bytes;
    RT_CHECK(field_ptr(h, field, lvl, &d, &bytes));
    if (layout == RT_LAYOUT_REF_GS) {
        std::vector<char> tmp(bytes);
        RT_CUDA(h->ctx, cudaMemcpyAsync(tmp.data(), d, bytes, cudaMemcpyDeviceToHost, h->ctx->stream));
        RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
        return convert_layout(h, field, lvl, true, tmp.data(), dst, bytes);
    }
    RT_CUDA(h->ctx, cudaMemcpyAsync(dst, d, bytes, cudaMemcpyDeviceToHost, h->ctx->stream));
    RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    return RT_OK;
}

extern "C" int rt_put_dev(rt_hier* h, int field, int lvl, const void* src) {
    if (!h || !src) return RT_EINVAL;
    if (h->parent && field != RT_FIELD_U && field != RT_FIELD_F && field != RT_FIELD_R)
        return rt_fail(h->ctx, RT_ESTATE, "a solve workspace takes only displacement, force and residual fields");
    void* d;
    size_t bytes;
    RT_CHECK(field_ptr(h, field, lvl, &d, &bytes));
    RT_CUDA(h->ctx, cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, h->ctx->stream));
    if (field == RT_FIELD_RHO || field == RT_FIELD_VFIX) {
        h->stencil_ready = false;
        h->design_epoch++;
    }
    return RT_OK;
}

extern "C" int rt_get_dev(rt_hier* h, int field, int lvl, void* dst) {
    if (!h || !dst) return RT_EINVAL;
    void* d;
    size_t bytes;
    RT_CHECK(field_ptr(h, field, lvl, &d, &bytes));
    RT_CUDA(h->ctx, cudaMemcpyAsync(dst, d, bytes, cudaMemcpyDeviceToDevice, h->ctx->stream));
    return RT_OK;
}

__global__ void k_fill_rho(long ne, const uint8_t* __restrict__ eact, float v, float* __restrict__ rho) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ne; e += (long)gridDim.x * blockDim.x)
        rho[e] = eact[e] ? v : 0.f;
}

extern "C" int rt_init_density(rt_hier* h, float rho) {
    if (!h) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    rt_level& L = h->L[0];
    h->stencil_ready = false;
    h->design_epoch++;
    return rt_launch(h->ctx, "init_density", [&] {
        k_fill_rho<<<(unsigned)std::min<long>((L.ne + 255) / 256, 148 * 16), 256, 0, h->ctx->stream>>>(L.ne, L.eact,
                                                                                                       rho, h->rho);
    });
}

// ---------------------------------------------------------------------------
// multigrid
// ---------------------------------------------------------------------------
static int estimate_lmax(rt_hier* h, int lvl);

// element weights rho^p and the inverted diagonal blocks of the finest level
static int refresh_fine(rt_hier* h) {
    if (h->parent) {  // weights and diagonal blocks belong to the parent (refreshed by its own calls)
        ws_sync(h);
        return RT_OK;
    }
    RT_CHECK(rtk::penalty_weights(h));
    return rtk::fine_dinv(h);
}

extern "C" int rt_update_stencil(rt_hier* h) {
    if (!h) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CUDA(h->ctx, cudaSetDevice(h->ctx->device));
    RT_CHECK(refresh_fine(h));
    const int nl = (int)h->L.size();
    for (int i = 1; i < nl; i++) {
        if (i == 1) RT_CHECK(rtk::galerkin_from_elements(h));
        else RT_CHECK(rtk::galerkin_from_stencil(h, i));
        if (h->P.coarse_bf16 && !h->L[i].st16)
            RT_CHECK(dalloc(h->ctx, &h->L[i].st16, 252 * (size_t)((h->L[i].nv + 31) / 32 * 32)));
        RT_CHECK(rtk::stencil_copies(h, i));
    }
    RT_CHECK(rtk::coarsest_setup(h));
    // spectral bound of D^-1 A per smoothed level, for the Chebyshev smoother
    for (int i = 0; i + 1 < nl; i++) RT_CHECK(estimate_lmax(h, i));
    h->stencil_ready = true;
    // a new design: the learned correction gets judged again (the verdict stands while only the
    // stencils of the same design are assembled again)
    if (h->design_epoch != h->unet_verdict_epoch) h->unet_off = false;
    return RT_OK;
}

extern "C" int rt_smoother_lmax(rt_hier* h, int lvl, double* lmax) {
    if (!h || !lmax || lvl < 0 || lvl + 1 >= (int)h->L.size()) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    if (!h->stencil_ready) return rt_fail(h->ctx, RT_ESTATE, "rt_update_stencil has not run");
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->ctx->hscal, h->scal + RT_SCAL_LMAX + lvl, sizeof(double),
                                    cudaMemcpyDeviceToHost, h->ctx->stream));
    RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    *lmax = h->ctx->hscal[0];
    return RT_OK;
}

template <typename T>
struct LvlVec;
template <>
struct LvlVec<double> {
    static double* u(rt_level& L) { return L.u; }
    static double* f(rt_level& L) { return L.f; }
    static double* r(rt_level& L) { return L.r; }
    static double* d(rt_level& L) { return L.d; }
};
template <>
struct LvlVec<float> {
    static float* u(rt_level& L) { return L.u32; }
    static float* f(rt_level& L) { return L.f32; }
    static float* r(rt_level& L) { return L.r32; }
    static float* d(rt_level& L) { return L.d32; }
};

// lmax = sqrt(|x|^2) after the power steps, then the level's Chebyshev coefficient table
__global__ void k_lmax_finish(const double* __restrict__ xx, double* __restrict__ lmax, double* __restrict__ table) {
    if (threadIdx.x == 0 && xx) lmax[0] = sqrt(xx[0]);
    __syncthreads();
    if (threadIdx.x < RT_CHEBY_MAXK) {
        double a, b;
        rt_cheby_coef(lmax[0], threadIdx.x, a, b);
        table[2 * threadIdx.x] = a;
        table[2 * threadIdx.x + 1] = b;
    }
}

// the tables belong to the operator: a workspace reads its parent's
static double* cheby_table(rt_hier* h, int lvl) {
    return (h->parent ? h->parent->scal : h->scal) + RT_SCAL_CHEB + 2 * RT_CHEBY_MAXK * lvl;
}

// v /= s and r /= s with s = sqrt(max(-v.r, tiny)) in slot out (the A-norm of v when r = -A v)
__global__ void k_anorm_scale(long n, const double* __restrict__ vr, double* __restrict__ out, double* __restrict__ v,
                              double* __restrict__ r) {
    const double s = sqrt(fmax(-vr[0], 1e-300));
    if (blockIdx.x == 0 && threadIdx.x == 0 && out) out[0] = s;
    const double is = 1.0 / s;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        v[i] *= is;
        r[i] *= is;
    }
}

// Lanczos step update: w = -w - alpha v - beta_prev vp
__global__ void k_lanczos_w(long n, double* __restrict__ w, const double* __restrict__ v,
                            const double* __restrict__ vp, const double* __restrict__ alpha,
                            const double* __restrict__ beta_prev) {
    const double a = alpha[0], b = beta_prev ? beta_prev[0] : 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        w[i] = -w[i] - a * v[i] - b * vp[i];
}

#define RT_LMAX_STEPS 30

// lmax(D^-1 A) of a smoothed level by RT_LMAX_STEPS Lanczos steps in the A inner product, in which
// M = D^-1 A is self-adjoint (no re-orthogonalisation: only the extreme Ritz value is used).
// r = f - A v with f = 0 gives -A v; one Jacobi step from u = 0 (omega = 1) gives D^-1 r = -M v.
// Step j, with v_j and r_j = -A v_j: w = -D^-1 r_j, alpha_j = r_j . D^-1 r_j,
// w -= alpha_j v_j + beta_{j-1} v_{j-1}, beta_j = |w|_A, v_{j+1} = w / beta_j.  Supported rows
// drop out (r = f = 0 there).  The largest eigenvalue of the tridiagonal matrix and the level's
// Chebyshev table stay on the device.
static int estimate_lmax(rt_hier* h, int lvl) {
    rt_level& L = h->L[lvl];
    rt_ctx* c = h->ctx;
    const long n = 3 * L.nv;
    double *vp = h->x, *v = h->rold, *r = h->q, *w = h->z, *r2 = h->rr, *zero = h->p;
    double* alpha = h->scal + 100;  // [RT_LMAX_STEPS] (the Lanczos eigen-solve's slots; not in use here)
    double* beta = h->scal + 164;
    const unsigned g = (unsigned)std::min<long>((n + 255) / 256, (long)c->sm_count * 16);
    auto residual = [&](const double* x, double* out) {
        return lvl == 0 ? rtk::fine_residual<double>(h, x, zero, out) : rtk::st_residual<double>(h, lvl, x, zero, out);
    };
    auto jacobi = [&](const double* f, double* out) {
        return lvl == 0 ? rtk::fine_jacobi<double>(h, zero, f, out, 1.0) : rtk::st_jacobi<double>(h, lvl, zero, f, out, 1.0);
    };
    RT_CUDA(c, cudaMemsetAsync(zero, 0, sizeof(double) * n, c->stream));
    RT_CUDA(c, cudaMemsetAsync(vp, 0, sizeof(double) * n, c->stream));
    RT_CHECK(rtk::rng_uniform(h, 0x51ab + lvl, n, v));
    RT_CHECK(residual(v, r));
    RT_CHECK(rtk::dot(h, n, v, r, h->scal + 292));
    RT_CHECK(rt_launch(c, "lmax_anorm", [&] { k_anorm_scale<<<g, 256, 0, c->stream>>>(n, h->scal + 292, nullptr, v, r); }));
    for (int it = 0; it < RT_LMAX_STEPS; it++) {
        RT_CHECK(jacobi(r, w));
        RT_CHECK(rtk::dot(h, n, r, w, alpha + it));
        RT_CHECK(rt_launch(c, "lmax_lanczos_w", [&] {
            k_lanczos_w<<<g, 256, 0, c->stream>>>(n, w, v, vp, alpha + it, it > 0 ? beta + it - 1 : nullptr);
        }));
        RT_CHECK(residual(w, r2));
        RT_CHECK(rtk::dot(h, n, w, r2, h->scal + 292));
        RT_CHECK(rt_launch(c, "lmax_anorm",
                           [&] { k_anorm_scale<<<g, 256, 0, c->stream>>>(n, h->scal + 292, beta + it, w, r2); }));
        // rotate: v_{j-1} <- v_j, v_j <- w, r_j <- r2
        std::swap(vp, v);
        std::swap(v, w);
        std::swap(r, r2);
    }
    double* lmax = h->scal + RT_SCAL_LMAX + lvl;
    RT_CHECK(rtk::tridiag_max_eig(h, RT_LMAX_STEPS, alpha, beta, lmax));
    return rt_launch(c, "lmax_finish", [&] {
        k_lmax_finish<<<1, 32, 0, c->stream>>>(nullptr, lmax, cheby_table(h, lvl));
    });
}

template <typename T>
static int level_residual(rt_hier* h, int lvl) {
    rt_level& L = h->L[lvl];
    if (lvl == 0) return rtk::fine_residual<T>(h, LvlVec<T>::u(L), LvlVec<T>::f(L), LvlVec<T>::r(L));
    return rtk::st_residual<T>(h, lvl, LvlVec<T>::u(L), LvlVec<T>::f(L), LvlVec<T>::r(L));
}

template <typename T>
static int level_smooth(rt_hier* h, int lvl, int smoother, int sweeps, double omega, bool backward) {
    rt_level& L = h->L[lvl];
    T* u = LvlVec<T>::u(L);
    T* f = LvlVec<T>::f(L);
    T* tmp = LvlVec<T>::r(L);
    const double* coef = cheby_table(h, lvl);
    if (smoother == RT_SMOOTH_CHEBY && sweeps > RT_CHEBY_MAXK)
        return rt_fail(h->ctx, RT_EINVAL, "Chebyshev smoothing takes at most 16 steps");
    if constexpr (sizeof(T) == 4) {
        // all steps in one cooperative launch where rt_autotune found that faster (not inside a
        // batched graph, whose instances run concurrently)
        if (smoother == RT_SMOOTH_CHEBY && lvl > 0 && sweeps > 0 && ((h->cheby_fused >> lvl) & 1u) &&
            !h->ctx->batch_capture)
            return rtk::st_cheby_fused(h, lvl, u, f, tmp, LvlVec<T>::d(L), coef, sweeps);
    }
    for (int s = 0; s < sweeps; s++) {
        if (smoother == RT_SMOOTH_JACOBI || smoother == RT_SMOOTH_CHEBY) {
            // ping-pong u -> tmp -> u
            const T* src = (s % 2 == 0) ? u : tmp;
            T* dst = (s % 2 == 0) ? tmp : u;
            if (smoother == RT_SMOOTH_CHEBY) {
                T* d = LvlVec<T>::d(L);
                if (lvl == 0) RT_CHECK(rtk::fine_cheby<T>(h, src, f, dst, d, coef, s));
                else RT_CHECK(rtk::st_cheby<T>(h, lvl, src, f, dst, d, coef, s));
            } else {
                if (lvl == 0) RT_CHECK(rtk::fine_jacobi<T>(h, src, f, dst, omega));
                else RT_CHECK(rtk::st_jacobi<T>(h, lvl, src, f, dst, omega));
            }
        } else {
            if (lvl == 0) RT_CHECK(rtk::fine_gs<T>(h, u, f, backward));
            else RT_CHECK(rtk::st_gs<T>(h, lvl, u, f, backward));
        }
    }
    if ((smoother == RT_SMOOTH_JACOBI || smoother == RT_SMOOTH_CHEBY) && (sweeps % 2) == 1)
        RT_CUDA(h->ctx, cudaMemcpyAsync(u, tmp, sizeof(T) * 3 * L.nv, cudaMemcpyDeviceToDevice, h->ctx->stream));
    return RT_OK;
}

// the multigrid cycle from level i down (level i's u is the caller's initial guess): smoothing,
// the coarse correction (cycle_gamma times on levels 1 .. cycle_gamma_levels (all when 0) unless
// the next level is the coarsest, whose solve is exact: gamma = 2 is the W-cycle), smoothing;
// pre/post mirror each other, so the
// cycle is symmetric when the smoother is (SGS, Jacobi, Chebyshev)
template <typename T>
static int mg_cycle(rt_hier* h, int i, int smoother, int pre, int post, double omega) {
    const int nl = (int)h->L.size();
    if (i == nl - 1) return rtk::coarsest_solve<T>(h, LvlVec<T>::f(h->L[i]), LvlVec<T>::u(h->L[i]));
    const int cs = h->P.coarse_sweeps;
    const int npre = (i > 0 && cs > 0) ? cs : pre, npost = (i > 0 && cs > 0) ? cs : post;
    RT_CHECK(level_smooth<T>(h, i, smoother, npre, omega, false));
    const int gl = h->P.cycle_gamma_levels;
    const int reps = (i > 0 && i + 1 < nl - 1 && h->P.cycle_gamma > 1 && (gl <= 0 || i <= gl)) ? h->P.cycle_gamma : 1;
    for (int g = 0; g < reps; g++) {
        RT_CHECK(level_residual<T>(h, i));
        RT_CHECK(rtk::restrict_<T>(h, i + 1, LvlVec<T>::r(h->L[i]), LvlVec<T>::f(h->L[i + 1])));
        RT_CUDA(h->ctx,
                cudaMemsetAsync(LvlVec<T>::u(h->L[i + 1]), 0, sizeof(T) * 3 * h->L[i + 1].nv, h->ctx->stream));
        RT_CHECK(mg_cycle<T>(h, i + 1, smoother, pre, post, omega));
        RT_CHECK(rtk::prolong_add<T>(h, i, LvlVec<T>::u(h->L[i + 1]), LvlVec<T>::u(h->L[i])));
    }
    return level_smooth<T>(h, i, smoother, npost, omega, smoother == RT_SMOOTH_SGS);
}

// HierarchyGrid::v_cycle (grid/Grid.cpp:1068-1113) over levels l0 .. coarsest
template <typename T>
static int vcycle_T(rt_hier* h, int smoother, int pre, int post, double omega, int l0 = 0) {
    return mg_cycle<T>(h, l0, smoother, pre, post, omega);
}

static int read_scalars(rt_hier* h, int first, int count, double* out) {
    rt_ctx* c = h->ctx;
    RT_CUDA(c, cudaMemcpyAsync(c->hscal, h->scal + first, sizeof(double) * count, cudaMemcpyDeviceToHost, c->stream));
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    memcpy(out, c->hscal, sizeof(double) * count);
    return RT_OK;
}

static int need_stencil(rt_hier* h) {
    ws_sync(h);
    if (!h->stencil_ready) return rt_fail(h->ctx, RT_ESTATE, "rt_update_stencil must run after the density or supports change");
    return RT_OK;
}

extern "C" int rt_vcycle(rt_hier* h, int pre, int post, double* rel_res) {
    if (!h || pre < 0 || post < 0) return RT_EINVAL;
    RT_CHECK(need_stencil(h));
    RT_CHECK(vcycle_T<double>(h, RT_SMOOTH_GS, pre, post, h->P.jacobi_omega));
    rt_level& L = h->L[0];
    RT_CHECK(rtk::fine_residual<double>(h, L.u, L.f, L.r));
    if (rel_res) {
        RT_CHECK(rtk::dot(h, 3 * L.nv, L.r, L.r, h->scal + 0));
        RT_CHECK(rtk::dot(h, 3 * L.nv, L.f, L.f, h->scal + 1));
        double s[2];
        RT_CHECK(read_scalars(h, 0, 2, s));
        *rel_res = std::sqrt(s[0]) / std::sqrt(s[1]);
    }
    return RT_OK;
}

extern "C" int rt_update_residual(rt_hier* h, int lvl) {
    if (!h || lvl < 0 || lvl >= (int)h->L.size()) return RT_EINVAL;
    if (lvl > 0) RT_CHECK(need_stencil(h));
    else RT_CHECK(refresh_fine(h));
    return level_residual<double>(h, lvl);
}

extern "C" int rt_smooth(rt_hier* h, int lvl, int smoother, int sweeps, double omega) {
    if (!h || lvl < 0 || lvl >= (int)h->L.size() || sweeps < 0) return RT_EINVAL;
    if (lvl > 0) RT_CHECK(need_stencil(h));
    else RT_CHECK(refresh_fine(h));
    return level_smooth<double>(h, lvl, smoother, sweeps, omega, smoother == RT_SMOOTH_SGS);
}

static int nan_fail(rt_hier* h, int it);

extern "C" int rt_smooth_f32(rt_hier* h, int lvl, int smoother, int sweeps, double omega) {
    if (!h || lvl < 0 || lvl + 1 >= (int)h->L.size() || sweeps < 0) return RT_EINVAL;
    if (smoother != RT_SMOOTH_JACOBI && smoother != RT_SMOOTH_CHEBY)
        return rt_fail(h->ctx, RT_EINVAL, "FP32 smoothing: Jacobi or Chebyshev");
    if (lvl > 0) RT_CHECK(need_stencil(h));
    else RT_CHECK(refresh_fine(h));
    if (smoother == RT_SMOOTH_CHEBY && !h->stencil_ready) return rt_fail(h->ctx, RT_ESTATE, "rt_update_stencil has not run");
    rt_level& L = h->L[lvl];
    const long n = 3 * L.nv;
    RT_CHECK(rtk::d2f(h, n, L.u, L.u32));
    RT_CHECK(rtk::d2f(h, n, L.f, L.f32));
    RT_CHECK(level_smooth<float>(h, lvl, smoother, sweeps, omega, false));
    RT_CHECK(rtk::f2d(h, n, L.u32, L.u));
    double e = 0;
    RT_CHECK(read_scalars(h, RT_SCAL_ERR, 1, &e));
    if (e != 0.0) return nan_fail(h, 0);
    return RT_OK;
}

extern "C" int rt_restrict_residual(rt_hier* h, int lvl) {
    if (!h || lvl < 1 || lvl >= (int)h->L.size()) return RT_EINVAL;
    ws_sync(h);
    return rtk::restrict_<double>(h, lvl, h->L[lvl - 1].r, h->L[lvl].f);
}

extern "C" int rt_prolongate_correction(rt_hier* h, int lvl) {
    if (!h || lvl < 0 || lvl + 1 >= (int)h->L.size()) return RT_EINVAL;
    ws_sync(h);
    return rtk::prolong_add<double>(h, lvl, h->L[lvl + 1].u, h->L[lvl].u);
}

extern "C" int rt_coarsest_solve(rt_hier* h) {
    if (!h) return RT_EINVAL;
    RT_CHECK(need_stencil(h));
    rt_level& L = h->L.back();
    return rtk::coarsest_solve<double>(h, L.f, L.u);
}

extern "C" int rt_apply_K_dev(rt_hier* h, const double* u, double* out) {
    if (!h || !u || !out) return RT_EINVAL;
    RT_CHECK(refresh_fine(h));
    return rtk::fine_applyK<double>(h, u, out);
}

extern "C" int rt_apply_K(rt_hier* h, const double* u, double* out) {
    if (!h || !u || !out) return RT_EINVAL;
    rt_level& L = h->L[0];
    const size_t b = sizeof(double) * 3 * L.nv;
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->x, u, b, cudaMemcpyHostToDevice, h->ctx->stream));
    RT_CHECK(rt_apply_K_dev(h, h->x, h->q));
    RT_CUDA(h->ctx, cudaMemcpyAsync(out, h->q, b, cudaMemcpyDeviceToHost, h->ctx->stream));
    RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    return RT_OK;
}

extern "C" int rt_compliance(rt_hier* h, double* cpl) {
    if (!h || !cpl) return RT_EINVAL;
    rt_level& L = h->L[0];
    RT_CHECK(rtk::dot(h, 3 * L.nv, L.f, L.u, h->scal + 2));
    return read_scalars(h, 2, 1, cpl);
}

// ---------------------------------------------------------------------------
// projection API (optimization/projection.h:16-65) and element compliance
// ---------------------------------------------------------------------------
__global__ void k_support_gather_soa(int nload, long nv, const int* __restrict__ nodes, const double* __restrict__ f,
                                     double* __restrict__ fs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nload; i += gridDim.x * blockDim.x) {
        const long v = nodes[i];
        fs[i] = f[v];
        fs[nload + i] = f[nv + v];
        fs[2 * nload + i] = f[2 * nv + v];
    }
}

__global__ void k_support_scatter_soa(int nload, long nv, const int* __restrict__ nodes,
                                      const double* __restrict__ fs, double* __restrict__ f) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nload; i += gridDim.x * blockDim.x) {
        const long v = nodes[i];
        f[v] = fs[i];
        f[nv + v] = fs[nload + i];
        f[2 * nv + v] = fs[2 * nload + i];
    }
}

static unsigned load_blocks(const rt_hier* h) {
    return (unsigned)std::max(1, std::min((h->nload + 255) / 256, h->ctx->sm_count * 8));
}

extern "C" int rt_force_project(rt_hier* h, double* f_dev) {
    if (!h || !f_dev) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    if (h->nload == 0) return rt_fail(h->ctx, RT_ESTATE, "forceProject: no load nodes (rt_set_load_nodes)");
    return rtk::project_load(h, f_dev);
}

extern "C" int rt_get_force_support(rt_hier* h, const double* f_dev, double* fs_dev) {
    if (!h || !f_dev || !fs_dev) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    if (h->nload == 0) return RT_OK;
    return rt_launch(h->ctx, "support_gather", [&] {
        k_support_gather_soa<<<load_blocks(h), 256, 0, h->ctx->stream>>>(h->nload, h->L[0].nv, h->load_nodes, f_dev,
                                                                         fs_dev);
    });
}

extern "C" int rt_set_force_support(rt_hier* h, const double* fs_dev, double* f_dev) {
    if (!h || !fs_dev || !f_dev) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CUDA(h->ctx, cudaMemsetAsync(f_dev, 0, sizeof(double) * 3 * h->L[0].nv, h->ctx->stream));
    if (h->nload == 0) return RT_OK;
    return rt_launch(h->ctx, "support_scatter", [&] {
        k_support_scatter_soa<<<load_blocks(h), 256, 0, h->ctx->stream>>>(h->nload, h->L[0].nv, h->load_nodes, fs_dev,
                                                                          f_dev);
    });
}

extern "C" int rt_displacement_project(rt_hier* h, double* u_dev) {
    if (!h || !u_dev) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    if (h->P.mode != RT_MODE_NSCF && h->P.mode != RT_MODE_NSFF) return RT_OK;  // supports fix the rigid modes
    if (h->Ru == nullptr) RT_CHECK(rtk::rigid_nodes(h));
    return rtk::displacement_project(h, u_dev);
}

extern "C" int rt_load_nodes(rt_hier* h, int* n, int* nodes) {
    if (!h || !n) return RT_EINVAL;
    *n = h->nload;
    if (nodes && h->nload > 0) {
        RT_CUDA(h->ctx, cudaMemcpyAsync(nodes, h->load_nodes, sizeof(int) * h->nload, cudaMemcpyDeviceToHost,
                                        h->ctx->stream));
        RT_CUDA(h->ctx, cudaStreamSynchronize(h->ctx->stream));
    }
    return RT_OK;
}

extern "C" int rt_element_compliance(rt_hier* h, const double* u_dev, float* ce_dev) {
    if (!h || !u_dev || !ce_dev) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    return rtk::element_compliance(h, u_dev, ce_dev);
}

extern "C" int rt_relative_residual(rt_hier* h, double* rel) {
    if (!h || !rel) return RT_EINVAL;
    rt_level& L = h->L[0];
    RT_CHECK(rtk::dot(h, 3 * L.nv, L.r, L.r, h->scal + 0));
    RT_CHECK(rtk::dot(h, 3 * L.nv, L.f, L.f, h->scal + 1));
    double s[2];
    RT_CHECK(read_scalars(h, 0, 2, s));
    *rel = std::sqrt(s[0]) / std::sqrt(s[1]);
    return RT_OK;
}

// ---------------------------------------------------------------------------
// MG-preconditioned flexible CG on level 0: x = L0.u (initial guess), b = L0.f
// scal slots: 10..13 r.z / rold.z (two parities), 20 p.q, 21 r.r, 22 b.b
// ---------------------------------------------------------------------------
// z = B r (the V-cycle, plus the learned correction when attached).  When dots is given and the
// form allows it, the FP32 path also leaves (z.r, z.rold) in dots[0..1] (fused with the widening
// of z) and returns with *dots_done set.
// the FP32 right-hand side of the V-cycle comes out of the x / r update (scaled by the r.r
// before that update, kept in scal[23]) instead of a separate conversion pass
static bool fused_f32_rhs(const rt_hier* h) { return h->P.precision == RT_FP32 && !h->P.krylov_fp32; }

// gate of the learned correction: counts the corrections run (scal[36]) and, inside a captured
// loop, sets the IF node that holds them
__global__ void k_learned_gate(const double* __restrict__ gate, double* __restrict__ count,
                               cudaGraphConditionalHandle hc, int use_cond) {
    if (threadIdx.x != 0) return;
    const bool on = gate[0] != 0.0;
    if (on) count[0] += 1.0;
    if (use_cond) cudaGraphSetConditional(hc, on ? 1u : 0u);
}

// runs fn's launches only while the gate scal[28] is on.  Inside a stream capture they become
// the body of an IF conditional node (captured on the context's auxiliary stream), so a loop
// whose gate went off launches none of them; outside a capture the gate is read on the host.
template <typename F>
static int learned_if(rt_hier* h, F&& fn) {
    rt_ctx* c = h->ctx;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    RT_CUDA(c, cudaStreamIsCapturing(c->stream, &cs));
    if (cs != cudaStreamCaptureStatusActive) {
        RT_CHECK(rt_launch(c, "learned_gate", [&] { k_learned_gate<<<1, 32, 0, c->stream>>>(h->scal + 28, h->scal + 36, 0, 0); }));
        double g = 0;
        RT_CHECK(read_scalars(h, 28, 1, &g));
        return g != 0.0 ? fn() : RT_OK;
    }
    if (!c->aux_stream) return rt_fail(c, RT_ESTATE, "learned correction captured without an auxiliary stream");
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    RT_CUDA(c, cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphConditionalHandle hc;
    RT_CUDA(c, cudaGraphConditionalHandleCreate(&hc, cg, 0, cudaGraphCondAssignDefault));
    RT_CHECK(rt_launch(c, "learned_gate", [&] { k_learned_gate<<<1, 32, 0, c->stream>>>(h->scal + 28, h->scal + 36, hc, 1); }));
    RT_CUDA(c, cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hc;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t ifn;
    RT_CUDA(c, cudaGraphAddNode(&ifn, cg, deps, nd, &cp));
    RT_CUDA(c, cudaStreamUpdateCaptureDependencies(c->stream, &ifn, 1, cudaStreamSetCaptureDependencies));
    RT_CUDA(c, cudaStreamBeginCaptureToGraph(c->aux_stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
    cudaStream_t saved = c->stream;
    c->stream = c->aux_stream;
    const long l0 = c->launches;
    const int st = fn();
    // the body's kernels are counted when they run (scal[36] corrections), not per iteration
    h->unet_kernels = c->launches - l0;
    c->launches = l0;
    c->stream = saved;
    cudaGraph_t body = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->aux_stream, &body);
    RT_CHECK(st);
    if (e != cudaSuccess) return rt_fail(c, RT_ECUDA, "capture of the learned correction failed: %s", cudaGetErrorString(e));
    return RT_OK;
}

// z = M^-1 r.  rr_dev: the scale (r.r of the residual the FP32 copy was made from);
// f32_ready: level 0's FP32 right-hand side already holds r / sqrt(rr_dev)
static int precondition(rt_hier* h, const double* r, double* z, const double* rr_dev, double* dots = nullptr,
                        bool* dots_done = nullptr, bool f32_ready = false) {
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    if (dots_done) *dots_done = false;
    if (h->P.precision == RT_FP32) {
        if (!f32_ready) RT_CHECK(rtk::d2f_scaled(h, n, r, L.f32, rr_dev));
        RT_CUDA(h->ctx, cudaMemsetAsync(L.u32, 0, sizeof(float) * n, h->ctx->stream));
        RT_CHECK(vcycle_T<float>(h, h->P.smoother, h->P.pre_sweeps, h->P.post_sweeps, h->P.jacobi_omega));
        if (dots) {
            RT_CHECK(rtk::f2d_scaled_dot2(h, n, L.u32, z, rr_dev, r, h->rold, dots));
            *dots_done = true;
        } else {
            RT_CHECK(rtk::f2d_scaled(h, n, L.u32, z, rr_dev));
        }
    } else if (h->P.precision == RT_FP64_FINE && h->L.size() > 1) {
        // FP64 smoothing and residual on the finest level (on r / z themselves), the coarse
        // V-cycle in FP32 on the restricted residual scaled by 1 / |r|, its correction added back
        double* saved_f = L.f;
        double* saved_u = L.u;
        L.f = const_cast<double*>(r);
        L.u = z;
        rt_level& L1 = h->L[1];
        int s = RT_OK;
        auto step = [&](int st) { if (s == RT_OK) s = st; };
        if (cudaMemsetAsync(z, 0, sizeof(double) * n, h->ctx->stream) != cudaSuccess) s = RT_ECUDA;
        step(level_smooth<double>(h, 0, h->P.smoother, h->P.pre_sweeps, h->P.jacobi_omega, false));
        step(level_residual<double>(h, 0));
        step(rtk::d2f_scaled(h, n, L.r, L.r32, rr_dev));
        step(rtk::restrict_<float>(h, 1, L.r32, L1.f32));
        if (s == RT_OK && cudaMemsetAsync(L1.u32, 0, sizeof(float) * 3 * L1.nv, h->ctx->stream) != cudaSuccess)
            s = RT_ECUDA;
        step(vcycle_T<float>(h, h->P.smoother, h->P.pre_sweeps, h->P.post_sweeps, h->P.jacobi_omega, 1));
        if (s == RT_OK && cudaMemsetAsync(L.u32, 0, sizeof(float) * n, h->ctx->stream) != cudaSuccess) s = RT_ECUDA;
        step(rtk::prolong_add<float>(h, 0, L1.u32, L.u32));
        step(rtk::f2d_scaled_add(h, n, L.u32, z, rr_dev));
        step(level_smooth<double>(h, 0, h->P.smoother, h->P.post_sweeps, h->P.jacobi_omega,
                                  h->P.smoother == RT_SMOOTH_SGS));
        L.f = saved_f;
        L.u = saved_u;
        if (s == RT_ECUDA) return rt_fail(h->ctx, RT_ECUDA, "hybrid V-cycle memset failed");
        RT_CHECK(s);
    } else {
        // run the FP64 V-cycle on level-0 f/u, using r/z as the level-0 vectors
        double* saved_f = L.f;
        double* saved_u = L.u;
        L.f = const_cast<double*>(r);
        L.u = z;
        RT_CUDA(h->ctx, cudaMemsetAsync(z, 0, sizeof(double) * n, h->ctx->stream));
        int s = vcycle_T<double>(h, h->P.smoother, h->P.pre_sweeps, h->P.post_sweeps, h->P.jacobi_omega);
        L.f = saved_f;
        L.u = saved_u;
        RT_CHECK(s);
    }
    // learned correction z += N(rho, r, z), run only while the gate in scal[28] is on; the dots
    // the widening of z already produced are recomputed for the corrected z.  Once the gate has
    // judged the network off for this design, the loop is captured without it: a conditional
    // node inside the captured loop body slows every iteration's launches, even when it skips
    if (h->unet && !h->unet_off)
        RT_CHECK(learned_if(h, [&]() -> int {
            RT_CHECK(rtk::dot(h, n, r, r, h->scal + 38));
            RT_CHECK(rtk::dot(h, n, z, z, h->scal + 37));
            RT_CHECK(rtu::correct(h->unet, h, r, h->scal + 38, h->scal + 37, h->scal + 28, z));
            if (h->unet_post > 0) {
                // smoothing steps on K z = r from the corrected z: damp what the network adds
                // at high frequencies, where K is largest
                double* saved_f = L.f;
                double* saved_u = L.u;
                L.f = const_cast<double*>(r);
                L.u = z;
                const int st = level_smooth<double>(h, 0, h->P.smoother, h->unet_post, h->P.jacobi_omega, false);
                L.f = saved_f;
                L.u = saved_u;
                RT_CHECK(st);
            }
            return (dots_done && *dots_done) ? rtk::dot2(h, n, z, r, h->rold, dots) : RT_OK;
        }));
    return RT_OK;
}

// p = z + beta p, flexible beta = (z.r - z.rold) / rz_prev; beta = 0 on the first iteration
__global__ void k_pcg_p_it(long n, const double* __restrict__ s, const double* __restrict__ it, double* __restrict__ p,
                           const double* __restrict__ z) {
    const bool first = it[0] == 0.0;
    const double den = s[2];
    const double beta = (first || den == 0.0) ? 0.0 : (s[0] - s[1]) / den;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = first ? z[i] : z[i] + beta * p[i];
}

// end of an iteration: it += 1, rz_prev = rz; optionally set the WHILE condition of the graph
__global__ void k_pcg_tail(double* __restrict__ scal, cudaGraphConditionalHandle cond, int use_cond) {
    if (threadIdx.x != 0) return;
    const double it = scal[24] + 1.0;
    scal[24] = it;
    scal[12] = scal[10];
    // learned-correction fallback: off for the rest of the solve once an iteration's residual
    // norm did not drop below ratio x the previous one
    if (scal[28] != 0.0 && scal[29] > 0.0 && !(scal[21] <= scal[27] * scal[27] * scal[29])) scal[28] = 0.0;
    scal[29] = scal[21];
    // precision fallback: the loop ends once |r| has not halved within scal[93] iterations (0: off);
    // scal[90] is the last halving's r.r, scal[91] its iteration, scal[92] the flag
    bool stalled = false;
    if (scal[93] > 0.0) {
        if (scal[21] <= 0.25 * scal[90]) {
            scal[90] = scal[21];
            scal[91] = it;
        } else if (it - scal[91] >= scal[93]) {
            scal[92] = 1.0;
            stalled = true;
        }
    }
    if (use_cond) {
        const double rr = scal[21], bb = scal[22] > 0 ? scal[22] : 1.0;
        const bool go = isfinite(rr) && sqrt(rr) > scal[25] * sqrt(bb) && it < scal[26] && !stalled;
        cudaGraphSetConditional(cond, go ? 1u : 0u);
    }
}

// one MG-PCG iteration, all scalars on the device (graph-capturable):
// scal[10] z.r, [11] z.rold, [12] previous z.r, [20] p.q, [21] r.r, [24] iteration
static int pcg_body(rt_hier* h, double* x, double* r, bool no_support, cudaGraphConditionalHandle cond,
                    int use_cond = 0) {
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    rt_ctx* c = h->ctx;
    bool dots_done = false;
    const bool fz = fused_f32_rhs(h);
    // the projection of z (no supports) must precede its dots: no fusion then
    RT_CHECK(precondition(h, r, h->z, h->scal + (fz ? 23 : 21), no_support ? nullptr : h->scal + 10, &dots_done, fz));
    if (no_support) RT_CHECK(rtk::displacement_project(h, h->z));
    if (!dots_done) RT_CHECK(rtk::dot2(h, n, h->z, r, h->rold, h->scal + 10));
    RT_CHECK(rt_launch(c, "pcg_update_p", [&] {
        k_pcg_p_it<<<(unsigned)std::min<long>((n + 255) / 256, (long)c->sm_count * 16), 256, 0, c->stream>>>(
            n, h->scal + 10, h->scal + 24, h->p, h->z);
    }));
    RT_CHECK(rtk::fine_applyK<double>(h, h->p, h->q));
    RT_CHECK(rtk::dot(h, n, h->p, h->q, h->scal + 20));
    RT_CHECK(rtk::pcg_update_xr_rr(h, n, h->scal + 10, h->scal + 20, x, r, h->p, h->q, h->rold, h->scal + 21,
                                   fz ? L.f32 : nullptr, h->scal + 23));
    return rt_launch(c, "pcg_tail", [&] { k_pcg_tail<<<1, 32, 0, c->stream>>>(h->scal, cond, use_cond); });
}

// the whole iteration loop as one graph: a WHILE conditional node whose body is one
// captured iteration; the body's last kernel decides whether to run again
static int pcg_graph_run(rt_hier* h, double* x, double* r, bool no_support) {
    rt_ctx* c = h->ctx;
    // the captured graph depends on the vectors, the solver settings, the operator epoch (launch
    // shapes, kernel variants, parameter changes) and the learned correction
    uint64_t key = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { key = (key ^ v) * 1099511628211ull; };
    mix((uint64_t)(uintptr_t)x);
    mix((uint64_t)(uintptr_t)h->unet);
    mix((uint64_t)h->unet_off);
    mix(h->graph_epoch);
    mix((uint64_t)c->wait_limit);
    mix((uint64_t)no_support);
    mix((uint64_t)h->P.precision | ((uint64_t)h->P.smoother << 8) | ((uint64_t)h->P.pre_sweeps << 16) |
        ((uint64_t)h->P.post_sweeps << 24) | ((uint64_t)h->P.cycle_gamma << 32) |
        ((uint64_t)h->P.coarse_sweeps << 40) | ((uint64_t)h->P.coarse_bf16 << 48));
    mix((uint64_t)(uint32_t)h->P.cycle_gamma_levels);
    uint64_t om;
    memcpy(&om, &h->P.jacobi_omega, 8);
    mix(om);
    if ((!h->pcg_exec || h->pcg_key != key) && h->pcg_exec_alt && h->pcg_key_alt == key) {
        std::swap(h->pcg_exec, h->pcg_exec_alt);
        std::swap(h->pcg_graph, h->pcg_graph_alt);
        std::swap(h->pcg_key, h->pcg_key_alt);
        std::swap(h->pcg_iter_kernels, h->pcg_iter_kernels_alt);
    }
    if (!h->pcg_exec || h->pcg_key != key) {
        // the current graph becomes the alternate one; the older alternate is released
        if (h->pcg_exec_alt) cudaGraphExecDestroy(h->pcg_exec_alt);
        if (h->pcg_graph_alt) cudaGraphDestroy(h->pcg_graph_alt);
        h->pcg_exec_alt = h->pcg_exec;
        h->pcg_graph_alt = h->pcg_graph;
        h->pcg_key_alt = h->pcg_key;
        h->pcg_iter_kernels_alt = h->pcg_iter_kernels;
        h->pcg_exec = nullptr;
        h->pcg_graph = nullptr;
        if (h->unet && !c->aux_stream) RT_CUDA(c, cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking));
        cudaGraph_t g;
        RT_CUDA(c, cudaGraphCreate(&g, 0));
        cudaGraphConditionalHandle cond;
        RT_CUDA(c, cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        RT_CUDA(c, cudaGraphAddNode(&node, g, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        RT_CUDA(c, cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        // captured launches are counted when the graph runs, once per executed iteration
        const long l0 = c->launches;
        int s = pcg_body(h, x, r, no_support, cond, 1);
        h->pcg_iter_kernels = c->launches - l0;
        c->launches = l0;
        cudaGraph_t captured = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &captured);
        if (s != RT_OK) { cudaGraphDestroy(g); return s; }
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return rt_fail(c, RT_ECUDA, "PCG graph capture failed: %s", cudaGetErrorString(e));
        }
        cudaGraphExec_t exec;
        e = cudaGraphInstantiate(&exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return rt_fail(c, RT_ECUDA, "PCG graph instantiation failed: %s", cudaGetErrorString(e));
        }
        h->pcg_graph = g;
        h->pcg_exec = exec;
        h->pcg_key = key;
    }
    RT_CUDA(c, cudaGraphLaunch(h->pcg_exec, c->stream));
    return RT_OK;
}

// r = b - K x (identity rows on supports), rold = 0, scal[22] = b.b, scal[21] = r.r (graph-capturable)
static int pcg_prologue(rt_hier* h, double* x, const double* b) {
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    double* r = h->rr;
    RT_CHECK(rtk::fine_applyK<double>(h, x, h->q));
    RT_CUDA(h->ctx, cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->ctx->stream));
    RT_CHECK(rtk::axpy(h, n, -1.0, h->q, r));
    RT_CHECK(rtk::mask_copy(h, n, r, r));
    RT_CUDA(h->ctx, cudaMemsetAsync(h->rold, 0, sizeof(double) * n, h->ctx->stream));
    RT_CHECK(rtk::dot(h, n, b, b, h->scal + 22));
    RT_CHECK(rtk::dot(h, n, r, r, h->scal + 21));
    if (!fused_f32_rhs(h)) return RT_OK;
    // the first iteration's FP32 right-hand side and its scale (later ones come from the x / r update)
    RT_CHECK(rtk::d2f_scaled(h, n, r, L.f32, h->scal + 21));
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->scal + 23, h->scal + 21, sizeof(double), cudaMemcpyDeviceToDevice, h->ctx->stream));
    return RT_OK;
}

// a solve that produced NaN: a stencil kernel whose bounded copy wait ran out writes NaN and
// flags RT_SCAL_ERR, anything else is a numerical breakdown
static int nan_fail(rt_hier* h, int it) {
    double e = 0;
    RT_CHECK(read_scalars(h, RT_SCAL_ERR, 1, &e));
    if (e != 0.0) {
        RT_CUDA(h->ctx, cudaMemsetAsync(h->scal + RT_SCAL_ERR, 0, sizeof(double), h->ctx->stream));
        RT_CUDA(h->ctx, cudaMemsetAsync(h->scal + RT_SCAL_GBAR, 0, sizeof(double) * RT_MAX_LEVELS, h->ctx->stream));
        if (e == 3.0)
            return rt_fail(h->ctx, RT_ECUDA, "a finest-level kernel gave up waiting for its TMA node-layer copies (iteration %d)", it);
        return rt_fail(h->ctx, RT_ECUDA, e == 2.0 ? "a fused Chebyshev sweep gave up at its grid barrier (iteration %d)"
                                                  : "a stencil-level kernel gave up waiting for its bulk copies (iteration %d)",
                       it);
    }
    return rt_fail(h->ctx, RT_ENAN, "NaN in PCG at iteration %d", it);
}

// ---------------------------------------------------------------------------
// FP32 Krylov form (rt_params.krylov_fp32 with precision RT_FP32): flexible CG whose vectors,
// operator products and V-cycles are all FP32 (every dot product summed in FP64), solving
// K d = r / |r| for the FP64 residual r = b - K x; x += |r| d, then the FP64 residual is
// recomputed and the next inner solve starts from it (iterative refinement)
// ---------------------------------------------------------------------------
static int ensure_krylov32(rt_hier* h) {
    if (h->p32k) return RT_OK;
    const size_t n = 3 * (size_t)h->L[0].nv;
    RT_CHECK(dalloc(h->ctx, &h->p32k, n));
    RT_CHECK(dalloc(h->ctx, &h->q32k, n));
    RT_CHECK(dalloc(h->ctx, &h->d32k, n));
    return dalloc(h->ctx, &h->ro32k, n);
}

// one inner iteration: z = V(res) (res is level 0's FP32 right-hand side, z its FP32 solution),
// flexible beta, p, q = K p, alpha, d += alpha p, res -= alpha q, then the loop test
static int pcg32_body(rt_hier* h, cudaGraphConditionalHandle cond, int use_cond) {
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    rt_ctx* c = h->ctx;
    RT_CUDA(c, cudaMemsetAsync(L.u32, 0, sizeof(float) * n, c->stream));
    RT_CHECK(vcycle_T<float>(h, h->P.smoother, h->P.pre_sweeps, h->P.post_sweeps, h->P.jacobi_omega));
    RT_CHECK(rtk::dot32_2(h, n, L.u32, L.f32, h->ro32k, h->scal + 10));
    RT_CHECK(rtk::pcg32_update_p(h, n, h->scal + 10, h->scal + 24, h->p32k, L.u32));
    RT_CHECK(rtk::fine_applyK<float>(h, h->p32k, h->q32k));
    RT_CHECK(rtk::dot32(h, n, h->p32k, h->q32k, h->scal + 20));
    RT_CHECK(rtk::pcg32_update_xr_rr(h, n, h->scal + 10, h->scal + 20, h->d32k, L.f32, h->p32k, h->q32k, h->ro32k,
                                     h->scal + 21));
    return rt_launch(c, "pcg_tail", [&] { k_pcg_tail<<<1, 32, 0, c->stream>>>(h->scal, cond, use_cond); });
}

// the inner loop as one graph with a WHILE conditional node (as pcg_graph_run)
static int pcg32_graph_run(rt_hier* h) {
    rt_ctx* c = h->ctx;
    uint64_t key = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { key = (key ^ v) * 1099511628211ull; };
    mix(h->graph_epoch);
    mix((uint64_t)c->wait_limit);
    mix((uint64_t)h->P.smoother | ((uint64_t)h->P.pre_sweeps << 8) | ((uint64_t)h->P.post_sweeps << 16) |
        ((uint64_t)h->P.cycle_gamma << 24) | ((uint64_t)h->P.coarse_sweeps << 32) | ((uint64_t)h->P.coarse_bf16 << 40));
    mix((uint64_t)(uint32_t)h->P.cycle_gamma_levels);
    uint64_t om;
    memcpy(&om, &h->P.jacobi_omega, 8);
    mix(om);
    if (!h->pcg32_exec || h->pcg32_key != key) {
        if (h->pcg32_exec) { cudaGraphExecDestroy(h->pcg32_exec); h->pcg32_exec = nullptr; }
        if (h->pcg32_graph) { cudaGraphDestroy(h->pcg32_graph); h->pcg32_graph = nullptr; }
        cudaGraph_t g;
        RT_CUDA(c, cudaGraphCreate(&g, 0));
        cudaGraphConditionalHandle cond;
        RT_CUDA(c, cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        RT_CUDA(c, cudaGraphAddNode(&node, g, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        RT_CUDA(c, cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        const long l0 = c->launches;
        int s = pcg32_body(h, cond, 1);
        h->pcg32_iter_kernels = c->launches - l0;
        c->launches = l0;
        cudaGraph_t captured = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &captured);
        if (s != RT_OK) { cudaGraphDestroy(g); return s; }
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return rt_fail(c, RT_ECUDA, "FP32 PCG graph capture failed: %s", cudaGetErrorString(e));
        }
        cudaGraphExec_t exec;
        e = cudaGraphInstantiate(&exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return rt_fail(c, RT_ECUDA, "FP32 PCG graph instantiation failed: %s", cudaGetErrorString(e));
        }
        h->pcg32_graph = g;
        h->pcg32_exec = exec;
        h->pcg32_key = key;
    }
    RT_CUDA(c, cudaGraphLaunch(h->pcg32_exec, c->stream));
    return RT_OK;
}

static int pcg_core(rt_hier* h, double* x, const double* b, double tol, int maxit, rt_solve_info* info, int* vcycles);

static int pcg32_core(rt_hier* h, double* x, const double* b, double tol, int maxit, rt_solve_info* info, int* vcycles) {
    RT_CHECK(ensure_krylov32(h));
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    RT_CHECK(pcg_prologue(h, x, b));
    double s[2];
    RT_CHECK(read_scalars(h, 21, 2, s));
    if (!std::isfinite(s[0]) || !std::isfinite(s[1])) {
        if (info) { info->status = RT_ENAN; info->iterations = 0; }
        return rt_fail(h->ctx, RT_ENAN, "PCG: the right-hand side or the initial residual is not finite");
    }
    const double bn = std::sqrt(s[1]) > 0 ? std::sqrt(s[1]) : 1.0;
    double rel = std::sqrt(s[0]) / bn;
    int it = 0;
    bool stalled = false;
    const bool fallback = h->P.precision_fallback > 0;
    while (rel > tol && it < maxit) {
        // the inner solve aims at the outer target, no tighter than 10^-(3 + krylov_fp32)
        const double floor_in = std::pow(10.0, -3.0 - std::min(std::max(h->P.krylov_fp32, 1), 4));
        const double tol_in = std::min(0.5, std::max(0.9 * tol / rel, floor_in));
        RT_CHECK(rtk::d2f_scaled(h, n, h->rr, L.f32, h->scal + 21));
        RT_CUDA(c, cudaMemcpyAsync(h->scal + 23, h->scal + 21, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        RT_CUDA(c, cudaMemsetAsync(h->d32k, 0, sizeof(float) * n, c->stream));
        RT_CUDA(c, cudaMemsetAsync(h->ro32k, 0, sizeof(float) * n, c->stream));
        // inner loop state: scal[24..29] iteration count, tolerance, budget, no learned
        // correction (ratio, gate, previous r.r); scal[21..22] the unit right-hand side's r.r
        // and b.b; scal[90..93] stall detection as in pcg_core
        const double st[6] = {0.0, tol_in, (double)(maxit - it), 0.0, 0.0, 1.0};
        memcpy(c->hscal + 8, st, sizeof(st));
        RT_CUDA(c, cudaMemcpyAsync(h->scal + 24, c->hscal + 8, sizeof(st), cudaMemcpyHostToDevice, c->stream));
        const double unit[2] = {1.0, 1.0};
        memcpy(c->hscal + 20, unit, sizeof(unit));
        RT_CUDA(c, cudaMemcpyAsync(h->scal + 21, c->hscal + 20, sizeof(unit), cudaMemcpyHostToDevice, c->stream));
        double sd[4] = {1.0, 0.0, 0.0, fallback ? (double)h->P.precision_fallback : 0.0};
        memcpy(c->hscal + 16, sd, sizeof(sd));
        RT_CUDA(c, cudaMemcpyAsync(h->scal + 90, c->hscal + 16, sizeof(sd), cudaMemcpyHostToDevice, c->stream));
        const bool graphed = h->use_graphs && !c->profile;
        if (graphed) {
            RT_CHECK(pcg32_graph_run(h));
        } else {
            for (int k = 0; k < maxit - it; k++) {
                RT_CHECK(pcg32_body(h, 0, 0));
                double s2 = 0, stall = 0;
                RT_CHECK(read_scalars(h, 21, 1, &s2));
                RT_CHECK(read_scalars(h, 92, 1, &stall));
                if (!std::isfinite(s2) || std::sqrt(s2) <= tol_in || stall != 0.0) break;
            }
        }
        double s3[4], stall = 0;
        RT_CHECK(read_scalars(h, 21, 4, s3));  // inner r.r, 1, |r|^2 of the outer residual, inner iterations
        RT_CHECK(read_scalars(h, 92, 1, &stall));
        if (!std::isfinite(s3[0])) {
            if (info) { info->status = RT_ENAN; info->iterations = it + (int)s3[3]; }
            return nan_fail(h, it + (int)s3[3]);
        }
        const int its_in = (int)s3[3];
        if (graphed) c->launches += h->pcg32_iter_kernels * its_in;
        RT_CHECK(rtk::axpy_f32_scaled(h, n, x, h->d32k, h->scal + 23));
        RT_CHECK(pcg_prologue(h, x, b));
        RT_CHECK(read_scalars(h, 21, 1, s));
        rel = std::sqrt(s[0]) / bn;
        it += its_in;
        if (its_in == 0) break;
        if (stall != 0.0) {
            stalled = true;
            break;
        }
    }
    if (fallback && stalled && rel > tol && it < maxit) {
        // the FP32 cycles stopped reducing |r|: continue from x with FP64 V-cycles and FP64 vectors
        const int saved = h->P.precision;
        h->P.precision = RT_FP64;
        rt_solve_info sub;
        memset(&sub, 0, sizeof(sub));
        int vc = 0;
        const int st2 = pcg_core(h, x, b, tol, maxit - it, &sub, &vc);
        h->P.precision = saved;
        RT_CHECK(st2);
        it += sub.iterations;
        rel = sub.rel_residual;
        h->fallbacks++;
    }
    *vcycles += it;
    if (info) {
        info->iterations = it;
        info->rel_residual = rel;
        info->status = rel <= tol ? RT_OK : RT_ENOCONV;
    }
    return RT_OK;
}

static int pcg_core(rt_hier* h, double* x, const double* b, double tol, int maxit, rt_solve_info* info, int* vcycles) {
    double* r = h->rr;
    if (h->P.precision == RT_FP32 && h->P.krylov_fp32 && !h->unet && h->P.mode != RT_MODE_NSCF &&
        h->P.mode != RT_MODE_NSFF)
        return pcg32_core(h, x, b, tol, maxit, info, vcycles);
    RT_CHECK(pcg_prologue(h, x, b));
    double s[2];
    RT_CHECK(read_scalars(h, 21, 2, s));
    if (!std::isfinite(s[0]) || !std::isfinite(s[1])) {
        if (info) { info->status = RT_ENAN; info->iterations = 0; }
        return rt_fail(h->ctx, RT_ENAN, "PCG: the right-hand side or the initial residual is not finite");
    }
    const double bn = std::sqrt(s[1]) > 0 ? std::sqrt(s[1]) : 1.0;
    double rel = std::sqrt(s[0]) / bn;
    int it = 0;
    // without supports K is singular (rigid modes): keep the search space in its range
    const bool no_support = (h->P.mode == RT_MODE_NSCF || h->P.mode == RT_MODE_NSFF);
    if (no_support && h->Ru == nullptr) RT_CHECK(rtk::rigid_nodes(h));
    if (rel > tol && maxit > 0) {
        // loop state on the device: scal[24] iteration count, scal[25] tol, scal[26] maxit,
        // scal[27..29] learned-correction fallback ratio, gate, previous r.r
        const bool learned_on = h->unet && !h->unet_off;
        double st[6] = {0.0, tol, (double)maxit, h->unet_fallback, learned_on ? 1.0 : 0.0, s[0]};
        memcpy(h->ctx->hscal + 8, st, sizeof(st));
        RT_CUDA(h->ctx, cudaMemcpyAsync(h->scal + 24, h->ctx->hscal + 8, sizeof(st), cudaMemcpyHostToDevice,
                                        h->ctx->stream));
        // scal[36]: learned corrections run in this solve
        RT_CUDA(h->ctx, cudaMemsetAsync(h->scal + 36, 0, sizeof(double), h->ctx->stream));
        if (h->unet) RT_CHECK(rtu::refresh(h->unet));
        // scal[90..93]: stall detection of the reduced-precision V-cycles (see k_pcg_tail)
        const bool fallback = h->P.precision != RT_FP64 && h->P.precision_fallback > 0;
        double sd[4] = {s[0], 0.0, 0.0, fallback ? (double)h->P.precision_fallback : 0.0};
        memcpy(h->ctx->hscal + 16, sd, sizeof(sd));
        RT_CUDA(h->ctx, cudaMemcpyAsync(h->scal + 90, h->ctx->hscal + 16, sizeof(sd), cudaMemcpyHostToDevice,
                                        h->ctx->stream));
        const bool graphed = h->use_graphs && !h->ctx->profile;
        if (graphed) {
            RT_CHECK(pcg_graph_run(h, x, r, no_support));
        } else {
            for (int k = 0; k < maxit; k++) {
                RT_CHECK(pcg_body(h, x, r, no_support, 0));
                double s2[4], stall = 0;
                RT_CHECK(read_scalars(h, 21, 4, s2));
                RT_CHECK(read_scalars(h, 92, 1, &stall));
                if (!std::isfinite(s2[0]) || std::sqrt(s2[0]) / bn <= tol || stall != 0.0) break;
            }
        }
        double s3[4], stall = 0;
        RT_CHECK(read_scalars(h, 21, 4, s3));  // rr, bb, (unused), it
        RT_CHECK(read_scalars(h, 92, 1, &stall));
        if (!std::isfinite(s3[0])) {
            if (info) { info->status = RT_ENAN; info->iterations = (int)s3[3]; }
            return nan_fail(h, (int)s3[3]);
        }
        rel = std::sqrt(s3[0]) / bn;
        it = (int)s3[3];
        if (graphed) h->ctx->launches += h->pcg_iter_kernels * it;
        if (h->unet) {
            double lg[9];
            RT_CHECK(read_scalars(h, 28, 9, lg));  // scal[28] gate at the end, scal[36] corrections run
            const long long applied = (long long)lg[8];
            h->unet_applied += applied;
            if (graphed) h->ctx->launches += h->unet_kernels * applied;
            if (learned_on && lg[0] == 0.0) {
                h->unet_off = true;
                h->unet_verdict_epoch = h->design_epoch;
            }
        }
        if (fallback && stall != 0.0 && rel > tol && it < maxit) {
            // continue from the current iterate with FP64 V-cycles (flexible CG restarts)
            const int saved = h->P.precision;
            h->P.precision = RT_FP64;
            rt_solve_info sub;
            memset(&sub, 0, sizeof(sub));
            int vc = 0;
            const int st2 = pcg_core(h, x, b, tol, maxit - it, &sub, &vc);
            h->P.precision = saved;
            RT_CHECK(st2);
            it += sub.iterations;
            rel = sub.rel_residual;
            h->fallbacks++;
        }
    }
    *vcycles += it;
    if (info) {
        info->iterations = it;
        info->rel_residual = rel;
        info->status = rel <= tol ? RT_OK : RT_ENOCONV;
    }
    return RT_OK;
}

extern "C" int rt_pcg(rt_hier* h, double tol, int maxit, rt_solve_info* info) {
    if (!h || tol <= 0 || maxit < 0) return RT_EINVAL;
    RT_CHECK(need_stencil(h));
    rt_solve_info loc;
    memset(&loc, 0, sizeof(loc));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, h->ctx->stream);
    rt_level& L = h->L[0];
    int vc = 0;
    int s = pcg_core(h, L.u, L.f, tol, maxit, &loc, &vc);
    cudaEventRecord(b, h->ctx->stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    loc.vcycles = vc;
    loc.seconds = ms * 1e-3;
    if (s == RT_OK) {
        RT_CHECK(rtk::dot(h, 3 * L.nv, L.f, L.u, h->scal + 2));
        RT_CHECK(read_scalars(h, 2, 1, &loc.value));
    }
    if (info) *info = loc;
    if (s != RT_OK) return s;
    return loc.status == RT_OK ? RT_OK : RT_ENOCONV;
}

// ---------------------------------------------------------------------------
// worst-case load
// ---------------------------------------------------------------------------
__global__ void k_multidot(long n, int m, const double* __restrict__ Q, const double* __restrict__ w,
                           double* __restrict__ partials) {
    // m <= 64 dots of w against the rows of Q; block partials [block][64]
    __shared__ double sh[64][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = 0; k < m; k++) {
        double s = 0;
        for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
            s += Q[(long)k * n + i] * w[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sh[k][warp] = s;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        double s = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += sh[k][q];
        partials[blockIdx.x * 64 + k] = s;
    }
}
__global__ void k_multidot_final(int nblocks, int m, const double* __restrict__ partials, double* __restrict__ out) {
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        double s = 0;
        for (int b = 0; b < nblocks; b++) s += partials[b * 64 + k];
        out[k] = s;
    }
}
__global__ void k_sub_multi(long n, int m, const double* __restrict__ Q, const double* __restrict__ hcoef,
                            double* __restrict__ w) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double s = w[i];
        for (int k = 0; k < m; k++) s -= hcoef[k] * Q[(long)k * n + i];
        w[i] = s;
    }
}
__global__ void k_combine(long n, int m, const double* __restrict__ Q, const double* __restrict__ y,
                          double* __restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = 0; k < m; k++) s += y[k] * Q[(long)k * n + i];
        out[i] = s;
    }
}
// store alpha_j = a and beta_j = sqrt(bb); w /= beta_j done by k_scale with the same slot
__global__ void k_store_ab(const double* __restrict__ adot, const double* __restrict__ bb, double* __restrict__ alpha,
                           double* __restrict__ beta, int j) {
    if (threadIdx.x == 0) {
        alpha[j] = adot[0];
        beta[j] = sqrt(bb[0]);
    }
}
// Ritz vector of the largest eigenvalue of T_k by three steps of inverse iteration
__global__ void k_tridiag_ritz(int k, const double* __restrict__ alpha, const double* __restrict__ beta,
                               const double* __restrict__ lam, double* __restrict__ y) {
    if (threadIdx.x != 0) return;
    double yy[64], cp[64], dp[64];
    for (int i = 0; i < k; i++) yy[i] = 1.0;
    const double shift = lam[0] * (1 + 1e-12) + 1e-300;
    for (int it = 0; it < 3; it++) {
        for (int i = 0; i < k; i++) {
            const double a = i > 0 ? beta[i - 1] : 0, b = alpha[i] - shift, c = i < k - 1 ? beta[i] : 0;
            const double den = b - (i > 0 ? a * cp[i - 1] : 0);
            cp[i] = c / den;
            dp[i] = (yy[i] - (i > 0 ? a * dp[i - 1] : 0)) / den;
        }
        double nrm = 0;
        for (int i = k - 1; i >= 0; i--) {
            yy[i] = dp[i] - (i < k - 1 ? cp[i] * yy[i + 1] : 0);
        }
        for (int i = 0; i < k; i++) nrm += yy[i] * yy[i];
        nrm = sqrt(nrm);
        for (int i = 0; i < k; i++) yy[i] /= nrm;
    }
    for (int i = 0; i < k; i++) y[i] = yy[i];
}
__global__ void k_diffnorm(long n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ partials) {
    __shared__ double sh[2][8];
    double s0 = 0, s1 = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double d = a[i] - b[i];
        s0 += d * d;
        s1 += b[i] * b[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
    }
    if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = s0; sh[1][threadIdx.x >> 5] = s1; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0, a1 = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) { a0 += sh[0][q]; a1 += sh[1][q]; }
        partials[blockIdx.x * 2] = a0;
        partials[blockIdx.x * 2 + 1] = a1;
    }
}
__global__ void k_final2(int nb, const double* __restrict__ partials, double* __restrict__ out) {
    if (threadIdx.x == 0) {
        double a0 = 0, a1 = 0;
        for (int b = 0; b < nb; b++) { a0 += partials[2 * b]; a1 += partials[2 * b + 1]; }
        out[0] = a0;
        out[1] = a1;
    }
}

static int multidot(rt_hier* h, long n, int m, const double* Q, const double* w, double* out) {
    RT_CHECK(rt_launch(h->ctx, "lanczos_multidot", [&] {
        k_multidot<<<RT_RED_BLOCKS / 2, 256, 0, h->ctx->stream>>>(n, m, Q, w, h->partials);
    }));
    return rt_launch(h->ctx, "lanczos_multidot_final", [&] {
        k_multidot_final<<<1, 64, 0, h->ctx->stream>>>(RT_RED_BLOCKS / 2, m, h->partials, out);
    });
}

static int lanczos(rt_hier* h, int k, double inner_tol, uint64_t seed, double* lambda, rt_solve_info* info) {
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[0];
    const long n = 3 * L.nv, nl = 3L * h->nload;
    if (h->nload == 0) return rt_fail(c, RT_ESTATE, "no load nodes");
    if (k < 1 || k > 60) return rt_fail(c, RT_EINVAL, "Lanczos k must be in [1, 60]");
    if (h->Qcap < k + 1) {
        cudaFree(h->Q);
        h->Q = nullptr;
        RT_CHECK(dalloc(c, &h->Q, (size_t)(k + 1) * nl));
        h->Qcap = k + 1;
    }
    double* alpha = h->scal + 100;  // [64]
    double* beta = h->scal + 164;   // [64]
    double* hc = h->scal + 240;     // [64] re-orthogonalisation coefficients, then the Ritz vector
    double* Q = h->Q;
    RT_CHECK(rtk::rng_uniform(h, seed, n, L.f));
    RT_CHECK(rtk::project_load(h, L.f));
    RT_CHECK(rtk::gather_load(h, L.f, Q));
    RT_CHECK(rtk::dot(h, nl, Q, Q, h->scal + 30));
    RT_CHECK(rtk::scale(h, nl, Q, h->scal + 30, true));
    int inner = 0, vcycles = 0, steps = 0;
    for (int j = 0; j < k; j++) {
        double* qj = Q + (long)j * nl;
        double* w = Q + (long)(j + 1) * nl;
        RT_CUDA(c, cudaMemsetAsync(L.f, 0, sizeof(double) * n, c->stream));
        RT_CHECK(rtk::scatter_load(h, qj, L.f));
        RT_CUDA(c, cudaMemsetAsync(L.u, 0, sizeof(double) * n, c->stream));
        rt_solve_info si;
        memset(&si, 0, sizeof(si));
        RT_CHECK(pcg_core(h, L.u, L.f, inner_tol, 500, &si, &vcycles));
        inner += si.iterations;
        // w = P S u
        RT_CUDA(c, cudaMemcpyAsync(h->z, L.u, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
        RT_CHECK(rtk::project_load(h, h->z));
        RT_CHECK(rtk::gather_load(h, h->z, w));
        RT_CHECK(rtk::dot(h, nl, w, qj, h->scal + 31));
        // CGS2 full re-orthogonalisation against q_0..q_j
        for (int pass = 0; pass < 2; pass++) {
            RT_CHECK(multidot(h, nl, j + 1, Q, w, hc));
            RT_CHECK(rt_launch(c, "lanczos_sub", [&] {
                k_sub_multi<<<(unsigned)std::min<long>((nl + 255) / 256, c->sm_count * 8), 256, 0, c->stream>>>(
                    nl, j + 1, Q, hc, w);
            }));
        }
        RT_CHECK(rtk::dot(h, nl, w, w, h->scal + 32));
        RT_CHECK(rt_launch(c, "lanczos_store_ab",
                           [&] { k_store_ab<<<1, 32, 0, c->stream>>>(h->scal + 31, h->scal + 32, alpha, beta, j); }));
        RT_CHECK(rtk::scale(h, nl, w, h->scal + 32, true));
        steps = j + 1;
        double ab[2];
        RT_CUDA(c, cudaMemcpyAsync(c->hscal, alpha + j, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        RT_CUDA(c, cudaMemcpyAsync(c->hscal + 1, beta + j, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        RT_CUDA(c, cudaStreamSynchronize(c->stream));
        ab[0] = c->hscal[0];
        ab[1] = c->hscal[1];
        if (!std::isfinite(ab[0]) || !std::isfinite(ab[1])) return rt_fail(c, RT_ENAN, "NaN in Lanczos");
        if (ab[1] < 1e-13 * std::fabs(ab[0])) break;
    }
    RT_CHECK(rtk::tridiag_max_eig(h, steps, alpha, beta, h->scal + 33));
    RT_CHECK(rt_launch(c, "lanczos_ritz", [&] { k_tridiag_ritz<<<1, 32, 0, c->stream>>>(steps, alpha, beta, h->scal + 33, hc); }));
    // worst-case load f = Q y on the load set, u = K^-1 f
    RT_CHECK(rt_launch(c, "lanczos_combine", [&] {
        k_combine<<<(unsigned)std::min<long>((nl + 255) / 256, c->sm_count * 8), 256, 0, c->stream>>>(nl, steps, Q, hc, h->fs_old);
    }));
    RT_CUDA(c, cudaMemsetAsync(L.f, 0, sizeof(double) * n, c->stream));
    RT_CHECK(rtk::scatter_load(h, h->fs_old, L.f));
    RT_CUDA(c, cudaMemsetAsync(L.u, 0, sizeof(double) * n, c->stream));
    rt_solve_info si;
    memset(&si, 0, sizeof(si));
    RT_CHECK(pcg_core(h, L.u, L.f, inner_tol, 500, &si, &vcycles));
    inner += si.iterations;
    RT_CHECK(read_scalars(h, 33, 1, lambda));
    if (info) {
        info->iterations = steps;
        info->inner_iterations = inner;
        info->vcycles = vcycles;
        info->rel_residual = si.rel_residual;
        info->value = *lambda;
        info->status = RT_OK;
    }
    return RT_OK;
}

// modifiedPM (optimization/optimization.cpp:123-261)
static int modified_pm(rt_hier* h, int maxit, uint64_t seed, double* lambda, rt_solve_info* info) {
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[0];
    const long n = 3 * L.nv, nl = 3L * h->nload;
    if (h->nload == 0) return rt_fail(c, RT_ESTATE, "no load nodes");
    const bool no_support = (h->P.mode == RT_MODE_NSCF || h->P.mode == RT_MODE_NSFF);
    if (no_support && h->Ru == nullptr) RT_CHECK(rtk::rigid_nodes(h));
    RT_CHECK(rtk::rng_uniform(h, seed, n, L.f));
    RT_CHECK(rtk::project_load(h, L.f));
    RT_CHECK(rtk::dot(h, n, L.f, L.f, h->scal + 30));
    RT_CHECK(rtk::scale(h, n, L.f, h->scal + 30, true));
    RT_CUDA(c, cudaMemsetAsync(L.u, 0, sizeof(double) * n, c->stream));
    RT_CHECK(rtk::gather_load(h, L.f, h->fs_old));
    double fch = 1, rel = 1;
    int itn = 0;
    while (itn++ < maxit && (fch > 1e-4 || rel > 1e-2)) {
        RT_CHECK(vcycle_T<double>(h, RT_SMOOTH_GS, 1, 1, h->P.jacobi_omega));
        RT_CHECK(rtk::fine_residual<double>(h, L.u, L.f, L.r));
        RT_CHECK(rtk::dot(h, n, L.r, L.r, h->scal + 0));
        RT_CHECK(rtk::dot(h, n, L.f, L.f, h->scal + 1));
        if (no_support) RT_CHECK(rtk::displacement_project(h, L.u));
        RT_CUDA(c, cudaMemcpyAsync(L.f, L.u, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
        RT_CHECK(rtk::project_load(h, L.f));
        RT_CHECK(rtk::dot(h, n, L.f, L.f, h->scal + 30));
        RT_CHECK(rtk::scale(h, n, L.f, h->scal + 30, true));
        RT_CHECK(rtk::gather_load(h, L.f, h->fs));
        RT_CHECK(rt_launch(c, "pm_diffnorm", [&] { k_diffnorm<<<64, 256, 0, c->stream>>>(nl, h->fs, h->fs_old, h->partials); }));
        RT_CHECK(rt_launch(c, "pm_diffnorm_final", [&] { k_final2<<<1, 32, 0, c->stream>>>(64, h->partials, h->scal + 3); }));
        RT_CUDA(c, cudaMemcpyAsync(h->fs_old, h->fs, sizeof(double) * nl, cudaMemcpyDeviceToDevice, c->stream));
        double s[5];
        RT_CHECK(read_scalars(h, 0, 5, s));
        rel = std::sqrt(s[0]) / std::sqrt(s[1]);
        fch = std::sqrt(s[3]) / std::sqrt(s[4]);
        if (!(rel <= 1e4)) return rt_fail(c, RT_ENAN, "modified power method diverged (rel_res %g)", rel);
    }
    RT_CHECK(rtk::dot(h, n, L.f, L.u, h->scal + 2));
    RT_CHECK(read_scalars(h, 2, 1, lambda));
    if (info) {
        info->iterations = itn - 1;
        info->vcycles = itn - 1;
        info->rel_residual = rel;
        info->value = *lambda;
        info->status = (fch <= 1e-4 && rel <= 1e-2) ? RT_OK : RT_ENOCONV;
    }
    return RT_OK;
}

static int block_lanczos(rt_hier* h, int bs, int nblk, double inner_tol, uint64_t seed, double* lambda,
                         rt_solve_info* info);

extern "C" int rt_worst_case(rt_hier* h, int method, int k, double inner_tol, uint64_t seed, double* lambda,
                             rt_solve_info* info) {
    if (!h || !lambda) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CHECK(need_stencil(h));
    rt_solve_info loc;
    memset(&loc, 0, sizeof(loc));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, h->ctx->stream);
    int s;
    if (method == RT_WORST_LANCZOS) s = lanczos(h, k, inner_tol, seed, lambda, &loc);
    else if (method == RT_WORST_BLOCK_LANCZOS) s = block_lanczos(h, 8, std::max(1, (k + 7) / 8), inner_tol, seed, lambda, &loc);
    else if (method == RT_WORST_MODPM) s = modified_pm(h, k > 0 ? k : 500, seed, lambda, &loc);
    else s = RT_EINVAL;
    cudaEventRecord(b, h->ctx->stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    loc.seconds = ms * 1e-3;
    if (info) *info = loc;
    return s;
}

// ---------------------------------------------------------------------------
// optimisation step
// ---------------------------------------------------------------------------
extern "C" int rt_filter_sensitivity(rt_hier* h, float radius) {
    if (!h || radius <= 0) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    return rtk::filter(h, radius);
}

extern "C" int rt_sensitivity(rt_hier* h, int filt) {
    if (!h) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CHECK(rtk::sensitivity(h, h->L[0].u));
    if (filt) RT_CHECK(rtk::filter(h, h->P.filter_radius));
    return RT_OK;
}

extern "C" int rt_oc_update(rt_hier* h, float vgoal, float* lambda_out, int* trials_out) {
    if (!h) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    rt_level& L = h->L[0];
    RT_CHECK(rtk::oc_maxabs(h, nullptr));
    double gmax;
    RT_CHECK(read_scalars(h, 50, 1, &gmax));
    float lo = 0, hi = (float)gmax, thr = (lo + hi) / 2, V = 2;
    const double nact = (double)L.n_act_elems;
    int itn = 0, trials = 0;
    do {
        thr = (lo + hi) / 2;
        RT_CHECK(rtk::oc_try(h, thr, h->ftmp, h->scal + 51));
        double vs;
        RT_CHECK(read_scalars(h, 51, 1, &vs));
        V = (float)(vs / nact);
        trials++;
        if (V > vgoal) lo = thr;
        else if (V < vgoal) hi = thr;
    } while (std::fabs(V - vgoal) > 1e-4f && itn++ < 30);
    RT_CHECK(rtk::oc_try(h, thr, h->rho, h->scal + 51));
    h->stencil_ready = false;
    h->design_epoch++;
    if (lambda_out) *lambda_out = thr;
    if (trials_out) *trials_out = trials;
    return RT_OK;
}

extern "C" int rt_oc_iteration(rt_hier* h, int method, int k, double inner_tol, uint64_t seed, float vgoal,
                               double* compliance_out) {
    if (!h) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CHECK(rt_update_stencil(h));
    double lam = 0;
    rt_solve_info info;
    RT_CHECK(rt_worst_case(h, method, k, inner_tol, seed, &lam, &info));
    RT_CHECK(rt_sensitivity(h, 1));
    RT_CHECK(rt_oc_update(h, vgoal, nullptr, nullptr));
    if (compliance_out) *compliance_out = lam;
    return RT_OK;
}

// ---------------------------------------------------------------------------
// launch-shape autotuner for the finest-level kernels
// ---------------------------------------------------------------------------
// a Chebyshev table for lmax = 2 (slot 299) so the fine kernels can be timed before any stencil exists
static int spare_cheby_table(rt_hier* h) {
    const double two = 2.0;
    RT_CUDA(h->ctx, cudaMemcpyAsync(h->scal + 299, &two, sizeof(double), cudaMemcpyHostToDevice, h->ctx->stream));
    return rt_launch(h->ctx, "lmax_finish", [&] {
        k_lmax_finish<<<1, 32, 0, h->ctx->stream>>>(nullptr, h->scal + 299, h->scal + RT_SCAL_CHEB_SPARE);
    });
}

static double time_fine_kernel(rt_hier* h, int prec, int mode, int reps) {
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[0];
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const double* coef = h->stencil_ready ? cheby_table(h, 0) : h->scal + RT_SCAL_CHEB_SPARE;
    auto run = [&]() -> int {
        if (prec == 1) {
            double *u = h->x, *f = h->q, *o = h->z, *d = h->p;
            switch (mode) {
                case 0: return rtk::fine_residual<double>(h, u, f, o);
                case 1: return rtk::fine_applyK<double>(h, u, o);
                case 2: return rtk::fine_jacobi<double>(h, u, f, o, 0.6);
                default: return rtk::fine_cheby<double>(h, u, f, o, d, coef, 1);
            }
        }
        float *u = L.u32, *f = L.f32, *o = L.r32, *d = L.d32;
        switch (mode) {
            case 0: return rtk::fine_residual<float>(h, u, f, o);
            case 1: return rtk::fine_applyK<float>(h, u, o);
            case 2: return rtk::fine_jacobi<float>(h, u, f, o, 0.6);
            default: return rtk::fine_cheby<float>(h, u, f, o, d, coef, 1);
        }
    };
    double best = 1e30;
    if (run() == RT_OK) {  // warm-up
        cudaEventRecord(a, c->stream);
        bool ok = true;
        for (int i = 0; i < reps && ok; i++) ok = run() == RT_OK;
        cudaEventRecord(b, c->stream);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ok) best = ms * 1e3 / reps;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

static int autotune_level_kernels(rt_hier* h, int reps);

extern "C" int rt_autotune(rt_hier* h, int reps) {
    if (!h) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    if (reps <= 0) reps = 5;
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    const bool was_profiling = c->profile;
    c->profile = false;
    // inputs: random u, f on the solver's scratch vectors (their contents do not persist across calls)
    RT_CHECK(refresh_fine(h));
    RT_CHECK(rtk::rng_uniform(h, 0xa770, n, h->x));
    RT_CHECK(rtk::rng_uniform(h, 0xa771, n, h->q));
    RT_CHECK(rtk::d2f(h, n, h->x, L.u32));
    RT_CHECK(rtk::d2f(h, n, h->q, L.f32));
    RT_CUDA(c, cudaMemsetAsync(h->p, 0, sizeof(double) * n, c->stream));
    RT_CUDA(c, cudaMemsetAsync(L.d32, 0, sizeof(float) * n, c->stream));
    if (!h->stencil_ready) RT_CHECK(spare_cheby_table(h));
    std::vector<rt_tile_cfg> cands;
    for (int ty : {2, 4, 8})
        for (int zc : {4, 8, 16, 32, 64}) cands.push_back(rt_tile_cfg{1, ty, zc});
    for (int ty : {2, 4})
        for (int zc : {8, 16, 32}) cands.push_back(rt_tile_cfg{2, ty, zc});
    for (int ty : {2, 4, 8})
        for (int zc : {8, 16, 32}) cands.push_back(rt_tile_cfg{0, ty, zc});
    for (int ty : {2, 4, 8})
        for (int zc : {8, 16, 32, 64}) cands.push_back(rt_tile_cfg{3, ty, zc});
    for (int ty : {2, 4, 8})
        for (int zc : {8, 16, 32, 64}) cands.push_back(rt_tile_cfg{4, ty, zc});  // FP32 only
    for (int ty : {4, 8, 16})
        for (int zc : {16, 32, 64}) cands.push_back(rt_tile_cfg{5, ty, zc});  // ty 16: FP32 only
    if (h->L[0].vx % 16 == 0)  // TMA-staged node layers: the flags' row pitch must be a multiple of 16 bytes
        for (int v : {6, 7})
            for (int ty : {4, 6, 8})
                for (int zc : {8, 16, 32, 64})
                    if (ty != 6 || v == 7) cands.push_back(rt_tile_cfg{v, ty, zc});
    for (int prec = 0; prec < 2; prec++)
        for (int mode = 0; mode < 4; mode++) {
            rt_tile_cfg best_cfg = h->tune[prec][mode];
            double best = 1e30;
            for (const rt_tile_cfg& cfg : cands) {
                if (cfg.zchunk > 2 * L.vz && cfg.zchunk != 4) continue;
                if (cfg.variant == 4 && prec == 1) continue;
                if (cfg.variant == 5 && cfg.ty == 16 && prec == 1) continue;
                h->tune[prec][mode] = cfg;
                const double t = time_fine_kernel(h, prec, mode, reps);
                if (t < best) { best = t; best_cfg = cfg; }
            }
            h->tune[prec][mode] = best_cfg;
            h->tune_us[prec][mode] = best;
        }
    RT_CHECK(autotune_level_kernels(h, reps));
    cudaGetLastError();
    h->graph_epoch++;  // launch shapes are baked into captured graphs
    c->profile = was_profiling;
    return RT_OK;
}

extern "C" int rt_tuning_info(rt_hier* h, int precision, int mode, int* variant, int* ty, int* zchunk, double* us) {
    if (!h || precision < 0 || precision > 1 || mode < 0 || mode > 3) return RT_EINVAL;
    const int pr = precision == RT_FP64 ? 1 : 0;
    const rt_tile_cfg& t = h->tune[pr][mode];
    if (variant) *variant = t.variant;
    if (ty) *ty = t.ty;
    if (zchunk) *zchunk = t.zchunk;
    if (us) *us = h->tune_us[pr][mode];
    return RT_OK;
}

extern "C" int rt_set_tuning(rt_hier* h, int precision, int mode, int variant, int ty, int zchunk) {
    if (!h || precision < 0 || precision > 1 || mode < 0 || mode > 3 || variant < 0 || variant > 7 || zchunk < 1)
        return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    if (variant == 4 && precision == RT_FP64) return rt_fail(h->ctx, RT_EINVAL, "variant 4 (packed FP32 pairs) is FP32 only");
    if (variant == 5) {
        if (ty != 4 && ty != 8 && ty != 16) return rt_fail(h->ctx, RT_EINVAL, "sum-factorised rows per tile must be 4, 8 or 16");
    } else if (variant == 6 || variant == 7) {
        if (ty != 4 && ty != 8 && !(variant == 7 && ty == 6))
            return rt_fail(h->ctx, RT_EINVAL, "TMA-staged rows per tile must be 4 or 8 (6 as well on 31-wide tiles)");
    } else if (variant != 2 && ty != 2 && ty != 4 && ty != 8) {
        return rt_fail(h->ctx, RT_EINVAL, "rows per tile must be 2, 4 or 8");
    }
    const int pr = precision == RT_FP64 ? 1 : 0;
    if (variant == 2 && ty != 2 && ty != 4) return rt_fail(h->ctx, RT_EINVAL, "prefetching rows per tile must be 2 or 4");
    h->tune[pr][mode] = rt_tile_cfg{variant, ty, zchunk};
    h->graph_epoch++;
    return RT_OK;
}

extern "C" int rt_bench_fine_kernel(rt_hier* h, int precision, int mode, int reps, double* us_per_launch) {
    if (!h || precision < 0 || precision > 1 || mode < 0 || mode > 3 || reps < 1) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    RT_CHECK(refresh_fine(h));
    RT_CHECK(rtk::rng_uniform(h, 0xbe7c, n, h->x));
    RT_CHECK(rtk::rng_uniform(h, 0xbe7d, n, h->q));
    RT_CHECK(rtk::d2f(h, n, h->x, L.u32));
    RT_CHECK(rtk::d2f(h, n, h->q, L.f32));
    if (!h->stencil_ready) RT_CHECK(spare_cheby_table(h));
    const double t = time_fine_kernel(h, precision == RT_FP64 ? 1 : 0, mode, reps);
    if (t >= 1e30) return rt_fail(c, RT_ECUDA, "kernel launch failed");
    if (us_per_launch) *us_per_launch = t;
    return RT_OK;
}

// one FP32 finest-level kernel at its current launch shape on level 0's vectors: u, f rounded to
// FP32, the result (mode 0 residual f - K u, 1 K u, 2 Jacobi step, 3 first Chebyshev step) widened into r
extern "C" int rt_fine_kernel_f32(rt_hier* h, int mode, double omega) {
    if (!h || mode < 0 || mode > 3) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CHECK(refresh_fine(h));
    if (mode == 3 && !h->stencil_ready) return rt_fail(h->ctx, RT_ESTATE, "rt_update_stencil has not run");
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    RT_CHECK(rtk::d2f(h, n, L.u, L.u32));
    RT_CHECK(rtk::d2f(h, n, L.f, L.f32));
    switch (mode) {
        case 0: RT_CHECK(rtk::fine_residual<float>(h, L.u32, L.f32, L.r32)); break;
        case 1: RT_CHECK(rtk::fine_applyK<float>(h, L.u32, L.r32)); break;
        case 2: RT_CHECK(rtk::fine_jacobi<float>(h, L.u32, L.f32, L.r32, omega)); break;
        default: RT_CHECK(rtk::fine_cheby<float>(h, L.u32, L.f32, L.r32, L.d32, cheby_table(h, 0), 0)); break;
    }
    return rtk::f2d(h, n, L.r32, L.r);
}

// one stencil-level kernel (residual, Jacobi or a Chebyshev step) on random inputs, timed with
// CUDA events on the context stream.  FP32: random u, f through the fine-level scratch vectors into
// the level's FP32 vectors (V-cycle scratch); FP64: the level's own u, f (overwritten).
static double time_level_kernel(rt_hier* h, int lvl, int precision, int mode, int reps) {
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[lvl];
    const long n = 3 * L.nv;
    double* ru = precision == RT_FP64 ? L.u : h->x;
    double* rf = precision == RT_FP64 ? L.f : h->q;
    if (rtk::rng_uniform(h, 0xbe7e, n, ru) != RT_OK || rtk::rng_uniform(h, 0xbe7f, n, rf) != RT_OK) return 1e30;
    if (precision != RT_FP64 && (rtk::d2f(h, n, ru, L.u32) != RT_OK || rtk::d2f(h, n, rf, L.f32) != RT_OK)) return 1e30;
    const double* coef = cheby_table(h, lvl);
    auto run = [&]() -> int {
        if (precision == RT_FP64) {
            switch (mode) {
                case 0: return rtk::st_residual<double>(h, lvl, L.u, L.f, L.r);
                case 2: return rtk::st_jacobi<double>(h, lvl, L.u, L.f, L.r, 0.6);
                default: return rtk::st_cheby<double>(h, lvl, L.u, L.f, L.r, L.d, coef, 1);
            }
        }
        switch (mode) {
            case 0: return rtk::st_residual<float>(h, lvl, L.u32, L.f32, L.r32);
            case 2: return rtk::st_jacobi<float>(h, lvl, L.u32, L.f32, L.r32, 0.6);
            default: return rtk::st_cheby<float>(h, lvl, L.u32, L.f32, L.r32, L.d32, coef, 1);
        }
    };
    if (run() != RT_OK) return 1e30;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, c->stream);
    int st = RT_OK;
    for (int i = 0; i < reps && st == RT_OK; i++) st = run();
    cudaEventRecord(b, c->stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return st == RT_OK ? ms * 1e3 / reps : 1e30;
}

extern "C" int rt_bench_level_kernel(rt_hier* h, int lvl, int precision, int mode, int reps, double* us_per_launch) {
    if (!h || lvl < 1 || lvl + 1 >= (int)h->L.size() || precision < RT_FP64 || precision > RT_FP32 || mode < 0 ||
        mode > 3 || mode == 1 || reps < 1)
        return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CHECK(need_stencil(h));
    const double t = time_level_kernel(h, lvl, precision, mode, reps);
    if (t >= 1e30) return rt_fail(h->ctx, RT_ECUDA, "kernel launch failed");
    if (us_per_launch) *us_per_launch = t;
    return RT_OK;
}

// the lane-split / bulk-copy choice for the FP32 smoother's stencil kernels, timed on the largest
// stencil level's Chebyshev step (FP32 stencils, and BF16 ones when they exist)
// a set of nsteps FP32 Chebyshev steps on stencil level lvl (random u, f), separate launches or one
// fused launch, captured as a graph as the solver runs it; device time per set in microseconds
static double time_level_sweeps(rt_hier* h, int lvl, bool fused, int nsteps, int reps) {
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[lvl];
    const long n = 3 * L.nv;
    if (rtk::rng_uniform(h, 0xbe80, n, h->x) != RT_OK || rtk::rng_uniform(h, 0xbe81, n, h->q) != RT_OK) return 1e30;
    if (rtk::d2f(h, n, h->x, L.u32) != RT_OK || rtk::d2f(h, n, h->q, L.f32) != RT_OK) return 1e30;
    const uint32_t saved = h->cheby_fused;
    h->cheby_fused = fused ? (saved | (1u << lvl)) : (saved & ~(1u << lvl));
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    double us = 1e30;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int st = level_smooth<float>(h, lvl, RT_SMOOTH_CHEBY, nsteps, 0.0, false);
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (st == RT_OK && e == cudaSuccess && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess &&
            cudaGraphLaunch(ge, c->stream) == cudaSuccess) {
            cudaEvent_t a, b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, c->stream);
            bool ok = true;
            for (int i = 0; i < reps && ok; i++) ok = cudaGraphLaunch(ge, c->stream) == cudaSuccess;
            cudaEventRecord(b, c->stream);
            cudaEventSynchronize(b);
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            double err = 0;
            if (ok && cudaStreamSynchronize(c->stream) == cudaSuccess && read_scalars(h, RT_SCAL_ERR, 1, &err) == RT_OK) {
                if (err == 0.0) {
                    us = ms * 1e3 / reps;
                } else {  // a barrier wait ran out: not a candidate; clear the error and barrier words
                    cudaMemsetAsync(h->scal + RT_SCAL_ERR, 0, sizeof(double), c->stream);
                    cudaMemsetAsync(h->scal + RT_SCAL_GBAR, 0, sizeof(double) * RT_MAX_LEVELS, c->stream);
                }
            }
        }
    }
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    h->cheby_fused = saved;
    return us;
}

static int autotune_level_kernels(rt_hier* h, int reps) {
    if (!h->stencil_ready || h->L.size() < 3) return RT_OK;
    // fused Chebyshev sweeps (one cooperative launch per smoothing) per stencil level, timed on
    // sets of 8 steps against the separate launches of the chosen lane-split / bulk variant.
    // The timings are recorded, the choice stays with the caller (rt_set_level_fused): alone the
    // fused sets are faster, but inside the solver's conditional-loop graphs the whole solve
    // measured slower with them
    const uint32_t keep = h->cheby_fused;
    if (rtk::st_cheby_fused_ok(h)) {
        for (int lvl = 1; lvl + 1 < (int)h->L.size() && lvl < 15; lvl++) {
            h->fused_us[lvl][0] = time_level_sweeps(h, lvl, false, 8, reps);
            h->fused_us[lvl][1] = time_level_sweeps(h, lvl, true, 8, reps);
        }
    }
    h->cheby_fused = keep;
    for (int t = 0; t < 2; t++) {
        if (t == 1 && !(h->P.coarse_bf16 && h->L[1].st16)) continue;
        const int saved_bf16 = h->P.coarse_bf16;
        h->P.coarse_bf16 = t;  // selects the stencil copy the FP32 smoother reads
        double best = 1e30;
        int best_v = h->st_variant[t];
        for (int v = 0; v < 2; v++) {
            h->st_variant[t] = v;
            const double us = time_level_kernel(h, 1, RT_FP32, 3, reps);
            h->st_us[t][v] = us;
            if (us < best) { best = us; best_v = v; }
        }
        h->st_variant[t] = best_v;
        h->P.coarse_bf16 = saved_bf16;
    }
    return RT_OK;
}

extern "C" int rt_set_level_fused(rt_hier* h, int lvl, int on) {
    if (!h || lvl < 1 || lvl + 1 >= (int)h->L.size() || lvl >= 15 || on < 0 || on > 2) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    if (on && !rtk::st_cheby_fused_ok(h))
        return rt_fail(h->ctx, RT_ECUDA, "the device cannot run the fused Chebyshev sweeps");
    h->cheby_fused = on ? (h->cheby_fused | (1u << lvl)) : (h->cheby_fused & ~(1u << lvl));
    h->cheby_stream = on == 2 ? (h->cheby_stream | (1u << lvl)) : (h->cheby_stream & ~(1u << lvl));
    h->graph_epoch++;
    return RT_OK;
}

extern "C" int rt_level_fused_info(rt_hier* h, int lvl, int* on, double* us_separate, double* us_fused) {
    if (!h || lvl < 1 || lvl + 1 >= (int)h->L.size() || lvl >= 15) return RT_EINVAL;
    if (on) *on = (int)((h->cheby_fused >> lvl) & 1u);
    if (us_separate) *us_separate = h->fused_us[lvl][0];
    if (us_fused) *us_fused = h->fused_us[lvl][1];
    return RT_OK;
}

extern "C" int rt_level_kernel_info(rt_hier* h, int stencil_type, int* variant, double* us_lane_split,
                                    double* us_bulk) {
    if (!h || stencil_type < 0 || stencil_type > 1) return RT_EINVAL;
    if (variant) *variant = h->st_variant[stencil_type];
    if (us_lane_split) *us_lane_split = h->st_us[stencil_type][0];
    if (us_bulk) *us_bulk = h->st_us[stencil_type][1];
    return RT_OK;
}

extern "C" int rt_set_level_kernel(rt_hier* h, int stencil_type, int variant) {
    if (!h || stencil_type < 0 || stencil_type > 1 || variant < 0 || variant > 1) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    h->st_variant[stencil_type] = variant;
    h->graph_epoch++;
    return RT_OK;
}

// ---------------------------------------------------------------------------
// solve workspaces and batched MG-PCG: many independent solves in one CUDA graph
// ---------------------------------------------------------------------------
static int make_workspace(rt_hier* p, rt_hier** out) {
    rt_ctx* c = p->ctx;
    rt_hier* w = new rt_hier();
    *out = w;  // the caller frees a partially built workspace
    w->ctx = c;
    rt_ctx_retain(c);
    w->uid = next_uid();
    w->parent = p;
    w->L.resize(p->L.size());
    for (size_t i = 0; i < p->L.size(); i++) {
        rt_level& a = w->L[i];
        const rt_level& b = p->L[i];
        a.nx = b.nx; a.ny = b.ny; a.nz = b.nz; a.vx = b.vx; a.vy = b.vy; a.vz = b.vz;
        a.nv = b.nv; a.ne = b.ne; a.ratio = b.ratio;
        const size_t n = 3 * (size_t)a.nv;
        RT_CHECK(dalloc(c, &a.u, n)); RT_CHECK(dalloc(c, &a.f, n)); RT_CHECK(dalloc(c, &a.r, n));
        RT_CHECK(dalloc(c, &a.d, n));
        RT_CHECK(dalloc(c, &a.u32, n)); RT_CHECK(dalloc(c, &a.f32, n)); RT_CHECK(dalloc(c, &a.r32, n));
        RT_CHECK(dalloc(c, &a.d32, n));
        RT_CUDA(c, cudaMemsetAsync(a.u, 0, sizeof(double) * n, c->stream));
        RT_CUDA(c, cudaMemsetAsync(a.f, 0, sizeof(double) * n, c->stream));
        RT_CUDA(c, cudaMemsetAsync(a.r, 0, sizeof(double) * n, c->stream));
        if (i + 1 == p->L.size()) {
            RT_CHECK(dalloc(c, &a.dvec, 3 * (size_t)b.na));
        }
    }
    const size_t n3 = 3 * (size_t)p->L[0].nv;
    RT_CHECK(dalloc(c, &w->x, n3)); RT_CHECK(dalloc(c, &w->rr, n3)); RT_CHECK(dalloc(c, &w->z, n3));
    RT_CHECK(dalloc(c, &w->p, n3)); RT_CHECK(dalloc(c, &w->q, n3)); RT_CHECK(dalloc(c, &w->rold, n3));
    RT_CHECK(dalloc(c, &w->partials, RT_PARTIALS));
    RT_CHECK(dalloc(c, &w->scal, RT_NSCAL));
    RT_CUDA(c, cudaMemsetAsync(w->scal, 0, sizeof(double) * RT_NSCAL, c->stream));
    ws_sync(w);
    return RT_OK;
}

extern "C" int rt_hier_workspace_create(rt_hier* parent, rt_hier** out) {
    if (!parent || !out) return RT_EINVAL;
    *out = nullptr;
    RT_NOT_WORKSPACE(parent);
    RT_CUDA(parent->ctx, cudaSetDevice(parent->ctx->device));
    rt_hier* w = nullptr;
    const int s = make_workspace(parent, &w);
    if (s != RT_OK) {
        if (w) free_workspace(w);
        return s;
    }
    *out = w;
    return RT_OK;
}

// start of one instance's loop in a batched graph: iteration state, and whether to iterate at all
__global__ void k_pcg_start(double* __restrict__ scal, double tol, double maxit, double stall,
                            cudaGraphConditionalHandle cond) {
    if (threadIdx.x != 0) return;
    scal[24] = 0.0;
    scal[25] = tol;
    scal[26] = maxit;
    scal[28] = 0.0;  // batched instances run without the learned correction
    scal[29] = scal[21];
    scal[90] = scal[21];  // stall detection of reduced-precision V-cycles (k_pcg_tail)
    scal[91] = 0.0;
    scal[92] = 0.0;
    scal[93] = stall;
    const double rr = scal[21], bb = scal[22] > 0 ? scal[22] : 1.0;
    const bool go = isfinite(rr) && sqrt(rr) > tol * sqrt(bb) && maxit > 0;
    cudaGraphSetConditional(cond, go ? 1u : 0u);
}

static bool no_support_mode(const rt_hier* h) { return h->P.mode == RT_MODE_NSCF || h->P.mode == RT_MODE_NSFF; }

// one graph: per instance, prologue (child graph) -> k_pcg_start -> WHILE(one PCG iteration);
// the instances share no node, so the device runs their kernels concurrently
static int build_batch_graph_(rt_ctx* c, rt_hier* const* hs, int n, double tol, int maxit, cudaGraph_t* out,
                              std::vector<long>* once_kernels, std::vector<long>* iter_kernels);

static int build_batch_graph(rt_ctx* c, rt_hier* const* hs, int n, double tol, int maxit, cudaGraph_t* out,
                             std::vector<long>* once_kernels, std::vector<long>* iter_kernels) {
    c->batch_capture = true;
    const int s = build_batch_graph_(c, hs, n, tol, maxit, out, once_kernels, iter_kernels);
    c->batch_capture = false;
    return s;
}

static int build_batch_graph_(rt_ctx* c, rt_hier* const* hs, int n, double tol, int maxit, cudaGraph_t* out,
                              std::vector<long>* once_kernels, std::vector<long>* iter_kernels) {
    cudaGraph_t g;
    RT_CUDA(c, cudaGraphCreate(&g, 0));
    // captured launches are counted when the graph runs (pcg_batch_core)
    const long l0 = c->launches;
    for (int i = 0; i < n; i++) {
        const long lp = c->launches;
        rt_hier* h = hs[i];
        double* x = h->L[0].u;
        const double* b = h->L[0].f;
        cudaGraphConditionalHandle cond;
        cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault);
        cudaGraph_t pg = nullptr;
        int s = RT_OK;
        if (e == cudaSuccess) e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            s = pcg_prologue(h, x, b);
            e = cudaStreamEndCapture(c->stream, &pg);
        }
        cudaGraphNode_t n1 = nullptr, n2 = nullptr, n3 = nullptr;
        if (e == cudaSuccess && s == RT_OK) e = cudaGraphAddChildGraphNode(&n1, g, nullptr, 0, pg);
        if (pg) cudaGraphDestroy(pg);
        if (e == cudaSuccess && s == RT_OK) {
            double* scal = h->scal;
            double tl = tol, mi = (double)maxit;
            double stall = (h->P.precision != RT_FP64 && h->P.precision_fallback > 0) ? (double)h->P.precision_fallback : 0.0;
            void* args[] = {(void*)&scal, (void*)&tl, (void*)&mi, (void*)&stall, (void*)&cond};
            cudaKernelNodeParams kp = {};
            kp.func = (void*)k_pcg_start;
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(32);
            kp.kernelParams = args;
            e = cudaGraphAddKernelNode(&n2, g, &n1, 1, &kp);
        }
        once_kernels->push_back(c->launches - lp + 1);
        const long lb = c->launches;
        cudaGraph_t body = nullptr;
        if (e == cudaSuccess && s == RT_OK) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            e = cudaGraphAddNode(&n3, g, &n2, 1, &cp);
            body = cp.conditional.phGraph_out[0];
        }
        if (e == cudaSuccess && s == RT_OK)
            e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess && s == RT_OK) {
            s = pcg_body(h, x, h->rr, no_support_mode(h), cond, 1);
            cudaGraph_t captured = nullptr;
            e = cudaStreamEndCapture(c->stream, &captured);
        }
        iter_kernels->push_back(c->launches - lb);
        if (s != RT_OK || e != cudaSuccess) {
            c->launches = l0;
            cudaGraphDestroy(g);
            if (s != RT_OK) return s;
            return rt_fail(c, RT_ECUDA, "batched PCG graph (instance %d): %s", i, cudaGetErrorString(e));
        }
    }
    c->launches = l0;
    *out = g;
    return RT_OK;
}

// key of a batched graph: the instances, their operator epochs and solver settings, tol, maxit
static uint64_t batch_key(rt_hier* const* hs, int n, double tol, int maxit) {
    uint64_t k = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { k = (k ^ v) * 1099511628211ull; };
    for (int i = 0; i < n; i++) {
        const rt_hier* h = hs[i];
        mix(h->uid);
        mix(h->graph_epoch);
        mix((uint64_t)h->P.precision | ((uint64_t)h->P.smoother << 4) | ((uint64_t)h->P.pre_sweeps << 8) |
            ((uint64_t)h->P.post_sweeps << 16) | ((uint64_t)h->P.mode << 24) | ((uint64_t)h->P.cycle_gamma << 32) |
            ((uint64_t)h->P.coarse_sweeps << 40) | ((uint64_t)h->P.precision_fallback << 48));
        mix((uint64_t)h->P.coarse_bf16);
        mix((uint64_t)(uint32_t)h->P.cycle_gamma_levels);
        uint64_t om;
        memcpy(&om, &h->P.jacobi_omega, 8);
        mix(om);
    }
    uint64_t tb;
    memcpy(&tb, &tol, 8);
    mix(tb);
    mix((uint64_t)maxit);
    return k;
}

static int pcg_batch_core(rt_hier* const* hs, int n, double tol, int maxit, rt_solve_info* infos) {
    rt_ctx* c = hs[0]->ctx;
    for (int i = 0; i < n; i++) {
        rt_hier* h = hs[i];
        if (h->ctx != c) return rt_fail(c, RT_EINVAL, "batched solves must share one context");
        for (int j = 0; j < i; j++)
            if (hs[j] == h) return rt_fail(c, RT_EINVAL, "instance %d appears twice in the batch", i);
        RT_CHECK(need_stencil(h));
        if (no_support_mode(h) && h->Ru == nullptr) {
            rt_hier* owner = h->parent ? h->parent : h;
            RT_CHECK(rtk::rigid_nodes(owner));
            ws_sync(h);
        }
    }
    cudaEvent_t ea, eb;
    cudaEventCreate(&ea);
    cudaEventCreate(&eb);
    cudaEventRecord(ea, c->stream);
    std::vector<long> batch_once, batch_iter;  // kernels of the graph run, per instance
    if (c->profile || !hs[0]->use_graphs) {
        // per-kernel events cannot sit inside a graph: run the instances one after the other
        for (int i = 0; i < n; i++) {
            rt_solve_info si;
            memset(&si, 0, sizeof(si));
            int vc = 0;
            RT_CHECK(pcg_core(hs[i], hs[i]->L[0].u, hs[i]->L[0].f, tol, maxit, &si, &vc));
        }
    } else {
        const uint64_t key = batch_key(hs, n, tol, maxit);
        rt_ctx::BatchGraph* bg = nullptr;
        for (auto& e : c->batch_graphs)
            if (e.key == key) bg = &e;
        if (!bg) {
            rt_ctx::BatchGraph nb;
            nb.key = key;
            for (int i = 0; i < n; i++) nb.uids.push_back(hs[i]->uid);
            RT_CHECK(build_batch_graph(c, hs, n, tol, maxit, &nb.graph, &nb.once_kernels, &nb.iter_kernels));
            cudaError_t e = cudaGraphInstantiate(&nb.exec, nb.graph, 0);
            if (e != cudaSuccess) {
                cudaGraphDestroy(nb.graph);
                return rt_fail(c, RT_ECUDA, "batched PCG graph instantiation failed: %s", cudaGetErrorString(e));
            }
            if (c->batch_graphs.size() >= 4) {  // keep the four most recent batches
                cudaGraphExecDestroy(c->batch_graphs.front().exec);
                cudaGraphDestroy(c->batch_graphs.front().graph);
                c->batch_graphs.erase(c->batch_graphs.begin());
            }
            c->batch_graphs.push_back(nb);
            bg = &c->batch_graphs.back();
        }
        RT_CUDA(c, cudaGraphLaunch(bg->exec, c->stream));
        batch_once = bg->once_kernels;
        batch_iter = bg->iter_kernels;
    }
    cudaEventRecord(eb, c->stream);
    cudaEventSynchronize(eb);
    float ms = 0;
    cudaEventElapsedTime(&ms, ea, eb);
    cudaEventDestroy(ea);
    cudaEventDestroy(eb);
    RT_CUDA(c, cudaGetLastError());
    for (int i = 0; i < n; i++) {
        rt_hier* h = hs[i];
        double sc[4], stall = 0;
        RT_CHECK(read_scalars(h, 21, 4, sc));  // r.r, b.b, (unused), iterations
        RT_CHECK(read_scalars(h, 92, 1, &stall));
        const double bn = sc[1] > 0 ? std::sqrt(sc[1]) : 1.0;
        double rel = std::sqrt(sc[0]) / bn;
        int its = (int)sc[3];
        if (!batch_iter.empty()) c->launches += batch_once[i] + batch_iter[i] * its;
        if (!std::isfinite(sc[0])) return nan_fail(h, its);
        if (stall != 0.0 && rel > tol && its < maxit) {
            // this instance's reduced-precision V-cycles stalled: continue it alone with FP64 ones
            const int saved = h->P.precision;
            h->P.precision = RT_FP64;
            rt_solve_info sub;
            memset(&sub, 0, sizeof(sub));
            int vc = 0;
            const int st2 = pcg_core(h, h->L[0].u, h->L[0].f, tol, maxit - its, &sub, &vc);
            h->P.precision = saved;
            RT_CHECK(st2);
            its += sub.iterations;
            rel = sub.rel_residual;
            h->fallbacks++;
        }
        if (infos) {
            rt_solve_info& si = infos[i];
            memset(&si, 0, sizeof(si));
            si.iterations = its;
            si.vcycles = its;
            si.rel_residual = rel;
            si.status = rel <= tol ? RT_OK : RT_ENOCONV;
            si.seconds = ms * 1e-3;
            RT_CHECK(rtk::dot(h, 3 * h->L[0].nv, h->L[0].f, h->L[0].u, h->scal + 2));
            RT_CHECK(read_scalars(h, 2, 1, &si.value));
        }
    }
    return RT_OK;
}

extern "C" int rt_pcg_batch(rt_hier* const* hs, int n, double tol, int maxit, rt_solve_info* infos) {
    if (!hs || n < 1 || tol <= 0 || maxit < 0) return RT_EINVAL;
    for (int i = 0; i < n; i++)
        if (!hs[i]) return RT_EINVAL;
    RT_CUDA(hs[0]->ctx, cudaSetDevice(hs[0]->ctx->device));
    return pcg_batch_core(hs, n, tol, maxit, infos);
}

// ---------------------------------------------------------------------------
// block Lanczos on the load-space compliance operator A = P S K^-1 S^T P:
// block size bs, nblk block steps, full CGS2 re-orthogonalisation, Rayleigh-Ritz on
// the projected (nblk bs)^2 matrix; each block step's bs inner solves run as one
// batched graph on bs solve workspaces
// ---------------------------------------------------------------------------

// cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major, overwritten);
// returns the largest eigenvalue and its unit eigenvector
static double sym_max_eig(int n, std::vector<double>& A, std::vector<double>& vec) {
    std::vector<double> V((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                const double a = A[(size_t)i * n + j] * A[(size_t)i * n + j];
                tot += a;
                if (i != j) off += a;
            }
        if (off <= 1e-30 * tot || off == 0) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = A[(size_t)p * n + q];
                if (apq == 0) continue;
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                // rotation angle zeroing A[p][q]: tan(2 phi) = 2 apq / (aqq - app)
                const double theta = (aqq - app) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                const double cs = 1 / std::sqrt(t * t + 1), sn = t * cs;
                for (int k = 0; k < n; k++) {  // A <- A J (columns p, q)
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = cs * akp - sn * akq;
                    A[(size_t)k * n + q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < n; k++) {  // A <- J^T A (rows p, q)
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = cs * apk - sn * aqk;
                    A[(size_t)q * n + k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < n; k++) {  // V <- V J
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = cs * vkp - sn * vkq;
                    V[(size_t)k * n + q] = sn * vkp + cs * vkq;
                }
            }
    }
    int best = 0;
    for (int i = 1; i < n; i++)
        if (A[(size_t)i * n + i] > A[(size_t)best * n + best]) best = i;
    vec.resize(n);
    for (int k = 0; k < n; k++) vec[k] = V[(size_t)k * n + best];
    return A[(size_t)best * n + best];
}

// w -= sum_c (Q_c . w) Q_c over columns [0, m), twice (CGS2); coef[c] accumulates both passes
static int cgs2(rt_hier* h, long nl, int m, const double* Q, double* w, double* dcoef, std::vector<double>& coef) {
    rt_ctx* c = h->ctx;
    coef.assign(m, 0.0);
    for (int pass = 0; pass < 2; pass++) {
        for (int c0 = 0; c0 < m; c0 += 64) {
            const int mm = std::min(64, m - c0);
            const double* Qc = Q + (long)c0 * nl;
            RT_CHECK(multidot(h, nl, mm, Qc, w, dcoef));
            RT_CHECK(rt_launch(c, "lanczos_sub", [&] {
                k_sub_multi<<<(unsigned)std::min<long>((nl + 255) / 256, c->sm_count * 8), 256, 0, c->stream>>>(
                    nl, mm, Qc, dcoef, w);
            }));
            RT_CUDA(c, cudaMemcpyAsync(c->hscal, dcoef, sizeof(double) * mm, cudaMemcpyDeviceToHost, c->stream));
            RT_CUDA(c, cudaStreamSynchronize(c->stream));
            for (int k = 0; k < mm; k++) coef[c0 + k] += c->hscal[k];
        }
    }
    return RT_OK;
}

// |w| into the host, then w /= |w|
static int normalize(rt_hier* h, long nl, double* w, double* norm) {
    RT_CHECK(rtk::dot(h, nl, w, w, h->scal + 34));
    double s;
    RT_CHECK(read_scalars(h, 34, 1, &s));
    *norm = std::sqrt(s);
    if (!(*norm > 0) || !std::isfinite(*norm)) return RT_OK;
    return rtk::scale(h, nl, w, h->scal + 34, true);
}

static int block_lanczos(rt_hier* h, int bs, int nblk, double inner_tol, uint64_t seed, double* lambda,
                         rt_solve_info* info) {
    rt_ctx* c = h->ctx;
    rt_level& L = h->L[0];
    const long n = 3 * L.nv, nl = 3L * h->nload;
    if (h->nload == 0) return rt_fail(c, RT_ESTATE, "no load nodes");
    if (bs < 1 || bs > 16 || nblk < 1 || (long)bs * nblk > 128)
        return rt_fail(c, RT_EINVAL, "block Lanczos needs 1 <= block size <= 16 and block size x steps <= 128");
    const int mcap = (nblk + 1) * bs;
    if (h->Qcap < mcap) {
        cudaFree(h->Q);
        h->Q = nullptr;
        RT_CHECK(dalloc(c, &h->Q, (size_t)mcap * nl));
        h->Qcap = mcap;
    }
    while ((int)h->wspool.size() < bs) {
        rt_hier* w = nullptr;
        const int s = make_workspace(h, &w);
        if (s != RT_OK) {
            if (w) free_workspace(w);
            return s;
        }
        h->wspool.push_back(w);
    }
    if (no_support_mode(h) && h->Ru == nullptr) RT_CHECK(rtk::rigid_nodes(h));
    double* Q = h->Q;
    double* dcoef = h->scal + 240;  // [64]
    const int m = nblk * bs;        // Krylov dimension
    std::vector<double> H((size_t)m * m, 0.0), coef;
    int inner = 0, vcycles = 0;
    // starting block: bs projected random loads, orthonormalised
    int ncol = 0;
    for (int i = 0; i < bs; i++) {
        double* qi = Q + (long)i * nl;
        RT_CHECK(rtk::rng_uniform(h, seed + 0x9e3779b97f4a7c15ull * (uint64_t)i, n, L.f));
        RT_CHECK(rtk::project_load(h, L.f));
        RT_CHECK(rtk::gather_load(h, L.f, qi));
        if (i > 0) RT_CHECK(cgs2(h, nl, i, Q, qi, dcoef, coef));
        double nr;
        RT_CHECK(normalize(h, nl, qi, &nr));
        if (!(nr > 0)) return rt_fail(c, RT_ENAN, "block Lanczos: degenerate starting block");
        ncol++;
    }
    std::vector<rt_hier*> ws(h->wspool.begin(), h->wspool.begin() + bs);
    std::vector<rt_solve_info> si(bs);
    int done_blocks = 0;
    for (int j = 0; j < nblk; j++) {
        // A Q_j: scatter each column into its workspace's right-hand side, solve all bs at once
        for (int i = 0; i < bs; i++) {
            rt_hier* w = ws[i];
            ws_sync(w);
            RT_CUDA(c, cudaMemsetAsync(w->L[0].f, 0, sizeof(double) * n, c->stream));
            RT_CHECK(rtk::scatter_load(w, Q + (long)(j * bs + i) * nl, w->L[0].f));
            RT_CUDA(c, cudaMemsetAsync(w->L[0].u, 0, sizeof(double) * n, c->stream));
        }
        RT_CHECK(pcg_batch_core(ws.data(), bs, inner_tol, 500, si.data()));
        for (int i = 0; i < bs; i++) {
            inner += si[i].iterations;
            vcycles += si[i].vcycles;
        }
        // new columns: orthogonalise against every earlier column; the coefficients and the
        // norm are column j bs + i of the projected matrix H = Q^T A Q
        bool breakdown = false;
        for (int i = 0; i < bs; i++) {
            const int col = (j + 1) * bs + i;
            double* wv = Q + (long)col * nl;
            RT_CUDA(c, cudaMemcpyAsync(h->z, ws[i]->L[0].u, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
            RT_CHECK(rtk::project_load(h, h->z));
            RT_CHECK(rtk::gather_load(h, h->z, wv));
            RT_CHECK(cgs2(h, nl, col, Q, wv, dcoef, coef));
            double nr;
            RT_CHECK(normalize(h, nl, wv, &nr));
            const int hc = j * bs + i;
            for (int r = 0; r < std::min(col, m); r++) H[(size_t)r * m + hc] = coef[r];
            if (col < m) H[(size_t)col * m + hc] = nr;
            if (!std::isfinite(nr)) return rt_fail(c, RT_ENAN, "NaN in block Lanczos");
            if (nr <= 1e-13 * std::fabs(H[(size_t)hc * m + hc])) breakdown = true;
        }
        done_blocks = j + 1;
        if (breakdown) break;  // invariant subspace: the Ritz values are exact
    }
    const int mk = done_blocks * bs;
    std::vector<double> T((size_t)mk * mk), y;
    for (int r = 0; r < mk; r++)
        for (int q = 0; q < mk; q++) T[(size_t)r * mk + q] = 0.5 * (H[(size_t)r * m + q] + H[(size_t)q * m + r]);
    const double theta = sym_max_eig(mk, T, y);
    // worst-case load f = Q y on the load set, u = K^-1 f
    double* dy = nullptr;
    RT_CHECK(dalloc(c, &dy, mk));
    RT_CUDA(c, cudaMemcpyAsync(dy, y.data(), sizeof(double) * mk, cudaMemcpyHostToDevice, c->stream));
    int st = rt_launch(c, "lanczos_combine", [&] {
        k_combine<<<(unsigned)std::min<long>((nl + 255) / 256, c->sm_count * 8), 256, 0, c->stream>>>(nl, mk, Q, dy,
                                                                                                      h->fs_old);
    });
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(dy);
    RT_CHECK(st);
    RT_CUDA(c, cudaMemsetAsync(L.f, 0, sizeof(double) * n, c->stream));
    RT_CHECK(rtk::scatter_load(h, h->fs_old, L.f));
    RT_CUDA(c, cudaMemsetAsync(L.u, 0, sizeof(double) * n, c->stream));
    rt_solve_info fin;
    memset(&fin, 0, sizeof(fin));
    RT_CHECK(pcg_core(h, L.u, L.f, inner_tol, 500, &fin, &vcycles));
    inner += fin.iterations;
    *lambda = theta;
    if (info) {
        info->iterations = done_blocks;
        info->inner_iterations = inner;
        info->vcycles = vcycles;
        info->rel_residual = fin.rel_residual;
        info->value = theta;
        info->status = RT_OK;
    }
    return RT_OK;
}

extern "C" int rt_worst_case_block(rt_hier* h, int block_size, int n_blocks, double inner_tol, uint64_t seed,
                                   double* lambda, rt_solve_info* info) {
    if (!h || !lambda || inner_tol <= 0) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CHECK(need_stencil(h));
    rt_solve_info loc;
    memset(&loc, 0, sizeof(loc));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, h->ctx->stream);
    const int s = block_lanczos(h, block_size, n_blocks, inner_tol, seed, lambda, &loc);
    cudaEventRecord(b, h->ctx->stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    loc.seconds = ms * 1e-3;
    if (info) *info = loc;
    return s;
}

// ---------------------------------------------------------------------------
// learned preconditioner: attach a network, harvest training samples
// ---------------------------------------------------------------------------
extern "C" int rt_hier_set_learned(rt_hier* h, rt_unet* u, double fallback_ratio) {
    if (!h) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    if (u && !rtu::box_matches(u, h))
        return rt_fail(h->ctx, RT_EINVAL, "the network's box must equal the finest level's node box");
    if (u && !(fallback_ratio > 0)) return rt_fail(h->ctx, RT_EINVAL, "fallback ratio must be positive");
    h->unet = u;
    h->unet_fallback = fallback_ratio;
    h->unet_off = false;
    h->unet_verdict_epoch = ~0ull;
    h->unet_applied = 0;
    h->graph_epoch++;
    return RT_OK;
}

extern "C" int rt_hier_set_learned_post(rt_hier* h, int sweeps) {
    if (!h || sweeps < 0 || sweeps > RT_CHEBY_MAXK) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    h->unet_post = sweeps;
    h->graph_epoch++;
    return RT_OK;
}

extern "C" int rt_hier_learned_stats(rt_hier* h, long long* applied, int* judged_off) {
    if (!h) return RT_EINVAL;
    if (applied) *applied = h->unet_applied;
    if (judged_off) *judged_off = h->unet_off ? 1 : 0;
    return RT_OK;
}

__global__ void k_zero_fixed(long n, long nv, const uint8_t* __restrict__ vact, const uint8_t* __restrict__ vfix,
                             int ws, double* __restrict__ f) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long v = i % nv;
        if (!vact[v] || (ws && vfix[v])) f[i] = 0.0;
    }
}

// one training sample from the solver: a random load on the free nodes, k PCG iterations
// (plain V-cycle) from zero give the residual r; the input packs (density, r, zv = one V-cycle
// applied to r), the target is the V-cycle's error on r: K^-1 r (PCG to 1e-10) minus zv
extern "C" int rt_unet_harvest(rt_hier* h, rt_unet* u, int k_iter, uint64_t seed, void* in_out, float* tgt_out) {
    if (!h || !u || !in_out || !tgt_out || k_iter < 0) return RT_EINVAL;
    RT_NOT_WORKSPACE(h);
    RT_CHECK(need_stencil(h));
    rt_ctx* c = h->ctx;
    if (!rtu::box_matches(u, h)) return rt_fail(c, RT_EINVAL, "the network's box must equal the finest node box");
    if (no_support_mode(h)) return rt_fail(c, RT_EINVAL, "training samples need a supported structure");
    rt_level& L = h->L[0];
    const long n = 3 * L.nv;
    rt_unet* saved = h->unet;
    h->unet = nullptr;
    double* zv = nullptr;
    int s = RT_OK;
    auto step = [&](int st) { if (s == RT_OK) s = st; return s == RT_OK; };
    if (cudaMallocAsync(&zv, sizeof(double) * n, c->stream) != cudaSuccess) {
        h->unet = saved;
        return rt_fail(c, RT_ENOMEM, "harvest scratch");
    }
    step(rtk::rng_uniform(h, seed, n, L.f));
    if (s == RT_OK)
        step(rt_launch(c, "zero_fixed", [&] {
            k_zero_fixed<<<(unsigned)std::min<long>((n + 255) / 256, c->sm_count * 16L), 256, 0, c->stream>>>(
                n, L.nv, L.vact, h->vfix, h->has_support ? 1 : 0, L.f);
        }));
    if (s == RT_OK) cudaMemsetAsync(L.u, 0, sizeof(double) * n, c->stream);
    if (s == RT_OK) step(pcg_prologue(h, L.u, L.f));
    if (s == RT_OK) {
        const double st[6] = {0.0, 0.0, (double)k_iter, 1.0, 0.0, 0.0};
        memcpy(c->hscal + 8, st, sizeof(st));
        cudaMemcpyAsync(h->scal + 24, c->hscal + 8, sizeof(st), cudaMemcpyHostToDevice, c->stream);
    }
    for (int i = 0; i < k_iter && s == RT_OK; i++) step(pcg_body(h, L.u, h->rr, false, 0, 0));
    // r_k becomes the right-hand side; r.r in scal[35]
    if (s == RT_OK) cudaMemcpyAsync(L.f, h->rr, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream);
    if (s == RT_OK) step(rtk::dot(h, n, L.f, L.f, h->scal + 35));
    if (s == RT_OK) step(precondition(h, L.f, zv, h->scal + 35));
    if (s == RT_OK) step(rtk::dot(h, n, zv, zv, h->scal + 37));
    if (s == RT_OK) step(rtu::pack(u, h, L.f, h->scal + 35, zv, h->scal + 37));
    if (s == RT_OK)
        cudaMemcpyAsync(in_out, rtu::input(u), sizeof(__nv_bfloat16) * 16 * rtu::voxels(u), cudaMemcpyDeviceToDevice,
                        c->stream);
    rt_solve_info si;
    memset(&si, 0, sizeof(si));
    int vc = 0;
    if (s == RT_OK) cudaMemsetAsync(L.u, 0, sizeof(double) * n, c->stream);
    if (s == RT_OK) step(pcg_core(h, L.u, L.f, 1e-10, 2000, &si, &vc));
    if (s == RT_OK) step(rtu::target(u, h, L.u, zv, h->scal + 37, tgt_out));
    cudaFreeAsync(zv, c->stream);
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    h->unet = saved;
    if (s != RT_OK) return s;
    if (e != cudaSuccess) return rt_fail(c, RT_ECUDA, "harvest: %s", cudaGetErrorString(e));
    if (si.status != RT_OK) return rt_fail(c, RT_ENOCONV, "harvest: the exact-error solve did not converge");
    return RT_OK;
}

extern "C" long long rt_hier_precision_fallbacks(rt_hier* h) { return h ? h->fallbacks : 0; }
