// The method of moving asymptotes for one inequality constraint, on the device: the alternative
// density update of optimization/mma_t.{h,cpp,cu} (class MMA::mma_t: mma_t(n, 1), init(lower,
// upper), update(df, dg, g), get_x).
//
// Per update (x^k the current design, L / U the asymptotes, alpha / beta the move bounds):
//   p_ij = (U_j - x_j)^2 (1.001 df_ij+ + 0.001 df_ij- + 1e-5 / (xmax_j - xmin_j)),
//   q_ij = (x_j - L_j)^2 (0.001 df_ij+ + 1.001 df_ij- + 1e-5 / (xmax_j - xmin_j))
// for the objective (i = 0) and the constraint (i = 1) (mma_t.cu:70-81); b = the constraint
// approximation at x^k minus g (mma_t.cu:83-89); a0 = 1, a = 0, c = 10, d = 1 (mma_t.h:229-237).
// The subproblem min f0~(x) + a0 z + c y + d y^2 / 2, f1~(x) - a z - y <= b, alpha <= x <= beta
// has z = 0 at its optimum (a = 0), and its dual is a concave function of the one multiplier
// lambda >= 0 with the monotone derivative
//   h(lambda) = sum_j p_1j / (U_j - x_j(lambda)) + q_1j / (x_j(lambda) - L_j) - y(lambda) - b,
//   x_j(lambda) = clamp((sqrt(P) L_j + sqrt(Q) U_j) / (sqrt(P) + sqrt(Q)), alpha_j, beta_j),
//   P = p_0j + lambda p_1j, Q = q_0j + lambda q_1j, y(lambda) = max(0, (lambda - c) / d).
// Its root (0 when h(0) <= 0) is bracketed and bisected; each evaluation is one pass over the
// design variables with a fixed-order block reduction.  The reference reaches the same optimum
// with a primal-dual interior-point method (mma_t.cu:330-500, epsilon down to 1e-6).  Then the
// asymptotes and move bounds move as in mma_t::adjust_asym (mma_t.cu:164-226).  State in FP64;
// the gradients are FP32 device arrays, as the reference's Scalar.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "rt_internal.h"

struct rt_mma {
    rt_ctx* ctx = nullptr;
    long long n = 0;
    double *xmin = nullptr, *xmax = nullptr, *x = nullptr, *low = nullptr, *upp = nullptr;
    double *alpha = nullptr, *beta = nullptr, *lastdx = nullptr, *pq = nullptr;
    double* partials = nullptr;  // RT_RED_BLOCKS block sums, then the total
    double* host = nullptr;      // pinned: one value read back per evaluation
    int stop_counter = 0;
    long long evaluations = 0;
};

namespace {

constexpr double kC = 10.0, kD = 1.0, kRaa0 = 1e-5;
constexpr int kBS = 256;

__device__ __forceinline__ double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ double x_of(double lam, double p0, double q0, double p1, double q1, double l, double u,
                                       double a, double b) {
    const double sp = sqrt(p0 + lam * p1), sq = sqrt(q0 + lam * q1);
    return clampd((sp * l + sq * u) / (sp + sq), a, b);
}

// fixed-order block sum of v into out[blockIdx.x]
__device__ __forceinline__ void block_sum(double v, double* out) {
    __shared__ double red[kBS / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < kBS / 32 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) out[blockIdx.x] = v;
    }
}

__global__ void k_mma_init(long long n, const double* __restrict__ xmin, const double* __restrict__ xmax,
                           double* __restrict__ x, double* __restrict__ low, double* __restrict__ upp,
                           double* __restrict__ alpha, double* __restrict__ beta, double* __restrict__ lastdx) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const double D = xmax[j] - xmin[j], xj = 0.5 * (xmin[j] + xmax[j]);
        const double l = clampd(xmin[j], xj - 10 * D, xj - 0.01 * D), u = clampd(xmax[j], xj + 0.01 * D, xj + 10 * D);
        x[j] = xj;
        low[j] = l;
        upp[j] = u;
        alpha[j] = fmax(fmax(xmin[j], l + 0.1 * (xj - l)), xj - 0.5 * D);
        beta[j] = fmin(fmin(xmax[j], u - 0.1 * (u - xj)), xj + 0.5 * D);
        lastdx[j] = 0.0;
    }
}

// p0, q0, p1, q1 and the block sums of the constraint approximation at x^k
__global__ void k_mma_pq(long long n, const float* __restrict__ df, const float* __restrict__ dg,
                         const double* __restrict__ xmin, const double* __restrict__ xmax,
                         const double* __restrict__ x, const double* __restrict__ low,
                         const double* __restrict__ upp, double* __restrict__ pq, double* __restrict__ partials) {
    double s = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const double ux = upp[j] - x[j], xl = x[j] - low[j], r = kRaa0 / (xmax[j] - xmin[j]);
        const double f0 = df[j], f1 = dg[j];
        const double f0p = f0 > 0 ? f0 : 0, f0m = f0 < 0 ? -f0 : 0, f1p = f1 > 0 ? f1 : 0, f1m = f1 < 0 ? -f1 : 0;
        const double p1 = ux * ux * (1.001 * f1p + 0.001 * f1m + r), q1 = xl * xl * (0.001 * f1p + 1.001 * f1m + r);
        pq[j] = ux * ux * (1.001 * f0p + 0.001 * f0m + r);
        pq[n + j] = xl * xl * (0.001 * f0p + 1.001 * f0m + r);
        pq[2 * n + j] = p1;
        pq[3 * n + j] = q1;
        s += p1 / ux + q1 / xl;
    }
    block_sum(s, partials);
}

// block sums of sum_j p1 / (U - x(lambda)) + q1 / (x(lambda) - L)
__global__ void k_mma_h(long long n, double lam, const double* __restrict__ pq, const double* __restrict__ low,
                        const double* __restrict__ upp, const double* __restrict__ alpha,
                        const double* __restrict__ beta, double* __restrict__ partials) {
    double s = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const double p1 = pq[2 * n + j], q1 = pq[3 * n + j];
        const double xj = x_of(lam, pq[j], pq[n + j], p1, q1, low[j], upp[j], alpha[j], beta[j]);
        s += p1 / (upp[j] - xj) + q1 / (xj - low[j]);
    }
    block_sum(s, partials);
}

// the new design, asymptotes and move bounds; block sums of |dx|^2
__global__ void k_mma_apply(long long n, double lam, const double* __restrict__ pq, const double* __restrict__ xmin,
                            const double* __restrict__ xmax, double* __restrict__ x, double* __restrict__ low,
                            double* __restrict__ upp, double* __restrict__ alpha, double* __restrict__ beta,
                            double* __restrict__ lastdx, double* __restrict__ partials) {
    const double tenth = (double)0.1f;  // the reference's float literal (mma_t.cu:214, 219)
    double s = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const double l = low[j], u = upp[j], xo = x[j];
        const double xn = x_of(lam, pq[j], pq[n + j], pq[2 * n + j], pq[3 * n + j], l, u, alpha[j], beta[j]);
        const double dx = xn - xo, D = xmax[j] - xmin[j], ld = lastdx[j];
        const double gam = dx * ld > 0 ? 1.2 : (dx * ld < 0 ? 0.7 : 1.0);
        const double nl = clampd(xn - gam * (xo - l), xn - 10 * D, xn - 0.01 * D);
        const double nu = clampd(xn + gam * (u - xo), xn + 0.01 * D, xn + 10 * D);
        double a = xmin[j], t = nl + tenth * (xn - nl);
        if (a < t) a = t;
        t = xn - 0.5 * D;
        if (a < t) a = t;
        double b = xmax[j];
        t = nu - tenth * (nu - xn);
        if (b > t) b = t;
        t = xn + 0.5 * D;
        if (b > t) b = t;
        low[j] = nl;
        upp[j] = nu;
        alpha[j] = a;
        beta[j] = b;
        lastdx[j] = dx;
        x[j] = xn;
        s += dx * dx;
    }
    block_sum(s, partials);
}

__global__ void k_mma_total(int nb, double* __restrict__ partials) {
    double v = 0;
    for (int i = threadIdx.x; i < nb; i += 32) v += partials[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partials[nb] = v;
}

__global__ void k_mma_to_rho(long long n, const double* __restrict__ x, const uint8_t* __restrict__ eact,
                             float* __restrict__ rho) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
        rho[j] = eact[j] ? (float)x[j] : 0.f;
}

int nblocks(const rt_mma* m) {
    const long long need = (m->n + kBS - 1) / kBS;
    return (int)(need < RT_RED_BLOCKS ? (need > 0 ? need : 1) : RT_RED_BLOCKS);
}

// the block sums' total, read back to the host
int total(rt_mma* m, double* out) {
    rt_ctx* c = m->ctx;
    const int nb = nblocks(m);
    RT_CHECK(rt_launch(c, "mma_total", [&] { k_mma_total<<<1, 32, 0, c->stream>>>(nb, m->partials); }));
    RT_CUDA(c, cudaMemcpyAsync(m->host, m->partials + nb, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    *out = m->host[0];
    return RT_OK;
}

int eval_h(rt_mma* m, double lam, double bconst, double* h) {
    rt_ctx* c = m->ctx;
    const int nb = nblocks(m);
    RT_CHECK(rt_launch(c, "mma_dual_derivative", [&] {
        k_mma_h<<<nb, kBS, 0, c->stream>>>(m->n, lam, m->pq, m->low, m->upp, m->alpha, m->beta, m->partials);
    }));
    double s = 0;
    RT_CHECK(total(m, &s));
    m->evaluations++;
    const double y = lam > kC ? (lam - kC) / kD : 0.0;
    *h = s - y - bconst;
    return RT_OK;
}

void free_mma(rt_mma* m) {
    double* bufs[] = {m->xmin, m->xmax, m->x, m->low, m->upp, m->alpha, m->beta, m->lastdx, m->pq, m->partials};
    for (double* b : bufs)
        if (b) cudaFree(b);
    if (m->host) cudaFreeHost(m->host);
}

}  // namespace

extern "C" int rt_mma_create(rt_ctx* ctx, long long n, const double* xmin, const double* xmax, double uniform_min,
                             double uniform_max, rt_mma** out) {
    if (!ctx || !out || n < 1) return RT_EINVAL;
    if ((xmin == nullptr) != (xmax == nullptr)) return rt_fail(ctx, RT_EINVAL, "MMA bounds: give both arrays or neither");
    if (!xmin && !(uniform_max > uniform_min)) return rt_fail(ctx, RT_EINVAL, "MMA bounds: upper must exceed lower");
    RT_CUDA(ctx, cudaSetDevice(ctx->device));
    rt_mma* m = new rt_mma();
    m->ctx = ctx;
    m->n = n;
    const size_t b = sizeof(double) * (size_t)n;
    cudaError_t e = cudaSuccess;
    double** arrs[] = {&m->xmin, &m->xmax, &m->x, &m->low, &m->upp, &m->alpha, &m->beta, &m->lastdx};
    for (double** a : arrs)
        if (e == cudaSuccess) e = cudaMalloc(a, b);
    if (e == cudaSuccess) e = cudaMalloc(&m->pq, 4 * b);
    if (e == cudaSuccess) e = cudaMalloc(&m->partials, sizeof(double) * (RT_RED_BLOCKS + 1));
    if (e == cudaSuccess) e = cudaMallocHost(&m->host, sizeof(double) * 2);
    if (e != cudaSuccess) {
        cudaGetLastError();
        free_mma(m);
        delete m;
        return rt_fail(ctx, RT_ENOMEM, "MMA state of %lld variables: %s", n, cudaGetErrorString(e));
    }
    int st = RT_OK;
    if (xmin) {
        if (cudaMemcpy(m->xmin, xmin, b, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(m->xmax, xmax, b, cudaMemcpyHostToDevice) != cudaSuccess)
            st = rt_fail(ctx, RT_ECUDA, "MMA bounds upload failed");
        for (long long j = 0; st == RT_OK && j < n; j++)
            if (!(xmax[j] > xmin[j])) st = rt_fail(ctx, RT_EINVAL, "MMA bounds: xmax[%lld] <= xmin[%lld]", j, j);
    } else {
        std::vector<double> lo((size_t)n, uniform_min), hi((size_t)n, uniform_max);
        if (cudaMemcpy(m->xmin, lo.data(), b, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(m->xmax, hi.data(), b, cudaMemcpyHostToDevice) != cudaSuccess)
            st = rt_fail(ctx, RT_ECUDA, "MMA bounds upload failed");
    }
    if (st == RT_OK)
        st = rt_launch(ctx, "mma_init", [&] {
            k_mma_init<<<nblocks(m), kBS, 0, ctx->stream>>>(n, m->xmin, m->xmax, m->x, m->low, m->upp, m->alpha,
                                                             m->beta, m->lastdx);
        });
    if (st == RT_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        st = rt_fail(ctx, RT_ECUDA, "MMA initialisation failed");
    if (st != RT_OK) {
        free_mma(m);
        delete m;
        return st;
    }
    rt_ctx_retain(ctx);
    *out = m;
    return RT_OK;
}

extern "C" int rt_mma_destroy(rt_mma* m) {
    if (!m) return RT_EINVAL;
    rt_ctx* c = m->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    free_mma(m);
    delete m;
    rt_ctx_release(c);
    return RT_OK;
}

extern "C" int rt_mma_update(rt_mma* m, const float* df_dev, const float* dg_dev, double g, int* stop,
                             double* lambda_out, double* dxnorm_out) {
    if (!m || !df_dev || !dg_dev) return RT_EINVAL;
    if (!std::isfinite(g)) return rt_fail(m->ctx, RT_ENAN, "MMA update: the constraint value is not finite");
    rt_ctx* c = m->ctx;
    RT_CUDA(c, cudaSetDevice(c->device));
    const int nb = nblocks(m);
    RT_CHECK(rt_launch(c, "mma_pq", [&] {
        k_mma_pq<<<nb, kBS, 0, c->stream>>>(m->n, df_dev, dg_dev, m->xmin, m->xmax, m->x, m->low, m->upp, m->pq,
                                            m->partials);
    }));
    double gk = 0;
    RT_CHECK(total(m, &gk));
    if (!std::isfinite(gk)) return rt_fail(c, RT_ENAN, "MMA update: a gradient is not finite");
    const double bconst = gk - g;
    double lam = 0, h = 0;
    RT_CHECK(eval_h(m, 0.0, bconst, &h));
    if (h > 0) {
        double lo = 0, hi = 1;
        for (int k = 0; k < 400; k++) {
            RT_CHECK(eval_h(m, hi, bconst, &h));
            if (!(h > 0)) break;
            lo = hi;
            hi *= 4;
        }
        for (int k = 0; k < 200 && hi - lo > 1e-15 * hi; k++) {
            const double mid = 0.5 * (lo + hi);
            RT_CHECK(eval_h(m, mid, bconst, &h));
            if (h > 0)
                lo = mid;
            else
                hi = mid;
        }
        lam = 0.5 * (lo + hi);
    }
    RT_CHECK(rt_launch(c, "mma_apply", [&] {
        k_mma_apply<<<nb, kBS, 0, c->stream>>>(m->n, lam, m->pq, m->xmin, m->xmax, m->x, m->low, m->upp, m->alpha,
                                               m->beta, m->lastdx, m->partials);
    }));
    double dx2 = 0;
    RT_CHECK(total(m, &dx2));
    const double dxn = std::sqrt(dx2);
    // mma_t::update (mma_t.cpp:38-48): a step shorter than 1e-3 counts towards the stop, which
    // is reported after more than 10 of them
    if (dxn < 1e-3) m->stop_counter++;
    if (stop) *stop = m->stop_counter > 10 ? 1 : 0;
    if (lambda_out) *lambda_out = lam;
    if (dxnorm_out) *dxnorm_out = dxn;
    return RT_OK;
}

extern "C" int rt_mma_x(rt_mma* m, const double** x_dev) {
    if (!m || !x_dev) return RT_EINVAL;
    *x_dev = m->x;
    return RT_OK;
}

extern "C" int rt_mma_get_x(rt_mma* m, double* x_host) {
    if (!m || !x_host) return RT_EINVAL;
    rt_ctx* c = m->ctx;
    RT_CUDA(c, cudaMemcpyAsync(x_host, m->x, sizeof(double) * m->n, cudaMemcpyDeviceToHost, c->stream));
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    return RT_OK;
}

extern "C" int rt_mma_set_density(rt_mma* m, rt_hier* h) {
    if (!m || !h) return RT_EINVAL;
    if (h->parent) return rt_fail(m->ctx, RT_ESTATE, "a solve workspace has no density of its own");
    if (h->ctx != m->ctx) return rt_fail(m->ctx, RT_EINVAL, "the MMA state and the hierarchy must share a context");
    rt_level& L = h->L[0];
    if (L.ne != m->n)
        return rt_fail(m->ctx, RT_EINVAL, "MMA state has %lld variables, the finest level %ld elements", m->n, L.ne);
    rt_ctx* c = m->ctx;
    h->stencil_ready = false;
    h->design_epoch++;
    return rt_launch(c, "mma_set_density", [&] {
        k_mma_to_rho<<<nblocks(m), kBS, 0, c->stream>>>(m->n, m->x, L.eact, h->rho);
    });
}

extern "C" long long rt_mma_evaluations(rt_mma* m) { return m ? m->evaluations : -1; }
