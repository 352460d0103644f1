// rt_coarsest.cu — coarsest-level direct solve on the device.
//
// The reference downloads the coarsest stencil, builds a dense matrix and
// factors it on the host with Eigen::BDCSVD (Grid::buildCoarsestSystem,
// grid/Grid.cpp:1884-1939), then does a D2H / svd.solve / H2D round trip every
// V-cycle (Grid::solve_fem_host, grid/Grid.cpp:1981-2043).  Here the dense
// matrix is assembled, inverted (Gauss-Jordan, one cooperative launch with a
// grid barrier per pivot) and applied (GEMV) without leaving the GPU.
// Without supports the matrix is singular with the rigid modes as null space;
// the minimum-norm solve of BDCSVD is reproduced as A^+ = (A + a R R^T)^-1 - R R^T / a.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "rt_internal.h"

namespace cg = cooperative_groups;

namespace {

__global__ void k_assemble_dense(int vx, int vy, int vz, long nv, int na, const int* __restrict__ aidx,
                                 const int* __restrict__ rowof, const double* __restrict__ st, double* __restrict__ A) {
    const int n = 3 * na;
    const long tot = (long)na * 27 * 9;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t / 243), q = (int)(t % 243), k = q / 9, rc = q % 9;
        const int v = aidx[i];
        const int x = v % vx, y = (v / vx) % vy, z = v / (vx * vy);
        const int jx = x + k % 3 - 1, jy = y + (k / 3) % 3 - 1, jz = z + k / 9 - 1;
        if (jx < 0 || jy < 0 || jz < 0 || jx >= vx || jy >= vy || jz >= vz) continue;
        const int j = rowof[jx + vx * (jy + vy * jz)];
        if (j < 0) continue;
        A[(long)(3 * i + rc / 3) * n + 3 * j + rc % 3] = st[(long)q * nv + v];
    }
}

__global__ void k_add_rrt(int n, int nr, const double* __restrict__ R, double alpha, double* __restrict__ A) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * n; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t / n), j = (int)(t % n);
        double s = 0;
        for (int a = 0; a < nr; a++) s += R[(long)a * n + i] * R[(long)a * n + j];
        A[t] += alpha * s;
    }
}

__global__ void k_trace(int n, const double* __restrict__ A, double* __restrict__ out) {
    __shared__ double sh[256];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += A[(long)i * n + i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0] / n;
}

// In-place Gauss-Jordan inversion of an SPD matrix (no pivoting needed).
// colbuf/rowbuf hold the pivot column and row of the current step; the
// threads that produce the next step's column/row write them during the
// update, so one grid barrier per step suffices.  status[0] != 0 reports a
// non-positive pivot.
__global__ void k_gauss_jordan(int n, double* __restrict__ A, double* __restrict__ colbuf,
                               double* __restrict__ rowbuf, int* __restrict__ status) {
    cg::grid_group grid = cg::this_grid();
    const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nth = (long)gridDim.x * blockDim.x;
    const long nn = (long)n * n;
    // step 0 buffers
    for (long i = tid; i < n; i += nth) {
        colbuf[i] = A[i * n + 0];
        rowbuf[i] = A[i];
    }
    grid.sync();
    for (int k = 0; k < n; k++) {
        const double* col = colbuf + (long)(k & 1) * n;
        const double* row = rowbuf + (long)(k & 1) * n;
        double* ncol = colbuf + (long)((k + 1) & 1) * n;
        double* nrow = rowbuf + (long)((k + 1) & 1) * n;
        const double pivot = row[k];
        if (!(pivot > 0)) {
            if (tid == 0) status[0] = k + 1;
            return;  // uniform across the grid: every thread read the same pivot
        }
        const double ip = 1.0 / pivot;
        for (long t = tid; t < nn; t += nth) {
            const int i = (int)(t / n), j = (int)(t % n);
            double v;
            if (i == k && j == k) v = ip;
            else if (i == k) v = row[j] * ip;
            else if (j == k) v = -col[i] * ip;
            else v = A[t] - col[i] * row[j] * ip;
            A[t] = v;
            if (j == k + 1) ncol[i] = v;
            if (i == k + 1) nrow[j] = v;
        }
        grid.sync();
    }
}

__global__ void k_sub_rrt(int n, int nr, const double* __restrict__ R, const double* __restrict__ alpha,
                          double* __restrict__ A) {
    const double ia = 1.0 / alpha[0];
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * n; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t / n), j = (int)(t % n);
        double s = 0;
        for (int a = 0; a < nr; a++) s += R[(long)a * n + i] * R[(long)a * n + j];
        A[t] -= s * ia;
    }
}

__global__ void k_add_rrt_dev(int n, int nr, const double* __restrict__ R, const double* __restrict__ alpha,
                              double* __restrict__ A) {
    const double a = alpha[0];
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < (long)n * n; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t / n), j = (int)(t % n);
        double s = 0;
        for (int q = 0; q < nr; q++) s += R[(long)q * n + i] * R[(long)q * n + j];
        A[t] += a * s;
    }
}

template <typename TI, typename TO>
__global__ void k_gather_active(int na, long nv, const int* __restrict__ aidx, const TI* __restrict__ f,
                                TO* __restrict__ d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
        const int v = aidx[i];
        d[3 * i] = (TO)f[v]; d[3 * i + 1] = (TO)f[nv + v]; d[3 * i + 2] = (TO)f[2 * nv + v];
    }
}

// u = Ainv d, one warp per row, scattered back to the node box (u zeroed first by the caller)
template <typename T, typename TU>
__global__ void k_gemv_scatter(int na, long nv, const int* __restrict__ aidx, const T* __restrict__ Ainv,
                               const T* __restrict__ d, TU* __restrict__ u) {
    const int n = 3 * na;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < n; i += nwarps) {
        T s = 0;
        const T* row = Ainv + (long)i * n;
        for (int j = lane; j < n; j += 32) s += row[j] * d[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) u[(long)(i % 3) * nv + aidx[i / 3]] = (TU)s;
    }
}

}  // namespace

namespace rtk {

int coarsest_setup(rt_hier* h) {
    rt_ctx* c = h->ctx;
    rt_level& L = h->L.back();
    const int na = L.na, n = 3 * na;
    if (na == 0) return rt_fail(c, RT_ESTATE, "coarsest level has no active node");
    // rowof on device (node -> active index)
    std::vector<int> aidx_h(na), rowof_h(L.nv, -1);
    RT_CUDA(c, cudaMemcpyAsync(aidx_h.data(), L.aidx, sizeof(int) * na, cudaMemcpyDeviceToHost, c->stream));
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int i = 0; i < na; i++) rowof_h[aidx_h[i]] = i;
    int* rowof = nullptr;
    double *colbuf = nullptr, *rowbuf = nullptr, *R = nullptr;
    int* status = nullptr;
    RT_CUDA(c, cudaMallocAsync(&rowof, sizeof(int) * L.nv, c->stream));
    RT_CUDA(c, cudaMallocAsync(&colbuf, sizeof(double) * 2 * n, c->stream));
    RT_CUDA(c, cudaMallocAsync(&rowbuf, sizeof(double) * 2 * n, c->stream));
    RT_CUDA(c, cudaMallocAsync(&status, sizeof(int), c->stream));
    RT_CUDA(c, cudaMemcpyAsync(rowof, rowof_h.data(), sizeof(int) * L.nv, cudaMemcpyHostToDevice, c->stream));
    RT_CUDA(c, cudaMemsetAsync(status, 0, sizeof(int), c->stream));
    RT_CUDA(c, cudaMemsetAsync(L.ainv, 0, sizeof(double) * (size_t)n * n, c->stream));
    RT_CHECK(rt_launch(c, "coarsest_assemble", [&] {
        long tot = (long)na * 243;
        unsigned g = (unsigned)std::min<long>((tot + 255) / 256, (long)c->sm_count * 8);
        k_assemble_dense<<<g, 256, 0, c->stream>>>(L.vx, L.vy, L.vz, L.nv, na, L.aidx, rowof, L.st, L.ainv);
    }));
    const bool no_support = (h->P.mode == RT_MODE_NSCF || h->P.mode == RT_MODE_NSFF);
    unsigned gnn = (unsigned)std::min<long>(((long)n * n + 255) / 256, (long)c->sm_count * 8);
    if (no_support) {
        // orthonormal rigid modes at the coarsest active nodes (positions are static)
        std::vector<double> Rh((size_t)6 * n, 0.0);
        for (int i = 0; i < na; i++) {
            int v = aidx_h[i];
            double p[3] = {(double)(v % L.vx), (double)((v / L.vx) % L.vy), (double)(v / (L.vx * L.vy))};
            double ph[3][3] = {{0, -p[2], p[1]}, {p[2], 0, -p[0]}, {-p[1], p[0], 0}};
            for (int t = 0; t < 3; t++) Rh[(size_t)t * n + 3 * i + t] = 1.0;
            for (int k = 0; k < 3; k++)
                for (int t = 0; t < 3; t++) Rh[(size_t)(3 + k) * n + 3 * i + t] = ph[t][k];
        }
        for (int a = 0; a < 6; a++) {
            for (int b = 0; b < a; b++) {
                double d = 0;
                for (int q = 0; q < n; q++) d += Rh[(size_t)a * n + q] * Rh[(size_t)b * n + q];
                for (int q = 0; q < n; q++) Rh[(size_t)a * n + q] -= d * Rh[(size_t)b * n + q];
            }
            double nn = 0;
            for (int q = 0; q < n; q++) nn += Rh[(size_t)a * n + q] * Rh[(size_t)a * n + q];
            nn = std::sqrt(nn);
            for (int q = 0; q < n; q++) Rh[(size_t)a * n + q] /= nn;
        }
        RT_CUDA(c, cudaMallocAsync(&R, sizeof(double) * 6 * n, c->stream));
        RT_CUDA(c, cudaMemcpyAsync(R, Rh.data(), sizeof(double) * 6 * n, cudaMemcpyHostToDevice, c->stream));
        RT_CHECK(rt_launch(c, "coarsest_trace", [&] { k_trace<<<1, 256, 0, c->stream>>>(n, L.ainv, h->scal + 60); }));
        RT_CHECK(rt_launch(c, "coarsest_add_rrt",
                           [&] { k_add_rrt_dev<<<gnn, 256, 0, c->stream>>>(n, 6, R, h->scal + 60, L.ainv); }));
    }
    // cooperative Gauss-Jordan
    int dev = c->device, nb_per_sm = 0;
    RT_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb_per_sm, k_gauss_jordan, 256, 0));
    int coop = 0;
    RT_CUDA(c, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop || nb_per_sm < 1) return rt_fail(c, RT_ECUDA, "cooperative launch unavailable");
    unsigned gblocks = (unsigned)std::min<long>((long)c->sm_count * std::min(nb_per_sm, 2), ((long)n * n + 255) / 256);
    if (gblocks < 1) gblocks = 1;
    double* Aptr = L.ainv;
    int nn_ = n;
    void* args[] = {&nn_, &Aptr, &colbuf, &rowbuf, &status};
    RT_CHECK(rt_launch(c, "coarsest_gauss_jordan", [&] {
        cudaLaunchCooperativeKernel((void*)k_gauss_jordan, gblocks, 256, args, 0, c->stream);
    }));
    if (no_support) {
        RT_CHECK(rt_launch(c, "coarsest_sub_rrt",
                           [&] { k_sub_rrt<<<gnn, 256, 0, c->stream>>>(n, 6, R, h->scal + 60, L.ainv); }));
        RT_CUDA(c, cudaFreeAsync(R, c->stream));
    }
    int st_h = 0;
    RT_CUDA(c, cudaMemcpyAsync(&st_h, status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    RT_CUDA(c, cudaFreeAsync(rowof, c->stream));
    RT_CUDA(c, cudaFreeAsync(colbuf, c->stream));
    RT_CUDA(c, cudaFreeAsync(rowbuf, c->stream));
    RT_CUDA(c, cudaFreeAsync(status, c->stream));
    RT_CUDA(c, cudaStreamSynchronize(c->stream));
    if (st_h != 0) return rt_fail(c, RT_ENAN, "coarsest matrix not positive definite (pivot %d)", st_h - 1);
    return RT_OK;
}

// u = A^-1 f on the coarsest level.  The inverse and the product are FP64 in both precisions
// of the V-cycle: the coarse operator's conditioning (the stiffness contrast survives the
// averaging) would amplify the rounding of an FP32 copy of the inverse.
template <typename T>
int coarsest_solve(rt_hier* h, const T* f, T* u) {
    rt_ctx* c = h->ctx;
    rt_level& L = h->L.back();
    RT_CHECK(rt_launch(c, sizeof(T) == 8 ? "coarsest_gather_f64" : "coarsest_gather_f32", [&] {
        k_gather_active<T, double><<<(L.na + 255) / 256, 256, 0, c->stream>>>(L.na, L.nv, L.aidx, f, L.dvec);
    }));
    RT_CUDA(c, cudaMemsetAsync(u, 0, sizeof(T) * 3 * L.nv, c->stream));
    const int n = 3 * L.na;
    return rt_launch(c, sizeof(T) == 8 ? "coarsest_gemv_f64" : "coarsest_gemv_f32", [&] {
        unsigned g = (unsigned)std::min<long>(((long)n * 32 + 255) / 256, (long)c->sm_count * 8);
        k_gemv_scatter<double, T><<<g, 256, 0, c->stream>>>(L.na, L.nv, L.aidx, L.ainv, L.dvec, u);
    });
}

template int coarsest_solve<double>(rt_hier*, const double*, double*);
template int coarsest_solve<float>(rt_hier*, const float*, float*);

}  // namespace rtk
