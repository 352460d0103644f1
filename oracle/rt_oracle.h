/*
 * rt_oracle.h — FP64 CPU restatement of robtop's multigrid solver hot path.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline / reference arm may load this library; the
 * product path (robtop_b200/) never calls it.
 *
 * Parity status: the reference (lavenklau/robtop) cannot be compiled here (it
 * needs Eigen 3.4, CGAL, OpenVDB, gflags, ... which are absent) and ships no
 * golden vectors, so this restatement is pinned only by the reference's own
 * known-answer tests (rigid-body null space, optimization/optimization.cpp:697;
 * aggregated-compliance eigenvalue vs modified power method,
 * utils/test_utils.cpp:1249-1296; BitSAT rank self-test,
 * optimization/optimization.cu:231-280) and by numpy's SVD for the
 * coarsest-level pseudo-inverse (the reference uses Eigen BDCSVD::solve,
 * grid/Grid.cpp:1927,2013).  Element-wise numeric parity is "parity unpinned".
 *
 * Layout conventions (shared with the CUDA library so results compare 1:1):
 *   level element box nx*ny*nz, node box (nx+1)*(ny+1)*(nz+1), x fastest;
 *   node vectors are SoA [3][nv] doubles; element arrays [ne];
 *   assembled stencils are [27*9][nv] doubles, entry ((k*9 + 3*row + col)*nv + v)
 *   couples node v to its neighbour v + d(k), d(k) = (k%3-1, k/3%3-1, k/9-1).
 */
#ifndef RT_ORACLE_H
#define RT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nz;       /* element box of this level */
    int ratio;            /* 0 on the finest level, else coarsening ratio (2 or 4) from the next finer real level */
    const uint8_t* eact;  /* element active flags [ne] */
    const uint8_t* vact;  /* node active flags [nv] */
    const uint8_t* vfix;  /* finest level only: support (Dirichlet) node flags [nv], may be NULL */
    const double* w;      /* finest level only: element stiffness weights rho^p (0 for void) [ne] */
    double* st;           /* coarse levels only: Galerkin stencil [243][nv] */
    double* u;            /* [3][nv] */
    double* f;            /* [3][nv] */
    double* r;            /* [3][nv] */
    double* ainv;         /* coarsest level only: dense (pseudo-)inverse [3na][3na] */
    int* aidx;            /* coarsest level only: active-node index -> node id [na] */
    int na;               /* coarsest level only: number of active nodes */
    double lmax;          /* smoothed levels: largest eigenvalue estimate of D^-1 A (Chebyshev) */
    double* d;            /* smoothed levels: Chebyshev direction [3][nv] */
} or_level;

enum { OR_SMOOTH_GS = 0, OR_SMOOTH_SGS = 1, OR_SMOOTH_JACOBI = 2, OR_SMOOTH_CHEBY = 3 };

/* Chebyshev smoothing on [lmax/30, 1.1 lmax] (not in the reference) */
void or_cheby_coef(double lmax, int k, double* a, double* b);
void or_fine_cheby(const or_level* L, const double* KE, const double* u, const double* f, double* unew, double* d,
                   int k);
void or_st_cheby(const or_level* L, const double* u, const double* f, double* unew, double* d, int k);
double or_lambda_max(or_level* L, int is_fine, const double* KE, uint64_t seed, int iters, double* work /*[6][3nv]*/);

/* element template (element/templateMatrix.cpp:15-124) */
void or_template_matrix(double E, double nu, double h, double* KE /* [576] row-major */);

/* occupancy on the reference's cubic bit grid (grid/Grid.cu:2555-2632, grid/Grid.cpp:455-505) */
void or_cube_vbits(int R, const uint32_t* ebits, uint32_t* vbits);
void or_cube_coarsen(int Rf, const uint32_t* ef, uint32_t* ec);
long or_bits_total(long nwords, const uint32_t* bits);
void or_bitsat_rank(long nwords, const uint32_t* bits, long nq, const long* q, int* rank);
/* reference GS-colour ordering (grid/Grid.cu:548-623, grid/Grid.cpp:2045-2106) */
void or_gs_maps(int vreso, const uint32_t* vbits, int nv_act, int* vlexi2gs, int* gs_num, int* nv_gs);

/* dense-box hierarchy helpers */
void or_node_active(int nx, int ny, int nz, const uint8_t* eact, uint8_t* vact);
void or_coarsen_elements(int nx, int ny, int nz, int ratio, const uint8_t* ef, uint8_t* ec);
void or_surface_nodes(int nx, int ny, int nz, const uint8_t* eact, uint8_t* surf);
void or_penalty_weights(long ne, const uint8_t* eact, const float* rho, float p, double* w);

/* finest-level matrix-free operator (grid/Grid.cu:1450-1557, 2439-2517, 792-1066) */
void or_fine_applyK(const or_level* L, const double* KE, const double* u, double* out);
void or_fine_residual(const or_level* L, const double* KE, const double* u, const double* f, double* r);
void or_fine_gs(const or_level* L, const double* KE, double* u, const double* f, int backward);
void or_fine_jacobi(const or_level* L, const double* KE, double* u, const double* f, double omega, double* tmp);

/* assembled-stencil levels (grid/Grid.cu:678-790, 1350-1448) */
void or_st_applyA(const or_level* L, const double* u, double* out);
void or_st_residual(const or_level* L, const double* u, const double* f, double* r);
void or_st_gs(const or_level* L, double* u, const double* f, int backward);
void or_st_jacobi(const or_level* L, double* u, const double* f, double omega, double* tmp);

/* transfers (grid/Grid.cu:1680-1895) */
void or_restrict(const or_level* fine, const or_level* coarse, const double* rf, double* fc);
void or_prolong_add(const or_level* fine, const or_level* coarse, const double* uc, double* uf);

/* Galerkin coarse stencils (grid/Grid.cu:120-506) */
void or_galerkin_from_elements(const or_level* fine, or_level* coarse, const double* KE, int with_support);
void or_galerkin_from_stencil(const or_level* fine, or_level* coarse);

/* coarsest direct solve (grid/Grid.cpp:1884-2043): dense (pseudo-)inverse */
int or_coarsest_setup(or_level* L, int no_support);
void or_coarsest_solve(const or_level* L);

/* V-cycle (grid/Grid.cpp:1068-1113) and MG-preconditioned CG */
double or_vcycle(or_level* levels, int nlev, const double* KE, int smoother, int npre, int npost,
                 double omega, int precond_mode);
int or_pcg(or_level* levels, int nlev, const double* KE, int smoother, int npre, int npost, double omega,
           double* x, const double* b, double tol, int maxit, double* relres_out, double* work /*[6][3nv]*/);

/* reductions */
double or_dot(long n, const double* a, const double* b);

/* worst-case load machinery (optimization/projection.cpp:129-360, optimization/optimization.cpp:123-261) */
void or_rng_uniform(uint64_t seed, long n, double* out);
int or_rigid_basis(int nload, const double* pos, const double* normal, int constrain_dir, double* Rd /*[6][3nload]*/);
void or_force_project(long nv, int nload, const int* load_nodes, const double* normal, int constrain_dir,
                      int nrig, const double* Rd, double* f);
void or_rigid_nodes(const or_level* L, double* Ru /*[6][3nv]*/);
void or_displacement_project(long nv, const double* Ru, double* u);
double or_modified_pm(or_level* levels, int nlev, const double* KE, int nload, const int* load_nodes,
                      const double* normal, int constrain_dir, int nrig, const double* Rd,
                      const double* Ru /* NULL when the structure has supports */, uint64_t seed,
                      int maxit, int* iters_out, double* fs_old /*[3nload]*/);
int or_lanczos(or_level* levels, int nlev, const double* KE, int smoother, int npre, int npost, double omega,
               int nload, const int* load_nodes, const double* normal, int constrain_dir, int nrig,
               const double* Rd, uint64_t seed, int k, double inner_tol, int inner_maxit,
               double* lambda_out, double* ritz_f /*[3nv]*/, double* work /*[(k+1)*3nload + 10*3nv]*/);
double or_tridiag_max_eig(int k, const double* alpha, const double* beta);

/* sensitivity, filter and OC update (optimization/optimization.cu:44-226, grid/Grid.cu:2323-2437) */
void or_sensitivity(int nx, int ny, int nz, const uint8_t* eact, const float* rho, float p, const double* KE,
                    const double* u, float* sens);
void or_filter(int nx, int ny, int nz, const uint8_t* eact, float radius, const float* sens, float* out);
void or_oc_try(long ne, const uint8_t* eact, const uint8_t* eshell, const float* rho, const float* sens,
               float lambda, float step, float damp, float rhomin, float* out);
float or_oc_update(long ne, const uint8_t* eact, const uint8_t* eshell, float* rho, const float* sens,
                   float vgoal, float step, float damp, float rhomin, long n_count, int* iters_out, float* tmp);

#ifdef __cplusplus
}
#endif

/* solid mesh voxeliser (or_voxel.c) */
void or_voxel_box(const float* coords, long nvert, int prefer_reso, int* reso, float bmin[3], float bmax[3],
                  float unit[3]);
void or_voxelize_solid(const float* coords, const int* tris, long ntri, int reso, const float bmin[3],
                       const float unit[3], uint32_t* bits);
void or_word_reverse(long nwords, uint32_t* w);
#endif
