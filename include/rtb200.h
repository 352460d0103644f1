/*
 * rtb200.h — C ABI of the B200-native (sm_100a) robtop solver hot path.
 *
 * The library replaces the GPU solver of lavenklau/robtop: the matrix-free
 * geometric multigrid for SIMP-penalised hex8 elasticity on a voxel grid
 * (grid/Grid.{h,cpp,cu}), the worst-case-load eigen-solve
 * (optimization/optimization.cpp:123-261, optimization/projection.*), and the
 * sensitivity / filter / OC density update (optimization/optimization.cu).
 *
 * Conventions
 *  - Every entry point returns an int status (RT_OK on success); the text of
 *    the last failure is available from rt_last_error(ctx).  The reference
 *    printed and continued (culib/cudaCommon.cuh:6-11) or called exit(-1)
 *    (optimization/optimization.cpp:81,234,254); this ABI never exits.
 *  - Pointers are plain host pointers unless the argument name ends in _dev.
 *  - "Dense" node vectors are SoA [3][nv] with nv = (nx+1)(ny+1)(nz+1), x
 *    fastest; element arrays are [ne] = nx*ny*nz, x fastest.  Level 0 is the
 *    finest grid.  RT_LAYOUT_REF_GS selects the reference's Gauss-Seidel
 *    colour-ordered, 32-padded layout (grid/Grid.cpp:2045-2106) instead.
 *  - A context owns one CUDA stream (or borrows the caller's); every call is
 *    ordered on it.  The context's own stream is non-blocking: a caller that writes
 *    an input _dev array on another stream, or reads an output one there, orders
 *    that work with the context's stream first (or passes its own stream at
 *    rt_ctx_create).  Contexts and hierarchies are independent of each other
 *    (the reference rebinds global __constant__ tables per level,
 *    grid/Grid.cu:48-75, and is not reentrant).
 */
#ifndef RTB200_H
#define RTB200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum rt_status {
    RT_OK = 0,
    RT_EINVAL = 1,    /* bad argument */
    RT_ECUDA = 2,     /* CUDA runtime error */
    RT_ENOCONV = 3,   /* iteration cap reached before the tolerance */
    RT_ENAN = 4,      /* NaN/Inf met in a solve */
    RT_ETIMEOUT = 5,  /* a bounded device wait gave up */
    RT_ENOMEM = 6,    /* device allocation failed */
    RT_ESTATE = 7     /* call out of order (e.g. solve before update_stencil) */
};

/* robtop's work modes, same order as grid::Mode (grid/Grid.h:139-144) */
enum rt_mode {
    RT_MODE_NSCF = 0, /* no support, load direction constrained to the surface normal */
    RT_MODE_NSFF = 1, /* no support, free load direction */
    RT_MODE_WSCF = 2, /* with support, constrained direction */
    RT_MODE_WSFF = 3  /* with support, free direction */
};

/* GS: the reference's 8-colour point-block Gauss-Seidel (forward in pre and post
 * smoothing, grid/Grid.cu:1068-1111); SGS: forward pre, backward post (symmetric
 * V-cycle); JACOBI: damped point-block Jacobi; CHEBY: Chebyshev polynomial in
 * D^-1 A of degree pre/post_sweeps on [lmax/30, 1.1 lmax], lmax estimated per
 * level by rt_update_stencil (one fused element-tile / stencil kernel per step). */
enum rt_smoother { RT_SMOOTH_GS = 0, RT_SMOOTH_SGS = 1, RT_SMOOTH_JACOBI = 2, RT_SMOOTH_CHEBY = 3 };
/* RT_FP64_FINE: the finest level's smoothing and residual in FP64, every coarser level in FP32 */
enum rt_precision { RT_FP64 = 0, RT_FP32 = 1, RT_FP64_FINE = 2 };
enum rt_layout { RT_LAYOUT_DENSE = 0, RT_LAYOUT_REF_GS = 1 };
enum rt_field { RT_FIELD_U = 0, RT_FIELD_F = 1, RT_FIELD_R = 2, RT_FIELD_RHO = 3, RT_FIELD_SENS = 4,
                RT_FIELD_STENCIL = 5, RT_FIELD_VACT = 6, RT_FIELD_EACT = 7, RT_FIELD_VFIX = 8,
                RT_FIELD_PENALTY = 9 /* level-0 element weights powf(rho, p), FP32, refreshed by rt_update_stencil */ };
enum rt_worst_method { RT_WORST_MODPM = 0, RT_WORST_LANCZOS = 1, RT_WORST_BLOCK_LANCZOS = 2 };

/* Parameter block: optimization/optimization.h:11-22 plus the solver knobs the
 * reference hard-codes (GS 1/1 sweeps, optimization/optimization.cpp:169). */
typedef struct rt_params {
    float power_penalty;    /* SIMP exponent p */
    float min_rho;          /* rho_min */
    float volume_ratio;     /* volume target */
    float design_step;      /* OC move limit */
    float damp_ratio;       /* OC damping exponent eta */
    float filter_radius;    /* sensitivity filter radius (the reference stores an int) */
    double youngs_modulus;  /* E */
    double poisson_ratio;   /* nu */
    double element_length;  /* h */
    int mode;               /* rt_mode */
    int skip_layer1;        /* 1: first coarse level is 4x coarser (the reference always sets this) */
    int smoother;           /* rt_smoother used by rt_pcg's V-cycle preconditioner */
    int pre_sweeps, post_sweeps;
    double jacobi_omega;
    int precision;          /* rt_precision of the V-cycle inside rt_pcg / rt_worst_case */
    int coarsest_elements;  /* halve while more elements than this are solid (the reference: 400,
                               grid/Grid.cpp:488); the coarsest level is solved densely (<= 12288 DOF) */
    int cycle_gamma;        /* coarse corrections per visit of levels >= 1: 1 V-cycle (the reference), 2 W */
    int coarse_sweeps;      /* smoothing steps on levels >= 1 (0: pre_sweeps / post_sweeps as on the finest) */
    int precision_fallback; /* N > 0: a PCG solve whose FP32 / FP64_FINE V-cycles stop reducing |r| (no halving
                               within N iterations; default 100) continues from its iterate with FP64 V-cycles;
                               0: off */
    int coarse_bf16;        /* 1: the FP32 smoother on levels >= 1 reads the stencils stored in BF16 (half the
                               bytes of the FP32 copy); residuals, restriction and the coarsest solve keep FP32 /
                               FP64 stencils.  0 (default): FP32 stencils */
    int krylov_fp32;        /* k = 1..4 (with precision RT_FP32, supported modes, no learned correction): the CG
                               vectors and the operator product of rt_pcg are FP32 too (dot products summed in
                               FP64); each inner solve of K d = r / |r| (to the outer target, at most down to
                               10^-(3+k)) is followed by x += |r| d and a fresh FP64 residual (iterative
                               refinement).  0 (default): FP64 flexible CG around the FP32 V-cycle */
    int cycle_gamma_levels; /* with cycle_gamma > 1: the coarse correction repeats on levels 1 .. this level
                               only (coarser levels are visited V-cycle fashion); 0 (default): on every level */
} rt_params;

typedef struct rt_solve_info {
    int iterations;         /* outer iterations (CG steps, power steps, Lanczos steps) */
    int inner_iterations;   /* CG steps inside Lanczos / refinement */
    int vcycles;            /* V-cycles applied */
    int status;             /* rt_status of the solve */
    double rel_residual;    /* final ||f - K u|| / ||f|| (FP64) */
    double value;           /* compliance f.u or the eigenvalue */
    double seconds;         /* device time of the call */
} rt_solve_info;

typedef struct rt_level_info {
    int nx, ny, nz;         /* element box of the level */
    int ratio;              /* 0 on level 0, else coarsening ratio to the next finer level */
    long long n_nodes;      /* nodes in the box */
    long long n_active_nodes;
    long long n_active_elements;
} rt_level_info;

typedef struct rt_ctx rt_ctx;
typedef struct rt_hier rt_hier;
typedef struct rt_unet rt_unet;
typedef struct rt_mma rt_mma;

/* ---- context ------------------------------------------------------------ */
int rt_ctx_create(int device, void* cuda_stream /* NULL: own stream */, rt_ctx** out);
/* releases the caller's handle (call once); hierarchies, workspaces and networks made on the
 * context keep it alive until they are destroyed, in any order */
void rt_ctx_destroy(rt_ctx* ctx);
const char* rt_last_error(rt_ctx* ctx);
int rt_ctx_sync(rt_ctx* ctx);
/* polls a device-side wait on other blocks may spend before it gives up (the grid barrier of the
 * fused Chebyshev sweeps; default 1 << 22, polls < 0 restores it, 0 gives up at the first poll).  No reference counterpart: a
 * test lowers it so that a wait runs out and the call reports RT_ECUDA with the reason, leaving
 * the context usable. */
int rt_ctx_set_wait_limit(rt_ctx* ctx, long long polls);
void rt_params_default(rt_params* p);
/* per-kernel device-time accounting (CUDA events around each launch) */
int rt_profile_enable(rt_ctx* ctx, int on);
int rt_profile_query(rt_ctx* ctx, int idx, char* name, int name_len, long long* launches, double* ms);
int rt_profile_reset(rt_ctx* ctx);
/* number of kernels this context has launched since creation */
long long rt_launch_count(rt_ctx* ctx);

/* ---- hierarchy ------------------------------------------------------------
 * replaces HierarchyGrid::genFromMesh(solid_bit, out_reso) (grid/Grid.cpp:455-712)
 * and Grid::build (grid/Grid.cpp:1513-1677).  The coarsening stops when at
 * most 400 elements are solid (grid/Grid.cpp:488). */
int rt_hier_create(rt_ctx* ctx, const rt_params* p, int nx, int ny, int nz, const uint8_t* eact, rt_hier** out);
/* solid_bits: cubic reso^3 bit grid, bit x + y*reso + z*reso^2, LSB-first words
 * (the bit layout genFromMesh(solid_bit, out_reso) takes) */
int rt_hier_create_from_bits(rt_ctx* ctx, const rt_params* p, int reso, const uint32_t* solid_bits, rt_hier** out);
void rt_hier_destroy(rt_hier* h);
int rt_hier_n_levels(rt_hier* h);
int rt_hier_level_info(rt_hier* h, int level, rt_level_info* out);
int rt_hier_set_params(rt_hier* h, const rt_params* p);
int rt_hier_get_params(rt_hier* h, rt_params* p);
/* element template (element/templateMatrix.cpp:31-124), 24x24 row-major */
int rt_template_matrix(rt_hier* h, double* KE);

/* occupancy hierarchy on the reference's cubic bit grid, on the device
 * (cubeGridSetSolidVertices_g, setSolidElementFromFineGrid_g: grid/Grid.cu:2555-2648) */
int rt_cube_vertex_bits(rt_ctx* ctx, int reso, const uint32_t* ebits, uint32_t* vbits);
int rt_cube_coarsen_bits(rt_ctx* ctx, int reso, const uint32_t* ebits_fine, uint32_t* ebits_coarse);

/* ---- mesh voxeliser ------------------------------------------------------- */
/* cube resolution the voxeliser uses for prefer_reso: the first power of two above it
 * (padd2SatifyResolution, voxelizer/voxelize_main.cpp:312-340); 0 if prefer_reso is
 * outside [1, 1023] */
int rt_voxel_resolution(int prefer_reso);
/* solid voxelisation of a closed triangle mesh (voxelize_mesh,
 * voxelizer/voxelize_main.cpp:344-402; the solid kernel voxelizer/voxelize_solid.cu:80-150).
 * vcoords [3 nvert] and tri_ids [3 ntri] are host arrays; every vertex index must lie in
 * [0, nvert).  solid_bits (host, capacity_words >= R^3 / 32 with R = rt_voxel_resolution)
 * receives bit x + y R + z R^2 of the padded cube, most significant bit first in each word
 * as the reference's voxeliser writes it; out_reso = (R, R, R), out_box = (min xyz, max xyz) */
int rt_voxelize_mesh(rt_ctx* ctx, const float* vcoords, long nvert, const int* tri_ids, long ntri, int prefer_reso,
                     uint32_t* solid_bits, long capacity_words, int out_reso[3], float out_box[6]);
/* HierarchyGrid::genFromMesh(pcoords, facevertices) (grid/Grid.cpp:184-205): voxelise, reverse
 * the words to least significant bit first, build the hierarchy (rt_hier_create_from_bits).
 * The reference's AABB tree of the surface (used for shell elements and normals) is not built. */
int rt_hier_create_from_mesh(rt_ctx* ctx, const rt_params* p, const float* vcoords, long nvert, const int* tri_ids,
                             long ntri, int prefer_reso, rt_hier** out);
/* device time of one voxelisation (event and row passes, mesh already on the device) */
int rt_bench_voxelize(rt_ctx* ctx, const float* vcoords, long nvert, const int* tri_ids, long ntri, int prefer_reso,
                      int reps, double* us_per_call);

/* ---- boundary conditions ------------------------------------------------- */
/* shell elements: eshell[ne] (dense level-0 element order) flags elements whose density the OC
 * update holds at 1 (the reference marks those within shell_width elements of the mesh surface,
 * HierarchyGrid::setSolidShellElement, grid/Grid.cpp:67-137); eshell = NULL clears them */
int rt_set_shell(rt_hier* h, const uint8_t* eshell);
/* surface nodes of level 0 (mark_surface_nodes_kernel, grid/Grid.cu:2005-2039), dense node order */
int rt_surface_nodes(rt_hier* h, uint8_t* surf);
/* support flags on level-0 nodes (Grid::computeProjectionMatrix, grid/Grid.cpp:1291-1403) */
int rt_set_support(rt_hier* h, const uint8_t* vfix);
/* load set: dense level-0 node ids with their outward unit normals [3*nload]
 * (setLoadNodes, optimization/projection.cpp:129-269) */
int rt_set_load_nodes(rt_hier* h, int nload, const int* nodes, const double* normals);

/* ---- fields ---------------------------------------------------------------
 * level-0 density: replaces Grid::init_rho / direct writes into getRho() */
int rt_init_density(rt_hier* h, float rho);
int rt_put(rt_hier* h, int field, int level, int layout, const void* src);
int rt_get(rt_hier* h, int field, int level, int layout, void* dst);
int rt_put_dev(rt_hier* h, int field, int level, const void* src_dev);
int rt_get_dev(rt_hier* h, int field, int level, void* dst_dev);
/* reference GS-order map of a level: vidmap[dense node] = GS slot or -1, and the GS slot count */
int rt_ref_gs_map(rt_hier* h, int level, int* vidmap, int* n_gs, int* gs_num /*[8]*/);

/* ---- multigrid operators (grid/Grid.cu) ----------------------------------- */
/* Galerkin coarse stencils + coarsest factorisation: HierarchyGrid::update_stencil (grid/Grid.cpp:2108-2119) */
int rt_update_stencil(rt_hier* h);
/* largest eigenvalue estimate of D^-1 A on a smoothed level (set by rt_update_stencil);
 * no counterpart in the reference (its GS smoother needs none) */
int rt_smoother_lmax(rt_hier* h, int level, double* lmax);
/* Grid::update_residual (grid/Grid.cu:1644-1678): r = f - K u on a level */
int rt_update_residual(rt_hier* h, int level);
/* Grid::gs_relax (grid/Grid.cu:1068-1111) and the other smoothers */
int rt_smooth(rt_hier* h, int level, int smoother, int sweeps, double omega);
/* Grid::restrict_residual (grid/Grid.cu:1796-1816): f[level] = P^T r[level-1] */
int rt_restrict_residual(rt_hier* h, int level);
/* Grid::prolongate_correction (grid/Grid.cu:1898-1915): u[level] += P u[level+1] */
int rt_prolongate_correction(rt_hier* h, int level);
/* Grid::solve_fem_host (grid/Grid.cpp:1981-2043), on the device: u = A^+ f on the coarsest level */
int rt_coarsest_solve(rt_hier* h);
/* HierarchyGrid::v_cycle (grid/Grid.cpp:1068-1113) on level-0 u/f; returns ||r||/||f|| */
int rt_vcycle(rt_hier* h, int pre, int post, double* rel_res);
/* Grid::applyK (grid/Grid.cu:2519-2532): out = K(rho) u on level 0, dense device vectors */
int rt_apply_K_dev(rt_hier* h, const double* u_dev, double* out_dev);
int rt_apply_K(rt_hier* h, const double* u, double* out);
/* Grid::compliance (grid/Grid.cpp:1976-1979): f.u on level 0 */
int rt_compliance(rt_hier* h, double* c);
/* forceProject (optimization/projection.cu:165-231, projection.cpp:289-360): f_dev (dense [3][nv]
 * device vector) <- P f: the load-node values projected onto the admissible loads of the work mode
 * (wsff: unchanged; *scf: normal component only; ns*: minus the rigid-mode components), every other
 * node set to zero */
int rt_force_project(rt_hier* h, double* f_dev);
/* getForceSupport (optimization/projection.cu:307-338): fs_dev [3][nload] (one array per component,
 * load nodes in increasing dense id) <- the load-node values of f_dev */
int rt_get_force_support(rt_hier* h, const double* f_dev, double* fs_dev);
/* setForceSupport (optimization/projection.cu:340-369): f_dev <- 0, then the load nodes <- fs_dev */
int rt_set_force_support(rt_hier* h, const double* fs_dev, double* f_dev);
/* displacementProject (optimization/projection.cpp:374-392): u_dev minus its components along the
 * orthonormalised rigid modes of the active nodes (no-support modes; a no-op with supports) */
int rt_displacement_project(rt_hier* h, double* u_dev);
/* getLoadNodes (optimization/projection.cpp:129-143): *n = number of load nodes; nodes (host,
 * may be null) <- their dense level-0 node ids in increasing order */
int rt_load_nodes(rt_hier* h, int* n, int* nodes);
/* Grid::elementCompliance (grid/Grid.cu:3434-3480): ce_dev[ne] (dense element order, device)
 * <- rho_e^p u_e.KE u_e for u_dev (dense [3][nv] device vector); 0 on inactive elements */
int rt_element_compliance(rt_hier* h, const double* u_dev, float* ce_dev);
/* Grid::relative_residual (grid/Grid.cu:1946-1951) */
int rt_relative_residual(rt_hier* h, double* rel);
/* Compliance f.u of two caller-owned FP64 device vectors of length n, written to
 * out_dev[0], without allocating any device memory: for callers that cannot call
 * cudaMalloc (all device memory handed to their own pool, or no allocation
 * allowed once their solve loop runs).  No counterpart in the reference.
 * The scratch is a fixed 512 KiB device array inside the library (held by every
 * GPU that loads it until exit); n must not exceed RT_NOALLOC_MAX_N, larger n is
 * rejected with RT_EINVAL and a message on stderr.  The array's address is looked
 * up on the first call per device (make that call before any stream capture).
 * All calls share the array: calls that overlap on the GPU race.  Runs on
 * cuda_stream (NULL: the legacy default stream) of the current device.  The
 * address is cached with the id of the context it belongs to and looked up again
 * when the current context changes (e.g. after cudaDeviceReset).  An error
 * already pending on the calling thread is reported as RT_ECUDA, not cleared. */
#define RT_NOALLOC_MAX_PARTIALS 65536
#define RT_NOALLOC_MAX_N (65536LL * 4096LL)
int rt_compliance_noalloc(const double* f_dev, const double* u_dev, long long n, double* out_dev,
                          void* cuda_stream);

/* Launch-shape autotuner (no counterpart in the reference): times every
 * finest-level kernel (residual, applyK, Jacobi, Chebyshev; FP32 and FP64) over
 * candidate tile shapes with CUDA events on the context stream and keeps the
 * fastest.  reps: timed launches per candidate (<= 0: 5). */
int rt_autotune(rt_hier* h, int reps);
/* chosen shape of a finest-level kernel; mode 0 residual, 1 applyK, 2 Jacobi, 3 Chebyshev;
 * variant 0 shared-memory element tile (ty 2, 4 or 8 node rows), 1 register-marching element kernel, 2 register marching with
 * each layer's output-stage loads issued before its element arithmetic, 3 shared-memory element tile software-pipelined
 * over z (element layer z+1 and node layer z share one barrier interval; ty 2, 4 or 8), 4 (FP32) variant 3 with
 * two elements per thread in packed FP32, 5 sum-factorised row marching (the element grid's Hadamard stages shared between
 * neighbouring elements, one warp per node row, one barrier per layer; ty 4, 8 or 16 node rows) */
int rt_tuning_info(rt_hier* h, int precision, int mode, int* variant, int* ty, int* zchunk, double* us);
/* set a finest-level kernel's launch shape explicitly (ty: 2, 4 or 8 rows for variants 0, 1, 3, 4; 2 or 4 for
 * variant 2; 4, 8 or 16 for variant 5) */
int rt_set_tuning(rt_hier* h, int precision, int mode, int variant, int ty, int zchunk);
/* time reps launches of one finest-level kernel at its current shape on random data
 * (device time per launch in microseconds, CUDA events on the context stream) */
int rt_bench_fine_kernel(rt_hier* h, int precision, int mode, int reps, double* us_per_launch);
/* sweeps steps of the FP32 smoother (RT_SMOOTH_JACOBI or RT_SMOOTH_CHEBY) on level lvl (0 .. coarsest-1):
 * the level's u, f rounded to FP32, smoothed with the kernels the mixed-precision V-cycle uses, u
 * widened back.  Same smoothing rule as rt_smooth (grid/Grid.cu:1068-1111 for the reference's GS). */
int rt_smooth_f32(rt_hier* h, int lvl, int smoother, int sweeps, double omega);
/* FP32 Chebyshev smoothing of stencil level lvl (1 .. coarsest-1) as one cooperative launch per
 * smoothing (the steps separated by a bounded grid barrier) instead of one launch per step.
 * on: 0 off, 1 on (the resident form when the level's nodes fit on the device at once, else the
 * streaming form), 2 on with the streaming form at any size.
 * Off by default.  rt_autotune times both forms on sets of 8 steps, captured as graphs, and
 * reports the times here without switching: alone the fused sets are faster, but inside the
 * solver's conditional-loop graphs whole solves measured slower with them.  Batched solves always
 * use separate launches (their instances run concurrently). */
int rt_set_level_fused(rt_hier* h, int lvl, int on);
int rt_level_fused_info(rt_hier* h, int lvl, int* on, double* us_separate, double* us_fused);
/* SIMT arithmetic peak of the context's device in TFLOP/s, from a project microbenchmark (16
 * independent FMA chains per thread, 8 blocks of 256 threads per SM, best of reps launches after one
 * warm-up): kind 0 FP32 FFMA, 1 FP32 packed FFMA2, 2 FP64 DFMA.  The matrix-free finest-level
 * operator is bound by this issue rate rather than by HBM.  No reference counterpart (measurement). */
int rt_bench_simt_peak(rt_ctx* c, int kind, int reps, double* tflops);
/* run one FP32 finest-level kernel at its current shape on level 0's vectors (u, f rounded to FP32)
 * and widen its result into level 0's residual vector: mode 0 f - K u, 1 K u, 2 a Jacobi step
 * u + omega D^-1 (f - K u), 3 the first Chebyshev step (needs rt_update_stencil) */
int rt_fine_kernel_f32(rt_hier* h, int mode, double omega);
/* the same for one stencil level lvl (1 .. coarsest-1): mode 0 residual, 2 Jacobi, 3 Chebyshev step;
 * precision RT_FP64 or RT_FP32 (FP32 smoothing reads the BF16 stencils when rt_params.coarse_bf16 is set).
 * Overwrites the level's vectors; needs rt_update_stencil. */
int rt_bench_level_kernel(rt_hier* h, int lvl, int precision, int mode, int reps, double* us_per_launch);
/* the kernel variant of the FP32 smoother's stencil levels, per stencil copy (stencil_type 0 FP32,
 * 1 BF16): 0 lane-split (4 lanes per node), 1 bulk-copy (each 32-node stencil run staged in shared
 * memory by cp.async.bulk).  rt_autotune times both on level 1 (after rt_update_stencil) and keeps
 * the faster; us_*: its measured Chebyshev-step times (0 before it ran). */
int rt_level_kernel_info(rt_hier* h, int stencil_type, int* variant, double* us_lane_split, double* us_bulk);
int rt_set_level_kernel(rt_hier* h, int stencil_type, int variant);

/* ---- solvers -------------------------------------------------------------- */
/* MG-preconditioned CG on level 0: u <- K^-1 f to ||r||/||f|| <= tol (solveFEM's role,
 * optimization/optimization.cpp:85-91).  Uses the precision/smoother in the params. */
int rt_pcg(rt_hier* h, double tol, int maxit, rt_solve_info* info);
/* number of solves on h (PCG, Lanczos inner solves, batched instances) that switched to FP64
 * V-cycles after stalling (rt_params.precision_fallback); no reference counterpart */
long long rt_hier_precision_fallbacks(rt_hier* h);
/* worst-case load: largest eigenvalue of P K^-1 P on the load set.
 * RT_WORST_MODPM restates modifiedPM (optimization/optimization.cpp:123-261);
 * RT_WORST_LANCZOS runs k Lanczos steps with PCG inner solves to inner_tol.
 * On return level-0 f holds the worst-case load and u = K^-1 f. */
int rt_worst_case(rt_hier* h, int method, int k, double inner_tol, uint64_t seed, double* lambda,
                  rt_solve_info* info);
/* RT_WORST_BLOCK_LANCZOS (rt_worst_case with k = Krylov dimension, block size 8) or this call:
 * block Lanczos with block_size starting loads and n_blocks block steps; each step's
 * block_size inner MG-PCG solves run concurrently as one batched CUDA graph (rt_pcg_batch)
 * on solve workspaces the hierarchy keeps.  Replaces the same role as rt_worst_case
 * (modifiedPM, optimization/optimization.cpp:123-261); no reference counterpart for the block form. */
int rt_worst_case_block(rt_hier* h, int block_size, int n_blocks, double inner_tol, uint64_t seed,
                        double* lambda, rt_solve_info* info);

/* ---- independent solves in one launch ------------------------------------- */
/* A solve workspace of `parent`: its own u/f/r and solver vectors on every level, the
 * parent's operator (densities, supports, stencils, coarsest inverse, launch shapes).
 * It accepts rt_put/rt_get of U, F, R, the level operators, rt_vcycle, rt_pcg and
 * rt_pcg_batch; calls that change the operator return RT_ESTATE.  Destroy it (with
 * rt_hier_destroy) before its parent.  No reference counterpart: the reference keeps one
 * global hierarchy (optimization/optimization.cpp:10). */
int rt_hier_workspace_create(rt_hier* parent, rt_hier** out);
/* rt_pcg on n hierarchies or workspaces of one context in ONE graph launch: every
 * instance's set-up and its WHILE-conditional PCG loop are independent branches of a
 * captured CUDA graph (cached per instance set), so the GPU runs them concurrently.
 * infos[i] as rt_pcg's; seconds is the whole batch. */
int rt_pcg_batch(rt_hier* const* hs, int n, double tol, int maxit, rt_solve_info* infos);

/* ---- optimisation step (optimization/optimization.cu) --------------------- */
/* computeSensitivity (optimization/optimization.cu:109-133) including the filter */
int rt_sensitivity(rt_hier* h, int filter);
/* Grid::filterSensitivity (grid/Grid.cu:2411-2437) alone */
int rt_filter_sensitivity(rt_hier* h, float radius);
/* updateDensities (optimization/optimization.cu:164-226); returns the multiplier */
int rt_oc_update(rt_hier* h, float vgoal, float* lambda_out, int* trials_out);
/* one OC iteration of optimization() (optimization/optimization.cpp:611-656):
 * update_stencil, worst-case solve, sensitivity+filter, OC update */
int rt_oc_iteration(rt_hier* h, int method, int k, double inner_tol, uint64_t seed, float vgoal,
                    double* compliance_out);

/* ---- method of moving asymptotes, one inequality constraint (optimization/mma_t.h:159-273) ---- */
/* mma_t(n, 1) + init(lower, upper) (optimization/mma_t.h:208-221, mma_t.cu:790-824): n design
 * variables with bounds xmin / xmax (host arrays), or, when both pointers are null, the uniform
 * bounds [uniform_min, uniform_max]; the design starts at the middle of its bounds */
int rt_mma_create(rt_ctx* ctx, long long n, const double* xmin, const double* xmax, double uniform_min,
                  double uniform_max, rt_mma** out);
int rt_mma_destroy(rt_mma* m);
/* mma_t::update (optimization/mma_t.cpp:18-51): one MMA step for min f0 s.t. f1 <= 0, from the
 * objective gradient df_dev and the constraint gradient dg_dev (device, n floats each, as the
 * reference's Scalar) and the constraint value g; the subproblem (a0 = 1, a = 0, c = 10, d = 1)
 * is solved exactly through its one-multiplier dual; *stop = 1 once more than 10 steps were
 * shorter than 1e-3 (the reference's stop rule); *lambda_out = the multiplier, *dxnorm_out = |dx|
 * (each may be null) */
int rt_mma_update(rt_mma* m, const float* df_dev, const float* dg_dev, double g, int* stop, double* lambda_out,
                  double* dxnorm_out);
/* mma_t::get_x: the design (device pointer owned by the state, n doubles), or a host copy */
int rt_mma_x(rt_mma* m, const double** x_dev);
int rt_mma_get_x(rt_mma* m, double* x_host);
/* setDensity(mma.get_x()) (utils/test_utils.cpp:1672): the design as the finest level's densities
 * (FP32, zero on inactive elements; n must be the element count of the dense finest level) */
int rt_mma_set_density(rt_mma* m, rt_hier* h);
/* dual-derivative evaluations run so far (each one pass over the design variables) */
long long rt_mma_evaluations(rt_mma* m);

/* ---- learned preconditioner (3D U-Net, BF16 activations, FP32 accumulation) ---- */
/* No reference counterpart.  One 3x3x3 convolution (zero padding 1) on the tensor cores:
 * out[v][n] (+)= bias[n] + sum_{tap,c} w[n][tap][c] in[v + offset(tap)][c], optional ReLU.
 * Device pointers; activations channels-last [v][stride] (v = x + X (y + Y z)), bf16;
 * w bf16 [cout][27][cin] with tap = 9 (dz+1) + 3 (dy+1) + (dx+1); out bf16 or float
 * (out_f32), accumulate only for float.  cin, cout multiples of 16 in [16, 128]. */
int rt_unet_conv3(rt_ctx* c, const void* in, int in_stride, int cin, const void* w, const float* bias, int cout,
                  void* out, int out_stride, int out_f32, int relu, int accumulate, int X, int Y, int Z);
/* kernel of every convolution in this process: 1 (default) halo tile (the input patch of P
 * z-planes read once into shared memory, every tap a shifted descriptor), 0 per-tap gather */
int rt_unet_set_conv_variant(int variant);

/* The U-Net (levels of 16/32/48/64 channels, two 3x3x3 convolutions + ReLU per level and side,
 * 2x2x2 average pooling, nearest upsampling with skip concatenation, 1x1x1 head to 3
 * channels; 684,851 parameters) over an X x Y x Z node box; weights He-initialised from seed. */
int rt_unet_create(rt_ctx* c, int X, int Y, int Z, uint64_t seed, rt_unet** out);
void rt_unet_destroy(rt_unet* u);
long long rt_unet_n_params(rt_unet* u);
/* FP32 master parameters (host arrays of rt_unet_n_params floats) */
int rt_unet_get_params(rt_unet* u, float* host);
int rt_unet_set_params(rt_unet* u, const float* host);
/* forward pass: in bf16 [V][16] and out float [V][3] device buffers (V = X Y Z) */
int rt_unet_forward(rt_unet* u, const void* in, float* out);
/* mean-squared-error gradients of one sample (no update); grads_host may be null */
int rt_unet_gradients(rt_unet* u, const void* in, const float* tgt, double* loss, float* grads_host);
/* one Adam step (b1 0.9, b2 0.999) on a batch of device samples in [batch][V][16], tgt [batch][V][3] */
int rt_unet_train_step(rt_unet* u, int batch, const void* in, const float* tgt, float lr, double* loss);
/* output unit of the network (rms of the scaled targets, fixed by the first harvest) */
double rt_unet_output_scale(rt_unet* u);
int rt_unet_set_output_scale(rt_unet* u, double oscale);
/* one (density, residual, MG-error) training sample from hierarchy h (node box = the network's):
 * a random load, k_iter plain MG-PCG iterations give the residual r and zv = Vcycle(r); input =
 * packed (log density, r / rms(r), support flag, zv / rms(zv)), target = (K^-1 r - zv) / rms(zv) /
 * output unit */
int rt_unet_harvest(rt_hier* h, rt_unet* u, int k_iter, uint64_t seed, void* in_out, float* tgt_out);
/* use the network inside rt_pcg / rt_worst_case: z = Vcycle(r) + N(rho, r, Vcycle(r)) (no
 * reference counterpart).  The correction is switched off once an iteration fails to reduce
 * ||r|| below fallback_ratio x its previous value (the plain V-cycle is the fallback and the
 * judge); that verdict holds for the design it was made on: for the following solves, and
 * across rt_update_stencil as long as the density, supports and parameters are unchanged, until
 * the design changes or the next rt_hier_set_learned.  Inside the captured PCG loop the
 * correction is the body of an IF node; once switched off, the loop is captured without it.
 * u = null detaches. */
int rt_hier_set_learned(rt_hier* h, rt_unet* u, double fallback_ratio);
/* finest-level smoothing steps (the hierarchy's smoother, FP64) applied to z after each learned
 * correction, on K z = r (0: none, the default) */
int rt_hier_set_learned_post(rt_hier* h, int sweeps);
/* corrections run since rt_hier_set_learned, and whether the gate has switched the network off
 * for the current design */
int rt_hier_learned_stats(rt_hier* h, long long* applied, int* judged_off);

#ifdef __cplusplus
}
#endif
#endif
