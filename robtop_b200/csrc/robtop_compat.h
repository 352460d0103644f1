// robtop_compat.h — the reference's C++ entry points, implemented on the C ABI.
//
// Same names, argument meaning and call order as lavenklau/robtop's
// optimization/optimization.h:28-82 and grid/Grid.h:172-692, so callers such as
// robtop.cpp:27-46 or the TestSuit routines link against this layer unchanged
// except for two documented differences:
//  * vectors returned by getForce()/getDisplacement()/getResidual() are device
//    pointers to the three components of the DENSE node box (SoA, x fastest),
//    not the reference's GS-colour-ordered arrays (use rt_get(...,
//    RT_LAYOUT_REF_GS, ...) for that order);
//  * setBoundaryCondition's force field returns std::array<double,3> instead of
//    Eigen::Matrix<double,3,1> (Eigen is not a dependency of this library).
// Errors throw std::runtime_error carrying rt_last_error(); the reference
// printed and continued or called exit(-1).  As in the reference, solveFEM() solves for the
// force the caller has set; a caller of the preloaded field sets it first with
// setForceSupport(getPreloadForce(), grids[0]->getForce()).
#pragma once
#include <array>
#include <cstdint>
#include <utility>
#include <functional>
#include <string>
#include <vector>

#include "../../include/rtb200.h"

namespace grid {

enum Mode {
    no_support_constrain_force_direction,
    no_support_free_force,
    with_support_constrain_force_direction,
    with_support_free_force
};

class HierarchyGrid;

// one level (grid::Grid, grid/Grid.h:172-532)
class Grid {
public:
    Grid(HierarchyGrid* owner, int layer);
    ~Grid();
    void update_residual(void);
    void gs_relax(int n_times = 1);
    void restrict_residual(void);
    void prolongate_correction(void);
    void solve_fem_host(void);
    void applyK(double* u[3], double* f[3]);
    double compliance(void);
    double relative_residual(void);
    double residual(void);
    void filterSensitivity(double radii);
    void init_rho(double rh0);
    void randForce(void);
    double unitizeForce(void);
    void reset_displacement(void);
    void reset_force(void);
    void reset_residual(void);
    double** getForce(void) { return _F; }
    double** getDisplacement(void) { return _U; }
    double** getResidual(void) { return _R; }
    float* getRho(void);
    float* getSens(void);
    int n_nodes(void) const { return (int)_n_active_nodes; }
    int n_rho(void) const { return (int)_n_active_elements; }
    long long n_box_nodes(void) const { return _nv; }
    double v3_dot(double* v[3], double* u[3]);
    double v3_norm(double* v[3]);
    void v3_copy(double* vsrc[3], double* vdst[3]);
    void v3_scale(double* v[3], double ampl);
    // grid/Grid.cu:2163-2200: a += alpha b, and a = alpha a + beta b
    void v3_add(double* a[3], double alpha, double* b[3]);
    void v3_add(double alpha, double* a[3], double beta, double* b[3]);
    // grid/Grid.cu:3434-3480: per-element compliance rho_e^p u_e.KE u_e of u into ce (device, dense element order)
    void elementCompliance(double* u[3], float* ce);
    // grid/Grid.cu:2255-2286: the support force held by the grid (device [3][nload]) and its change
    double** getSupportForce(void);
    double supportForceCh(void);
    double supportForceCh(double* f[3]);
    double supportForceNorm(void);
    int _layer = 0;

private:
    friend class HierarchyGrid;
    HierarchyGrid* _H;
    long long _nv = 0, _n_active_nodes = 0, _n_active_elements = 0;
    double* _U[3];
    double* _F[3];
    double* _R[3];
    double* _FS[3] = {nullptr, nullptr, nullptr};  // support force, [3][nload] device (level 0)
    double* _FS_new = nullptr;                        // scratch [3][nload] for supportForceCh
    int _FS_n = -1;                                   // load-node count the support arrays were sized for
    void ensure_support(void);
    double* _tmp = nullptr;
};

// grid::HierarchyGrid (grid/Grid.h:534-692)
class HierarchyGrid {
public:
    HierarchyGrid(void);
    ~HierarchyGrid();
    void genFromMesh(const std::vector<unsigned int>& solid_bit, int out_reso[3]);
    // grid/Grid.cpp:184-205: voxelise the closed triangle mesh at the preferred resolution
    void genFromMesh(const std::vector<float>& pcoords, const std::vector<int>& facevertices);
    void set_prefer_reso(int preferreso) { _prefer_reso = preferreso; }
    void update_stencil(void);
    double v_cycle(int pre_relax = 1, int post_relax = 1);
    void setMode(Mode mode);
    Grid* operator[](int i) { return _grids[i]; }
    int n_grid(void) { return (int)_grids.size(); }
    void set_skip_layer(bool isskip) { _params.skip_layer1 = isskip ? 1 : 0; }
    bool isForceFree(void) { return _mode == no_support_free_force || _mode == with_support_free_force; }
    bool hasSupport(void) { return _mode == with_support_constrain_force_direction || _mode == with_support_free_force; }
    double elementLength(void) { return _params.element_length; }
    void resetAllResidual(void);
    // grid/Grid.cpp:727-764, 809-839 (the reference writes and reads OpenVDB grids): the level-0
    // densities as a raw file, magic "RTB200D1", int32 nx, ny, nz, then nx*ny*nz float32 (x fastest)
    void writeDensity(const std::string& filename);
    void readDensity(const std::string& filename);

    std::function<bool(double[3])> _inLoadArea;
    std::function<bool(double[3])> _inFixedArea;
    std::function<std::array<double, 3>(double[3])> _loadField;
    Mode _mode = with_support_free_force;

    // library handles (for callers that mix the C ABI in)
    rt_ctx* ctx(void) { return _ctx; }
    rt_hier* hier(void) { return _h; }
    rt_params& params(void) { return _params; }
    void check(int status, const char* what);
    const std::vector<int>& loadNodes(void) const { return _load_nodes; }
    const std::vector<double>& preloadForce(void) const { return _preload; }

private:
    rt_ctx* _ctx = nullptr;
    rt_hier* _h = nullptr;
    rt_params _params;
    int _prefer_reso = 128;  // grid/Grid.h:541
    std::vector<Grid*> _grids;
    std::vector<int> _load_nodes;
    std::vector<double> _preload;  // [3*nload] load field at the load nodes
};

}  // namespace grid

// mem/gpu_manager_t.h: the reference's device-buffer manager, the members its callers use.
// Buffers come from the library's CUDA runtime; callers of this layer allocate through it
// rather than linking a CUDA runtime of their own.
class gpu_manager_t {
public:
    static void upload_buf(void* dst, const void* src, size_t size);
    static void download_buf(void* host_dst, const void* dev_src, size_t n);
    static void initMem(void* pdata, size_t len, char value = 0);
    void* add_buf(const std::string& name, size_t size, const void* src = nullptr);
    void* add_buf(size_t size, const void* src = nullptr);
    void delete_buf(const std::string& name);
    void delete_buf(void* pbuf);
    size_t size(void);
    ~gpu_manager_t();

private:
    struct Buf {
        std::string name;
        void* p;
        size_t size;
    };
    std::vector<Buf> _bufs;
    int _anonymous = 0;
};

extern gpu_manager_t gpu_manager;

// optimization/optimization.h:11-22
struct Parameter {
    float damp_ratio;
    float design_step;
    float power_penalty;
    float volume_ratio;
    float volume_decrease;
    int filter_radius;
    float min_rho;
    int gridreso;
    float youngs_modulu;
    float poisson_ratio;
};

extern Parameter params;
extern grid::HierarchyGrid grids;

// optimization/optimization.h:28-82
void buildGrids(const std::vector<unsigned int>& solid_bit, int reso);
// optimization/optimization.cpp:14-19: the mesh form
void buildGrids(const std::vector<float>& coords, const std::vector<int>& trifaces);
void setParameters(float volRatio, float volDecrease, float designStep, float filterRadi, float dampRatio,
                   float powerPenal, float min_density, int gridreso, float youngs_modulu, float poisson_ratio,
                   float shell_width, bool logdensity, bool logcompliance);
void setWorkMode(const std::string& modestr);
void solveFEM(void);
double modifiedPM(void);
void computeSensitivity(void);
float updateDensities(float Vgoal);
void optimization(int max_iter = 100);
// the worst-case compliance of each iteration of the last optimization() (the reference writes it
// to the file "cworst"), and with volumes != nullptr the volume goals ("vrec")
const std::vector<double>& optimizationRecords(std::vector<double>* volumes = nullptr);
grid::HierarchyGrid& getGrids(void);
void setBoundaryCondition(std::function<bool(double[3])> fixarea, std::function<bool(double[3])> loadarea,
                          std::function<std::array<double, 3>(double[3])> forcefield);
void uploadTemplateMatrix(void);
void initDensities(double rho);
void update_stencil(void);
void test_rigid_displacement(void);

// optimization/optimization.h:28-82, the remaining entry points
void setOutpurDir(const std::string& dirname);
const std::string& getOutputDir(void);
void selfTest(void);
double inCompleteModiPM(double fch_thres = 1e-2);
double MGPSOR(void);
std::pair<double, double> RayleighGradient(double* u[3], double* g[3]);
double Pnorm(double* u[3]);
double Knorm(double* u[3]);
bool checkAdjointVariable(void);

// optimization/projection.h:16-65 (dense level-0 node ids instead of GS ids; support-force
// arrays hold the load nodes in increasing id)
const std::vector<int>& getLoadNodes(void);
int n_loadnodes(void);
void forceProject(double* f_dev[3]);
void forceProject(std::vector<double> fsupport[3]);
void getForceSupport(double const* const f_dev[3], double* fsup[3]);
void getForceSupport(double const* const f_dev[3], std::vector<double> fs[3]);
void setForceSupport(double const* const fsup[3], double* f_dev[3]);
void displacementProject(double* u_dev[3]);
double** getPreloadForce(void);

// setDensity (utils/test_utils.cpp:1672): densities of the dense finest level from a device
// array (FP32); the volume ratio of the current densities over the active elements
// (Grid::volumeRatio)
void setDensity(const float* rho_dev);
double volumeRatio(void);

// optimization/mma_t.h:159-273: the method of moving asymptotes with one constraint (the
// reference's TestSuit::test2011 / testtest2011 drive it with the volume constraint).  The
// subproblem is solved exactly through its one-multiplier dual; the state is FP64, the
// gradients and the design view FP32 device arrays, as the reference's Scalar.
namespace MMA {
class mma_t {
public:
    struct XView {
        float* p;
        float* data() { return p; }
    };
    mma_t(int ndim, int nConstrain, double err_tol = 1e-7);
    ~mma_t();
    mma_t(const mma_t&) = delete;
    mma_t& operator=(const mma_t&) = delete;
    void init(float lower_bound, float upper_bound);
    void init(const float* lower_bound_host, const float* upper_bound_host);
    // one step: df (device, n), dg[0] (device, n) and g (device, 1 value); true once the
    // reference's stop rule fires (more than 10 steps shorter than 1e-3)
    bool update(float* dev_df, float** dg, float* dev_g);
    XView get_x(void);  // FP32 device copy of the design, valid until the next update
    int n_dim(void) const { return _n; }
    int n_constrain(void) const { return 1; }

private:
    int _n;
    ::rt_mma* _m = nullptr;
    float* _x32 = nullptr;
};
}  // namespace MMA

