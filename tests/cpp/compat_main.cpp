// compat_main.cpp — drives the library through the reference's own C++ entry
// points, in the order robtop.cpp:27-46 and TestSuit::testOrdinaryTopopt
// (utils/test_utils.cpp:589-660) call them, and prints the results as
// "key value" lines for tests/test_gpu_compat.py to compare with the oracle.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../robtop_b200/csrc/robtop_compat.h"

int main(int argc, char** argv) {
    const int nx = 24, ny = 12, nz = 12, R = 32;
    // cantilever: x = 0 clamped, load on the bottom edge of the x = nx face
    setParameters(0.4f, 0.0f, 0.03f, 2.0f, 0.5f, 3.0f, 1e-3f, R, 1e6f, 0.4f, 0.0f, false, false);
    setWorkMode("wsff");
    const int nload = ny + 1;
    setBoundaryCondition([](double p[3]) { return p[0] == 0.0; },
                         [=](double p[3]) { return p[0] == nx && p[2] == 0.0; },
                         [=](double p[3]) { return std::array<double, 3>{0.0, 0.0, -1.0 / nload}; });
    std::vector<unsigned int> bits((R * R * R + 31) / 32, 0u);
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                const long t = x + (long)R * (y + (long)R * z);
                bits[t >> 5] |= 1u << (t & 31);
            }
    buildGrids(bits, R);
    uploadTemplateMatrix();
    initDensities(0.4);
    update_stencil();
    printf("levels %d\n", getGrids().n_grid());
    printf("load_nodes %zu\n", getGrids().loadNodes().size());
    test_rigid_displacement();
    solveFEM();
    printf("compliance %.17g\n", getGrids()[0]->compliance());
    printf("rel_residual %.17g\n", getGrids()[0]->relative_residual());
    const double mu = modifiedPM();
    printf("worst_compliance %.17g\n", mu);
    computeSensitivity();
    const float g = updateDensities(0.4f);
    printf("oc_multiplier %.9g\n", g);
    std::vector<float> rho((size_t)nx * ny * nz);
    rt_get(getGrids().hier(), RT_FIELD_RHO, 0, RT_LAYOUT_DENSE, rho.data());
    double s = 0;
    for (float r : rho) s += r;
    printf("volume %.9g\n", s / rho.size());
    // the mesh form of buildGrids (optimization/optimization.cpp:14-19): a 24 x 12 x 12 box
    // of 12 triangles, voxelised at gridreso R - 1 (cube 32^3)
    setParameters(0.4f, 0.0f, 0.03f, 2.0f, 0.5f, 3.0f, 1e-3f, R - 1, 1e6f, 0.4f, 0.0f, false, false);
    const std::vector<float> coords = {0, 0, 0, 24, 0, 0, 24, 12, 0, 0, 12, 0, 0, 0, 12, 24, 0, 12, 24, 12, 12, 0, 12, 12};
    const std::vector<int> faces = {0, 2, 1, 0, 3, 2, 4, 5, 6, 4, 6, 7, 0, 1, 5, 0, 5, 4,
                                    2, 3, 7, 2, 7, 6, 0, 4, 7, 0, 7, 3, 1, 2, 6, 1, 6, 5};
    buildGrids(coords, faces);
    rt_level_info li;
    rt_hier_level_info(getGrids().hier(), 0, &li);
    printf("mesh_levels %d\n", getGrids().n_grid());
    printf("mesh_elements %lld\n", li.n_active_elements);
    printf("ok 1\n");
    return 0;
}
