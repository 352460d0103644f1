// compat_main.cpp — drives the library through the reference's own C++ entry
// points, in the order robtop.cpp:27-46 and TestSuit::testOrdinaryTopopt
// (utils/test_utils.cpp:589-660) call them, and prints the results as
// "key value" lines for tests/test_gpu_compat.py to compare with the oracle.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../robtop_b200/csrc/robtop_compat.h"

int main(int argc, char** argv) {
    setvbuf(stdout, nullptr, _IONBF, 0);  // every line reaches the test even if a call throws
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
    // TestSuit::testOrdinaryTopopt (utils/test_utils.cpp:594): the preloaded force, then solveFEM
    setForceSupport(getPreloadForce(), getGrids()[0]->getForce());
    solveFEM();
    printf("compliance %.17g\n", getGrids()[0]->compliance());
    printf("rel_residual %.17g\n", getGrids()[0]->relative_residual());
    const double mu = modifiedPM();
    printf("worst_compliance %.17g\n", mu);
    // the adjoint identity of checkAdjointVariable (optimization/optimization.cu:353-402) holds for
    // N^T lambda = 2 u_w - 2 mu K u_w; a zero vector fails it
    grid::Grid* g0 = getGrids()[0];
    g0->applyK(g0->getDisplacement(), g0->getForce());
    g0->v3_add(2.0, g0->getDisplacement(), -2.0 * mu, g0->getForce());
    printf("adjoint_ok %d\n", checkAdjointVariable() ? 1 : 0);
    g0->reset_displacement();
    printf("adjoint_zero_ok %d\n", checkAdjointVariable() ? 1 : 0);
    // element compliance of the worst-case displacement sums to u.K u (on the displacement
    // with its support nodes zeroed: K u has identity rows there, the element sums do not)
    const double mu2 = modifiedPM();
    {
        const long long nvb0 = g0->n_box_nodes();
        std::vector<double> uh(3 * nvb0), kuh(3 * nvb0);
        std::vector<uint8_t> fix(nvb0);
        rt_get(getGrids().hier(), RT_FIELD_U, 0, RT_LAYOUT_DENSE, uh.data());
        rt_get(getGrids().hier(), RT_FIELD_VFIX, 0, RT_LAYOUT_DENSE, fix.data());
        double ufix = 0;
        for (long long v = 0; v < nvb0; v++)
            if (fix[v])
                for (int c = 0; c < 3; c++) {
                    ufix = std::max(ufix, std::fabs(uh[c * nvb0 + v]));
                    uh[c * nvb0 + v] = 0;
                }
        printf("worst_u_support_max %.17g\n", ufix);
        rt_put(getGrids().hier(), RT_FIELD_U, 0, RT_LAYOUT_DENSE, uh.data());
        rt_apply_K(getGrids().hier(), uh.data(), kuh.data());
        double uku = 0;
        for (long long i = 0; i < 3 * nvb0; i++) uku += uh[i] * kuh[i];
        printf("worst_uKu %.17g\n", uku);
    }
    float* ce = (float*)gpu_manager.add_buf("element compliance", sizeof(float) * nx * ny * nz);
    g0->elementCompliance(g0->getDisplacement(), ce);
    std::vector<float> ceh((size_t)nx * ny * nz);
    gpu_manager_t::download_buf(ceh.data(), ce, sizeof(float) * ceh.size());
    gpu_manager.delete_buf(ce);
    double csum = 0;
    for (float v : ceh) csum += v;
    printf("element_compliance_sum %.17g\n", csum);
    printf("worst_compliance2 %.17g\n", mu2);
    // projection API (wsff: the projection keeps the load-node values, zeroes every other node)
    printf("n_loadnodes %d\n", n_loadnodes());
    std::vector<double> fs[3];
    getForceSupport(g0->getForce(), fs);
    double fs2 = 0;
    for (int c = 0; c < 3; c++)
        for (double v : fs[c]) fs2 += v * v;
    printf("support_norm2 %.17g\n", fs2);
    printf("pnorm %.17g\n", Pnorm(g0->getForce()));
    forceProject(g0->getForce());
    printf("projected_norm2 %.17g\n", g0->v3_dot(g0->getForce(), g0->getForce()));
    double* fsd = (double*)gpu_manager.add_buf(sizeof(double) * 3 * n_loadnodes());
    double* fsp[3] = {fsd, fsd + n_loadnodes(), fsd + 2 * n_loadnodes()};
    getForceSupport(g0->getForce(), fsp);
    g0->reset_force();
    setForceSupport(fsp, g0->getForce());
    printf("restored_norm2 %.17g\n", g0->v3_dot(g0->getForce(), g0->getForce()));
    gpu_manager.delete_buf(fsd);
    // the Rayleigh quotient R(u) = |P u|^2 / u.K u of the worst-case displacement and its gradient
    const long long nvb = g0->n_box_nodes();
    double* gm = (double*)gpu_manager.add_buf("gradient", sizeof(double) * 3 * nvb);
    double* gv[3] = {gm, gm + nvb, gm + 2 * nvb};
    const double mu3 = modifiedPM();
    const auto pk = RayleighGradient(g0->getDisplacement(), gv);
    printf("rayleigh_pnorm %.17g\n", pk.first);
    printf("rayleigh_knorm %.17g\n", pk.second);
    printf("rayleigh_grad_norm %.17g\n", g0->v3_norm(gv));
    printf("worst_compliance3 %.17g\n", mu3);
    gpu_manager.delete_buf(gm);
    // the incomplete power method and the preconditioned eigen-iteration
    printf("incomplete_pm %.17g\n", inCompleteModiPM(1e-2));
    printf("mgpsor %.17g\n", MGPSOR());
    selfTest();
    computeSensitivity();
    const float g = updateDensities(0.4f);
    printf("oc_multiplier %.9g\n", g);
    std::vector<float> rho((size_t)nx * ny * nz);
    rt_get(getGrids().hier(), RT_FIELD_RHO, 0, RT_LAYOUT_DENSE, rho.data());
    double s = 0;
    for (float r : rho) s += r;
    printf("volume %.9g\n", s / rho.size());
    // density file round trip (writeDensity / readDensity)
    setOutpurDir("/tmp");
    const std::string dfile = getOutputDir() + "/rtb200_density_test.bin";
    getGrids().writeDensity(dfile);
    initDensities(0.9);
    getGrids().readDensity(dfile);
    std::vector<float> rho2(rho.size());
    rt_get(getGrids().hier(), RT_FIELD_RHO, 0, RT_LAYOUT_DENSE, rho2.data());
    printf("density_roundtrip %d\n", rho2 == rho ? 1 : 0);
    // the optimisation loop with its stop test (volume goal 0.4 throughout)
    optimization(12);
    std::vector<double> vols;
    const std::vector<double>& crec = optimizationRecords(&vols);
    printf("opt_iterations %zu\n", crec.size());
    printf("opt_first_compliance %.17g\n", crec.front());
    printf("opt_last_compliance %.17g\n", crec.back());
    printf("opt_last_volume_goal %.9g\n", vols.back());
    // TestSuit::testtest2011 (utils/test_utils.cpp:1750-1800): MMA steps on the densities with
    // the volume constraint scaled by 1e3 and the sensitivity by 1e5
    {
        rt_level_info l0;
        rt_hier_level_info(getGrids().hier(), 0, &l0);
        const int ne = l0.nx * l0.ny * l0.nz;
        std::vector<uint8_t> act(ne);
        rt_get(getGrids().hier(), RT_FIELD_EACT, 0, RT_LAYOUT_DENSE, act.data());
        long long na = 0;
        for (uint8_t a : act) na += a;
        std::vector<float> dvh(ne), sh(ne);
        for (int e = 0; e < ne; e++) dvh[e] = act[e] ? 1e3f / (float)na : 0.f;
        float* dv = (float*)gpu_manager.add_buf("mma dv", sizeof(float) * ne, dvh.data());
        float* sdev = (float*)gpu_manager.add_buf("mma sens", sizeof(float) * ne);
        float* vdev = (float*)gpu_manager.add_buf("mma v", sizeof(float));
        MMA::mma_t mma(ne, 1);
        mma.init(1e-3f, 1.0f);
        double c_mma = 0;
        for (int itn = 0; itn < 3; itn++) {
            setDensity(mma.get_x().data());
            update_stencil();
            const float v = 1e3f * (float)(volumeRatio() - 0.4);
            gpu_manager_t::upload_buf(vdev, &v, sizeof(float));
            c_mma = modifiedPM();
            computeSensitivity();
            gpu_manager_t::download_buf(sh.data(), getGrids()[0]->getSens(), sizeof(float) * ne);
            for (float& x : sh) x *= 1e5f;
            gpu_manager_t::upload_buf(sdev, sh.data(), sizeof(float) * ne);
            mma.update(sdev, &dv, vdev);
        }
        setDensity(mma.get_x().data());
        printf("mma_volume %.9g\n", volumeRatio());
        printf("mma_compliance %.17g\n", c_mma);
        gpu_manager.delete_buf(dv);
        gpu_manager.delete_buf(sdev);
        gpu_manager.delete_buf(vdev);
    }
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
