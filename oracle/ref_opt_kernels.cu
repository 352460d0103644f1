// The reference's optimization/optimization.cu, included unchanged, and launchers of two of its
// kernels for oracle/ref_kernels_driver.cu (which binds the __constant__ tables they read).
// Test infrastructure only.
#include "optimization.cu"

void ref_launch_sensitivity(int nv, float* rho, float* sens) {
    computeSensitivity_kernel<<<(nv + 511) / 512, 512>>>(nv, rho, 0.0, sens);
}

void ref_launch_oc_try(int nv, const float* rho, float* sens, float thres, float step, float damp, float rhomin,
                       float* newrho) {
    trySensMultiplier_kernel<<<(nv + 511) / 512, 512>>>(nv, rho, sens, thres, step, damp, rhomin, newrho);
}

// symbols grid/Grid.cu declares extern and the reference defines in optimization/projection.cu
// (not compiled here); the four kernels driven by this library do not read them
__constant__ double* gLoadtangent[2][3];
__constant__ double* gLoadnormal[3];
gBitSAT<unsigned int> vid2loadid;
