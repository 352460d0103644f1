// C ABI around the reference's own element stiffness routine (element/templateMatrix.cpp:31-124,
// compiled unchanged from the reference sources against the stubs in oracle/ref_stubs/):
// ref_template_matrix(h, E, nu, out[576]) runs initTemplateMatrix and copies the 24x24 KE.
// Test infrastructure: it pins the oracle's or_template_matrix to the reference.
#include <cstring>

#include "templateMatrix.h"

extern "C" void ref_template_matrix(double h, double E, double nu, double* out) {
    gpu_manager_t gm;
    initTemplateMatrix(h, gm, E, nu);
    std::memcpy(out, getTemplateMatrixElements(), sizeof(double) * 576);
}
