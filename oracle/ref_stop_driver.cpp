// Test infrastructure: drives the reference's own snippet::converge_criteria
// (utils/snippet.h:156-213), compiled unchanged from the reference's header, so that the stop
// test of the optimisation loop can be checked against it.  Only tests load the library.
//
// converge_criteria::update calls an unqualified abs() on a double.  Built with g++ as-is, the
// only abs that lookup finds from namespace snippet is the C library's int abs(int): the change
// is truncated to an integer before the division, so every change below 1 reads as 0.  Where the
// C++ overloads are visible in the global namespace (MSVC, for which the header was written) the
// change is the floating-point one.  REF_STOP_FLOAT_ABS makes std::abs visible in namespace
// snippet before the header is read, which gives the second behaviour from the same source.
#include <cstdio>

#ifdef REF_STOP_FLOAT_ABS
#include <cmath>
#include <cstdlib>
namespace snippet {
using std::abs;
}
#endif

#include "snippet.h"

extern "C" __attribute__((visibility("default"))) void ref_converge_run(int n_constrain, int max_counter,
                                                                        double thres, int n, const double* values,
                                                                        const double* constraints, int* stop) {
    snippet::converge_criteria crit(n_constrain, max_counter, thres);
    for (int i = 0; i < n; i++) {
        double g[8];
        for (int j = 0; j < n_constrain && j < 8; j++) g[j] = constraints[(long)i * n_constrain + j];
        stop[i] = crit.update(values[i], g) ? 1 : 0;
    }
    fflush(stdout);
}
