// Project-written stand-in for the reference's matlab/matlab_utils.h (which needs the MATLAB
// engine): the matrix hand-off to a MATLAB session is a no-op here.
#pragma once
#include <string>
template <class M>
void eigen2ConnectedMatlab(const std::string&, const M&) {}
