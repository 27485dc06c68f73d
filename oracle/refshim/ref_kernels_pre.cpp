// The reference's element-wise preprocessing kernels (src/kernels/ffc.cl,
// src/kernels/conebeam.cl) compiled unchanged as C++ through clc_shim.hpp, in a
// translation unit of their own so that the float overloads of log/sqrt they
// need do not change how the other kernels compile.  Test infrastructure only.
#include <cmath>

#include "clc_shim.hpp"
using std::isinf;
using std::isnan;
using std::log;
using std::sqrt;
#include "ffc.cl.cpp"
#include "conebeam.cl.cpp"
