// The reference's OpenCL kernels (src/kernels/{backproject,filter,fft,forwardproject}.cl),
// compiled unchanged as C++ through clc_shim.hpp after ref.mk rewrote their
// vector literals into the build folder.  Test infrastructure only.
#include "clc_shim.hpp"
#include "backproject.cl.cpp"
#include "filter.cl.cpp"
#include "fft.cl.cpp"
#include "forwardproject.cl.cpp"
