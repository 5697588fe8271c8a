// dugma_mex.hpp -- the reference's four C++ entry points, exported with their exact
// signatures (C++ linkage) by libdugma_b200.so so that the reference's MEX gateways
// link against it unchanged.  Each forwards to the C ABI in dugma.h; on failure it
// prints the reason to stderr and returns (the reference calls exit()).
#pragma once

// init.cu:249-259, declared by init.cpp:9-19
void init(double* X, double* X_C, double* Y, double* Y_C, double* Coef, int N, int M, int D, float* Ptr[6]);
// update_sig.cu:319-321, declared by update_sig.cpp:7; sig[0] = NaN on failure
void cpd(float* Ptr[6], double* R, double* t, double* N, double* M, double* D, float sig[1]);
// compi.cu:511-513, declared by compi.cpp:7; all 640 entries NaN on failure
void cpd(float* Ptr[6], double* R, double* t, double* N, double* M, double* D, double* sig, double coefficient[640]);
// fr_m.cu:14-16, declared by fr_m.cpp:7 (no cudaDeviceReset)
void fr_m(float* Ptr[6]);
