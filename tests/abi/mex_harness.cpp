// mex_harness.cpp -- calls libdugma_b200.so through the reference's four C++ entry points
// (include/dugma_mex.hpp) in the order and with the arguments the MEX gateways and DUGMA.m
// use them: init (init.cpp:65), update_sig's cpd (update_sig.cpp:45), compi's cpd
// (compi.cpp:45), fr_m (fr_m.cpp:26).  Test infrastructure: tests/test_abi.py links it
// (CPU) and tests/test_gpu_parity.py runs it and compares with the Python mirror (GPU).
//
//   mex_harness <input> <output>
// input:  int32 N, M, D; then FP64 X (N*D), X_C (N*D*D), Y (M*D), Y_C (M*D*D), R (D*D,
//         column-major), t (D)  -- the MATLAB layouts
// output: FP64 Coef, sigma (the FP32 value widened), then the 640 coefficients
#include <cstdio>
#include <cstdint>
#include <vector>

#include "dugma_mex.hpp"

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: mex_harness <input> <output>\n");
        return 2;
    }
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t hdr[3];
    if (std::fread(hdr, sizeof(hdr), 1, f) != 1) return 2;
    const int N = hdr[0], M = hdr[1], D = hdr[2];
    std::vector<double> X((size_t)N * D), XC((size_t)N * D * D), Y((size_t)M * D), YC((size_t)M * D * D), R(D * D),
        t(D);
    for (auto* v : {&X, &XC, &Y, &YC, &R, &t})
        if (std::fread(v->data(), sizeof(double), v->size(), f) != v->size()) return 2;
    std::fclose(f);

    double coef_ok = 0;
    float* Ptr[6];
    init(X.data(), XC.data(), Y.data(), YC.data(), &coef_ok, N, M, D, Ptr);
    double Nd = N, Md = M, Dd = D;
    float sig[1] = {0};
    cpd(Ptr, R.data(), t.data(), &Nd, &Md, &Dd, sig);
    double sigd = sig[0];
    double coef[640];
    cpd(Ptr, R.data(), t.data(), &Nd, &Md, &Dd, &sigd, coef);
    fr_m(Ptr);

    std::FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    std::fwrite(&coef_ok, sizeof(double), 1, o);
    std::fwrite(&sigd, sizeof(double), 1, o);
    std::fwrite(coef, sizeof(double), 640, o);
    std::fclose(o);
    return coef_ok == 1.0 ? 0 : 1;
}
