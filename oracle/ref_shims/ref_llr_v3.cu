// Checker shim (test infrastructure): compiles the reference's
// src/llr/aerial_llr_v3.cu unchanged, from the reference tree (the include
// path is given by oracle/Makefile), and exposes its FP64 host model cpu_ref
// (:61-79) and its kernels llr_v1_baseline (:84-108) and
// llr_v3_reg_template<N> (:219-229) through a C ABI.  Output goes to
// oracle/_ref/ only.
#define main aerial_llr_v3_reference_main
#include "src/llr/aerial_llr_v3.cu"
#undef main

extern "C" void ref_llr_v3_cpu_ref(const half2c* in, const float* ni, float* out, int N, int nPamBits) {
    for (int i = 0; i < N; i++)
        cpu_ref(__half2float(in[i].re), __half2float(in[i].im), ni[i], nPamBits, out + (size_t)i * 2 * nPamBits);
}

// Device pointers; launch shapes as in the reference's main() (:292, :302).
extern "C" int ref_llr_v3_v1(const half2c* d_in, const float* d_ni, __half* d_out, int N, int nPamBits) {
    llr_v1_baseline<<<(N + 511) / 512, 512>>>(d_in, d_ni, d_out, N, nPamBits);
    return (int)cudaDeviceSynchronize();
}
extern "C" int ref_llr_v3_v3(const half2c* d_in, const float* d_ni, __half* d_out, int N, int nPamBits) {
    dim3 b(512), g((N + 511) / 512);
    if (nPamBits == 2) llr_v3_reg_template<2><<<g, b>>>(d_in, d_ni, d_out, N);
    else if (nPamBits == 3) llr_v3_reg_template<3><<<g, b>>>(d_in, d_ni, d_out, N);
    else if (nPamBits == 4) llr_v3_reg_template<4><<<g, b>>>(d_in, d_ni, d_out, N);
    else return -1;
    return (int)cudaDeviceSynchronize();
}

// Launch only (no synchronization), for event timing by the caller:
// which = 1 (llr_v1_baseline) or 3 (llr_v3_reg_template, nPamBits 2..4).
extern "C" int ref_llr_v3_launch(int which, const half2c* d_in, const float* d_ni, __half* d_out, int N,
                                 int nPamBits) {
    dim3 b(512), g((N + 511) / 512);
    if (which == 1) llr_v1_baseline<<<g, b>>>(d_in, d_ni, d_out, N, nPamBits);
    else if (nPamBits == 2) llr_v3_reg_template<2><<<g, b>>>(d_in, d_ni, d_out, N);
    else if (nPamBits == 3) llr_v3_reg_template<3><<<g, b>>>(d_in, d_ni, d_out, N);
    else if (nPamBits == 4) llr_v3_reg_template<4><<<g, b>>>(d_in, d_ni, d_out, N);
    else return -1;
    return (int)cudaGetLastError();
}
