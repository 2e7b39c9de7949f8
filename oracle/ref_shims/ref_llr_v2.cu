// Checker shim (test infrastructure): compiles the reference's
// src/llr/aerial_llr_bench_v2.cu unchanged from the reference tree and exposes
// cpu_computePamLlr_ref (:72-107), llr_v1_baseline (:114-156) and
// llr_v2_smem_warp (:174-229) through a C ABI.  Output goes to oracle/_ref/.
#define main aerial_llr_bench_v2_reference_main
#include "src/llr/aerial_llr_bench_v2.cu"
#undef main

extern "C" void ref_llr_v2_cpu_ref(const half2c* in, const float* ni, float* out, int N, int nPamBits) {
    for (int i = 0; i < N; i++)
        cpu_computePamLlr_ref(__half2float(in[i].re), __half2float(in[i].im), ni[i], nPamBits,
                              out + (size_t)i * 2 * nPamBits);
}
extern "C" int ref_llr_v2_v1(const half2c* d_in, const float* d_ni, __half* d_out, int N, int nPamBits) {
    llr_v1_baseline<<<(N + 255) / 256, 256>>>(d_in, d_ni, d_out, N, nPamBits);
    return (int)cudaDeviceSynchronize();
}
extern "C" int ref_llr_v2_v2(const half2c* d_in, const float* d_ni, __half* d_out, int N, int nPamBits) {
    llr_v2_smem_warp<<<(N + V2_SYMS_PER_BLOCK - 1) / V2_SYMS_PER_BLOCK, V2_SYMS_PER_BLOCK * V2_THREADS_PER_SYM>>>(
        d_in, d_ni, d_out, N, nPamBits);
    return (int)cudaDeviceSynchronize();
}
