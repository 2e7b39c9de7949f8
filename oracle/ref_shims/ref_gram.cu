// Checker shim (test infrastructure): compiles the reference's
// src/aerial_bottleneck.cu unchanged from the reference tree and exposes
// gram_scalar (:56-80) and coef_apply_scalar (:88-124) with the launch
// shapes of its main() (:174-179).  64 antennas, 8 layers (compile-time).
#define main aerial_bottleneck_reference_main
#include "src/aerial_bottleneck.cu"
#undef main

extern "C" int ref_gram_shape(int* nAnt, int* nLayers) { *nAnt = N_BS_ANTS; *nLayers = N_LAYERS; return 0; }
extern "C" int ref_gram(const cf32* M, const cf32* H, cf32* G, int nSC) {
    dim3 blk(N_LAYERS, N_LAYERS), grd(N_SC_PRB, (nSC + N_SC_PRB - 1) / N_SC_PRB);
    gram_scalar<<<grd, blk>>>(M, H, G, nSC);
    return (int)cudaDeviceSynchronize();
}
extern "C" int ref_gram_coef_apply(const cf32* C, const cf32* Y, cf32* O, int nSC, int nSym) {
    dim3 blk(N_SC_PRB, nSym), grd((nSC + N_SC_PRB - 1) / N_SC_PRB, N_LAYERS);
    coef_apply_scalar<<<grd, blk>>>(C, Y, O, nSC, nSym);
    return (int)cudaDeviceSynchronize();
}

// Launch only (no synchronization), for event timing by the caller.
extern "C" int ref_gram_launch(const cf32* M, const cf32* H, cf32* G, int nSC) {
    dim3 blk(N_LAYERS, N_LAYERS), grd(N_SC_PRB, (nSC + N_SC_PRB - 1) / N_SC_PRB);
    gram_scalar<<<grd, blk>>>(M, H, G, nSC);
    return (int)cudaGetLastError();
}
