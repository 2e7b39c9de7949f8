// Checker shim (test infrastructure): compiles the reference's
// src/aerial_coef_wmma.cu unchanged from the reference tree and exposes its
// three coef_apply kernels (:71-104, :146-239, :250-337) with the launch
// shapes of its main() (:400-407).  Shapes are the file's compile-time
// constants: 64 antennas, 8 layers, 12 subcarriers per PRB.  nSym <= 16.
#define main aerial_coef_wmma_reference_main
#include "src/aerial_coef_wmma.cu"
#undef main

extern "C" int ref_coef_shape(int* nAnt, int* nLayers, int* nScPrb) {
    *nAnt = N_BS_ANTS; *nLayers = N_LAYERS; *nScPrb = N_SC_PRB;
    return 0;
}
extern "C" int ref_coef_v1(const cf32* C, const cf32* Y, cf32* O, int nSC, int nSym) {
    dim3 blk(N_SC_PRB, nSym), grd((nSC + N_SC_PRB - 1) / N_SC_PRB, N_LAYERS);
    coef_apply_v1_scalar<<<grd, blk>>>(C, Y, O, nSC, nSym);
    return (int)cudaDeviceSynchronize();
}
extern "C" int ref_coef_v2(const cf32* C, const cf32* Y, cf32* O, int nSC, int nSym) {
    coef_apply_v2_wmma<<<nSC, 32>>>(C, Y, O, nSC, nSym);
    return (int)cudaDeviceSynchronize();
}
extern "C" int ref_coef_v3(const cf32* C, const cf32* Y, cf32* O, int nSC, int nSym) {
    coef_apply_v3_wmma_multiw<<<(nSC + SC_PER_BLK - 1) / SC_PER_BLK, SC_PER_BLK * 32>>>(C, Y, O, nSC, nSym);
    return (int)cudaDeviceSynchronize();
}
// Event-timed launches on the default stream (the reference's own timing
// pattern, :443-458): returns the median of `iters` launch times in ms.
extern "C" float ref_coef_time(int which, const cf32* C, const cf32* Y, cf32* O, int nSC, int nSym, int iters) {
    cudaEvent_t s, e; cudaEventCreate(&s); cudaEventCreate(&e);
    float* t = (float*)malloc(sizeof(float) * iters);
    for (int i = 0; i < iters; i++) {
        cudaEventRecord(s);
        if (which == 1) {
            dim3 blk(N_SC_PRB, nSym), grd((nSC + N_SC_PRB - 1) / N_SC_PRB, N_LAYERS);
            coef_apply_v1_scalar<<<grd, blk>>>(C, Y, O, nSC, nSym);
        } else if (which == 2) {
            coef_apply_v2_wmma<<<nSC, 32>>>(C, Y, O, nSC, nSym);
        } else {
            coef_apply_v3_wmma_multiw<<<(nSC + SC_PER_BLK - 1) / SC_PER_BLK, SC_PER_BLK * 32>>>(C, Y, O, nSC, nSym);
        }
        cudaEventRecord(e); cudaEventSynchronize(e);
        cudaEventElapsedTime(&t[i], s, e);
    }
    float m = (float)median_ms(t, iters);
    free(t); cudaEventDestroy(s); cudaEventDestroy(e);
    return m;
}

// Launch only (no synchronization), for event timing by the caller on the
// default stream: which = 1 (V1 scalar), 2 (V2 WMMA), 3 (V3 WMMA 4 warps).
extern "C" int ref_coef_launch(int which, const cf32* C, const cf32* Y, cf32* O, int nSC, int nSym) {
    if (which == 1) {
        dim3 blk(N_SC_PRB, nSym), grd((nSC + N_SC_PRB - 1) / N_SC_PRB, N_LAYERS);
        coef_apply_v1_scalar<<<grd, blk>>>(C, Y, O, nSC, nSym);
    } else if (which == 2) {
        coef_apply_v2_wmma<<<nSC, 32>>>(C, Y, O, nSC, nSym);
    } else {
        coef_apply_v3_wmma_multiw<<<(nSC + SC_PER_BLK - 1) / SC_PER_BLK, SC_PER_BLK * 32>>>(C, Y, O, nSC, nSym);
    }
    return (int)cudaGetLastError();
}
