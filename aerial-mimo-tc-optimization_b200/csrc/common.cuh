// common.cuh -- shared device/host helpers of the B200 equalization library.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <atomic>
#include <cmath>
#include <mutex>

#include "../../include/aerial_eq.h"

namespace aeq {

using cf = float2;  // {re, im}: the reference's struct cf32 (src/aerial_coef_wmma.cu:60)

// Status helper: map the last launch error to an ABI status.
inline int launch_status() {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AERIAL_OK : (int)e;
}

// Status of a runtime call.  A failed call also leaves its error in the
// calling thread's last-error state, where the next launch check
// (launch_status) would read it as that launch's own; once returned here it
// is cleared.  Sticky errors (a faulted context) stay, as the runtime keeps
// them.
inline int rt_status(cudaError_t e) {
    if (e == cudaSuccess) return AERIAL_OK;
    (void)cudaGetLastError();
    return (int)e;
}

inline cudaStream_t to_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kMaxDevices = 64;                 // devices with cached per-device state
constexpr int kMaxSmemPerCta = 227 * 1024;      // B200 dynamic shared memory per block

// cuCtxGetCurrent / cuCtxGetId from the driver, looked up once.
struct CtxQuery {
    PFN_cuCtxGetCurrent_v4000 current = nullptr;
    PFN_cuCtxGetId_v12000 id = nullptr;
};
inline const CtxQuery& ctx_query() {
    static std::once_flag once;
    static CtxQuery q;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult r;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r) == cudaSuccess &&
            r == cudaDriverEntryPointSuccess)
            q.current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &r) == cudaSuccess &&
            r == cudaDriverEntryPointSuccess)
            q.id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
    });
    return q;
}

// Unique ID of the calling thread's current context, 0 if there is none yet
// or the driver cannot say.
inline unsigned long long current_ctx_id() {
    const CtxQuery& q = ctx_query();
    if (!q.current || !q.id) return 0;
    CUcontext ctx = nullptr;
    if (q.current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    unsigned long long id = 0;
    return q.id(ctx, &id) == CUDA_SUCCESS ? id : 0;
}

// SM count of the current device, looked up once per device.
inline int sm_count() {
    static std::atomic<int> cache[kMaxDevices];
    int dev = 0;
    cudaGetDevice(&dev);
    const bool cached = dev >= 0 && dev < kMaxDevices;
    int n = cached ? cache[dev].load(std::memory_order_relaxed) : 0;
    if (!n) {
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
        if (cached) cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

// Raises kernel K's dynamic shared-memory limit to the per-block maximum,
// once per device (the launch's own request then sets its occupancy).
template <auto K>
int allow_max_smem() {
    static std::mutex mu;
    static bool done[kMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return rt_status(e);
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < kMaxDevices && done[dev]) return AERIAL_OK;
    e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemPerCta);
    if (e != cudaSuccess) return rt_status(e);
    if (dev >= 0 && dev < kMaxDevices) done[dev] = true;
    return AERIAL_OK;
}

// cma() of src/aerial_coef_wmma.cu:61-64 with the contraction nvcc applies to
// `acc + a*b - c*d`: re = fma(-a.im, b.im, fma(a.re, b.re, acc.re)),
// im = fma(a.im, b.re, fma(a.re, b.im, acc.im)).  Written with explicit
// round-to-nearest fmas so the result does not depend on -fmad.
__device__ __forceinline__ cf cma(cf a, cf b, cf acc) {
    cf r;
    r.x = __fmaf_rn(-a.y, b.y, __fmaf_rn(a.x, b.x, acc.x));
    r.y = __fmaf_rn(a.y, b.x, __fmaf_rn(a.x, b.y, acc.y));
    return r;
}

// Per-dimension Gray-PAM decision distances D_i = 2^(n-1-i) / sqrt(2(4^n-1)/3)
// of unit-energy QAM with 2n bits; D[n-1] is the half spacing `dist`.
// (The same values as the LUT of src/llr/aerial_llr_v3.cu:42-49, computed.)
struct PamLut {
    float d[4];
};
inline PamLut pam_lut(int n) {
    PamLut p{{0.f, 0.f, 0.f, 0.f}};
    double norm = std::sqrt(2.0 * (double)((1 << (2 * n)) - 1) / 3.0);
    float r = (float)(1.0 / norm);
    for (int i = 0; i < n; i++) p.d[i] = r * (float)(1 << (n - 1 - i));
    return p;
}

// Max-log PAM LLRs of one complex symbol, the arithmetic of llr_v1_baseline
// (src/llr/aerial_llr_v3.cu:90-107): soft-bit chain sb[i+1] = D_i - |sb[i]|,
// pMD[i] = (dist + |sb[i]|)^2, minDist1 = (|sb[n-1]| - dist)^2,
// llr_i = +-(pMD[i] - minDist1) * noise, clamped to +-65504.
// out[2*bit + iq].  Every operation is explicitly rounded so the result is
// bit-identical to llr_v1_baseline as nvcc 12.9 compiles it for sm_100a:
// for 16/64/256-QAM it rounds each square separately; for QPSK (N = 1) its
// final subtraction is contracted into fma(-t, t, pMD) with t = |sb| - dist,
// and that is restated here.
template <int N>
__device__ __forceinline__ void pam_llr(float pamI, float pamQ, float noise, const PamLut& L,
                                        float* out) {
    const float dist = L.d[N - 1];
#pragma unroll
    for (int iq = 0; iq < 2; iq++) {
        float sb = iq == 0 ? pamI : pamQ;
        float pmd[N];
        unsigned sign = 0;
#pragma unroll
        for (int i = 0; i < N; i++) {
            float a = fabsf(sb);
            float m = __fadd_rn(dist, a);
            pmd[i] = __fmul_rn(m, m);
            if (sb < 0.f) sign |= 1u << i;
            if (i < N - 1) sb = __fsub_rn(L.d[i], a);
        }
        const float t = __fsub_rn(fabsf(sb), dist);
        const float md1 = __fmul_rn(t, t);
#pragma unroll
        for (int i = 0; i < N; i++) {
            const float diff = (N == 1) ? __fmaf_rn(-t, t, pmd[i]) : __fsub_rn(pmd[i], md1);
            float llr = __fmul_rn(diff, noise);
            if (sign & (1u << i)) llr = -llr;
            out[2 * i + iq] = fmaxf(-65504.f, fminf(65504.f, llr));
        }
    }
}

}  // namespace aeq
