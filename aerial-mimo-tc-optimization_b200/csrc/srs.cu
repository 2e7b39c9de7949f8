// srs.cu -- SRS filter multiply (srsFilterMultiply of the reference,
// src/srs/srs_wmma_bench.cu:57-90 and :102-231):
//   H_est[blk][ant][k_out][p] = sum_k (W[k_out][k] * FOCC[p][k % F]) * SRS[blk][ant][k]
// The reference accumulates in FP16 (__hfma in V1, an FP16 accumulator in
// V2); here the filter taps W*FOCC are formed in FP32 once per CTA and the
// K-term sums are FP32, rounded once at the store.  complex_conjmul (:43-47)
// computes the plain product despite its name; the plain product is kept.
//
// One CTA per (SRS block, 16-antenna slab): the K*P*K filter taps of the
// block are built in shared memory laid out [k][k_out][p] so a warp reading
// tap k for consecutive outputs is conflict-free; the 16 SRS rows of the
// slab are staged once.  Threads map to outputs in the reference's
// [ant][k_out][p] order, so the stores are coalesced.
#include "common.cuh"

namespace aeq {

constexpr int kSrsAntPerCta = 16;

template <bool TO_CHANNEL>
__global__ void __launch_bounds__(256) srs_filter_kernel(const __half2* __restrict__ srs,
                                                          const __half2* __restrict__ W,
                                                          const __half2* __restrict__ focc, void* __restrict__ out,
                                                          int nAnt, int K, int P, int F) {
    extern __shared__ float2 sm[];
    float2* taps = sm;                          // [K][K][P]: taps[(k*K + ko)*P + p]
    float2* rows = sm + (long)K * K * P;        // [16][K]
    const int blk = blockIdx.x;
    const int ant0 = blockIdx.y * kSrsAntPerCta;
    const int nA = min(kSrsAntPerCta, nAnt - ant0);
    const int KP = K * P;
    for (int e = threadIdx.x; e < K * KP; e += blockDim.x) {
        const int k = e / KP, r = e % KP, ko = r / P, p = r % P;
        const float2 w = __half22float2(W[ko * K + k]);
        const float2 f = __half22float2(focc[p * F + (k % F)]);
        taps[e] = make_float2(w.x * f.x - w.y * f.y, w.x * f.y + w.y * f.x);
    }
    const __half2* s = srs + ((long)blk * nAnt + ant0) * K;
    for (int e = threadIdx.x; e < nA * K; e += blockDim.x) rows[e] = __half22float2(s[e]);
    __syncthreads();
    for (int o = threadIdx.x; o < nA * KP; o += blockDim.x) {
        const int a = o / KP, r = o % KP;   // r = ko*P + p
        const float2* row = rows + a * K;
        float re = 0.f, im = 0.f;
        for (int k = 0; k < K; k++) {
            const float2 t = taps[k * KP + r], x = row[k];
            re = fmaf(t.x, x.x, re);
            re = fmaf(-t.y, x.y, re);
            im = fmaf(t.x, x.y, im);
            im = fmaf(t.y, x.x, im);
        }
        const int ant = ant0 + a;
        if (TO_CHANNEL) {
            // H[sc = blk*K + ko][ant][layer = p], nLayers = P
            const int ko = r / P, p = r % P;
            float2* H = reinterpret_cast<float2*>(out);
            H[(((long)blk * K + ko) * nAnt + ant) * P + p] = make_float2(re, im);
        } else {
            __half2* H = reinterpret_cast<__half2*>(out);
            H[((long)blk * nAnt + ant) * KP + r] = __floats2half2_rn(re, im);
        }
    }
}

static int launch_srs(bool toChannel, void* out, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC,
                      int nAnt, int nBlocks, int K, int P, int F, cudaStream_t st) {
    if (!out || !SRS || !W || !FOCC || nAnt < 1 || nBlocks < 1 || K < 1 || K > 48 || P < 1 || P > 16 || F < 1)
        return AERIAL_ERR_INVALID_ARG;
    const size_t smem = sizeof(float2) * ((size_t)K * K * P + (size_t)kSrsAntPerCta * K);
    if (smem > 200 * 1024) return AERIAL_ERR_UNSUPPORTED;
    dim3 grid(nBlocks, (nAnt + kSrsAntPerCta - 1) / kSrsAntPerCta);
    if (toChannel) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(srs_filter_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        srs_filter_kernel<true><<<grid, 256, smem, st>>>((const __half2*)SRS, (const __half2*)W,
                                                         (const __half2*)FOCC, out, nAnt, K, P, F);
    } else {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(srs_filter_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        srs_filter_kernel<false><<<grid, 256, smem, st>>>((const __half2*)SRS, (const __half2*)W,
                                                          (const __half2*)FOCC, out, nAnt, K, P, F);
    }
    return launch_status();
}

}  // namespace aeq

using namespace aeq;

extern "C" int aerial_srs_filter(aerial_ch2* H_est, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC,
                                 int nAnt, int nBlocks, int K, int nPorts, int foccLen, void* stream) {
    return launch_srs(false, H_est, SRS, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen, to_stream(stream));
}

extern "C" int aerial_srs_to_channel(aerial_cf32* H, const aerial_ch2* SRS, const aerial_ch2* W,
                                     const aerial_ch2* FOCC, int nAnt, int nBlocks, int K, int nPorts, int foccLen,
                                     void* stream) {
    return launch_srs(true, H, SRS, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen, to_stream(stream));
}
