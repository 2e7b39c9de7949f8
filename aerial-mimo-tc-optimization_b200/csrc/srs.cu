// srs.cu -- SRS filter multiply (srsFilterMultiply of the reference,
// src/srs/srs_wmma_bench.cu:57-90 and :102-231):
//   H_est[blk][ant][k_out][p] = sum_k (W[k_out][k] * FOCC[p][k % F]) * SRS[blk][ant][k]
// The reference accumulates in FP16 (__hfma in V1, an FP16 accumulator in
// V2).  Here the sums run on the tensor cores with FP32 accumulation and the
// FP32 accuracy of a scalar FP32 sum; complex_conjmul (:43-47) computes the
// plain product despite its name, and the plain product is kept.
//
// Tensor-core form (mma.sync m16n8k16, FP16 operands, FP32 accumulate).  Per
// SRS block it is the complex GEMM out[ant][n] = sum_k S[ant][k] T[n][k] with
// n = k_out * P + p and taps T[n][k] = W[k_out][k] FOCC[p][k % F], embedded as
// a real GEMM:
//   A[ant][2k + r]   = (Re, Im) of S[ant][k]   -- the SRS row as stored, so a
//                                                thread's A register IS one
//                                                complex half2 sample
//   B[2k][2n] = Re T, B[2k+1][2n] = -Im T     -> column 2n   = Re out
//   B[2k][2n+1] = Im T, B[2k+1][2n+1] = Re T  -> column 2n+1 = Im out
// and a thread's accumulator pair (d0, d1) is one complex output.
// Precision: S is FP16 and exact as an operand.  Each tap, a product of two
// FP16 values formed in FP32, is split T = T_hi + T_lo into two FP16 parts
// (22 significant bits), and each k-step issues the two products S T_hi and
// S T_lo into the same FP32 accumulator.  FP16 x FP16 products are exact, so
// the result carries the error of an FP32 sum (about 2^-22 relative), not the
// FP16 rounding of the reference's taps.
//
// Output order.  Output tiles go in groups of four: tile jj of group q puts
// output n = 16 q + 4 c + jj in its complex column c, so after the four tiles
// of a group a lane holds four consecutive outputs of its antenna rows (one
// 16-byte store), and the four tiles give eight independent accumulators.
// Inside each k-step, K slot c (and c + 4) holds tap 2c (and 2c + 1), so a
// lane's two A registers of a row are one 8-byte load.  Both are column / row
// permutations of the same GEMM.
//
// Work split: the taps of one slice of groups are built once per CTA in
// shared memory, already in the B-fragment order (one 16-byte load per lane
// gives b0, b1 of T_hi and T_lo), so one build serves every SRS block the CTA
// visits.  Each warp takes (SRS block, 32-antenna) items in turn: its A
// fragments (two 16-antenna m-tiles, the whole K) are loaded once from global
// memory, then it sweeps the slice's groups.
#include <algorithm>

#include "common.cuh"

namespace aeq {

constexpr int kSrsWarps = 8;                 // warps per CTA
constexpr int kSrsMaxK = 48;                 // taps of the SRS filter (H_est layout)
constexpr int kChestMaxK = 96;               // pilots of the interpolation filter (channel layout)
constexpr int kSrsSliceBytes = 96 * 1024;    // taps of one slice of output groups
constexpr int kSrsGroupBytes = 4 * 32 * 16;  // one k-step of a group: 4 tiles x 32 lanes x 16 B

__device__ __forceinline__ void mma_f16(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                        uint32_t b1) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t h2bits(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// FP16 hi/lo parts of the pair (x, y): hi = rn(v), lo = rn(v - hi).
__device__ __forceinline__ void split_h2(float x, float y, uint32_t& hi, uint32_t& lo) {
    const __half2 h = __floats2half2_rn(x, y);
    const float2 hf = __half22float2(h);
    hi = h2bits(h);
    lo = h2bits(__floats2half2_rn(x - hf.x, y - hf.y));
}

// KS: k-steps of 8 complex taps (K <= 8 KS); MT: 16-antenna m-tiles per warp
// item (two up to 48 taps, one above, to bound the A registers).  K input
// taps per antenna, Ko filter outputs per block (Ko = K for the SRS filter).
// Grid: x = CTAs walking the (block, 16 MT-antenna) items, y = slices of NQ
// output groups (16 complex outputs per group).
template <int KS, int MT, bool TO_CHANNEL>
__global__ void __launch_bounds__(kSrsWarps * 32, 2) srs_filter_tc_kernel(const __half2* __restrict__ srs,
                                                                          const __half2* __restrict__ W,
                                                                          const __half2* __restrict__ focc,
                                                                          void* __restrict__ out, int nAnt,
                                                                          int nBlocks, int K, int Ko, int P, int F, int NQ) {
    extern __shared__ uint4 bfrag[];            // [group][kstep][tile][lane]: {b0 hi, b1 hi, b0 lo, b1 lo}
    const int N = Ko * P;                        // complex outputs per antenna
    const int nGroups = (N + 15) / 16;
    const int q0 = blockIdx.y * NQ;
    const int nq = min(NQ, nGroups - q0);
    for (int e = threadIdx.x; e < nq * KS * 128; e += blockDim.x) {
        const int l = e & 31, jj = (e >> 5) & 3, ks = (e >> 7) % KS, q = q0 + e / (128 * KS);
        const int g = l >> 2, c = l & 3;
        const int n = 16 * q + 4 * (g >> 1) + jj;
        uint32_t hi[2], lo[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = ks * 8 + 2 * c + h;    // K slot c + 4h
            float2 t = make_float2(0.f, 0.f);
            if (n < N && k < K) {
                const int ko = n / P, p = n % P;
                const float2 w = __half22float2(W[ko * K + k]);
                const float2 f = __half22float2(focc[p * F + (k % F)]);
                t = make_float2(w.x * f.x - w.y * f.y, w.x * f.y + w.y * f.x);
            }
            // even output column: (Re T, -Im T) -> Re out; odd: (Im T, Re T) -> Im out
            if (g & 1) split_h2(t.y, t.x, hi[h], lo[h]);
            else split_h2(t.x, -t.y, hi[h], lo[h]);
        }
        bfrag[e] = make_uint4(hi[0], hi[1], lo[0], lo[1]);
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, c = lane & 3;
    constexpr int kAntPerItem = 16 * MT;
    const int antGroups = (nAnt + kAntPerItem - 1) / kAntPerItem;
    const long items = (long)nBlocks * antGroups;
    const long nw = (long)gridDim.x * kSrsWarps;
    const uint32_t fb = (uint32_t)__cvta_generic_to_shared(bfrag) + lane * 16;
    const bool pairK = (K & 1) == 0;             // taps 2c, 2c + 1 of a row are one 8-byte load
    for (long it = (long)blockIdx.x * kSrsWarps + (threadIdx.x >> 5); it < items; it += nw) {
        const int blk = (int)(it / antGroups);
        const int ant0 = (int)(it - (long)blk * antGroups) * kAntPerItem;
        // A fragments: rows ant0 + 16 mt + g (+8 rr), taps 8 ks + 2c (+1)
        uint32_t a[MT][KS][4];
#pragma unroll
        for (int mt = 0; mt < MT; mt++) {
#pragma unroll
            for (int rr = 0; rr < 2; rr++) {
                const int ant = ant0 + 16 * mt + g + 8 * rr;
                const bool av = ant < nAnt;
                const __half2* row = srs + ((long)blk * nAnt + (av ? ant : 0)) * K;
#pragma unroll
                for (int ks = 0; ks < KS; ks++) {
                    const int k = ks * 8 + 2 * c;
                    uint32_t v0 = 0u, v1 = 0u;
                    if (av && k < K) {
                        if (pairK) {
                            const uint2 v = __ldg(reinterpret_cast<const uint2*>(row + k));
                            v0 = v.x;
                            v1 = v.y;
                        } else {
                            v0 = h2bits(__ldg(row + k));
                            if (k + 1 < K) v1 = h2bits(__ldg(row + k + 1));
                        }
                    }
                    a[mt][ks][rr] = v0;
                    a[mt][ks][rr + 2] = v1;
                }
            }
        }
        for (int q = 0; q < nq; q++) {
            float d[4][MT][4];
#pragma unroll
            for (int jj = 0; jj < 4; jj++)
#pragma unroll
                for (int mt = 0; mt < MT; mt++)
#pragma unroll
                    for (int r = 0; r < 4; r++) d[jj][mt][r] = 0.f;
#pragma unroll
            for (int ks = 0; ks < KS; ks++) {
#pragma unroll
                for (int jj = 0; jj < 4; jj++) {
                    uint4 b;
                    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n"
                                 : "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
                                 : "r"(fb + (uint32_t)(((q * KS + ks) * 4 + jj) * 512)));
#pragma unroll
                    for (int mt = 0; mt < MT; mt++) {
                        mma_f16(d[jj][mt], a[mt][ks][0], a[mt][ks][1], a[mt][ks][2], a[mt][ks][3], b.x, b.y);
                        mma_f16(d[jj][mt], a[mt][ks][0], a[mt][ks][1], a[mt][ks][2], a[mt][ks][3], b.z, b.w);
                    }
                }
            }
            // lane holds outputs n0 .. n0 + 3 of rows (mt, rr): (Re, Im) = d[jj][mt][2 rr], [2 rr + 1]
            const int n0 = 16 * (q0 + q) + 4 * c;
            if (n0 >= N) continue;
            const bool full = n0 + 3 < N;
#pragma unroll
            for (int mt = 0; mt < MT; mt++) {
#pragma unroll
                for (int rr = 0; rr < 2; rr++) {
                    const int ant = ant0 + 16 * mt + g + 8 * rr;
                    if (ant >= nAnt) continue;
                    if constexpr (TO_CHANNEL) {
                        // H[sc = blk*Ko + ko][ant][layer = p], nLayers = P
                        float2* H = reinterpret_cast<float2*>(out);
                        if (P == 4 && full) {
                            float2* dst = H + (((long)blk * Ko + n0 / 4) * nAnt + ant) * 4;
                            __stcs(reinterpret_cast<float4*>(dst),
                                   make_float4(d[0][mt][2 * rr], d[0][mt][2 * rr + 1], d[1][mt][2 * rr],
                                               d[1][mt][2 * rr + 1]));
                            __stcs(reinterpret_cast<float4*>(dst + 2),
                                   make_float4(d[2][mt][2 * rr], d[2][mt][2 * rr + 1], d[3][mt][2 * rr],
                                               d[3][mt][2 * rr + 1]));
                        } else {
#pragma unroll
                            for (int jj = 0; jj < 4; jj++) {
                                const int n = n0 + jj;
                                if (n < N)
                                    __stcs(H + (((long)blk * Ko + n / P) * nAnt + ant) * P + n % P,
                                           make_float2(d[jj][mt][2 * rr], d[jj][mt][2 * rr + 1]));
                            }
                        }
                    } else {
                        unsigned* H = reinterpret_cast<unsigned*>(out) + ((long)blk * nAnt + ant) * N + n0;
                        uint32_t v[4];
#pragma unroll
                        for (int jj = 0; jj < 4; jj++)
                            v[jj] = h2bits(__floats2half2_rn(d[jj][mt][2 * rr], d[jj][mt][2 * rr + 1]));
                        if (full && (N & 3) == 0) {
                            __stcs(reinterpret_cast<uint4*>(H), make_uint4(v[0], v[1], v[2], v[3]));
                        } else {
#pragma unroll
                            for (int jj = 0; jj < 4; jj++)
                                if (n0 + jj < N) __stcs(H + jj, v[jj]);
                        }
                    }
                }
            }
        }
    }
}

template <int KS, bool TO_CHANNEL>
static int launch_srs_tc(void* out, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC, int nAnt,
                         int nBlocks, int K, int Ko, int P, int F, cudaStream_t st) {
    constexpr int MT = KS <= 6 ? 2 : 1;
    auto kern = srs_filter_tc_kernel<KS, MT, TO_CHANNEL>;
    const int s = allow_max_smem<srs_filter_tc_kernel<KS, MT, TO_CHANNEL>>();
    if (s != AERIAL_OK) return s;
    const int nGroups = (Ko * P + 15) / 16;
    const int groupBytes = KS * kSrsGroupBytes;
    const int NQ = std::min(nGroups, kSrsSliceBytes / groupBytes);
    const int slices = (nGroups + NQ - 1) / NQ;
    const size_t smem = (size_t)NQ * groupBytes;
    int perSm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kSrsWarps * 32, smem);
    if (e != cudaSuccess) return (int)e;
    const long items = (long)nBlocks * ((nAnt + 16 * MT - 1) / (16 * MT));
    const long ctasForItems = (items + kSrsWarps - 1) / kSrsWarps;
    // enough CTAs to fill the GPU once per slice; each walks its share of items
    long gx = std::max(1L, (long)sm_count() * std::max(1, perSm) / slices);
    gx = std::min(gx, ctasForItems);
    dim3 grid((unsigned)gx, (unsigned)slices);
    kern<<<grid, kSrsWarps * 32, smem, st>>>((const __half2*)SRS, (const __half2*)W, (const __half2*)FOCC, out,
                                             nAnt, nBlocks, K, Ko, P, F, NQ);
    return launch_status();
}

// H_est layout (the SRS filter): up to 48 taps.
static int launch_srs_est(void* out, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC, int nAnt,
                          int nBlocks, int K, int P, int F, cudaStream_t st) {
    switch ((K + 7) / 8) {
        case 1: return launch_srs_tc<1, false>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        case 2: return launch_srs_tc<2, false>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        case 3: return launch_srs_tc<3, false>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        case 4: return launch_srs_tc<4, false>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        case 5: return launch_srs_tc<5, false>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        default: return launch_srs_tc<6, false>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
    }
}

// Channel layout H[blk*Ko + ko][ant][p]: up to 96 input taps.
static int launch_srs_chan(void* out, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC, int nAnt,
                           int nBlocks, int K, int Ko, int P, int F, cudaStream_t st) {
    switch ((K + 7) / 8) {
        case 1: return launch_srs_tc<1, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 2: return launch_srs_tc<2, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 3: return launch_srs_tc<3, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 4: return launch_srs_tc<4, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 5: return launch_srs_tc<5, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 6: return launch_srs_tc<6, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 7: return launch_srs_tc<7, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 8: return launch_srs_tc<8, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 9: return launch_srs_tc<9, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 10: return launch_srs_tc<10, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 11: return launch_srs_tc<11, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        default: return launch_srs_tc<12, true>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
    }
}

static bool srs_args_ok(const void* out, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC, int nAnt,
                        int nBlocks, int K, int maxK, int Ko, int P, int F) {
    return out && SRS && W && FOCC && nAnt >= 1 && nBlocks >= 1 && K >= 1 && K <= maxK && Ko >= 1 && Ko <= 4096 &&
           P >= 1 && P <= 16 && F >= 1;
}

}  // namespace aeq

using namespace aeq;

extern "C" int aerial_srs_filter(aerial_ch2* H_est, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC,
                                 int nAnt, int nBlocks, int K, int nPorts, int foccLen, void* stream) {
    if (!srs_args_ok(H_est, SRS, W, FOCC, nAnt, nBlocks, K, kSrsMaxK, K, nPorts, foccLen)) return AERIAL_ERR_INVALID_ARG;
    return launch_srs_est(H_est, SRS, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen, to_stream(stream));
}

extern "C" int aerial_srs_to_channel(aerial_cf32* H, const aerial_ch2* SRS, const aerial_ch2* W,
                                     const aerial_ch2* FOCC, int nAnt, int nBlocks, int K, int nPorts, int foccLen,
                                     void* stream) {
    if (!srs_args_ok(H, SRS, W, FOCC, nAnt, nBlocks, K, kSrsMaxK, K, nPorts, foccLen)) return AERIAL_ERR_INVALID_ARG;
    return launch_srs_chan(H, SRS, W, FOCC, nAnt, nBlocks, K, K, nPorts, foccLen, to_stream(stream));
}

extern "C" int aerial_chest_interp(aerial_cf32* H, const aerial_ch2* Yp, const aerial_ch2* Wf, const aerial_ch2* OCC,
                                   int nAnt, int nBlocks, int nPilot, int nOut, int nPorts, int occLen, void* stream) {
    if (!srs_args_ok(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, kChestMaxK, nOut, nPorts, occLen))
        return AERIAL_ERR_INVALID_ARG;
    return launch_srs_chan(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, nPorts, occLen, to_stream(stream));
}
