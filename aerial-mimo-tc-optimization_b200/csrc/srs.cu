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
#include <cstdint>
#include <mutex>
#include <utility>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"

namespace aeq {

constexpr int kSrsWarps = 8;                 // warps per CTA
constexpr int kSrsMaxK = 48;                 // taps of the SRS filter (H_est layout)
constexpr int kChestMaxK = 96;               // pilots of the interpolation filter (channel layout)
constexpr int kSrsSliceBytes = 96 * 1024;    // taps of one slice of output groups
constexpr int kSrsGroupBytes = 4 * 32 * 16;  // one k-step of a group: 4 tiles x 32 lanes x 16 B

// Output layouts of the filter kernels: the SRS filter's FP16
// H_est[blk][ant][k_out][p]; the PUSCH channel H[blk*Ko + k_out][ant][p] as
// complex64 (the equalizer's drop-in format) or as complex half (its FP16 I/O
// format).
enum OutLayout : int { kOutEst16 = 0, kOutChan32 = 1, kOutChan16 = 2 };

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
template <int KS, int MT, int OUTL>
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
                    if constexpr (OUTL == kOutChan16) {
                        // H[sc = blk*Ko + ko][ant][layer = p] as complex half
                        uint32_t* H = reinterpret_cast<uint32_t*>(out);
                        uint32_t v[4];
#pragma unroll
                        for (int jj = 0; jj < 4; jj++)
                            v[jj] = h2bits(__floats2half2_rn(d[jj][mt][2 * rr], d[jj][mt][2 * rr + 1]));
                        if (P == 4 && full && (reinterpret_cast<uintptr_t>(H) & 15) == 0) {
                            __stcs(reinterpret_cast<uint4*>(H + (((long)blk * Ko + n0 / 4) * nAnt + ant) * 4),
                                   make_uint4(v[0], v[1], v[2], v[3]));
                        } else {
#pragma unroll
                            for (int jj = 0; jj < 4; jj++) {
                                const int n = n0 + jj;
                                if (n < N) __stcs(H + (((long)blk * Ko + n / P) * nAnt + ant) * P + n % P, v[jj]);
                            }
                        }
                    } else if constexpr (OUTL == kOutChan32) {
                        // H[sc = blk*Ko + ko][ant][layer = p], nLayers = P
                        float2* H = reinterpret_cast<float2*>(out);
                        if (P == 4 && full && (reinterpret_cast<uintptr_t>(H) & 15) == 0) {
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
                        if (full && (N & 3) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0) {
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

// ---------------------------------------------------------------------------
// The interpolation filter on the 5th-generation tensor cores (tcgen05).
//
// The filter taps are shared by every block, so blocks stack along M with no
// wasted products: one GEMM C[m][n] = sum_k A[m][k] B[k][n] with m = (block,
// antenna) rows of the pilot input as stored (row-major, K = (pilot, re/im)
// interleaved FP16: K-major), and n = (output subcarrier, port, re/im).
//   - A tiles of 128 rows x 64 K arrive by TMA with the 128-byte swizzle, the
//     canonical K-major layout of the UMMA shared-memory descriptor.
//   - B (taps, real-embedded as in the mma.sync kernel, split hi/lo) is built
//     once per CTA in shared memory in the same swizzled layout, for the
//     CTA's tile of 128 real output columns (64 complex outputs).
//   - One elected thread issues tcgen05.mma (M = 128, N = NTL = 128 or 192
//     real columns, K = 16, FP16 operands, FP32 accumulate in TMEM): the hi
//     products then the lo products into one accumulator.  Two TMEM
//     accumulators let the epilogue of one M tile overlap the MMAs of the
//     next.
//   - Warps 2-9 read the accumulator rows with tcgen05.ld (one TMEM lane =
//     one (block, antenna) row per thread; two warps per TMEM sub-partition,
//     each half of the tile's columns) and store the channel layout; for 4
//     ports a thread's 4 consecutive outputs are one 256-bit store and a
//     warp's 32 antennas are 1 KB contiguous per instruction.  (Two 16-byte
//     stores per thread left every 32-byte sector of a request half written:
//     ncu showed 32 sectors per request and L1 at 76 %.  Staging the outputs
//     in shared memory for TMA tensor stores measured slower than these
//     direct stores, with 64-byte, 32-byte or 1 KB box rows.)
// Warp roles: 0 = TMA producer, 1 = TMEM owner + MMA issuer, 2-9 = epilogue.
// Every wait is bounded: on a timeout the CTA raises an abort flag, every
// role leaves its loop, and the kernel still frees its TMEM and returns
// (counted in g_umma_timeouts).
// ---------------------------------------------------------------------------
constexpr int kUmmaM = 128;                  // rows per M tile (TMEM lanes)
constexpr int kUmmaN = 128;                  // real output columns per CTA tile (192 where shared memory allows)
constexpr int kUmmaKB = 64;                  // K elements per swizzle atom (128 bytes of FP16)
constexpr int kUmmaAtomBytes = kUmmaM * 128; // one 128 x 64 FP16 atom column block: 16 KB
constexpr int kUmmaEpiWarps = 8;            // two per TMEM sub-partition, each half of the columns
constexpr int kUmmaThreads = 64 + 32 * kUmmaEpiWarps;
constexpr long kUmmaWaitLimit = 1L << 22;    // mbarrier polls before a wait gives up

__device__ unsigned g_umma_timeouts;         // waits that gave up (diagnostic; stays 0)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
    for (long i = 0; i < kUmmaWaitLimit; i++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 1023) == 1023 && *abort) return false;
    }
    *abort = 1;
    atomicAdd(&g_umma_timeouts, 1u);
    return false;
}

// UMMA shared-memory descriptor, K-major, 128-byte swizzle: start address,
// LBO = 16 B (unused by swizzled K-major), SBO = 1024 B (8 rows of 128 B),
// version 1, base offset 0, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// Instruction descriptor, kind::f16: FP32 accumulator, FP16 A and B, both
// K-major, N = n, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kUmmaM >> 4) << 24);
}
// TMEM columns for two accumulators of n columns (a power of two >= 32).
__host__ __device__ constexpr int umma_tmem_cols(int n) { return 2 * n <= 256 ? 256 : 512; }

// Byte offset of FP16 element (row r, k) in a K-major 128-byte-swizzled atom
// column block of 128-byte rows (k < 64): 16-byte chunk index XOR (r mod 8).
__device__ __forceinline__ uint32_t sw128_off(int r, int k) {
    return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 3) ^ r) & 7) << 4) + (k & 7) * 2);
}

// KB: 64-element K atoms (2 nPilot <= 64 KB); NTL: real output columns per
// tile (NTL / 2 complex outputs); OUTL: the output layout (OutLayout).
// nSrs input symbols (1, 2 or 4; tmA is [nSrs][rows][2 nPilot]) give the
// average of their filter outputs: the K loop runs over every symbol's A
// tile into one FP32 accumulator, with the taps scaled by 1/nSrs (exact for
// these counts), so (1/S) sum_s f(in_s) is one GEMM with K extended over S.
template <int KB, int NTL, int OUTL>
__global__ void __launch_bounds__(kUmmaThreads, 1) chest_umma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                                      const __half2* __restrict__ Wf,
                                                                      const __half2* __restrict__ occ,
                                                                      void* __restrict__ out, int nAnt, int nBlocks,
                                                                      int nPilot, int nOut, int P, int F, int nSrs) {
    extern __shared__ __align__(1024) uint8_t usm_raw[];
    // 128-byte swizzle atoms must start on 1024-byte boundaries of the shared window
    uint8_t* usm = usm_raw + ((1024u - (smem_u32(usm_raw) & 1023u)) & 1023u);
    // layout: A stages [2][nSrs x KB atoms of 128 rows] | B [hi, lo][KB atoms of NTL rows] | barriers | TMEM slot
    constexpr int kBAtom = NTL * 128;             // bytes of one B atom column block
    constexpr int kTCols = umma_tmem_cols(NTL);
    const uint32_t aStage = (uint32_t)nSrs * KB * kUmmaAtomBytes;
    uint8_t* sA = usm;
    uint8_t* sB = usm + 2 * aStage;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sB + 2 * KB * kBAtom);
    // bars: full[2], empty[2], tfull[2], tempty[2]
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 8);
    volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int N = nOut * P;                       // complex outputs per row
    const int nt = blockIdx.y;                    // tile of NTL / 2 complex outputs
    const long M = (long)nBlocks * nAnt;
    const long nMT = (M + kUmmaM - 1) / kUmmaM;

    if (threadIdx.x == 0) {
        for (int b = 0; b < 8; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bars + b)),
                         "r"(b >= 6 ? kUmmaEpiWarps : 1));   // tempty: one arrival per epilogue warp
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(kTCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    // B's K columns past 2 nPilot inside the last atom must read as zero
    for (int e = threadIdx.x; e < 2 * KB * kBAtom / 16; e += blockDim.x)
        reinterpret_cast<uint4*>(sB)[e] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    // B tile: rows r = 2 j + (re/im output) for complex output n = NTL/2 nt + j,
    // K columns 2 kc + (re/im input); (Re T, -Im T) / (Im T, Re T) pairs.
    for (int e = threadIdx.x; e < (NTL / 2) * nPilot; e += blockDim.x) {
        const int j = e / nPilot, kc = e - j * nPilot;
        const int n = (NTL / 2) * nt + j;
        float2 t = make_float2(0.f, 0.f);
        if (n < N) {
            const float2 w = __half22float2(Wf[(n / P) * nPilot + kc]);
            const float2 f = __half22float2(occ[(n % P) * F + (kc % F)]);
            t = make_float2(w.x * f.x - w.y * f.y, w.x * f.y + w.y * f.x);
            if (nSrs > 1) t = make_float2(t.x * (1.f / nSrs), t.y * (1.f / nSrs));   // a power of two: exact
        }
        uint32_t hi0, lo0, hi1, lo1;
        split_h2(t.x, -t.y, hi0, lo0);           // row 2j: Re out
        split_h2(t.y, t.x, hi1, lo1);            // row 2j+1: Im out
        const int k = 2 * kc, kb = k >> 6, kin = k & 63;
        uint8_t* bh = sB + kb * kBAtom;
        uint8_t* bl = sB + (KB + kb) * kBAtom;
        *reinterpret_cast<uint32_t*>(bh + sw128_off(2 * j, kin)) = hi0;
        *reinterpret_cast<uint32_t*>(bl + sw128_off(2 * j, kin)) = lo0;
        *reinterpret_cast<uint32_t*>(bh + sw128_off(2 * j + 1, kin)) = hi1;
        *reinterpret_cast<uint32_t*>(bl + sw128_off(2 * j + 1, kin)) = lo1;
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tbase = *tslot;

    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + 2), tfull0 = smem_u32(bars + 4),
                   tempty0 = smem_u32(bars + 6);
    if (warp == 0) {
        if (lane == 0) {
            long i = 0;
            for (long mt = blockIdx.x; mt < nMT && !*abort; mt += gridDim.x, i++) {
                const int s = (int)(i & 1);
                if (!mbar_wait(empty0 + 8 * s, (uint32_t)(((i >> 1) & 1) ^ 1), abort)) break;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(full0 + 8 * s),
                             "r"(aStage)
                             : "memory");
                for (int q = 0; q < nSrs; q++)
#pragma unroll
                    for (int kb = 0; kb < KB; kb++)
                        asm volatile(
                            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                            "[%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
                                smem_u32(sA + s * aStage + (uint32_t)(q * KB + kb) * kUmmaAtomBytes)),
                            "l"(reinterpret_cast<uint64_t>(&tmA)), "r"(kb * kUmmaKB), "r"((int)(mt * kUmmaM)), "r"(q),
                            "r"(full0 + 8 * s)
                            : "memory");
            }
            // leave no copy in flight: the last two stages' loads have landed
            for (long d = (i > 2 ? i - 2 : 0); d < i; d++) mbar_wait(full0 + 8 * (d & 1), (uint32_t)((d >> 1) & 1), abort);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            long i = 0;
            for (long mt = blockIdx.x; mt < nMT && !*abort; mt += gridDim.x, i++) {
                const int s = (int)(i & 1), a = (int)(i & 1);
                const uint32_t ph = (uint32_t)((i >> 1) & 1);
                if (!mbar_wait(tempty0 + 8 * a, ph ^ 1, abort)) break;
                if (!mbar_wait(full0 + 8 * s, ph, abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t dt = tbase + (uint32_t)(a * NTL);
                const uint32_t a0 = smem_u32(sA + s * aStage);
                const uint32_t b0 = smem_u32(sB);
#pragma unroll
                for (int part = 0; part < 2; part++) {
                    for (int q = 0; q < nSrs; q++) {
#pragma unroll
                        for (int kb = 0; kb < KB; kb++) {
#pragma unroll
                            for (int kk = 0; kk < kUmmaKB / 16; kk++) {
                                if (kb * kUmmaKB + kk * 16 >= 2 * nPilot) break;   // K steps past the pilots
                                const uint64_t ad =
                                    umma_desc_sw128(a0 + (uint32_t)(q * KB + kb) * kUmmaAtomBytes + kk * 32);
                                const uint64_t bd = umma_desc_sw128(b0 + (part * KB + kb) * kBAtom + kk * 32);
                                const uint32_t acc = (part | q | kb | kk) ? 1u : 0u;
                                asm volatile(
                                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dt),
                                    "l"(ad), "l"(bd), "r"(umma_idesc(NTL)), "r"(acc)
                                    : "memory");
                            }
                        }
                    }
                }
                // stage s is free and accumulator a is full once these MMAs complete
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 empty0 + 8 * s)
                             : "memory");
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 tfull0 + 8 * a)
                             : "memory");
            }
        }
    } else {
        // epilogue: TMEM sub-partition (warp mod 4) holds rows 32 (warp mod 4) .. +31
        const int sp = warp & 3;
        const int row = sp * 32 + lane;
        long i = 0;
        for (long mt = blockIdx.x; mt < nMT && !*abort; mt += gridDim.x, i++) {
            const int a = (int)(i & 1);
            if (!mbar_wait(tfull0 + 8 * a, (uint32_t)((i >> 1) & 1), abort)) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const long m = mt * kUmmaM + row;
            const bool mv = m < M;
            const int blk = mv ? (int)(m / nAnt) : 0;
            const int ant = mv ? (int)(m - (long)blk * nAnt) : 0;
#pragma unroll 1
            for (int c = ((warp - 2) >> 2) * (NTL / 64); c < (((warp - 2) >> 2) + 1) * (NTL / 64); c++) {
                uint32_t v[32];
                const uint32_t ta = tbase + ((uint32_t)(sp * 32) << 16) + (uint32_t)(a * NTL + c * 32);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                    "[%32];\n"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(ta));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                const int nb = (NTL / 2) * nt + 16 * c;  // complex outputs nb .. nb + 15 of this row
                if (!mv) continue;
                if constexpr (OUTL == kOutChan16) {
                    // channel as complex half: a subcarrier's 4 ports are one 16-byte
                    // store, a warp's 32 antennas 512 contiguous bytes.  (Pairing
                    // lanes by a shuffle into 256-bit stores measured no faster.)
                    uint32_t h[16];
#pragma unroll
                    for (int jj = 0; jj < 16; jj++)
                        h[jj] = h2bits(__floats2half2_rn(__uint_as_float(v[2 * jj]), __uint_as_float(v[2 * jj + 1])));
                    uint32_t* H = reinterpret_cast<uint32_t*>(out);
                    if (P == 4 && (reinterpret_cast<uintptr_t>(H) & 15) == 0) {
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            if (nb + 4 * q >= N) break;
                            __stcs(reinterpret_cast<uint4*>(H + (((long)blk * nOut + (nb >> 2) + q) * nAnt + ant) * 4),
                                   make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]));
                        }
                    } else {
#pragma unroll
                        for (int jj = 0; jj < 16; jj++) {
                            const int n = nb + jj;
                            if (n < N) __stcs(H + (((long)blk * nOut + n / P) * nAnt + ant) * P + n % P, h[jj]);
                        }
                    }
                    continue;
                }
                if constexpr (OUTL == kOutEst16) {
                    // H_est[blk][ant][n]: the row's 16 outputs are 64 contiguous bytes of half2
                    uint32_t h[16];
#pragma unroll
                    for (int jj = 0; jj < 16; jj++)
                        h[jj] = h2bits(__floats2half2_rn(__uint_as_float(v[2 * jj]), __uint_as_float(v[2 * jj + 1])));
                    uint32_t* dst = reinterpret_cast<uint32_t*>(out) + m * N + nb;
                    if (nb + 16 <= N && (N & 7) == 0 && (reinterpret_cast<uintptr_t>(out) & 31) == 0) {
#pragma unroll
                        for (int hh = 0; hh < 2; hh++)
                            asm volatile("st.global.cs.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"l"(dst + 8 * hh),
                                         "r"(h[8 * hh]), "r"(h[8 * hh + 1]), "r"(h[8 * hh + 2]), "r"(h[8 * hh + 3]),
                                         "r"(h[8 * hh + 4]), "r"(h[8 * hh + 5]), "r"(h[8 * hh + 6]), "r"(h[8 * hh + 7])
                                         : "memory");
                    } else {
#pragma unroll
                        for (int jj = 0; jj < 16; jj++)
                            if (nb + jj < N) __stcs(dst + jj, h[jj]);
                    }
                    continue;
                }
                float2* H = reinterpret_cast<float2*>(out);
                if (P == 4 && (reinterpret_cast<uintptr_t>(H) & 31) == 0) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        if (nb + 4 * q >= N) break;
                        float2* dst = H + (((long)blk * nOut + (nb >> 2) + q) * nAnt + ant) * 4;
                        asm volatile("st.global.cs.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"l"(dst),
                                     "r"(v[8 * q]), "r"(v[8 * q + 1]), "r"(v[8 * q + 2]), "r"(v[8 * q + 3]),
                                     "r"(v[8 * q + 4]), "r"(v[8 * q + 5]), "r"(v[8 * q + 6]), "r"(v[8 * q + 7])
                                     : "memory");
                    }
                } else {
#pragma unroll
                    for (int jj = 0; jj < 16; jj++) {
                        const int n = nb + jj;
                        if (n < N)
                            __stcs(H + (((long)blk * nOut + n / P) * nAnt + ant) * P + n % P,
                                   make_float2(__uint_as_float(v[2 * jj]), __uint_as_float(v[2 * jj + 1])));
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(tempty0 + 8 * a) : "memory");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(kTCols));
}

// cuTensorMapEncodeTiled from the driver, looked up once.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Shapes the tcgen05 kernel takes: pilot rows whose byte stride (4 nPilot)
// is a multiple of 16, up to 96 pilots, from a 16-byte aligned array.  The
// tensor map is encoded per call; a shape it rejects falls back to the
// mma.sync kernel.
static bool chest_umma_ok(const aerial_ch2* Yp, int nPilot, long rows) {
    // TMA row coordinates are 32-bit: more rows take the mma.sync kernel
    return nPilot % 4 == 0 && nPilot <= 96 && (reinterpret_cast<uintptr_t>(Yp) & 15) == 0 &&
           rows <= (long)INT32_MAX - kUmmaM;
}

template <int KB, int NTL, int OUTL>
static int launch_chest_umma(void* out, const aerial_ch2* Yp, const aerial_ch2* Wf, const aerial_ch2* OCC, int nAnt,
                             int nBlocks, int nPilot, int nOut, int P, int F, int nSrs, cudaStream_t st) {
    auto enc = tensor_map_encoder();
    if (!enc) return AERIAL_ERR_UNSUPPORTED;
    const long M = (long)nBlocks * nAnt;
    // A stages (nSrs x KB atoms each) + B + barriers, TMEM slot, abort flag
    // and the 1024-byte alignment slack; at least 120 KB so one CTA (its TMEM
    // columns) runs per SM
    const size_t smem = std::max<size_t>((size_t)2 * nSrs * KB * kUmmaAtomBytes + (size_t)2 * KB * NTL * 128 +
                                             8 * sizeof(uint64_t) + 16 + 1024,
                                         120 * 1024);
    if (smem > (size_t)kMaxSmemPerCta) return AERIAL_ERR_UNSUPPORTED;
    CUtensorMap tm;
    // [nSrs][M rows][2 nPilot]: K extent 2 nPilot; a 64-element box past it
    // (nPilot < 32 KB) reads zeros
    const cuuint64_t dims[3] = {(cuuint64_t)(2 * nPilot), (cuuint64_t)M, (cuuint64_t)nSrs};
    const cuuint64_t strides[2] = {(cuuint64_t)(4 * nPilot), (cuuint64_t)M * 4 * nPilot};
    const cuuint32_t box[3] = {(cuuint32_t)kUmmaKB, (cuuint32_t)kUmmaM, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<aerial_ch2*>(Yp), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return AERIAL_ERR_UNSUPPORTED;
    const int s = allow_max_smem<chest_umma_kernel<KB, NTL, OUTL>>();
    if (s != AERIAL_OK) return s;
    const int nNT = (2 * nOut * P + NTL - 1) / NTL;
    const long nMT = (M + kUmmaM - 1) / kUmmaM;
    long gx = std::max(1L, (long)sm_count() / nNT);
    gx = std::min(gx, nMT);
    dim3 grid((unsigned)gx, (unsigned)nNT);
    chest_umma_kernel<KB, NTL, OUTL><<<grid, kUmmaThreads, smem, st>>>(tm, (const __half2*)Wf, (const __half2*)OCC, out,
                                                                   nAnt, nBlocks, nPilot, nOut, P, F, nSrs);
    return launch_status();
}

// The filter on tcgen05 when the shape allows it; AERIAL_ERR_UNSUPPORTED
// (nothing launched) otherwise, and the caller takes the mma.sync kernel.
// nSrs > 1 averages that many consecutive input symbols.
template <int OUTL>
static int try_chest_umma(void* out, const aerial_ch2* Yp, const aerial_ch2* Wf, const aerial_ch2* OCC, int nAnt,
                          int nBlocks, int nPilot, int nOut, int P, int F, cudaStream_t st, int nSrs = 1) {
    if (!chest_umma_ok(Yp, nPilot, (long)nBlocks * nAnt)) return AERIAL_ERR_UNSUPPORTED;
    // 192-column tiles where more than 128 real output columns exist and the
    // operands fit (up to 64 pilots); 128 otherwise
    const bool wide = 2 * nOut * P > kUmmaN && nPilot <= 64;
    switch ((nPilot + 31) / 32) {
        case 1:
            return wide ? launch_chest_umma<1, 192, OUTL>(out, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, P, F, nSrs, st)
                        : launch_chest_umma<1, 128, OUTL>(out, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, P, F, nSrs, st);
        case 2:
            return wide ? launch_chest_umma<2, 192, OUTL>(out, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, P, F, nSrs, st)
                        : launch_chest_umma<2, 128, OUTL>(out, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, P, F, nSrs, st);
        default: return launch_chest_umma<3, 128, OUTL>(out, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, P, F, nSrs, st);
    }
}

template <int KS, int OUTL>
static int launch_srs_tc(void* out, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC, int nAnt,
                         int nBlocks, int K, int Ko, int P, int F, cudaStream_t st) {
    constexpr int MT = KS <= 6 ? 2 : 1;
    auto kern = srs_filter_tc_kernel<KS, MT, OUTL>;
    const int s = allow_max_smem<srs_filter_tc_kernel<KS, MT, OUTL>>();
    if (s != AERIAL_OK) return s;
    const int nGroups = (Ko * P + 15) / 16;
    const int groupBytes = KS * kSrsGroupBytes;
    const int NQ = std::min(nGroups, kSrsSliceBytes / groupBytes);
    const int slices = (nGroups + NQ - 1) / NQ;
    const size_t smem = (size_t)NQ * groupBytes;
    int perSm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kSrsWarps * 32, smem);
    if (e != cudaSuccess) return rt_status(e);
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
        case 1: return launch_srs_tc<1, kOutEst16>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        case 2: return launch_srs_tc<2, kOutEst16>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        case 3: return launch_srs_tc<3, kOutEst16>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        case 4: return launch_srs_tc<4, kOutEst16>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        case 5: return launch_srs_tc<5, kOutEst16>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
        default: return launch_srs_tc<6, kOutEst16>(out, SRS, W, FOCC, nAnt, nBlocks, K, K, P, F, st);
    }
}

// Channel layout H[blk*Ko + ko][ant][p] (OUTL: complex64 or complex half): up
// to 96 input taps.
template <int OUTL>
static int launch_srs_chan(void* out, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC, int nAnt,
                           int nBlocks, int K, int Ko, int P, int F, cudaStream_t st) {
    switch ((K + 7) / 8) {
        case 1: return launch_srs_tc<1, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 2: return launch_srs_tc<2, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 3: return launch_srs_tc<3, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 4: return launch_srs_tc<4, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 5: return launch_srs_tc<5, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 6: return launch_srs_tc<6, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 7: return launch_srs_tc<7, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 8: return launch_srs_tc<8, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 9: return launch_srs_tc<9, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 10: return launch_srs_tc<10, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        case 11: return launch_srs_tc<11, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
        default: return launch_srs_tc<12, OUTL>(out, SRS, W, FOCC, nAnt, nBlocks, K, Ko, P, F, st);
    }
}

static bool srs_args_ok(const void* out, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC, int nAnt,
                        int nBlocks, int K, int maxK, int Ko, int P, int F) {
    return out && SRS && W && FOCC && nAnt >= 1 && nBlocks >= 1 && K >= 1 && K <= maxK && Ko >= 1 && Ko <= 4096 &&
           P >= 1 && P <= 16 && F >= 1;
}

}  // namespace aeq

using namespace aeq;

// Bounded waits of the tcgen05 filter kernel that gave up on the current
// device (the kernel then leaves its loops, frees its TMEM and returns).
extern "C" int aerial_kernel_timeouts(unsigned int* count) {
    if (!count) return AERIAL_ERR_INVALID_ARG;
    const cudaError_t e = cudaMemcpyFromSymbol(count, g_umma_timeouts, sizeof(unsigned int));
    return rt_status(e);
}

extern "C" int aerial_srs_filter(aerial_ch2* H_est, const aerial_ch2* SRS, const aerial_ch2* W, const aerial_ch2* FOCC,
                                 int nAnt, int nBlocks, int K, int nPorts, int foccLen, void* stream) {
    if (!srs_args_ok(H_est, SRS, W, FOCC, nAnt, nBlocks, K, kSrsMaxK, K, nPorts, foccLen)) return AERIAL_ERR_INVALID_ARG;
    const int r = try_chest_umma<kOutEst16>(H_est, SRS, W, FOCC, nAnt, nBlocks, K, K, nPorts, foccLen, to_stream(stream));
    if (r != AERIAL_ERR_UNSUPPORTED) return r;
    return launch_srs_est(H_est, SRS, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen, to_stream(stream));
}

extern "C" int aerial_srs_to_channel(aerial_cf32* H, const aerial_ch2* SRS, const aerial_ch2* W,
                                     const aerial_ch2* FOCC, int nAnt, int nBlocks, int K, int nPorts, int foccLen,
                                     void* stream) {
    if (!srs_args_ok(H, SRS, W, FOCC, nAnt, nBlocks, K, kSrsMaxK, K, nPorts, foccLen)) return AERIAL_ERR_INVALID_ARG;
    const int r = try_chest_umma<kOutChan32>(H, SRS, W, FOCC, nAnt, nBlocks, K, K, nPorts, foccLen, to_stream(stream));
    if (r != AERIAL_ERR_UNSUPPORTED) return r;
    return launch_srs_chan<kOutChan32>(H, SRS, W, FOCC, nAnt, nBlocks, K, K, nPorts, foccLen, to_stream(stream));
}

extern "C" int aerial_srs_to_channel_avg(aerial_cf32* H, const aerial_ch2* SRS, int nSrsSym, const aerial_ch2* W,
                                         const aerial_ch2* FOCC, int nAnt, int nBlocks, int K, int nPorts, int foccLen,
                                         void* stream) {
    if (nSrsSym != 1 && nSrsSym != 2 && nSrsSym != 4) return AERIAL_ERR_INVALID_ARG;
    if (nSrsSym == 1) return aerial_srs_to_channel(H, SRS, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen, stream);
    if (!srs_args_ok(H, SRS, W, FOCC, nAnt, nBlocks, K, kSrsMaxK, K, nPorts, foccLen)) return AERIAL_ERR_INVALID_ARG;
    // the average runs inside the tcgen05 kernel's K loop only
    return try_chest_umma<kOutChan32>(H, SRS, W, FOCC, nAnt, nBlocks, K, K, nPorts, foccLen, to_stream(stream),
                                      nSrsSym);
}

extern "C" int aerial_chest_interp(aerial_cf32* H, const aerial_ch2* Yp, const aerial_ch2* Wf, const aerial_ch2* OCC,
                                   int nAnt, int nBlocks, int nPilot, int nOut, int nPorts, int occLen, void* stream) {
    if (!srs_args_ok(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, kChestMaxK, nOut, nPorts, occLen))
        return AERIAL_ERR_INVALID_ARG;
    const int r = try_chest_umma<kOutChan32>(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, nPorts, occLen,
                                             to_stream(stream));
    if (r != AERIAL_ERR_UNSUPPORTED) return r;
    return launch_srs_chan<kOutChan32>(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, nPorts, occLen, to_stream(stream));
}

extern "C" int aerial_chest_interp_h(aerial_ch2* H, const aerial_ch2* Yp, const aerial_ch2* Wf, const aerial_ch2* OCC,
                                     int nAnt, int nBlocks, int nPilot, int nOut, int nPorts, int occLen,
                                     void* stream) {
    if (!srs_args_ok(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, kChestMaxK, nOut, nPorts, occLen))
        return AERIAL_ERR_INVALID_ARG;
    const int r = try_chest_umma<kOutChan16>(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, nPorts, occLen,
                                             to_stream(stream));
    if (r != AERIAL_ERR_UNSUPPORTED) return r;
    return launch_srs_chan<kOutChan16>(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, nPorts, occLen, to_stream(stream));
}

namespace aeq {

// Load every filter-kernel instantiation on the current device and raise its
// shared-memory limit (aerial_prepare): the first launch of a kernel
// otherwise pays the driver's lazy module loading, milliseconds inside a
// serving loop's first SRS update.
template <int KS, int OUTL>
static int prepare_srs_tc() {
    constexpr int MT = KS <= 6 ? 2 : 1;
    cudaFuncAttributes at;
    const cudaError_t e = cudaFuncGetAttributes(&at, srs_filter_tc_kernel<KS, MT, OUTL>);
    return e == cudaSuccess ? allow_max_smem<srs_filter_tc_kernel<KS, MT, OUTL>>() : rt_status(e);
}
template <int OUTL, int... KS>
static int prepare_srs_tc_all(std::integer_sequence<int, KS...>) {
    int s = AERIAL_OK;
    ((s = s ? s : prepare_srs_tc<KS + 1, OUTL>()), ...);
    return s;
}
template <int KB, int NTL, int OUTL>
static int prepare_umma() {
    cudaFuncAttributes at;
    const cudaError_t e = cudaFuncGetAttributes(&at, chest_umma_kernel<KB, NTL, OUTL>);
    return e == cudaSuccess ? allow_max_smem<chest_umma_kernel<KB, NTL, OUTL>>() : rt_status(e);
}
template <int OUTL>
static int prepare_umma_all() {
    int s = prepare_umma<1, 128, OUTL>();
    if (!s) s = prepare_umma<1, 192, OUTL>();
    if (!s) s = prepare_umma<2, 128, OUTL>();
    if (!s) s = prepare_umma<2, 192, OUTL>();
    if (!s) s = prepare_umma<3, 128, OUTL>();
    return s;
}

int prepare_srs_kernels() {
    int s = prepare_umma_all<kOutEst16>();
    if (!s) s = prepare_umma_all<kOutChan32>();
    if (!s) s = prepare_umma_all<kOutChan16>();
    if (!s) s = prepare_srs_tc_all<kOutEst16>(std::make_integer_sequence<int, 6>{});
    if (!s) s = prepare_srs_tc_all<kOutChan32>(std::make_integer_sequence<int, 12>{});
    if (!s) s = prepare_srs_tc_all<kOutChan16>(std::make_integer_sequence<int, 12>{});
    return s;
}

}  // namespace aeq
