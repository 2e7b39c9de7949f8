// fused.cu -- the fused PUSCH equalization kernel: Gram + matched filter on
// the tensor cores, FP32 MMSE solve (LDL^H elimination with the inverse
// accumulated in the same sweep), unbiasing and max-log LLR, in
// one persistent launch over any mix of cells.  Only H and Y_rx are read
// from HBM and only LLRs (optionally Y_eq) are written; G, C and Y_eq stay in
// registers / shared memory.
//
// Formulation (per subcarrier, L layers, A antennas, S symbols):
//   G = H^H H + s2 I          (L x L, Hermitian)
//   Z = H^H Y^T               (L x S, the matched filter)
//   X = G^-1 Z                (= C Y^T with C = G^-1 H^H, C never formed)
//   mu_l = 1 - s2 (G^-1)_ll ; Y_eq = X / mu ; noiseInv_l = mu_l / (s2 (G^-1)_ll)
// This is algebraically the reference chain gram -> solve -> coef_apply
// (src/aerial_bottleneck.cu:56-80, src/aerial_coef_wmma.cu:71-104) followed by
// computePamLlr (src/llr/aerial_llr_v3.cu:84-108); it replaces the L x A
// coefficient matrix by an L x S right-hand side (S = 11 << A = 64).
//
// Tensor-core mapping (mma.sync m16n8k16, FP32 accumulate).  A complex GEMM
// out[r][n] = sum_k conj(H[k][r]) B[k][n] is embedded as a real GEMM with
//   A_emb rows 0..7 = (Re, Im) pairs of H[k][r]       -> Re out
//   A_emb rows 8..15 = (-Im, Re) pairs of H[k][r]     -> Im out
//   B_emb = (Re, Im) pairs of B[k][n]
// and the K index interleaving (k, re/im).  With that choice a thread's A
// fragment register IS the complex tap H[k][layer] packed as a half2 and its
// B fragment register IS B[k][n] packed, so operands go from global memory
// to registers with no shared-memory staging or shuffles.  For the Gram
// n-tile B = H, i.e. the same registers as A.  Thread (g = lane/4, c = lane%4)
// covers antennas 8j+2c and 8j+2c+1 of k-step j (the K order is permuted
// inside each k-step; A and B use the same permutation).
#include <cstdlib>

#include "common.cuh"

namespace aeq {

constexpr int kMaxCells = AERIAL_MAX_CELLS;

// Subcarriers per group: GS = min(32 / LT, cap).  32 / LT fills every lane
// of the FP32 solve and of the LLR epilogue (LT lanes per subcarrier); a
// smaller cap shortens each group's operand pass (GS x chunks items), which
// an uneven batch needs so that no warp is left with a few long groups: on
// the uneven 16-cell batch a cap of 4 (idle solve lanes on 1-, 2- and
// 4-layer tiles) measured 54.3 us against 66.6 us for a cap of 8.
// The cap is a tuning parameter (aerial_tuning.sc_per_group, searched by the
// autotuner).
constexpr int kDefaultGroupCap = 4;

struct FusedCell {
    const float2* H;
    const float2* Y;
    float* llr;
    float2* yeq;
    long group0;     // first global group index of this cell
    float sigma2;    // noise variance in the units the kernel sees (times scale^2)
    float scale;     // power-of-two operand scale (FP16 operands), else 1
    int nSC, A, L, nSym, nPam, LT, vecY, vecH, lgHalfL;
    int GS;          // subcarriers per group = min(32 / LT, group cap)
    int nChunk;      // 16-antenna chunks per subcarrier
    int hrs;         // staged channel-row stride (bytes)
    PamLut lut;
};

struct FusedParams {
    FusedCell cell[kMaxCells];
    int nCells;
    int epiBytes;    // per-warp epilogue region (bytes)
    int stageBytes;  // per operand stage (bytes)
    int exactTile;   // shared exact layer tile (2, 4, 8, 16) or 0: selects the kernel
    int nStages;     // operand stages per warp of that kernel
    int exactChunks; // with an exact tile: every cell has nAnt == 16 * exactChunks (2, 4, 8), else 0
    int fmt;         // AERIAL_FMT_* shared by every cell
    int scaled;      // some cell's FP16 operands are scaled (selects the kernel)
    int halfMixed;   // complex-half cells in a mixed batch (fused_eq_kernel_hg)
    int walkSlot;    // counter slot of the dynamic group walk, or -1 (static round-robin walk)
    long totalGroups;
};

// ---------------------------------------------------------------------------
// Group walk.  Every warp starts at group gw (its static first group).  With
// walkSlot < 0 it then takes groups gw + nw, gw + 2 nw, ... (round-robin);
// with a slot (the unrolled kernels) it takes each further group as nw + a
// ticket from the slot's counter in device memory, so warps that run ahead
// take more groups and the launch ends when the work is done, not when the
// warp with the most or the slowest groups is.  The last warp to finish
// resets the slot's two words (next ticket, warps done) for the slot's next
// launch.  The host gives each stream and each graph its own slot, so
// launches that can overlap never share one.  A subcarrier's result does not
// depend on the warp that computes it: both walks give the same LLRs bit for
// bit.  Measured, same box: 64 100 MHz slots 213.6 -> 209.3 us; the 12-slot
// precision-stress launch 337 -> 316 us with BF16X3 operands, 265 -> 256 us
// with FP16 operands.
// ---------------------------------------------------------------------------
constexpr int kWalkSlots = 64;
__device__ unsigned int g_walk[2 * kWalkSlots];

__device__ __forceinline__ long walk_next(const FusedParams& p, long nw, long staticNext, int lane) {
    if (p.walkSlot < 0) return staticNext;
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(&g_walk[2 * p.walkSlot], 1u);
    return nw + (long)__shfl_sync(0xffffffffu, t, 0);
}

// Called once by every warp of the launch, last.
__device__ __forceinline__ void walk_done(const FusedParams& p, long nw) {
    if (p.walkSlot < 0) return;
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        unsigned* w = g_walk + 2 * p.walkSlot;
        __threadfence();                                 // this warp's tickets precede its count
        if (atomicAdd(w + 1, 1u) == (unsigned)(nw - 1)) {
            atomicExch(w, 0u);
            atomicExch(w + 1, 0u);
        }
    }
}


// Packed FP32 pairs (fma.rn.f32x2 and friends, two IEEE operations per
// instruction on sm_100a).
__device__ __forceinline__ unsigned long long pk2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
// Two complex samples times the (exact, power-of-two) operand scale ss = (s, s).
__device__ __forceinline__ float4 scale4(float4 v, unsigned long long ss) {
    const float2 a = upk2(mul2(pk2(v.x, v.y), ss));
    const float2 b = upk2(mul2(pk2(v.z, v.w), ss));
    return make_float4(a.x, a.y, b.x, b.y);
}

// ---------------------------------------------------------------------------
// operand packing
// ---------------------------------------------------------------------------
template <int P>
__device__ __forceinline__ uint32_t pack2(float re, float im) {
    if constexpr (P == AERIAL_PREC_FP16) {
        __half2 h = __floats2half2_rn(re, im);
        return *reinterpret_cast<uint32_t*>(&h);
    } else {
        __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
        return *reinterpret_cast<uint32_t*>(&h);
    }
}
// (re, im) -> (-im, re): swap the halves and flip the sign bit of the new low half.
__device__ __forceinline__ uint32_t jrot(uint32_t p) { return __byte_perm(p, 0, 0x1032) ^ 0x8000u; }

// (x.re, x.im) - (h.re, h.im) as one packed FP32 subtraction (exact here:
// h is x rounded to fewer bits).
__device__ __forceinline__ float2 sub2(float re, float im, float2 h) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(re, im)), "l"(pk2(h.x, h.y)));
    return upk2(d);
}
// bf16 hi/lo split of a complex pair: x = hi + lo to ~16 mantissa bits.
__device__ __forceinline__ void split_bf16(float re, float im, uint32_t& hi, uint32_t& lo) {
    __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
    const float2 r = sub2(re, im, __bfloat1622float2(h));
    __nv_bfloat162 l = __floats2bfloat162_rn(r.x, r.y);
    hi = *reinterpret_cast<uint32_t*>(&h);
    lo = *reinterpret_cast<uint32_t*>(&l);
}
// fp16 hi/lo split: x = hi + lo to ~22 significant bits, for operands the
// host has normalized (set_operand_scale) so that lo stays a normal half.
__device__ __forceinline__ void split_fp16(float re, float im, uint32_t& hi, uint32_t& lo) {
    __half2 h = __floats2half2_rn(re, im);
    const float2 r = sub2(re, im, __half22float2(h));
    __half2 l = __floats2half2_rn(r.x, r.y);
    hi = *reinterpret_cast<uint32_t*>(&h);
    lo = *reinterpret_cast<uint32_t*>(&l);
}
template <int P>
__device__ __forceinline__ void split2(float re, float im, uint32_t& hi, uint32_t& lo) {
    if constexpr (P == AERIAL_PREC_FP16X3)
        split_fp16(re, im, hi, lo);
    else
        split_bf16(re, im, hi, lo);
}

template <int P>
__device__ __forceinline__ void mma16816(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    if constexpr (P == AERIAL_PREC_FP16 || P == AERIAL_PREC_FP16X3) {
        asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    } else {
        asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
}

// ---------------------------------------------------------------------------
// per-warp shared-memory layout for layer tile LT (GS = 32/LT subcarriers), in
// float2 units.  G rows (later Lc^-1 rows) and Z rows of each subcarrier;
// row strides are even so pairs of complex values are one 16-byte access,
// and each subcarrier's block is offset by 16 bytes so the GS blocks that a
// warp reads in the same instruction fall in different banks.
// ---------------------------------------------------------------------------
template <int LT>
struct WarpSmem {
    static constexpr int GS = 32 / LT;
    static constexpr int RS = (LT + 3) & ~1;         // G row stride (even: float4-aligned)
    static constexpr int ZS = 16 + 2;                // Z row stride (16 symbols)
    static constexpr int GB = LT * RS + 2;           // per-subcarrier G block
    static constexpr int ZB = LT * ZS + 2;           // per-subcarrier Z block
    static constexpr int offG = 0;
    static constexpr int offZ = GS * GB;
    static constexpr int total = offZ + GS * ZB;
    // every float4 access (row starts, pair offsets, block and warp offsets)
    // must stay 16-byte aligned
    static_assert(RS % 2 == 0 && ZS % 2 == 0 && GB % 2 == 0 && ZB % 2 == 0 && offZ % 2 == 0 && total % 2 == 0,
                  "shared-memory layout must keep 16-byte alignment");
};

__host__ __device__ constexpr int warp_smem_bytes(int LT) {
    return LT == 1 ? WarpSmem<1>::total * 8
         : LT == 2 ? WarpSmem<2>::total * 8
         : LT == 4 ? WarpSmem<4>::total * 8
         : LT == 8 ? WarpSmem<8>::total * 8
                   : WarpSmem<16>::total * 8;
}

// The fields of a cell a warp needs, read once from kernel-parameter space.
struct CellView {
    const float2* H;
    const float2* Y;
    float* llr;
    float2* yeq;
    float s2;
    int nSC, A, L, nSym, nPam, vecY;
    PamLut lut;
};

__device__ __forceinline__ CellView view_of(const FusedCell& c) {
    CellView v;
    v.H = c.H; v.Y = c.Y; v.llr = c.llr; v.yeq = c.yeq; v.s2 = c.sigma2;
    v.nSC = c.nSC; v.A = c.A; v.L = c.L; v.nSym = c.nSym; v.nPam = c.nPam; v.vecY = c.vecY;
    v.lut = c.lut;
    return v;
}

// ---------------------------------------------------------------------------
// Operand staging.  Each warp streams its (subcarrier, 16-antenna chunk)
// items through a ring of shared-memory stages with cp.async (16-byte
// global -> shared copies that need no registers).  The ring runs ahead
// across group boundaries, so while a warp does the FP32 solve and the LLR
// epilogue of one group, the first chunks of its next group are in flight.
//
// Stage layout (bytes): 16 channel rows H[a][0..L-1] at a stride HRS (padded
// so the fragment reads H[2c][g] of a warp hit distinct banks), then up to
// 16 received rows Y[s][a0..a0+15] of 128 bytes whose 16-byte pieces are
// XOR-swizzled by (s & 1) * 4 (conflict-free 16-byte fragment reads).
// ---------------------------------------------------------------------------
// Stages per warp: three for exact tiles up to 8 layers, two for the generic
// kernel and the 16-layer tile, whose larger epilogue regions would otherwise
// cost resident warps.  Measured same-box A/B (sustained): the 8-layer cell
// 250 -> 244 us with three stages instead of four (12 resident warps instead
// of 10), the uneven 16-cell batch 57.0 -> 54.6 us and the 16-layer cell
// 411 -> 398 us with two instead of three.
__host__ __device__ constexpr int stages_of(int exactTile) { return exactTile == 0 || exactTile == 16 ? 2 : 3; }
constexpr int CHUNK = 16;       // antennas per stage (two k-steps)

__host__ __device__ constexpr int hrs_of(int L) {
    return (((8 * L + 15) & ~15) + 16) < 48 ? 48 : (((8 * L + 15) & ~15) + 16);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(__cvta_generic_to_global(src))
                 : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(__cvta_generic_to_global(src))
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ float2 lds64(uint32_t a) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ float4 lds128(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}

// Gram blocks kept: (0,0) for LT <= 8; (0,0), (1,0), (1,1) for LT = 16.
// Fragment reads of one staged chunk (two k-steps) and their MMAs.  Thread
// (g, c) of k-step kk owns the antenna pair 8kk + 2c, +1 of the chunk.
//
// FULL: all 16 antennas of the chunk exist, so no antenna mask is applied.
// Rows of symbols past nSym are never masked: each received row only feeds
// its own Z column, and columns past nSym are never read.
// yo[kk][nt]: the lane's received-row fragment offsets in a stage (row
// 8 nt + g, clamped to row 0 past nSym, antenna pair 8 kk + 2 c, swizzled),
// fixed per cell.
// SC: FP16 operands of a cell whose noise level lies outside the range where
// raw FP16 is safe are multiplied by the cell's power-of-two scale ss = (s, s)
// before they are rounded (exact; the cell's sigma2 carries s^2, so G^-1 Z,
// mu and the LLRs are unchanged).
template <int LT, int P, bool LEXACT, bool FULL, bool SC = false>
__device__ __forceinline__ void mma_stage(uint32_t st, int hrs, int nRows, int L, const uint32_t (&yo)[2][2],
                                          float (*gacc)[4], float (*zacc)[2][4], bool z2, int g, int c,
                                          unsigned long long ss = 0) {
    constexpr int NMT = LT > 8 ? 2 : 1;
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
        const int a0 = 8 * kk + 2 * c;
        if (!FULL && 8 * kk >= nRows) break;             // uniform: tail chunk of 8 antennas
        const bool v0 = FULL || a0 < nRows, v1 = FULL || a0 + 1 < nRows;
        float4 hv[NMT];
#pragma unroll
        for (int mt = 0; mt < NMT; mt++) {
            const int l = g + 8 * mt;
            const bool lv = LEXACT || l < L;             // LEXACT: every lane's layer exists (L == LT)
            const int la = lv ? l : 0;                   // padded layers read row data they then discard
            const float2 h0 = lds64(st + a0 * hrs + la * 8);
            const float2 h1 = lds64(st + (a0 + 1) * hrs + la * 8);
            hv[mt] = make_float4((lv && v0) ? h0.x : 0.f, (lv && v0) ? h0.y : 0.f, (lv && v1) ? h1.x : 0.f,
                                 (lv && v1) ? h1.y : 0.f);
        }
        float4 yv[2];
#pragma unroll
        for (int nt = 0; nt < 2; nt++) {
            const float4 y = lds128(st + yo[kk][nt]);
            yv[nt] = FULL ? y : make_float4(v0 ? y.x : 0.f, v0 ? y.y : 0.f, v1 ? y.z : 0.f, v1 ? y.w : 0.f);
        }
        if constexpr (SC) {
#pragma unroll
            for (int mt = 0; mt < NMT; mt++) hv[mt] = scale4(hv[mt], ss);
#pragma unroll
            for (int nt = 0; nt < 2; nt++) yv[nt] = scale4(yv[nt], ss);
        }
        if constexpr (P == AERIAL_PREC_BF16X3 || P == AERIAL_PREC_FP16X3) {
            uint32_t ah[NMT][2], al[NMT][2];
#pragma unroll
            for (int mt = 0; mt < NMT; mt++) {
                split2<P>(hv[mt].x, hv[mt].y, ah[mt][0], al[mt][0]);
                split2<P>(hv[mt].z, hv[mt].w, ah[mt][1], al[mt][1]);
            }
            uint32_t yh[2][2], yl[2][2];
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                split2<P>(yv[nt].x, yv[nt].y, yh[nt][0], yl[nt][0]);
                split2<P>(yv[nt].z, yv[nt].w, yh[nt][1], yl[nt][1]);
            }
#pragma unroll
            for (int mt = 0; mt < NMT; mt++) {
                const uint32_t h0 = ah[mt][0], h1 = jrot(ah[mt][0]), h2 = ah[mt][1], h3 = jrot(ah[mt][1]);
                const uint32_t l0 = al[mt][0], l1 = jrot(al[mt][0]), l2 = al[mt][1], l3 = jrot(al[mt][1]);
#pragma unroll
                for (int nt = 0; nt <= mt; nt++) {
                    float* d = gacc[mt + nt];
                    mma16816<P>(d, h0, h1, h2, h3, ah[nt][0], ah[nt][1]);
                    mma16816<P>(d, h0, h1, h2, h3, al[nt][0], al[nt][1]);
                    mma16816<P>(d, l0, l1, l2, l3, ah[nt][0], ah[nt][1]);
                }
#pragma unroll
                for (int nt = 0; nt < 2; nt++) {
                    if (nt == 1 && !z2) break;
                    mma16816<P>(zacc[mt][nt], h0, h1, h2, h3, yh[nt][0], yh[nt][1]);
                    mma16816<P>(zacc[mt][nt], h0, h1, h2, h3, yl[nt][0], yl[nt][1]);
                    mma16816<P>(zacc[mt][nt], l0, l1, l2, l3, yh[nt][0], yh[nt][1]);
                }
            }
        } else {
            uint32_t a[NMT][2];
#pragma unroll
            for (int mt = 0; mt < NMT; mt++) {
                a[mt][0] = pack2<P>(hv[mt].x, hv[mt].y);
                a[mt][1] = pack2<P>(hv[mt].z, hv[mt].w);
            }
            uint32_t b[2][2];
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                b[nt][0] = pack2<P>(yv[nt].x, yv[nt].y);
                b[nt][1] = pack2<P>(yv[nt].z, yv[nt].w);
            }
#pragma unroll
            for (int mt = 0; mt < NMT; mt++) {
                const uint32_t a0r = a[mt][0], a1r = jrot(a[mt][0]), a2r = a[mt][1], a3r = jrot(a[mt][1]);
#pragma unroll
                for (int nt = 0; nt <= mt; nt++) mma16816<P>(gacc[mt + nt], a0r, a1r, a2r, a3r, a[nt][0], a[nt][1]);
#pragma unroll
                for (int nt = 0; nt < 2; nt++) {
                    if (nt == 1 && !z2) break;
                    mma16816<P>(zacc[mt][nt], a0r, a1r, a2r, a3r, b[nt][0], b[nt][1]);
                }
            }
        }
    }
}

// Accumulators of subcarrier q of the group -> per-warp shared memory.
// Fragment (row g, cols 2c, 2c+1) and (row g+8, ...) = Re / Im of
// out[8mt+g][8nt+2c], out[8mt+g][8nt+2c+1]: one 16-byte store each.
template <int LT>
__device__ __forceinline__ void store_acc(float2* sm, float (*gacc)[4], float (*zacc)[2][4], int q, int g, int c) {
    using W = WarpSmem<LT>;
    constexpr int NMT = LT > 8 ? 2 : 1;
    float2* sG = sm + W::offG + q * W::GB;
    float2* sZ = sm + W::offZ + q * W::ZB;
#pragma unroll
    for (int mt = 0; mt < NMT; mt++) {
        const int r = 8 * mt + g;
#pragma unroll
        for (int nt = 0; nt <= mt; nt++) {
            const float* d = gacc[mt + nt];
            const int n = 8 * nt + 2 * c;
            if (r < LT && n < LT)
                *reinterpret_cast<float4*>(sG + r * W::RS + n) = make_float4(d[0], d[2], d[1], d[3]);
        }
#pragma unroll
        for (int nt = 0; nt < 2; nt++) {
            const float* d = zacc[mt][nt];
            const int s = 8 * nt + 2 * c;
            if (r < LT) *reinterpret_cast<float4*>(sZ + r * W::ZS + s) = make_float4(d[0], d[2], d[1], d[3]);
        }
    }
}

template <int N>
__device__ __forceinline__ void write_llr(float* dst, const float* o) {
    if constexpr (N == 2) {
        __stcs(reinterpret_cast<float4*>(dst), make_float4(o[0], o[1], o[2], o[3]));
    } else if constexpr (N == 4) {
        __stcs(reinterpret_cast<float4*>(dst), make_float4(o[0], o[1], o[2], o[3]));
        __stcs(reinterpret_cast<float4*>(dst + 4), make_float4(o[4], o[5], o[6], o[7]));
    } else {
#pragma unroll
        for (int j = 0; j < 2 * N; j += 2) __stcs(reinterpret_cast<float2*>(dst + j), make_float2(o[j], o[j + 1]));
    }
}

// The same LLRs stored as __half (the reference's LLR storage), rounded to
// nearest from the clamped FP32 values: 2N halves = 4N bytes per symbol.
__device__ __forceinline__ unsigned half2_bits(float lo, float hi) {
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&h);
}
template <int N>
__device__ __forceinline__ void write_llr_h(char* dst, const float* o) {
    if constexpr (N == 4) {
        __stcs(reinterpret_cast<uint4*>(dst), make_uint4(half2_bits(o[0], o[1]), half2_bits(o[2], o[3]),
                                                          half2_bits(o[4], o[5]), half2_bits(o[6], o[7])));
    } else if constexpr (N == 2) {
        __stcs(reinterpret_cast<uint2*>(dst), make_uint2(half2_bits(o[0], o[1]), half2_bits(o[2], o[3])));
    } else {
#pragma unroll
        for (int j = 0; j < 2 * N; j += 2) __stcs(reinterpret_cast<unsigned*>(dst + 2 * j), half2_bits(o[j], o[j + 1]));
    }
}

// Max-log PAM demapper of the fused epilogue: the formula of llr_v1_baseline
// (src/llr/aerial_llr_v3.cu:90-107) evaluated on a scaled axis.  With
// r = sqrt(noiseInv), the soft estimate and the distances D_i scaled by r,
//   (pm_i - t^2) * noiseInv = (r m_i)^2 - (r t)^2,
// so each LLR is one fma(-t', t', m'^2) with no noise multiply.  For the last
// soft bit m = D + a and t = a - D with the same a, so m^2 - t^2 = 4 D a
// exactly: one multiply (and QPSK is that term alone).  The +-65504 clamp is
// applied to the magnitude and the soft bit's sign copied in with one bit
// operation.  It differs from the reference's rounding by a few FP32 ulps of
// each LLR (the plain chain keeps the bit-exact form).
template <int N>
__device__ __forceinline__ void pam_llr_scaled(float pI, float pQ, const float* d, float* out) {
    const float dist = d[N - 1];
    const float dist4 = 4.f * dist;
#pragma unroll
    for (int iq = 0; iq < 2; iq++) {
        float sb = iq ? pQ : pI;
        float pm[N], sg[N];
#pragma unroll
        for (int i = 0; i < N - 1; i++) {
            const float a = fabsf(sb);
            const float m = dist + a;
            pm[i] = m * m;
            sg[i] = sb;
            sb = d[i] - a;
        }
        sg[N - 1] = sb;
        const float aL = fabsf(sb);
        const float t = aL - dist;
#pragma unroll
        for (int i = 0; i < N; i++) {
            const float v = fminf(i == N - 1 ? dist4 * aL : fmaf(-t, t, pm[i]), 65504.f);
            out[2 * i + iq] = __int_as_float(__float_as_int(v) ^ (__float_as_int(sg[i]) & 0x80000000));
        }
    }
}

// One symbol of a layer row: Y_eq = x / mu (when YE), LLRs of x * r / mu at
// lp; H16: Y_eq as half2 and LLRs as __half.
template <int N, bool YE, bool H16>
__device__ __forceinline__ void emit1(char* lp, char* ye, float2 x, float invMu, float scl, const float* d) {
    if constexpr (YE) {
        if constexpr (H16)
            __stcs(reinterpret_cast<unsigned*>(ye), half2_bits(x.x * invMu, x.y * invMu));
        else
            __stcs(reinterpret_cast<float2*>(ye), make_float2(x.x * invMu, x.y * invMu));
    }
    float o[2 * N];
    pam_llr_scaled<N>(x.x * scl, x.y * scl, d, o);
    if constexpr (H16)
        write_llr_h<N>(lp, o);
    else
        write_llr<N>(reinterpret_cast<float*>(lp), o);
}

__device__ __forceinline__ void lds2x64(uint32_t a, unsigned long long& v0, unsigned long long& v1) {
    asm volatile("ld.shared.v2.b64 {%0, %1}, [%2];\n" : "=l"(v0), "=l"(v1) : "r"(a));
}

// X[i][s] = sum_m Ginv[i][m] Z[m][s] for symbol pairs, then unbias and demap;
// lp / ye walk the row's LLRs and equalized symbols.  The sums run on packed
// pairs: with Z[m][s] = (zr, zi) as stored,
//   P_s = sum_m (Re g_m, Re g_m) * (zr, zi),  Q_s = sum_m (Im g_m, Im g_m) * (zr, zi)
//   X_s = (P.x - Q.y, P.y + Q.x),
// four packed FMAs per m and symbol pair instead of eight scalar ones.
template <int LT, int N, bool YE, bool H16>
__device__ __forceinline__ void emit_row(const float2* sZ, const float2* gi, char* lp, char* ye, int nSym,
                                         float invMu, float scl, const float* d) {
    using W = WarpSmem<LT>;
    constexpr int LB = 2 * N * (H16 ? 2 : 4);      // LLR bytes per symbol
    constexpr int YB = H16 ? 4 : 8;                // Y_eq bytes per symbol
    unsigned long long gr[LT], gq[LT];
#pragma unroll
    for (int m = 0; m < LT; m++) {
        gr[m] = pk2(gi[m].x, gi[m].x);
        gq[m] = pk2(gi[m].y, gi[m].y);
    }
    const uint32_t zb = (uint32_t)__cvta_generic_to_shared(sZ);
#pragma unroll 1
    for (int s = 0; s < nSym; s += 2) {
        unsigned long long P0, Q0, P1, Q1;
#pragma unroll
        for (int m = 0; m < LT; m++) {
            unsigned long long z0, z1;
            lds2x64(zb + (m * W::ZS + s) * 8, z0, z1);
            if (m == 0) {
                P0 = mul2(gr[0], z0);
                Q0 = mul2(gq[0], z0);
                P1 = mul2(gr[0], z1);
                Q1 = mul2(gq[0], z1);
            } else {
                P0 = fma2(gr[m], z0, P0);
                Q0 = fma2(gq[m], z0, Q0);
                P1 = fma2(gr[m], z1, P1);
                Q1 = fma2(gq[m], z1, Q1);
            }
        }
        const float2 p0 = upk2(P0), q0 = upk2(Q0), p1 = upk2(P1), q1 = upk2(Q1);
        emit1<N, YE, H16>(lp, ye, make_float2(p0.x - q0.y, p0.y + q0.x), invMu, scl, d);
        if (s + 1 < nSym)
            emit1<N, YE, H16>(lp + LB, ye + YB, make_float2(p1.x - q1.y, p1.y + q1.x), invMu, scl, d);
        lp += 2 * LB;
        if constexpr (YE) ye += 2 * YB;
    }
}

// Lane (sc, i): layer row i of subcarrier sc.  Lanes without an output row
// return at once.
template <int LT, int N, bool H16>
__device__ __forceinline__ void solve_emit(const CellView& cl, const float2* sZ, const float2* gi, long sc, int i,
                                           bool out, float invMu, float nInv) {
    if (!out) return;
    const long row = sc * cl.L + i;
    char* lp = reinterpret_cast<char*>(cl.llr) + row * cl.nSym * (2 * N) * (H16 ? 2 : 4);
    const float r = sqrtf(nInv);
    const float scl = invMu * r;
    float d[N];
#pragma unroll
    for (int k = 0; k < N; k++) d[k] = cl.lut.d[k] * r;
    if (cl.yeq)
        emit_row<LT, N, true, H16>(sZ, gi, lp, reinterpret_cast<char*>(cl.yeq) + row * cl.nSym * (H16 ? 4 : 8),
                                   cl.nSym, invMu, scl, d);
    else
        emit_row<LT, N, false, H16>(sZ, gi, lp, nullptr, cl.nSym, invMu, scl, d);
}

// 1/x: the approximate reciprocal plus one Newton-Raphson step y (2 - x y).
__device__ __forceinline__ float rcp_nr(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y * fmaf(-x, y, 2.f);
}

// Row of LT complex values from shared memory (16-byte pieces; rows start
// 16-byte aligned, WarpSmem keeps every row stride even).
template <int LT>
__device__ __forceinline__ void get_row(const float2* row, float2 (&b)[LT]) {
    if constexpr (LT == 1) {
        b[0] = row[0];
    } else {
#pragma unroll
        for (int m = 0; m < LT; m += 2) {
            const float4 t = *reinterpret_cast<const float4*>(row + m);
            b[m] = make_float2(t.x, t.y);
            b[m + 1] = make_float2(t.z, t.w);
        }
    }
}

// ---------------------------------------------------------------------------
// The FP32 solve of one group of GS subcarriers whose G and Z are in the
// warp's epilogue region: LT lanes per subcarrier.
// ---------------------------------------------------------------------------
// H16: Y_eq and LLRs are stored as half precision (the FP16 I/O format).
template <int LT, int P, bool H16 = false>
__device__ __noinline__ void solve_group(const CellView cl, long sc0, int nValid, int smemOff, int lane) {
    using W = WarpSmem<LT>;
    extern __shared__ float4 smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw) + smemOff;
    // ---- solve phase: lane = (q, i), LT lanes per subcarrier ----
    // G^-1 by Gauss-Jordan elimination in place, lane i holding row i in
    // registers; X = G^-1 Z then reads Z from shared memory.
    const int q = lane / LT, i = lane % LT;
    const long sc = sc0 + q;
    const bool scValid = q < nValid;
    const bool real = i < cl.L;          // padded layers (i >= L) carry an identity block
    float2* sG = sm + W::offG + q * W::GB;
    const float2* sZ = sm + W::offZ + q * W::ZB;
    const float s2 = cl.s2;

    // Row i of G + s2 I.  The 16-layer tile keeps the Gram blocks (0,0),
    // (1,0) and (1,1) only, so rows 0-7 take columns 8-15 as conj(G[m][i]).
    // Subcarriers past the group's end solve s2 I (never stored).
    float2 r[LT];
    if constexpr (LT > 8) {
        float2 lo[8];
        get_row<8>(sG + i * W::RS, lo);
#pragma unroll
        for (int m = 0; m < 8; m++) r[m] = lo[m];
        const bool up = i < 8;
#pragma unroll
        for (int m = 8; m < LT; m++) {
            const float2 v = sG[up ? m * W::RS + i : i * W::RS + m];
            r[m] = make_float2(v.x, up ? -v.y : v.y);
        }
    } else {
        get_row<LT>(sG + i * W::RS, r);
    }
#pragma unroll
    for (int m = 0; m < LT; m++) {
        float2 v = (scValid && real) ? r[m] : make_float2(0.f, 0.f);
        if (m == i) v = real ? make_float2(v.x + s2, 0.f) : make_float2(1.f, 0.f);
        r[m] = v;
    }

    // Gauss-Jordan sweep, step k: row k as it stands before the step
    // (published to shared memory by lane k at the end of step k - 1)
    // eliminates column k from every other row:
    //   p = 1 / b_kk,  f_i = r_ik p  (f_k = 1 - p),
    //   r_ij -= f_i b_kj  (j != k),   r_ik = delta_ik - f_i,
    // which leaves row k as b_k p and, after LT steps, G^-1 in the rows.  On
    // the trailing block (i, j > k) the update is the right-looking LDL^H
    // (square-root-free Cholesky) step of G, and the pivots b_kk are the
    // diagonal of D in G = L D L^H: real and positive for the Hermitian
    // positive definite G, so no pivoting is needed.  The other rows and
    // columns accumulate the inverse in the same sweep.  Every lane does
    // LT - 1 useful complex multiply-adds per step (no idle triangle), and the
    // broadcast of row k is LT / 2 shared loads.
    if constexpr (LT == 1) {
        // one layer: G^-1 = 1 / g
        r[0] = make_float2(rcp_nr(fmaxf(r[0].x, 1e-30f)), -0.f);
    } else {
        // The row is held planar for the sweep: for each column pair h,
        // X[h] = (Re r_2h, Re r_2h+1) and Y[h] = (Im r_2h, Im r_2h+1), and the
        // published row k is stored the same way (one 16-byte piece per pair:
        // Re, Re, Im, Im), so the update
        //   Re r_j = fma(-fx, Re b_j, fma(fy, Im b_j, Re r_j))
        //   Im r_j = fma(-fx, Im b_j, fma(-fy, Re b_j, Im r_j))
        // is four packed FMAs per column pair, in the same order of rounding
        // as the scalar form.  Column k's updated value is discarded.
        constexpr int NP = LT / 2;
        unsigned long long X[NP], Y[NP];
#pragma unroll
        for (int h = 0; h < NP; h++) {
            X[h] = pk2(r[2 * h].x, r[2 * h + 1].x);
            Y[h] = pk2(r[2 * h].y, r[2 * h + 1].y);
        }
        auto put_planar = [&](float2* row) {
#pragma unroll
            for (int h = 0; h < NP; h++) {
                const float2 x = upk2(X[h]), y = upk2(Y[h]);
                *reinterpret_cast<float4*>(row + 2 * h) = make_float4(x.x, x.y, y.x, y.y);
            }
        };
        if (i == 0) put_planar(sG);
#pragma unroll
        for (int k = 0; k < LT; k++) {
            __syncwarp();
            const float* bk = reinterpret_cast<const float*>(sG + k * W::RS);
            const float piv = fmaxf(bk[4 * (k >> 1) + (k & 1)], 1e-30f);
            const float p = rcp_nr(piv);
            const bool mine = i == k;
            const float2 xk = upk2(X[k >> 1]), yk = upk2(Y[k >> 1]);
            const float rkx = (k & 1) ? xk.y : xk.x, rky = (k & 1) ? yk.y : yk.x;
            const float fx = mine ? 1.f - p : rkx * p;
            const float fy = mine ? 0.f : rky * p;
            const unsigned long long nfx = pk2(-fx, -fx), pfy = pk2(fy, fy), nfy = pk2(-fy, -fy);
#pragma unroll
            for (int h = 0; h < NP; h++) {
                const float4 t = *reinterpret_cast<const float4*>(bk + 4 * h);
                const unsigned long long bx = pk2(t.x, t.y), by = pk2(t.z, t.w);
                X[h] = fma2(nfx, bx, fma2(pfy, by, X[h]));
                Y[h] = fma2(nfx, by, fma2(nfy, bx, Y[h]));
            }
            const float nx = mine ? p : -fx, ny = -fy;
            const float2 xs = upk2(X[k >> 1]), ys = upk2(Y[k >> 1]);
            X[k >> 1] = (k & 1) ? pk2(xs.x, nx) : pk2(nx, xs.y);
            Y[k >> 1] = (k & 1) ? pk2(ys.x, ny) : pk2(ny, ys.y);
            if (k + 1 < LT && i == k + 1) put_planar(sG + (k + 1) * W::RS);
        }
#pragma unroll
        for (int h = 0; h < NP; h++) {
            const float2 x = upk2(X[h]), y = upk2(Y[h]);
            r[2 * h] = make_float2(x.x, y.x);
            r[2 * h + 1] = make_float2(x.y, y.y);
        }
    }
    float gii = r[0].x;
#pragma unroll
    for (int m = 1; m < LT; m++) gii = (i == m) ? r[m].x : gii;

    // X row i = Ginv[i][:] Z, two symbols at a time, each pair demapped and
    // stored as soon as it is complete.
    const float t = s2 * gii;           // 1 - mu = s2 (G^-1)_ii
    const float mu = fmaxf(1.0f - t, 1e-30f);
    const float invMu = 1.0f / mu;
    const float nInv = mu / fmaxf(t, 1e-30f);
    const bool out = scValid && real;
    switch (cl.nPam) {
        case 1: solve_emit<LT, 1, H16>(cl, sZ, r, sc, i, out, invMu, nInv); break;
        case 2: solve_emit<LT, 2, H16>(cl, sZ, r, sc, i, out, invMu, nInv); break;
        case 3: solve_emit<LT, 3, H16>(cl, sZ, r, sc, i, out, invMu, nInv); break;
        default: solve_emit<LT, 4, H16>(cl, sZ, r, sc, i, out, invMu, nInv); break;
    }
    __syncwarp();   // shared memory is reused by the next group
}

// Per-warp shared memory of a launch: the epilogue region (largest footprint
// of the layer tiles present) followed by the operand stages.
inline int stage_bytes_of(const FusedParams& p) {
    int b = 0;
    for (int ci = 0; ci < p.nCells; ci++) {
        const int v = CHUNK * hrs_of(p.cell[ci].L) + 128 * p.cell[ci].nSym;
        b = v > b ? v : b;
    }
    return (b + 15) & ~15;
}
inline int epi_bytes_of(const FusedParams& p) {
    int b = 0;
    for (int ci = 0; ci < p.nCells; ci++) {
        const int v = warp_smem_bytes(p.cell[ci].LT);
        b = v > b ? v : b;
    }
    return (b + 15) & ~15;
}

// Stage the copies of one item (subcarrier base pointers hs / ys, chunk ch)
// of cell cl into the stage at shared address st.  Subcarriers of a group
// are contiguous, so the producer only advances pointers between items.
__device__ __forceinline__ void stage_item(const FusedCell& cl, const float2* hs, const float2* ys, int ch,
                                           uint32_t st, int lane) {
    const int L = cl.L, A = cl.A, nSym = cl.nSym, hrs = cl.hrs;
    const int nRows = min(CHUNK, A - CHUNK * ch);
    const float2* hsrc = hs + CHUNK * ch * L;
    if (cl.vecH) {                      // L even: 16-byte pieces, L/2 per row
        const int half = L >> 1;
        const int n = nRows * half;
        if (cl.lgHalfL >= 0) {
            const int sh = cl.lgHalfL;
            for (int e = lane; e < n; e += 32) cp_async16(st + (e >> sh) * hrs + (e & (half - 1)) * 16, hsrc + 2 * e);
        } else {
            for (int e = lane; e < n; e += 32) {
                const int row = e / half;
                cp_async16(st + row * hrs + (e - row * half) * 16, hsrc + 2 * e);
            }
        }
    } else {                            // 8-byte pieces
        const int n = nRows * L;
        for (int e = lane; e < n; e += 32) {
            const int row = e / L;
            cp_async8(st + row * hrs + (e - row * L) * 8, hsrc + e);
        }
    }
    const uint32_t yst = st + CHUNK * hrs;
    const float2* ysrc = ys + CHUNK * ch;
    for (int e = lane; e < nSym * 8; e += 32) {
        const int s = e >> 3, k = e & 7;
        const int a = 2 * k;
        if (a < nRows) {
            const uint32_t d = yst + s * 128 + ((k ^ ((s & 1) << 2)) << 4);
            const float2* src = ysrc + (long)s * A + a;
            if (cl.vecY && a + 1 < nRows) {
                cp_async16(d, src);
            } else {
                cp_async8(d, src);
                if (a + 1 < nRows) cp_async8(d + 8, src + 1);
            }
        }
    }
}

// stage_item for a launch whose cells all have L == LF (even): strides and
// piece mapping are compile-time constants.
template <int LF>
__device__ __forceinline__ void stage_item_exact(const FusedCell& cl, const float2* hs, const float2* ys, int ch,
                                                 uint32_t st, int lane) {
    constexpr int HRS = hrs_of(LF);
    constexpr int HALF = LF / 2;
    const int A = cl.A, nSym = cl.nSym;
    const int nRows = min(CHUNK, A - CHUNK * ch);
    const float2* hsrc = hs + CHUNK * ch * LF;
    const int n = nRows * HALF;
#pragma unroll
    for (int k = 0; k < (CHUNK * HALF + 31) / 32; k++) {
        const int e = lane + 32 * k;
        if (e < n) cp_async16(st + (e / HALF) * HRS + (e % HALF) * 16, hsrc + 2 * e);
    }
    const uint32_t yst = st + CHUNK * HRS;
    const float2* ysrc = ys + CHUNK * ch;
    if (nRows == CHUNK) {
#pragma unroll
        for (int k = 0; k < 4; k++) {                  // up to 16 rows x 8 pieces
            const int e = lane + 32 * k;
            const int s = e >> 3, kk = e & 7;
            if (s < nSym) cp_async16(yst + s * 128 + ((kk ^ ((s & 1) << 2)) << 4), ysrc + (long)s * A + 2 * kk);
        }
    } else {
        for (int e = lane; e < nSym * 8; e += 32) {
            const int s = e >> 3, kk = e & 7;
            const int a = 2 * kk;
            if (a < nRows) {
                const uint32_t d = yst + s * 128 + ((kk ^ ((s & 1) << 2)) << 4);
                const float2* src = ysrc + (long)s * A + a;
                if (a + 1 < nRows) cp_async16(d, src);
                else cp_async8(d, src);
            }
        }
    }
}

// A full 16-antenna chunk of a launch whose cells all have L == LF: the
// channel rows are 16 * LF / 2 pieces of 16 bytes (lane e -> row e / (LF/2),
// piece e % (LF/2)), the received rows 8 pieces each (lane -> row lane / 8 + 4k,
// piece lane % 8).  hLaneS / yLaneS are the lane's stage offsets of its first
// pieces, ys points at the lane's first received piece, yStep = 4 rows, and
// nYk is the lane's count of received rows below nSym.
template <int LF>
__device__ __forceinline__ void stage_full(uint32_t st, uint32_t hLaneS, uint32_t yLaneS, const float2* hsrc,
                                           const float2* ys, int yStep, int nYk, int lane) {
    constexpr int HRS = hrs_of(LF);
    constexpr int HALF = LF / 2;
    constexpr int NP = CHUNK * HALF;                    // channel pieces per chunk
    constexpr int RPK = 32 / HALF;                      // channel rows per 32 pieces
#pragma unroll
    for (int k = 0; k < (NP + 31) / 32; k++)
        if (NP >= 32 * (k + 1) || lane < NP - 32 * k) cp_async16(st + hLaneS + k * RPK * HRS, hsrc + 2 * lane + 64 * k);
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (k < nYk) cp_async16(st + yLaneS + 512 * k, ys + k * yStep);
}

__device__ __forceinline__ int group_valid(const FusedCell& cl, long grp) {
    return (int)min((long)cl.GS, (long)cl.nSC - (grp - cl.group0) * cl.GS);
}

// LTF = 0: any mix of cells.  LTF in {2, 4, 8, 16}: every cell has
// nLayers == LTF and 16-byte aligned H / Y_rx (the host checks), so the layer
// tile, strides and masks are compile-time constants.
// SC: the launch has cells whose FP16 operands are scaled (mma_stage).
template <int P, int LTF, bool SC = false>
__global__ void __launch_bounds__(256, 2) fused_eq_kernel(const __grid_constant__ FusedParams p) {
    extern __shared__ float4 smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warpsPerCta = blockDim.x >> 5;
    const int g = lane >> 2, c = lane & 3;
    constexpr int NST = stages_of(LTF);
    const int warpBytes = p.epiBytes + NST * p.stageBytes;
    const int smemOff = wib * (warpBytes / 8);
    float2* sm = reinterpret_cast<float2*>(smem_raw) + smemOff;
    const uint32_t stBase =
        (uint32_t)__cvta_generic_to_shared(reinterpret_cast<char*>(smem_raw) + (long)wib * warpBytes + p.epiBytes);
    const long gw = (long)blockIdx.x * warpsPerCta + wib;
    const long nw = (long)gridDim.x * warpsPerCta;
    const long total = p.totalGroups;
    if (gw >= total) return;

    // ---- producer cursor (registers): group, cell, subcarrier, chunk ----
    // Per-lane staging offsets are fixed for the whole launch (exact tile) or
    // for a cell (received-row pieces), so a full chunk costs a few adds and
    // its cp.async instructions.
    uint32_t hLaneS = 0, yLaneS = 0;
    if constexpr (LTF != 0) {
        constexpr int HALF = LTF / 2;
        hLaneS = (lane / HALF) * hrs_of(LTF) + (lane % HALF) * 16;
        yLaneS = CHUNK * hrs_of(LTF) + (lane >> 3) * 128 + (((lane & 7) ^ (((lane >> 3) & 1) << 2)) << 4);
    }
    long pg = gw;
    int pci = 0;
    while (pci + 1 < p.nCells && pg >= p.cell[pci + 1].group0) pci++;
    int pq = 0, pch = 0, pslot = 0, pValid, pNChunk, pNFull, pYStep, pYLane, pYk;
    int pExact = 0;                                       // generic kernel: this cell's exact tile, or 0
    long pHsc, pYsc;
    const float2* phs;
    const float2* pys;
    auto load_pcell = [&]() {
        const FusedCell& cl = p.cell[pci];
        const int A = cl.A, nSym = cl.nSym;
        pNChunk = cl.nChunk;
        pNFull = A / CHUNK;
        pHsc = (long)A * (LTF != 0 ? LTF : cl.L);
        pYsc = (long)nSym * A;
        pValid = group_valid(cl, pg);
        const long sc = (pg - cl.group0) * cl.GS;
        phs = cl.H + sc * pHsc;
        pys = cl.Y + sc * pYsc;
        pYStep = 4 * A;                                   // received rows s and s + 4
        pYLane = (lane >> 3) * A + 2 * (lane & 7);        // this lane's first piece
        pYk = min(4, max(0, (nSym - (lane >> 3) + 3) >> 2));
        if constexpr (LTF == 0) {
            // a cell whose layers fill its tile stages full chunks like the
            // exact-tile kernels, with this cell's lane offsets
            pExact = (cl.L == cl.LT && cl.LT >= 2 && cl.vecH && cl.vecY) ? cl.LT : 0;
            if (pExact) {
                const int half = cl.L / 2;
                hLaneS = (lane / half) * cl.hrs + (lane % half) * 16;
                yLaneS = CHUNK * cl.hrs + (lane >> 3) * 128 + (((lane & 7) ^ (((lane >> 3) & 1) << 2)) << 4);
            }
        }
    };
    load_pcell();
    auto produce = [&]() {
        if (pg < total) {
            const uint32_t st = stBase + pslot * p.stageBytes;
            if constexpr (LTF != 0) {
                if (pch < pNFull)
                    stage_full<LTF>(st, hLaneS, yLaneS, phs + CHUNK * pch * LTF, pys + CHUNK * pch + pYLane, pYStep,
                                    pYk, lane);
                else
                    stage_item_exact<LTF>(p.cell[pci], phs, pys, pch, st, lane);
            } else {
                if (pExact && pch < pNFull) {
                    const float2* hsrc = phs + CHUNK * pch * pExact;
                    const float2* ysrc = pys + CHUNK * pch + pYLane;
                    switch (pExact) {
                        case 2: stage_full<2>(st, hLaneS, yLaneS, hsrc, ysrc, pYStep, pYk, lane); break;
                        case 4: stage_full<4>(st, hLaneS, yLaneS, hsrc, ysrc, pYStep, pYk, lane); break;
                        case 8: stage_full<8>(st, hLaneS, yLaneS, hsrc, ysrc, pYStep, pYk, lane); break;
                        default: stage_full<16>(st, hLaneS, yLaneS, hsrc, ysrc, pYStep, pYk, lane); break;
                    }
                } else {
                    stage_item(p.cell[pci], phs, pys, pch, st, lane);
                }
            }
            if (++pch == pNChunk) {
                pch = 0;
                if (++pq < pValid) {
                    phs += pHsc;
                    pys += pYsc;
                } else {
                    pq = 0;
                    pg += nw;
                    if (pg < total) {
                        while (pci + 1 < p.nCells && pg >= p.cell[pci + 1].group0) pci++;
                        load_pcell();
                    }
                }
            }
        }
        cp_async_commit();
        pslot = pslot == NST - 1 ? 0 : pslot + 1;
    };
#pragma unroll
    for (int k = 0; k < NST - 1; k++) produce();

    // ---- consumer: cell constants in registers, reloaded per group ----
    long grp = gw;
    int ci = 0;
    while (ci + 1 < p.nCells && grp >= p.cell[ci + 1].group0) ci++;
    int q = 0, ch = 0, cslot = 0, nValid, cNChunk, cNFull, cA, cL, cLT, cHrs;
    bool cExact = false;                                  // generic kernel: L fills the tile, aligned rows
    bool z2;
    uint32_t yo[2][2];
    unsigned long long ss = 0;                            // (scale, scale) of the cell's operands
    auto load_ccell = [&]() {
        const FusedCell& cl = p.cell[ci];
        if constexpr (SC) ss = pk2(cl.scale, cl.scale);
        nValid = group_valid(cl, grp);
        cA = cl.A;
        cNChunk = cl.nChunk;
        cNFull = cl.A / CHUNK;
        cL = cl.L;
        cLT = LTF != 0 ? LTF : cl.LT;
        cHrs = cl.hrs;
        cExact = cl.L == cl.LT && cl.LT >= 2 && cl.vecH && cl.vecY;
        z2 = cl.nSym > 8;
        const uint32_t ys = CHUNK * (LTF != 0 ? hrs_of(LTF) : cl.hrs);
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int r = 8 * nt + g;
                const int ra = r < cl.nSym ? r : 0;      // rows past nSym are not staged: read row 0 instead
                yo[kk][nt] = ys + ra * 128 + (((4 * kk + c) ^ ((ra & 1) << 2)) << 4);
            }
    };
    load_ccell();
    float gacc[3][4], zacc[2][2][4];
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
        for (int e = 0; e < 4; e++) gacc[b][e] = 0.f;
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 2; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) zacc[mt][nt][e] = 0.f;

    while (true) {
        __syncwarp();                              // every lane is done with the slot refilled now
        produce();
        cp_async_wait<NST - 1>();                  // this item's copies (own lane) have landed
        __syncwarp();                              // ... and every lane's
        const uint32_t st = stBase + cslot * p.stageBytes;
        cslot = cslot == NST - 1 ? 0 : cslot + 1;
        if constexpr (LTF != 0) {
            if (ch < cNFull)
                mma_stage<LTF, P, true, true, SC>(st, hrs_of(LTF), CHUNK, LTF, yo, gacc, zacc, z2, g, c, ss);
            else
                mma_stage<LTF, P, true, false, SC>(st, hrs_of(LTF), cA - CHUNK * ch, LTF, yo, gacc, zacc, z2, g, c,
                                                   ss);
        } else {
            const int nRows = min(CHUNK, cA - CHUNK * ch);
            if (cExact && nRows == CHUNK) {
                switch (cLT) {
                    case 2: mma_stage<2, P, true, true, SC>(st, cHrs, CHUNK, 2, yo, gacc, zacc, z2, g, c, ss); break;
                    case 4: mma_stage<4, P, true, true, SC>(st, cHrs, CHUNK, 4, yo, gacc, zacc, z2, g, c, ss); break;
                    case 8: mma_stage<8, P, true, true, SC>(st, cHrs, CHUNK, 8, yo, gacc, zacc, z2, g, c, ss); break;
                    default: mma_stage<16, P, true, true, SC>(st, cHrs, CHUNK, 16, yo, gacc, zacc, z2, g, c, ss); break;
                }
            } else switch (cLT) {
                case 1: mma_stage<1, P, false, false, SC>(st, cHrs, nRows, cL, yo, gacc, zacc, z2, g, c, ss); break;
                case 2: mma_stage<2, P, false, false, SC>(st, cHrs, nRows, cL, yo, gacc, zacc, z2, g, c, ss); break;
                case 4: mma_stage<4, P, false, false, SC>(st, cHrs, nRows, cL, yo, gacc, zacc, z2, g, c, ss); break;
                case 8: mma_stage<8, P, false, false, SC>(st, cHrs, nRows, cL, yo, gacc, zacc, z2, g, c, ss); break;
                default: mma_stage<16, P, false, false, SC>(st, cHrs, nRows, cL, yo, gacc, zacc, z2, g, c, ss); break;
            }
        }
        if (++ch < cNChunk) continue;
        ch = 0;
        if constexpr (LTF != 0) {
            store_acc<LTF>(sm, gacc, zacc, q, g, c);
        } else {
            switch (cLT) {
                case 1: store_acc<1>(sm, gacc, zacc, q, g, c); break;
                case 2: store_acc<2>(sm, gacc, zacc, q, g, c); break;
                case 4: store_acc<4>(sm, gacc, zacc, q, g, c); break;
                case 8: store_acc<8>(sm, gacc, zacc, q, g, c); break;
                default: store_acc<16>(sm, gacc, zacc, q, g, c); break;
            }
        }
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int e = 0; e < 4; e++) gacc[b][e] = 0.f;
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++)
#pragma unroll
                for (int e = 0; e < 4; e++) zacc[mt][nt][e] = 0.f;
        if (++q < nValid) continue;
        __syncwarp();
        {
            const FusedCell& cl = p.cell[ci];
            const CellView v = view_of(cl);
            const long sc0 = (grp - cl.group0) * cl.GS;
            if constexpr (LTF != 0) {
                solve_group<LTF, P>(v, sc0, nValid, smemOff, lane);
            } else {
                switch (cLT) {
                    case 1: solve_group<1, P>(v, sc0, nValid, smemOff, lane); break;
                    case 2: solve_group<2, P>(v, sc0, nValid, smemOff, lane); break;
                    case 4: solve_group<4, P>(v, sc0, nValid, smemOff, lane); break;
                    case 8: solve_group<8, P>(v, sc0, nValid, smemOff, lane); break;
                    default: solve_group<16, P>(v, sc0, nValid, smemOff, lane); break;
                }
            }
        }
        q = 0;
        grp += nw;
        if (grp >= total) break;
        while (ci + 1 < p.nCells && grp >= p.cell[ci + 1].group0) ci++;
        load_ccell();
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Exact-antenna variant: every cell of the launch has nLayers == LTF and
// nAnt == 16 * NCH.  A subcarrier's NCH chunks are unrolled, so the stage
// the producer fills at each step (chunk k + NST - 1 of this subcarrier, or
// an early chunk of the next one) is known at compile time, and its copies
// are a per-lane subcarrier pointer plus immediate offsets.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int stages_of_a(int ltf, int nch) {
    return stages_of(ltf) < nch + 1 ? stages_of(ltf) : nch + 1;
}

// One subcarrier's operands as the producing lane sees them: its first
// channel piece, its first received piece, its count of received rows.
struct ScPtr {
    const float2* h;
    const float2* y;
    int yk;
};

// Chunk j of subcarrier s into the stage at st (A = 16 NCH antennas).
template <int LF, int NCH>
__device__ __forceinline__ void stage_chunk(uint32_t st, uint32_t hLaneS, uint32_t yLaneS, const ScPtr& s, int j,
                                            int lane) {
    constexpr int HRS = hrs_of(LF);
    constexpr int HALF = LF / 2;
    constexpr int NP = CHUNK * HALF;
    constexpr int RPK = 32 / HALF;
    constexpr int A = CHUNK * NCH;
#pragma unroll
    for (int k = 0; k < (NP + 31) / 32; k++)
        if (NP >= 32 * (k + 1) || lane < NP - 32 * k)
            cp_async16(st + hLaneS + k * RPK * HRS, s.h + CHUNK * j * LF + 64 * k);
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (k < s.yk) cp_async16(st + yLaneS + 512 * k, s.y + CHUNK * j + 4 * k * A);
}

// Register budget: 128 per thread (16 resident warps) for tiles up to 8
// layers; the 16-layer tile's shared memory admits 12 resident warps at most,
// so it takes what it needs (140 registers, no spills in its 16 x 16 solve):
// 12-slot precision-stress launch 334 against 341-343 us with BF16X3 operands,
// same box, bit-identical.
template <int P, int LTF, int NCH, bool SC = false>
__global__ void __launch_bounds__(256, LTF == 16 ? 1 : 2) fused_eq_kernel_a(const __grid_constant__ FusedParams p) {
    constexpr int NST = stages_of_a(LTF, NCH);
    constexpr int A = CHUNK * NCH;
    constexpr int HRS = hrs_of(LTF);
    constexpr long HSC = (long)A * LTF;               // channel float2 per subcarrier
    extern __shared__ float4 smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warpsPerCta = blockDim.x >> 5;
    const int g = lane >> 2, c = lane & 3;
    const int warpBytes = p.epiBytes + NST * p.stageBytes;
    const int smemOff = wib * (warpBytes / 8);
    float2* sm = reinterpret_cast<float2*>(smem_raw) + smemOff;
    const uint32_t stBase =
        (uint32_t)__cvta_generic_to_shared(reinterpret_cast<char*>(smem_raw) + (long)wib * warpBytes + p.epiBytes);
    const long gw = (long)blockIdx.x * warpsPerCta + wib;
    const long nw = (long)gridDim.x * warpsPerCta;
    const long total = p.totalGroups;
    if (gw >= total) {
        walk_done(p, nw);
        return;
    }

    constexpr int HALF = LTF / 2;
    const uint32_t hLaneS = (lane / HALF) * HRS + (lane % HALF) * 16;
    const uint32_t yLaneS = CHUNK * HRS + (lane >> 3) * 128 + (((lane & 7) ^ (((lane >> 3) & 1) << 2)) << 4);
    const int yLaneG = (lane >> 3) * A + 2 * (lane & 7);

    // first subcarrier of group grp (in cell ci) as seen by this lane
    auto first_sc = [&](int cell, long grp) -> ScPtr {
        const FusedCell& cl = p.cell[cell];
        const long sc = (grp - cl.group0) * cl.GS;
        ScPtr s;
        s.h = cl.H + sc * HSC + 2 * lane;
        s.y = cl.Y + sc * cl.nSym * A + yLaneG;
        s.yk = min(4, max(0, (cl.nSym - (lane >> 3) + 3) >> 2));
        return s;
    };

    long grp = gw;
    int ci = 0;
    while (ci + 1 < p.nCells && grp >= p.cell[ci + 1].group0) ci++;
    int nValid, nSym;
    bool z2;
    uint32_t yo[2][2];
    unsigned long long ss = 0;                           // (scale, scale) of the cell's operands
    auto load_cell = [&]() {
        const FusedCell& cl = p.cell[ci];
        if constexpr (SC) ss = pk2(cl.scale, cl.scale);
        nValid = group_valid(cl, grp);
        nSym = cl.nSym;
        z2 = nSym > 8;
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int r = 8 * nt + g;
                const int ra = r < nSym ? r : 0;         // rows past nSym are not staged: read row 0 instead
                yo[kk][nt] = CHUNK * HRS + ra * 128 + (((4 * kk + c) ^ ((ra & 1) << 2)) << 4);
            }
    };
    load_cell();
    ScPtr cur = first_sc(ci, grp);

    int pslot = 0, cslot = 0;
#pragma unroll
    for (int j = 0; j < NST - 1; j++) {
        stage_chunk<LTF, NCH>(stBase + pslot * p.stageBytes, hLaneS, yLaneS, cur, j, lane);
        cp_async_commit();
        pslot = pslot == NST - 1 ? 0 : pslot + 1;
    }

    float gacc[3][4], zacc[2][2][4];
    int q = 0;
    long nextGrp = total;                                // the warp's next group, set with its last subcarrier
    while (true) {
        // the subcarrier after this one in the warp's order, if any
        ScPtr nxt = cur;
        bool hasNxt = true;
        if (q + 1 < nValid) {
            nxt.h = cur.h + HSC;
            nxt.y = cur.y + (long)nSym * A;
        } else {
            const long ng = walk_next(p, nw, grp + nw, lane);
            nextGrp = ng;
            hasNxt = ng < total;
            if (hasNxt) {
                int nc = ci;
                while (nc + 1 < p.nCells && ng >= p.cell[nc + 1].group0) nc++;
                nxt = first_sc(nc, ng);
            }
        }
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int e = 0; e < 4; e++) gacc[b][e] = 0.f;
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++)
#pragma unroll
                for (int e = 0; e < 4; e++) zacc[mt][nt][e] = 0.f;
        // The 16-layer tile's chunk body is large (three MMAs per product with
        // BF16X3): fully unrolled over 8 chunks the loop outgrows the
        // instruction cache (no_instruction stalls 0.88 cycles per issue on
        // the precision-stress launch).  Same box, bit-identical, BF16X3 /
        // FP16 operands: unrolled by 8 315.7 / 256.4 us, by 4 303.5 / 248.2,
        // by 2 299.5 / 238.0, not unrolled 293-295 / 240 us.  The 8-layer
        // tile with 128 antennas (8 chunks) is unrolled by 4: 16 cells of
        // 106 PRB, BF16X3 94.7-96.6 -> 92.6-92.8 us (FP16 88.5 us either way).
#pragma unroll(LTF == 16 ? 1 : (LTF == 8 && NCH == 8 ? 4 : NCH))
        for (int k = 0; k < NCH; k++) {
            __syncwarp();                              // every lane is done with the slot refilled now
            const uint32_t pst = stBase + pslot * p.stageBytes;
            if (k + NST - 1 < NCH)
                stage_chunk<LTF, NCH>(pst, hLaneS, yLaneS, cur, k + NST - 1, lane);
            else if (hasNxt)
                stage_chunk<LTF, NCH>(pst, hLaneS, yLaneS, nxt, k + NST - 1 - NCH, lane);
            cp_async_commit();
            pslot = pslot == NST - 1 ? 0 : pslot + 1;
            cp_async_wait<NST - 1>();                  // this chunk's copies (own lane) have landed
            __syncwarp();                              // ... and every lane's
            mma_stage<LTF, P, true, true, SC>(stBase + cslot * p.stageBytes, HRS, CHUNK, LTF, yo, gacc, zacc, z2, g,
                                              c, ss);
            cslot = cslot == NST - 1 ? 0 : cslot + 1;
        }
        store_acc<LTF>(sm, gacc, zacc, q, g, c);
        cur = nxt;
        if (++q < nValid) continue;
        __syncwarp();
        {
            const FusedCell& cl = p.cell[ci];
            solve_group<LTF, P>(view_of(cl), (grp - cl.group0) * cl.GS, nValid, smemOff, lane);
        }
        q = 0;
        grp = nextGrp;
        if (grp >= total) break;
        while (ci + 1 < p.nCells && grp >= p.cell[ci + 1].group0) ci++;
        load_cell();
    }
    cp_async_wait<0>();
    walk_done(p, nw);
}

// ---------------------------------------------------------------------------
// FP16 I/O variant (cell format AERIAL_FMT_CF16): H and Y_rx are complex
// half (4 bytes) in HBM, Y_eq is written as complex half and the LLRs as
// __half.  Same tile, unrolled chunks and epilogue as fused_eq_kernel_a with
// FP16 operands; the staged samples ARE the MMA operand registers, so no
// conversion runs between shared memory and the tensor cores.
//
// Stage layout (bytes): 16 channel rows of LF half2 at stride hrs16_of(LF)
// (48 B for 8 layers, 16 B for 4), then up to 16 received rows of 64 B
// (16 antennas) whose 8-byte antenna-pair granules are XOR-swizzled by
// (sym & 2) << 1; both make every fragment read of a warp conflict-free.
// ---------------------------------------------------------------------------
// (2 layers: 8-byte rows, contiguous, so one 16-byte copy stages two rows)
__host__ __device__ constexpr int hrs16_of(int L) { return L == 16 ? 80 : L == 8 ? 48 : L == 4 ? 16 : 8; }

struct ScPtrH {
    const char* h;   // the lane's channel piece of the subcarrier's first chunk
    const char* y;   // the lane's received piece (row lane / 4, antennas 4 (lane % 4) ..)
    int yk;          // rows (lane / 4) and (lane / 4 + 8) below nSym: 0, 1 or 2
};

template <int LF, int NCH>
__device__ __forceinline__ void stage_chunk_h(uint32_t st, uint32_t hLaneS, uint32_t yLaneS, const ScPtrH& s,
                                              int j, int lane) {
    constexpr int NP = CHUNK * LF / 4;                 // 16-byte channel pieces per chunk
    constexpr int A = CHUNK * NCH;
    if (NP >= 32 || lane < NP) cp_async16(st + hLaneS, s.h + j * CHUNK * LF * 4);
    // 16 layers: 64 pieces, the second 32 are antenna rows 8-15
    if (NP > 32) cp_async16(st + hLaneS + 8 * hrs16_of(LF), s.h + j * CHUNK * LF * 4 + 512);
    if (s.yk > 0) cp_async16(st + yLaneS, s.y + j * 64);
    if (s.yk > 1) cp_async16(st + yLaneS + 512, s.y + j * 64 + 8 * A * 4);
}

__device__ __forceinline__ uint32_t lds32(uint32_t a) {
    uint32_t v;
    asm volatile("ld.shared.b32 %0, [%1];\n" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint2 lds64u(uint32_t a) {
    uint2 v;
    asm volatile("ld.shared.v2.b32 {%0, %1}, [%2];\n" : "=r"(v.x), "=r"(v.y) : "r"(a));
    return v;
}

// One full chunk: hb = stage + the lane's channel offset (antenna 2c, layer g),
// yo[kk][nt] = its received-pair offsets.
// 16 layers: two m-tiles (layers g and g + 8, 32 bytes apart in a row), the
// Gram blocks (0,0), (1,0), (1,1) and both matched-filter m-tiles, each
// accumulator fed in the complex64 kernel's order (mma_stage).
template <int LT>
__device__ __forceinline__ void mma_stage_h(uint32_t st, uint32_t hb, const uint32_t (&yo)[2][2],
                                            float (*gacc)[4], float (*zacc)[2][4], bool z2) {
    constexpr int HRS = hrs16_of(LT);
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
        const uint32_t h0 = lds32(hb + 8 * kk * HRS);
        const uint32_t h1 = lds32(hb + (8 * kk + 1) * HRS);
        const uint2 y0 = lds64u(st + yo[kk][0]);
        const uint2 y1 = lds64u(st + yo[kk][1]);
        const uint32_t r0 = jrot(h0), r1 = jrot(h1);
        mma16816<AERIAL_PREC_FP16>(gacc[0], h0, r0, h1, r1, h0, h1);
        mma16816<AERIAL_PREC_FP16>(zacc[0][0], h0, r0, h1, r1, y0.x, y0.y);
        if (z2) mma16816<AERIAL_PREC_FP16>(zacc[0][1], h0, r0, h1, r1, y1.x, y1.y);
        if constexpr (LT == 16) {
            const uint32_t u0 = lds32(hb + 8 * kk * HRS + 32);
            const uint32_t u1 = lds32(hb + (8 * kk + 1) * HRS + 32);
            const uint32_t q0 = jrot(u0), q1 = jrot(u1);
            mma16816<AERIAL_PREC_FP16>(gacc[1], u0, q0, u1, q1, h0, h1);
            mma16816<AERIAL_PREC_FP16>(gacc[2], u0, q0, u1, q1, u0, u1);
            mma16816<AERIAL_PREC_FP16>(zacc[1][0], u0, q0, u1, q1, y0.x, y0.y);
            if (z2) mma16816<AERIAL_PREC_FP16>(zacc[1][1], u0, q0, u1, q1, y1.x, y1.y);
        }
    }
}

template <int LTF, int NCH>
__global__ void __launch_bounds__(256, 2) fused_eq_kernel_h(const __grid_constant__ FusedParams p) {
    constexpr int NST = stages_of_a(LTF, NCH);
    constexpr int A = CHUNK * NCH;
    constexpr int HRS = hrs16_of(LTF);
    constexpr long HSCB = (long)A * LTF * 4;          // channel bytes per subcarrier
    extern __shared__ float4 smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warpsPerCta = blockDim.x >> 5;
    const int g = lane >> 2, c = lane & 3;
    const int warpBytes = p.epiBytes + NST * p.stageBytes;
    const int smemOff = wib * (warpBytes / 8);
    float2* sm = reinterpret_cast<float2*>(smem_raw) + smemOff;
    const uint32_t stBase =
        (uint32_t)__cvta_generic_to_shared(reinterpret_cast<char*>(smem_raw) + (long)wib * warpBytes + p.epiBytes);
    const long gw = (long)blockIdx.x * warpsPerCta + wib;
    const long nw = (long)gridDim.x * warpsPerCta;
    const long total = p.totalGroups;
    if (gw >= total) {
        walk_done(p, nw);
        return;
    }

    const int s0 = lane >> 2, q4 = lane & 3;
    const uint32_t hLaneS = LTF == 16 ? (lane >> 2) * HRS + (lane & 3) * 16
                          : LTF == 8  ? (lane >> 1) * HRS + (lane & 1) * 16
                                      : lane * HRS;
    const uint32_t yLaneS = CHUNK * HRS + s0 * 64 + ((q4 ^ (((s0 >> 1) & 1) << 1)) << 4);
    const long yLaneB = (long)(s0 * A + 4 * q4) * 4;

    auto first_sc = [&](int cell, long grp) -> ScPtrH {
        const FusedCell& cl = p.cell[cell];
        const long sc = (grp - cl.group0) * cl.GS;
        ScPtrH s;
        s.h = reinterpret_cast<const char*>(cl.H) + sc * HSCB + 16 * lane;
        s.y = reinterpret_cast<const char*>(cl.Y) + sc * cl.nSym * A * 4 + yLaneB;
        s.yk = (s0 < cl.nSym ? 1 : 0) + (s0 + 8 < cl.nSym ? 1 : 0);
        return s;
    };

    long grp = gw;
    int ci = 0;
    while (ci + 1 < p.nCells && grp >= p.cell[ci + 1].group0) ci++;
    int nValid, nSym;
    bool z2;
    uint32_t yo[2][2];
    auto load_cell = [&]() {
        const FusedCell& cl = p.cell[ci];
        nValid = group_valid(cl, grp);
        nSym = cl.nSym;
        z2 = nSym > 8;
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int r = 8 * nt + g;
                const int ra = r < nSym ? r : 0;         // rows past nSym are not staged: read row 0 instead
                yo[kk][nt] = CHUNK * HRS + ra * 64 + (((4 * kk + c) ^ ((ra & 2) << 1)) << 3);
            }
    };
    load_cell();
    ScPtrH cur = first_sc(ci, grp);
    const uint32_t hoff = 2 * c * HRS + 4 * g;

    int pslot = 0, cslot = 0;
#pragma unroll
    for (int j = 0; j < NST - 1; j++) {
        stage_chunk_h<LTF, NCH>(stBase + pslot * p.stageBytes, hLaneS, yLaneS, cur, j, lane);
        cp_async_commit();
        pslot = pslot == NST - 1 ? 0 : pslot + 1;
    }

    float gacc[3][4], zacc[2][2][4];
    int q = 0;
    long nextGrp = total;                                // the warp's next group, set with its last subcarrier
    while (true) {
        ScPtrH nxt = cur;
        bool hasNxt = true;
        if (q + 1 < nValid) {
            nxt.h = cur.h + HSCB;
            nxt.y = cur.y + (long)nSym * A * 4;
        } else {
            const long ng = walk_next(p, nw, grp + nw, lane);
            nextGrp = ng;
            hasNxt = ng < total;
            if (hasNxt) {
                int nc = ci;
                while (nc + 1 < p.nCells && ng >= p.cell[nc + 1].group0) nc++;
                nxt = first_sc(nc, ng);
            }
        }
        constexpr int NMT = LTF > 8 ? 2 : 1;
#pragma unroll
        for (int b = 0; b < (NMT == 2 ? 3 : 1); b++)
#pragma unroll
            for (int e = 0; e < 4; e++) gacc[b][e] = 0.f;
#pragma unroll
        for (int mt = 0; mt < NMT; mt++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++)
#pragma unroll
                for (int e = 0; e < 4; e++) zacc[mt][nt][e] = 0.f;
        // 16 layers: unrolled by 2 for the instruction cache (the 12-slot
        // complex-half precision-stress launch 180.7 -> 174.6 us, same box,
        // bit-identical)
#pragma unroll(LTF == 16 ? 2 : NCH)
        for (int k = 0; k < NCH; k++) {
            __syncwarp();                              // every lane is done with the slot refilled now
            const uint32_t pst = stBase + pslot * p.stageBytes;
            if (k + NST - 1 < NCH)
                stage_chunk_h<LTF, NCH>(pst, hLaneS, yLaneS, cur, k + NST - 1, lane);
            else if (hasNxt)
                stage_chunk_h<LTF, NCH>(pst, hLaneS, yLaneS, nxt, k + NST - 1 - NCH, lane);
            cp_async_commit();
            pslot = pslot == NST - 1 ? 0 : pslot + 1;
            cp_async_wait<NST - 1>();                  // this chunk's copies (own lane) have landed
            __syncwarp();                              // ... and every lane's
            const uint32_t st = stBase + cslot * p.stageBytes;
            mma_stage_h<LTF>(st, st + hoff, yo, gacc, zacc, z2);
            cslot = cslot == NST - 1 ? 0 : cslot + 1;
        }
        store_acc<LTF>(sm, gacc, zacc, q, g, c);
        cur = nxt;
        if (++q < nValid) continue;
        __syncwarp();
        {
            const FusedCell& cl = p.cell[ci];
            solve_group<LTF, AERIAL_PREC_FP16, true>(view_of(cl), (grp - cl.group0) * cl.GS, nValid, smemOff, lane);
        }
        q = 0;
        grp = nextGrp;
        if (grp >= total) break;
        while (ci + 1 < p.nCells && grp >= p.cell[ci + 1].group0) ci++;
        load_cell();
    }
    cp_async_wait<0>();
    walk_done(p, nw);
}

// ---------------------------------------------------------------------------
// FP16 I/O for a mixed batch: any mix of complex-half cells whose layers fill
// their tile (2, 4, 8 or 16) and whose antenna counts are multiples of 16.
// Staging, fragment reads and epilogue are fused_eq_kernel_h's per cell (the
// layer tile by switch, the chunk count at run time) and the group walk is
// the mixed-batch kernel's.
// ---------------------------------------------------------------------------
// Chunk j of one subcarrier: h / y are the lane's pieces of its first chunk.
template <int LF>
__device__ __forceinline__ void stage_chunk_hr(uint32_t st, uint32_t hLaneS, uint32_t yLaneS, const char* h,
                                               const char* y, int yk, int j, int A, int lane) {
    constexpr int NP = CHUNK * LF / 4;                 // 16-byte channel pieces per chunk
    if (NP >= 32 || lane < NP) cp_async16(st + hLaneS, h + j * CHUNK * LF * 4);
    if (NP > 32) cp_async16(st + hLaneS + 8 * hrs16_of(LF), h + j * CHUNK * LF * 4 + 512);
    if (yk > 0) cp_async16(st + yLaneS, y + j * 64);
    if (yk > 1) cp_async16(st + yLaneS + 512, y + j * 64 + 8 * A * 4);
}

// The lane's channel-piece offset in a stage for layer tile LT.
__host__ __device__ constexpr uint32_t h_lane_stage(int LT, int lane) {
    return LT == 16 ? (lane >> 2) * hrs16_of(16) + (lane & 3) * 16
         : LT == 8  ? (lane >> 1) * hrs16_of(8) + (lane & 1) * 16
         : LT == 4  ? lane * hrs16_of(4)
                    : lane * 16;                       // 2 layers: rows 2 lane, 2 lane + 1
}

__global__ void __launch_bounds__(256, 2) fused_eq_kernel_hg(const __grid_constant__ FusedParams p) {
    constexpr int NST = 2;
    extern __shared__ float4 smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warpsPerCta = blockDim.x >> 5;
    const int g = lane >> 2, c = lane & 3;
    const int warpBytes = p.epiBytes + NST * p.stageBytes;
    const int smemOff = wib * (warpBytes / 8);
    float2* sm = reinterpret_cast<float2*>(smem_raw) + smemOff;
    const uint32_t stBase =
        (uint32_t)__cvta_generic_to_shared(reinterpret_cast<char*>(smem_raw) + (long)wib * warpBytes + p.epiBytes);
    const long gw = (long)blockIdx.x * warpsPerCta + wib;
    const long nw = (long)gridDim.x * warpsPerCta;
    const long total = p.totalGroups;
    if (gw >= total) return;
    const int s0 = lane >> 2, q4 = lane & 3;

    // ---- producer cursor: group, cell, subcarrier, chunk ----
    long pg = gw;
    int pci = 0;
    while (pci + 1 < p.nCells && pg >= p.cell[pci + 1].group0) pci++;
    int pq = 0, pch = 0, pslot = 0, pValid, pNCh, pLT, pYk, pA, pHscB, pYscB;
    uint32_t pHLaneS, pYLaneS;
    const char* ph;
    const char* py;
    auto load_pcell = [&]() {
        const FusedCell& cl = p.cell[pci];
        const int hrs = hrs16_of(cl.L);
        pValid = group_valid(cl, pg);
        pLT = cl.LT;
        pA = cl.A;
        pNCh = cl.nChunk;
        pHscB = cl.A * cl.L * 4;
        pYscB = cl.nSym * cl.A * 4;
        const long sc = (pg - cl.group0) * cl.GS;
        ph = reinterpret_cast<const char*>(cl.H) + sc * pHscB + 16 * lane;
        py = reinterpret_cast<const char*>(cl.Y) + sc * pYscB + (s0 * cl.A + 4 * q4) * 4;
        pYk = (s0 < cl.nSym ? 1 : 0) + (s0 + 8 < cl.nSym ? 1 : 0);
        pHLaneS = h_lane_stage(pLT, lane);
        pYLaneS = CHUNK * hrs + s0 * 64 + ((q4 ^ (((s0 >> 1) & 1) << 1)) << 4);
    };
    load_pcell();
    auto produce = [&]() {
        if (pg < total) {
            const uint32_t st = stBase + pslot * p.stageBytes;
            switch (pLT) {
                case 2: stage_chunk_hr<2>(st, pHLaneS, pYLaneS, ph, py, pYk, pch, pA, lane); break;
                case 4: stage_chunk_hr<4>(st, pHLaneS, pYLaneS, ph, py, pYk, pch, pA, lane); break;
                case 8: stage_chunk_hr<8>(st, pHLaneS, pYLaneS, ph, py, pYk, pch, pA, lane); break;
                default: stage_chunk_hr<16>(st, pHLaneS, pYLaneS, ph, py, pYk, pch, pA, lane); break;
            }
            if (++pch == pNCh) {
                pch = 0;
                if (++pq < pValid) {
                    ph += pHscB;
                    py += pYscB;
                } else {
                    pq = 0;
                    pg += nw;
                    if (pg < total) {
                        while (pci + 1 < p.nCells && pg >= p.cell[pci + 1].group0) pci++;
                        load_pcell();
                    }
                }
            }
        }
        cp_async_commit();
        pslot = pslot == NST - 1 ? 0 : pslot + 1;
    };
    produce();

    // ---- consumer ----
    long grp = gw;
    int ci = 0;
    while (ci + 1 < p.nCells && grp >= p.cell[ci + 1].group0) ci++;
    int q = 0, ch = 0, cslot = 0, nValid, cNCh, cLT;
    bool z2;
    uint32_t yo[2][2], hoff;
    auto load_ccell = [&]() {
        const FusedCell& cl = p.cell[ci];
        const int hrs = hrs16_of(cl.L);
        nValid = group_valid(cl, grp);
        cNCh = cl.nChunk;
        cLT = cl.LT;
        z2 = cl.nSym > 8;
        hoff = 2 * c * hrs + 4 * g;
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int r = 8 * nt + g;
                const int ra = r < cl.nSym ? r : 0;      // rows past nSym are not staged: read row 0 instead
                yo[kk][nt] = CHUNK * hrs + ra * 64 + (((4 * kk + c) ^ ((ra & 2) << 1)) << 3);
            }
    };
    load_ccell();
    float gacc[3][4], zacc[2][2][4];
    auto clear_acc = [&]() {
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int e = 0; e < 4; e++) gacc[b][e] = 0.f;
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++)
#pragma unroll
                for (int e = 0; e < 4; e++) zacc[mt][nt][e] = 0.f;
    };
    clear_acc();
    while (true) {
        __syncwarp();                              // every lane is done with the slot refilled now
        produce();
        cp_async_wait<NST - 1>();                  // this chunk's copies (own lane) have landed
        __syncwarp();                              // ... and every lane's
        const uint32_t st = stBase + cslot * p.stageBytes;
        cslot = cslot == NST - 1 ? 0 : cslot + 1;
        switch (cLT) {
            case 2: mma_stage_h<2>(st, st + hoff, yo, gacc, zacc, z2); break;
            case 4: mma_stage_h<4>(st, st + hoff, yo, gacc, zacc, z2); break;
            case 8: mma_stage_h<8>(st, st + hoff, yo, gacc, zacc, z2); break;
            default: mma_stage_h<16>(st, st + hoff, yo, gacc, zacc, z2); break;
        }
        if (++ch < cNCh) continue;
        ch = 0;
        switch (cLT) {
            case 2: store_acc<2>(sm, gacc, zacc, q, g, c); break;
            case 4: store_acc<4>(sm, gacc, zacc, q, g, c); break;
            case 8: store_acc<8>(sm, gacc, zacc, q, g, c); break;
            default: store_acc<16>(sm, gacc, zacc, q, g, c); break;
        }
        clear_acc();
        if (++q < nValid) continue;
        __syncwarp();
        {
            const FusedCell& cl = p.cell[ci];
            const CellView v = view_of(cl);
            const long sc0 = (grp - cl.group0) * cl.GS;
            switch (cLT) {
                case 2: solve_group<2, AERIAL_PREC_FP16, true>(v, sc0, nValid, smemOff, lane); break;
                case 4: solve_group<4, AERIAL_PREC_FP16, true>(v, sc0, nValid, smemOff, lane); break;
                case 8: solve_group<8, AERIAL_PREC_FP16, true>(v, sc0, nValid, smemOff, lane); break;
                default: solve_group<16, AERIAL_PREC_FP16, true>(v, sc0, nValid, smemOff, lane); break;
            }
        }
        q = 0;
        grp += nw;
        if (grp >= total) break;
        while (ci + 1 < p.nCells && grp >= p.cell[ci + 1].group0) ci++;
        load_ccell();
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int layer_tile(int L) {
    int t = 1;
    while (t < L) t <<= 1;
    return t;
}

// The layer tile shared by every cell when each has nLayers == tile in
// {2, 4, 8, 16} and 16-byte aligned H / Y_rx; 0 otherwise (generic kernel).
static int exact_tile(const FusedParams& p) {
    const int lt = p.cell[0].LT;
    if (lt < 2) return 0;
    for (int i = 0; i < p.nCells; i++) {
        const FusedCell& c = p.cell[i];
        if (c.LT != lt || c.L != lt || !c.vecH || !c.vecY) return 0;
    }
    return lt;
}

}  // namespace aeq

// Power-of-two scale for a cell's FP16 operands, from its noise variance.
// FP16 keeps 11 significant bits only between 2^-14 and 65504, so H and Y_rx
// are rounded raw only while sigma2 lies in [2^-16, 2^7) (noise standard
// deviation 2^-8 ... 11.3: received samples up to about 75 dB above the
// noise stay below 65504, and channel taps 20 dB under it stay normal).
// Outside that window the operands are multiplied by s = 2^k with
// s^2 sigma2 in [2^-10, 2^-8) before rounding, and sigma2 by s^2: G, Z and
// G^-1 then scale by exact powers of two, which X = G^-1 Z, mu and the LLRs
// do not see.  sigma2 = 0 (zero forcing) or non-finite takes no scale.
extern "C" float aerial_fp16_operand_scale(float sigma2) {
    if (!(sigma2 > 0.f) || !(sigma2 < INFINITY)) return 1.f;
    int e = 0;
    (void)frexpf(sigma2, &e);             // sigma2 in [2^(e-1), 2^e)
    const int E = e - 1;
    if (E >= -16 && E <= 6) return 1.f;
    int k = (-10 - E) >= 0 ? (-10 - E + 1) / 2 : -((E + 10) / 2);   // ceil((-10 - E) / 2)
    k = k > 60 ? 60 : (k < -60 ? -60 : k);
    return ldexpf(1.f, k);
}

namespace aeq {

// Group size of every cell (min(32 / LT, cap)) and the first group index of
// each, in launch order.  Warps take groups round-robin (warp w: groups w,
// w + nw, ...).  Measured on the uneven 16-cell batch (configuration 4), same
// box, against this walk with cap 4 (54.3 us): a snake walk over cells sorted
// by estimated group cost 56.3 us, sorting alone 56.3-58.3 us, cap 8 with the
// plain walk 66.6 us; the autotuner's launch shapes recover 54.3 us in every
// variant, and no variant beats the plain walk.  Outputs are bit-identical
// across all of them.
void set_groups(FusedParams& p, int cap) {
    if (cap < 1) cap = kDefaultGroupCap;
    long g0 = 0;
    for (int i = 0; i < p.nCells; i++) {
        FusedCell& f = p.cell[i];
        f.GS = 32 / f.LT < cap ? 32 / f.LT : cap;
        f.group0 = g0;
        g0 += (f.nSC + f.GS - 1) / f.GS;
    }
    p.totalGroups = g0;
}

// warpBytes: the per-warp shared memory of the launch (epilogue region of the
// largest layer-tile footprint present, which is not monotonic in the tile,
// plus the kernel's operand stages).
int build_fused_params(const aerial_cell_desc* cells, int nCells, FusedParams& p, int& warpBytes) {
    if (!cells || nCells < 1 || nCells > kMaxCells) return AERIAL_ERR_INVALID_ARG;
    warpBytes = 0;
    for (int i = 0; i < nCells; i++) {
        const aerial_cell_desc& c = cells[i];
        if (c.nPRB < 1 || c.nPRB > AERIAL_MAX_PRB) return AERIAL_ERR_INVALID_ARG;
        const int nSC = c.nPRB * 12;
        if (!c.H || !c.Y_rx || !c.llr || c.nAnt < 1 || c.nAnt > AERIAL_MAX_ANTS || c.nLayers < 1 ||
            c.nLayers > AERIAL_MAX_LAYERS || c.nSym < 1 || c.nSym > AERIAL_MAX_SYMS || c.nPamBits < 1 ||
            c.nPamBits > 4 || !(c.sigma2 >= 0.f))
            return AERIAL_ERR_INVALID_ARG;
        if (((uintptr_t)c.H & 7) || ((uintptr_t)c.Y_rx & 7) || ((uintptr_t)c.llr & 7) || ((uintptr_t)c.Y_eq & 7))
            return AERIAL_ERR_INVALID_ARG;
        FusedCell& f = p.cell[i];
        f.H = (const float2*)c.H;
        f.Y = (const float2*)c.Y_rx;
        f.llr = c.llr;
        f.yeq = (float2*)c.Y_eq;
        f.sigma2 = c.sigma2;
        f.scale = 1.f;                  // set_operand_scale decides, once the precision is known
        f.nSC = nSC;
        f.A = c.nAnt;
        f.L = c.nLayers;
        f.nSym = c.nSym;
        f.nPam = c.nPamBits;
        f.LT = layer_tile(c.nLayers);
        f.vecY = ((c.nAnt % 2) == 0 && ((uintptr_t)c.Y_rx & 15) == 0) ? 1 : 0;
        f.vecH = ((c.nLayers % 2) == 0 && ((uintptr_t)c.H & 15) == 0) ? 1 : 0;
        {
            const int half = c.nLayers / 2;
            f.lgHalfL = (half > 0 && (half & (half - 1)) == 0) ? __builtin_ctz(half) : -1;
        }
        f.lut = pam_lut(c.nPamBits);
        f.nChunk = (c.nAnt + CHUNK - 1) / CHUNK;
        f.hrs = hrs_of(c.nLayers);
        // LLR rows of 2*nPam floats are written as float4 for nPam 2/4: need 16 B alignment
        if ((c.nPamBits == 2 || c.nPamBits == 4) && ((uintptr_t)c.llr & 15)) return AERIAL_ERR_INVALID_ARG;
    }
    p.nCells = nCells;
    p.scaled = 0;
    p.walkSlot = -1;
    set_groups(p, kDefaultGroupCap);
    p.fmt = cells[0].format;
    for (int i = 0; i < nCells; i++)
        if (cells[i].format != p.fmt || (p.fmt != AERIAL_FMT_CF32 && p.fmt != AERIAL_FMT_CF16))
            return AERIAL_ERR_INVALID_ARG;
    p.epiBytes = epi_bytes_of(p);
    p.stageBytes = stage_bytes_of(p);
    p.exactTile = exact_tile(p);
    p.exactChunks = 0;
    if (p.exactTile) {
        const int a = p.cell[0].A;
        // 16-layer tiles unroll too: on the 12-slot 273 PRB x 128 antenna
        // launch, same box, 277 against 302 us with FP16 operands and 359
        // against 365 us with BF16X3, bit-identical (the runtime chunk loop
        // of the 16-layer tile spills registers, the unrolled one does not)
        bool same = a == 32 || a == 64 || a == 128;
        for (int i = 1; i < nCells && same; i++) same = p.cell[i].A == a;
        if (same) p.exactChunks = a / CHUNK;
    }
    p.halfMixed = 0;
    if (p.fmt == AERIAL_FMT_CF16) {
        // half-format cells run an FP16 I/O kernel: a uniform batch of exact
        // 4-, 8- or 16-layer tiles with 32 / 64 / 128 antennas takes the
        // unrolled one; any other mix whose cells fill 2-, 4-, 8- or 16-layer
        // tiles with a multiple of 16 antennas takes the mixed-batch one.
        // H and Y_rx must be 16-byte aligned.
        if (p.exactTile == 16) {
            const int a = p.cell[0].A;
            bool same = a == 32 || a == 64 || a == 128;
            for (int i = 1; i < nCells && same; i++) same = p.cell[i].A == a;
            p.exactChunks = same ? a / CHUNK : 0;
        }
        if ((p.exactTile != 4 && p.exactTile != 8 && p.exactTile != 16) || !p.exactChunks) {
            for (int i = 0; i < nCells; i++) {
                const FusedCell& f = p.cell[i];
                if (f.L != f.LT || f.LT < 2 || f.A % CHUNK || ((uintptr_t)f.H & 15) || ((uintptr_t)f.Y & 15))
                    return AERIAL_ERR_UNSUPPORTED;
            }
            p.halfMixed = 1;
            p.exactTile = 0;
            p.exactChunks = 0;
        }
        int b = 0;
        for (int i = 0; i < nCells; i++) {
            const int v = CHUNK * hrs16_of(p.cell[i].L) + 64 * p.cell[i].nSym;
            b = v > b ? v : b;
        }
        p.stageBytes = (b + 15) & ~15;
    }
    p.nStages = p.exactChunks ? stages_of_a(p.exactTile, p.exactChunks) : stages_of(p.exactTile);
    warpBytes = p.epiBytes + p.nStages * p.stageBytes;
    return AERIAL_OK;
}

// FP16 operands from complex64 cells: each cell's power-of-two scale
// (aerial_fp16_operand_scale) and its sigma2 in the scaled units; p.scaled
// selects the kernels that apply it.  Other precisions keep the FP32 range
// and complex-half cells are read as stored: no scale.  Call once per
// parameter block, after build_fused_params.
//
// FP16X3 operands are always normalized, to s^2 sigma2 in [1/4, 1): the low
// half of each split then stays a normal half (22 significant bits in all)
// for channel taps down to about 40 dB under the noise, and received samples
// up to about 90 dB above it stay below 65504.  Its kernels always apply the
// scale (a cell with s = 1 multiplies by one).
static float fp16x3_operand_scale(float sigma2) {
    if (!(sigma2 > 0.f) || !(sigma2 < INFINITY)) return 1.f;
    int e = 0;
    (void)frexpf(sigma2, &e);             // sigma2 in [2^(e-1), 2^e)
    const int E = e - 1;
    int k = (-2 - E) >= 0 ? (-2 - E + 1) / 2 : -((E + 2) / 2);      // ceil((-2 - E) / 2)
    k = k > 60 ? 60 : (k < -60 ? -60 : k);
    return ldexpf(1.f, k);
}

void set_operand_scale(FusedParams& p, int prec) {
    p.scaled = prec == AERIAL_PREC_FP16X3 ? 1 : 0;
    for (int i = 0; i < p.nCells; i++) {
        FusedCell& f = p.cell[i];
        f.scale = 1.f;
        if (p.fmt != AERIAL_FMT_CF32) continue;
        float s = 1.f;
        if (prec == AERIAL_PREC_FP16) s = aerial_fp16_operand_scale(f.sigma2);
        else if (prec == AERIAL_PREC_FP16X3) s = fp16x3_operand_scale(f.sigma2);
        if (s != 1.f) {
            f.scale = s;
            f.sigma2 = f.sigma2 * s * s;      // exact: s is a power of two
            p.scaled = 1;
        }
    }
}

struct LaunchShape {
    int warps, ctasPerSm;
};

// Launch shapes are limited by 16 resident warps per SM (128 registers per
// thread) and by shared memory (operand ring + epilogue region per warp).
constexpr int kSmemPerSm = 220 * 1024;
constexpr int kWarpsPerSm = 16;

static int max_ctas(int warps, int warpBytes) {
    int k = kSmemPerSm / (warps * warpBytes);
    if (k > kWarpsPerSm / warps) k = kWarpsPerSm / warps;
    if (k > 8) k = 8;
    return k;
}

// Four-warp CTAs, as many per SM as fit; smaller CTAs only where a four-warp
// CTA does not fit.  Smaller CTAs can pack more warps into the leftover shared
// memory, but that measured slower where it happens for the standard shapes:
// 64 100 MHz slots (8 layers, 64 antennas; 15 KB per warp), same box, 4 x 3
// (12 resident warps) 213.6 us and 2 x 6 213.6 us against 228 us for 2 x 7
// (14 warps); BF16X3 operands 230 against 244 us.  Where both reach 16 warps
// (the 4-layer 20 MHz slots) the four-warp CTAs were the fastest too.
static LaunchShape default_shape(int warpBytes) {
    for (int w : {4, 3, 2}) {
        const int k = max_ctas(w, warpBytes);
        if (k >= 1) return {w, k};
    }
    return {1, max_ctas(1, warpBytes) > 0 ? max_ctas(1, warpBytes) : 1};
}

// A resolved launch: kernel instantiation, grid, block and dynamic shared
// memory.  Resolving also raises the kernel's shared-memory limit once.
struct LaunchPlan {
    const void* func;
    dim3 grid, block;
    int smem;
};

// Grid: enough CTAs for every group, at most ctasPerSm per SM.
static void fill_plan(const void* func, const FusedParams& p, int warpBytes, LaunchShape sh, LaunchPlan& out) {
    long need = (p.totalGroups + sh.warps - 1) / sh.warps;
    long grid = (long)sm_count() * sh.ctasPerSm;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    out.func = func;
    out.grid = dim3((unsigned)grid);
    out.block = dim3(sh.warps * 32);
    out.smem = sh.warps * warpBytes;
}

template <int P, int LTF, bool SC>
static int plan_v(const FusedParams& p, int warpBytes, LaunchShape sh, LaunchPlan& out) {
    const int s = allow_max_smem<fused_eq_kernel<P, LTF, SC>>();
    if (s) return s;
    fill_plan(reinterpret_cast<const void*>(fused_eq_kernel<P, LTF, SC>), p, warpBytes, sh, out);
    return AERIAL_OK;
}

template <int P, int LTF, int NCH, bool SC>
static int plan_a(const FusedParams& p, int warpBytes, LaunchShape sh, LaunchPlan& out) {
    const int s = allow_max_smem<fused_eq_kernel_a<P, LTF, NCH, SC>>();
    if (s) return s;
    fill_plan(reinterpret_cast<const void*>(fused_eq_kernel_a<P, LTF, NCH, SC>), p, warpBytes, sh, out);
    return AERIAL_OK;
}

template <int P, int LTF, bool SC>
static int plan_an(const FusedParams& p, int warpBytes, LaunchShape sh, LaunchPlan& out) {
    switch (p.exactChunks) {
        case 2: return plan_a<P, LTF, 2, SC>(p, warpBytes, sh, out);
        case 4: return plan_a<P, LTF, 4, SC>(p, warpBytes, sh, out);
        default: return plan_a<P, LTF, 8, SC>(p, warpBytes, sh, out);
    }
}

template <int LTF, int NCH>
static int plan_h(const FusedParams& p, int warpBytes, LaunchShape sh, LaunchPlan& out) {
    const int s = allow_max_smem<fused_eq_kernel_h<LTF, NCH>>();
    if (s) return s;
    fill_plan(reinterpret_cast<const void*>(fused_eq_kernel_h<LTF, NCH>), p, warpBytes, sh, out);
    return AERIAL_OK;
}

template <int LTF>
static int plan_hn(const FusedParams& p, int warpBytes, LaunchShape sh, LaunchPlan& out) {
    switch (p.exactChunks) {
        case 2: return plan_h<LTF, 2>(p, warpBytes, sh, out);
        case 4: return plan_h<LTF, 4>(p, warpBytes, sh, out);
        default: return plan_h<LTF, 8>(p, warpBytes, sh, out);
    }
}

template <int P, bool SC>
static int plan_p(const FusedParams& p, int warpBytes, LaunchShape sh, LaunchPlan& out) {
    if (p.fmt == AERIAL_FMT_CF16) {
        if (P != AERIAL_PREC_FP16) return AERIAL_ERR_UNSUPPORTED;
        if (p.halfMixed) {
            const int s = allow_max_smem<fused_eq_kernel_hg>();
            if (s) return s;
            fill_plan(reinterpret_cast<const void*>(fused_eq_kernel_hg), p, warpBytes, sh, out);
            return AERIAL_OK;
        }
        return p.exactTile == 4   ? plan_hn<4>(p, warpBytes, sh, out)
             : p.exactTile == 8   ? plan_hn<8>(p, warpBytes, sh, out)
                                  : plan_hn<16>(p, warpBytes, sh, out);
    }
    if (p.exactChunks) {
        switch (p.exactTile) {
            case 2: return plan_an<P, 2, SC>(p, warpBytes, sh, out);
            case 4: return plan_an<P, 4, SC>(p, warpBytes, sh, out);
            case 8: return plan_an<P, 8, SC>(p, warpBytes, sh, out);
            default: return plan_an<P, 16, SC>(p, warpBytes, sh, out);
        }
    }
    switch (p.exactTile) {
        case 2: return plan_v<P, 2, SC>(p, warpBytes, sh, out);
        case 4: return plan_v<P, 4, SC>(p, warpBytes, sh, out);
        case 8: return plan_v<P, 8, SC>(p, warpBytes, sh, out);
        case 16: return plan_v<P, 16, SC>(p, warpBytes, sh, out);
        default: return plan_v<P, 0, SC>(p, warpBytes, sh, out);
    }
}

int plan_fused(const FusedParams& p, int warpBytes, int prec, LaunchShape sh, LaunchPlan& out) {
    if (sh.warps < 1 || sh.warps > 8 || sh.ctasPerSm < 1 || sh.ctasPerSm > 8) return AERIAL_ERR_INVALID_ARG;
    if ((long)sh.warps * warpBytes * sh.ctasPerSm > 227 * 1024 || (long)sh.warps * warpBytes > 227 * 1024)
        return AERIAL_ERR_UNSUPPORTED;
    switch (prec) {
        case AERIAL_PREC_FP16:
            return p.scaled ? plan_p<AERIAL_PREC_FP16, true>(p, warpBytes, sh, out)
                            : plan_p<AERIAL_PREC_FP16, false>(p, warpBytes, sh, out);
        case AERIAL_PREC_BF16: return plan_p<AERIAL_PREC_BF16, false>(p, warpBytes, sh, out);
        case AERIAL_PREC_BF16X3: return plan_p<AERIAL_PREC_BF16X3, false>(p, warpBytes, sh, out);
        case AERIAL_PREC_FP16X3: return plan_p<AERIAL_PREC_FP16X3, true>(p, warpBytes, sh, out);
        default: return AERIAL_ERR_UNSUPPORTED;
    }
}

// ---------------------------------------------------------------------------
// Slots of the dynamic group walk, per device.  A stream that launches the
// fused kernel holds one (matched by its process-unique stream ID) and a
// graph reserves one for its lifetime.  The table's lock is held from the
// choice of a slot to the event recorded behind the launch, and a slot passes
// to another stream or a graph only once that event has completed, so two
// launches that may run at the same time never share a counter.  A launch
// being captured into a graph, one that finds no slot free, and every launch
// while AERIAL_STATIC_WALK is set to a non-zero value take the static walk.
// ---------------------------------------------------------------------------
struct WalkSlot {
    unsigned long long stream = 0;   // 1 + ID of the owning stream, 0 if none
    bool graph = false;              // reserved by a graph (or retired after a failed record)
    cudaEvent_t last = nullptr;      // recorded behind the slot's latest launch
};
struct WalkTable {
    unsigned long long ctx = 0;      // context the slots (and their events) belong to, 0 if unused
    WalkSlot s[kWalkSlots];
};
// A device's tables, one per context (the device's primary context, or a
// new one after a device reset): a table is never handed to another context,
// and a launch in a fifth context on one device takes the static walk.
constexpr int kWalkContexts = 4;
struct WalkDevice {
    std::mutex m;
    WalkTable t[kWalkContexts];
};
static WalkDevice g_walk_devices[kMaxDevices];

static bool walk_static_forced() {
    const char* e = std::getenv("AERIAL_STATIC_WALK");
    return e && e[0] && !(e[0] == '0' && e[1] == 0);
}

// The current context's table with its device's lock taken, or nullptr
// (static walk).
static WalkTable* walk_table_locked(std::unique_lock<std::mutex>& lk, int* devOut = nullptr) {
    if (walk_static_forced()) return nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    if (dev < 0 || dev >= kMaxDevices) return nullptr;
    const unsigned long long ctx = current_ctx_id();
    if (ctx == 0) return nullptr;
    WalkDevice& d = g_walk_devices[dev];
    lk = std::unique_lock<std::mutex>(d.m);
    WalkTable* t = nullptr;
    for (WalkTable& c : d.t)
        if (c.ctx == ctx) t = &c;
    for (int k = 0; k < kWalkContexts && !t; k++)
        if (d.t[k].ctx == 0) {
            t = &d.t[k];
            t->ctx = ctx;
        }
    if (!t) {
        lk.unlock();
        return nullptr;
    }
    if (devOut) *devOut = dev;
    return t;
}

// The unrolled kernels (uniform batches) take the dynamic walk: they ask for
// their next group a subcarrier ahead of needing it.  The mixed-tile kernels'
// producer cursor would ask at the moment it stages the group, and on the
// uneven 16-cell batch that measured slower (57.4-58.2 against 54.3 us; with
// the ticket taken a whole group ahead still 58.4 against 54.2 us), so they
// keep the static walk.
static bool walk_applies(const FusedParams& p) { return p.exactChunks != 0 && !p.halfMixed; }

static bool walk_slot_idle(WalkSlot& w) {
    if (!w.last) return true;
    if (cudaEventQuery(w.last) == cudaSuccess) return true;
    (void)cudaGetLastError();        // not ready (its launch still runs): not an error, clear it
    return false;
}

static int walk_free_slot(WalkTable* t) {
    for (int i = 0; i < kWalkSlots; i++)
        if (!t->s[i].graph && !t->s[i].stream && !t->s[i].last) return i;
    for (int i = 0; i < kWalkSlots; i++)
        if (!t->s[i].graph && walk_slot_idle(t->s[i])) return i;
    return -1;
}

static int walk_slot_for_stream(WalkTable* t, cudaStream_t st) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    unsigned long long id = 0;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone ||
        cudaStreamGetId(st, &id) != cudaSuccess) {
        (void)cudaGetLastError();
        return -1;
    }
    for (int i = 0; i < kWalkSlots; i++)
        if (!t->s[i].graph && t->s[i].stream == id + 1) return i;
    const int i = walk_free_slot(t);
    if (i >= 0) t->s[i].stream = id + 1;
    return i;
}

// The event behind a launch that used slot i on stream st.  If it cannot be
// recorded the slot's state is unknown, and the slot is retired.
static int walk_record(WalkTable* t, int i, cudaStream_t st) {
    WalkSlot& w = t->s[i];
    cudaError_t e = cudaSuccess;
    if (!w.last) e = cudaEventCreateWithFlags(&w.last, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(w.last, st);
    if (e != cudaSuccess) {
        w.graph = true;
        w.stream = 0;
    }
    return rt_status(e);
}

int launch_fused(FusedParams& p, int warpBytes, int prec, LaunchShape sh, cudaStream_t st) {
    LaunchPlan pl;
    int s = plan_fused(p, warpBytes, prec, sh, pl);
    if (s) return s;
    std::unique_lock<std::mutex> lk;
    WalkTable* t = walk_applies(p) ? walk_table_locked(lk) : nullptr;
    p.walkSlot = t ? walk_slot_for_stream(t, st) : -1;
    void* args[] = {&p};
    const cudaError_t e = cudaLaunchKernel(pl.func, pl.grid, pl.block, args, (size_t)pl.smem, st);
    if (e != cudaSuccess) return rt_status(e);
    return p.walkSlot >= 0 ? walk_record(t, p.walkSlot, st) : AERIAL_OK;
}

// Resolve precision and launch shape from an optional tuning struct.
// A shape tuned on one batch may be applied to another whose cells need more
// shared memory per warp (a host-pipeline sub-batch, say): its CTAs per SM
// are then reduced to what fits instead of failing the launch.
static void resolve_tuning(const aerial_tuning* tuning, int warpBytes, int& prec, LaunchShape& sh, int& gsCap) {
    sh = default_shape(warpBytes);
    prec = AERIAL_PREC_FP16;
    gsCap = kDefaultGroupCap;
    if (tuning) {
        prec = tuning->precision;
        if (tuning->sc_per_group > 0) gsCap = tuning->sc_per_group;
        if (tuning->warps_per_cta) sh.warps = tuning->warps_per_cta;
        if (tuning->ctas_per_sm) sh.ctasPerSm = tuning->ctas_per_sm;
        if (sh.warps >= 1 && sh.ctasPerSm > 1 && (long)sh.warps * warpBytes * sh.ctasPerSm > kSmemPerSm) {
            const int k = kSmemPerSm / (sh.warps * warpBytes);
            sh.ctasPerSm = k >= 1 ? k : 1;
        }
    }
}

}  // namespace aeq

using namespace aeq;

extern "C" int aerial_pusch_eq_fused(const aerial_cell_desc* cells, int nCells, const aerial_tuning* tuning,
                                     void* stream) {
    FusedParams p;
    int warpBytes = 0;
    int s = build_fused_params(cells, nCells, p, warpBytes);
    if (s) return s;
    LaunchShape sh;
    int prec, gsCap;
    resolve_tuning(tuning, warpBytes, prec, sh, gsCap);
    if (gsCap != kDefaultGroupCap) set_groups(p, gsCap);
    set_operand_scale(p, prec);
    return launch_fused(p, warpBytes, prec, sh, to_stream(stream));
}

// ---------------------------------------------------------------------------
// Autotuner: time each candidate tile and launch shape on the caller's cells
// and keep the fastest.  Candidates are the group cap (subcarriers solved
// together per warp: 4, 8 or 32, for batches with tiles of 4 layers or fewer,
// where the cap changes anything) crossed with (warps per CTA, CTAs per SM)
// pairs whose shared memory fits one SM; each is timed with CUDA events over
// a few launches after one warm-up launch.  The reference's analogue is its
// templated shape sweep over antennas and symbols (src/coef_scaling.cu:221-250).
// ---------------------------------------------------------------------------
extern "C" int aerial_autotune(const aerial_cell_desc* cells, int nCells, aerial_tuning* best, float* bestUs,
                               void* stream) {
    if (!best) return AERIAL_ERR_INVALID_ARG;
    FusedParams base, p;
    int warpBytes = 0;
    int s = build_fused_params(cells, nCells, base, warpBytes);
    if (s) return s;
    cudaStream_t st = to_stream(stream);
    const int prec = best->precision;
    struct Cand {
        LaunchShape sh;
        int cap;
    };
    int caps[3] = {kDefaultGroupCap, 0, 0}, nCaps = 1;
    bool smallTile = false;
    for (int i = 0; i < base.nCells; i++) smallTile |= base.cell[i].LT <= 4;
    if (smallTile) {
        caps[nCaps++] = 8;
        caps[nCaps++] = 32;
    }
    Cand cand[48];
    int nc = 0;
    const LaunchShape def = default_shape(warpBytes);
    for (int ic = 0; ic < nCaps; ic++) {
        bool hasDef = false;
        for (int w : {2, 3, 4, 6, 8}) {
            const int k = max_ctas(w, warpBytes);
            if (k >= 1) cand[nc++] = {{w, k}, caps[ic]};
            if (k >= 2) cand[nc++] = {{w, k - 1}, caps[ic]};
            hasDef |= w == def.warps && ((k >= 1 && k == def.ctasPerSm) || (k >= 2 && k - 1 == def.ctasPerSm));
        }
        if (!hasDef) cand[nc++] = {def, caps[ic]};
    }
    // Rounds interleave the candidates so clock drift under the power cap
    // hits all of them alike; a candidate's time is its best round.  Within
    // 2 % of the fastest, the shape with more resident warps wins (it holds
    // more operand copies in flight once clocks settle), then the default cap.
    float t[48];
    for (int ic = 0; ic < nc; ic++) t[ic] = 1e30f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int rounds = 3, reps = 8;
    for (int rd = 0; rd < rounds && !s; rd++) {
        for (int ic = 0; ic < nc && !s; ic++) {
            const LaunchShape& sh = cand[ic].sh;
            p = base;                                // unscaled sigma2, default groups
            set_groups(p, cand[ic].cap);
            set_operand_scale(p, prec);
            if ((s = launch_fused(p, warpBytes, prec, sh, st))) break;
            cudaEventRecord(e0, st);
            for (int r = 0; r < reps && !s; r++) s = launch_fused(p, warpBytes, prec, sh, st);
            cudaEventRecord(e1, st);
            if (s) break;
            cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) {
                s = rt_status(e);
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= reps;
            t[ic] = ms < t[ic] ? ms : t[ic];
        }
    }
    float fastest = 1e30f;
    for (int ic = 0; ic < nc; ic++) fastest = t[ic] < fastest ? t[ic] : fastest;
    Cand bestC{def, kDefaultGroupCap};
    float bestT = 1e30f;
    int bestWarps = -1;
    for (int ic = 0; ic < nc; ic++) {
        if (t[ic] > fastest * 1.02f) continue;
        const int w = cand[ic].sh.warps * cand[ic].sh.ctasPerSm;
        const bool better = w > bestWarps ||
                            (w == bestWarps && cand[ic].cap == kDefaultGroupCap && bestC.cap != kDefaultGroupCap) ||
                            (w == bestWarps && cand[ic].cap == bestC.cap && t[ic] < bestT);
        if (better) {
            bestWarps = w;
            bestT = t[ic];
            bestC = cand[ic];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s) return s;
    best->warps_per_cta = bestC.sh.warps;
    best->ctas_per_sm = bestC.sh.ctasPerSm;
    best->sc_per_group = bestC.cap;
    if (bestUs) *bestUs = bestT * 1000.f;
    return AERIAL_OK;
}

// ---------------------------------------------------------------------------
// CUDA graph of the persistent launch.  The graph holds one kernel node built
// directly (no stream capture); aerial_eq_graph_update re-points it at new
// slot buffers / noise levels of the same cell shapes with
// cudaGraphExecKernelNodeSetParams, so a slot loop replays one executable
// graph per slot without re-instantiation.
// ---------------------------------------------------------------------------
struct aerial_eq_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t node = nullptr;
    FusedParams params;
    LaunchPlan plan;
    int prec = AERIAL_PREC_FP16;
    LaunchShape shape{};
    int gsCap = kDefaultGroupCap;
    int dev = -1;                    // device of the graph's walk slot (params.walkSlot)
    WalkTable* walk = nullptr;       // table of that slot
};

static void release_walk_slot(aerial_eq_graph* g) {
    const int i = g->params.walkSlot;
    if (i < 0 || !g->walk) return;
    std::lock_guard<std::mutex> lk(g_walk_devices[g->dev].m);
    g->walk->s[i].graph = false;     // reusable once the event behind its last replay completes
}

static cudaKernelNodeParams node_params(aerial_eq_graph* g, void** args) {
    cudaKernelNodeParams kp{};
    kp.func = const_cast<void*>(g->plan.func);
    kp.gridDim = g->plan.grid;
    kp.blockDim = g->plan.block;
    kp.sharedMemBytes = (unsigned)g->plan.smem;
    kp.kernelParams = args;
    kp.extra = nullptr;
    return kp;
}

extern "C" int aerial_eq_graph_create(const aerial_cell_desc* cells, int nCells, const aerial_tuning* tuning,
                                      aerial_eq_graph** out) {
    if (!out) return AERIAL_ERR_INVALID_ARG;
    *out = nullptr;
    aerial_eq_graph* g = new aerial_eq_graph();
    int warpBytes = 0;
    int s = build_fused_params(cells, nCells, g->params, warpBytes);
    if (!s) {
        resolve_tuning(tuning, warpBytes, g->prec, g->shape, g->gsCap);
        if (g->gsCap != kDefaultGroupCap) set_groups(g->params, g->gsCap);
        set_operand_scale(g->params, g->prec);
        s = plan_fused(g->params, warpBytes, g->prec, g->shape, g->plan);
    }
    if (!s) {
        // the graph's own walk slot: its replays are ordered among themselves
        std::unique_lock<std::mutex> lk;
        WalkTable* t = walk_applies(g->params) ? walk_table_locked(lk, &g->dev) : nullptr;
        int held = 0;                // graphs hold at most kWalkSlots - 16: streams keep slots
        for (int k = 0; t && k < kWalkSlots; k++) held += t->s[k].graph ? 1 : 0;
        const int i = t && held < kWalkSlots - 16 ? walk_free_slot(t) : -1;
        if (i >= 0) {
            t->s[i].graph = true;
            t->s[i].stream = 0;
            g->walk = t;
        }
        g->params.walkSlot = i;
    }
    cudaError_t e = cudaSuccess;
    if (!s) e = cudaGraphCreate(&g->graph, 0);
    if (!s && e == cudaSuccess) {
        void* args[] = {&g->params};
        cudaKernelNodeParams kp = node_params(g, args);
        e = cudaGraphAddKernelNode(&g->node, g->graph, nullptr, 0, &kp);
    }
    if (!s && e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (!s && e != cudaSuccess) s = rt_status(e);
    if (s) {
        if (g->exec) cudaGraphExecDestroy(g->exec);
        if (g->graph) cudaGraphDestroy(g->graph);
        release_walk_slot(g);
        delete g;
        return s;
    }
    *out = g;
    return AERIAL_OK;
}

extern "C" int aerial_eq_graph_update(aerial_eq_graph* g, const aerial_cell_desc* cells, int nCells) {
    if (!g || !cells || nCells != g->params.nCells) return AERIAL_ERR_INVALID_ARG;
    FusedParams np;
    int warpBytes = 0;
    int s = build_fused_params(cells, nCells, np, warpBytes);
    if (s) return s;
    for (int i = 0; i < nCells; i++) {
        const FusedCell &a = np.cell[i], &b = g->params.cell[i];
        if (a.nSC != b.nSC || a.A != b.A || a.L != b.L || a.nSym != b.nSym || a.nPam != b.nPam ||
            a.vecH != b.vecH || a.vecY != b.vecY || np.fmt != g->params.fmt)
            return AERIAL_ERR_UNSUPPORTED;      // a new shape or format needs a new graph
    }
    // The new noise levels may move a cell in or out of FP16 operand scaling,
    // which selects another kernel instantiation: re-plan the node (an
    // executable graph's kernel node may change its function).
    if (g->gsCap != kDefaultGroupCap) set_groups(np, g->gsCap);
    set_operand_scale(np, g->prec);
    np.walkSlot = g->params.walkSlot;
    LaunchPlan pl;
    s = plan_fused(np, warpBytes, g->prec, g->shape, pl);
    if (s) return s;
    g->params = np;
    g->plan = pl;
    void* args[] = {&g->params};
    cudaKernelNodeParams kp = node_params(g, args);
    cudaError_t e = cudaGraphExecKernelNodeSetParams(g->exec, g->node, &kp);
    return rt_status(e);
}

extern "C" int aerial_eq_graph_launch(aerial_eq_graph* g, void* stream) {
    if (!g) return AERIAL_ERR_INVALID_ARG;
    const int i = g->params.walkSlot;
    if (i < 0 || !g->walk) return rt_status(cudaGraphLaunch(g->exec, to_stream(stream)));
    std::lock_guard<std::mutex> lk(g_walk_devices[g->dev].m);
    const cudaError_t e = cudaGraphLaunch(g->exec, to_stream(stream));
    if (e != cudaSuccess) return rt_status(e);
    return walk_record(g->walk, i, to_stream(stream));
}

extern "C" int aerial_eq_graph_destroy(aerial_eq_graph* g) {
    if (!g) return AERIAL_ERR_INVALID_ARG;
    cudaError_t e1 = g->exec ? cudaGraphExecDestroy(g->exec) : cudaSuccess;
    cudaError_t e2 = g->graph ? cudaGraphDestroy(g->graph) : cudaSuccess;
    release_walk_slot(g);
    delete g;
    const int s1 = rt_status(e1), s2 = rt_status(e2);
    return s1 ? s1 : s2;
}

namespace aeq {

// ---------------------------------------------------------------------------
// Load every fused-kernel instantiation on the current device and raise its
// shared-memory limit, so the first launch of a variant inside a latency-
// critical loop does not pay module loading.
// ---------------------------------------------------------------------------
template <int P, int LTF, bool SC>
static int prepare_v() {
    cudaFuncAttributes at;
    const cudaError_t e = cudaFuncGetAttributes(&at, fused_eq_kernel<P, LTF, SC>);
    return e == cudaSuccess ? allow_max_smem<fused_eq_kernel<P, LTF, SC>>() : rt_status(e);
}

template <int P, int LTF, int NCH, bool SC>
static int prepare_a() {
    cudaFuncAttributes at;
    const cudaError_t e = cudaFuncGetAttributes(&at, fused_eq_kernel_a<P, LTF, NCH, SC>);
    return e == cudaSuccess ? allow_max_smem<fused_eq_kernel_a<P, LTF, NCH, SC>>() : rt_status(e);
}

template <int P, int LTF, bool SC>
static int prepare_an() {
    int s = prepare_a<P, LTF, 2, SC>();
    if (!s) s = prepare_a<P, LTF, 4, SC>();
    if (!s) s = prepare_a<P, LTF, 8, SC>();
    return s;
}

template <int LTF, int NCH>
static int prepare_h() {
    cudaFuncAttributes at;
    const cudaError_t e = cudaFuncGetAttributes(&at, fused_eq_kernel_h<LTF, NCH>);
    return e == cudaSuccess ? allow_max_smem<fused_eq_kernel_h<LTF, NCH>>() : rt_status(e);
}

template <int P, bool SC = false>
static int prepare_p() {
    int s = prepare_an<P, 2, SC>();
    if (!s) s = prepare_an<P, 4, SC>();
    if (!s) s = prepare_an<P, 8, SC>();
    if (!s) s = prepare_an<P, 16, SC>();
    if (!s) s = prepare_v<P, 0, SC>();
    if (!s) s = prepare_v<P, 2, SC>();
    if (!s) s = prepare_v<P, 4, SC>();
    if (!s) s = prepare_v<P, 8, SC>();
    if (!s) s = prepare_v<P, 16, SC>();
    return s;
}

int prepare_fused_kernels() {
    int s = prepare_p<AERIAL_PREC_FP16>();
    if (!s) {
        cudaFuncAttributes at;
        const cudaError_t e = cudaFuncGetAttributes(&at, fused_eq_kernel_hg);
        s = e == cudaSuccess ? allow_max_smem<fused_eq_kernel_hg>() : rt_status(e);
    }
    if (!s) s = prepare_p<AERIAL_PREC_FP16, true>();
    if (!s) s = prepare_h<4, 2>();
    if (!s) s = prepare_h<4, 4>();
    if (!s) s = prepare_h<4, 8>();
    if (!s) s = prepare_h<8, 2>();
    if (!s) s = prepare_h<8, 4>();
    if (!s) s = prepare_h<8, 8>();
    if (!s) s = prepare_h<16, 2>();
    if (!s) s = prepare_h<16, 4>();
    if (!s) s = prepare_h<16, 8>();
    if (!s) s = prepare_p<AERIAL_PREC_BF16>();
    if (!s) s = prepare_p<AERIAL_PREC_BF16X3>();
    if (!s) s = prepare_p<AERIAL_PREC_FP16X3, true>();
    return s;
}

}  // namespace aeq
