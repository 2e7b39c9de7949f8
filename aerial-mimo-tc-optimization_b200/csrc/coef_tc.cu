// coef_tc.cu -- coef_apply on the tensor cores: the semantics of
// coef_apply_v2_wmma (src/aerial_coef_wmma.cu:146-239), FP16 operands and
// FP32 accumulation, without its shared-memory staging.
//
// Y_eq[l][s] = sum_a C[l][a] Y[s][a] (no conjugate) as a real-embedded
// mma.sync m16n8k16: with B pairs (Re Y, Im Y), A row l carries
// (Re C, -Im C) -> Re out and A row l+8 carries (Im C, Re C) -> Im out.
// Thread (g, c) of k-step j owns antennas 8j+2c and 8j+2c+1, so its A operand
// is C[l][8j+2c .. +1] and its B operand Y[s][8j+2c .. +1]: one 16-byte load
// each, straight into registers.  One warp per subcarrier; L <= 16 (two
// m-tiles), nSym <= 16 (two n-tiles).
#include "common.cuh"

namespace aeq {

__device__ __forceinline__ uint32_t h2u(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

__device__ __forceinline__ void mma_f16(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                        uint32_t b1) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float4 ld_pair(const float2* p, int a0, int A, bool vec) {
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (vec && a0 + 1 < A) return __ldg(reinterpret_cast<const float4*>(p + a0));
    if (a0 < A) { float2 t = __ldg(p + a0); v.x = t.x; v.y = t.y; }
    if (a0 + 1 < A) { float2 t = __ldg(p + a0 + 1); v.z = t.x; v.w = t.y; }
    return v;
}

__global__ void __launch_bounds__(256) coef_apply_tc_kernel(const float2* __restrict__ C, const float2* __restrict__ Y,
                                                             float2* __restrict__ O, int nSC, int nSym, int L, int A,
                                                             int vec) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, c = lane & 3;
    const long w0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    const int nK = (A + 7) >> 3;
    const int nMT = L > 8 ? 2 : 1;
    const int nNT = nSym > 8 ? 2 : 1;
    for (long sc = w0; sc < nSC; sc += nw) {
        float acc[2][2][4] = {};
        const float2* Cs = C + sc * (long)L * A;
        const float2* Ys = Y + sc * (long)nSym * A;
        for (int j = 0; j < nK; j++) {
            const int a0 = 8 * j + 2 * c;
            uint32_t b[2][2];
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int s = 8 * nt + g;
                float4 y = (nt < nNT && s < nSym) ? ld_pair(Ys + (long)s * A, a0, A, vec) : make_float4(0, 0, 0, 0);
                b[nt][0] = h2u(__floats2half2_rn(y.x, y.y));
                b[nt][1] = h2u(__floats2half2_rn(y.z, y.w));
            }
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                if (mt >= nMT) break;
                const int l = 8 * mt + g;
                float4 cv = l < L ? ld_pair(Cs + (long)l * A, a0, A, vec) : make_float4(0, 0, 0, 0);
                const uint32_t p0 = h2u(__floats2half2_rn(cv.x, cv.y)), p1 = h2u(__floats2half2_rn(cv.z, cv.w));
                const uint32_t r0 = p0 ^ 0x80000000u, r1 = p1 ^ 0x80000000u;          // (Re, -Im)
                const uint32_t i0 = __byte_perm(p0, 0, 0x1032), i1 = __byte_perm(p1, 0, 0x1032);  // (Im, Re)
#pragma unroll
                for (int nt = 0; nt < 2; nt++)
                    if (nt < nNT) mma_f16(acc[mt][nt], r0, i0, r1, i1, b[nt][0], b[nt][1]);
            }
        }
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int l = 8 * mt + g, s = 8 * nt + 2 * c;
                if (mt < nMT && nt < nNT && l < L) {
                    float2* o = O + (sc * L + l) * (long)nSym;
                    if (s < nSym) o[s] = make_float2(acc[mt][nt][0], acc[mt][nt][2]);
                    if (s + 1 < nSym) o[s + 1] = make_float2(acc[mt][nt][1], acc[mt][nt][3]);
                }
            }
    }
}

}  // namespace aeq

using namespace aeq;

extern "C" int aerial_coef_apply_tc(const aerial_cf32* C, const aerial_cf32* Y_rx, aerial_cf32* Y_eq, int nSC,
                                    int nSym, int nLayers, int nAnt, void* stream) {
    if (!C || !Y_rx || !Y_eq || nSC < 1 || nSym < 1 || nSym > AERIAL_MAX_SYMS || nLayers < 1 ||
        nLayers > AERIAL_MAX_LAYERS || nAnt < 1 || nAnt > AERIAL_MAX_ANTS)
        return AERIAL_ERR_INVALID_ARG;
    const int vec = ((nAnt % 2) == 0 && ((uintptr_t)C & 15) == 0 && ((uintptr_t)Y_rx & 15) == 0) ? 1 : 0;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long blocks = ((long)nSC + 7) / 8;
    long cap = (long)nsm * 8;
    if (blocks > cap) blocks = cap;
    coef_apply_tc_kernel<<<(unsigned)blocks, 256, 0, to_stream(stream)>>>(
        (const float2*)C, (const float2*)Y_rx, (float2*)Y_eq, nSC, nSym, nLayers, nAnt, vec);
    return launch_status();
}
