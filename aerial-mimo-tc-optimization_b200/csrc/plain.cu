// plain.cu -- the plain FP32 chain: one kernel per stage, the reference's
// scalar method (Gram, coef_apply, LLR) plus the FP32 Cholesky MMSE solve the
// reference lacks.  Every stage is bit-exact with the CPU restatement in the
// checker because each output element is accumulated in the same order with
// the same fused multiply-adds.
#include "common.cuh"

namespace aeq {

// ---------------------------------------------------------------------------
// Gram: G[sc][r][c] = sum_k cma(conj(H[k][r]), H[k][c]) (+ sigma2 if r == c).
// gram_scalar (src/aerial_bottleneck.cu:56-80) with M = H^H; one thread per
// output element, the antenna sum in order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) gram_kernel(const cf* __restrict__ H, float sigma2,
                                                    cf* __restrict__ G, long total, int A, int L) {
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int c = (int)(t % L);
    int r = (int)((t / L) % L);
    long sc = t / ((long)L * L);
    const cf* h = H + sc * (long)A * L;
    cf acc = make_float2(0.f, 0.f);
    for (int k = 0; k < A; k++) {
        cf m = __ldg(&h[k * L + r]);
        m.y = -m.y;
        acc = cma(m, __ldg(&h[k * L + c]), acc);
    }
    if (r == c) acc.x = __fadd_rn(acc.x, sigma2);
    G[t] = acc;
}

// ---------------------------------------------------------------------------
// MMSE coefficients.  One block per subcarrier.
//   1. Cholesky G = Lc Lc^H, column by column; thread i computes Lc[i][j]
//      (its whole sum in order), so the arithmetic is the serial
//      specification's.
//   2. Thread a solves G x = conj(H[a][:]) -> column a of C.
//   3. Thread l sums mu_l = Re sum_a C[l][a] H[a][l] in antenna order.
//   4. C[l][:] *= 1/mu_l; noiseInv[l] = mu_l / (1 - mu_l).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) mmse_coef_kernel(const cf* __restrict__ G,
                                                         const cf* __restrict__ H, cf* __restrict__ C,
                                                         float* __restrict__ noiseInv, int A, int L) {
    extern __shared__ float2 sm[];
    cf* sL = sm;                  // [L][L]
    cf* sX = sm + L * L;          // [L][A]
    float* sInv = (float*)(sX + (long)L * A);   // [L]
    float* sMuInv = sInv + L;                    // [L]
    const long sc = blockIdx.x;
    const cf* g = G + sc * L * L;
    const cf* h = H + sc * (long)A * L;
    const int tid = threadIdx.x;

    for (int j = 0; j < L; j++) {
        if (tid == 0) {
            float s = g[j * L + j].x;
            for (int k = 0; k < j; k++) {
                cf x = sL[j * L + k];
                s = __fmaf_rn(-x.x, x.x, s);
                s = __fmaf_rn(-x.y, x.y, s);
            }
            if (!(s > 0.f)) s = 1e-30f;
            float d = __fsqrt_rn(s);
            sInv[j] = __fdiv_rn(1.0f, d);
            sL[j * L + j] = make_float2(d, 0.f);
        }
        __syncthreads();
        const float iv = sInv[j];
        for (int i = j + 1 + tid; i < L; i += blockDim.x) {
            cf acc = g[i * L + j];
            for (int k = 0; k < j; k++) {
                cf a = sL[i * L + k], b = sL[j * L + k];
                acc.x = __fmaf_rn(-a.x, b.x, acc.x);
                acc.x = __fmaf_rn(-a.y, b.y, acc.x);
                acc.y = __fmaf_rn(-a.y, b.x, acc.y);
                acc.y = __fmaf_rn(a.x, b.y, acc.y);
            }
            sL[i * L + j] = make_float2(__fmul_rn(acc.x, iv), __fmul_rn(acc.y, iv));
        }
        __syncthreads();
    }

    for (int a = tid; a < A; a += blockDim.x) {
        cf w[AERIAL_MAX_LAYERS], x[AERIAL_MAX_LAYERS];
        for (int i = 0; i < L; i++) {
            cf hv = __ldg(&h[a * L + i]);
            cf acc = make_float2(hv.x, -hv.y);
            for (int k = 0; k < i; k++) {
                cf lv = sL[i * L + k], y = w[k];
                acc.x = __fmaf_rn(-lv.x, y.x, acc.x);
                acc.x = __fmaf_rn(lv.y, y.y, acc.x);
                acc.y = __fmaf_rn(-lv.x, y.y, acc.y);
                acc.y = __fmaf_rn(-lv.y, y.x, acc.y);
            }
            w[i] = make_float2(__fmul_rn(acc.x, sInv[i]), __fmul_rn(acc.y, sInv[i]));
        }
        for (int i = L - 1; i >= 0; i--) {
            cf acc = w[i];
            for (int k = i + 1; k < L; k++) {
                cf lv = sL[k * L + i], y = x[k];
                acc.x = __fmaf_rn(-lv.x, y.x, acc.x);
                acc.x = __fmaf_rn(-lv.y, y.y, acc.x);
                acc.y = __fmaf_rn(-lv.x, y.y, acc.y);
                acc.y = __fmaf_rn(lv.y, y.x, acc.y);
            }
            x[i] = make_float2(__fmul_rn(acc.x, sInv[i]), __fmul_rn(acc.y, sInv[i]));
        }
        for (int l = 0; l < L; l++) sX[l * A + a] = x[l];
    }
    __syncthreads();
    for (int l = tid; l < L; l += blockDim.x) {
        float mu = 0.f;
        for (int a = 0; a < A; a++) {
            cf c = sX[l * A + a], hv = __ldg(&h[a * L + l]);
            mu = __fmaf_rn(c.x, hv.x, mu);
            mu = __fmaf_rn(-c.y, hv.y, mu);
        }
        sMuInv[l] = __fdiv_rn(1.0f, mu);
        noiseInv[sc * L + l] = __fdiv_rn(mu, __fsub_rn(1.0f, mu));
    }
    __syncthreads();
    cf* c = C + sc * (long)L * A;
    for (int e = tid; e < L * A; e += blockDim.x) {
        cf v = sX[e];
        float im = sMuInv[e / A];
        c[e] = make_float2(__fmul_rn(v.x, im), __fmul_rn(v.y, im));
    }
}

// ---------------------------------------------------------------------------
// coef_apply, coef_apply_v1_scalar (src/aerial_coef_wmma.cu:71-104): grid
// (PRBs, layers), block (12 subcarriers, nSym); C[sc][layer][:] staged in
// shared memory; each thread sums its antenna products in order.
// ---------------------------------------------------------------------------
__global__ void coef_apply_kernel(const cf* __restrict__ C, const cf* __restrict__ Y,
                                  cf* __restrict__ O, int nSC, int nSym, int L, int A) {
    extern __shared__ float2 sC[];  // [A][12]
    const int prb = blockIdx.x, layer = blockIdx.y;
    const int scl = threadIdx.x, sym = threadIdx.y;
    const int sc = prb * 12 + scl;
    const int nt = blockDim.x * blockDim.y;
    for (int e = threadIdx.y * blockDim.x + threadIdx.x; e < A * 12; e += nt) {
        int s2 = e / A, a = e % A;
        int scc = prb * 12 + s2;
        if (scc < nSC) sC[a * 12 + s2] = __ldg(&C[((long)scc * L + layer) * A + a]);
    }
    __syncthreads();
    if (sc >= nSC || sym >= nSym) return;
    const cf* y = Y + ((long)sc * nSym + sym) * A;
    cf acc = make_float2(0.f, 0.f);
    for (int a = 0; a < A; a++) acc = cma(sC[a * 12 + scl], __ldg(&y[a]), acc);
    O[((long)sc * L + layer) * nSym + sym] = acc;
}

// ---------------------------------------------------------------------------
// LLR demapper: one thread per symbol (llr_v1_baseline / llr_v3 shape).
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(512) llr_f16_kernel(const __half2* __restrict__ in,
                                                       const float* __restrict__ ni,
                                                       __half* __restrict__ out, int count, PamLut lut) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    __half2 v = in[idx];
    float o[2 * N];
    pam_llr<N>(__low2float(v), __high2float(v), ni[idx], lut, o);
    __half* dst = out + (long)idx * 2 * N;
#pragma unroll
    for (int j = 0; j < 2 * N; j += 2) *reinterpret_cast<__half2*>(dst + j) = __floats2half2_rn(o[j], o[j + 1]);
}

template <int N>
__global__ void __launch_bounds__(512) llr_f32_kernel(const cf* __restrict__ in, const float* __restrict__ ni,
                                                       float* __restrict__ out, int count, int symsPerNoise,
                                                       PamLut lut) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    cf v = in[idx];
    float o[2 * N];
    pam_llr<N>(v.x, v.y, ni[idx / symsPerNoise], lut, o);
    float* dst = out + (long)idx * 2 * N;
#pragma unroll
    for (int j = 0; j < 2 * N; j += 2) *reinterpret_cast<float2*>(dst + j) = make_float2(o[j], o[j + 1]);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static bool shape_ok(int nSC, int nSym, int L, int A) {
    return nSC >= 1 && nSC <= 12 * AERIAL_MAX_PRB && nSym >= 1 && nSym <= AERIAL_MAX_SYMS && L >= 1 && L <= AERIAL_MAX_LAYERS && A >= 1 &&
           A <= AERIAL_MAX_ANTS;
}

int launch_gram(const cf* H, float sigma2, cf* G, int nSC, int A, int L, cudaStream_t st) {
    long total = (long)nSC * L * L;
    gram_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(H, sigma2, G, total, A, L);
    return launch_status();
}

int launch_mmse_coef(const cf* G, const cf* H, cf* C, float* nI, int nSC, int A, int L, cudaStream_t st) {
    size_t smem = sizeof(cf) * ((size_t)L * L + (size_t)L * A) + sizeof(float) * 2 * L;
    int threads = A < 32 ? 32 : (A > 256 ? 256 : ((A + 31) / 32) * 32);
    if (smem > 48 * 1024) cudaFuncSetAttribute(mmse_coef_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    mmse_coef_kernel<<<nSC, threads, smem, st>>>(G, H, C, nI, A, L);
    return launch_status();
}

int launch_coef_apply(const cf* C, const cf* Y, cf* O, int nSC, int nSym, int L, int A, cudaStream_t st) {
    dim3 blk(12, nSym), grd((nSC + 11) / 12, L);
    size_t smem = sizeof(cf) * (size_t)A * 12;
    coef_apply_kernel<<<grd, blk, smem, st>>>(C, Y, O, nSC, nSym, L, A);
    return launch_status();
}

int launch_llr_f32(const cf* in, const float* ni, float* out, int N, int n, int spn, cudaStream_t st) {
    PamLut lut = pam_lut(n);
    unsigned g = (unsigned)((N + 511) / 512);
    switch (n) {
        case 1: llr_f32_kernel<1><<<g, 512, 0, st>>>(in, ni, out, N, spn, lut); break;
        case 2: llr_f32_kernel<2><<<g, 512, 0, st>>>(in, ni, out, N, spn, lut); break;
        case 3: llr_f32_kernel<3><<<g, 512, 0, st>>>(in, ni, out, N, spn, lut); break;
        default: llr_f32_kernel<4><<<g, 512, 0, st>>>(in, ni, out, N, spn, lut); break;
    }
    return launch_status();
}

}  // namespace aeq

namespace aeq {

// Load the plain chain's kernels on the current device (aerial_prepare).
template <typename K>
static int prepare_one(K* k) {
    cudaFuncAttributes at;
    return rt_status(cudaFuncGetAttributes(&at, k));
}
int prepare_plain_kernels() {
    int s = prepare_one(gram_kernel);
    if (!s) s = prepare_one(mmse_coef_kernel);
    if (!s) s = prepare_one(coef_apply_kernel);
    if (!s) s = prepare_one(llr_f16_kernel<1>);
    if (!s) s = prepare_one(llr_f16_kernel<2>);
    if (!s) s = prepare_one(llr_f16_kernel<3>);
    if (!s) s = prepare_one(llr_f16_kernel<4>);
    if (!s) s = prepare_one(llr_f32_kernel<1>);
    if (!s) s = prepare_one(llr_f32_kernel<2>);
    if (!s) s = prepare_one(llr_f32_kernel<3>);
    if (!s) s = prepare_one(llr_f32_kernel<4>);
    return s;
}

}  // namespace aeq

using namespace aeq;

extern "C" int aerial_gram(const aerial_cf32* H, float sigma2, aerial_cf32* G, int nSC, int nAnt, int nLayers,
                           void* stream) {
    if (!H || !G || !shape_ok(nSC, 1, nLayers, nAnt)) return AERIAL_ERR_INVALID_ARG;
    return launch_gram((const cf*)H, sigma2, (cf*)G, nSC, nAnt, nLayers, to_stream(stream));
}

extern "C" int aerial_mmse_coef(const aerial_cf32* G, const aerial_cf32* H, aerial_cf32* C, float* noiseInv, int nSC,
                                int nAnt, int nLayers, void* stream) {
    if (!G || !H || !C || !noiseInv || !shape_ok(nSC, 1, nLayers, nAnt)) return AERIAL_ERR_INVALID_ARG;
    return launch_mmse_coef((const cf*)G, (const cf*)H, (cf*)C, noiseInv, nSC, nAnt, nLayers, to_stream(stream));
}

extern "C" int aerial_coef_apply(const aerial_cf32* C, const aerial_cf32* Y_rx, aerial_cf32* Y_eq, int nSC, int nSym,
                                 int nLayers, int nAnt, void* stream) {
    if (!C || !Y_rx || !Y_eq || !shape_ok(nSC, nSym, nLayers, nAnt)) return AERIAL_ERR_INVALID_ARG;
    return launch_coef_apply((const cf*)C, (const cf*)Y_rx, (cf*)Y_eq, nSC, nSym, nLayers, nAnt, to_stream(stream));
}

extern "C" int aerial_llr(const aerial_ch2* softEst, const float* noiseInv, uint16_t* llrOut, int N, int nPamBits,
                          void* stream) {
    if (!softEst || !noiseInv || !llrOut || N < 1 || nPamBits < 1 || nPamBits > 4) return AERIAL_ERR_INVALID_ARG;
    PamLut lut = pam_lut(nPamBits);
    unsigned g = (unsigned)((N + 511) / 512);
    cudaStream_t st = to_stream(stream);
    const __half2* in = (const __half2*)softEst;
    __half* out = (__half*)llrOut;
    switch (nPamBits) {
        case 1: llr_f16_kernel<1><<<g, 512, 0, st>>>(in, noiseInv, out, N, lut); break;
        case 2: llr_f16_kernel<2><<<g, 512, 0, st>>>(in, noiseInv, out, N, lut); break;
        case 3: llr_f16_kernel<3><<<g, 512, 0, st>>>(in, noiseInv, out, N, lut); break;
        default: llr_f16_kernel<4><<<g, 512, 0, st>>>(in, noiseInv, out, N, lut); break;
    }
    return launch_status();
}

extern "C" int aerial_llr_f32(const aerial_cf32* softEst, const float* noiseInv, float* llrOut, int N, int nPamBits,
                              int nSymPerNoise, void* stream) {
    if (!softEst || !noiseInv || !llrOut || N < 1 || nPamBits < 1 || nPamBits > 4 || nSymPerNoise < 1)
        return AERIAL_ERR_INVALID_ARG;
    return launch_llr_f32((const cf*)softEst, noiseInv, llrOut, N, nPamBits, nSymPerNoise, to_stream(stream));
}

// ---------------------------------------------------------------------------
// The plain chain over cells: workspace holds G, C, noiseInv and Y_eq of the
// largest cell; cells run one after another on `stream`.
// ---------------------------------------------------------------------------
static size_t plain_ws_cell(const aerial_cell_desc& c) {
    size_t nSC = (size_t)c.nPRB * 12;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return al(nSC * c.nLayers * c.nLayers * sizeof(cf)) + al(nSC * c.nLayers * c.nAnt * sizeof(cf)) +
           al(nSC * c.nLayers * sizeof(float)) + al(nSC * c.nLayers * c.nSym * sizeof(cf));
}

extern "C" size_t aerial_pusch_eq_plain_workspace(const aerial_cell_desc* cells, int nCells) {
    size_t m = 0;
    for (int i = 0; cells && i < nCells; i++) {
        size_t w = plain_ws_cell(cells[i]);
        if (w > m) m = w;
    }
    return m;
}

extern "C" int aerial_pusch_eq_plain(const aerial_cell_desc* cells, int nCells, void* workspace, size_t wsBytes,
                                     void* stream) {
    if (!cells || nCells < 1 || !workspace) return AERIAL_ERR_INVALID_ARG;
    cudaStream_t st = to_stream(stream);
    for (int i = 0; i < nCells; i++) {
        const aerial_cell_desc& c = cells[i];
        if (c.nPRB < 1 || c.nPRB > AERIAL_MAX_PRB) return AERIAL_ERR_INVALID_ARG;
        int nSC = c.nPRB * 12;
        if (!c.H || !c.Y_rx || !c.llr || c.nPamBits < 1 || c.nPamBits > 4 || !shape_ok(nSC, c.nSym, c.nLayers, c.nAnt))
            return AERIAL_ERR_INVALID_ARG;
        if (c.format != AERIAL_FMT_CF32) return AERIAL_ERR_UNSUPPORTED;   // the FP32 chain reads complex64 only
        if (plain_ws_cell(c) > wsBytes) return AERIAL_ERR_INVALID_ARG;
        auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
        char* p = (char*)workspace;
        cf* G = (cf*)p;
        p += al((size_t)nSC * c.nLayers * c.nLayers * sizeof(cf));
        cf* C = (cf*)p;
        p += al((size_t)nSC * c.nLayers * c.nAnt * sizeof(cf));
        float* nI = (float*)p;
        p += al((size_t)nSC * c.nLayers * sizeof(float));
        cf* Yeq = c.Y_eq ? (cf*)c.Y_eq : (cf*)p;
        int s;
        if ((s = launch_gram((const cf*)c.H, c.sigma2, G, nSC, c.nAnt, c.nLayers, st))) return s;
        if ((s = launch_mmse_coef(G, (const cf*)c.H, C, nI, nSC, c.nAnt, c.nLayers, st))) return s;
        if ((s = launch_coef_apply(C, (const cf*)c.Y_rx, Yeq, nSC, c.nSym, c.nLayers, c.nAnt, st))) return s;
        if ((s = launch_llr_f32(Yeq, nI, c.llr, nSC * c.nLayers * c.nSym, c.nPamBits, c.nSym, st))) return s;
    }
    return AERIAL_OK;
}

// ---------------------------------------------------------------------------
// The plain chain for callers that must not allocate device memory.
//
// Some hosts cannot call cudaMalloc on the path that equalizes a slot: a
// real-time receiver loop where an allocation may block or synchronize the
// device and miss the slot deadline, or a plugin inside a framework that owns
// all device memory and hands out none.  This entry point keeps the plain
// chain's intermediates (G, C, noiseInv, Y_eq) in one file-scope device array
// instead of a caller workspace.  The array is part of the module image, so
// every GPU that loads this library holds it until the process exits.
//
// The array's host-side name is only a stand-in for the device symbol; the
// device address comes from cudaGetSymbolAddress, made with the device
// current.  The address belongs to the CUDA context that loaded the module:
// a cudaDeviceReset, or a second context on the same device, gets its own
// copy of the array.  The address is therefore cached per device together
// with the unique ID of the context it was looked up in (cuCtxGetId, which a
// new context never reuses even where its handle value is recycled), and
// looked up again whenever a call runs in a different context.  The first
// call in each context does that lookup, so make it before any stream
// capture.  All calls share the one array and it keeps the last call's
// contents: every scratch byte a call reads is first written by that same
// call, so nothing needs clearing, but calls that overlap on the GPU (two
// streams, two threads) race on it.
// ---------------------------------------------------------------------------
#include <mutex>

static __device__ __align__(256) unsigned char g_plain_static_scratch[AERIAL_STATIC_SCRATCH_BYTES];

static int static_scratch_address(void** out) {
    static std::mutex mu;
    static void* addr[64] = {};
    static unsigned long long ctxOf[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return rt_status(e);
    if (dev < 0 || dev >= 64) return AERIAL_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long ctx = current_ctx_id();
    if (ctx != 0 && addr[dev] && ctxOf[dev] == ctx) {
        *out = addr[dev];
        return AERIAL_OK;
    }
    // no cached address for this context (or no context yet: the runtime
    // makes the device's primary context current inside this call)
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_plain_static_scratch);
    if (e != cudaSuccess) return rt_status(e);
    addr[dev] = p;
    ctxOf[dev] = current_ctx_id();    // 0 when unknown: looked up again next call
    *out = p;
    return AERIAL_OK;
}

// The checks aerial_pusch_eq_plain makes per cell, so a malformed cell gets
// AERIAL_ERR_INVALID_ARG / AERIAL_ERR_UNSUPPORTED before the size comparison
// (negative shapes would otherwise wrap in the workspace arithmetic).
static int plain_cell_check(const aerial_cell_desc& c) {
    if (c.nPRB < 1 || c.nPRB > AERIAL_MAX_PRB) return AERIAL_ERR_INVALID_ARG;
    if (!c.H || !c.Y_rx || !c.llr || c.nPamBits < 1 || c.nPamBits > 4 ||
        !shape_ok(c.nPRB * 12, c.nSym, c.nLayers, c.nAnt))
        return AERIAL_ERR_INVALID_ARG;
    if (c.format != AERIAL_FMT_CF32) return AERIAL_ERR_UNSUPPORTED;
    return AERIAL_OK;
}

extern "C" int aerial_pusch_eq_plain_static(const aerial_cell_desc* cells, int nCells, void* stream) {
    if (!cells || nCells < 1) return AERIAL_ERR_INVALID_ARG;
    for (int i = 0; i < nCells; i++) {
        const int s = plain_cell_check(cells[i]);
        if (s != AERIAL_OK) return s;
    }
    if (aerial_pusch_eq_plain_workspace(cells, nCells) > (size_t)AERIAL_STATIC_SCRATCH_BYTES)
        return AERIAL_ERR_SCRATCH_LIMIT;
    void* scratch = nullptr;
    const int s = static_scratch_address(&scratch);
    if (s != AERIAL_OK) return s;
    return aerial_pusch_eq_plain(cells, nCells, scratch, (size_t)AERIAL_STATIC_SCRATCH_BYTES, stream);
}
