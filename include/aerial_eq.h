/*
 * aerial_eq.h -- C ABI of the B200 PUSCH receiver equalization path.
 *
 * Drop-in boundary for the per-subcarrier equalization chain of
 * ebaenamar/aerial-mimo-tc-optimization: Gram, MMSE coefficient solve,
 * coef_apply, max-log LLR demapper and SRS filter multiply, plus the fused
 * chain and a slot-serving loop.  The reference has no library API; its
 * kernel-entry argument lists and buffer layouts are the interface, and each
 * entry point below names the reference kernel it replaces (file:line inside
 * the reference project).
 *
 * Conventions (all entry points):
 *   - Buffers are DEVICE pointers owned by the caller unless stated
 *     otherwise; nothing is allocated, freed or synchronised by a call.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Work is enqueued asynchronously on it.
 *   - Return value: AERIAL_OK (0), an AERIAL_ERR_* code for bad arguments,
 *     or a cudaError_t value (1..999) from the launch.  Nothing calls
 *     exit(); the reference's CUDA_CHECK -> exit(1) becomes a status.
 *   - Complex numbers are interleaved {re, im} pairs: aerial_cf32 is the
 *     reference's `struct cf32 { float re, im; }` (src/aerial_coef_wmma.cu:60);
 *     aerial_ch2 is `struct half2c` / `struct ch2` of IEEE binary16 bits
 *     (src/llr/aerial_llr_v3.cu:51, src/srs/srs_wmma_bench.cu:41).
 *
 * Layouts (row-major):
 *   H      [nSC][nAnt][nLayers]      channel      (src/aerial_bottleneck.cu:58)
 *   Y_rx   [nSC][nSym][nAnt]         received     (src/aerial_coef_wmma.cu:73)
 *   C      [nSC][nLayers][nAnt]      coefficients (src/aerial_coef_wmma.cu:72)
 *   G      [nSC][nLayers][nLayers]   Gram         (src/aerial_bottleneck.cu:59)
 *   Y_eq   [nSC][nLayers][nSym]      equalized    (src/aerial_coef_wmma.cu:74)
 *   LLR    [nSC*nLayers*nSym][2*nPamBits] in the order
 *          bit0_I, bit0_Q, bit1_I, bit1_Q, ...  (src/llr/aerial_llr_v3.cu:92,105)
 *
 * Noise convention: noiseInv = 1/nu where nu is the complex noise variance of
 * the (unbiased) equalized symbol, so LLR = (d_opposite^2 - d_nearest^2)/nu
 * per real dimension of a unit-energy constellation.  The MMSE stages produce
 * nu_l = sigma2 (G^-1)_ll / (1 - sigma2 (G^-1)_ll) for layer l, where sigma2
 * is the complex noise variance per receive antenna.
 */
#ifndef AERIAL_EQ_H
#define AERIAL_EQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float re, im; } aerial_cf32;
typedef struct { uint16_t re, im; } aerial_ch2;

enum {
    AERIAL_OK = 0,
    AERIAL_ERR_INVALID_ARG = 1001,   /* null pointer, non-positive or too-large size */
    AERIAL_ERR_UNSUPPORTED = 1002,   /* shape outside the supported envelope */
    AERIAL_ERR_NO_DEVICE = 1003,     /* no usable sm_100 device */
    AERIAL_ERR_BUDGET = 1004,        /* serving: request exceeds the memory budget */
    AERIAL_ERR_QUEUE_FULL = 1005,    /* serving: submission queue full */
    AERIAL_ERR_TIMEOUT = 1006,       /* a bounded wait ran out */
    AERIAL_ERR_NOT_FOUND = 1007,     /* serving: unknown cell or request */
    AERIAL_ERR_SCRATCH_LIMIT = 1008  /* request needs more than the library's static scratch */
};

/* Supported envelope: 1 <= nLayers <= 16, 1 <= nSym <= 16, 1 <= nAnt <= 256,
 * 1 <= nPamBits <= 4 (QPSK..256QAM), 1 <= nPRB <= AERIAL_MAX_PRB per cell
 * descriptor (nSC = 12 nPRB; the per-stage entry points take nSC up to
 * 12 AERIAL_MAX_PRB).  The PRB bound keeps every symbol index of a cell
 * (nSC x nLayers x nSym) inside 32 bits. */
#define AERIAL_MAX_PRB 524288
#define AERIAL_MAX_LAYERS 16
#define AERIAL_MAX_SYMS 16
#define AERIAL_MAX_ANTS 256
#define AERIAL_MAX_CELLS 64

const char* aerial_error_string(int status);
int aerial_version(void);

/* Diagnostic with no counterpart in the reference: the number of mbarrier
 * waits in this library's tcgen05 kernels (the SRS / DMRS filter multiply)
 * that ran out of their iteration limit on the current device since the
 * library was loaded.  0 in correct operation; a kernel whose wait gives up
 * leaves its loops, frees its tensor memory and returns (its output is then
 * not valid).  Synchronizes with the device (a device-to-host copy). */
int aerial_kernel_timeouts(unsigned int* count);

/* Load every kernel of the library on the current device and set its launch
 * attributes.  Optional: without it the first launch of each kernel variant
 * pays the driver's lazy module loading (milliseconds), which a latency-
 * critical slot loop should do before it starts.  aerial_server_create calls it. */
int aerial_prepare(void);

/* ------------------------------------------------------------------------ */
/* Per-stage entry points (the plain FP32 chain; bit-exact restatements of   */
/* the reference's scalar kernels where the reference has the stage).        */
/* ------------------------------------------------------------------------ */

/* Y_eq[sc][l][s] = sum_a C[sc][l][a] * Y_rx[sc][s][a], FP32, antennas summed
 * in order with the reference's fused multiply-adds (bit-exact).
 * Replaces coef_apply_v1_scalar(C, Y_rx, Y_eq, nSC, nSym)
 * (src/aerial_coef_wmma.cu:71-75); N_LAYERS and N_BS_ANTS become runtime. */
int aerial_coef_apply(const aerial_cf32* C, const aerial_cf32* Y_rx, aerial_cf32* Y_eq,
                      int nSC, int nSym, int nLayers, int nAnt, void* stream);

/* Same product on the tensor cores (FP16 operands, FP32 accumulation): the
 * semantics of coef_apply_v2_wmma (src/aerial_coef_wmma.cu:146-239). */
int aerial_coef_apply_tc(const aerial_cf32* C, const aerial_cf32* Y_rx, aerial_cf32* Y_eq,
                         int nSC, int nSym, int nLayers, int nAnt, void* stream);

/* G[sc] = H[sc]^H H[sc] + sigma2 I, FP32 (bit-exact with gram_scalar given
 * M = H^H, then one FP32 add of sigma2 on the diagonal).
 * Replaces gram_scalar(M, H, G, nSC) (src/aerial_bottleneck.cu:56-60); M is
 * dropped because the MMSE Gram is Hermitian, sigma2 is added. */
int aerial_gram(const aerial_cf32* H, float sigma2, aerial_cf32* G,
                int nSC, int nAnt, int nLayers, void* stream);

/* MMSE coefficients C[sc] = diag(1/mu) G^-1 H^H (FP32 Cholesky of G, forward
 * and backward substitution per antenna), mu_l = Re (G^-1 H^H H)_ll, and
 * noiseInv[sc][l] = mu_l / (1 - mu_l).  No reference counterpart (the
 * reference's coef_apply consumes a random C). */
int aerial_mmse_coef(const aerial_cf32* G, const aerial_cf32* H, aerial_cf32* C, float* noiseInv,
                     int nSC, int nAnt, int nLayers, void* stream);

/* Max-log PAM LLR demapper, FP16 in / FP16 out, bit-exact with the
 * reference.  Replaces llr_v1_baseline(in, ni, out, N, nPamBits)
 * (src/llr/aerial_llr_v3.cu:84-86) and llr_v3_reg_template (:219-229). */
int aerial_llr(const aerial_ch2* softEst, const float* noiseInv, uint16_t* llrOut,
               int N, int nPamBits, void* stream);

/* Same demapper with complex64 input and float32 output (the layout the
 * fused chain writes).  noiseInv index = idx / nSymPerNoise (1 = per
 * symbol, as the reference; nSym = one value per (sc, layer)). */
int aerial_llr_f32(const aerial_cf32* softEst, const float* noiseInv, float* llrOut,
                   int N, int nPamBits, int nSymPerNoise, void* stream);

/* SRS filter multiply, FP16 in/out with FP32 accumulation:
 *   H_est[blk][ant][k_out][p] = sum_k (W[k_out][k] * FOCC[p][k % foccLen]) * SRS[blk][ant][k]
 * Replaces srs_filter_v1_scalar<K,N_PORTS,FOCC_LENGTH>(H_est, SRS, W, FOCC,
 * nAnt, nBlocks) (src/srs/srs_wmma_bench.cu:57-63); template arguments are
 * runtime.  The reference's complex_conjmul (:43-47) computes the plain
 * product W*FOCC (no conjugate); that behaviour is kept. */
int aerial_srs_filter(aerial_ch2* H_est, const aerial_ch2* SRS, const aerial_ch2* W,
                      const aerial_ch2* FOCC, int nAnt, int nBlocks, int K, int nPorts,
                      int foccLen, void* stream);

/* SRS filter multiply straight into the PUSCH channel layout: writes
 * H[sc][ant][layer] (complex64) for sc = blk*K + k_out, layer = port, so a
 * cell's resident channel is refreshed in place.  FP32 accumulation. */
int aerial_srs_to_channel(aerial_cf32* H, const aerial_ch2* SRS, const aerial_ch2* W,
                          const aerial_ch2* FOCC, int nAnt, int nBlocks, int K, int nPorts,
                          int foccLen, void* stream);

/* aerial_srs_to_channel over nSrsSym (1, 2 or 4) SRS symbols, averaged:
 *   H = (1 / nSrsSym) sum_s srs_to_channel(SRS_s),
 * with SRS holding the symbols one after another ([sym][blk][ant][K]).  The
 * average is one FP32 sum: the tcgen05 kernel's K loop runs over every
 * symbol with the taps scaled by 1/nSrsSym (exact for these counts).
 * nSrsSym > 1 needs the tcgen05 path (K a multiple of 4, SRS 16-byte
 * aligned, and K <= 32 for 4 symbols, whose operand stages must fit in
 * shared memory); other shapes return AERIAL_ERR_UNSUPPORTED. */
int aerial_srs_to_channel_avg(aerial_cf32* H, const aerial_ch2* SRS, int nSrsSym, const aerial_ch2* W,
                              const aerial_ch2* FOCC, int nAnt, int nBlocks, int K, int nPorts,
                              int foccLen, void* stream);

/* Frequency-interpolation filter of DMRS channel estimation, straight into
 * the PUSCH channel layout (complex64):
 *   H[blk*nOut + o][ant][p] = sum_k Wf[o][k] * OCC[p][k % occLen] * Yp[blk][ant][k]
 * for k < nPilot (<= 96) received pilot REs per filter block and nOut output
 * subcarriers per block; Wf is [nOut][nPilot], OCC [nPorts][occLen], all
 * complex half.  This is the [64 x 96] x [96 x 4] GEMM per output subcarrier
 * (64 antennas, 96 pilots, 4 ports, batched over subcarriers, symbols and
 * blocks) that the reference names as future work (README.md:200, cuPHY
 * channel_est.cu, not in the reference); it has no reference kernel, and the
 * sum is the SRS filter multiply's with nOut != nPilot allowed (nOut ==
 * nPilot gives aerial_srs_to_channel's result bit for bit).  FP32
 * accumulation. */
int aerial_chest_interp(aerial_cf32* H, const aerial_ch2* Yp, const aerial_ch2* Wf,
                        const aerial_ch2* OCC, int nAnt, int nBlocks, int nPilot, int nOut,
                        int nPorts, int occLen, void* stream);

/* The same filter writing the channel as complex half (H[blk*nOut + o][ant][p]
 * in aerial_ch2): the H input of an AERIAL_FMT_CF16 cell.  Each value is
 * aerial_chest_interp's FP32 sum rounded once to half (round to nearest
 * even), bit for bit.  New: the reference has no FP16 channel producer. */
int aerial_chest_interp_h(aerial_ch2* H, const aerial_ch2* Yp, const aerial_ch2* Wf,
                          const aerial_ch2* OCC, int nAnt, int nBlocks, int nPilot, int nOut,
                          int nPorts, int occLen, void* stream);

/* ------------------------------------------------------------------------ */
/* Fused chain: Gram -> FP32 MMSE solve -> apply -> LLR in one kernel; G, C */
/* and Y_eq stay on chip, only LLRs (and optionally Y_eq) are written.       */
/* ------------------------------------------------------------------------ */

/* Storage format of a cell's buffers (aerial_cell_desc.format).
 *  AERIAL_FMT_CF32: H, Y_rx, Y_eq complex float32 (aerial_cf32), LLRs float32
 *                   -- the drop-in layout.
 *  AERIAL_FMT_CF16: H, Y_rx, Y_eq complex half (aerial_ch2), LLRs __half --
 *                   half the bytes; the LLR storage of the reference's
 *                   demapper (src/llr/aerial_llr_v3.cu:84-108).  Supported,
 *                   with FP16 operands, for any mix of cells whose nLayers is
 *                   2, 4, 8 or 16 and whose nAnt is a multiple of 16, with
 *                   16-byte aligned H and Y_rx (else AERIAL_ERR_UNSUPPORTED);
 *                   uniform batches of 4, 8 or 16 layers and 32, 64 or 128
 *                   antennas take an unrolled kernel. */
enum { AERIAL_FMT_CF32 = 0, AERIAL_FMT_CF16 = 1 };

/* One cell-slot.  nSC = 12 * nPRB.  Y_eq may be NULL.  Pointer types name
 * the AERIAL_FMT_CF32 layout; with AERIAL_FMT_CF16 they point at the half
 * formats of the same shapes.  All cells of one launch share a format. */
typedef struct {
    const aerial_cf32* H;      /* [nSC][nAnt][nLayers] */
    const aerial_cf32* Y_rx;   /* [nSC][nSym][nAnt] */
    float* llr;                /* [nSC*nLayers*nSym][2*nPamBits] float32 */
    aerial_cf32* Y_eq;         /* optional [nSC][nLayers][nSym] (unbiased) */
    float sigma2;              /* noise variance per receive antenna */
    int nPRB, nAnt, nLayers, nSym, nPamBits;
    int format;                /* AERIAL_FMT_*; 0 (zero-initialised) = CF32 */
} aerial_cell_desc;

/* Operand precision of the tensor-core products.
 *
 * Input range.  BF16 and BF16X3 keep the FP32 exponent range.  FP16 keeps 11
 * significant bits only between 2^-14 and 65504, so the complex64 path scales
 * each cell's H and Y_rx by an exact power of two s before rounding them to
 * FP16 whenever its sigma2 lies outside [2^-16, 2^7), bringing s^2 sigma2 into
 * [2^-10, 2^-8), and uses s^2 sigma2 as the noise variance.  Scaling H, Y_rx
 * and sigma2 together by any power of two therefore leaves Y_eq, the noise
 * estimates and the LLRs unchanged.  The scale comes from sigma2 alone: it
 * assumes sigma2 is the noise of the same samples, and within the window the
 * raw operands cover received samples up to about 75 dB above the noise.
 * sigma2 = 0 (zero forcing) takes no scale, so H and Y_rx must then lie within
 * the FP16 range themselves.  AERIAL_FMT_CF16 cells are read as stored: their
 * producer chooses the scale (aerial_fp16_operand_scale gives the one the
 * complex64 path would use). */
enum {
    AERIAL_PREC_FP16 = 0,      /* FP16 operands, FP32 accumulation */
    AERIAL_PREC_BF16 = 1,      /* BF16 operands, FP32 accumulation */
    AERIAL_PREC_BF16X3 = 2,    /* BF16 hi/lo split, 3 products, FP32 accumulation */
    AERIAL_PREC_FP32 = 3,      /* FP32 CUDA-core products: the plain chain
                                  (aerial_pusch_eq_plain, the serving loop's
                                  plain mode); the fused entry points return
                                  AERIAL_ERR_UNSUPPORTED */
    AERIAL_PREC_FP16X3 = 4     /* FP16 hi/lo split (about 22 significant bits),
                                  3 products, FP32 accumulation; complex64
                                  cells only, operands always normalized by a
                                  power of two to s^2 sigma2 in [1/4, 1) so the
                                  low halves stay normal */
};

/* The power-of-two operand scale the FP16 path applies to a complex64 cell
 * with noise variance sigma2 (1 inside the window above, or for sigma2 = 0).
 * A producer writing complex-half H and Y_rx can store them times this scale
 * and pass sigma2 times its square.  Host function, no device work.  New:
 * the reference converts FP32 to FP16 unscaled
 * (src/aerial_coef_wmma.cu:165-192) on U(-0.5, 0.5) data only. */
float aerial_fp16_operand_scale(float sigma2);

/* Launch shape; zero fields take the autotuned / default value.  A shape
 * whose CTAs per SM do not fit the launch's shared memory (e.g. one tuned on
 * a different batch) runs with the CTAs per SM that fit. */
typedef struct {
    int precision;             /* AERIAL_PREC_* */
    int warps_per_cta;         /* 0 = default */
    int ctas_per_sm;           /* 0 = default */
    int sc_per_group;          /* cap on the subcarriers a warp solves together
                                  (min(32 / layer tile, cap)); 0 = default (4:
                                  short groups, so no warp of an uneven batch
                                  is left with a few long ones) */
} aerial_tuning;

/* Equalize nCells cell-slots in ONE persistent launch (cells may differ in
 * PRBs, antennas, layers, symbols and modulation).  `cells` is a HOST array
 * (copied into the launch's parameters); its buffers are device pointers.
 * Results per subcarrier do not depend on which other cells share the
 * launch.  nCells <= AERIAL_MAX_CELLS.  tuning may be NULL.
 * Work distribution: a uniform batch (every cell the same 2/4/8/16-layer
 * tile and 32/64/128 antennas) hands its groups of subcarriers to warps from
 * a counter in the library's device memory, one counter per stream that
 * launches and per graph (64 per device), so launches that may overlap never
 * share one; a launch being stream-captured, one that finds no counter free,
 * mixed batches, and every launch while the environment variable
 * AERIAL_STATIC_WALK is set to a non-zero value use a fixed round-robin
 * assignment instead.  The outputs are the same bit for bit either way.
 * No reference counterpart as one kernel: the reference chains gram_scalar,
 * coef_apply and a demapper as separate launches (src/pipeline_overlap.cu:293-301). */
int aerial_pusch_eq_fused(const aerial_cell_desc* cells, int nCells, const aerial_tuning* tuning,
                          void* stream);

/* The fused chain on HOST buffers: each cell's H, Y_rx, llr (and optional
 * Y_eq) are host pointers (page-locked for the copies to overlap).  Cells
 * run in batches of cellsPerBatch (0 = automatic: batches of at least 4 MiB
 * of input) through three internal streams, so host-to-device copies, fused
 * launches and device-to-host copies of successive batches overlap.  The
 * caller's device workspace (256-byte aligned, size from
 * aerial_pusch_eq_host_workspace) stages the batches.  Everything is
 * enqueued asynchronously behind the work already on `stream`, and `stream`
 * waits for all of it: synchronize `stream` before reading the outputs.  Any
 * number of cells; the first call on a device creates the internal streams,
 * and calls from several host threads take turns while they enqueue.  On an
 * error return the batches enqueued before the failing one still run, and
 * `stream` still waits for them.
 * Replaces the reference's blocking cudaMemcpy staging around its launches
 * (src/aerial_coef_wmma.cu:396-397, :414-416). */
int aerial_pusch_eq_host_workspace(const aerial_cell_desc* cells, int nCells, int cellsPerBatch,
                                   size_t* bytes);
int aerial_pusch_eq_host(const aerial_cell_desc* cells, int nCells, const aerial_tuning* tuning,
                         int cellsPerBatch, void* workspace, size_t workspaceBytes, void* stream);

/* The plain FP32 chain for the same cells: aerial_gram, aerial_mmse_coef,
 * aerial_coef_apply and aerial_llr_f32 per cell, intermediates in the
 * caller's workspace (size from aerial_pusch_eq_plain_workspace).  This is
 * the reference's stage-by-stage scalar method on the GPU. */
size_t aerial_pusch_eq_plain_workspace(const aerial_cell_desc* cells, int nCells);
int aerial_pusch_eq_plain(const aerial_cell_desc* cells, int nCells, void* workspace,
                          size_t workspaceBytes, void* stream);

/* The plain chain for callers that cannot allocate device memory -- a
 * real-time slot loop where cudaMalloc may block or synchronize the device,
 * or a plugin whose host framework owns all device memory.  No counterpart in
 * the reference.  Same cells and results as aerial_pusch_eq_plain, but the
 * intermediates live in one static device array of
 * AERIAL_STATIC_SCRATCH_BYTES (16 MiB) inside this library, held on every GPU
 * that loads it until exit; a batch whose largest cell needs more (see
 * aerial_pusch_eq_plain_workspace; e.g. a 273-PRB, 128-antenna, 16-layer
 * cell) is rejected with AERIAL_ERR_SCRATCH_LIMIT before anything runs.
 * Malformed cells return AERIAL_ERR_INVALID_ARG (or AERIAL_ERR_UNSUPPORTED
 * for a complex-half cell) before the size check.  The first call in each
 * CUDA context looks up the array's device address: once per device, and
 * again after a cudaDeviceReset or in a second context on the same device,
 * each of which holds its own copy of the array (make that call before any
 * stream capture).  Calls share the array, so calls that overlap on the GPU
 * race; nothing is allocated or freed. */
#define AERIAL_STATIC_SCRATCH_BYTES (16u << 20)
int aerial_pusch_eq_plain_static(const aerial_cell_desc* cells, int nCells, void* stream);

/* The same fused launch as an executable CUDA graph (one kernel node, built
 * without stream capture).  aerial_eq_graph_update re-points the node at new
 * buffers / sigma2 of cells with the same shapes (AERIAL_ERR_UNSUPPORTED if a
 * shape changes); launching replays the graph on `stream`.  A graph of a
 * uniform batch holds its own work counter (see aerial_pusch_eq_fused) until
 * it is destroyed; replays of one graph must not overlap one another, which
 * CUDA already ensures for launches of one executable graph.  No counterpart
 * in the reference (it has no graphs). */
typedef struct aerial_eq_graph aerial_eq_graph;
int aerial_eq_graph_create(const aerial_cell_desc* cells, int nCells, const aerial_tuning* tuning,
                           aerial_eq_graph** out);
int aerial_eq_graph_update(aerial_eq_graph* graph, const aerial_cell_desc* cells, int nCells);
int aerial_eq_graph_launch(aerial_eq_graph* graph, void* stream);
int aerial_eq_graph_destroy(aerial_eq_graph* graph);

/* ------------------------------------------------------------------------ */
/* Slot-serving loop                                                          */
/*                                                                            */
/* Cells are registered once; their channel estimate H and noise variance     */
/* stay resident in device memory owned by the server (refreshed by           */
/* aerial_server_set_channel or, on the device, by an SRS filter-multiply     */
/* update).  A slot request names the slot's received samples and LLR output  */
/* in device memory.  Requests are admitted against a device-memory budget   */
/* (resident channels + the buffers of every admitted request); one that does */
/* not fit waits, in arrival order.  A dispatcher thread launches whatever is */
/* admitted and pending as one fused kernel whenever one of the server's      */
/* streams is free, so batches overlap on the device; results per subcarrier  */
/* are independent of the batch.  No counterpart in the reference, whose     */
/* multi-cell study runs one kernel per cell on its own stream                */
/* (src/multicell_contention.cu:167-235).                                     */
/* ------------------------------------------------------------------------ */
enum { AERIAL_SERVER_FUSED = 0, AERIAL_SERVER_PLAIN = 1 };

typedef struct {
    int64_t memory_budget_bytes;  /* device-memory admission budget */
    int streams;                  /* batches in flight at once (1..16) */
    int max_batch;                /* cell-slots per launch (1..AERIAL_MAX_CELLS) */
    int precision;                /* AERIAL_PREC_* of the fused kernel */
    int mode;                     /* AERIAL_SERVER_FUSED, or AERIAL_SERVER_PLAIN: the plain FP32
                                     chain request by request (comparison) */
    int queue_capacity;           /* pending requests accepted (0 = unbounded) */
    int start_paused;             /* 1: queue without dispatching until aerial_server_pause(s, 0) */
    float deadline_us;            /* slot deadline counted by the statistics */
    float batch_window_us;        /* launch a batch smaller than min_batch only once its oldest
                                     slot has waited this long (0 = launch at once) */
    int min_batch;                /* see batch_window_us (0 or 1 = no minimum) */
} aerial_server_config;

typedef struct {
    uint64_t request_id;
    int cell_id;
    int status;                   /* 0 or the launch's status */
    float latency_us;             /* completion - arrival */
} aerial_server_completion;

typedef struct {
    long slots_done;
    float p50_us, p99_us, max_us, mean_us;   /* slot latency: completion - arrival */
    float queue_p99_us;           /* arrival -> launch */
    float service_p99_us;         /* launch -> completion observed */
    long deadline_misses;
    long res_done;                /* equalized REs (subcarrier x symbol) */
    double span_s;                /* first arrival -> last completion */
    double res_per_s;
    long batches;
    float mean_batch;             /* cell-slots per launch */
    long srs_updates;
    int64_t budget_used_bytes;
    long pending;
    /* where the tail comes from (host clock) */
    float submit_lag_p99_us, submit_lag_max_us;   /* arrival stamp -> submit call (client side) */
    float dispatch_gap_max_us;    /* longest dispatcher iteration while work was pending or in flight */
    float launch_call_max_us;     /* longest host call that enqueued a batch */
    long misses_late_submit;      /* deadline misses submitted more than half a deadline late */
} aerial_server_statistics;

typedef struct aerial_server aerial_server;

int aerial_server_create(const aerial_server_config* cfg, aerial_server** out);
int aerial_server_destroy(aerial_server* server);
int aerial_server_add_cell(aerial_server* server, int nPRB, int nAnt, int nLayers, int nSym, int nPamBits,
                           float sigma2, int* cellId);
/* Copy a channel estimate (host or device memory) into the cell's resident H. */
int aerial_server_set_channel(aerial_server* server, int cellId, const aerial_cf32* H, float sigma2);
/* Queue an SRS update: filter multiply into the cell's resident H (one SRS
 * port per layer, K subcarriers per block); slots queued after it see it. */
int aerial_server_srs_update(aerial_server* server, int cellId, const aerial_ch2* SRS, const aerial_ch2* W,
                             const aerial_ch2* FOCC, int K, int foccLen, uint64_t* requestId);
/* The same over nSrsSym (1, 2 or 4) SRS symbols whose estimates are averaged
 * (aerial_srs_to_channel_avg); aerial_server_srs_update is nSrsSym = 1. */
int aerial_server_srs_update_n(aerial_server* server, int cellId, const aerial_ch2* SRS, int nSrsSym,
                               const aerial_ch2* W, const aerial_ch2* FOCC, int K, int foccLen,
                               uint64_t* requestId);
/* Queue one slot: Y_rx [nSC][nSym][nAnt] in, LLRs out (device memory).
 * arrival_ns: steady-clock arrival time in ns (0 = now). */
int aerial_server_submit(aerial_server* server, int cellId, const aerial_cf32* Y_rx, float* llr,
                         int64_t arrival_ns, uint64_t* requestId);
int aerial_server_poll(aerial_server* server, aerial_server_completion* out, int maxOut, int* nOut);
int aerial_server_wait(aerial_server* server, uint64_t requestId, int timeout_ms);
int aerial_server_drain(aerial_server* server, int timeout_ms);
int aerial_server_pause(aerial_server* server, int paused);
int aerial_server_stats(aerial_server* server, aerial_server_statistics* out);
/* Forget the latency samples and counters gathered so far (e.g. after warm-up). */
int aerial_server_reset_stats(aerial_server* server);
/* Fault injection for tests: the nth device allocation the server makes from
 * now on (nth >= 1; aerial_server_add_cell makes one for the resident channel
 * and, in AERIAL_SERVER_PLAIN mode, one workspace per stream when the cell is
 * the largest so far) fails with cudaErrorMemoryAllocation without calling
 * the CUDA runtime; 0 disarms.  Host side only.  A failed allocation leaves
 * the server as it was. */
int aerial_server_inject_alloc_failure(aerial_server* server, int nth);

/* ------------------------------------------------------------------------ */
/* Autotuner                                                                  */
/* ------------------------------------------------------------------------ */

/* Time the fused kernel on `cells` for each candidate group cap and launch
 * shape and write the fastest into *best (precision is taken from *best on
 * entry; sc_per_group, warps_per_cta and ctas_per_sm are written).
 * Runs synchronously on `stream`.  Returns the best time in microseconds via
 * *bestUs (may be NULL). */
int aerial_autotune(const aerial_cell_desc* cells, int nCells, aerial_tuning* best, float* bestUs,
                    void* stream);

#ifdef __cplusplus
}
#endif
#endif /* AERIAL_EQ_H */
