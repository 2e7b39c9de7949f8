// host.cu -- the fused chain on HOST buffers: the cells' H and Y_rx are copied
// in, equalized and their LLRs (and optional Y_eq) copied back, pipelined over
// three internal streams so that the host-to-device copies of one batch of
// cells, the fused launch of the previous batch and the device-to-host copies
// of the one before run at the same time (the PCIe link, not the kernel,
// bounds this path).
//
// The reference stages every buffer with blocking cudaMemcpy around its
// launches (src/aerial_coef_wmma.cu:396-397 and :414-416, src/pipeline_overlap.cu:225-231);
// this entry point is that call pattern made asynchronous.
#include <mutex>

#include "common.cuh"

namespace aeq {

constexpr int kPipeSlots = 3;          // internal streams / workspace slots
constexpr size_t kAlign = 256;
// A batch carries at least this many input bytes, so small cells do not pay
// one copy setup per cell (the automatic batch size).
constexpr size_t kMinBatchBytes = 4u << 20;

struct HostPipe {
    cudaStream_t s[kPipeSlots];
    cudaEvent_t start, join[kPipeSlots];
};

static std::mutex g_pipe_mu;
static HostPipe* g_pipes[64];

static size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }

struct CellBytes {
    size_t h, y, llr, yeq;
};

// Complex samples are 8 bytes and LLRs 4 in AERIAL_FMT_CF32, half that in
// AERIAL_FMT_CF16.
static CellBytes cell_bytes(const aerial_cell_desc& c) {
    const size_t nSC = (size_t)c.nPRB * 12;
    const size_t cs = c.format == AERIAL_FMT_CF16 ? 4 : 8;
    CellBytes b;
    b.h = nSC * c.nAnt * c.nLayers * cs;
    b.y = nSC * c.nSym * c.nAnt * cs;
    b.llr = nSC * c.nLayers * c.nSym * 2 * c.nPamBits * (cs / 2);
    b.yeq = c.Y_eq ? nSC * c.nLayers * c.nSym * cs : 0;
    return b;
}

static size_t cell_footprint(const aerial_cell_desc& c) {
    const CellBytes b = cell_bytes(c);
    return align_up(b.h) + align_up(b.y) + align_up(b.llr) + align_up(b.yeq);
}

// Host-side envelope of one cell (the device-side checks run again on the
// staged descriptors inside aerial_pusch_eq_fused).
static bool host_cell_ok(const aerial_cell_desc& c) {
    return c.H && c.Y_rx && c.llr && c.nPRB >= 1 && c.nPRB <= AERIAL_MAX_PRB && c.nAnt >= 1 && c.nAnt <= AERIAL_MAX_ANTS && c.nLayers >= 1 &&
           c.nLayers <= AERIAL_MAX_LAYERS && c.nSym >= 1 && c.nSym <= AERIAL_MAX_SYMS && c.nPamBits >= 1 &&
           c.nPamBits <= 4 && c.sigma2 >= 0.f && (c.format == AERIAL_FMT_CF32 || c.format == AERIAL_FMT_CF16);
}

// Cells per batch: the caller's value, or the smallest count whose input
// bytes reach kMinBatchBytes (at least one cell), capped by the fused
// launch's cell limit.
static int batch_size(const aerial_cell_desc* cells, int nCells, int cellsPerBatch) {
    if (cellsPerBatch > 0) return cellsPerBatch < AERIAL_MAX_CELLS ? cellsPerBatch : AERIAL_MAX_CELLS;
    size_t in = 0;
    for (int i = 0; i < nCells; i++) {
        const CellBytes b = cell_bytes(cells[i]);
        in += b.h + b.y;
    }
    const size_t perCell = in / (size_t)nCells;
    size_t k = perCell ? (kMinBatchBytes + perCell - 1) / perCell : 1;
    if (k < 1) k = 1;
    if (k > AERIAL_MAX_CELLS) k = AERIAL_MAX_CELLS;
    return (int)k;
}

// Bytes of one workspace slot: the largest batch's footprint.
static size_t slot_bytes(const aerial_cell_desc* cells, int nCells, int bs) {
    size_t best = 0;
    for (int b0 = 0; b0 < nCells; b0 += bs) {
        size_t v = 0;
        for (int i = b0; i < nCells && i < b0 + bs; i++) v += cell_footprint(cells[i]);
        best = v > best ? v : best;
    }
    return best;
}

// The internal streams and events of the current device, created on the
// first call on that device.
static int host_pipe(HostPipe** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return rt_status(e);
    if (dev < 0 || dev >= 64) return AERIAL_ERR_UNSUPPORTED;
    if (!g_pipes[dev]) {
        HostPipe* p = new HostPipe();
        for (int k = 0; k < kPipeSlots && e == cudaSuccess; k++) {
            e = cudaStreamCreateWithFlags(&p->s[k], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->join[k], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->start, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            delete p;  // the handles made so far stay with the context
            return rt_status(e);
        }
        g_pipes[dev] = p;
    }
    *out = g_pipes[dev];
    return AERIAL_OK;
}

}  // namespace aeq

using namespace aeq;

extern "C" int aerial_pusch_eq_host_workspace(const aerial_cell_desc* cells, int nCells, int cellsPerBatch,
                                              size_t* bytes) {
    if (!cells || !bytes || nCells < 1 || cellsPerBatch < 0) return AERIAL_ERR_INVALID_ARG;
    for (int i = 0; i < nCells; i++)
        if (!host_cell_ok(cells[i])) return AERIAL_ERR_INVALID_ARG;
    const int bs = batch_size(cells, nCells, cellsPerBatch);
    const int nBatch = (nCells + bs - 1) / bs;
    const int slots = nBatch < kPipeSlots ? nBatch : kPipeSlots;
    *bytes = (size_t)slots * slot_bytes(cells, nCells, bs);
    return AERIAL_OK;
}

extern "C" int aerial_pusch_eq_host(const aerial_cell_desc* cells, int nCells, const aerial_tuning* tuning,
                                    int cellsPerBatch, void* workspace, size_t workspaceBytes, void* stream) {
    if (!cells || nCells < 1 || cellsPerBatch < 0 || !workspace || ((uintptr_t)workspace & (kAlign - 1)))
        return AERIAL_ERR_INVALID_ARG;
    for (int i = 0; i < nCells; i++)
        if (!host_cell_ok(cells[i])) return AERIAL_ERR_INVALID_ARG;
    const int bs = batch_size(cells, nCells, cellsPerBatch);
    const int nBatch = (nCells + bs - 1) / bs;
    const int slots = nBatch < kPipeSlots ? nBatch : kPipeSlots;
    const size_t perSlot = slot_bytes(cells, nCells, bs);
    if (workspaceBytes < (size_t)slots * perSlot) return AERIAL_ERR_INVALID_ARG;

    std::lock_guard<std::mutex> lock(g_pipe_mu);
    HostPipe* hp = nullptr;
    int st = host_pipe(&hp);
    if (st) return st;
    const cudaStream_t caller = to_stream(stream);
    cudaError_t e = cudaEventRecord(hp->start, caller);
    for (int k = 0; k < slots && e == cudaSuccess; k++) e = cudaStreamWaitEvent(hp->s[k], hp->start, 0);
    if (e != cudaSuccess) return rt_status(e);

    // Batch b runs on stream b % slots with workspace slot b % slots: the
    // stream order keeps a slot's next batch behind its previous copies out.
    aerial_cell_desc dev[AERIAL_MAX_CELLS];
    for (int b = 0; b < nBatch && st == AERIAL_OK; b++) {
        const int k = b % slots;
        const cudaStream_t s = hp->s[k];
        char* base = static_cast<char*>(workspace) + (size_t)k * perSlot;
        const int c0 = b * bs, n = (nCells - c0) < bs ? (nCells - c0) : bs;
        for (int j = 0; j < n && e == cudaSuccess; j++) {
            const aerial_cell_desc& c = cells[c0 + j];
            const CellBytes cb = cell_bytes(c);
            aerial_cell_desc& d = dev[j];
            d = c;
            d.H = reinterpret_cast<const aerial_cf32*>(base);
            base += align_up(cb.h);
            d.Y_rx = reinterpret_cast<const aerial_cf32*>(base);
            base += align_up(cb.y);
            d.llr = reinterpret_cast<float*>(base);
            base += align_up(cb.llr);
            d.Y_eq = c.Y_eq ? reinterpret_cast<aerial_cf32*>(base) : nullptr;
            base += align_up(cb.yeq);
            e = cudaMemcpyAsync(const_cast<aerial_cf32*>(d.H), c.H, cb.h, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(const_cast<aerial_cf32*>(d.Y_rx), c.Y_rx, cb.y, cudaMemcpyHostToDevice, s);
        }
        if (e != cudaSuccess) break;
        st = aerial_pusch_eq_fused(dev, n, tuning, s);
        if (st) break;
        for (int j = 0; j < n && e == cudaSuccess; j++) {
            const aerial_cell_desc& c = cells[c0 + j];
            const CellBytes cb = cell_bytes(c);
            e = cudaMemcpyAsync(c.llr, dev[j].llr, cb.llr, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess && c.Y_eq) e = cudaMemcpyAsync(c.Y_eq, dev[j].Y_eq, cb.yeq, cudaMemcpyDeviceToHost, s);
        }
    }
    // Join every internal stream back into the caller's stream, also after an
    // error, so the caller's stream never runs ahead of copies in flight.
    cudaError_t je = cudaSuccess;
    for (int k = 0; k < slots; k++) {
        cudaError_t r = cudaEventRecord(hp->join[k], hp->s[k]);
        if (r == cudaSuccess) r = cudaStreamWaitEvent(caller, hp->join[k], 0);
        if (r != cudaSuccess && je == cudaSuccess) je = r;
    }
    if (st) return st;
    if (e != cudaSuccess) return rt_status(e);
    return rt_status(je);
}
