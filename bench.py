#!/usr/bin/env python3
"""Benchmark of the fused PUSCH equalization path (Gram + MMSE solve + apply + LLR).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): a batch of S cell-slots of the 100 MHz reference cell --
132 PRB = 1584 subcarriers, 64 receive antennas, 8 layers, 11 data symbols,
256-QAM, SNR 25 dB, per-PRB channel with a per-subcarrier perturbation --
equalized by ONE persistent fused launch.  Inputs are seeded synthetic slots
generated on the device (S * 15.4 MB of H + Y_rx, S * 4.46 MB of LLRs), larger
than L2 at the default S = 64 (1.27 GB per step).  Metric: equalized REs/s, RE = one
(subcarrier, data symbol) of one cell with all its layers.

One JSON line is printed by rank 0.  Under torchrun each rank equalizes its
own S slots (independent cells, no collective on the data path: weak
scaling); the elapsed time is the max over ranks.

--impl reference times the reference's scalar FP32 chain restated as host
C code (the checker library), on the host cores, over a bounded sample of
the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "equalized REs/s (Gram+solve+apply+LLR)"
UNIT = "REs/s"
WORKLOAD = ("PUSCH equalization, 132 PRB = 1584 subcarriers x 64 Rx antennas x 8 layers x 11 data symbols, "
            "256-QAM, SNR 25 dB, per-PRB CN(0,1/64) channel + per-subcarrier perturbation; "
            "Gram -> FP32 Cholesky MMSE -> apply -> max-log LLR (float32)")
WORKLOADS = {
    1: ("plain-chain cell: 24 PRB = 288 subcarriers x 32 Rx antennas x 4 layers x 11 data symbols, 16-QAM, "
        "SNR 20 dB, i.i.d. CN(0,1/32) channel"),
    2: WORKLOAD,
    3: ("precision stress: 273 PRB = 3276 subcarriers x 128 Rx antennas x 16 layers x 11 data symbols, 256-QAM, "
        "SNR 30 dB, exponentially correlated (rho = 0.7) receive antennas"),
    4: ("uneven 16-cell batch in one persistent launch: PRB in {24,51,106,132,273}, antennas in {16,32,64}, "
        "layers in {2,4,8}, QPSK..256-QAM, SNR U(10,30) dB, from a seed"),
}
DEFAULT_SLOTS = {1: 960, 2: 64, 3: 12, 4: 16}
DEFAULT_PRECISION = {1: "fp16", 2: "fp16", 3: "bf16x3", 4: "fp16", 5: "fp16"}
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5],
                    help="benchmark configuration (2 = the headline 100 MHz cell)")
    ap.add_argument("--slots", type=int, default=0, help="cell-slots per step per GPU (0 = the config's default)")
    ap.add_argument("--precision", default="", choices=["", "fp16", "bf16", "bf16x3", "fp16x3"])
    ap.add_argument("--io", default="cf32", choices=["cf32", "fp16"],
                    help="storage of H / Y_rx / LLRs: cf32 = the drop-in complex64 layout (default); fp16 = complex "
                         "half in, __half LLRs out (configs 1, 2 and 3 with FP16 operands), reported as its own line")
    ap.add_argument("--duration", type=float, default=1.0, help="serving run length in seconds (config 5)")
    ap.add_argument("--window-us", type=float, default=-1.0,
                    help="serving batching window (config 5; -1 = the default, 0 = launch at once)")
    ap.add_argument("--min-batch", type=int, default=-1, help="serving minimum batch before the window ends (-1 = default)")
    ap.add_argument("--serve-streams", type=int, default=0, help="serving batches in flight (0 = default)")
    ap.add_argument("--srs-symbols", type=int, default=4, choices=[1, 2, 4],
                    help="SRS symbols averaged by each serving SRS update (config 5)")
    ap.add_argument("--soak", type=float, default=1.5, help="seconds of untimed load before timing (clock steady state)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip plain-chain / EVM / latency extras")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def ncu_traffic_per_slot(config: int):
    """DRAM bytes per cell-slot of the fused kernel for this benchmark
    configuration, from the committed ncu summary (None if not captured)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("fused_eq_kernel", {}).get(f"config{config}", {}).get("dram_bytes_per_slot")
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons while the GPU is loaded."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def host_cell(wl, cfg: int):
    """One host-resident slot of a configuration for the CPU baseline."""
    if cfg in (1, 2, 3):
        return wl.config_cell(cfg, seed=42)
    return wl.multicell(16, seed=42)[0]


def cell_seeds(cfg: int, slots: int, rank: int):
    """The generator seed of each cell of a rank's step.  Ranks draw from
    disjoint seed sets (weak scaling: every rank equalizes its own slots):
    1000 rank + 17 i + 1 never repeats across ranks for i < 1000, and the
    16-cell batch's per-cell seeds (base + 1000 i) stay below the next rank's
    base of 1,000,000 rank."""
    if cfg in (2, 3):
        return [1000 * rank + 17 * i + 1 for i in range(slots)]
    if cfg == 1:
        per = -(-slots // 64)
        return [1000 * rank + 17 * i + 1 for i in range(-(-slots // per))]
    if cfg == 4:
        base = 42 + 1_000_000 * rank
        return [base + 1000 * i for i in range(slots)]
    raise ValueError(cfg)


def build_cells(wl, cfg: int, slots: int, rank: int, dev):
    """The step's cell-slots.  Slots of one configuration share sigma2, so for
    the small configuration 1 consecutive slots are laid out contiguously and
    described as one cell of slots x 24 PRBs (at most 64 descriptors a launch)."""
    seeds = cell_seeds(cfg, slots, rank)
    if cfg in (2, 3):
        return [wl.config_cell(cfg, seed=sd, device=dev) for sd in seeds]
    if cfg == 1:
        per = -(-slots // 64)
        return [wl.make_cell(24 * per, 32, 4, 11, 16, 20.0, "iid", seed=sd, device=dev) for sd in seeds]
    if cfg == 4:
        return wl.multicell(slots, seed=seeds[0], device=dev)
    raise ValueError(cfg)


def work_walk(cells) -> str:
    """How the timed launch hands groups of subcarriers to warps: uniform
    batches of the unrolled kernels take tickets from a per-stream counter,
    mixed batches (and every launch under AERIAL_STATIC_WALK=1) walk
    round-robin.  Outputs are identical either way."""
    shapes = {(c.nLayers, c.nAnt) for c in cells}
    uniform = len(shapes) == 1 and cells[0].nLayers in (2, 4, 8, 16) and cells[0].nAnt in (32, 64, 128)
    if uniform and os.environ.get("AERIAL_STATIC_WALK", "0") in ("", "0"):
        return "dynamic: groups handed to warps from a per-stream counter"
    return "static round-robin"


def max_over_ranks(values, world: int, device=None):
    """Element-wise max of per-rank timings (ms) across the process group.

    Every rank calls it at the same point with the same number of values.
    With world == 1 it returns the values unchanged."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def whole_job_rate(units_per_rank_per_step: int, steps: int, world: int, max_elapsed_ms: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time (weak scaling)."""
    return world * units_per_rank_per_step * steps / (max_elapsed_ms / 1e3)


def cpu_chain_rate(orc, cell, seconds: float):
    """REs/s of the scalar FP32 chain on the host cores over a bounded sample."""
    H, Y = cell.H.numpy(), cell.Y.numpy()
    args = (cell.sigma2, cell.nSC, cell.nAnt, cell.nLayers, cell.nSym, cell.nPamBits)
    orc.chain_f32(H[:12], Y[:12], cell.sigma2, 12, cell.nAnt, cell.nLayers, cell.nSym, cell.nPamBits)
    t0 = time.perf_counter()
    runs = 0
    while True:
        orc.chain_f32(H, Y, *args)
        runs += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return runs * cell.n_re / el, runs, el


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def run_reference(a, rank):
    if rank != 0:
        return
    from oracle import oracle as orc

    wl = importlib.import_module("aerial-mimo-tc-optimization_b200.workload")
    cores = os.cpu_count() or 1
    orc.set_threads(cores)
    cell = host_cell(wl, a.config if a.config in (1, 2, 3, 4) else 2)
    H, Y = cell.H.numpy(), cell.Y.numpy()
    # calibrate one slot, then size each step so the whole run stays within ~2 minutes
    t0 = time.perf_counter()
    orc.chain_f32(H, Y, cell.sigma2, cell.nSC, cell.nAnt, cell.nLayers, cell.nSym, cell.nPamBits)
    t_slot = time.perf_counter() - t0
    frac = min(1.0, 100.0 / max(1, a.steps + a.warmup) / max(t_slot, 1e-6))
    nprb = max(1, int(round(cell.nPRB * frac)))
    nsc = 12 * nprb
    Hs, Ys = H[:nsc], Y[:nsc]
    args = (cell.sigma2, nsc, cell.nAnt, cell.nLayers, cell.nSym, cell.nPamBits)
    for _ in range(a.warmup):
        orc.chain_f32(Hs, Ys, *args)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        orc.chain_f32(Hs, Ys, *args)
    el = time.perf_counter() - t0
    v = a.steps * nsc * cell.nSym / el
    sample = f"{nprb} of {cell.nPRB} PRB ({nsc} subcarriers) of one slot per step, OpenMP over subcarriers"
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * el / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOADS.get(a.config, WORKLOAD), "benchmark_config": a.config, "sample": sample},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "notes": "scalar FP32 chain of the reference (gram_scalar, Cholesky solve, coef_apply_v1_scalar, "
                 "llr_v1_baseline) restated as C and run on the host cores",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def main():
    a = parse()
    if not a.precision:
        a.precision = DEFAULT_PRECISION[a.config]
    if not a.slots:
        a.slots = DEFAULT_SLOTS.get(a.config, 64)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank)
        return

    import torch
    import torch.distributed as dist

    aeq = importlib.import_module("aerial-mimo-tc-optimization_b200")
    wl = importlib.import_module("aerial-mimo-tc-optimization_b200.workload")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    if a.config == 5:
        run_serving(a, aeq, wl, dev)
        return
    S = a.slots
    cells = build_cells(wl, a.config, S, rank, dev)
    half = a.io == "fp16"
    if half:
        if a.config not in (1, 2, 3, 4) or a.precision != "fp16":
            raise SystemExit("--io fp16 runs configurations 1-4 with fp16 operands "
                             "(configuration 3: --precision fp16)")
        a.no_extras = True          # the extras run the complex64 plain chain
        # the same slots stored as complex half; the complex64 copies are dropped
        for c in cells:
            c.H = torch.view_as_real(c.H).to(torch.float16).contiguous()
            c.Y = torch.view_as_real(c.Y).to(torch.float16).contiguous()
        torch.cuda.empty_cache()
    fmt = aeq.FMT_CF16 if half else aeq.FMT_CF32
    ldt = torch.float16 if half else torch.float32
    llrs = [torch.empty(c.llr_numel, dtype=ldt, device=dev) for c in cells]
    descs = [aeq.cell_desc(c.H, c.Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, fmt=fmt)
             for c, l in zip(cells, llrs)]
    tun = aeq.make_tuning(a.precision)
    if os.environ.get("AERIAL_AUTOTUNE", "1") == "1":
        tun, _ = aeq.autotune(descs, a.precision)
    stream = torch.cuda.current_stream()
    res_per_step = sum(c.n_re for c in cells)
    bytes_per_step = sum(c.algorithmic_bytes() for c in cells) // (2 if half else 1)
    in_bytes_per_step = sum(c.H.numel() * c.H.element_size() + c.Y.numel() * c.Y.element_size() for c in cells)
    out_bytes_per_step = sum(l.numel() * l.element_size() for l in llrs)

    # Configuration 4 is specified as one persistent launch under a CUDA graph:
    # its step replays the captured launch (aerial_eq_graph_launch)
    graph = aeq.FusedGraph(descs, tun) if a.config == 4 else None

    def step():
        if graph is not None:
            graph.launch(stream)
        else:
            aeq.pusch_eq_fused(descs, tun, stream)

    flush = None
    if bytes_per_step < 2 * L2_BYTES:
        # the step fits (or nearly fits) in L2: flush it before every timed launch
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    t_end = time.time() + a.soak
    while time.time() < t_end:
        for _ in range(50):
            step()
        torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")          # ncu --nvtx --nvtx-include "timed/" lists these launches
    e0.record(stream)
    for i in range(a.steps):
        if flush is not None:
            flush.fill_(float(i))
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier()
    clocks = sampler.stop()
    launch_ms = [s.elapsed_time(e) for s, e in ev]
    # with L2 flushes between launches only the launches are timed
    elapsed_ms = e0.elapsed_time(e1) if flush is None else sum(launch_ms)
    elapsed_ms, launch_avg_ms = max_over_ranks([elapsed_ms, statistics.mean(launch_ms)], world, dev)
    value = whole_job_rate(res_per_step, a.steps, world, elapsed_ms)
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_step / (launch_avg_ms / 1e3) / 1e9
    tr = None if half else ncu_traffic_per_slot(a.config)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": (tr * S) if tr else None, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": bytes_per_step}

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not a.no_e2e:
        hH = [c.H.cpu().pin_memory() for c in cells]
        hY = [c.Y.cpu().pin_memory() for c in cells]
        hL = [torch.empty(c.llr_numel, dtype=ldt).pin_memory() for c in cells]
        hd = [aeq.host_cell_desc(h, y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, fmt=fmt)
              for c, h, y, l in zip(cells, hH, hY, hL)]
        ws = torch.empty(aeq.pusch_eq_host_workspace(hd), dtype=torch.uint8, device=dev)

        def e2e_step():
            aeq.pusch_eq_host(hd, ws, tun, 0, stream)

        k2 = max(3, min(a.steps, 20))
        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(k2):
            e2e_step()
        s1.record(stream)
        torch.cuda.synchronize()
        e2e_ms, = max_over_ranks([s0.elapsed_time(s1)], world, dev)
        e2e = {"value": whole_job_rate(res_per_step, k2, world, e2e_ms), "unit": UNIT,
               "h2d_bytes_per_step": in_bytes_per_step, "d2h_bytes_per_step": out_bytes_per_step,
               "steps": k2,
               "path": "aerial_pusch_eq_host: pinned host H, Y_rx -> device -> fused launch -> pinned host LLR, "
                       "batches overlapped over three streams"}
        # the end-to-end output must equal the resident run's, bit for bit
        torch.cuda.synchronize()
        for i in sorted({0, len(cells) - 1}):
            if not torch.equal(hL[i], llrs[i].cpu()):
                raise RuntimeError(f"end-to-end LLRs of cell {i} differ from the resident launch")
        e2e["parity"] = "host-buffer LLRs equal the resident launch's (checked on the first and last cell)"
        # the box's own host link: the step's inputs copied alone, one stream,
        # from the same pinned buffers onto the device copies they came from
        link_ms = []
        for _ in range(2):
            c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            c0.record(stream)
            with torch.cuda.stream(stream):
                for c, h, y in zip(cells, hH, hY):
                    c.H.copy_(h, non_blocking=True)
                    c.Y.copy_(y, non_blocking=True)
            c1.record(stream)
            torch.cuda.synchronize()
            link_ms.append(c0.elapsed_time(c1))
        link_gbs = in_bytes_per_step / (min(link_ms) / 1e3) / 1e9
        e2e["h2d_link_gbs"] = link_gbs
        e2e["h2d_link_frac"] = in_bytes_per_step / (e2e_ms / k2 / 1e3) / 1e9 / link_gbs
        e2e["link"] = ("h2d_link_gbs: the step's H and Y_rx copied alone from pinned memory on one stream; "
                       "h2d_link_frac: the end-to-end step's input bytes per second over that")

    extras = {}
    cpu_base = None
    if rank == 0 and world == 1 and not a.no_extras:
        extras = bench_extras(aeq, wl, cells, llrs, descs, tun, stream, a)
        if a.config == 2:
            for key, fn in (("path_rates", lambda: path_rates(aeq, descs, res_per_step, bytes_per_step, stream)),
                            ("other_configs", lambda: other_configs(aeq, wl, dev, stream, a))):
                try:   # reported beside the headline; never fatal for the timing line
                    extras[key] = fn()
                except Exception as e:
                    extras[key] = {"error": f"{type(e).__name__}: {e}"}
        if a.config == 4:
            extras["tiles"] = compare_tiles(aeq, descs, tun, stream, a, flush)
            extras["per_cell_streams_vs_batched"] = compare_streams(aeq, descs, tun, a, flush)
            extras["sm_partition_strategies"] = sm_partition_strategies(aeq, wl, aeq.make_tuning("fp16"), dev)
            extras["graph_vs_direct_launch_us"] = {
                "graph_replay": _time_launches(lambda: graph.launch(stream), stream),
                "direct": _time_launches(lambda: aeq.pusch_eq_fused(descs, tun, stream), stream),
                "note": "back-to-back launches of the 16-cell batch, CUDA events around 50"}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        from oracle import oracle as orc

        cores = os.cpu_count() or 1
        orc.set_threads(cores)
        hc = host_cell(wl, a.config)
        v, runs, el = cpu_chain_rate(orc, hc, a.cpu_seconds)
        cpu_base = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                    "sample": f"{runs} full slot(s) ({hc.nSC} subcarriers) in {el:.1f} s, OpenMP over subcarriers"}
        if "srs_filter" in extras:
            r, runs, el = srs_cpu_rate(orc, min(5.0, a.cpu_seconds))
            extras["srs_filter"]["cpu_baseline"] = {
                "value": r, "unit": "SRS blocks/s", "cores": cores, "kind": "port",
                "sample": f"{runs} x the reference's 66-block launch (srs_filter_v1_scalar restated, FP16 "
                          f"arithmetic) in {el:.1f} s, OpenMP over outputs"}
        if not half:
            try:   # the oracle as the checker of slot 0; reported, never fatal for the timing line
                extras["accuracy_vs_fp64"] = accuracy_vs_fp64(orc, aeq, cells, llrs, descs, tun, stream)
                if a.config == 2 and not a.no_extras:
                    c3 = build_cells(wl, 3, 1, 0, dev)
                    l3 = [torch.empty(c3[0].llr_numel, dtype=torch.float32, device=dev)]
                    d3 = [aeq.cell_desc(c3[0].H, c3[0].Y, l3[0], c3[0].sigma2, c3[0].nPRB, c3[0].nAnt,
                                        c3[0].nLayers, c3[0].nSym, c3[0].nPamBits)]
                    extras["accuracy_vs_fp64_config3"] = accuracy_vs_fp64(
                        orc, aeq, c3, l3, d3, aeq.make_tuning("bf16x3"), stream)
            except Exception as e:
                extras["accuracy_vs_fp64"] = {"error": str(e)}
        if a.config == 2 and not a.no_extras:
            try:   # the reference's own kernels on this GPU: a baseline, from the checker libraries
                extras["reference_kernels_on_b200"] = reference_kernels_on_b200(aeq, wl, dev)
            except Exception as e:
                extras["reference_kernels_on_b200"] = {"error": str(e)}

    if graph is not None:
        graph.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC + (" with FP16 I/O" if half else ""), "value": value, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": elapsed_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": a.precision + " operands / fp32 accumulate and solve" + ("; complex-half in, __half LLRs out"
                                                                           if half else ""),
        "data": "synthetic (seeded, generated on device)",
        "config": {"workload": WORKLOADS[a.config], "benchmark_config": a.config, "cells_per_step": len(cells),
                   "slots_per_step_per_gpu": S, "res_per_step_per_gpu": res_per_step,
                   "l2": (f"inputs larger than L2 ({bytes_per_step / 1e6:.0f} MB touched per step per GPU)"
                          if flush is None else
                          f"L2 flushed before each timed launch ({bytes_per_step / 1e6:.0f} MB per step)"),
                   "precision": a.precision, "io": a.io, "tuning": {"warps_per_cta": tun.warps_per_cta,
                                                         "ctas_per_sm": tun.ctas_per_sm},
                   "launch": "CUDA graph replay of the persistent launch" if graph is not None
                             else "one persistent launch per step",
                   "work_walk": work_walk(cells),
                   "parallelism": f"independent cell-slots per GPU x{world}"},
        "roofline": roof,
        "cpu_baseline": cpu_base,
        "e2e": e2e,
        "gpu_launches": a.steps,
        "clocks": clocks,
    }
    line.update(extras)
    print(json.dumps(line), flush=True)


class ServingWorkload:
    """Configuration 5's cells and buffers: 40 cells with shapes drawn as the
    16-cell batch, two received slots per cell (alternated), a ring of 16 LLR
    outputs per cell, and SRS operands (K = 12, one port per layer, averaged
    over `srs_syms` SRS symbols)."""

    def __init__(self, aeq, wl, dev, srs_syms, n_cells=40):
        import torch

        self.aeq, self.n_cells, self.srs_syms = aeq, n_cells, srs_syms
        shapes = wl.multicell_shapes(n_cells, seed=5)
        self.cells, self.Ys, self.rings, self.srs_ops = [], [], [], []
        for i, (p, A, L, q, snr) in enumerate(shapes):
            c = wl.make_cell(p, A, L, 11, q, snr, "iid", seed=5000 + i, device=dev)
            extra = wl.make_cell(p, A, L, 11, q, snr, "iid", seed=7000 + i, device=dev)
            self.cells.append(c)
            self.Ys.append([c.Y, extra.Y])
            self.rings.append([torch.empty(c.llr_numel, dtype=torch.float32, device=dev) for _ in range(16)])
            g = torch.Generator(device=dev)
            g.manual_seed(9000 + i)
            nblk = c.nSC // 12
            self.srs_ops.append([(torch.randn(n, generator=g, device=dev) * 0.5).half().view(torch.int16).contiguous()
                                 for n in (2 * srs_syms * nblk * A * 12, 2 * 12 * 12, 2 * L * 12)])

    def arrivals(self, duration, n_active, per_slot_s=500e-6, seed=11):
        """Poisson slot arrivals of the first n_active cells, mean one per per_slot_s each."""
        import numpy as np

        rng = np.random.default_rng(seed)
        out = []
        for ci in range(n_active):
            t = rng.exponential(per_slot_s)
            while t < duration:
                out.append((t, ci))
                t += rng.exponential(per_slot_s)
        out.sort()
        return out

    def serve(self, arrivals, mode, precision, streams, window_us=0.0, min_batch=0, srs_every=20):
        """Replay an arrival trace against a fresh server; its statistics."""
        import gc

        import torch

        aeq = self.aeq
        lib = aeq.lib()
        srv = aeq.Server(memory_budget_bytes=16 << 30, streams=streams, max_batch=64, precision=precision,
                         mode=mode, deadline_us=500.0, batch_window_us=window_us, min_batch=min_batch)
        active = sorted({ci for _, ci in arrivals})
        ids = {}
        for ci in active:
            c = self.cells[ci]
            k = srv.add_cell(c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, c.sigma2)
            srv.set_channel(k, c.H, c.sigma2)
            ids[ci] = k
        # one untimed SRS update and slot per cell (first launch of every shape), then reset the statistics
        for ci in active:
            ops = self.srs_ops[ci]
            assert lib.aerial_server_srs_update_n(srv._h, ids[ci], ctypes.c_void_p(ops[0].data_ptr()), self.srs_syms,
                                                  ctypes.c_void_p(ops[1].data_ptr()), ctypes.c_void_p(ops[2].data_ptr()),
                                                  12, 12, None) == 0
            srv.submit(ids[ci], self.Ys[ci][0], self.rings[ci][0])
        srv.drain(60000)
        srv.poll(max_out=4096)
        srv.reset_stats()
        yp = {ci: [ctypes.c_void_p(y.data_ptr()) for y in self.Ys[ci]] for ci in active}
        rp = {ci: [ctypes.c_void_p(r.data_ptr()) for r in self.rings[ci]] for ci in active}
        sp = {ci: [ctypes.c_void_p(t.data_ptr()) for t in self.srs_ops[ci]] for ci in active}
        count = dict.fromkeys(active, 0)
        handle = srv._h
        submit, srs_update = lib.aerial_server_submit, lib.aerial_server_srs_update_n
        torch.cuda.synchronize()
        t0 = time.monotonic_ns() + 20_000_000
        plan = [(t0 + int(t * 1e9), ci) for t, ci in arrivals]
        errors = 0
        gc_was = gc.isenabled()
        gc.disable()                    # no collector pause inside the trace (the client is Python)
        try:
            for target, ci in plan:
                while time.monotonic_ns() < target:
                    pass
                k = count[ci]
                count[ci] = k + 1
                if k and k % srs_every == 0:
                    errors += srs_update(handle, ids[ci], sp[ci][0], self.srs_syms, sp[ci][1], sp[ci][2],
                                         12, 12, None) != 0
                errors += submit(handle, ids[ci], yp[ci][k % 2], rp[ci][k % 16], target, None) != 0
        finally:
            if gc_was:
                gc.enable()
        srv.drain(600000)
        st = srv.stats()
        srv.close()
        st["submit_errors"] = int(errors)
        st["miss_rate"] = st["deadline_misses"] / max(1, st["slots_done"])
        # misses of requests the load generator submitted half a deadline late or more
        # are the client's; the rest are the server's own
        st["server_miss_rate"] = (st["deadline_misses"] - st["misses_late_submit"]) / max(1, st["slots_done"])
        st["slots_offered"] = len(arrivals)
        st["streams"], st["batch_window_us"], st["min_batch"] = streams, window_us, min_batch
        return st


SERVE_KEYS = ("slots_offered", "slots_done", "p50_us", "p99_us", "max_us", "mean_us", "queue_p99_us",
              "service_p99_us", "deadline_misses", "miss_rate", "server_miss_rate", "res_per_s", "batches", "mean_batch", "srs_updates",
              "submit_errors", "submit_lag_p99_us", "submit_lag_max_us", "dispatch_gap_max_us", "launch_call_max_us",
              "misses_late_submit", "streams", "batch_window_us", "min_batch")

# Configuration 5's dispatcher settings: batches in flight and batching window.
SERVE_STREAMS, SERVE_WINDOW_US, SERVE_MIN_BATCH = 2, 20.0, 2
# Cells whose Poisson load the plain FP32 chain, request by request, sustains
# (the kernel comparison runs both paths on this lighter trace).
SERVE_LIGHT_CELLS = 4


def serving_summary(a, aeq, wl, dev, duration, streams, window_us, min_batch, compare_plain=True):
    """Configuration 5 on one trace: the fused batched loop at the full 40-cell
    load; and, on a lighter trace of SERVE_LIGHT_CELLS cells that the plain
    FP32 chain sustains, both paths, so their p99 compares kernels rather
    than an unbounded queue."""
    w = ServingWorkload(aeq, wl, dev, a.srs_symbols)
    full = w.serve(w.arrivals(duration, w.n_cells), aeq.SERVER_FUSED, a.precision, streams, window_us, min_batch)
    out = {"fused_batched": {k: full[k] for k in SERVE_KEYS}}
    if compare_plain:
        light = w.arrivals(duration, SERVE_LIGHT_CELLS)
        lf = w.serve(light, aeq.SERVER_FUSED, a.precision, streams, window_us, min_batch)
        lp = w.serve(light, aeq.SERVER_PLAIN, a.precision, streams, 0.0, 0)
        out["light_load"] = {
            "cells": SERVE_LIGHT_CELLS,
            "fused_batched": {k: lf[k] for k in SERVE_KEYS},
            "plain_fp32_per_request": {k: lp[k] for k in SERVE_KEYS},
            "p99_ratio_plain_over_fused": lp["p99_us"] / max(lf["p99_us"], 1e-9)}
    return out


def run_serving(a, aeq, wl, dev):
    """Configuration 5: 40 cells submit slots as Poisson arrivals (mean one
    slot per 500 us per cell) to the serving loop; every 20th slot of a cell
    is preceded by an SRS channel update (filter multiply, K = 12, one port per
    layer, averaged over 4 SRS symbols)."""
    streams = a.serve_streams or SERVE_STREAMS
    window = SERVE_WINDOW_US if a.window_us < 0 else a.window_us
    min_batch = SERVE_MIN_BATCH if a.min_batch < 0 else a.min_batch
    res = serving_summary(a, aeq, wl, dev, a.duration, streams, window, min_batch)
    fused = res["fused_batched"]
    line = {
        "metric": "serving: equalized REs/s with p99 slot latency (deadline 500 us)", "value": fused["res_per_s"],
        "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "benchmark_config": 5,
        "config": {"workload": (f"40 cells, Poisson slot arrivals (mean one per 500 us per cell) for "
                                f"{a.duration:.1f} s, shapes drawn as the 16-cell batch, SRS update (filter multiply "
                                f"averaged over {a.srs_symbols} SRS symbols) every 20 slots, 16 GB admission "
                                f"budget, {streams} streams, up to 64 slots a launch"),
                   "precision": a.precision},
        "data": "synthetic (seeded, generated on device)",
    }
    line.update(res)
    print(json.dumps(line), flush=True)


def compare_tiles(aeq, descs, tuned, stream, a, flush):
    """Configuration 4: autotuned launch shape against the fixed default shape."""
    import torch

    def timed(t, k=20):
        e = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for i in range(k):
            if flush is not None:
                flush.fill_(float(i))
            e[i][0].record(stream)
            aeq.pusch_eq_fused(descs, t, stream)
            e[i][1].record(stream)
        torch.cuda.synchronize()
        ms = sorted(x.elapsed_time(y) for x, y in e)
        return 1e3 * ms[len(ms) // 2]

    fixed = aeq.make_tuning(a.precision)
    return {"autotuned_us": timed(tuned), "fixed_default_us": timed(fixed),
            "autotuned_shape": {"warps_per_cta": tuned.warps_per_cta, "ctas_per_sm": tuned.ctas_per_sm}}


def compare_streams(aeq, descs, tuned, a, flush):
    """Configuration 4, the reference's multi-cell stream study
    (src/multicell_contention.cu:205-235) restated for this path: the 16 cells
    as one launch per cell on 16 concurrent streams (per-cell latency and
    makespan, against each cell alone) versus all cells in one persistent
    batched launch.  A device sleep ahead of each start event keeps host-side
    call overhead out of every interval."""
    import torch

    n = len(descs)
    streams = [torch.cuda.Stream() for _ in range(n)]
    main = torch.cuda.current_stream()
    reps = 10

    def med(v):
        v = sorted(v)
        return v[len(v) // 2]

    alone = []
    for d in descs:
        t = []
        for r in range(reps):
            if flush is not None:
                flush.fill_(float(r))
            torch.cuda._sleep(2_000_000)     # the launch is enqueued before e0 fires
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(main)
            aeq.pusch_eq_fused([d], tuned, main)
            e1.record(main)
            torch.cuda.synchronize()
            t.append(1e3 * e0.elapsed_time(e1))
        alone.append(med(t))
    per_cell, span = [[] for _ in range(n)], []
    for r in range(reps):
        if flush is not None:
            flush.fill_(float(r))
        torch.cuda.synchronize()
        torch.cuda._sleep(2_000_000)         # every launch is enqueued before g0 fires
        g0 = torch.cuda.Event(enable_timing=True)
        g0.record(main)
        ev = []
        for d, st in zip(descs, streams):
            st.wait_event(g0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            aeq.pusch_eq_fused([d], tuned, st)
            e1.record(st)
            ev.append((e0, e1))
        torch.cuda.synchronize()
        for c, (e0, e1) in enumerate(ev):
            per_cell[c].append(1e3 * e0.elapsed_time(e1))
        span.append(max(1e3 * g0.elapsed_time(e1) for _, e1 in ev))
    batched = []
    for r in range(reps):
        if flush is not None:
            flush.fill_(float(r))
        torch.cuda._sleep(2_000_000)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        aeq.pusch_eq_fused(descs, tuned, main)
        e1.record(main)
        torch.cuda.synchronize()
        batched.append(1e3 * e0.elapsed_time(e1))
    lat = [med(v) for v in per_cell]
    return {"cells": n, "alone_us_mean": sum(alone) / n,
            "streams_per_cell_latency_us_mean": sum(lat) / n,
            "streams_mean_degradation_vs_alone": sum(l / al for l, al in zip(lat, alone)) / n,
            "streams_makespan_us": med(span), "batched_launch_us": med(batched),
            "makespan_ratio_streams_over_batched": med(span) / med(batched)}


def prb_range_desc(aeq, cell, llr, prb0, nprb):
    """Subcarriers [12 prb0, 12 (prb0 + nprb)) of a device cell as a cell of
    its own: the same buffers at an offset (H[nSC][A][L], Y_rx[nSC][nSym][A],
    LLRs per subcarrier in the Y_eq order)."""
    sc0 = 12 * prb0
    return aeq.cell_desc(cell.H[sc0:], cell.Y[sc0:], llr[sc0 * (cell.llr_numel // cell.nSC):], cell.sigma2, nprb,
                         cell.nAnt, cell.nLayers, cell.nSym, cell.nPamBits)


def sm_partition_strategies(aeq, wl, tuned, dev, max_cells=8, reps=20):
    """The reference's SM-partitioning study (src/adaptive_smpartition.cu:165-436)
    restated with the fused launch, on cells of the 100 MHz shape (132 PRB x 64
    antennas x 8 layers x 11 symbols, 256-QAM), for N = 1..8 cells:
      A  one launch per cell on N concurrent streams;
      B  the N launches back to back on one stream;
      C  as A, even cells on a high-priority stream, odd cells on a low one;
      D  ONE cell's PRB range split into N chunks, one launch per chunk on N
         streams (the same total work as one cell);
      E  launches two at a time on two streams, each pair after the previous;
      F  all N cells in one persistent batched launch (this library's method).
    Per-cell latency is event-timed on each cell's stream; the makespan runs
    from a start event that every stream waits on to the last cell's end, with
    every launch enqueued before the start fires.  L2
    is flushed before every repetition (the N cells of 19.9 MB each fit in
    L2 otherwise).  Medians over `reps` repetitions; degradation is the per-cell
    latency over the cell alone."""
    import torch

    cells = [wl.config_cell(2, seed=300 + i, device=dev) for i in range(max_cells)]
    llrs = [torch.empty(c.llr_numel, dtype=torch.float32, device=dev) for c in cells]
    descs = [aeq.cell_desc(c.H, c.Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
             for c, l in zip(cells, llrs)]
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    main = torch.cuda.current_stream()
    plain = [torch.cuda.Stream() for _ in range(max_cells)]
    lo_p, hi_p = torch.cuda.Stream.priority_range()
    prio = [torch.cuda.Stream(priority=hi_p if i % 2 == 0 else lo_p) for i in range(max_cells)]

    def med(v):
        v = sorted(v)
        return v[len(v) // 2]

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def run(plan):
        """plan: list of (stream, [descs], after) launches; `after` = indices of
        the launches whose ends this one waits for, or None for the start event.
        Returns per-launch latencies and the makespan over `reps` repetitions."""
        lat, span = [[] for _ in plan], []
        for r in range(reps + 3):
            flush.fill_(float(r))
            # ~1 ms of device sleep ahead of the start event: every launch is
            # enqueued before the start fires, so no interval holds host-side
            # call overhead
            torch.cuda._sleep(2_000_000)
            g0 = ev()
            g0.record(main)
            ends = []
            for k, (st, ds, after) in enumerate(plan):
                for w in ([g0] if after is None else [ends[j][1] for j in after]):
                    st.wait_event(w)
                e0, e1 = ev(), ev()
                e0.record(st)
                aeq.pusch_eq_fused(ds, tuned, st)
                e1.record(st)
                ends.append((e0, e1))
            for st, _, _ in plan:
                main.wait_stream(st)
            torch.cuda.synchronize()
            if r < 3:
                continue
            for k, (e0, e1) in enumerate(ends):
                lat[k].append(1e3 * e0.elapsed_time(e1))
            span.append(max(1e3 * g0.elapsed_time(e1) for _, e1 in ends))
        return [med(v) for v in lat], med(span)

    iso, _ = run([(plain[0], [descs[0]], None)])
    iso = iso[0]
    out = {"cell": "132 PRB x 64 antennas x 8 layers x 11 symbols, 256-QAM, complex64 in, float32 LLRs",
           "alone_us": iso, "reps": reps, "l2": "flushed before every repetition",
           "strategies": {}}
    rows = {k: [] for k in "ABCDEF"}
    for n in range(1, max_cells + 1):
        def row(lat, span):
            pc = sum(lat) / len(lat)
            return {"n": n, "per_cell_us": pc, "makespan_us": span, "degradation": pc / iso,
                    "cells_per_s": n / (span * 1e-6)}
        lat, span = run([(plain[i], [descs[i]], None) for i in range(n)])
        rows["A"].append(row(lat, span))
        lat, span = run([(plain[0], [descs[i]], None if i == 0 else [i - 1]) for i in range(n)])
        rows["B"].append(row(lat, span))
        lat, span = run([(prio[i], [descs[i]], None) for i in range(n)])
        r = row(lat, span)
        r["high_priority_us"] = sum(lat[0::2]) / len(lat[0::2])
        r["low_priority_us"] = sum(lat[1::2]) / len(lat[1::2]) if n > 1 else None
        rows["C"].append(r)
        per = -(-cells[0].nPRB // n)
        chunks = [(p0, min(per, cells[0].nPRB - p0)) for p0 in range(0, cells[0].nPRB, per)]
        lat, span = run([(plain[i], [prb_range_desc(aeq, cells[0], llrs[0], p0, m)], None)
                         for i, (p0, m) in enumerate(chunks)])
        rows["D"].append({"n": n, "chunks": len(chunks), "per_chunk_us": sum(lat) / len(lat),
                          "makespan_us": span, "speedup_vs_alone": iso / span})
        if n >= 2:
            plan = [(plain[i % 2], [descs[i]], None if i < 2 else [2 * (i // 2) - 2, 2 * (i // 2) - 1])
                    for i in range(n)]
            lat, span = run(plan)
            rows["E"].append(row(lat, span))
        lat, span = run([(main, descs[:n], None)])   # every cell's results land at the launch's end
        rows["F"].append(row(lat * n, span))
    names = {"A": "unrestricted concurrent streams", "B": "serial on one stream",
             "C": "stream priority, alternating high/low", "D": "one cell split by PRB range over N streams",
             "E": "pairs of streams, serial between pairs", "F": "one persistent batched launch"}
    for k in "ABCDEF":
        out["strategies"][k] = {"name": names[k], "rows": rows[k]}
    del flush
    return out


def bench_extras(aeq, wl, cells, llrs, descs, tun, stream, a):
    """Plain FP32 chain on the same slots, single-slot latency, the SRS filter multiply."""
    import numpy as np
    import torch

    out = {}
    # plain FP32 chain on the same S slots (stage-by-stage, the reference's method)
    ws = torch.empty(aeq.pusch_eq_plain_workspace(descs), dtype=torch.uint8, device=llrs[0].device)
    for _ in range(2):
        aeq.pusch_eq_plain(descs, ws, stream)
    torch.cuda.synchronize()
    k = 10
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(k):
        aeq.pusch_eq_plain(descs, ws, stream)
    s1.record(stream)
    torch.cuda.synchronize()
    plain = sum(c.n_re for c in cells) * k / (s0.elapsed_time(s1) / 1e3)
    out["plain_fp32_chain"] = {"value": plain, "unit": UNIT, "kernels_per_cell": 4}
    # single-slot latency (one cell per launch), L2 flushed between launches
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=llrs[0].device)
    lat = []
    for i in range(60):
        flush.fill_(float(i))
        s0.record(stream)
        aeq.pusch_eq_fused([descs[i % len(descs)]], tun, stream)
        s1.record(stream)
        torch.cuda.synchronize()
        if i >= 10:
            lat.append(s0.elapsed_time(s1) * 1e3)
    lat.sort()
    out["single_slot_latency_us"] = {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                                     "note": f"one {cells[0].nSC}-SC cell per launch, L2 flushed before each"}
    out["srs_filter"] = bench_srs(aeq, llrs[0].device, stream)
    out["chest_interp"] = bench_chest(aeq, llrs[0].device, stream)
    return out


def accuracy_vs_fp64(orc, aeq, cells, llrs, descs, tun, stream):
    """Checker: slot 0 against the FP64 model of the oracle, through the fused
    launch at the bench's operand precision (the top-level keys), and under
    `by_path` at every operand precision and through the plain FP32 chain
    (the reference's method), so the precisions compare at the same EVM.
    `hard_bit_mismatch` counts every sign flip against FP64, unmasked;
    `flip_max_abs_llr64_rel` is the largest |LLR64| at a flip over max |LLR64|."""
    import numpy as np
    import torch

    c = cells[0]
    y64, _, l64 = orc.chain_f64(c.H.cpu().numpy(), c.Y.cpu().numpy(), c.sigma2, c.nSC, c.nAnt, c.nLayers, c.nSym,
                                c.nPamBits)
    bits = c.bits.cpu().numpy().reshape(-1)

    def run(fn):
        llr = torch.empty(c.llr_numel, dtype=torch.float32, device=c.H.device)
        yeq = torch.empty(c.nSC * c.nLayers * c.nSym, dtype=torch.complex64, device=c.H.device)
        d = aeq.cell_desc(c.H, c.Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=yeq)
        fn(d)
        torch.cuda.synchronize()
        y = yeq.cpu().numpy().astype(np.complex128)
        l = llr.cpu().numpy().astype(np.float64)
        flips = (l < 0) != (l64 < 0)
        scale = float(np.abs(l64).max())
        return {"evm_db": float(10 * np.log10(np.sum(np.abs(y - y64) ** 2) / np.sum(np.abs(y64) ** 2))),
                "llr_max_abs_err": float(np.abs(l - l64).max()), "llr_scale": scale,
                "hard_bit_mismatch": int(np.sum(flips)), "bits": int(l.size),
                "flip_max_abs_llr64_rel": float(np.abs(l64[flips]).max() / scale) if flips.any() else 0.0,
                "ber_vs_tx": float(np.mean((l < 0).astype(np.uint8) != bits))}

    out = run(lambda d: aeq.pusch_eq_fused([d], tun, stream))
    by = {}
    for name in ("fp16", "bf16", "bf16x3", "fp16x3"):
        by["fused_" + name] = run(lambda d: aeq.pusch_eq_fused([d], aeq.make_tuning(name), stream))
    ws = torch.empty(aeq.pusch_eq_plain_workspace(descs[:1]), dtype=torch.uint8, device=c.H.device)
    by["plain_fp32_chain"] = run(lambda d: aeq.pusch_eq_plain([d], ws, stream))
    out["by_path"] = by
    return out


def path_rates(aeq, descs, res_per_step, bytes_per_step, stream, k=20):
    """The headline step (same slots, same launch) at each operand precision:
    mean launch time, REs/s and HBM fraction, so the accuracy of each path in
    `accuracy_vs_fp64.by_path` sits next to its cost."""
    peak, _ = measured_peaks()
    out = {}
    for name in ("fp16", "bf16", "bf16x3", "fp16x3"):
        t = aeq.make_tuning(name)
        us = _time_launches(lambda: aeq.pusch_eq_fused(descs, t, stream), stream, k)
        out["fused_" + name] = {"us_per_launch": us, "res_per_s": res_per_step / (us * 1e-6),
                                "hbm_frac": bytes_per_step / (us * 1e-6) / 1e9 / peak}
    return out


def _timed_flushed(fn, stream, flush, k=20):
    """Mean of k event-timed launches, L2 flushed before each (inputs near or
    below the L2 size)."""
    import torch

    for _ in range(3):
        fn()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
    for i in range(k):
        if flush is not None:
            flush.fill_(float(i))
        ev[i][0].record(stream)
        fn()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    return 1e3 * statistics.mean(x.elapsed_time(y) for x, y in ev)


def other_configs(aeq, wl, dev, stream, a):
    """Configurations 3, 4 and 5 in compact form for the default line, each a
    few seconds: the 12-slot precision-stress launch per operand precision;
    the uneven 16-cell batch as a CUDA graph replay, autotuned against the
    fixed default shape; and one second of the serving loop."""
    import torch

    peak, _ = measured_peaks()
    out = {}
    # configuration 3: 12 slots of 273 PRB x 128 antennas x 16 layers (1.3 GB: larger than L2)
    cells = build_cells(wl, 3, 12, 0, dev)
    llrs = [torch.empty(c.llr_numel, dtype=torch.float32, device=dev) for c in cells]
    descs = [aeq.cell_desc(c.H, c.Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
             for c, l in zip(cells, llrs)]
    res = sum(c.n_re for c in cells)
    nbytes = sum(c.algorithmic_bytes() for c in cells)
    c3 = {"workload": WORKLOADS[3], "slots": len(cells)}
    for name in ("bf16x3", "fp16x3", "fp16"):
        t = aeq.make_tuning(name)
        us = _time_launches(lambda: aeq.pusch_eq_fused(descs, t, stream), stream, 10)
        c3[name] = {"us_per_launch": us, "res_per_s": res / (us * 1e-6),
                    "hbm_frac": nbytes / (us * 1e-6) / 1e9 / peak}
    out["config3"] = c3
    del cells, llrs, descs
    torch.cuda.empty_cache()
    # configuration 4: the uneven 16-cell batch, one persistent launch replayed as a CUDA graph
    cells = build_cells(wl, 4, 16, 0, dev)
    llrs = [torch.empty(c.llr_numel, dtype=torch.float32, device=dev) for c in cells]
    descs = [aeq.cell_desc(c.H, c.Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
             for c, l in zip(cells, llrs)]
    res = sum(c.n_re for c in cells)
    nbytes = sum(c.algorithmic_bytes() for c in cells)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    tuned, _ = aeq.autotune(descs, "fp16")
    fixed = aeq.make_tuning("fp16")
    g = aeq.FusedGraph(descs, tuned)
    try:
        us = _timed_flushed(lambda: g.launch(stream), stream, flush)
    finally:
        g.close()
    out["config4"] = {
        "workload": WORKLOADS[4], "launch": "CUDA graph replay of the persistent launch, L2 flushed before each",
        "us_per_launch": us, "res_per_s": res / (us * 1e-6), "hbm_frac": nbytes / (us * 1e-6) / 1e9 / peak,
        "autotuned_us": _timed_flushed(lambda: aeq.pusch_eq_fused(descs, tuned, stream), stream, flush),
        "fixed_default_us": _timed_flushed(lambda: aeq.pusch_eq_fused(descs, fixed, stream), stream, flush),
        "autotuned": {"warps_per_cta": tuned.warps_per_cta, "ctas_per_sm": tuned.ctas_per_sm,
                      "sc_per_group": tuned.sc_per_group}}
    del cells, llrs, descs, flush
    torch.cuda.empty_cache()
    # configuration 5: one second of the serving loop
    a5 = argparse.Namespace(**vars(a))
    a5.precision = DEFAULT_PRECISION[5]
    out["config5"] = serving_summary(a5, aeq, wl, dev, 1.0, SERVE_STREAMS, SERVE_WINDOW_US, SERVE_MIN_BATCH)
    out["config5"]["duration_s"] = 1.0
    return out


def reference_stages_on_b200(aeq, dev, med):
    """Single launches at the reference's own shapes (L2-warm, the kernel time
    alone): its coef_apply V1 / V2 / V3 (src/aerial_coef_wmma.cu:400-407),
    gram_scalar (src/aerial_bottleneck.cu:174-179), llr V1 / V3 at 256-QAM
    (src/llr/aerial_llr_v3.cu:292) and SRS filter V1 / V2 (66 blocks, K = 24,
    4 ports, FOCC length 8: src/srs/srs_wmma_bench.cu:347), each beside this
    library's entry point for the same stage."""
    import torch

    reflib = os.path.join(ROOT, "oracle", "_ref")
    VP, CI = ctypes.c_void_p, ctypes.c_int
    lc = ctypes.CDLL(os.path.join(reflib, "libref_coef.so"))
    lg = ctypes.CDLL(os.path.join(reflib, "libref_gram.so"))
    ll = ctypes.CDLL(os.path.join(reflib, "libref_llr_v3.so"))
    ls = ctypes.CDLL(os.path.join(reflib, "libref_srs.so"))
    lc.ref_coef_launch.argtypes = [CI, VP, VP, VP, CI, CI]
    lg.ref_gram_launch.argtypes = [VP, VP, VP, CI]
    ll.ref_llr_v3_launch.argtypes = [CI, VP, VP, VP, CI, CI]
    ls.ref_srs_launch.argtypes = [CI, VP, VP, VP, VP, CI, CI]
    g = torch.Generator(device=dev)
    g.manual_seed(7)

    def crand(*shape):
        return torch.complex(torch.rand(shape, generator=g, device=dev) - 0.5,
                             torch.rand(shape, generator=g, device=dev) - 0.5)

    nSC, S, L, A = 1584, 11, 8, 64
    out = {}
    C, Y = crand(nSC, L, A), crand(nSC, S, A)
    O = torch.empty(nSC, L, S, dtype=torch.complex64, device=dev)
    p = (C.data_ptr(), Y.data_ptr(), O.data_ptr(), nSC, S)
    out["coef_apply"] = {
        "reference_v1_scalar": med(lambda: lc.ref_coef_launch(1, *p)),
        "reference_v2_wmma": med(lambda: lc.ref_coef_launch(2, *p)),
        "reference_v3_wmma": med(lambda: lc.ref_coef_launch(3, *p)),
        "aerial_coef_apply (bit-exact V1)": med(lambda: aeq.coef_apply(C, Y, O, nSC, S, L, A)),
        "aerial_coef_apply_tc (V2 semantics)": med(lambda: aeq.coef_apply_tc(C, Y, O, nSC, S, L, A))}
    H = crand(nSC, A, L)
    M = H.conj().transpose(1, 2).contiguous()
    G = torch.empty(nSC, L, L, dtype=torch.complex64, device=dev)
    out["gram"] = {"reference_gram_scalar": med(lambda: lg.ref_gram_launch(M.data_ptr(), H.data_ptr(), G.data_ptr(),
                                                                           nSC)),
                   "aerial_gram": med(lambda: aeq.gram(H, 0.01, G, nSC, A, L))}
    N, nb = nSC * L * S, 4
    soft = ((torch.rand(2 * N, generator=g, device=dev) - 0.5) * 1.4).half()
    ni = torch.rand(N, generator=g, device=dev) * 10 + 1
    lo = torch.empty(N * 2 * nb, dtype=torch.float16, device=dev)
    lp = (soft.data_ptr(), ni.data_ptr(), lo.data_ptr(), N, nb)
    out["llr_256qam"] = {"reference_v1": med(lambda: ll.ref_llr_v3_launch(1, *lp)),
                         "reference_v3": med(lambda: ll.ref_llr_v3_launch(3, *lp)),
                         "aerial_llr (bit-exact V1)": med(lambda: aeq.llr(soft, ni, lo, N, nb))}
    K, P, F, nBlk = 24, 4, 8, 66
    srs = ((torch.rand(nBlk * A * K * 2, generator=g, device=dev) - 0.5) * 1.4).half()
    W = ((torch.rand(K * K * 2, generator=g, device=dev) - 0.5) * 1.4).half()
    fo = ((torch.rand(P * F * 2, generator=g, device=dev) - 0.5) * 1.4).half()
    he = torch.empty(nBlk * A * K * P * 2, dtype=torch.float16, device=dev)
    sp = (he.data_ptr(), srs.data_ptr(), W.data_ptr(), fo.data_ptr(), A, nBlk)
    out["srs_filter"] = {"reference_v1_scalar": med(lambda: ls.ref_srs_launch(1, *sp)),
                         "reference_v2_wmma": med(lambda: ls.ref_srs_launch(2, *sp)),
                         "aerial_srs_filter": med(lambda: aeq.srs_filter(he, srs, W, fo, A, nBlk, K, P, F))}
    return out


def reference_kernels_on_b200(aeq, wl, dev, slots=64):
    """Baseline: the reference's own kernels, compiled unchanged from its
    sources into the checker libraries (oracle/_ref), on this GPU over the
    headline step's 64 cell-slots: gram_scalar -> coef_apply_v2_wmma -> llr_v3
    (three launches, no MMSE solve: the reference has none), against one fused
    launch of this library with the solve.  The reference's C and the LLR
    input are random (its benchmarks do not chain data).  Median of 20
    event-timed repetitions after 3 warm-ups; 1.3 GB of inputs (larger than
    L2).  Shapes: src/aerial_bottleneck.cu:174-179, src/aerial_coef_wmma.cu:400-404,
    src/llr/aerial_llr_v3.cu:292."""
    import torch

    reflib = os.path.join(ROOT, "oracle", "_ref")
    need = [os.path.join(reflib, f"libref_{n}.so") for n in ("gram", "coef", "llr_v3")]
    if not all(os.path.exists(x) for x in need):
        return {"unavailable": "oracle/_ref not built (make -C oracle ref needs the reference sources)"}
    VP, CI = ctypes.c_void_p, ctypes.c_int
    lg, lc, ll = (ctypes.CDLL(x) for x in need)
    lg.ref_gram_launch.argtypes = [VP, VP, VP, CI]
    lc.ref_coef_launch.argtypes = [CI, VP, VP, VP, CI, CI]
    ll.ref_llr_v3_launch.argtypes = [CI, VP, VP, VP, CI, CI]
    nSC1, S, L, A, nb = 1584, 11, 8, 64, 4
    cells = [wl.config_cell(2, seed=17 * i + 1, device=dev) for i in range(slots)]
    nS = nSC1 * slots
    Hs = torch.cat([x.H for x in cells])
    Ys = torch.cat([x.Y for x in cells])
    Ms = Hs.conj().transpose(1, 2).contiguous()
    Gs = torch.empty(nS, L, L, dtype=torch.complex64, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    Cs = torch.complex(torch.rand((nS, L, A), generator=g, device=dev) - 0.5,
                       torch.rand((nS, L, A), generator=g, device=dev) - 0.5)
    Os = torch.empty(nS, L, S, dtype=torch.complex64, device=dev)
    Ns = nS * L * S
    soft = ((torch.rand(2 * Ns, generator=g, device=dev) - 0.5) * 1.4).half()
    ni = torch.rand(Ns, generator=g, device=dev) * 10 + 1
    lo = torch.empty(Ns * 2 * nb, dtype=torch.float16, device=dev)
    llrs = [torch.empty(x.llr_numel, dtype=torch.float32, device=dev) for x in cells]
    descs = [aeq.cell_desc(x.H, x.Y, l, x.sigma2, x.nPRB, x.nAnt, x.nLayers, x.nSym, x.nPamBits)
             for x, l in zip(cells, llrs)]
    tun = aeq.make_tuning("fp16")
    stream = torch.cuda.current_stream()    # the checker libraries launch on the default stream

    def ref_chain():
        lg.ref_gram_launch(Ms.data_ptr(), Hs.data_ptr(), Gs.data_ptr(), nS)
        lc.ref_coef_launch(2, Cs.data_ptr(), Ys.data_ptr(), Os.data_ptr(), nS, S)
        ll.ref_llr_v3_launch(3, soft.data_ptr(), ni.data_ptr(), lo.data_ptr(), Ns, nb)

    def med(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        t = []
        for _ in range(20):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda._sleep(200000)     # the GPU stays busy while the host enqueues
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            t.append(1e3 * e0.elapsed_time(e1))
        return statistics.median(t)

    t_ref = med(ref_chain)
    t_fused = med(lambda: aeq.pusch_eq_fused(descs, tun, stream))
    stages = reference_stages_on_b200(aeq, dev, med)
    return {"per_stage_us": stages, "slots": slots, "subcarriers": nS,
            "reference_gram_coefv2_llrv3_us": t_ref, "reference_res_per_s": nS * S / (t_ref * 1e-6),
            "fused_us": t_fused, "fused_res_per_s": nS * S / (t_fused * 1e-6), "speedup": t_ref / t_fused,
            "note": "reference: three unfused launches without a solve, from oracle/_ref; fused: Gram + MMSE "
                    "solve + apply + LLR in one launch"}


def _time_launches(fn, stream, k=50):
    import torch

    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e3 / k


def write_fill_gbs(buf, stream):
    """Write-only HBM rate on this GPU: torch's fill of `buf`'s bytes as 4-byte
    words (no reads; torch's FP16 fill is slower than its 4-byte fill), GB/s.
    Context for the filter kernels, whose traffic is 80-89 % writes."""
    import torch

    words = (torch.view_as_real(buf) if buf.is_complex() else buf).reshape(-1).view(torch.int32)
    return words.numel() * 4 / (_time_launches(lambda: words.fill_(0), stream) * 1e-6) / 1e9


def bench_chest(aeq, dev, stream):
    """DMRS frequency-interpolation filter: the [64 x 96] x [96 x 4] product per output subcarrier named by the
    reference (README.md:200) -- 64 antennas, 96 pilot REs and 96 output subcarriers per 8-PRB block, 4 ports,
    OCC length 2 -- over 34 blocks (272 PRB) x 40 cells x 2 DMRS symbols = 2,720 blocks per launch, written as
    the complex64 PUSCH channel (602 MB touched: larger than L2)."""
    import torch

    nPilot, nOut, P, F, nAnt = 96, 96, 4, 2, 64
    nBlk = 34 * 40 * 2
    g = torch.Generator(device=dev)
    g.manual_seed(9)
    yp = ((torch.rand(nBlk * nAnt * nPilot * 2, generator=g, device=dev) - 0.5) * 1.4).half()
    wf = ((torch.rand(nOut * nPilot * 2, generator=g, device=dev) - 0.5) * 0.1).half()
    occ = ((torch.rand(P * F * 2, generator=g, device=dev) - 0.5) * 1.4).half()
    H = torch.empty(nBlk * nOut * nAnt * P, dtype=torch.complex64, device=dev)
    us = _time_launches(lambda: aeq.chest_interp(H, yp, wf, occ, nAnt, nBlk, nPilot, nOut, P, F, stream), stream)
    nbytes = 2 * (yp.numel() + wf.numel() + occ.numel()) + 8 * H.numel()
    flops = 8.0 * nBlk * nAnt * nPilot * nOut * P
    peak, kind = measured_peaks()
    gbs = nbytes / (us * 1e-6) / 1e9
    # the same filter writing the channel as complex half (the H of an FP16 I/O cell)
    H16 = torch.empty(H.numel(), 2, dtype=torch.float16, device=dev)
    us16 = _time_launches(lambda: aeq.chest_interp_h(H16, yp, wf, occ, nAnt, nBlk, nPilot, nOut, P, F, stream), stream)
    nbytes16 = 2 * (yp.numel() + wf.numel() + occ.numel()) + 4 * H.numel()
    fp16 = {"us_per_launch": us16, "bytes_per_launch": nbytes16, "achieved_gbs": nbytes16 / (us16 * 1e-6) / 1e9,
            "hbm_frac": nbytes16 / (us16 * 1e-6) / 1e9 / peak}
    return {"us_per_launch": us, "blocks_per_launch": nBlk, "bytes_per_launch": nbytes,
            "achieved_gbs": gbs, "hbm_frac": gbs / peak, "peak_gbs": peak, "peak_kind": kind,
            "write_share": 8 * H.numel() / nbytes, "write_fill_gbs": write_fill_gbs(H, stream),
            "fp16_channel": fp16,
            "gflops": flops / (us * 1e-6) / 1e9, "tensor_gflops": 2 * flops / (us * 1e-6) / 1e9,
            "shape": f"{nBlk} blocks x {nAnt} antennas, {nPilot} pilots -> {nOut} subcarriers x {P} ports, "
                     f"OCC length {F}; FP16 in, complex64 channel out; tensor cores (FP16 operands, taps split "
                     "hi/lo), FP32 accumulate"}


def srs_cpu_rate(orc, seconds: float):
    """The reference's srs_filter_v1_scalar (FP16 arithmetic) restated in C, on the host cores: SRS blocks/s on
    the reference's own launch (66 blocks x 64 antennas, K = 24, 4 ports, FOCC length 8), repeated."""
    K, P, F, nBlk, nAnt = 24, 4, 8, 66, 64
    s, w, f = orc.ref_srs_inputs(42, nBlk * nAnt * K, K * K, P * F)
    orc.srs_v1_f16(s, w, f, nAnt, nBlk, K, P, F)
    t0 = time.perf_counter()
    runs = 0
    while True:
        orc.srs_v1_f16(s, w, f, nAnt, nBlk, K, P, F)
        runs += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return runs * nBlk / el, runs, el


def bench_srs(aeq, dev, stream):
    """SRS filter multiply (srsFilterMultiply, src/srs/srs_wmma_bench.cu:57-90) at the reference's shape -- 66
    blocks x 64 antennas, K = 24 taps, 4 ports, FOCC length 8 -- for 40 cells x 4 SRS symbols per launch
    (10,560 blocks, 324 MB touched: larger than L2).  Algorithmic bytes: SRS in + W + FOCC + H_est out (FP16)."""
    import torch

    K, P, F, nAnt = 24, 4, 8, 64
    nBlk = 66 * 40 * 4
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    srs = ((torch.rand(nBlk * nAnt * K * 2, generator=g, device=dev) - 0.5) * 1.4).half()
    W = ((torch.rand(K * K * 2, generator=g, device=dev) - 0.5) * 1.4).half()
    focc = ((torch.rand(P * F * 2, generator=g, device=dev) - 0.5) * 1.4).half()
    out = torch.empty(nBlk * nAnt * K * P * 2, dtype=torch.float16, device=dev)
    us = _time_launches(lambda: aeq.srs_filter(out, srs, W, focc, nAnt, nBlk, K, P, F, stream), stream)
    nbytes = 2 * (srs.numel() + W.numel() + focc.numel() + out.numel())
    flops = 8.0 * nBlk * nAnt * K * P * K
    peak, kind = measured_peaks()
    gbs = nbytes / (us * 1e-6) / 1e9
    return {"us_per_launch": us, "blocks_per_launch": nBlk, "blocks_per_s": nBlk / (us * 1e-6),
            "bytes_per_launch": nbytes,
            "achieved_gbs": gbs, "hbm_frac": gbs / peak, "peak_gbs": peak, "peak_kind": kind,
            "write_share": 2 * out.numel() / nbytes, "write_fill_gbs": write_fill_gbs(out, stream),
            "gflops": flops / (us * 1e-6) / 1e9,
            "shape": f"{nBlk} blocks x {nAnt} antennas, K={K}, P={P}, FOCC length {F}, FP16 in/out, "
                     "tensor cores (FP16 operands, taps split hi/lo), FP32 accumulate"}


if __name__ == "__main__":
    main()
