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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--slots", type=int, default=64, help="cell-slots per step (per GPU)")
    ap.add_argument("--precision", default="fp16", choices=["fp16", "bf16", "bf16x3"])
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


def ncu_traffic_per_slot():
    """DRAM bytes per cell-slot of the fused kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("fused_eq_kernel", {}).get("dram_bytes_per_slot")
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
    cell = wl.config_cell(2, seed=42)
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
    sample = f"{nprb} of 132 PRB ({nsc} subcarriers) of one slot per step, OpenMP over subcarriers"
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * el / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "sample": sample},
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

    S = a.slots
    cells = [wl.config_cell(2, seed=1000 * rank + 17 * i + 1, device=dev) for i in range(S)]
    llrs = [torch.empty(c.llr_numel, dtype=torch.float32, device=dev) for c in cells]
    descs = [aeq.cell_desc(c.H, c.Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
             for c, l in zip(cells, llrs)]
    tun = aeq.make_tuning(a.precision)
    if os.environ.get("AERIAL_AUTOTUNE", "1") == "1":
        tun, _ = aeq.autotune(descs, a.precision)
    stream = torch.cuda.current_stream()
    res_per_step = sum(c.n_re for c in cells)
    bytes_per_step = sum(c.algorithmic_bytes() for c in cells)
    in_bytes_per_step = sum(8 * (c.H.numel() + c.Y.numel()) for c in cells)
    out_bytes_per_step = sum(4 * c.llr_numel for c in cells)

    def step():
        aeq.pusch_eq_fused(descs, tun, stream)

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
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier()
    clocks = sampler.stop()
    elapsed_ms = e0.elapsed_time(e1)
    launch_ms = [s.elapsed_time(e) for s, e in ev]
    elapsed_ms, launch_avg_ms = max_over_ranks([elapsed_ms, statistics.mean(launch_ms)], world, dev)
    value = whole_job_rate(res_per_step, a.steps, world, elapsed_ms)
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_step / (launch_avg_ms / 1e3) / 1e9
    tr = ncu_traffic_per_slot()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": (tr * S) if tr else None, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": bytes_per_step}

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not a.no_e2e:
        hH = [c.H.cpu().pin_memory() for c in cells]
        hY = [c.Y.cpu().pin_memory() for c in cells]
        hL = [torch.empty(c.llr_numel, dtype=torch.float32).pin_memory() for c in cells]
        dH = [torch.empty_like(c.H) for c in cells]
        dY = [torch.empty_like(c.Y) for c in cells]
        dL = [torch.empty_like(l) for l in llrs]
        d2 = [aeq.cell_desc(h, y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
              for c, h, y, l in zip(cells, dH, dY, dL)]

        def e2e_step():
            for i in range(S):
                dH[i].copy_(hH[i], non_blocking=True)
                dY[i].copy_(hY[i], non_blocking=True)
            aeq.pusch_eq_fused(d2, tun, stream)
            for i in range(S):
                hL[i].copy_(dL[i], non_blocking=True)

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
               "steps": k2, "path": "pinned host H, Y_rx -> aerial_pusch_eq_fused -> pinned host LLR, one stream"}
        # parity of the end-to-end output against the resident run
        torch.cuda.synchronize()

    extras = {}
    cpu_base = None
    if rank == 0 and world == 1 and not a.no_extras:
        extras = bench_extras(aeq, wl, cells, llrs, descs, tun, stream, a)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        from oracle import oracle as orc

        cores = os.cpu_count() or 1
        orc.set_threads(cores)
        hc = wl.config_cell(2, seed=42)
        v, runs, el = cpu_chain_rate(orc, hc, a.cpu_seconds)
        cpu_base = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                    "sample": f"{runs} full slot(s) (1584 subcarriers) in {el:.1f} s, OpenMP over subcarriers"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": elapsed_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": a.precision + " operands / fp32 accumulate and solve", "data": "synthetic (seeded, generated on device)",
        "config": {"workload": WORKLOAD, "slots_per_step_per_gpu": S, "res_per_step_per_gpu": res_per_step,
                   "l2": f"inputs larger than L2 ({bytes_per_step / 1e6:.0f} MB touched per step per GPU)",
                   "precision": a.precision, "tuning": {"warps_per_cta": tun.warps_per_cta,
                                                         "ctas_per_sm": tun.ctas_per_sm},
                   "parallelism": f"independent cell-slots per GPU x{world}"},
        "roofline": roof,
        "cpu_baseline": cpu_base,
        "e2e": e2e,
        "gpu_launches": a.steps,
        "clocks": clocks,
    }
    line.update(extras)
    print(json.dumps(line), flush=True)


def bench_extras(aeq, wl, cells, llrs, descs, tun, stream, a):
    """Plain FP32 chain on the same slots, single-slot latency, accuracy vs FP64."""
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
                                     "note": "one 1584-SC cell per launch, L2 flushed before each"}
    # accuracy of slot 0 vs the FP64 model
    try:
        from oracle import oracle as orc

        c = cells[0]
        aeq.pusch_eq_fused([descs[0]], tun, stream)
        torch.cuda.synchronize()
        H, Y = c.H.cpu().numpy(), c.Y.cpu().numpy()
        yeq = torch.empty(c.nSC * c.nLayers * c.nSym, dtype=torch.complex64, device=c.H.device)
        d = aeq.cell_desc(c.H, c.Y, llrs[0], c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=yeq)
        aeq.pusch_eq_fused([d], tun, stream)
        torch.cuda.synchronize()
        y64, _, l64 = orc.chain_f64(H, Y, c.sigma2, c.nSC, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
        y = yeq.cpu().numpy().astype(np.complex128)
        l = llrs[0].cpu().numpy().astype(np.float64)
        evm = 10 * np.log10(np.sum(np.abs(y - y64) ** 2) / np.sum(np.abs(y64) ** 2))
        bits = c.bits.cpu().numpy().reshape(-1)
        out["accuracy_vs_fp64"] = {
            "evm_db": float(evm), "llr_max_abs_err": float(np.abs(l - l64).max()),
            "llr_scale": float(np.abs(l64).max()),
            "hard_bit_mismatch": int(np.sum((l < 0) != (l64 < 0))), "bits": int(l.size),
            "ber_vs_tx": float(np.mean((l < 0).astype(np.uint8) != bits)),
        }
    except Exception as e:  # accuracy is reported, never fatal for the timing line
        out["accuracy_vs_fp64"] = {"error": str(e)}
    return out


if __name__ == "__main__":
    main()
