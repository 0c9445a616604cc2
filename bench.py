#!/usr/bin/env python3
"""Benchmark of the fused batched-indicator path on B200.

Workload (one "step"): the 13-indicator pass (SMA20, EMA14, WMA14, RSI14,
MACD 12/26/9, ATR14, ADX14, BBANDS 20/2/2, STOCH 14/3/3, CCI14, OBV, MFI14,
WILLR14 -> 18 float planes) over 4000 series x 234 bars of seeded synthetic
OHLCV, evaluated by ONE fused kernel launch replayed from a CUDA graph.

Metric: indicator-bars/s = 13 * numSeries * seriesLen / step time (whole job:
summed over ranks for N > 1, each rank processing its own 4000-series batch).

Timing: W warm-up steps, then K steps each timed with CUDA events on the
launch stream; before every timed step a 256 MiB buffer is written to flush the
126 MB L2, so every step reads its inputs from HBM. Multi-GPU: one process per
GPU, barrier + device sync around the timed region, max over ranks.

`--impl reference` times the reference's own CPU implementation of the same
pass (vendored TA-Lib 0.8.3 C + StreamStates.h compiled from the reference
tree into oracle/_ref; ADX/CCI/WILLR have no CPU code in the reference and use
the project's FP64 port) on all host threads, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

S_DEFAULT, T_DEFAULT = 4000, 234
METRIC = "indicator-bars/s"
CONFIG = {"workload": "fused 13-indicator pass, uniform batch 4000 series x 234 bars OHLCV float32, one CUDA-graph launch",
          "indicators": "SMA20 EMA14 WMA14 RSI14 MACD12/26/9 ATR14 ADX14 BBANDS20/2/2 STOCH14/3/3 CCI14 OBV MFI14 WILLR14",
          "num_series": S_DEFAULT, "series_len": T_DEFAULT, "l2": "flushed before every timed step (256 MiB write)"}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                line = out.stdout.strip().splitlines()[0] if out.stdout.strip() else ""
                if line:
                    self.samples.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.1)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "pass13_4000x234.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["dram_bytes_per_launch"])
        except Exception:
            return None
    return None


def run_ours(args, rank, world, local):
    import torch
    import tacuda_b200 as tb
    from tacuda_b200 import synthetic, workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    S, T = args.series, args.length
    data = synthetic.ohlcv(S, T, seed=2024 + rank)
    planes = {k: torch.from_numpy(data[k]).to(dev) for k in ("high", "low", "close", "volume")}
    outs = {name: torch.empty((S, T), dtype=torch.float32, device=dev) for name in workloads.PASS13_OUTPUTS}

    def jobs_for(outmap):
        jobs = []
        for _, fam, p, fp, onames in workloads.PASS13:
            jobs.append(tb.make_job(fam, p, fp, [outmap[o].data_ptr() for o in onames]))
        return jobs

    series = tb.make_series({k: v.data_ptr() for k, v in planes.items()}, S, T)
    jobs = jobs_for(outs)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    # plain mode: one launch per indicator (each re-reads its inputs)
    def plain_once(s):
        for j in jobs:
            tb.fused_batch_d(series, [j], s)

    with torch.cuda.stream(stream):
        launches0 = tb.launch_count()
        tb.fused_batch_d(series, jobs, stream.cuda_stream)  # eager warm-up, also first-call setup
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            tb.fused_batch_d(series, jobs, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.fill_(1)
            g.replay()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            for i in range(args.steps):
                flush.fill_(i & 0xff)
                ev[i][0].record(stream)
                g.replay()
                ev[i][1].record(stream)
            torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
    times = [a.elapsed_time(b) for a, b in ev]
    ms = sum(times) / len(times)

    # plain path timing (same flush discipline)
    pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for _ in range(max(1, args.warmup)):
            flush.fill_(2)
            plain_once(stream.cuda_stream)
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.fill_(i & 0xff)
            pev[i][0].record(stream)
            plain_once(stream.cuda_stream)
            pev[i][1].record(stream)
        torch.cuda.synchronize()
    plain_ms = sum(a.elapsed_time(b) for a, b in pev) / args.steps

    # end to end through the host-memory C-ABI call (pinned host buffers)
    hplanes = {k: torch.from_numpy(data[k]).pin_memory() for k in ("high", "low", "close", "volume")}
    houts = {name: torch.empty((S, T), dtype=torch.float32).pin_memory() for name in workloads.PASS13_OUTPUTS}
    hseries = tb.make_series({k: v.data_ptr() for k, v in hplanes.items()}, S, T)
    hjobs = jobs_for(houts)
    with torch.cuda.stream(stream):
        for _ in range(max(1, args.warmup)):
            tb.fused_batch(hseries, hjobs, stream.cuda_stream)
        torch.cuda.synchronize()
        eev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for i in range(args.steps):
            eev[i][0].record(stream)
            tb.fused_batch(hseries, hjobs, stream.cuda_stream)
            eev[i][1].record(stream)
        torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in eev) / args.steps
    h2d = sum(v.numel() * 4 for v in hplanes.values())
    d2h = sum(v.numel() * 4 for v in houts.values())

    # correctness spot check of the timed outputs against the eager host run
    for name in workloads.PASS13_OUTPUTS:
        a, b = outs[name].cpu().numpy(), houts[name].numpy()
        if not np.array_equal(np.isnan(a), np.isnan(b)) or not np.allclose(a, b, equal_nan=True, rtol=0, atol=0):
            raise SystemExit(f"bench: graph replay and host call disagree on {name}")

    stats = {"ms": ms, "plain_ms": plain_ms, "e2e_ms": e2e_ms, "times": times}
    if world > 1:
        t = torch.tensor([ms, plain_ms, e2e_ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        stats["ms"], stats["plain_ms"], stats["e2e_ms"] = (float(x) for x in t.tolist())
    del g
    return stats, clocks.summary(), h2d, d2h, launches0


def cpu_baseline_pass13(S, T, threads, seed=2024):
    """Reference CPU path of the 13-indicator pass on `threads` host threads."""
    from oracle import oracle as O
    from tacuda_b200 import synthetic, workloads

    data = synthetic.ohlcv(S, T, seed=seed)
    t0 = time.perf_counter()
    for _, fam, p, fp, _ in workloads.PASS13:
        kw = workloads.ORACLE_PARAMS[fam](p, fp)
        if fam in O.REF_FAMILIES and O.ref_available():
            O.ref_run(fam, data, threads=threads, **kw)
        else:
            O.run(fam, data, threads=threads, **kw)
    return time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--series", type=int, default=S_DEFAULT)
    ap.add_argument("--length", type=int, default=T_DEFAULT)
    args = ap.parse_args()
    rank, world, local = dist_env()
    n_ind = 13
    work_per_step = n_ind * args.series * args.length  # indicator-bars per rank

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        threads = O.host_threads()
        for _ in range(args.warmup):
            cpu_baseline_pass13(args.series, args.length, threads)
        ts = [cpu_baseline_pass13(args.series, args.length, threads) for _ in range(args.steps)]
        sec = sum(ts) / len(ts)
        v = work_per_step / sec
        kind = "reference" if O.ref_available() else "port"
        sample = (f"full workload per step ({args.series}x{args.length}, 13 indicators); SMA EMA WMA RSI MACD ATR "
                  "BBANDS STOCH via the reference's vendored TA-Lib 0.8.3 C, OBV MFI via its StreamStates.h, "
                  "ADX CCI WILLR via the project's FP64 port (no reference CPU code)")
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "indicator-bars/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(CONFIG, num_series=args.series, series_len=args.length),
                "cpu_baseline": {"value": v, "unit": "indicator-bars/s", "cores": threads, "kind": kind,
                                 "sample": sample},
                "e2e": {"value": v, "unit": "indicator-bars/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stats, clocks, h2d, d2h, _ = run_ours(args, rank, world, local)
    if rank == 0:
        from tacuda_b200 import workloads
        peak, peak_kind = measured_peak()
        ms = stats["ms"]
        value = work_per_step * world / (ms * 1e-3)
        algo_bytes = workloads.PASS13_FUSED_BYTES_PER_BAR * args.series * args.length
        achieved = algo_bytes / (ms * 1e-3) / 1e9
        traffic = committed_traffic()
        # CPU baseline: the reference CPU path on a bounded sample (1000 series)
        from oracle import oracle as O
        threads = O.host_threads()
        cs = min(args.series, 1000)
        cpu_baseline_pass13(cs, args.length, threads)
        csec = statistics.median(cpu_baseline_pass13(cs, args.length, threads) for _ in range(3))
        cpu_v = n_ind * cs * args.length / csec
        line = {
            "metric": METRIC, "value": value, "unit": "indicator-bars/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG, num_series=args.series, series_len=args.length),
            "e2e": {"value": work_per_step * world / (stats["e2e_ms"] * 1e-3), "unit": "indicator-bars/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": stats["e2e_ms"],
                    "path": "ct_b200_fused_batch (host pointers, pinned)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": algo_bytes, "peak_source": peak_kind},
            "cpu_baseline": {"value": cpu_v, "unit": "indicator-bars/s", "cores": threads,
                             "kind": "reference" if O.ref_available() else "port",
                             "sample": f"{cs} of the {args.series} series, all 13 indicators, median of 3"},
            "plain": {"ms_per_step": stats["plain_ms"], "value": work_per_step * world / (stats["plain_ms"] * 1e-3),
                      "launches_per_step": 13, "fused_speedup": stats["plain_ms"] / ms},
            "gpu_launches": args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
