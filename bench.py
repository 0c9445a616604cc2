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

    def _sample(self):
        try:
            out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                  "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
            line = out.stdout.strip().splitlines()[0] if out.stdout.strip() else ""
            if line:
                self.samples.append([x.strip() for x in line.split(",")])
        except Exception:
            pass

    def _run(self):
        while not self._stop.is_set():
            self._sample()
            self._stop.wait(0.1)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        # one more sample right at the end of the region (a region of a few
        # milliseconds is shorter than one nvidia-smi query)
        self._sample()

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


def max_over_ranks(values, device):
    """Element-wise max of per-rank timings over the process group (the job's
    time is its slowest rank's)."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def whole_job_value(work_per_rank, world, ms):
    """Whole-job throughput: every rank processes its own batch (weak scaling),
    so the job does world x the per-rank work in the slowest rank's time."""
    return work_per_rank * world / (ms * 1e-3)


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

    # each job alone (one launch), same flush discipline: the per-family cost
    per_family = {}
    with torch.cuda.stream(stream):
        for (name, *_), j in zip(workloads.PASS13, jobs):
            ts = []
            for i in range(max(1, args.warmup) + args.steps):
                flush.fill_(i & 0xff)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                tb.fused_batch_d(series, [j], stream.cuda_stream)
                b.record(stream)
                b.synchronize()
                if i >= max(1, args.warmup):
                    ts.append(a.elapsed_time(b))
            per_family[name] = statistics.median(ts) * 1e3

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

    # the autotuner on this shape: every candidate launch shape timed, the
    # fastest kept (the timed steps above use the heuristic plan; tuning last,
    # since the tuned plan then serves this shape in the whole process)
    plan = tb.Plan(jobs, S, T)
    heuristic = plan.describe()
    plan.autotune(series, jobs, stream.cuda_stream)
    tuned = {"heuristic": dict(heuristic, engine=tb.Plan.ENGINES.get(heuristic["mode"])),
             "chosen": dict(plan.describe(), engine=tb.Plan.ENGINES.get(plan.describe()["mode"])),
             "candidates": plan.candidates()}
    plan.close()

    stats = {"ms": ms, "plain_ms": plain_ms, "e2e_ms": e2e_ms, "times": times, "per_family_us": per_family,
             "autotune": tuned}
    if world > 1:
        stats["ms"], stats["plain_ms"], stats["e2e_ms"] = max_over_ranks([ms, plain_ms, e2e_ms], dev)
    del g
    return stats, clocks.summary(), h2d, d2h, launches0


def _event_ms(fn, reps, warm=2, stream=None):
    """Median CUDA-event time of fn() on the current stream."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def run_extras(dev, peak):
    """The other measured workloads, each timed with CUDA events (inputs larger
    than L2 where the workload is; the single 100,000-bar series is latency-bound and L2-resident)."""
    import torch
    import tacuda_b200 as tb
    from tacuda_b200 import synthetic, workloads
    from tacuda_b200 import torch_api as TA
    out = {}
    torch.cuda.synchronize()

    # one 100,000-bar close series, SMA20 EMA30 RSI14 MACD12/26/9
    x = torch.from_numpy(synthetic.single_close(100_000, seed=11).astype(np.float32)).to(dev).reshape(1, -1)
    o1 = {n: torch.empty_like(x) for n in ("sma", "ema", "rsi", "macd", "sig", "hist")}
    j1 = [tb.make_job("sma", (20,), (), [o1["sma"].data_ptr()]), tb.make_job("ema", (30,), (), [o1["ema"].data_ptr()]),
          tb.make_job("rsi", (14,), (), [o1["rsi"].data_ptr()]),
          tb.make_job("macd", (12, 26, 9), (), [o1[k].data_ptr() for k in ("macd", "sig", "hist")])]
    s1 = tb.make_series({"close": x.data_ptr()}, 1, x.shape[1])
    st = torch.cuda.current_stream().cuda_stream
    # the synchronous call (stream 0: returns when done, as the reference's
    # stream-0 calls do), then the same launch replayed from a CUDA graph on a
    # user stream (device time, no host work between steps)
    sync_ms = _event_ms(lambda: tb.fused_batch_d(s1, j1, 0), 20)
    p_ms = _event_ms(lambda: [tb.fused_batch_d(s1, [j], 0) for j in j1], 20)
    side = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(side):
        tb.fused_batch_d(s1, j1, side.cuda_stream)
        torch.cuda.synchronize()
        g1 = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g1, stream=side):
            tb.fused_batch_d(s1, j1, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        f_ms = _event_ms(lambda: g1.replay(), 20)
    del g1
    out["single_series_100k"] = {"workload": "1 series x 100,000 bars: SMA20 EMA30 RSI14 MACD12/26/9 (6 outputs)",
                                  "fused_us": f_ms * 1e3, "fused_path": "one fused launch replayed from a CUDA graph",
                                  "sync_call_us": sync_ms * 1e3, "plain_us": p_ms * 1e3,
                                  "plain_path": "four synchronous single-job calls on stream 0",
                                  "value": 4 * 100_000 / (f_ms * 1e-3), "unit": "indicator-bars/s",
                                  "bound": "latency"}
    del x, o1

    # 10,000 ragged series (log-uniform 50..20,000 bars), 13-pass + 61 CDL int32
    lengths = synthetic.ragged_lengths(10_000, 50, 20_000, seed=7)
    planes, off = synthetic.ragged_ohlcv(lengths, seed=4)
    N = int(off[-1])
    dp = {k: torch.from_numpy(v).to(dev) for k, v in planes.items()}
    doff = torch.from_numpy(off).to(dev)
    outs = {n: torch.empty(N, device=dev) for n in workloads.PASS13_OUTPUTS}
    names = tb.cdl_names()
    mask = sum(1 << k for k, n in enumerate(names) if n not in ("bullish_engulfing", "bearish_engulfing"))
    cdl = torch.empty((len(names), N), dtype=torch.int32, device=dev)
    jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    jobs.append(tb.make_job("cdl", (), (), [cdl.data_ptr()], cdl_mask=mask, cdl_stride=N, cdl_int32=True))
    ser = tb.make_series({k: v.data_ptr() for k, v in dp.items()}, len(lengths), 0, doff.data_ptr())
    plan = tb.Plan(jobs, len(lengths), 0, off)
    fused = _event_ms(lambda: plan.execute(ser, jobs, st), 5)
    heuristic = plan.describe()
    plan.autotune(ser, jobs, st)
    tuned_ms = _event_ms(lambda: plan.execute(ser, jobs, st), 5)
    tuned = {"heuristic": dict(heuristic, engine=tb.Plan.ENGINES.get(heuristic["mode"])),
             "chosen": dict(plan.describe(), engine=tb.Plan.ENGINES.get(plan.describe()["mode"])),
             "candidates": plan.candidates(), "tuned_ms": tuned_ms}
    plans = [tb.Plan([j], len(lengths), 0, off) for j in jobs]
    plain = _event_ms(lambda: [pl.execute(ser, [j], st) for pl, j in zip(plans, jobs)], 3)
    ncdl = bin(mask).count("1")
    bytes3 = N * (20 + 4 * len(workloads.PASS13_OUTPUTS) + 4 * ncdl)
    gbs = bytes3 / (fused * 1e-3) / 1e9
    out["ragged_10k_13pass_cdl61"] = {
        "workload": f"10,000 ragged series (sum {N} bars), 13-indicator pass + 61 CDL int32, one plan (2 launches)",
        "ms": fused, "plain_ms": plain, "fused_speedup": plain / fused, "autotune": tuned,
        "value": (13 + ncdl) * N / (fused * 1e-3), "unit": "indicator-bars/s",
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                     "algorithmic_bytes_per_launch": bytes3},
        "l2": "inputs and outputs far larger than L2"}
    for pl in plans:
        pl.close()
    plan.close()
    del dp, doff, outs, cdl

    # per-series alpha EMA/MACD/RSI, forward and adjoint, 4096 x 2048
    rng = np.random.default_rng(4)
    c4 = torch.from_numpy(synthetic.ohlcv(4096, 2048, seed=4)["close"]).to(dev)
    a4 = torch.from_numpy(rng.uniform(0.01, 0.5, 4096).astype(np.float32)).to(dev)
    w4 = [torch.from_numpy(rng.standard_normal((4096, 2048)).astype(np.float32)).to(dev) for _ in range(5)]
    ck = TA.alpha_forward(c4, a4)[5]
    fwd = _event_ms(lambda: TA.alpha_forward(c4, a4), 5)
    bwd = _event_ms(lambda: TA.alpha_backward(c4, a4, ck, w4), 5)
    n4 = 4096 * 2048
    out["alpha_adjoint_4096x2048"] = {
        "workload": "4096 series x 2048 bars, EMA14 MACD12/26/9 RSI14 with per-series alpha; adjoint of a "
                    "N(0,1)-weighted sum of the 5 outputs; checkpoints every 256 bars",
        "forward_ms": fwd, "adjoint_ms": bwd, "adjoint_over_forward": bwd / fwd,
        "forward_GBs": n4 * 24 / (fwd * 1e-3) / 1e9, "adjoint_GBs": n4 * 28 / (bwd * 1e-3) / 1e9}
    del c4, a4, w4, ck

    # batch streams: 4096 series, EMA14 and MACD12/26/9 handles, 64 bars per append
    # (host buffers in and out, synchronous, as the reference's append)
    import ctypes as ct
    lib = tb.get_lib()
    Ss, n = 4096, 64
    dd = synthetic.ohlcv(Ss, 16 * n, seed=9)["close"]
    outs_e = np.empty((Ss, n), np.float32)
    outs_m = [np.empty((Ss, n), np.float32) for _ in range(3)]
    he, hm = ct.c_void_p(), ct.c_void_p()
    lib.ct_ema_stream_batch_create(14, Ss, ct.byref(he))
    lib.ct_macd_stream_batch_create(12, 26, 9, Ss, ct.byref(hm))
    chunks = [np.ascontiguousarray(dd[:, i * n:(i + 1) * n]) for i in range(16)]
    P = ct.c_void_p
    for i in range(2):
        lib.ct_ema_stream_batch_append(he, chunks[i].ctypes.data_as(P), n, outs_e.ctypes.data_as(P))
    t0 = time.perf_counter()
    for i in range(2, 16):
        lib.ct_ema_stream_batch_append(he, chunks[i].ctypes.data_as(P), n, outs_e.ctypes.data_as(P))
    ema_ms = (time.perf_counter() - t0) * 1e3 / 14
    for i in range(2):
        lib.ct_macd_stream_batch_append(hm, chunks[i].ctypes.data_as(P), n, *(o.ctypes.data_as(P) for o in outs_m))
    t0 = time.perf_counter()
    for i in range(2, 16):
        lib.ct_macd_stream_batch_append(hm, chunks[i].ctypes.data_as(P), n, *(o.ctypes.data_as(P) for o in outs_m))
    macd_ms = (time.perf_counter() - t0) * 1e3 / 14
    lib.ct_stream_batch_destroy(he)
    lib.ct_stream_batch_destroy(hm)
    out["stream_append_4096x64"] = {
        "workload": "batch streams of 4096 series, 64 bars per append, host buffers, synchronous (host wall clock "
                    "per append, copies included)",
        "ema14_ms_per_append": ema_ms, "macd_ms_per_append": macd_ms,
        "ema14_bars_per_s": Ss * n / (ema_ms * 1e-3), "macd_bars_per_s": Ss * n / (macd_ms * 1e-3)}

    # 4 series x 50,000,000 bars with a +1e4 level, look-back across tiles
    T5 = 50_000_000
    x5 = torch.from_numpy(synthetic.level_walk(4, T5, seed=5)).to(dev)
    y5 = torch.from_numpy(synthetic.level_walk(4, T5, seed=6)).to(dev)
    o5 = {n: torch.empty_like(x5) for n in ("sma", "stddev", "var", "linearreg", "correl", "ema")}
    j5 = [tb.make_job("sma", (200,), (), [o5["sma"].data_ptr()]),
          tb.make_job("stddev", (200,), (1.0,), [o5["stddev"].data_ptr()]),
          tb.make_job("var", (200,), (), [o5["var"].data_ptr()]),
          tb.make_job("linearreg", (200,), (), [o5["linearreg"].data_ptr()]),
          tb.make_job("correl", (30,), (), [o5["correl"].data_ptr()], inputs=("close", "aux")),
          tb.make_job("ema", (500,), (), [o5["ema"].data_ptr()])]
    s5 = tb.make_series({"close": x5.data_ptr(), "aux": y5.data_ptr()}, 4, T5)
    ms5 = _event_ms(lambda: tb.fused_batch_d(s5, j5, st), 3, warm=1)
    bytes5 = 4 * T5 * (8 + 4 * len(o5))
    g5 = bytes5 / (ms5 * 1e-3) / 1e9
    out["long_rows_4x50M"] = {
        "workload": "4 series x 50,000,000 bars (+1e4 level): SMA/STDDEV/VAR/LINEARREG 200, CORREL30, EMA500, "
                    "FP64 carries, decoupled look-back",
        "ms": ms5, "value": 6 * 4 * T5 / (ms5 * 1e-3), "unit": "indicator-bars/s",
        "roofline": {"bound": "hbm", "achieved": g5, "peak": peak, "unit": "GB/s", "frac": g5 / peak,
                     "algorithmic_bytes_per_launch": bytes5}}
    del x5, y5, o5
    torch.cuda.synchronize()
    return out


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


def profile_case(case: str) -> None:
    """Small self-contained workloads for ncu captures of single kernels: each
    runs its launch three times, so a capture can skip the first two.
      pass13       13-indicator fused pass, 4000 x 234 bars (the headline shape)
      pass13_2000  the same pass over 4000 x 2000 bars
      cdl          candle tile kernel, 61 patterns, 4000 x 2000 bars
      alpha        alpha forward + adjoint, 4096 x 2048 bars
      lb5          long-row jobs through look-back, 4 x 2,000,000 bars
      fam:<names>  jobs of the 13-indicator pass alone (comma-separated), 4000 x 234 bars
      single100k   SMA20 EMA30 RSI14 MACD12/26/9 over one 100,000-bar series"""
    import torch
    import tacuda_b200 as tb
    from tacuda_b200 import synthetic, workloads
    if case in ("pass13", "pass13_2000", "cdl") or case.startswith("fam:"):
        S, T = (4000, 2000) if case in ("pass13_2000", "cdl") else (4000, 234)
        d = synthetic.ohlcv(S, T, seed=5)
        dp = {k: torch.from_numpy(v).cuda() for k, v in d.items()}
        ser = tb.make_series({k: v.data_ptr() for k, v in dp.items() if k in tb.PLANE_ID}, S, T)
        if case == "cdl":
            names = tb.cdl_names()
            mask = sum(1 << k for k, n in enumerate(names) if n not in ("bullish_engulfing", "bearish_engulfing"))
            out = torch.empty((len(names), S, T), dtype=torch.int32, device="cuda")
            jobs = [tb.make_job("cdl", (), (), [out.data_ptr()], cdl_mask=mask, cdl_stride=S * T, cdl_int32=True)]
        else:
            outs = {n: torch.empty((S, T), device="cuda") for n in workloads.PASS13_OUTPUTS}
            only = case[4:].split(",") if case.startswith("fam:") else None
            jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on])
                    for name, fam, p, fp, on in workloads.PASS13 if only is None or name in only]
            if not jobs:
                raise SystemExit(f"unknown job {only!r}")
        for _ in range(3):
            tb.fused_batch_d(ser, jobs, 0)
    elif case == "single100k":
        x = torch.from_numpy(synthetic.single_close(100_000, seed=11).astype(np.float32)).cuda().reshape(1, -1)
        o = {n: torch.empty_like(x) for n in ("sma", "ema", "rsi", "macd", "sig", "hist")}
        jobs = [tb.make_job("sma", (20,), (), [o["sma"].data_ptr()]), tb.make_job("ema", (30,), (), [o["ema"].data_ptr()]),
                tb.make_job("rsi", (14,), (), [o["rsi"].data_ptr()]),
                tb.make_job("macd", (12, 26, 9), (), [o[k].data_ptr() for k in ("macd", "sig", "hist")])]
        ser = tb.make_series({"close": x.data_ptr()}, 1, x.shape[1])
        for _ in range(3):
            tb.fused_batch_d(ser, jobs, 0)
    elif case == "alpha":
        from tacuda_b200 import torch_api as TA
        rng = np.random.default_rng(4)
        c = torch.from_numpy(synthetic.ohlcv(4096, 2048, seed=4)["close"]).cuda()
        a = torch.from_numpy(rng.uniform(0.01, 0.5, 4096).astype(np.float32)).cuda()
        w = [torch.from_numpy(rng.standard_normal((4096, 2048)).astype(np.float32)).cuda() for _ in range(5)]
        for _ in range(3):
            ck = TA.alpha_forward(c, a)[5]
            TA.alpha_backward(c, a, ck, w)
    elif case == "lb5":
        S, T = 4, 2_000_000
        x = torch.from_numpy(synthetic.level_walk(S, T, seed=5)).cuda()
        y = torch.from_numpy(synthetic.level_walk(S, T, seed=6)).cuda()
        o = {n: torch.empty_like(x) for n in ("sma", "stddev", "var", "linearreg", "correl", "ema")}
        jobs = [tb.make_job("sma", (200,), (), [o["sma"].data_ptr()]),
                tb.make_job("stddev", (200,), (1.0,), [o["stddev"].data_ptr()]),
                tb.make_job("var", (200,), (), [o["var"].data_ptr()]),
                tb.make_job("linearreg", (200,), (), [o["linearreg"].data_ptr()]),
                tb.make_job("correl", (30,), (), [o["correl"].data_ptr()], inputs=("close", "aux")),
                tb.make_job("ema", (500,), (), [o["ema"].data_ptr()])]
        ser = tb.make_series({"close": x.data_ptr(), "aux": y.data_ptr()}, S, T)
        for _ in range(3):
            tb.fused_batch_d(ser, jobs, 0)
    else:
        raise SystemExit(f"unknown case {case!r}")
    torch.cuda.synchronize()
    print("ok", case)


REF_GPU_FUSED = {  # FusedFamily codes of src/api/BatchFused.h and the planes each call reads
    "sma": (1, "c"), "ema": (2, "c"), "wma": (8, "c"), "rsi": (3, "c"), "macd": (5, "c"), "atr": (4, "hlc"),
    "bbands": (6, "c"), "stoch": (7, "hlc"), "obv": (14, "cv"), "mfi": (15, "hlcv")}
REF_GPU_PLAIN = {"sma": 1, "ema": 2, "wma": 3, "rsi": 4, "atr": 5, "adx": 6, "bbands": 7, "stoch": 8, "cci": 9,
                 "obv": 10, "mfi": 11, "willr": 12}


def reference_gpu_pass13(S, T, steps, warmup):
    """The reference's own GPU kernels for the 13-indicator pass on this GPU,
    built from its sources into oracle/_ref/libtaref_gpu.so: the batch path
    its ct_*_batch_d entries take at this shape (fused row kernels for ten
    families, the short-row ADX kernel, the flat-matrix CCI and WILLR), one
    call after another on one stream; and its per-series path
    (TACUDA_BATCH_FUSED=0: an indicator object's calculate() per series)."""
    import ctypes as ct
    import torch
    from tacuda_b200 import synthetic, workloads
    so = ROOT / "oracle" / "_ref" / "libtaref_gpu.so"
    if not so.exists() or not torch.cuda.is_available():
        return {"unavailable": "oracle/_ref/libtaref_gpu.so not built" if not so.exists() else "no GPU"}
    lib = ct.CDLL(str(so))
    P, I, F = ct.c_void_p, ct.c_int, ct.c_float
    lib.refgpu_fused.argtypes = [I, P, P, P, P, P, P, P, I, I, I, I, I, F, F, P]
    lib.refgpu_adx.argtypes = [P, P, P, P, I, I, I, I, P]
    lib.refgpu_cci.argtypes = [P, P, P, P, I, I, I, P]
    lib.refgpu_willr.argtypes = [P, P, P, P, I, I, I, P]
    has_plain = hasattr(lib, "refgpu_plain")
    if has_plain:
        lib.refgpu_plain.argtypes = [I, P, P, P, P, P, P, P, I, I, I, I, F, F, P]
    d = synthetic.ohlcv(S, T, seed=2024)
    dv = {k: torch.from_numpy(d[k]).cuda() for k in ("high", "low", "close", "volume")}
    pl = {"h": dv["high"].data_ptr(), "l": dv["low"].data_ptr(), "c": dv["close"].data_ptr(),
          "v": dv["volume"].data_ptr()}
    outs = {n: torch.empty((S, T), device="cuda") for n in workloads.PASS13_OUTPUTS}
    st = torch.cuda.Stream()
    sh = ct.c_void_p(st.cuda_stream)
    calls = {}
    for name, fam, p, fp, onames in workloads.PASS13:
        o = [outs[n].data_ptr() for n in onames] + [None] * (3 - len(onames))
        if name in REF_GPU_FUSED:
            code, ins = REF_GPU_FUSED[name]
            a = [pl[k] for k in ins] + [None] * (4 - len(ins))
            pp = tuple(p) + (0, 0, 0)
            if name == "stoch":
                pp = (p[0], p[1], p[1])
            up, dn = (fp[0], fp[1]) if fp else (2.0, 2.0)
            calls[name] = (lambda code=code, a=a, o=o, pp=pp, up=up, dn=dn:
                           lib.refgpu_fused(code, *a, *o, T, S, pp[0], pp[1], pp[2], up, dn, sh))
        elif name == "adx":
            calls[name] = lambda o=o, p=p: lib.refgpu_adx(pl["h"], pl["l"], pl["c"], o[0], T, S, p[0], 0, sh)
        elif name == "cci":
            calls[name] = lambda o=o, p=p: lib.refgpu_cci(pl["h"], pl["l"], pl["c"], o[0], T, S, p[0], sh)
        elif name == "willr":
            calls[name] = lambda o=o, p=p: lib.refgpu_willr(pl["h"], pl["l"], pl["c"], o[0], T, S, p[0], sh)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn, n, w):
        ts = []
        with torch.cuda.stream(st):
            for i in range(w + n):
                flush.fill_(i & 0xff)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(st)
                rc = fn()
                b.record(st)
                b.synchronize()
                if any(x not in (None, 0) for x in (rc if isinstance(rc, list) else [rc])):
                    raise RuntimeError(f"reference GPU call failed: {rc}")
                if i >= w:
                    ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    res = {"shape": f"{S}x{T}", "timing": "CUDA events on one stream, L2 flushed before each step, median",
           "batch_path_us": timed(lambda: [calls[n]() for n, *_ in workloads.PASS13], steps, warmup) * 1e3,
           "batch_path_per_indicator_us": {n: timed(calls[n], steps, warmup) * 1e3 for n, *_ in workloads.PASS13}}
    if has_plain:
        def plain(name):
            fam = REF_GPU_PLAIN[name]
            spec = next(x for x in workloads.PASS13 if x[0] == name)
            p, fp, onames = spec[2], spec[3], spec[4]
            o = [outs[n].data_ptr() for n in onames] + [None] * (3 - len(onames))
            up, dn = (fp[0], fp[1]) if fp else (2.0, 2.0)
            return lambda: lib.refgpu_plain(fam, pl["h"], pl["l"], pl["c"], pl["v"], *o, T, S,
                                            p[0] if p else 0, p[1] if len(p) > 1 else 0, up, dn, sh)
        per = {n: timed(plain(n), 2, 1) for n in REF_GPU_PLAIN}
        res["per_series_path_ms"] = sum(per.values())
        res["per_series_path_per_indicator_ms"] = per
        res["per_series_path_note"] = ("12 of the 13 indicators: MACD's per-series entry runs MACDEXT, whose "
                                       "moving-average and TA-Lib runner sources are not in the bridge")
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--series", type=int, default=S_DEFAULT)
    ap.add_argument("--length", type=int, default=T_DEFAULT)
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="skip the other measured workloads (single long series, ragged + candles, "
                         "alpha adjoint, 4 x 50M bars)")
    ap.add_argument("--case", default=None,
                    help="run one small profiling workload three times and exit (for ncu captures): pass13, "
                         "pass13_2000, cdl, alpha, lb5 or fam:<job of the 13-indicator pass>")
    args = ap.parse_args()
    if args.case:
        profile_case(args.case)
        return
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
        try:
            line["reference_gpu"] = reference_gpu_pass13(args.series, args.length, max(3, min(args.steps, 10)),
                                                         max(1, args.warmup))
        except Exception as e:  # context only: the CPU arm above is the reference measurement
            line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
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
        value = whole_job_value(work_per_step, world, ms)
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
                         "traffic_source": "copied from profiles/pass13_4000x234.json (ncu dram__bytes_read.sum + "
                                           "dram__bytes_write.sum of one launch), not measured by this run",
                         "algorithmic_bytes_per_launch": algo_bytes, "peak_source": peak_kind},
            "cpu_baseline": {"value": cpu_v, "unit": "indicator-bars/s", "cores": threads,
                             "kind": "reference" if O.ref_available() else "port",
                             "sample": f"{cs} of the {args.series} series, all 13 indicators, median of 3"},
            "plain": {"ms_per_step": stats["plain_ms"], "value": work_per_step * world / (stats["plain_ms"] * 1e-3),
                      "launches_per_step": 13, "fused_speedup": stats["plain_ms"] / ms,
                      "per_family_us": stats["per_family_us"]},
            "autotune": stats["autotune"],
            "gpu_launches": args.steps,
            "clocks": clocks,
        }
        if args.extras:
            line["other_workloads"] = run_extras(torch.device("cuda", local), peak)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
