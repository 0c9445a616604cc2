"""Parity at the measured workloads' own shapes, with the error of every output
stated against the FP64 oracle, and the autotuner.

  * 4000 series x 234 bars, the 13-indicator pass (the headline workload),
    on the default plan and on each engine;
  * 1 series x 100,000 bars, SMA20 EMA30 RSI14 MACD12/26/9;
  * 5,000 ragged series of 50..20,000 bars (log-uniform; half the 10,000 rows
    of the measured ragged workload, same length law), the 13-indicator pass;
  * 4 level-offset series of 2,000,000 bars (TACUDA_B200_PRECISION_BARS
    raises it, 50,000,000 for the measured long-row workload) through every
    precision variant.

With TACUDA_B200_ERROR_TABLE=<file>, every comparison appends one JSON line
(workload, output, largest error in units of the tolerance, float32 bit
differences from the oracle rounded to float, values compared, and the
largest relative error where the precision table wants it).
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

import tacuda_b200 as tb
from oracle import oracle as O
from tacuda_b200 import synthetic, workloads
from tolerance import compare, compare_ragged

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def record(workload, output, stats, n, **extra):
    path = os.environ.get("TACUDA_B200_ERROR_TABLE")
    if not path:
        return
    line = {"workload": workload, "output": output, "max_scaled_error": stats[0], "bit_diffs": stats[1],
            "values": int(n)}
    line.update(extra)
    with open(path, "a") as f:
        f.write(json.dumps(line) + "\n")


def pass13_jobs(outs):
    return [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]


def pass13_oracle(planes, offsets=None):
    ref = {}
    for _, fam, p, fp, onames in workloads.PASS13:
        kw = workloads.ORACLE_PARAMS[fam](p, fp)
        res = O.run(fam, planes, offsets=offsets, **kw) if offsets is not None else O.run(fam, planes, **kw)
        for name, r in zip(onames, res):
            ref[name] = r
    return ref


@pytest.fixture(scope="module")
def config2():
    S, T = 4000, 234
    d = synthetic.ohlcv(S, T, seed=2024)
    return S, T, d, pass13_oracle(d)


@pytest.fixture()
def pinned_mode(request):
    old = os.environ.get("TACUDA_B200_MODE")
    if request.param:
        os.environ["TACUDA_B200_MODE"] = request.param
    else:
        os.environ.pop("TACUDA_B200_MODE", None)
    yield request.param or "default"
    if old is None:
        os.environ.pop("TACUDA_B200_MODE", None)
    else:
        os.environ["TACUDA_B200_MODE"] = old


@pytest.mark.parametrize("pinned_mode", [None, "sp", "ws"], indirect=True)
def test_pass13_4000x234_matches_oracle(config2, pinned_mode):
    S, T, d, ref = config2
    dp = {k: torch.from_numpy(v).cuda() for k, v in d.items() if k in tb.PLANE_ID}
    outs = {n: torch.full((S, T), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = pass13_jobs(outs)
    tb.fused_batch_d(tb.make_series({k: v.data_ptr() for k, v in dp.items()}, S, T), jobs, 0)
    torch.cuda.synchronize()
    for name in workloads.PASS13_OUTPUTS:
        g = outs[name].cpu().numpy()
        stats = compare(g, ref[name], f"4000x234 [{pinned_mode}] {name}")
        record(f"4000x234 pass13 [{pinned_mode}]", name, stats, np.count_nonzero(~np.isnan(ref[name])))


def test_single_series_100k_matches_oracle():
    T = 100_000
    x = synthetic.single_close(T, seed=11).astype(np.float32).reshape(1, T)
    dx = torch.from_numpy(x).cuda()
    names = ("sma", "ema", "rsi", "macd", "macd_signal", "macd_hist")
    outs = {n: torch.full((1, T), 777.0, device="cuda") for n in names}
    jobs = [tb.make_job("sma", (20,), (), [outs["sma"].data_ptr()]),
            tb.make_job("ema", (30,), (), [outs["ema"].data_ptr()]),
            tb.make_job("rsi", (14,), (), [outs["rsi"].data_ptr()]),
            tb.make_job("macd", (12, 26, 9), (), [outs[k].data_ptr() for k in names[3:]])]
    tb.fused_batch_d(tb.make_series({"close": dx.data_ptr()}, 1, T), jobs, 0)
    torch.cuda.synchronize()
    d = {"close": x}
    ref = {"sma": O.run("sma", d, period=20)[0], "ema": O.run("ema", d, period=30)[0],
           "rsi": O.run("rsi", d, period=14)[0]}
    ref.update(zip(names[3:], O.run("macd", d, fast=12, slow=26, signal=9)))
    for n in names:
        stats = compare(outs[n].cpu().numpy(), ref[n], f"1x100k {n}")
        record("1x100000 SMA20 EMA30 RSI14 MACD", n, stats, np.count_nonzero(~np.isnan(ref[n])))


def test_ragged_5000_series_matches_oracle():
    lengths = synthetic.ragged_lengths(5000, 50, 20_000, seed=7)
    planes, off = synthetic.ragged_ohlcv(lengths, seed=4)
    N = int(off[-1])
    dp = {k: torch.from_numpy(v).cuda() for k, v in planes.items()}
    doff = torch.from_numpy(off).cuda()
    outs = {n: torch.full((N,), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = pass13_jobs(outs)
    plan = tb.Plan(jobs, len(lengths), 0, off)
    plan.execute(tb.make_series({k: v.data_ptr() for k, v in dp.items()}, len(lengths), 0, doff.data_ptr()), jobs, 0)
    torch.cuda.synchronize()
    engine = tb.Plan.ENGINES.get(plan.describe()["mode"])
    plan.close()
    del dp, doff
    for _, fam, p, fp, onames in workloads.PASS13:
        res = O.run(fam, planes, offsets=off, **workloads.ORACLE_PARAMS[fam](p, fp))
        for name, r in zip(onames, res):
            stats = compare_ragged(outs[name].cpu().numpy(), r, off, f"ragged {name}")
            record(f"5000 ragged rows 50..20000 ({N} bars) pass13 [{engine}]", name, stats,
                   np.count_nonzero(~np.isnan(r)))
        del res


PREC_JOBS = [("sma", (200,), (), dict(period=200)), ("stddev", (200,), (1.0,), dict(period=200, nbdev=1.0)),
             ("var", (200,), (), dict(period=200)), ("linearreg", (200,), (), dict(period=200)),
             ("correl", (30,), (), dict(period=30)), ("ema", (500,), (), dict(period=500))]
# bound on |gpu - ref| / max|ref of the row| per variant; plain FP32 has none
# (its running sums lose the digits the 1e4 level cancels) and is only recorded
PREC_BOUND = {"fp64": 1e-6, "fp32c": 1e-6, "fp32/fp64carry": 1e-5, "fp32": None}


@pytest.mark.parametrize("prec", list(PREC_BOUND))
def test_long_rows_precision_variants(prec):
    S, T = 4, int(os.environ.get("TACUDA_B200_PRECISION_BARS", 2_000_000))
    x = synthetic.level_walk(S, T, seed=5)
    y = synthetic.level_walk(S, T, seed=6)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    outs = {n: torch.full((S, T), 777.0, device="cuda") for n, *_ in PREC_JOBS}
    jobs = [tb.make_job(n, p, fp, [outs[n].data_ptr()], inputs=("close", "aux") if n == "correl" else None,
                        precision=prec) for n, p, fp, _ in PREC_JOBS]
    series = tb.make_series({"close": dx.data_ptr(), "aux": dy.data_ptr()}, S, T)
    tb.fused_batch_d(series, jobs, 0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    tb.fused_batch_d(series, jobs, 0)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    d = {"close": x, "x": x, "y": y}
    for n, _, _, kw in PREC_JOBS:
        ref = O.run(n, d, **kw)[0]
        g = outs[n].cpu().numpy().astype(np.float64)
        np.testing.assert_array_equal(np.isnan(g), np.isnan(ref), err_msg=f"{prec} {n} NaN mask")
        m = ~np.isnan(ref)
        scale = np.nanmax(np.abs(ref), axis=1, keepdims=True)
        err = np.where(m, np.abs(g - ref), 0.0)
        scaled = float(np.max(err / scale))
        big = m & (np.abs(ref) > 1e-12 * scale)
        rel = float(np.max(err[big] / np.abs(ref[big]))) if big.any() else 0.0
        bits = int(np.count_nonzero(g[m].astype(np.float32).view(np.uint32) !=
                                    ref[m].astype(np.float32).view(np.uint32)))
        record(f"4x{T} level walk [{prec}]", n, (scaled, bits), np.count_nonzero(m), max_rel=rel, launch_ms=ms)
        if PREC_BOUND[prec] is not None:
            assert scaled <= PREC_BOUND[prec], f"{prec} {n}: {scaled}"
        del ref, g, err


def _check_autotuned(plan):
    cands = plan.candidates()
    assert len(cands) >= 2 and all(c["ms"] > 0 for c in cands)
    best = min(cands, key=lambda c: c["ms"])
    chosen = plan.describe()
    assert tb.Plan.ENGINES[chosen["mode"]] == best["engine"]
    if best["engine"] != "row-parallel":
        assert (chosen["bars_per_lane"], chosen["warps_per_block"]) == (best["bars_per_lane"],
                                                                         best["warps_per_block"])
    else:
        assert (chosen["parts"], chosen["groups"]) == (best["parts"], best["groups"])
    return cands


def test_autotune_4000x234_picks_fastest_and_matches_oracle(config2):
    S, T, d, ref = config2
    dp = {k: torch.from_numpy(v).cuda() for k, v in d.items() if k in tb.PLANE_ID}
    outs = {n: torch.full((S, T), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = pass13_jobs(outs)
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items()}, S, T)
    plan = tb.Plan(jobs, S, T)
    plan.autotune(series, jobs, 0)
    _check_autotuned(plan)
    for v in outs.values():
        v.fill_(777.0)
    plan.execute(series, jobs, 0)
    torch.cuda.synchronize()
    for name in workloads.PASS13_OUTPUTS:
        compare(outs[name].cpu().numpy(), ref[name], f"autotuned 4000x234 {name}")
    plan.close()


def test_autotune_ragged_picks_fastest_and_matches_oracle():
    lengths = synthetic.ragged_lengths(1200, 50, 5000, seed=12)
    planes, off = synthetic.ragged_ohlcv(lengths, seed=13)
    N = int(off[-1])
    dp = {k: torch.from_numpy(v).cuda() for k, v in planes.items()}
    doff = torch.from_numpy(off).cuda()
    outs = {n: torch.full((N,), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = pass13_jobs(outs)
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items()}, len(lengths), 0, doff.data_ptr())
    plan = tb.Plan(jobs, len(lengths), 0, off)
    plan.autotune(series, jobs, 0)
    _check_autotuned(plan)
    for v in outs.values():
        v.fill_(777.0)
    plan.execute(series, jobs, 0)
    torch.cuda.synchronize()
    ref = pass13_oracle(planes, off)
    for name in workloads.PASS13_OUTPUTS:
        compare_ragged(outs[name].cpu().numpy(), ref[name], off, f"autotuned ragged {name}")
    plan.close()


TUNE_CHILD = r"""
import json, sys, torch
sys.path.insert(0, sys.argv[1])
import tacuda_b200 as tb
from tacuda_b200 import synthetic, workloads
S, T = 640, 96
d = synthetic.ohlcv(S, T, seed=3)
dp = {k: torch.from_numpy(v).cuda() for k, v in d.items() if k in tb.PLANE_ID}
outs = {n: torch.empty((S, T), device="cuda") for n in workloads.PASS13_OUTPUTS}
jobs = [tb.make_job(f, p, fp, [outs[o].data_ptr() for o in on]) for _, f, p, fp, on in workloads.PASS13]
plan = tb.Plan(jobs, S, T)
if sys.argv[2] == "tune":
    plan.autotune(tb.make_series({k: v.data_ptr() for k, v in dp.items()}, S, T), jobs, 0)
print(json.dumps(plan.describe()))
"""


def test_tune_cache_round_trip(tmp_path):
    """A plan tuned in one process is found in TACUDA_B200_TUNE_CACHE by the
    next process that plans the same shape and job set."""
    cache = tmp_path / "tune.txt"
    env = dict(os.environ, TACUDA_B200_TUNE_CACHE=str(cache))
    env.pop("TACUDA_B200_MODE", None)

    def child(arg):
        out = subprocess.run([sys.executable, "-c", TUNE_CHILD, str(ROOT), arg], env=env, capture_output=True,
                             text=True, timeout=600)
        assert out.returncode == 0, out.stderr[-2000:]
        return json.loads(out.stdout.strip().splitlines()[-1])

    tuned = child("tune")
    assert cache.exists() and cache.read_text().strip(), "autotune wrote no cache entry"
    assert child("plan") == tuned
