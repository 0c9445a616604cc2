"""GPU parity: every family through its reference-named C entry point
(ct_*_batch_d) against the FP64 oracle, over shapes that exercise single and
multi-round rows, tiny rows and every round width; plus the fused multi-job
launch, ragged plans and the reference's row-independence invariants."""
import ctypes as ct
import os

import numpy as np
import pytest
import torch

import tacuda_b200 as tb
from gpu_util import DEFAULTS, SPECS, call_batch_d, device_planes, to_np
from test_oracle_pin import qstick_inf_rows
from oracle import oracle as O
from tacuda_b200 import synthetic, workloads
from tolerance import compare

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 16), (17, 19), (67, 234), (3, 513), (4, 3000)]


def oracle_data(d):
    out = dict(d)
    out["x"] = d["close"]
    out["y"] = d["open"]
    return out


def run_case(name, params, shape, seed=6):
    d = oracle_data(synthetic.ohlcv(*shape, seed=seed))
    if name.startswith("rolling_") and params["period"] > shape[1]:
        # ClubPack.cu:409-413: a rolling period above the row length is an invalid argument
        with pytest.raises(RuntimeError, match="code 4"):
            call_batch_d(name, device_planes(d), params)
        return []
    got = to_np(call_batch_d(name, device_planes(d), params))
    ref = O.run(name, d, **params)
    stats = []
    for i, (g, r) in enumerate(zip(got, ref)):
        stats.append(compare(g, r, f"{name}{params}[{i}] {shape}"))
    return stats


@pytest.fixture(params=["sp", "ws", "lb"])
def mode(request):
    """Every engine: row-parallel (a CTA per 32 rows, "sp"), warp-scan (a warp
    per series, "ws"), and look-back (a warp per tile chained by decoupled
    look-back, "lb")."""
    os.environ["TACUDA_B200_MODE"] = request.param
    yield request.param
    del os.environ["TACUDA_B200_MODE"]


@pytest.mark.parametrize("name", sorted(SPECS))
@pytest.mark.parametrize("shape", SHAPES)
def test_family_matches_oracle(name, shape, mode):
    run_case(name, DEFAULTS[name], shape)


VARIANTS = {
    "sma": [dict(period=1), dict(period=2), dict(period=64), dict(period=200)],
    "ema": [dict(period=1), dict(period=2), dict(period=63), dict(period=500)],
    "wma": [dict(period=1), dict(period=2), dict(period=64)],
    "rsi": [dict(period=1), dict(period=2), dict(period=3), dict(period=64)],
    "atr": [dict(period=1), dict(period=2), dict(period=64)],
    "natr": [dict(period=1), dict(period=2), dict(period=63)],
    "adx": [dict(period=2), dict(period=5), dict(period=30)],
    "dx": [dict(period=1), dict(period=5)],
    "macd": [dict(fast=26, slow=12, signal=9), dict(fast=2, slow=3, signal=2), dict(fast=5, slow=35, signal=1)],
    "bbands": [dict(period=2, up=1.5, dn=2.5), dict(period=64, up=2.0, dn=2.0)],
    "stoch": [dict(k=2, d=1), dict(k=5, d=5), dict(k=30, d=8)],
    "stddev": [dict(period=2, nbdev=1.0), dict(period=200, nbdev=1.0)],
    "var": [dict(period=2), dict(period=200)],
    "linearreg": [dict(period=2), dict(period=200)],
    "cci": [dict(period=2), dict(period=40)],
    "mfi": [dict(period=2), dict(period=64)],
    "willr": [dict(period=1), dict(period=50)],
    "min": [dict(period=1), dict(period=33)],
    "max": [dict(period=1), dict(period=33)],
    "adosc": [dict(fast=10, slow=3), dict(fast=2, slow=2)],
    "dema": [dict(period=1), dict(period=30)],
    "tema": [dict(period=2), dict(period=20)],
    "t3": [dict(period=1, vfactor=0.7), dict(period=8, vfactor=0.4)],
    "correl": [dict(period=2), dict(period=100)],
    "roc": [dict(period=1), dict(period=2), dict(period=300)],
    "rma": [dict(period=1), dict(period=2), dict(period=60)],
    "midprice": [dict(period=1), dict(period=2), dict(period=40)],
    "midpoint": [dict(period=1), dict(period=2), dict(period=40)],
    "momentum": [dict(period=1), dict(period=250)],
    "qstick": [dict(period=1), dict(period=2), dict(period=64)],
    "aroon": [dict(period=1), dict(period=2), dict(period=25), dict(period=90)],
    "aroonosc": [dict(period=1), dict(period=14), dict(period=90)],
}


@pytest.mark.parametrize("name,params", [(n, p) for n, ps in VARIANTS.items() for p in ps])
def test_parameter_corpus(name, params, mode):
    run_case(name, params, (7, 1300), seed=17)


def test_fused_pass_matches_oracle_and_single_calls(mode):
    S, T = 67, 700
    d = synthetic.ohlcv(S, T, seed=8)
    dp = device_planes(d)
    outs = {n: torch.full((S, T), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items() if k in tb.PLANE_ID}, S, T)
    tb.fused_batch_d(series, jobs, 0)
    torch.cuda.synchronize()
    for _, fam, p, fp, onames in workloads.PASS13:
        kw = workloads.ORACLE_PARAMS[fam](p, fp)
        ref = O.run(fam, d, **kw)
        single = to_np(call_batch_d(fam, dp, kw))
        for name, r, s in zip(onames, ref, single):
            g = outs[name].cpu().numpy()
            compare(g, r, f"fused {name}")
            np.testing.assert_array_equal(g.view(np.uint32), s.view(np.uint32), err_msg=f"fused vs single {name}")


def test_stream_zero_and_user_stream_agree():
    d = synthetic.ohlcv(33, 400, seed=9)
    dp = device_planes(d)
    a = to_np(call_batch_d("macd", dp, DEFAULTS["macd"]))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b = call_batch_d("macd", dp, DEFAULTS["macd"], stream=s.cuda_stream)
    s.synchronize()
    b = to_np(b)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.parametrize("name", ["ema", "rsi", "macd", "atr", "adx", "bbands", "stoch", "cci", "mfi", "obv", "willr"])
def test_row_independence(name, mode):
    """With the engine pinned, as the reference pins its fused path with
    TACUDA_BATCH_FUSED=1, rows, their order, batch size and future bars cannot
    change a row (tests/python/batch_fused.py:296-310). No round width is
    pinned: every engine's plan depends on the row alone."""
    try:
        S, T = 67, 234
        d = oracle_data(synthetic.ohlcv(S, T, seed=6))
        p = DEFAULTS[name]
        full = to_np(call_batch_d(name, device_planes(d), p))
        perm = np.random.default_rng(7).permutation(S)
        shuf = to_np(call_batch_d(name, device_planes({k: v[perm] for k, v in d.items()}), p))
        one = to_np(call_batch_d(name, device_planes({k: v[31:32] for k, v in d.items()}), p))
        pre = to_np(call_batch_d(name, device_planes({k: np.ascontiguousarray(v[:, :117]) for k, v in d.items()}), p))
        for a, b, c, e in zip(full, shuf, one, pre):
            np.testing.assert_array_equal(a[perm].view(np.uint32), b.view(np.uint32))
            np.testing.assert_array_equal(a[31:32].view(np.uint32), c.view(np.uint32))
            np.testing.assert_array_equal(a[:, :117].view(np.uint32), e.view(np.uint32))
        for at in (0, 110, 233):
            bad = {k: v.copy() for k, v in d.items()}
            for v in bad.values():
                v[0, at] = np.nan
            poisoned = to_np(call_batch_d(name, device_planes(bad), p))
            for a, b in zip(full, poisoned):
                np.testing.assert_array_equal(a[1:].view(np.uint32), b[1:].view(np.uint32))
    finally:
        pass


def test_known_answers_on_gpu(mode):
    flat = {k: np.full((3, 129), 100.0 if k != "volume" else 1000.0, np.float32)
            for k in ("open", "high", "low", "close", "volume")}
    dp = device_planes(flat)
    for name in ("sma", "ema", "rsi", "macd", "bbands", "cci", "willr", "adx", "stoch", "mfi", "atr"):
        got = to_np(call_batch_d(name, dp, DEFAULTS[name]))
        ref = O.run(name, flat, **DEFAULTS[name])
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(np.isnan(g), np.isnan(r))
            np.testing.assert_array_equal(g[~np.isnan(g)], r[~np.isnan(r)].astype(np.float32), err_msg=name)
    x = np.array([[1e30, 1.0, -1e30, 1.0, np.nan, 2.0]], np.float32)
    out = to_np(call_batch_d("ema", device_planes({"close": x}), dict(period=1)))[0]
    np.testing.assert_array_equal(out.view(np.uint32), x.view(np.uint32))
    x = np.arange(1.0, 40.0, dtype=np.float32)[None, :]
    m, s, h = to_np(call_batch_d("macd", device_planes({"close": x}), dict(fast=2, slow=3, signal=1)))
    assert np.all(np.isnan(m[:, :2])) and np.all(m[:, 2:] == 0.5) and np.all(s[:, 2:] == 0.5) and np.all(h[:, 2:] == 0)
    c = np.array([[1, 2, 1, 2, 1]], np.float32)
    sv = {"close": c, "high": c + 1, "low": c - 1, "volume": np.array([[10, -1, 10, -1, 10]], np.float32)}
    out = to_np(call_batch_d("mfi", device_planes(sv), dict(period=2)))[0]
    np.testing.assert_array_equal(out[:, 2:], -25.0)


def test_leading_nan_and_interior_nan_semantics(mode):
    d = synthetic.ohlcv(5, 600, seed=12)
    for v in d.values():
        v[1, :37] = np.nan
        v[2, 300] = np.nan
    d = oracle_data(d)
    dp = device_planes(d)
    for name in ("ema", "rsi", "macd", "sma", "bbands", "willr", "min", "max", "dema", "roc", "rma",
                 "medprice", "typprice", "midprice", "rocp", "rocr", "rocr100", "momentum", "avgprice",
                 "wclprice", "midpoint", "ibs", "marketfi", "qstick"):
        got = to_np(call_batch_d(name, dp, DEFAULTS[name]))
        ref = O.run(name, d, **DEFAULTS[name])
        for i, (g, r) in enumerate(zip(got, ref)):
            compare(g, r, f"nan {name}[{i}]")


def test_ragged_plan_matches_oracle(mode):
    lengths = synthetic.ragged_lengths(300, 1, 5000, seed=3)
    lengths[:5] = [0, 1, 2, 1024, 4097]
    planes, off = synthetic.ragged_ohlcv(lengths, seed=4)
    dp = {k: torch.from_numpy(v).to("cuda") for k, v in planes.items()}
    doff = torch.from_numpy(off).to("cuda")
    N = int(off[-1])
    outs = {n: torch.full((N,), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    plan = tb.Plan(jobs, len(lengths), 0, off)
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items()}, len(lengths), 0, doff.data_ptr())
    plan.execute(series, jobs, 0)
    torch.cuda.synchronize()
    for _, fam, p, fp, onames in workloads.PASS13:
        ref = O.run(fam, planes, offsets=off, **workloads.ORACLE_PARAMS[fam](p, fp))
        for name, r in zip(onames, ref):
            g = outs[name].cpu().numpy()
            for s in range(len(lengths)):
                a, b = off[s], off[s + 1]
                if b > a:
                    compare(g[a:b], r[a:b], f"ragged {name} row {s} len {b - a}")
    plan.close()


def test_graph_capture_replay_equals_eager(mode):
    S, T = 67, 234
    d = synthetic.ohlcv(S, T, seed=6)
    dp = device_planes(d)
    outs = {n: torch.empty((S, T), device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items()}, S, T)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        tb.fused_batch_d(series, jobs, s.cuda_stream)
    s.synchronize()
    eager = {k: v.clone() for k, v in outs.items()}
    g = torch.cuda.CUDAGraph()
    n0 = tb.launch_count()
    with torch.cuda.graph(g, stream=s):
        tb.fused_batch_d(series, jobs, torch.cuda.current_stream().cuda_stream)
    assert tb.launch_count() - n0 == 1
    for _ in range(3):
        for v in outs.values():
            v.fill_(float("nan"))
            v.view(torch.int32).fill_(0x5A5A5A5A)
        g.replay()
        torch.cuda.synchronize()
        for k in outs:
            assert torch.equal(outs[k].view(torch.int32), eager[k].view(torch.int32)), k
    del g


LOOKBACK_FAMILIES = ["ema", "dema", "tema", "t3", "rsi", "macd", "atr", "natr", "adx", "dx", "obv", "ad", "adosc",
                     "min", "max", "correl", "sma", "stoch", "mfi", "rma", "roc", "midprice", "midpoint", "ibs", "qstick"]
SINGLE_INPUT = {"ema", "dema", "tema", "t3", "rsi", "macd", "min", "max", "sma", "rma", "roc", "midpoint"}


@pytest.mark.parametrize("bars", ["4", "16"])
@pytest.mark.parametrize("name", LOOKBACK_FAMILIES)
def test_lookback_long_rows(name, bars):
    """Rows of hundreds of tiles chained by look-back (checkpoints every 32
    tiles, warm-up spanning tiles, a leading NaN run ending inside a later
    tile) match the oracle, and repeated launches are bit-identical."""
    os.environ["TACUDA_B200_MODE"] = "lb"
    os.environ["TACUDA_B200_BARS_PER_LANE"] = bars
    try:
        d = oracle_data(synthetic.ohlcv(3, 30000, seed=21))
        if name in SINGLE_INPUT:
            d["close"][1, :1500] = np.nan
        if name == "correl":
            d["x"][2, 20000] = np.inf
        p = dict(DEFAULTS[name])
        if name in ("ema", "rsi", "dema"):
            p["period"] = 300
        dp = device_planes(d)
        got = to_np(call_batch_d(name, dp, p))
        again = to_np(call_batch_d(name, dp, p))
        ref = O.run(name, d, **p)
        for i, (g, a, r) in enumerate(zip(got, again, ref)):
            compare(g, r, f"lookback {name}[{i}] bars/lane {bars}")
            np.testing.assert_array_equal(g.view(np.uint32), a.view(np.uint32))
    finally:
        del os.environ["TACUDA_B200_MODE"]
        del os.environ["TACUDA_B200_BARS_PER_LANE"]


def test_lookback_fused_pass_on_long_rows():
    """The 13-indicator fused pass over three 60000-bar rows in look-back mode
    (the default plan for few long rows) matches the oracle."""
    S, T = 3, 60000
    d = synthetic.ohlcv(S, T, seed=23)
    dp = device_planes(d)
    outs = {n: torch.full((S, T), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items() if k in tb.PLANE_ID}, S, T)
    plan = tb.Plan(jobs, S, T)
    assert plan.describe()["mode"] == 2
    plan.execute(series, jobs, 0)
    torch.cuda.synchronize()
    for _, fam, p, fp, onames in workloads.PASS13:
        ref = O.run(fam, d, **workloads.ORACLE_PARAMS[fam](p, fp))
        for name, r in zip(onames, ref):
            compare(outs[name].cpu().numpy(), r, f"lookback fused {name}")
    plan.close()


@pytest.mark.parametrize("name", ["ema", "macd", "rsi", "adx", "obv", "t3", "correl", "atr"])
def test_lookback_beyond_checkpoint_span(name):
    """Rows of 2,344 tiles (128-bar rounds): several checkpoint spans of 1,024
    tiles, whole-group aggregates, and (single-input families) a 200,000-bar
    leading NaN run that keeps the first 1,500 tiles in warm-up."""
    os.environ["TACUDA_B200_MODE"] = "lb"
    os.environ["TACUDA_B200_BARS_PER_LANE"] = "4"
    try:
        d = oracle_data(synthetic.ohlcv(2, 300_000, seed=29))
        if name in SINGLE_INPUT:
            d["close"][1, :200_000] = np.nan
        p = DEFAULTS[name]
        dp = device_planes(d)
        got = to_np(call_batch_d(name, dp, p))
        again = to_np(call_batch_d(name, dp, p))
        ref = O.run(name, d, **p)
        for i, (g, a, r) in enumerate(zip(got, again, ref)):
            compare(g, r, f"span {name}[{i}]")
            np.testing.assert_array_equal(g.view(np.uint32), a.view(np.uint32))
    finally:
        del os.environ["TACUDA_B200_MODE"]
        del os.environ["TACUDA_B200_BARS_PER_LANE"]


PREC_JOBS = [("sma", dict(period=200)), ("stddev", dict(period=200, nbdev=1.0)), ("var", dict(period=200)),
             ("linearreg", dict(period=200)), ("correl", dict(period=30)), ("ema", dict(period=500)),
             ("bbands", dict(period=20, up=2.0, dn=1.5)), ("wma", dict(period=30)), ("sum", dict(period=50))]
# tolerance of each precision variant against the FP64 oracle on a +1e4-level
# random walk: |gpu - ref| <= tol*|ref| + tol*max|ref row|. Plain FP32 has no
# bound there (its running sums lose the digits the level offset cancels); it
# is only checked for its NaN mask, and its error is what the long-series
# precision report measures.
PREC_TOL = {"fp32": None, "fp32c": 1e-6, "fp32/fp64carry": 1e-5}


@pytest.mark.parametrize("engine", ["ws", "lb"])
@pytest.mark.parametrize("prec", sorted(PREC_TOL))
def test_precision_variants_on_level_offset_rows(prec, engine):
    """FP32, compensated FP32 and FP32-with-FP64-carry variants of the long
    window families and the EMA, against the FP64 oracle on level-offset
    rows (the long-series precision stress at a testable size)."""
    os.environ["TACUDA_B200_MODE"] = engine
    try:
        S, T = 3, 20000
        x = synthetic.level_walk(S, T, seed=41)
        y = synthetic.level_walk(S, T, seed=42)
        d = {"close": x, "x": x, "y": y, "aux": y}
        dx = torch.from_numpy(x).cuda()
        dy = torch.from_numpy(y).cuda()
        for name, params in PREC_JOBS:
            fam = name
            nout = 3 if name == "bbands" else 1
            outs = [torch.full((S, T), 777.0, device="cuda") for _ in range(nout)]
            spec_p = tuple(v for k, v in params.items() if k == "period")
            fp = tuple(v for k, v in params.items() if k in ("nbdev", "up", "dn"))
            job = tb.make_job(fam, spec_p, fp, [o.data_ptr() for o in outs],
                              inputs=("close", "aux") if name == "correl" else None, precision=prec)
            series = tb.make_series({"close": dx.data_ptr(), "aux": dy.data_ptr()}, S, T)
            tb.fused_batch_d(series, [job], 0)
            torch.cuda.synchronize()
            ref = O.run(name, d, **params)
            tol = PREC_TOL[prec]
            for i, (g, r) in enumerate(zip(outs, ref)):
                g = g.cpu().numpy().astype(np.float64)
                np.testing.assert_array_equal(np.isnan(g), np.isnan(r), err_msg=f"{prec} {name} NaN mask")
                if tol is None:
                    continue
                m = ~np.isnan(r)
                bound = tol * np.abs(r[m]) + tol * np.max(np.abs(r[m]))
                err = np.abs(g[m] - r[m])
                assert np.all(err <= bound), f"{prec} {engine} {name}[{i}]: worst excess {np.max(err - bound)}"
    finally:
        del os.environ["TACUDA_B200_MODE"]


@pytest.mark.parametrize("S,T", [(4000, 234), (37, 50), (9, 3001)])
def test_host_entry_matches_device_entry(S, T):
    """ct_b200_fused_batch (host buffers; large batches pipelined in row
    chunks over auxiliary streams) gives the device entry point's bits."""
    d = synthetic.ohlcv(S, T, seed=31)
    dp = device_planes(d)
    douts = {n: torch.full((S, T), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = [tb.make_job(fam, p, fp, [douts[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    tb.fused_batch_d(tb.make_series({k: v.data_ptr() for k, v in dp.items() if k in tb.PLANE_ID}, S, T), jobs, 0)
    torch.cuda.synchronize()
    hp = {k: torch.from_numpy(v).pin_memory() for k, v in d.items()}
    houts = {n: torch.full((S, T), 555.0).pin_memory() for n in workloads.PASS13_OUTPUTS}
    hjobs = [tb.make_job(fam, p, fp, [houts[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    s = torch.cuda.Stream()
    tb.fused_batch(tb.make_series({k: v.data_ptr() for k, v in hp.items() if k in tb.PLANE_ID}, S, T), hjobs,
                   s.cuda_stream)
    for n in workloads.PASS13_OUTPUTS:
        np.testing.assert_array_equal(houts[n].numpy().view(np.uint32), douts[n].cpu().numpy().view(np.uint32),
                                      err_msg=n)


FLOAT_KERNELS = {"roc": [dict(period=1), dict(period=10), dict(period=700)], "medprice": [{}], "typprice": [{}],
                 "midprice": [dict(period=1), dict(period=7), dict(period=100)],
                 "rocp": [dict(period=1), dict(period=33)], "rocr": [dict(period=2), dict(period=64)],
                 "rocr100": [dict(period=5)], "momentum": [dict(period=1), dict(period=9)],
                 "avgprice": [{}], "wclprice": [{}],
                 "midpoint": [dict(period=1), dict(period=7), dict(period=100)], "change": [dict(period=4)],
                 "rolling_mean": [dict(period=1), dict(period=30)], "rolling_max": [dict(period=7)],
                 "rolling_min": [dict(period=200)], "rolling_std": [dict(period=1), dict(period=25)],
                 "ibs": [{}], "marketfi": [{}]}


@pytest.mark.parametrize("name", sorted(FLOAT_KERNELS))
def test_float_kernel_families_bit_exact(name, mode):
    """The ROC family, MOM, the price transforms, MIDPRICE and MIDPOINT repeat
    the reference kernels' float arithmetic, so every output word equals the
    oracle's float result, with zeros (the ratios' zero divisor), NaN and
    infinite bars and a leading NaN run mixed in."""
    d = synthetic.ohlcv(9, 2500, seed=41)
    d["close"][1, ::97] = 0.0
    d["close"][2, 50:60] = np.nan
    d["close"][6, :300] = np.nan
    d["close"][7, 1500] = np.inf  # the rolling statistics are NaN wherever a window holds it
    d["high"][3, 400:410] = np.nan
    d["low"][4, 1000] = -np.inf
    d["high"][5, :] = np.nan  # whole windows of NaN: MIDPRICE stays NaN there
    dp = device_planes(d)
    for p in FLOAT_KERNELS[name]:
        got = to_np(call_batch_d(name, dp, p))[0]
        ref = O.run(name, d, **p)[0].astype(np.float32)
        np.testing.assert_array_equal(np.isnan(got), np.isnan(ref), err_msg=f"{name}{p}")
        m = ~np.isnan(ref)
        np.testing.assert_array_equal(got[m].view(np.uint32), ref[m].view(np.uint32), err_msg=f"{name}{p}")


@pytest.mark.parametrize("name", ["aroon", "aroonosc"])
def test_aroon_bit_exact(name, mode):
    """AROON and AROONOSC repeat the reference kernels' float arithmetic
    (src/indicators/Aroon.cu, AroonOscillator.cu), so every output word equals
    the oracle's float result, with ties (flat highs and lows, where the most
    recent bar wins), NaN and infinite bars, and a NaN at the current bar."""
    d = synthetic.ohlcv(8, 1500, seed=43)
    d["high"][1, 100:160] = 105.0
    d["low"][1, 100:160] = 95.0
    d["high"][2, 300:310] = np.nan
    d["low"][3, 500] = np.nan
    d["high"][4, 700] = np.inf
    d["low"][5, 800] = -np.inf
    d["high"][6, :] = np.nan
    dp = device_planes(d)
    for p in (1, 7, 14, 40, 100):
        got = to_np(call_batch_d(name, dp, dict(period=p)))
        ref = O.run(name, d, period=p)
        for i, (g, r) in enumerate(zip(got, ref)):
            r = r.astype(np.float32)
            np.testing.assert_array_equal(np.isnan(g), np.isnan(r), err_msg=f"{name}[{i}] p={p}")
            m = ~np.isnan(r)
            np.testing.assert_array_equal(g[m].view(np.uint32), r[m].view(np.uint32), err_msg=f"{name}[{i}] p={p}")


def test_rma_period_one_propagates_nan(mode):
    """TA_RMA has no period-1 shortcut: fma(0, NaN, x) keeps a NaN from an
    interior bar to the end of the row (unlike EMA(1), which copies)."""
    x = np.array([[np.nan, 1.0, 2.0, np.nan, 3.0, 4.0]], np.float32)
    got = to_np(call_batch_d("rma", device_planes({"close": x}), dict(period=1)))[0]
    ref = O.run("rma", {"close": x}, period=1)[0]
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    assert np.isnan(got[0, 3:]).all() and (got[0, 1:3] == [1.0, 2.0]).all()


NEW_JOBS = [("roc", (10,), {"period": 10}), ("rma", (14,), {"period": 14}), ("medprice", (), {}),
            ("typprice", (), {}), ("midprice", (14,), {"period": 14}), ("ema", (14,), {"period": 14}),
            ("rocr100", (7,), {"period": 7}), ("momentum", (3,), {"period": 3}), ("avgprice", (), {}),
            ("wclprice", (), {}), ("midpoint", (20,), {"period": 20}), ("rolling_std", (15,), {"period": 15}),
            ("rolling_max", (9,), {"period": 9})]


def test_fused_pass_with_price_transforms_roc_rma(mode):
    """ROC, RMA, MEDPRICE, TYPPRICE and MIDPRICE share one fused launch with an
    EMA job on uniform rows (bit-equal to their single entry points) and on a
    ragged plan (against the oracle)."""
    S, T = 41, 900
    d = synthetic.ohlcv(S, T, seed=43)
    dp = device_planes(d)
    outs = [torch.full((S, T), 777.0, device="cuda") for _ in NEW_JOBS]
    jobs = [tb.make_job(fam, p, (), [o.data_ptr()]) for (fam, p, _), o in zip(NEW_JOBS, outs)]
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items() if k in tb.PLANE_ID}, S, T)
    tb.fused_batch_d(series, jobs, 0)
    torch.cuda.synchronize()
    for (fam, _, kw), o in zip(NEW_JOBS, outs):
        g = o.cpu().numpy()
        compare(g, O.run(fam, d, **kw)[0], f"fused {fam}")
        single = to_np(call_batch_d(fam, dp, kw))[0]
        np.testing.assert_array_equal(g.view(np.uint32), single.view(np.uint32), err_msg=f"fused vs single {fam}")

    lengths = synthetic.ragged_lengths(120, 1, 3000, seed=44)
    lengths[:4] = [0, 1, 15, 2049]
    planes, off = synthetic.ragged_ohlcv(lengths, seed=45)
    rp = {k: torch.from_numpy(v).to("cuda") for k, v in planes.items()}
    doff = torch.from_numpy(off).to("cuda")
    N = int(off[-1])
    routs = [torch.full((N,), 777.0, device="cuda") for _ in NEW_JOBS]
    rjobs = [tb.make_job(fam, p, (), [o.data_ptr()]) for (fam, p, _), o in zip(NEW_JOBS, routs)]
    plan = tb.Plan(rjobs, len(lengths), 0, off)
    rseries = tb.make_series({k: v.data_ptr() for k, v in rp.items()}, len(lengths), 0, doff.data_ptr())
    plan.execute(rseries, rjobs, 0)
    torch.cuda.synchronize()
    for (fam, _, kw), o in zip(NEW_JOBS, routs):
        ref = O.run(fam, planes, offsets=off, **kw)[0]
        g = o.cpu().numpy()
        for s in range(len(lengths)):
            a, b = off[s], off[s + 1]
            if b > a:
                compare(g[a:b], ref[a:b], f"ragged {fam} row {s} len {b - a}")
    plan.close()


def test_talib_runner_prefix_rule(mode):
    """IBS and MARKETFI start at the first bar where no input is NaN; a row
    with no complete bar evaluates its last bar only (src/compat/Talib08.cu:72-84)."""
    d = synthetic.ohlcv(6, 700, seed=47)
    d["close"][1, :40] = np.nan
    d["volume"][2, :333] = np.nan
    d["close"][3, :] = np.nan
    d["high"][3, -1] = d["low"][3, -1]  # zero range on the last bar: IBS gives 0.5 there
    d["volume"][4, :] = np.nan
    d["volume"][5, 100] = 0.0
    dp = device_planes(d)
    d["open"][4, 500] = np.nan  # QSTICK: NaN from here to the end of the row
    dp = device_planes(d)
    for name, p in (("ibs", {}), ("marketfi", {}), ("qstick", dict(period=10))):
        got = to_np(call_batch_d(name, dp, p))[0]
        ref = O.run(name, d, **p)[0]
        compare(got, ref, f"prefix {name}")
    assert np.isnan(to_np(call_batch_d("qstick", dp, dict(period=10)))[0][4, 500:]).all()
    # infinite close - open differences: TA_QSTICK's running sum is inf while
    # one is in the window and NaN for good once it leaves
    q = qstick_inf_rows()
    got = to_np(call_batch_d("qstick", device_planes(q), dict(period=10)))[0]
    ref = O.run("qstick", q, period=10)[0]
    for kind in (np.isposinf, np.isneginf):
        np.testing.assert_array_equal(kind(got), kind(ref))
    fin = np.isfinite(ref)
    compare(np.where(fin, got, np.nan), np.where(fin, ref, np.nan), "qstick with infinite differences")
    assert to_np(call_batch_d("ibs", dp, {}))[0][3, -1] == 0.5
