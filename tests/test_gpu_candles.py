"""GPU: the 63 candle families bit-exact against the oracle (which is pinned
bit-exactly to the reference's CandleUtils.h), through the per-pattern
reference entry points and the one-pass int32 engine, uniform and ragged."""
import os

import numpy as np
import pytest
import torch

import tacuda_b200 as tb
from gpu_util import call_cdl, device_planes, to_np
from oracle import oracle as O
from tacuda_b200 import synthetic

pytestmark = pytest.mark.gpu
NAMES = tb.cdl_names()


@pytest.fixture(params=["tile", "sp"])
def engine(request):
    """Bar-parallel tile kernel (default) and the series-parallel engine."""
    if request.param == "sp":
        os.environ["TACUDA_B200_MODE"] = "sp"
    yield request.param
    os.environ.pop("TACUDA_B200_MODE", None)


def candle_data(S, T, seed):
    d = synthetic.ohlcv(S, T, seed=seed)
    # a few rows with coarse prices: doji, equal bodies and gaps become common
    rng = np.random.default_rng(seed)
    for s in range(min(S, 4)):
        base = np.round(100 + np.cumsum(rng.integers(-3, 4, T)) * 0.25, 2).astype(np.float32)
        o = base
        c = np.roll(base, -1)
        c[-1] = base[-1]
        d["open"][s], d["close"][s] = o, c
        d["high"][s] = np.maximum(o, c) + np.float32(0.25) * rng.integers(0, 3, T).astype(np.float32)
        d["low"][s] = np.minimum(o, c) - np.float32(0.25) * rng.integers(0, 3, T).astype(np.float32)
    return d


@pytest.mark.parametrize("k", range(63))
def test_candle_family_bit_exact(k, engine):
    d = candle_data(40, 300, seed=100 + k)
    out = to_np([call_cdl(k, device_planes(d), NAMES[k])])[0]
    ref = O.cdl(k, d["open"], d["high"], d["low"], d["close"])
    np.testing.assert_array_equal(out, ref.astype(np.float32), err_msg=NAMES[k])


def test_all_patterns_one_pass_int32(engine):
    S, T = 600, 333
    d = candle_data(S, T, seed=7)
    dp = device_planes(d)
    out = torch.full((63, S, T), 77, dtype=torch.int32, device="cuda")
    lib = tb.get_lib()
    import ctypes as ct
    rc = lib.ct_b200_cdl_batch_d(*(ct.c_void_p(dp[p].data_ptr()) for p in ("open", "high", "low", "close")),
                                 ct.c_void_p(out.data_ptr()), T, S, ct.c_uint64((1 << 63) - 1), None)
    tb.call_status(rc, "ct_b200_cdl_batch_d")
    got = out.cpu().numpy()
    total = 0
    for k in range(63):
        ref = O.cdl(k, d["open"], d["high"], d["low"], d["close"])
        np.testing.assert_array_equal(got[k], ref, err_msg=NAMES[k])
        total += int(np.count_nonzero(ref))
    assert total > 1000


def test_candles_ragged_plan_split_jobs(engine):
    lengths = synthetic.ragged_lengths(200, 1, 3000, seed=9)
    lengths[:4] = [0, 1, 15, 2049]
    planes, off = synthetic.ragged_ohlcv(lengths, seed=10)
    dp = {k: torch.from_numpy(v).to("cuda") for k, v in planes.items()}
    N = int(off[-1])
    out = torch.full((63, N), 55, dtype=torch.int32, device="cuda")
    groups = [list(range(i, 63, 7)) for i in range(7)]
    jobs = [tb.make_job("cdl", (), (), [out.data_ptr()], cdl_mask=sum(1 << k for k in g), cdl_stride=N,
                        cdl_int32=True) for g in groups]
    plan = tb.Plan(jobs, len(lengths), 0, off)
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items()}, len(lengths), 0,
                            torch.from_numpy(off).to("cuda").data_ptr())
    plan.execute(series, jobs, 0)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for k in range(63):
        ref = O.cdl(k, planes["open"], planes["high"], planes["low"], planes["close"], offsets=off)
        np.testing.assert_array_equal(got[k], ref, err_msg=NAMES[k])
    plan.close()


def test_indicators_and_candles_in_one_plan():
    """A plan mixing the 13-indicator pass with a candle job (int32, all 61
    TA-Lib patterns) over ragged rows: both parts match the oracle."""
    from tacuda_b200 import workloads
    from tolerance import compare
    lengths = synthetic.ragged_lengths(150, 1, 4000, seed=12)
    lengths[:3] = [0, 17, 1500]
    planes, off = synthetic.ragged_ohlcv(lengths, seed=13)
    dp = {k: torch.from_numpy(v).to("cuda") for k, v in planes.items()}
    doff = torch.from_numpy(off).to("cuda")
    N = int(off[-1])
    outs = {n: torch.full((N,), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    cdl = torch.full((63, N), 55, dtype=torch.int32, device="cuda")
    mask = sum(1 << k for k, n in enumerate(NAMES) if n not in ("bullish_engulfing", "bearish_engulfing"))
    jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    jobs.append(tb.make_job("cdl", (), (), [cdl.data_ptr()], cdl_mask=mask, cdl_stride=N, cdl_int32=True))
    plan = tb.Plan(jobs, len(lengths), 0, off)
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items()}, len(lengths), 0, doff.data_ptr())
    plan.execute(series, jobs, 0)
    torch.cuda.synchronize()
    for _, fam, p, fp, onames in workloads.PASS13:
        ref = O.run(fam, planes, offsets=off, **workloads.ORACLE_PARAMS[fam](p, fp))
        for name, r in zip(onames, ref):
            compare(outs[name].cpu().numpy(), r, f"mixed plan {name}")
    got = cdl.cpu().numpy()
    for k in range(63):
        if (mask >> k) & 1:
            ref = O.cdl(k, planes["open"], planes["high"], planes["low"], planes["close"], offsets=off)
            np.testing.assert_array_equal(got[k], ref, err_msg=NAMES[k])
        else:
            assert np.all(got[k] == 55)
    plan.close()
