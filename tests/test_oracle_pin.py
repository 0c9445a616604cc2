"""CPU: the project's FP64 oracle against the reference's own CPU code.

Pins oracle/ta_oracle.c and oracle/oracle_candles.c against (a) the committed
golden fixtures generated from the reference build (tests/golden), and (b) the
reference build itself (oracle/_ref) on fresh seeded data when it is present.
Families without reference CPU code (ADX, DX, CCI, WILLR, CORREL, SUM, MIN,
MAX) are pinned by known-answer tests.
"""
import os
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tacuda_b200 import synthetic
from tolerance import compare

GOLD = np.load(Path(__file__).with_name("golden") / "golden_ref.npz")
CASES = {
    "sma": dict(period=20), "ema": dict(period=14), "wma": dict(period=14), "rsi": dict(period=14),
    "stddev": dict(period=20, nbdev=1.0), "var": dict(period=20), "linearreg": dict(period=14),
    "dema": dict(period=10), "tema": dict(period=8), "t3": dict(period=5, vfactor=0.7),
    "macd": dict(fast=12, slow=26, signal=9), "bbands": dict(period=20, up=2.0, dn=2.0),
    "atr": dict(period=14), "trange": {}, "stoch": dict(k=14, d=3), "obv": {}, "ad": {},
    "mfi": dict(period=14), "adosc": dict(fast=3, slow=10), "natr": dict(period=14),
    "roc": dict(period=10), "rma": dict(period=14), "medprice": {}, "typprice": {}, "midprice": dict(period=14),
    "rocp": dict(period=10), "ibs": {}, "marketfi": {}, "qstick": dict(period=10),
}


def gold_inputs():
    return {k[3:]: GOLD[k] for k in GOLD.files if k.startswith("in_")}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden(name):
    d = gold_inputs()
    res = O.run(name, d, **CASES[name])
    for i, r in enumerate(res):
        ref = GOLD[f"{name}_{i}"]
        # float32-rounded reference states (OBV/AD/ADOSC/MFI/NATR) compare at float precision
        compare(r, ref, f"{name}[{i}]", rtol=1e-6, row_atol=1e-9 if ref.dtype == np.float64 else 1e-7)


def test_oracle_candles_match_golden():
    d = gold_inputs()
    for k in range(63):
        got = O.cdl(k, d["open"], d["high"], d["low"], d["close"])
        np.testing.assert_array_equal(got, GOLD[f"cdl_{k}"], err_msg=f"candle {k}")


def test_golden_fixture_has_signals():
    total = sum(int(np.count_nonzero(GOLD[f"cdl_{k}"])) for k in range(63))
    assert total > 500


@pytest.mark.skipif(not O.ref_available(), reason="reference CPU build not present")
@pytest.mark.parametrize("shape,seed", [((32, 257), 1), ((3, 1200), 2), ((17, 19), 3)])
def test_oracle_matches_reference_build(shape, seed):
    d = synthetic.ohlcv(*shape, seed=seed)
    for name, p in CASES.items():
        a = O.run(name, d, **p)
        b = O.ref_run(name, d, **p)
        for i, (x, y) in enumerate(zip(a, b)):
            compare(x, y, f"{name}[{i}] {shape}", rtol=1e-6, row_atol=1e-9 if np.asarray(y).dtype == np.float64 else 1e-7)
    for k in range(63):
        np.testing.assert_array_equal(O.cdl(k, d["open"], d["high"], d["low"], d["close"]),
                                      O.ref_cdl(k, d["open"], d["high"], d["low"], d["close"]), err_msg=f"candle {k}")


def qstick_inf_rows():
    """Rows whose close - open differences hold infinities: TA_QSTICK's running
    sum turns NaN for good once an infinite difference leaves the window."""
    d = synthetic.ohlcv(4, 300, seed=31)
    d["close"][0, 100] = np.inf                       # inf for 10 bars, then NaN
    d["close"][1, 50] = np.inf
    d["open"][1, 53] = np.inf                         # -inf difference: NaN at once
    d["open"][2, 5] = -np.inf                         # inf inside the first window
    d["close"][3, 200] = np.inf
    d["open"][3, 200] = np.inf                        # inf - inf: a NaN difference
    return d


@pytest.mark.skipif(not O.ref_available(), reason="reference CPU build not present")
def test_qstick_infinite_difference_matches_reference_build():
    d = qstick_inf_rows()
    a = O.run("qstick", d, period=10)[0]
    b = O.ref_run("qstick", d, period=10)[0]
    for kind in (np.isnan, np.isposinf, np.isneginf):
        np.testing.assert_array_equal(kind(a), kind(b))
    fin = np.isfinite(b)
    compare(np.where(fin, a, np.nan), np.where(fin, b, np.nan), "qstick with infinite differences", rtol=1e-6,
            row_atol=1e-9)


def test_aroon_known_answers():
    """src/indicators/Aroon.cu: rising highs put the high at the current bar
    (up = 100), falling lows the low there too (down = 100); flat windows tie
    and the most recent bar wins (100); the oscillator is up - down; warm-up
    NaN for the first p bars."""
    T, p = 40, 10
    h = np.arange(T, dtype=np.float32)[None, :] + 100.0
    lo = (200.0 - np.arange(T, dtype=np.float32))[None, :]
    dn, up = O.run("aroon", {"high": h, "low": lo}, period=p)
    assert np.isnan(up[0, :p]).all() and (up[0, p:] == 100.0).all() and (dn[0, p:] == 100.0).all()
    flat = np.full((1, T), 50.0, np.float32)
    dn, up = O.run("aroon", {"high": flat, "low": flat}, period=p)
    assert (up[0, p:] == 100.0).all() and (dn[0, p:] == 100.0).all()
    # the highest high 3 bars back, the lowest low at the window's oldest bar
    h2 = np.full((1, 12), 10.0, np.float32)
    h2[0, 8] = 20.0
    l2 = np.full((1, 12), 5.0, np.float32)
    l2[0, 1] = 1.0
    dn, up = O.run("aroon", {"high": h2, "low": l2}, period=p)
    assert up[0, 11] == np.float32(100.0) * np.float32(p - 3) / np.float32(p)
    assert dn[0, 11] == np.float32(0.0)
    osc = O.run("aroonosc", {"high": h2, "low": l2}, period=p)[0]
    assert osc[0, 11] == up[0, 11] - dn[0, 11]
    # a NaN high at the current bar keeps the current bar (strict comparisons)
    h3 = h2.copy()
    h3[0, 11] = np.nan
    assert O.run("aroon", {"high": h3, "low": l2}, period=p)[1][0, 11] == 100.0


def test_qstick_infinite_difference_rule():
    a = O.run("qstick", qstick_inf_rows(), period=10)[0]
    assert np.isposinf(a[0, 100:110]).all() and np.isnan(a[0, 110:]).all() and np.isfinite(a[0, 9:100]).all()
    assert np.isposinf(a[1, 50:53]).all() and np.isnan(a[1, 53:]).all()
    assert np.isposinf(a[2, 9:15]).all() and np.isnan(a[2, 15:]).all()
    assert np.isfinite(a[3, 9:200]).all() and np.isnan(a[3, 200:]).all()


# ---- known answers (tests/cpp/test_edge_cases.cpp, tests/python/batch_fused.py) ----

def flat(T=129, value=100.0):
    return {k: np.full((3, T), value if k != "volume" else 1000.0, np.float32)
            for k in ("open", "high", "low", "close", "volume")}


def test_flat_series_known_answers():
    d = flat()
    assert np.allclose(O.run("sma", d, period=20)[0][:, 19:], 100.0)
    assert np.allclose(O.run("ema", d, period=14)[0][:, 13:], 100.0)
    assert np.allclose(O.run("rsi", d, period=14)[0][:, 14:], 50.0)
    m, s, h = O.run("macd", d, fast=12, slow=26, signal=9)
    assert np.all(m[:, 33:] == 0.0) and np.all(h[:, 33:] == 0.0)
    assert np.all(O.run("cci", d, period=14)[0][:, 13:] == 0.0)
    assert np.all(O.run("willr", d, period=14)[0][:, 13:] == 0.0)
    assert np.all(O.run("adx", d, period=14)[0][:, 27:] == 0.0)
    assert np.all(np.isnan(O.run("adx", d, period=14)[0][:, :27]))
    assert np.all(O.run("correl", {"x": d["close"], "y": d["close"]}, period=10)[0][:, 9:] == 0.0)


def test_atr_constant_range_is_range():
    # H - L = 10 everywhere, closes inside: ATR = 10 (test_edge_cases.cpp:162-183)
    T = 60
    c = np.full((1, T), 100.0, np.float32)
    d = {"high": c + 5, "low": c - 5, "close": c}
    out = O.run("atr", d, period=14)[0]
    assert np.allclose(out[:, 14:], 10.0) and np.all(np.isnan(out[:, :14]))


def test_ema_period_one_passthrough():
    x = np.array([[1e30, 1.0, -1e30, 1.0, np.nan, 2.0]], np.float32)
    out = O.run("ema", {"close": x}, period=1)[0]
    np.testing.assert_array_equal(out.astype(np.float32), x)


def test_macd_2_3_1_constants():
    x = np.arange(1.0, 40.0, dtype=np.float32)[None, :]
    m, s, h = O.run("macd", {"close": x}, fast=2, slow=3, signal=1)
    assert np.all(np.isnan(m[:, :2]))
    assert np.all(m[:, 2:] == 0.5) and np.all(s[:, 2:] == 0.5) and np.all(h[:, 2:] == 0.0)


def test_mfi_signed_volume():
    c = np.array([[1, 2, 1, 2, 1]], np.float32)
    d = {"close": c, "high": c + 1, "low": c - 1, "volume": np.array([[10, -1, 10, -1, 10]], np.float32)}
    out = O.run("mfi", d, period=2)[0]
    np.testing.assert_array_equal(out[:, 2:], -25.0)


def test_minmax_and_sum_windows():
    x = np.array([[3, 1, 4, 1, 5, 9, 2, 6]], np.float32)
    np.testing.assert_array_equal(O.run("max", {"close": x}, period=3)[0][0, 2:], [4, 4, 5, 9, 9, 9])
    np.testing.assert_array_equal(O.run("min", {"close": x}, period=3)[0][0, 2:], [1, 1, 1, 1, 2, 2])
    np.testing.assert_array_equal(O.run("sum", {"close": x}, period=3)[0][0, 2:], [8, 6, 10, 15, 16, 17])


def test_willr_clamp_and_range():
    d = synthetic.ohlcv(8, 200, seed=4)
    w = O.run("willr", d, period=14)[0][:, 13:]
    assert np.all((w <= 0) & (w >= -100))


def test_window_nan_only_poisons_its_windows():
    x = (100 + np.cumsum(np.random.default_rng(0).normal(0, 1, 80))).astype(np.float32)[None, :]
    y = x.copy()
    y[0, 40] = np.nan
    a = O.run("sma", {"close": x}, period=5)[0]
    b = O.run("sma", {"close": y}, period=5)[0]
    assert np.all(np.isnan(b[0, 40:45]))
    np.testing.assert_array_equal(a[0, 45:], b[0, 45:])
    np.testing.assert_array_equal(a[0, :40], b[0, :40])


def test_leading_nan_delays_recurrences():
    x = (100 + np.cumsum(np.random.default_rng(1).normal(0, 1, 60))).astype(np.float32)
    y = np.concatenate([np.full(7, np.nan, np.float32), x])[None, :]
    for name, p in (("ema", dict(period=10)), ("rsi", dict(period=10)), ("macd", dict(fast=3, slow=6, signal=4))):
        a = O.run(name, {"close": x[None, :]}, **p)
        b = O.run(name, {"close": y}, **p)
        for u, v in zip(a, b):
            assert np.all(np.isnan(v[0, :7]))
            np.testing.assert_array_equal(u[0], v[0, 7:])


def test_roc_zero_divisor_and_float_order():
    # ROC.cu:18-20: 0 where the earlier bar is 0, float ((x - prev) / prev) * 100
    x = np.array([[0.0, 1.0, 2.0, 3.0, 0.5, np.nan, 7.0]], np.float32)
    got = O.run("roc", {"close": x}, period=2)[0][0]
    assert np.isnan(got[:2]).all()
    assert got[2] == 0.0
    exp = np.float32((np.float32(3.0) - np.float32(1.0)) / np.float32(1.0)) * np.float32(100.0)
    assert got[3] == exp
    assert got[4] == np.float32(np.float32(np.float32(0.5) - np.float32(2.0)) / np.float32(2.0)) * np.float32(100.0)
    assert np.isnan(got[5]) and got[6] == np.float32(np.float32(7.0 - 0.5) / np.float32(0.5)) * np.float32(100.0)


def test_price_transforms_known_answers():
    h = np.array([[3.0, 5.0, np.nan, 9.0]], np.float32)
    l = np.array([[1.0, 2.0, 4.0, 1.0]], np.float32)
    c = np.array([[2.0, 4.0, 4.0, 1.0]], np.float32)
    med = O.run("medprice", {"high": h, "low": l})[0][0]
    typ = O.run("typprice", {"high": h, "low": l, "close": c})[0][0]
    np.testing.assert_array_equal(med[[0, 1, 3]], [2.0, 3.5, 5.0])
    assert np.isnan(med[2]) and np.isnan(typ[2])
    assert typ[0] == 2.0 and typ[1] == np.float32(np.float32(11.0) / np.float32(3.0))
    # MIDPRICE: fmaxf/fminf skip the NaN high inside the window
    mid = O.run("midprice", {"high": h, "low": l}, period=2)[0][0]
    assert np.isnan(mid[0])
    np.testing.assert_array_equal(mid[1:], [3.0, 3.5, 5.0])


def test_rma_is_wilder_average():
    x = np.array([[np.nan, np.nan, 1.0, 2.0, 3.0, 4.0, 5.0]], np.float32)
    got = O.run("rma", {"close": x}, period=3)[0][0]
    assert np.isnan(got[:4]).all()
    assert got[4] == 2.0
    # fma(wBeta, 2, wAlpha * 4) with wBeta = 2/3: 8/3 up to the coefficients' rounding
    assert abs(got[5] - 8.0 / 3.0) < 1e-14


def test_ratio_momentum_and_price_known_answers():
    # ROCR.cu / ROCR100.cu / Momentum.cu / AvgPrice.cu / WclPrice.cu / MIDPOINT.cu
    f = np.float32
    x = np.array([[np.nan, 0.0, 4.0, 3.0, 6.0, 1.5]], np.float32)
    assert np.isnan(O.run("rocr", {"close": x}, period=1)[0][0, :2]).all()
    np.testing.assert_array_equal(O.run("rocr", {"close": x}, period=1)[0][0, 2:], [0.0, f(3.0) / f(4.0), 2.0, 0.25])
    np.testing.assert_array_equal(O.run("rocr100", {"close": x}, period=2)[0][0, 3:],
                                  [0.0, f(f(6.0) / f(4.0)) * f(100.0), f(f(1.5) / f(3.0)) * f(100.0)])
    mom = O.run("momentum", {"close": x}, period=2)[0][0]
    assert np.isnan(mom[:3]).all() and (mom[3:] == [3.0, 2.0, -1.5]).all()
    o = np.array([[1.0, 2.0]], np.float32)
    h = np.array([[4.0, 3.0]], np.float32)
    l = np.array([[0.5, 1.0]], np.float32)
    c = np.array([[2.5, 2.0]], np.float32)
    np.testing.assert_array_equal(O.run("avgprice", {"open": o, "high": h, "low": l, "close": c})[0][0], [2.0, 2.0])
    np.testing.assert_array_equal(O.run("wclprice", {"high": h, "low": l, "close": c})[0][0],
                                  [f(f(4.5) + f(5.0)) * f(0.25), 2.0])
    # MIDPOINT: leading NaN windows stay NaN, interior NaN is skipped by fmaxf/fminf
    y = np.array([[np.nan, np.nan, 1.0, 5.0, np.nan, 3.0]], np.float32)
    mp = O.run("midpoint", {"close": y}, period=2)[0][0]
    assert np.isnan(mp[:3]).all()
    np.testing.assert_array_equal(mp[3:], [3.0, 5.0, 3.0])


def test_rolling_strict_known_answers():
    # ClubPack.cu:375-407: any non-finite bar in the window gives NaN
    x = np.array([[1.0, 2.0, np.inf, 4.0, 5.0, 6.0]], np.float32)
    mean = O.run("rolling_mean", {"close": x}, period=2)[0][0]
    assert np.isnan(mean[[0, 2, 3]]).all()
    np.testing.assert_array_equal(mean[[1, 4, 5]], [1.5, 4.5, 5.5])
    np.testing.assert_array_equal(O.run("rolling_max", {"close": x}, period=2)[0][0, 4:], [5.0, 6.0])
    np.testing.assert_array_equal(O.run("rolling_min", {"close": x}, period=2)[0][0, 4:], [4.0, 5.0])
    std = O.run("rolling_std", {"close": x}, period=2)[0][0]
    np.testing.assert_array_equal(std[[1, 4, 5]], [0.5, 0.5, 0.5])
    np.testing.assert_array_equal(O.run("change", {"close": x}, period=1)[0][0, 4:], [1.0, 1.0])


# The reference's own TA-Lib 0.8.3 fixture for RMA(close, 14) on a 96-bar OHLC
# series (tests/fixtures/talib08_typed.json, checked by its Node binding test
# tests/node/talib08_typed.js:36). Read from the reference tree where it exists.
REF_TREE = Path(os.environ.get("TACUDA_REFERENCE_TREE", "/root/reference"))
RMA_FIXTURE = REF_TREE / "tests" / "fixtures" / "talib08_typed.json"


@pytest.mark.skipif(not RMA_FIXTURE.exists(), reason="reference tree not present")
def test_rma_matches_reference_talib_fixture():
    import json
    f = json.loads(RMA_FIXTURE.read_text())
    close = np.array([f["close"]], np.float64)
    assert np.array_equal(close.astype(np.float32).astype(np.float64), close)  # float32 values
    want = np.array([[np.nan if v is None else v for v in f["rma"]]])
    got = O.run("rma", {"close": close.astype(np.float32)}, period=14)[0]
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
    m = ~np.isnan(want)
    np.testing.assert_allclose(got[m], want[m], rtol=1e-14, atol=0)
