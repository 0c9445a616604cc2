"""Generate the golden fixtures in this directory from the reference's own CPU
code (oracle/_ref/libtaref.so: the vendored TA-Lib 0.8.3 C, StreamStates.h and
CandleUtils.h compiled from the reference tree by oracle/Makefile).

    python tests/golden/make_golden.py

Writes golden_ref.npz: seeded OHLCV inputs (6 series x 160 bars, plus a flat
series and a series with a gap/doji-rich shape) and, per family and candle
pattern, the reference outputs. The fixtures pin the project's oracle and the
CUDA path without needing the reference tree at test time.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from tacuda_b200 import synthetic  # noqa: E402

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


def inputs():
    d = synthetic.ohlcv(6, 160, seed=31)
    # a flat row and a row with repeated prices (doji and equal-body cases)
    for k in d:
        d[k][4, :] = 100.0 if k != "volume" else 1000.0
    rng = np.random.default_rng(5)
    base = np.round(100 + np.cumsum(rng.integers(-2, 3, 160)) * 0.5, 1).astype(np.float32)
    d["open"][5] = base
    d["close"][5] = np.roll(base, -1)
    d["high"][5] = np.maximum(d["open"][5], d["close"][5]) + np.float32(0.5)
    d["low"][5] = np.minimum(d["open"][5], d["close"][5]) - np.float32(0.5)
    return d


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libtaref.so missing: build it with `make -C oracle` where the reference tree exists")
    d = inputs()
    out = {f"in_{k}": v for k, v in d.items()}
    for name, p in CASES.items():
        res = O.ref_run(name, d, **p)
        for i, r in enumerate(res):
            out[f"{name}_{i}"] = np.asarray(r)
    for k in range(63):
        out[f"cdl_{k}"] = O.ref_cdl(k, d["open"], d["high"], d["low"], d["close"])
    np.savez_compressed(Path(__file__).with_name("golden_ref.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
