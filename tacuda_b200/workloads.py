"""Named job sets of the measured workloads (parameters as the reference's
fused-batch benchmark uses them: period 14 by default, 20 for the SMA and
BBANDS windows, MACD 12/26/9, STOCH 14/3/3; benchmarks/benchmark_batch_fused.py
and tests/python/batch_fused.py:24-29 in the reference).
"""
from __future__ import annotations

# (name, family, params, fparams, output names)
PASS13 = (
    ("sma", "sma", (20,), (), ("sma",)),
    ("ema", "ema", (14,), (), ("ema",)),
    ("wma", "wma", (14,), (), ("wma",)),
    ("rsi", "rsi", (14,), (), ("rsi",)),
    ("macd", "macd", (12, 26, 9), (), ("macd", "macd_signal", "macd_hist")),
    ("atr", "atr", (14,), (), ("atr",)),
    ("adx", "adx", (14,), (), ("adx",)),
    ("bbands", "bbands", (20,), (2.0, 2.0), ("bb_upper", "bb_middle", "bb_lower")),
    ("stoch", "stoch", (14, 3), (), ("stoch_k", "stoch_d")),
    ("cci", "cci", (14,), (), ("cci",)),
    ("obv", "obv", (), (), ("obv",)),
    ("mfi", "mfi", (14,), (), ("mfi",)),
    ("willr", "willr", (14,), (), ("willr",)),
)

PASS13_OUTPUTS = tuple(o for spec in PASS13 for o in spec[4])  # 18 planes

# oracle parameter names per family (oracle/oracle.py FAMILIES)
ORACLE_PARAMS = {
    "sma": lambda p, f: dict(period=p[0]),
    "ema": lambda p, f: dict(period=p[0]),
    "wma": lambda p, f: dict(period=p[0]),
    "rsi": lambda p, f: dict(period=p[0]),
    "macd": lambda p, f: dict(fast=p[0], slow=p[1], signal=p[2]),
    "atr": lambda p, f: dict(period=p[0]),
    "natr": lambda p, f: dict(period=p[0]),
    "trange": lambda p, f: dict(),
    "adx": lambda p, f: dict(period=p[0]),
    "dx": lambda p, f: dict(period=p[0]),
    "bbands": lambda p, f: dict(period=p[0], up=f[0], dn=f[1]),
    "stoch": lambda p, f: dict(k=p[0], d=p[1]),
    "cci": lambda p, f: dict(period=p[0]),
    "obv": lambda p, f: dict(),
    "ad": lambda p, f: dict(),
    "adosc": lambda p, f: dict(fast=p[0], slow=p[1]),
    "mfi": lambda p, f: dict(period=p[0]),
    "willr": lambda p, f: dict(period=p[0]),
    "sum": lambda p, f: dict(period=p[0]),
    "min": lambda p, f: dict(period=p[0]),
    "max": lambda p, f: dict(period=p[0]),
    "stddev": lambda p, f: dict(period=p[0], nbdev=(f[0] if f else 1.0)),
    "var": lambda p, f: dict(period=p[0]),
    "linearreg": lambda p, f: dict(period=p[0]),
    "correl": lambda p, f: dict(period=p[0]),
    "dema": lambda p, f: dict(period=p[0]),
    "tema": lambda p, f: dict(period=p[0]),
    "t3": lambda p, f: dict(period=p[0], vfactor=f[0]),
}

# bytes per series-bar of the 13-indicator pass when fused: inputs high, low,
# close, volume (16 B) + 18 float outputs (72 B)
PASS13_FUSED_BYTES_PER_BAR = 16 + 4 * len(PASS13_OUTPUTS)
# the same pass as 13 separate launches, each re-reading its own inputs
PASS13_PLAIN_BYTES_PER_BAR = 4 * (1 + 1 + 1 + 1 + 1 + 3 + 3 + 1 + 3 + 3 + 2 + 4 + 3) + 4 * len(PASS13_OUTPUTS)
