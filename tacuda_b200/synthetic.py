"""Seeded synthetic market data with the shapes and distributions of the
workloads this library is measured on (no public dataset is involved).

* ``ohlcv(S, T, seed)``: per-series close as a geometric random walk from 100
  with log-return sigma drawn from U(0.005, 0.03); open = previous close;
  high = max(open, close) * (1 + |N(0, 0.004^2)|); low = min(open, close) *
  (1 - |N(0, 0.004^2)|); volume ~ lognormal(10, 1). float32 planes (S, T).
* ``ragged_lengths(S, lo, hi, seed)``: lengths log-uniform in [lo, hi].
* ``single_close(T, seed)``: one geometric random walk from 100 with
  log-returns N(0, 0.01^2), float64 (callers cast to float32).
* ``level_walk(S, T, seed)``: additive random walk with sigma 0.01 around a
  +1e4 level (a cancellation stress for window moments), float32.
"""
from __future__ import annotations

import numpy as np


def ohlcv(S: int, T: int, seed: int = 2024, close0: float = 100.0) -> dict:
    rng = np.random.default_rng(seed)
    sigma = rng.uniform(0.005, 0.03, size=(S, 1))
    r = rng.standard_normal((S, T)) * sigma
    close = close0 * np.exp(np.cumsum(r, axis=1))
    opn = np.empty_like(close)
    opn[:, 0] = close0
    opn[:, 1:] = close[:, :-1]
    hi = np.maximum(opn, close) * (1.0 + np.abs(rng.normal(0.0, 0.004, (S, T))))
    lo = np.minimum(opn, close) * (1.0 - np.abs(rng.normal(0.0, 0.004, (S, T))))
    vol = rng.lognormal(10.0, 1.0, (S, T))
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return {"open": f(opn), "high": f(hi), "low": f(lo), "close": f(close), "volume": f(vol)}


def ragged_lengths(S: int, lo: int = 50, hi: int = 20000, seed: int = 7) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), S))).astype(np.int64)


def offsets_of(lengths) -> np.ndarray:
    off = np.zeros(len(lengths) + 1, dtype=np.int64)
    np.cumsum(np.asarray(lengths, dtype=np.int64), out=off[1:])
    return off


def ragged_ohlcv(lengths, seed: int = 2024) -> tuple[dict, np.ndarray]:
    """Flat planes for rows of the given lengths (generated as one long matrix
    row by row so each row follows the ``ohlcv`` distribution)."""
    off = offsets_of(lengths)
    total = int(off[-1])
    planes = {k: np.empty(total, dtype=np.float32) for k in ("open", "high", "low", "close", "volume")}
    rng = np.random.default_rng(seed)
    chunk = 512
    for s0 in range(0, len(lengths), chunk):
        s1 = min(len(lengths), s0 + chunk)
        Tm = int(max(lengths[s0:s1]))
        d = ohlcv(s1 - s0, Tm, seed=int(rng.integers(1 << 31)))
        for s in range(s0, s1):
            n = int(lengths[s])
            for k in planes:
                planes[k][off[s]:off[s] + n] = d[k][s - s0, :n]
    return planes, off


def single_close(T: int = 100_000, seed: int = 11) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return 100.0 * np.exp(np.cumsum(rng.normal(0.0, 0.01, T)))


def level_walk(S: int, T: int, seed: int = 5, level: float = 1e4, sigma: float = 0.01) -> np.ndarray:
    out = np.empty((S, T), dtype=np.float32)
    rng = np.random.default_rng(seed)
    block = 1 << 22
    for s in range(S):
        acc = 0.0
        for t0 in range(0, T, block):
            t1 = min(T, t0 + block)
            steps = np.cumsum(rng.normal(0.0, sigma, t1 - t0)) + acc
            acc = float(steps[-1])
            out[s, t0:t1] = (level + steps).astype(np.float32)
    return out
