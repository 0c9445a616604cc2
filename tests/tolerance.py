"""Parity criteria shared by the tests.

Float outputs: NaN positions must match exactly; finite values must satisfy
|gpu - ref| <= 1e-5 * |ref| + 1e-6 * max|ref of the row|, i.e. 1e-5 relative,
with values near zero judged against the row's own scale at 1e-6 (oscillators
and MACD lines cross zero, where a pure relative bound is undefined).
Candle signals and every integer output must be bit-exact.
"""
from __future__ import annotations

import numpy as np

RTOL = 1e-5
ROW_ATOL = 1e-6


def compare(got, ref, name: str, rtol: float = RTOL, row_atol: float = ROW_ATOL):
    """Return (max scaled error, float32 bit differences); raise on failure."""
    g = np.asarray(got, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    assert g.shape == r.shape, f"{name}: shape {g.shape} vs {r.shape}"
    ng, nr = np.isnan(g), np.isnan(r)
    if not np.array_equal(ng, nr):
        idx = np.argwhere(ng != nr)[0]
        raise AssertionError(f"{name}: NaN positions differ first at {tuple(idx)} (gpu {g[tuple(idx)]}, ref {r[tuple(idx)]})")
    m = ~nr
    if not m.any():
        return 0.0, 0
    absr = np.where(m, np.abs(r), 0.0)
    scale = absr.max(axis=-1, keepdims=True) if r.ndim > 1 else absr.max()
    tol = rtol * np.abs(r) + row_atol * np.broadcast_to(scale, r.shape)
    err = np.abs(g - r)
    bad = m & (err > tol)
    if bad.any():
        idx = tuple(np.argwhere(bad)[0])
        raise AssertionError(f"{name}: {int(bad.sum())} values off, first at {idx}: gpu {g[idx]!r} ref {r[idx]!r}")
    scaled = np.where(m, err / np.maximum(tol, 1e-300), 0.0)
    bits = int(np.count_nonzero(g[m].astype(np.float32).view(np.uint32) != r[m].astype(np.float32).view(np.uint32)))
    return float(scaled.max()), bits


def compare_ragged(got, ref, offsets, name: str, rtol: float = RTOL, row_atol: float = ROW_ATOL):
    """compare() for a ragged batch stored flat: the near-zero allowance uses
    each row's own max |ref| (rows given by offsets[s]..offsets[s+1])."""
    g = np.asarray(got, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    off = np.asarray(offsets, dtype=np.int64)
    assert g.shape == r.shape, f"{name}: shape {g.shape} vs {r.shape}"
    ng, nr = np.isnan(g), np.isnan(r)
    if not np.array_equal(ng, nr):
        idx = int(np.argwhere(ng != nr)[0][0])
        raise AssertionError(f"{name}: NaN positions differ first at {idx} (gpu {g[idx]}, ref {r[idx]})")
    m = ~nr
    if not m.any():
        return 0.0, 0
    absr = np.where(m, np.abs(r), 0.0)
    lens = np.diff(off)
    keep = lens > 0
    starts = off[:-1][keep]
    row_max = np.maximum.reduceat(absr, starts) if len(starts) else np.zeros(0)
    scale = np.repeat(row_max, lens[keep])
    tol = rtol * np.abs(r) + row_atol * scale
    err = np.abs(g - r)
    bad = m & (err > tol)
    if bad.any():
        idx = int(np.argwhere(bad)[0][0])
        row = int(np.searchsorted(off, idx, side="right") - 1)
        raise AssertionError(f"{name}: {int(bad.sum())} values off, first at {idx} (row {row}): "
                             f"gpu {g[idx]!r} ref {r[idx]!r}")
    scaled = np.where(m, err / np.maximum(tol, 1e-300), 0.0)
    bits = int(np.count_nonzero(g[m].astype(np.float32).view(np.uint32) != r[m].astype(np.float32).view(np.uint32)))
    return float(scaled.max()), bits
