"""Test infrastructure only: FP64 reference for the per-series-alpha EMA / MACD
/ RSI and their gradients.

The forward is the TA-Lib recurrence structure written out bar by bar in torch
float64 (vectorised across series), so torch autograd through it is the
"unrolled recurrence" reference gradient; `finite_difference` gives FP64
central differences of the same forward. With alpha = 2/(p+1) (EMA, MACD fast
line) and 1/p (RSI) the forward reduces to talib08's TA_EMA / TA_MACD /
TA_RSI (src/compat/talib08_formulas.inc:5546-5627, 9316-9505, 13996-14115),
which tests/test_alpha.py checks against the pinned oracle. Finite inputs only.
"""
from __future__ import annotations

import numpy as np
import torch


def talib_coeffs(p: int) -> tuple[float, float]:
    """TA_EMA's coefficients for period p: (beta, k)."""
    b = (p - 1) / (p + 1)
    k = 1.0 - b
    if b < 0.5:
        b = 1.0 - k
    return b, k


def _ema_stage(x, p, start, beta, k, T):
    """One TA-Lib EMA stage over columns t of x (S, T): inputs counted from
    `start`, summed, mean of the first p at count start+p-1, then
    beta*y + k*x. Returns a list of per-bar tensors (S,)."""
    S = x.shape[0]
    y = torch.zeros(S, dtype=x.dtype)
    out = []
    for t in range(T):
        r = t - start
        if r < 0:
            pass
        elif p == 1:
            y = x[:, t]
        elif r < p - 1:
            y = y + x[:, t]
        elif r == p - 1:
            y = (y + x[:, t]) / p
        else:
            y = beta * y + k * x[:, t]
        out.append(y)
    return out


def forward(close, alpha, ema_period=14, fast=12, slow=26, signal=9, rsi_period=14):
    """close (S, T) and alpha (S,) as float64 tensors. Returns ema, macd,
    signal, hist, rsi as (S, T) float64 tensors, NaN in warm-up."""
    S, T = close.shape
    a = alpha
    b = 1.0 - a
    nan = torch.full((S,), float("nan"), dtype=close.dtype)
    ema = _ema_stage(close, ema_period, 0, b, a, T)
    bs, ks = talib_coeffs(slow)
    sl = _ema_stage(close, slow, 0, bs, ks, T)
    fa = _ema_stage(close, fast, slow - fast, b, a, T)
    m = [fa[t] - sl[t] if t >= slow - 1 else torch.zeros(S, dtype=close.dtype) for t in range(T)]
    bg, kg = talib_coeffs(signal)
    # the signal stage counts from slow-1
    g = torch.zeros(S, dtype=close.dtype)
    sig = []
    start, ready = slow - 1, slow + signal - 2
    for t in range(T):
        if t < start:
            pass
        elif t < ready:
            g = g + m[t]
        elif t == ready:
            g = (g + m[t]) / signal
        elif signal == 1:
            g = m[t]
        else:
            g = bg * g + kg * m[t]
        sig.append(g)
    # RSI with Wilder smoothing coefficient alpha
    inv = 1.0 / rsi_period
    gain = torch.zeros(S, dtype=close.dtype)
    loss = torch.zeros(S, dtype=close.dtype)
    rsi = []
    for t in range(T):
        if t >= 1:
            d = close[:, t] - close[:, t - 1]
            u = torch.clamp(d, min=0.0)
            v = torch.clamp(-d, min=0.0)
            if t < rsi_period:
                gain, loss = gain + u, loss + v
            elif t == rsi_period:
                gain, loss = (gain + u) * inv, (loss + v) * inv
            else:
                gain, loss = b * gain + a * u, b * loss + a * v
        if t >= rsi_period:
            tot = gain + loss
            safe = torch.where(tot > 0, tot, torch.ones_like(tot))
            rsi.append(torch.where(tot > 0, 100.0 * gain / safe, torch.full_like(tot, 50.0)))
        else:
            rsi.append(nan)
    ema_o = torch.stack([ema[t] if t >= ema_period - 1 else nan for t in range(T)], 1)
    ok = [t >= ready for t in range(T)]
    macd_o = torch.stack([m[t] if ok[t] else nan for t in range(T)], 1)
    sig_o = torch.stack([sig[t] if ok[t] else nan for t in range(T)], 1)
    hist_o = torch.stack([m[t] - sig[t] if ok[t] else nan for t in range(T)], 1)
    return ema_o, macd_o, sig_o, hist_o, torch.stack(rsi, 1)


def loss_of(outs, weights):
    """Weighted sum of the outputs over their non-warm-up bars."""
    total = 0.0
    for o, w in zip(outs, weights):
        if w is None:
            continue
        total = total + torch.where(torch.isnan(o), torch.zeros_like(o), o * w).sum()
    return total


def gradients(close, alpha, weights, **params):
    """Unrolled-recurrence autograd reference: dL/dclose (S, T), dL/dalpha (S,)."""
    c = torch.as_tensor(close, dtype=torch.float64).clone().requires_grad_(True)
    a = torch.as_tensor(alpha, dtype=torch.float64).clone().requires_grad_(True)
    w = [None if x is None else torch.as_tensor(x, dtype=torch.float64) for x in weights]
    L = loss_of(forward(c, a, **params), w)
    gc, ga = torch.autograd.grad(L, (c, a))
    return gc.numpy(), ga.numpy()


def finite_difference(close, alpha, weights, which, h=1e-6, **params):
    """FP64 central differences of L with respect to the listed entries:
    which = [("alpha", s) | ("close", s, t), ...]."""
    c0 = torch.as_tensor(close, dtype=torch.float64)
    a0 = torch.as_tensor(alpha, dtype=torch.float64)
    w = [None if x is None else torch.as_tensor(x, dtype=torch.float64) for x in weights]
    res = []
    for item in which:
        vals = []
        for sgn in (1.0, -1.0):
            c, a = c0.clone(), a0.clone()
            if item[0] == "alpha":
                a[item[1]] += sgn * h
            else:
                c[item[1], item[2]] += sgn * h
            with torch.no_grad():
                vals.append(float(loss_of(forward(c, a, **params), w)))
        res.append((vals[0] - vals[1]) / (2 * h))
    return np.array(res)
