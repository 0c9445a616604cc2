"""Thin torch layer over the C ABI: device tensors in, device tensors out, on
the current CUDA stream. The compute is the library's kernels; torch only
supplies memory and the stream.

`alpha_indicators(close, alpha, ...)` is differentiable: its backward is the
library's hand-written adjoint (ct_b200_alpha_backward_d), which reads the
checkpoints the forward kernel wrote (the recurrence state every 256 bars)
instead of keeping per-bar state.
"""
from __future__ import annotations

import ctypes as ct

import torch

from . import call_status, ctB200AlphaParams, get_lib

ALPHA_OUTPUTS = ("ema", "macd", "signal", "hist", "rsi")


def _ptr(t):
    return ct.c_void_p(t.data_ptr()) if t is not None else ct.c_void_p(0)


def _stream():
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def _params(ema_period, fast, slow, signal, rsi_period):
    return ctB200AlphaParams(ema_period, fast, slow, signal, rsi_period)


def _check(close, alpha):
    if close.device.type != "cuda" or alpha.device.type != "cuda":
        raise ValueError("close and alpha must be CUDA tensors")
    if close.dtype != torch.float32 or alpha.dtype != torch.float32:
        raise TypeError("close and alpha must be float32")
    if close.dim() != 2 or alpha.dim() != 1 or alpha.shape[0] != close.shape[0]:
        raise ValueError("close must be (numSeries, seriesLen) and alpha (numSeries,)")


def alpha_forward(close, alpha, ema_period=14, fast=12, slow=26, signal=9, rsi_period=14):
    """Forward pass: returns (ema, macd, signal, hist, rsi, checkpoints)."""
    _check(close, alpha)
    close = close.contiguous()
    alpha = alpha.contiguous()
    S, T = close.shape
    outs = [torch.empty_like(close) for _ in ALPHA_OUTPUTS]
    nck = int(get_lib().ct_b200_alpha_checkpoint_doubles(T))
    ckpt = torch.empty((S, nck), dtype=torch.float64, device=close.device)
    p = _params(ema_period, fast, slow, signal, rsi_period)
    rc = get_lib().ct_b200_alpha_forward_d(_ptr(close), _ptr(alpha), T, S, ct.byref(p), *(_ptr(o) for o in outs),
                                           _ptr(ckpt), _stream())
    call_status(rc, "ct_b200_alpha_forward_d")
    return (*outs, ckpt)


def alpha_backward(close, alpha, ckpt, weights, ema_period=14, fast=12, slow=26, signal=9, rsi_period=14):
    """Adjoint: weights is a 5-sequence of (numSeries, seriesLen) tensors or
    None (dL/d each output); returns (dL/dclose, dL/dalpha)."""
    _check(close, alpha)
    S, T = close.shape
    ws = [None if w is None else w.to(torch.float32).contiguous() for w in weights]
    dx = torch.empty_like(close)
    da = torch.empty_like(alpha)
    p = _params(ema_period, fast, slow, signal, rsi_period)
    rc = get_lib().ct_b200_alpha_backward_d(_ptr(close.contiguous()), _ptr(alpha.contiguous()), T, S, ct.byref(p),
                                            _ptr(ckpt), *(_ptr(w) for w in ws), _ptr(dx), _ptr(da), _stream())
    call_status(rc, "ct_b200_alpha_backward_d")
    return dx, da


class AlphaIndicators(torch.autograd.Function):
    """EMA, MACD (line, signal, histogram) and RSI with a per-series alpha."""

    @staticmethod
    def forward(ctx, close, alpha, ema_period, fast, slow, signal, rsi_period):
        *outs, ckpt = alpha_forward(close, alpha, ema_period, fast, slow, signal, rsi_period)
        ctx.save_for_backward(close, alpha, ckpt)
        ctx.periods = (ema_period, fast, slow, signal, rsi_period)
        return tuple(outs)

    @staticmethod
    def backward(ctx, *grads):
        # warm-up bars are NaN in the forward and carry no gradient
        close, alpha, ckpt = ctx.saved_tensors
        ws = [None if g is None else torch.nan_to_num(g, nan=0.0) for g in grads]
        dx, da = alpha_backward(close, alpha, ckpt, ws, *ctx.periods)
        return dx, da, None, None, None, None, None


def alpha_indicators(close, alpha, ema_period=14, fast=12, slow=26, signal=9, rsi_period=14):
    """Differentiable (ema, macd, signal, hist, rsi) of close (S, T) with a
    smoothing coefficient alpha (S,) per series; float32 CUDA tensors."""
    return AlphaIndicators.apply(close, alpha, ema_period, fast, slow, signal, rsi_period)
