"""Per-series-alpha EMA / MACD / RSI and the hand-written adjoint.

CPU: the FP64 reference reduces to the pinned TA-Lib oracle at TA-Lib's
coefficients, its autograd gradient agrees with FP64 central differences, and
the C entry points validate their arguments. GPU: forward against the FP64
reference, the adjoint against the unrolled-recurrence autograd gradient and
against central differences (h = 1e-6), through the C ABI and through the
torch autograd.Function."""
import ctypes as ct

import numpy as np
import pytest
import torch

import tacuda_b200 as tb
from oracle import alpha_oracle as A
from oracle import oracle as O
from tacuda_b200 import synthetic
from tolerance import compare

PARAMS = dict(ema_period=14, fast=12, slow=26, signal=9, rsi_period=14)


def _data(S, T, seed):
    d = synthetic.ohlcv(S, T, seed=seed)
    rng = np.random.default_rng(seed + 1)
    alpha = rng.uniform(0.01, 0.5, S).astype(np.float32)
    w = [rng.standard_normal((S, T)).astype(np.float32) for _ in range(5)]
    return d["close"], alpha, w


def grad_close(g, r, label):
    """Gradient tolerance: |g - r| <= 1e-4*|r| + 1e-5*max|r| (float32 results
    of an FP64 adjoint against the FP64 autograd reference)."""
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    tol = 1e-4 * np.abs(r) + 1e-5 * np.max(np.abs(r))
    bad = np.abs(g - r) > tol
    assert not bad.any(), f"{label}: {bad.sum()} entries off, worst {np.max(np.abs(g - r) - tol)}"


def test_reference_reduces_to_talib_at_talib_coefficients():
    d = synthetic.ohlcv(5, 400, seed=3)
    c = torch.tensor(d["close"], dtype=torch.float64)
    S = c.shape[0]
    ema = A.forward(c, torch.full((S,), 2.0 / 15, dtype=torch.float64), **PARAMS)[0].numpy()
    compare(ema.astype(np.float32), O.run("ema", d, period=14)[0], "alpha EMA at 2/(p+1)")
    outs = A.forward(c, torch.full((S,), 2.0 / 13, dtype=torch.float64), **PARAMS)
    for o, r in zip(outs[1:4], O.run("macd", d, fast=12, slow=26, signal=9)):
        compare(o.numpy().astype(np.float32), r, "alpha MACD at 2/(fast+1)")
    rsi = A.forward(c, torch.full((S,), 1.0 / 14, dtype=torch.float64), **PARAMS)[4].numpy()
    compare(rsi.astype(np.float32), O.run("rsi", d, period=14)[0], "alpha RSI at 1/p")


def test_reference_gradient_matches_central_differences():
    close, alpha, w = _data(3, 320, seed=5)
    gc, ga = A.gradients(close, alpha, w, **PARAMS)
    which = [("alpha", 0), ("alpha", 2), ("close", 1, 0), ("close", 1, 40), ("close", 2, 319)]
    fd = A.finite_difference(close, alpha, w, which, **PARAMS)
    got = np.array([ga[0], ga[2], gc[1, 0], gc[1, 40], gc[2, 319]])
    np.testing.assert_allclose(got, fd, rtol=1e-5, atol=1e-6 * np.max(np.abs(fd)))


def test_entry_points_validate_arguments():
    lib = tb.get_lib()
    p = tb.ctB200AlphaParams(14, 12, 26, 9, 14)
    fake = ct.c_void_p(16)
    rc = lib.ct_b200_alpha_forward_d(None, fake, 10, 1, ct.byref(p), None, None, None, None, None, fake, None)
    assert rc == 4 and "null pointer" in tb.get_last_error()
    bad = tb.ctB200AlphaParams(14, 30, 26, 9, 14)  # fast > slow
    rc = lib.ct_b200_alpha_forward_d(fake, fake, 10, 1, ct.byref(bad), None, None, None, None, None, fake, None)
    assert rc == 4 and "invalid periods" in tb.get_last_error()
    rc = lib.ct_b200_alpha_backward_d(fake, fake, 10, 1, ct.byref(p), fake, None, None, None, None, None, None,
                                      fake, None)
    assert rc == 4
    assert lib.ct_b200_alpha_checkpoint_doubles(256) == 6
    assert lib.ct_b200_alpha_checkpoint_doubles(257) == 12


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(1, 30), (16, 700), (5, 2048), (3, 10000)])
def test_forward_matches_reference(shape):
    from tacuda_b200 import torch_api as TA
    close, alpha, _ = _data(*shape, seed=11)
    outs = TA.alpha_forward(torch.from_numpy(close).cuda(), torch.from_numpy(alpha).cuda(), **PARAMS)
    ref = A.forward(torch.tensor(close, dtype=torch.float64), torch.tensor(alpha, dtype=torch.float64), **PARAMS)
    for name, g, r in zip(TA.ALPHA_OUTPUTS, outs[:5], ref):
        compare(g.cpu().numpy(), r.numpy(), f"alpha forward {name} {shape}")


@pytest.mark.gpu
def test_forward_at_talib_coefficients_matches_talib_oracle():
    from tacuda_b200 import torch_api as TA
    d = synthetic.ohlcv(9, 500, seed=13)
    c = torch.from_numpy(d["close"]).cuda()
    a = torch.full((9,), 2.0 / 15, device="cuda")
    ema = TA.alpha_forward(c, a, **PARAMS)[0].cpu().numpy()
    compare(ema, O.run("ema", d, period=14)[0], "gpu alpha EMA at 2/(p+1)")


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(3, 40), (8, 600), (4, 2048), (2, 10000), (37, 300)])
def test_adjoint_matches_unrolled_autograd(shape):
    from tacuda_b200 import torch_api as TA
    close, alpha, w = _data(*shape, seed=17)
    c, a = torch.from_numpy(close).cuda(), torch.from_numpy(alpha).cuda()
    *_, ck = TA.alpha_forward(c, a, **PARAMS)
    ws = [torch.from_numpy(x).cuda() for x in w]
    dx, da = TA.alpha_backward(c, a, ck, ws, **PARAMS)
    dx2, da2 = TA.alpha_backward(c, a, ck, ws, **PARAMS)
    assert torch.equal(dx, dx2) and torch.equal(da, da2)
    gc, ga = A.gradients(close, alpha, w, **PARAMS)
    grad_close(dx.cpu().numpy(), gc, f"dL/dclose {shape}")
    grad_close(da.cpu().numpy(), ga, f"dL/dalpha {shape}")


@pytest.mark.gpu
def test_adjoint_matches_central_differences():
    from tacuda_b200 import torch_api as TA
    close, alpha, w = _data(4, 530, seed=19)
    c, a = torch.from_numpy(close).cuda(), torch.from_numpy(alpha).cuda()
    *_, ck = TA.alpha_forward(c, a, **PARAMS)
    dx, da = TA.alpha_backward(c, a, ck, [torch.from_numpy(x).cuda() for x in w], **PARAMS)
    which = [("alpha", 0), ("alpha", 3), ("close", 0, 5), ("close", 2, 255), ("close", 2, 256), ("close", 3, 529)]
    fd = A.finite_difference(close.astype(np.float64), alpha.astype(np.float64), w, which, **PARAMS)
    dx, da = dx.cpu().numpy(), da.cpu().numpy()
    got = np.array([da[0], da[3], dx[0, 5], dx[2, 255], dx[2, 256], dx[3, 529]])
    np.testing.assert_allclose(got, fd, rtol=1e-4, atol=1e-5 * np.max(np.abs(fd)))


@pytest.mark.gpu
def test_autograd_function_uses_the_adjoint():
    from tacuda_b200 import torch_api as TA
    close, alpha, w = _data(6, 400, seed=23)
    c = torch.from_numpy(close).cuda().requires_grad_(True)
    a = torch.from_numpy(alpha).cuda().requires_grad_(True)
    outs = TA.alpha_indicators(c, a, **PARAMS)
    ws = [torch.from_numpy(x).cuda() for x in w]
    L = sum(torch.nansum(o * x) for o, x in zip(outs, ws))
    gc, ga = torch.autograd.grad(L, (c, a))
    rc, ra = A.gradients(close, alpha, w, **PARAMS)
    grad_close(gc.cpu().numpy(), rc, "autograd dL/dclose")
    grad_close(ga.cpu().numpy(), ra, "autograd dL/dalpha")
