"""GPU: a bounded wait that runs out is reported, on every stream, and the
context stays usable (the reference reports a failed synchronisation as a
failed call, src/api/api_batch.cu:327-337).

TACUDA_B200_TEST_STALL=1 makes one wait of a launch run out on purpose: the
row-parallel engine's producer never announces its first chunk (its job warps
give up after 1 ms), the look-back engine never takes its first tile (the
tiles waiting for it give up after 64 polls). No GPU fault: the kernels return
with the device's error word set."""
from __future__ import annotations

import ctypes as ct
import os

import pytest
import torch

import tacuda_b200 as tb
from gpu_util import DEFAULTS, call_batch_d, device_planes, to_np
from oracle import oracle as O
from tacuda_b200 import synthetic
from tolerance import compare

pytestmark = pytest.mark.gpu

KERNEL_FAILED = 3


def _status(name, dp, stream=0):
    """ct_<name>_batch_d without raising; returns the status code."""
    try:
        call_batch_d(name, dp, DEFAULTS[name], stream=stream)
    except RuntimeError as e:
        return int(str(e).split("code ")[1].split(" ")[0])
    return 0


@pytest.fixture
def stall():
    os.environ["TACUDA_B200_TEST_STALL"] = "1"
    yield
    os.environ.pop("TACUDA_B200_TEST_STALL", None)


@pytest.mark.parametrize("mode,shape", [("sp", (64, 234)), ("lb", (2, 8192))])
def test_stream_zero_call_reports_the_timeout(mode, shape):
    d = synthetic.ohlcv(*shape, seed=3)
    dp = device_planes(d)
    os.environ["TACUDA_B200_MODE"] = mode
    try:
        assert tb.take_device_error() == 0
        os.environ["TACUDA_B200_TEST_STALL"] = "1"
        try:
            rc = _status("ema", dp)
        finally:
            os.environ.pop("TACUDA_B200_TEST_STALL", None)
        assert rc == KERNEL_FAILED
        assert "ran out" in tb.get_last_error()
        assert tb.take_device_error() == 0  # the synchronous call consumed it
        # the context is usable and the next call is correct
        got = to_np(call_batch_d("ema", dp, DEFAULTS["ema"]))[0]
        compare(got, O.run("ema", d, **DEFAULTS["ema"])[0], f"ema after timeout [{mode}]")
    finally:
        del os.environ["TACUDA_B200_MODE"]


@pytest.mark.parametrize("mode,shape", [("sp", (64, 234)), ("lb", (2, 8192))])
def test_user_stream_timeout_is_observable(mode, shape, stall):
    dp = device_planes(synthetic.ohlcv(*shape, seed=4))
    os.environ["TACUDA_B200_MODE"] = mode
    try:
        s = torch.cuda.Stream()
        assert _status("ema", dp, stream=s.cuda_stream) == 0  # asynchronous: launched fine
        s.synchronize()
        assert tb.take_device_error() == 1
        assert tb.take_device_error() == 0
    finally:
        del os.environ["TACUDA_B200_MODE"]


def test_static_entry_reports_the_timeout(stall):
    S, T = 2, 8192
    dp = device_planes(synthetic.ohlcv(S, T, seed=5))
    out = torch.empty((S, T), device="cuda")
    job = tb.make_job("ema", (14,), (), [out.data_ptr()])
    series = tb.make_series({"close": dp["close"].data_ptr()}, S, T)
    rc = tb.get_lib().ct_b200_fused_lookback_static_d(ct.byref(series), tb.job_array([job]), 1, None)
    assert rc == KERNEL_FAILED
    assert tb.take_device_error() == 0
