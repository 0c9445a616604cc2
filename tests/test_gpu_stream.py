"""Batch streams (the reference's include/tacuda_stream.h:155-269): appends
of uneven chunk sizes continue every series' state, so their outputs equal one
batch call over the concatenated bars - checked against the FP64 oracle, and
against this library's own batch entry point, within the tolerance."""
import ctypes as ct

import numpy as np
import pytest
import torch

import tacuda_b200 as tb
from gpu_util import DEFAULTS, call_batch_d, device_planes, to_np
from oracle import oracle as O
from tacuda_b200 import synthetic
from tolerance import compare

pytestmark = pytest.mark.gpu

_P = ct.c_void_p
# family: (create args, inputs in append order, outputs)
FAMS = {
    "sma": ((20,), ["close"], 1), "ema": ((14,), ["close"], 1), "wma": ((14,), ["close"], 1),
    "rsi": ((14,), ["close"], 1), "atr": ((14,), ["high", "low", "close"], 1),
    "natr": ((14,), ["high", "low", "close"], 1), "obv": ((), ["close", "volume"], 1),
    "ad": ((), ["high", "low", "close", "volume"], 1), "macd": ((12, 26, 9), ["close"], 3),
    "bbands": ((20, 2.0, 2.0), ["close"], 3),
}
CHUNKS = [1, 5, 300, 17, 128, 700, 3, 256]


def _create(lib, name, args, S):
    h = _P()
    f = getattr(lib, f"ct_{name}_stream_batch_create")
    cargs = [ct.c_float(a) if isinstance(a, float) else ct.c_int(a) for a in args]
    rc = f(*cargs, ct.c_int(S), ct.byref(h))
    tb.call_status(rc, f"ct_{name}_stream_batch_create")
    return h


def _append(lib, name, h, data, t0, n, nout):
    S = next(iter(data.values())).shape[0]
    _, ins, _ = FAMS[name]
    chunk = [np.ascontiguousarray(data[k][:, t0:t0 + n]) for k in ins]
    outs = [np.full((S, n), 777.0, np.float32) for _ in range(nout)]
    args = [h] + [c.ctypes.data_as(_P) for c in chunk] + [ct.c_int(n)] + [o.ctypes.data_as(_P) for o in outs]
    rc = getattr(lib, f"ct_{name}_stream_batch_append")(*args)
    tb.call_status(rc, f"ct_{name}_stream_batch_append")
    return outs


@pytest.mark.parametrize("name", sorted(FAMS))
def test_appends_equal_one_batch_over_the_concatenation(name):
    lib = tb.get_lib()
    args, ins, nout = FAMS[name]
    S, T = 37, sum(CHUNKS)
    d = synthetic.ohlcv(S, T, seed=51)
    h = _create(lib, name, args, S)
    try:
        parts, t0 = [], 0
        for n in CHUNKS:
            parts.append(_append(lib, name, h, d, t0, n, nout))
            t0 += n
        bars = ct.c_longlong()
        assert lib.ct_stream_batch_bars(h, ct.byref(bars)) == 0 and bars.value == T
        got = [np.concatenate([p[i] for p in parts], axis=1) for i in range(nout)]
        params = DEFAULTS[name] if name != "bbands" else dict(period=20, up=2.0, dn=2.0)
        ref = O.run(name, d, **params)
        mine = to_np(call_batch_d(name, device_planes(d), params))
        for i in range(nout):
            compare(got[i], ref[i], f"stream {name}[{i}] vs oracle")
            compare(got[i], mine[i].astype(np.float64), f"stream {name}[{i}] vs batch")
    finally:
        lib.ct_stream_batch_destroy(h)


def test_reset_restarts_every_series_and_handles_are_checked():
    lib = tb.get_lib()
    S, T = 9, 600
    d = synthetic.ohlcv(S, T, seed=52)
    h = _create(lib, "macd", (12, 26, 9), S)
    try:
        first = _append(lib, "macd", h, d, 0, 400, 3)
        _append(lib, "macd", h, d, 400, 200, 3)
        assert lib.ct_stream_batch_reset(h) == 0
        again = _append(lib, "macd", h, d, 0, 400, 3)
        for a, b in zip(first, again):
            np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        lb, ns, no = ct.c_int(), ct.c_int(), ct.c_int()
        assert lib.ct_stream_batch_lookback(h, ct.byref(lb)) == 0 and lb.value == 26 + 9 - 2
        assert lib.ct_stream_batch_series(h, ct.byref(ns)) == 0 and ns.value == S
        assert lib.ct_stream_batch_outputs(h, ct.byref(no)) == 0 and no.value == 3
        assert lib.ct_stream_batch_set_exec(h, ct.c_int(2)) == 0
        assert lib.ct_stream_batch_set_exec(h, ct.c_int(1)) != 0  # CPU execution is not offered
        x = np.zeros((S, 1), np.float32)
        o = [np.zeros((S, 1), np.float32) for _ in range(3)]
        rc = lib.ct_macd_stream_batch_append(h, x.ctypes.data_as(_P), ct.c_int(0), *(v.ctypes.data_as(_P) for v in o))
        assert rc == 4 and "n must be > 0" in tb.get_last_error()
        rc = lib.ct_sma_stream_batch_append(h, x.ctypes.data_as(_P), ct.c_int(1), o[0].ctypes.data_as(_P))
        assert rc == 4 and "different indicator" in tb.get_last_error()
    finally:
        assert lib.ct_stream_batch_destroy(h) == 0
    lb = ct.c_int()
    assert lib.ct_stream_batch_lookback(h, ct.byref(lb)) == 4  # destroyed handle
