"""GPU: the allocation-free look-back entry point (static device scratch)
against the look-back engine of the regular fused entry point, whose scratch
comes from the stream-ordered pool, and against the FP64 oracle. Kept in its own file, collected last, so
it also runs after every other test has used the library."""
import ctypes as ct
import os

import numpy as np
import pytest
import torch

import tacuda_b200 as tb
from oracle import oracle as O
from tacuda_b200 import synthetic, workloads
from tolerance import compare

pytestmark = pytest.mark.gpu


def _entry():
    f = tb.get_lib().ct_b200_fused_lookback_static_d
    f.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]
    f.restype = ct.c_int
    return f


def _jobs(S, T, seed, extra):
    """The 13-indicator pass, plus (extra) two appended families (QSTICK, RMA),
    which run on the look-back engine's second set of kernels."""
    d = synthetic.ohlcv(S, T, seed=seed)
    dp = {k: torch.from_numpy(v).cuda() for k, v in d.items()}
    spec = [(fam, p, fp, on) for _, fam, p, fp, on in workloads.PASS13]
    if extra:
        spec += [("qstick", (10,), (), ("qstick",)), ("rma", (14,), (), ("rma",))]
    names = [n for *_, on in spec for n in on]
    outs = {n: torch.full((S, T), 777.0, device="cuda") for n in names}
    jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for fam, p, fp, on in spec]
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items() if k in tb.PLANE_ID}, S, T)
    return d, outs, jobs, series, spec


@pytest.mark.parametrize("on_stream", [False, True], ids=["null-stream", "user-stream"])
@pytest.mark.parametrize("extra", [False, True], ids=["pass13", "pass13+qstick+rma"])
@pytest.mark.parametrize("k", [4, 8, 16])
def test_static_scratch_matches_pool_scratch_twice(k, extra, on_stream, monkeypatch):
    """Two calls in a row of the static-scratch entry give the bits of the
    pool-scratch look-back launch, and both agree with the FP64 oracle."""
    S, T = 2, 40000
    d, outs, jobs, series, spec = _jobs(S, T, seed=31 + k, extra=extra)
    monkeypatch.setenv("TACUDA_B200_BARS_PER_LANE", str(k))
    monkeypatch.setenv("TACUDA_B200_MODE", "lb")
    tb.fused_batch_d(series, jobs, 0)
    monkeypatch.delenv("TACUDA_B200_MODE")
    torch.cuda.synchronize()
    ref = {n: v.cpu().numpy() for n, v in outs.items()}
    for fam, p, fp, on in spec:
        params = workloads.ORACLE_PARAMS[fam](p, fp) if fam in workloads.ORACLE_PARAMS else {"period": p[0]}
        for name, want in zip(on, O.run(fam, d, **params)):
            compare(ref[name], want, f"pool look-back {name}")
    arr = tb.job_array(jobs)
    f = _entry()
    stream = torch.cuda.Stream() if on_stream else None
    for call in range(2):
        for v in outs.values():
            v.fill_(777.0)
        torch.cuda.synchronize()
        rc = f(ct.addressof(series), ct.addressof(arr), len(jobs), stream.cuda_stream if stream else None)
        tb.call_status(rc, "ct_b200_fused_lookback_static_d")
        if stream is not None:
            stream.synchronize()
        torch.cuda.synchronize()
        for name, v in outs.items():
            got = v.cpu().numpy()
            assert np.array_equal(got.view(np.uint32), ref[name].view(np.uint32)), f"static call {call} {name}"
    assert tb.take_device_error() == 0


def test_static_scratch_rejects_oversized_batch():
    # 16000 rows x 4096 bars: far more descriptors than the 8 MiB array holds
    # (real buffers, although the host rejects the batch before any launch)
    S, T = 16000, 4096
    x = torch.zeros((S, T), device="cuda")
    y = torch.empty_like(x)
    jobs = [tb.make_job("ema", (14,), (), [y.data_ptr()])]
    series = tb.make_series({"close": x.data_ptr()}, S, T)
    arr = tb.job_array(jobs)
    rc = _entry()(ct.addressof(series), ct.addressof(arr), 1, None)
    assert rc == 4  # CT_STATUS_INVALID_ARGUMENT
    msg = tb.get_lib().ct_get_last_error().decode()
    assert "more than the static" in msg
