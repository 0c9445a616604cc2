"""GPU: the allocation-free look-back entry point (static device scratch)
against the look-back engine of the regular fused entry point, whose scratch
comes from the stream-ordered pool. Kept in its own file, collected last, so
it also runs after every other test has used the library."""
import ctypes as ct
import os

import pytest
import torch

import tacuda_b200 as tb
from tacuda_b200 import synthetic, workloads
from tolerance import compare

pytestmark = pytest.mark.gpu


def _entry():
    f = tb.get_lib().ct_b200_fused_lookback_static_d
    f.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]
    f.restype = ct.c_int
    return f


def _pass13(S, T, seed):
    d = synthetic.ohlcv(S, T, seed=seed)
    dp = {k: torch.from_numpy(v).cuda() for k, v in d.items()}
    outs = {n: torch.full((S, T), 777.0, device="cuda") for n in workloads.PASS13_OUTPUTS}
    jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
    series = tb.make_series({k: v.data_ptr() for k, v in dp.items() if k in tb.PLANE_ID}, S, T)
    return dp, outs, jobs, series


def test_static_scratch_matches_pool_scratch_twice():
    S, T = 2, 40000
    dp, outs, jobs, series = _pass13(S, T, seed=31)
    os.environ["TACUDA_B200_MODE"] = "lb"
    try:
        tb.fused_batch_d(series, jobs, 0)
    finally:
        del os.environ["TACUDA_B200_MODE"]
    torch.cuda.synchronize()
    ref = {k: v.clone() for k, v in outs.items()}
    arr = tb.job_array(jobs)
    f = _entry()
    for call in range(2):
        for v in outs.values():
            v.fill_(777.0)
        rc = f(ct.addressof(series), ct.addressof(arr), len(jobs), None)
        tb.call_status(rc, "ct_b200_fused_lookback_static_d")
        torch.cuda.synchronize()
        for k in outs:
            compare(outs[k].cpu().numpy(), ref[k].cpu().numpy().astype("float64"), f"static call {call} {k}")


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
