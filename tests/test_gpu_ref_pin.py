"""GPU: the CUDA path against the reference's own GPU kernels (fixtures of
tests/golden/golden_ref_gpu.npz, see tests/test_oracle_pin_refgpu.py), through
the reference-named C entry points, on every engine."""
from __future__ import annotations

import os

import pytest

from gpu_util import call_batch_d, device_planes, to_np
from refgpu_cases import cases, load
from tolerance import compare

pytestmark = pytest.mark.gpu

G = load()
CASES = list(cases(G)) if G is not None else []


@pytest.fixture(params=["sp", "ws", "lb"])
def engine(request):
    os.environ["TACUDA_B200_MODE"] = request.param
    yield request.param
    del os.environ["TACUDA_B200_MODE"]


@pytest.mark.skipif(G is None, reason="golden_ref_gpu.npz not generated")
@pytest.mark.parametrize("case,key,fam,params,data,want", CASES, ids=[c[1] for c in CASES])
def test_cuda_matches_reference_gpu(case, key, fam, params, data, want, engine):
    got = to_np(call_batch_d(fam, device_planes(data), params))[0]
    compare(got, want, f"{key} [{engine}]")
