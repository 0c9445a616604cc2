"""CPU: the project's FP64 oracle against the reference's own GPU kernels.

ADX, DX, CCI, WILLR, CORREL and the fused SUM / MIN / MAX windows have no CPU
code in the reference; their reference behaviour is its CUDA. The fixtures in
tests/golden/golden_ref_gpu.npz are that CUDA's outputs on seeded inputs (made
on a GPU by tests/golden/make_golden_gpu.py from oracle/_ref/libtaref_gpu.so,
which oracle/Makefile compiles from the reference tree): the short-row and
per-series paths of ADX / DX / CORREL, the flat rows plan of CCI / WILLR and
the fused windows of SUM / MIN / MAX. NaN positions must match exactly; values
within the float tolerance of tests/tolerance.py."""
from __future__ import annotations

import pytest

from oracle import oracle as O
from refgpu_cases import cases, load
from tolerance import compare

G = load()
pytestmark = pytest.mark.skipif(G is None, reason="golden_ref_gpu.npz not generated")

CASES = list(cases(G)) if G is not None else []


@pytest.mark.parametrize("case,key,fam,params,data,want", CASES, ids=[c[1] for c in CASES])
def test_oracle_matches_reference_gpu(case, key, fam, params, data, want):
    got = O.run(fam, data, **params)[0]
    compare(got, want, key)


def test_fixture_covers_every_reference_only_family():
    fams = {c[2] for c in CASES}
    assert {"adx", "dx", "cci", "willr", "correl", "sum", "min", "max"} <= fams
