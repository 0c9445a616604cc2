"""Cases of tests/golden/golden_ref_gpu.npz (outputs of the reference's own
GPU kernels, made by tests/golden/make_golden_gpu.py) and the oracle / C-entry
call each one corresponds to."""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "golden_ref_gpu.npz"

_PAT = re.compile(r"^(adx|dx|cci|willr|correl|sum|min|max)(\d+)(?:_path(\d))?$")


def load():
    if not GOLDEN.exists():
        return None
    z = np.load(GOLDEN)
    return {k: z[k] for k in z.files}


def cases(g):
    """Yield (case, key, family, params, data, want)."""
    inputs = {}
    for kk, vv in g.items():
        case, name = kk.split("/", 1)
        if name.startswith("in_"):
            inputs.setdefault(case, {})[name[3:]] = vv
    for key in sorted(g):
        case, name = key.split("/", 1)
        m = _PAT.match(name)
        if not m:
            continue
        data = dict(inputs[case])
        data["x"] = data["close"]
        data["y"] = data["aux"]
        yield case, key, m.group(1), {"period": int(m.group(2))}, data, g[key]
