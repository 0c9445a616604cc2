"""Generate golden_ref_gpu.npz from the reference's own GPU code
(oracle/_ref/libtaref_gpu.so: the reference's short-row, fused-row and ADX / DX
/ CCI / WILLR / CORREL kernels for sm_100a, compiled from the reference tree by
oracle/Makefile, target refgpu). Runs on a machine with a GPU:

    python tests/golden/make_golden_gpu.py [out.npz]

These are the families whose only reference implementation is CUDA. The
fixtures hold seeded inputs and the reference's outputs of the paths its batch
entry points take:
  * ADX, DX, CORREL: the short-row kernel (rows of at most 1024 bars) and the
    per-series path (longer rows);
  * CCI, WILLR: the flat rows plan (one call over the flattened matrix, NaN
    warm-up per row);
  * SUM, MIN, MAX: the fused window kernels.
They pin the project's FP64 oracle (tests/test_oracle_pin_refgpu.py) and the
CUDA path (tests/test_gpu_ref_pin.py) without the reference tree at test time.
"""
from __future__ import annotations

import ctypes as ct
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from tacuda_b200 import synthetic  # noqa: E402

LIB = ROOT / "oracle" / "_ref" / "libtaref_gpu.so"
FUSED = {"sum": 11, "min": 12, "max": 13}  # src/api/BatchFused.h FusedFamily


def inputs():
    """Cases: name -> planes (S, T) float32."""
    cases = {}
    d = synthetic.ohlcv(24, 234, seed=11)
    d["aux"] = synthetic.ohlcv(24, 234, seed=12)["close"]
    # row 20 flat, row 21 with zero ranges, rows 22/23 with NaN bars
    for k in ("open", "high", "low", "close", "aux"):
        d[k][20] = 100.0
    d["volume"][20] = 1000.0
    for k in ("open", "high", "low", "close"):
        d[k][21, 100:140] = 50.0
    for k in ("high", "low", "close", "open", "aux"):
        d[k][22, 60] = np.nan
        d[k][23, 0] = np.nan
        d[k][23, 150] = np.nan
    cases["short"] = d
    long = synthetic.ohlcv(3, 1500, seed=13)
    long["aux"] = synthetic.ohlcv(3, 1500, seed=14)["close"]
    cases["long"] = long
    return cases


def main():
    import torch

    lib = ct.CDLL(str(LIB))
    P, I, F = ct.c_void_p, ct.c_int, ct.c_float
    for fn in ("refgpu_adx", "refgpu_dx"):
        getattr(lib, fn).argtypes = [P, P, P, P, I, I, I, I, P]
    lib.refgpu_correl.argtypes = [P, P, P, I, I, I, I, P]
    lib.refgpu_cci.argtypes = [P, P, P, P, I, I, I, P]
    lib.refgpu_willr.argtypes = [P, P, P, P, I, I, I, P]
    lib.refgpu_fused.argtypes = [I, P, P, P, P, P, P, P, I, I, I, I, I, F, F, P]
    out = {}
    for case, d in inputs().items():
        S, T = d["close"].shape
        dev = {k: torch.from_numpy(v).cuda() for k, v in d.items()}
        for k, v in d.items():
            out[f"{case}/in_{k}"] = v
        h, l, c, x, y = (dev[k].data_ptr() for k in ("high", "low", "close", "close", "aux"))

        def fresh():
            return torch.full((S, T), 777.0, device="cuda")

        def keep(name, t, rc):
            torch.cuda.synchronize()
            if rc != 0:
                raise SystemExit(f"{case}/{name}: reference call failed ({rc})")
            out[f"{case}/{name}"] = t.cpu().numpy()

        paths = (0, 1) if T <= 1024 else (1,)
        for p in (2, 14, 30):
            for path in paths:
                o = fresh()
                keep(f"adx{p}_path{path}", o, lib.refgpu_adx(h, l, c, o.data_ptr(), T, S, p, path, None))
                o = fresh()
                keep(f"dx{p}_path{path}", o, lib.refgpu_dx(h, l, c, o.data_ptr(), T, S, p, path, None))
            o = fresh()
            keep(f"cci{p}", o, lib.refgpu_cci(h, l, c, o.data_ptr(), T, S, p, None))
            o = fresh()
            keep(f"willr{p}", o, lib.refgpu_willr(h, l, c, o.data_ptr(), T, S, p, None))
        for p in (2, 30):
            for path in paths:
                o = fresh()
                keep(f"correl{p}_path{path}", o, lib.refgpu_correl(x, y, o.data_ptr(), T, S, p, path, None))
        for name, fam in FUSED.items():
            for p in (1, 5, 20):
                o = fresh()
                keep(f"{name}{p}", o, lib.refgpu_fused(fam, c, None, None, None, o.data_ptr(), None, None, T, S, p, 0,
                                                       0, 2.0, 2.0, None))
    dst = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).with_name("golden_ref_gpu.npz")
    np.savez_compressed(dst, **out)
    print("wrote", len(out), "arrays to", dst)


if __name__ == "__main__":
    main()
