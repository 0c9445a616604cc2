"""Small, self-contained workloads for ncu captures of single kernels (one GPU;
each case runs its launch three times so a capture can skip the first two).

    python tests/profile_cases.py cdl      # candle tile kernel, 61 patterns, 4000 x 2000 bars
    python tests/profile_cases.py pass13   # 13-indicator fused pass, 4000 x 2000 bars
    python tests/profile_cases.py alpha    # alpha forward + adjoint, 4096 x 2048 bars
    python tests/profile_cases.py lb5      # long-series jobs through look-back, 4 x 2,000,000 bars

The commands in profiles/*.md run these cases under `ncu`.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main(case: str) -> None:
    import torch
    import tacuda_b200 as tb
    from tacuda_b200 import synthetic, workloads
    if case in ("cdl", "pass13"):
        S, T = 4000, 2000
        d = synthetic.ohlcv(S, T, seed=5)
        dp = {k: torch.from_numpy(v).cuda() for k, v in d.items()}
        ser = tb.make_series({k: v.data_ptr() for k, v in dp.items()}, S, T)
        if case == "cdl":
            names = tb.cdl_names()
            mask = sum(1 << k for k, n in enumerate(names) if n not in ("bullish_engulfing", "bearish_engulfing"))
            out = torch.empty((len(names), S, T), dtype=torch.int32, device="cuda")
            jobs = [tb.make_job("cdl", (), (), [out.data_ptr()], cdl_mask=mask, cdl_stride=S * T, cdl_int32=True)]
        else:
            outs = {n: torch.empty((S, T), device="cuda") for n in workloads.PASS13_OUTPUTS}
            jobs = [tb.make_job(fam, p, fp, [outs[o].data_ptr() for o in on]) for _, fam, p, fp, on in workloads.PASS13]
        for _ in range(3):
            tb.fused_batch_d(ser, jobs, 0)
    elif case == "alpha":
        from tacuda_b200 import torch_api as TA
        rng = np.random.default_rng(4)
        c = torch.from_numpy(synthetic.ohlcv(4096, 2048, seed=4)["close"]).cuda()
        a = torch.from_numpy(rng.uniform(0.01, 0.5, 4096).astype(np.float32)).cuda()
        w = [torch.from_numpy(rng.standard_normal((4096, 2048)).astype(np.float32)).cuda() for _ in range(5)]
        for _ in range(3):
            ck = TA.alpha_forward(c, a)[5]
            TA.alpha_backward(c, a, ck, w)
    elif case == "lb5":
        S, T = 4, 2_000_000
        x = torch.from_numpy(synthetic.level_walk(S, T, seed=5)).cuda()
        y = torch.from_numpy(synthetic.level_walk(S, T, seed=6)).cuda()
        o = {n: torch.empty_like(x) for n in ("sma", "stddev", "var", "linearreg", "correl", "ema")}
        jobs = [tb.make_job("sma", (200,), (), [o["sma"].data_ptr()]),
                tb.make_job("stddev", (200,), (1.0,), [o["stddev"].data_ptr()]),
                tb.make_job("var", (200,), (), [o["var"].data_ptr()]),
                tb.make_job("linearreg", (200,), (), [o["linearreg"].data_ptr()]),
                tb.make_job("correl", (30,), (), [o["correl"].data_ptr()], inputs=("close", "aux")),
                tb.make_job("ema", (500,), (), [o["ema"].data_ptr()])]
        ser = tb.make_series({"close": x.data_ptr(), "aux": y.data_ptr()}, S, T)
        for _ in range(3):
            tb.fused_batch_d(ser, jobs, 0)
    else:
        raise SystemExit(f"unknown case {case!r}")
    torch.cuda.synchronize()
    print("ok", case)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "pass13")
