"""Long-series precision stress: error of each precision variant against the
FP64 oracle on 4 series x 50,000,000 bars of a random walk (sigma 0.01) on a
+1e4 level, for SMA(200), STDDEV(200), VAR(200), LINEARREG(200), CORREL(30)
of two such walks and EMA(500), all through the look-back engine; with the
device time of each fused launch.

    python tests/precision_report.py [--bars 50000000] [--out report.json]

Needs a GPU; prints one JSON object (per variant: ms, and per indicator the
largest relative error over bars with |ref| > 1e-12*max|ref| and the largest
error scaled by the row's max |ref|).
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

JOBS = [("sma", (200,), (), dict(period=200)), ("stddev", (200,), (1.0,), dict(period=200, nbdev=1.0)),
        ("var", (200,), (), dict(period=200)), ("linearreg", (200,), (), dict(period=200)),
        ("correl", (30,), (), dict(period=30)), ("ema", (500,), (), dict(period=500))]
VARIANTS = ("fp64", "fp32", "fp32c", "fp32/fp64carry")


def main():
    import torch
    import tacuda_b200 as tb
    from oracle import oracle as O
    from tacuda_b200 import synthetic

    ap = argparse.ArgumentParser()
    ap.add_argument("--bars", type=int, default=50_000_000)
    ap.add_argument("--series", type=int, default=4)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    S, T = args.series, args.bars
    x = synthetic.level_walk(S, T, seed=5)
    y = synthetic.level_walk(S, T, seed=6)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    outs = {n: torch.empty_like(dx) for n, *_ in JOBS}
    series = tb.make_series({"close": dx.data_ptr(), "aux": dy.data_ptr()}, S, T)
    report = {"workload": f"{S} series x {T} bars, random walk sigma 0.01 on a 1e4 level", "variants": {}}
    data = {"close": x, "x": x, "y": y}
    for var in VARIANTS:
        jobs = [tb.make_job(n, p, fp, [outs[n].data_ptr()], inputs=("close", "aux") if n == "correl" else None,
                            precision=var) for n, p, fp, _ in JOBS]
        tb.fused_batch_d(series, jobs, 0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tb.fused_batch_d(series, jobs, 0)
        e1.record()
        torch.cuda.synchronize()
        entry = {"ms": e0.elapsed_time(e1), "errors": {}}
        for n, _, _, kw in JOBS:
            ref = O.run(n, data, **kw)[0]
            g = outs[n].cpu().numpy().astype(np.float64)
            m = ~np.isnan(ref)
            scale = np.nanmax(np.abs(ref), axis=1, keepdims=True)
            err = np.abs(g - ref)
            big = m & (np.abs(ref) > 1e-12 * scale)
            rel = float(np.max(err[big] / np.abs(ref[big]))) if big.any() else 0.0
            entry["errors"][n] = {"max_rel": rel, "max_scaled": float(np.nanmax(err / scale)),
                                  "nan_mask_exact": bool(np.array_equal(np.isnan(g), ~m))}
            del ref, g, err
        report["variants"][var] = entry
        print(json.dumps({var: entry}), flush=True)
    text = json.dumps(report, indent=1)
    print(text)
    if args.out:
        Path(args.out).write_text(text)


if __name__ == "__main__":
    main()
