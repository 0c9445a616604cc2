"""Helpers for the GPU tests: calling the reference-named C entry points with
torch device buffers."""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

import tacuda_b200 as tb

HLC = ["high", "low", "close"]
HLCV = ["high", "low", "close", "volume"]
# name: (C symbol, input planes, outputs, scalars (type, oracle param name or constant))
SPECS = {
    "sma": ("ct_sma_batch_d", ["close"], 1, [("i", "period")]),
    "ema": ("ct_ema_batch_d", ["close"], 1, [("i", "period")]),
    "wma": ("ct_wma_batch_d", ["close"], 1, [("i", "period")]),
    "rsi": ("ct_rsi_batch_d", ["close"], 1, [("i", "period")]),
    "dema": ("ct_dema_batch_d", ["close"], 1, [("i", "period")]),
    "tema": ("ct_tema_batch_d", ["close"], 1, [("i", "period")]),
    "t3": ("ct_t3_batch_d", ["close"], 1, [("i", "period"), ("f", "vfactor")]),
    "stddev": ("ct_stddev_batch_d", ["close"], 1, [("i", "period")]),
    "var": ("ct_var_batch_d", ["close"], 1, [("i", "period")]),
    "sum": ("ct_sum_batch_d", ["close"], 1, [("i", "period")]),
    "max": ("ct_max_batch_d", ["close"], 1, [("i", "period")]),
    "min": ("ct_min_batch_d", ["close"], 1, [("i", "period")]),
    "linearreg": ("ct_linearreg_batch_d", ["close"], 1, [("i", "period")]),
    "atr": ("ct_atr_batch_d", HLC, 1, [("i", "period"), ("f", 0.0)]),
    "natr": ("ct_natr_batch_d", HLC, 1, [("i", "period")]),
    "trange": ("ct_trange_batch_d", HLC, 1, []),
    "adx": ("ct_adx_batch_d", HLC, 1, [("i", "period")]),
    "dx": ("ct_dx_batch_d", HLC, 1, [("i", "period")]),
    "willr": ("ct_willr_batch_d", HLC, 1, [("i", "period")]),
    "cci": ("ct_cci_batch_d", HLC, 1, [("i", "period")]),
    "macd": ("ct_macd_batch_d", ["close"], 3, [("i", "fast"), ("i", "slow"), ("i", "signal"), ("i", 1)]),
    "bbands": ("ct_bbands_batch_d", ["close"], 3, [("i", "period"), ("f", "up"), ("f", "dn")]),
    "stoch": ("ct_stochastic_batch_d", HLC, 2, [("i", "k"), ("i", "d")]),
    "obv": ("ct_obv_batch_d", ["close", "volume"], 1, []),
    "mfi": ("ct_mfi_batch_d", HLCV, 1, [("i", "period")]),
    "ad": ("ct_ad_batch_d", HLCV, 1, []),
    "adosc": ("ct_adosc_batch_d", HLCV, 1, [("i", "fast"), ("i", "slow")]),
    "correl": ("ct_correl_batch_d", ["x", "y"], 1, [("i", "period")]),
    "roc": ("ct_roc_batch_d", ["close"], 1, [("i", "period")]),
    "rma": ("ct_rma_batch_d", ["close"], 1, [("i", "period")]),
    "medprice": ("ct_medprice_batch_d", ["high", "low"], 1, []),
    "typprice": ("ct_typprice_batch_d", HLC, 1, []),
    "midprice": ("ct_midprice_batch_d", ["high", "low"], 1, [("i", "period")]),
    "rocp": ("ct_rocp_batch_d", ["close"], 1, [("i", "period")]),
    "rocr": ("ct_rocr_batch_d", ["close"], 1, [("i", "period")]),
    "rocr100": ("ct_rocr100_batch_d", ["close"], 1, [("i", "period")]),
    "momentum": ("ct_momentum_batch_d", ["close"], 1, [("i", "period")]),
    "avgprice": ("ct_avgprice_batch_d", ["open", "high", "low", "close"], 1, []),
    "wclprice": ("ct_wclprice_batch_d", HLC, 1, []),
    "midpoint": ("ct_midpoint_batch_d", ["close"], 1, [("i", "period")]),
    "change": ("ct_change_batch_d", ["close"], 1, [("i", "period")]),
    "rolling_mean": ("ct_rolling_mean_batch_d", ["close"], 1, [("i", "period")]),
    "rolling_max": ("ct_rolling_max_batch_d", ["close"], 1, [("i", "period")]),
    "rolling_min": ("ct_rolling_min_batch_d", ["close"], 1, [("i", "period")]),
    "rolling_std": ("ct_rolling_std_batch_d", ["close"], 1, [("i", "period")]),
    "ibs": ("ct_ibs_batch_d", HLC, 1, []),
    "marketfi": ("ct_marketfi_batch_d", ["high", "low", "volume"], 1, []),
    "qstick": ("ct_qstick_batch_d", ["open", "close"], 1, [("i", "period")]),
    "aroon": ("ct_aroon_batch_d", ["high", "low"], 2, [("i", "period")]),
    "aroonosc": ("ct_aroonosc_batch_d", ["high", "low"], 1, [("i", "period")]),
}

DEFAULTS = {
    "sma": dict(period=20), "ema": dict(period=14), "wma": dict(period=14), "rsi": dict(period=14),
    "dema": dict(period=10), "tema": dict(period=8), "t3": dict(period=5, vfactor=0.7),
    "stddev": dict(period=20, nbdev=1.0), "var": dict(period=20), "sum": dict(period=20), "max": dict(period=20),
    "min": dict(period=20), "linearreg": dict(period=14), "atr": dict(period=14), "natr": dict(period=14),
    "trange": {}, "adx": dict(period=14), "dx": dict(period=14), "willr": dict(period=14), "cci": dict(period=14),
    "macd": dict(fast=12, slow=26, signal=9), "bbands": dict(period=20, up=2.0, dn=2.0), "stoch": dict(k=14, d=3),
    "obv": {}, "mfi": dict(period=14), "ad": {}, "adosc": dict(fast=3, slow=10), "correl": dict(period=30),
    "roc": dict(period=10), "rma": dict(period=14), "medprice": {}, "typprice": {}, "midprice": dict(period=14),
    "rocp": dict(period=10), "rocr": dict(period=10), "rocr100": dict(period=10), "momentum": dict(period=10),
    "avgprice": {}, "wclprice": {}, "midpoint": dict(period=14), "change": dict(period=10),
    "rolling_mean": dict(period=20), "rolling_max": dict(period=20), "rolling_min": dict(period=20),
    "rolling_std": dict(period=20), "ibs": {}, "marketfi": {}, "qstick": dict(period=10),
    "aroon": dict(period=14), "aroonosc": dict(period=14),
}


def device_planes(data: dict, dev="cuda") -> dict:
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in data.items()}


def call_batch_d(name: str, dplanes: dict, params: dict, stream=0, outs=None):
    """Run ct_<name>_batch_d; returns the list of output tensors."""
    sym, ins, nout, scal = SPECS[name]
    S, T = dplanes[ins[0]].shape
    if outs is None:
        outs = [torch.full((S, T), 12345.0, device=dplanes[ins[0]].device) for _ in range(nout)]
    args = [ct.c_void_p(dplanes[k].data_ptr()) for k in ins] + [ct.c_void_p(o.data_ptr()) for o in outs]
    args += [ct.c_int(T), ct.c_int(S)]
    for typ, key in scal:
        v = params[key] if isinstance(key, str) else key
        args.append(ct.c_int(int(v)) if typ == "i" else ct.c_float(float(v)))
    args += [ct.c_int(0), ct.c_void_p(stream)]
    rc = getattr(tb.get_lib(), sym)(*args)
    tb.call_status(rc, sym)
    return outs


def to_np(ts):
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in ts]


def call_cdl(k: int, dplanes: dict, name: str, stream=0):
    """ct_cdl_<name>_batch_d for pattern k (float signal plane)."""
    S, T = dplanes["open"].shape
    out = torch.full((S, T), 12345.0, device=dplanes["open"].device)
    sym = f"ct_cdl_{name}_batch_d"
    args = [ct.c_void_p(dplanes[p].data_ptr()) for p in ("open", "high", "low", "close")]
    args += [ct.c_void_p(out.data_ptr()), ct.c_int(T), ct.c_int(S), ct.c_int(0), ct.c_void_p(stream)]
    tb.call_status(getattr(tb.get_lib(), sym)(*args), sym)
    return out
