"""Test infrastructure only: ctypes front-end to the CPU checkers.

``liboracle.so`` is the project's FP64 restatement (ta_oracle.c,
oracle_candles.c). ``_ref/libtaref.so`` is the reference's own CPU code compiled
from the reference tree (ref_bridge.cpp); it exists only where that tree was
available at build time (it is then shipped as a prebuilt file).

Only tests, ``__graft_entry__.smoke`` and bench.py's CPU baseline use this
module; the product library never imports it.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libtaref.so"

# name: (family id, input planes, output planes, int params, float params)
FAMILIES = {
    "sma": (0, ("close",), ("out",), ("period",), ()),
    "ema": (1, ("close",), ("out",), ("period",), ()),
    "wma": (2, ("close",), ("out",), ("period",), ()),
    "rsi": (3, ("close",), ("out",), ("period",), ()),
    "macd": (4, ("close",), ("macd", "signal", "hist"), ("fast", "slow", "signal"), ()),
    "atr": (5, ("high", "low", "close"), ("out",), ("period",), ()),
    "natr": (6, ("high", "low", "close"), ("out",), ("period",), ()),
    "trange": (7, ("high", "low", "close"), ("out",), (), ()),
    "adx": (8, ("high", "low", "close"), ("out",), ("period",), ()),
    "dx": (9, ("high", "low", "close"), ("out",), ("period",), ()),
    "bbands": (10, ("close",), ("upper", "middle", "lower"), ("period",), ("up", "dn")),
    "stoch": (11, ("high", "low", "close"), ("slowk", "slowd"), ("k", "d"), ()),
    "cci": (12, ("high", "low", "close"), ("out",), ("period",), ()),
    "obv": (13, ("close", "volume"), ("out",), (), ()),
    "ad": (14, ("high", "low", "close", "volume"), ("out",), (), ()),
    "adosc": (15, ("high", "low", "close", "volume"), ("out",), ("fast", "slow"), ()),
    "mfi": (16, ("high", "low", "close", "volume"), ("out",), ("period",), ()),
    "willr": (17, ("high", "low", "close"), ("out",), ("period",), ()),
    "sum": (18, ("close",), ("out",), ("period",), ()),
    "min": (19, ("close",), ("out",), ("period",), ()),
    "max": (20, ("close",), ("out",), ("period",), ()),
    "stddev": (21, ("close",), ("out",), ("period",), ("nbdev",)),
    "var": (22, ("close",), ("out",), ("period",), ()),
    "linearreg": (23, ("close",), ("out",), ("period",), ()),
    "correl": (24, ("x", "y"), ("out",), ("period",), ()),
    "dema": (25, ("close",), ("out",), ("period",), ()),
    "tema": (26, ("close",), ("out",), ("period",), ()),
    "t3": (27, ("close",), ("out",), ("period",), ("vfactor",)),
    "roc": (28, ("close",), ("out",), ("period",), ()),
    "rma": (29, ("close",), ("out",), ("period",), ()),
    "medprice": (30, ("high", "low"), ("out",), (), ()),
    "typprice": (31, ("high", "low", "close"), ("out",), (), ()),
    "midprice": (32, ("high", "low"), ("out",), ("period",), ()),
    "rocp": (33, ("close",), ("out",), ("period",), ()),
    "rocr": (34, ("close",), ("out",), ("period",), ()),
    "rocr100": (35, ("close",), ("out",), ("period",), ()),
    "momentum": (36, ("close",), ("out",), ("period",), ()),
    "avgprice": (37, ("open", "high", "low", "close"), ("out",), (), ()),
    "wclprice": (38, ("high", "low", "close"), ("out",), (), ()),
    "midpoint": (39, ("close",), ("out",), ("period",), ()),
    "change": (36, ("close",), ("out",), ("period",), ()),  # src/indicators/Change.cu: MOM's arithmetic
    "rolling_mean": (40, ("close",), ("out",), ("period",), ()),
    "rolling_max": (41, ("close",), ("out",), ("period",), ()),
    "rolling_min": (42, ("close",), ("out",), ("period",), ()),
    "rolling_std": (43, ("close",), ("out",), ("period",), ()),
    "ibs": (44, ("high", "low", "close"), ("out",), (), ()),
    "marketfi": (45, ("high", "low", "volume"), ("out",), (), ()),
    "qstick": (46, ("open", "close"), ("out",), ("period",), ()),
    "aroon": (47, ("high", "low"), ("down", "up"), ("period",), ()),
    "aroonosc": (48, ("high", "low"), ("out",), ("period",), ()),
}

_P = ct.c_void_p
_lib = None
_ref = None


def _load():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run make -C oracle)")
        lib = ct.CDLL(str(ORACLE_SO))
        lib.orc_batch.argtypes = [ct.c_int, _P, ct.c_int, ct.c_int, _P, _P, _P, ct.c_int]
        lib.orc_batch_ragged.argtypes = [ct.c_int, _P, ct.c_int, _P, _P, _P, _P, ct.c_int]
        lib.orc_cdl.argtypes = [ct.c_int, _P, _P, _P, _P, ct.c_int, ct.c_int, _P, ct.c_int]
        lib.orc_cdl_ragged.argtypes = [ct.c_int, _P, _P, _P, _P, ct.c_int, _P, _P, ct.c_int]
        lib.orc_cdl_lookback.argtypes = [ct.c_int]
        _lib = lib
    return _lib


def _f4(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptrs(arrays):
    arr = (ct.c_void_p * max(1, len(arrays)))()
    for i, a in enumerate(arrays):
        arr[i] = a.ctypes.data
    return arr


def run(name: str, data: dict, threads: int = 0, offsets=None, **params):
    """Run family ``name`` over the planes in ``data`` (2-D (S, T) arrays, or 1-D
    flat arrays with ``offsets`` of length S+1). Returns a tuple of float64
    arrays shaped like the inputs."""
    fid, ins, outs, ipn, fpn = FAMILIES[name]
    lib = _load()
    planes = [_f4(data[k]) for k in ins]
    shape = planes[0].shape
    res = [np.empty(shape, dtype=np.float64) for _ in outs]
    ip = np.array([int(params[k]) for k in ipn] or [0], dtype=np.int32)
    fp = np.array([float(params[k]) for k in fpn] or [0.0], dtype=np.float64)
    if offsets is None:
        S, T = shape
        rc = lib.orc_batch(fid, _ptrs(planes), S, T, ip.ctypes.data, fp.ctypes.data,
                           _ptrs(res), threads)
    else:
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        rc = lib.orc_batch_ragged(fid, _ptrs(planes), len(off) - 1, off.ctypes.data,
                                  ip.ctypes.data, fp.ctypes.data, _ptrs(res), threads)
    if rc != 0:
        raise ValueError(f"oracle rejected {name} {params}")
    return tuple(res)


def cdl_count() -> int:
    return 63


def cdl_lookback(k: int) -> int:
    return int(_load().orc_cdl_lookback(k))


def cdl(k: int, o, h, l, c, threads: int = 0, offsets=None):
    lib = _load()
    o, h, l, c = (_f4(a) for a in (o, h, l, c))
    out = np.empty(o.shape, dtype=np.int32)
    if offsets is None:
        S, T = o.shape
        rc = lib.orc_cdl(k, o.ctypes.data, h.ctypes.data, l.ctypes.data, c.ctypes.data,
                         S, T, out.ctypes.data, threads)
    else:
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        rc = lib.orc_cdl_ragged(k, o.ctypes.data, h.ctypes.data, l.ctypes.data,
                                c.ctypes.data, len(off) - 1, off.ctypes.data,
                                out.ctypes.data, threads)
    if rc != 0:
        raise ValueError(f"bad candle pattern {k}")
    return out


# ------------------------------------------------------------------ reference

def ref_available() -> bool:
    return REF_SO.exists()


def _load_ref():
    global _ref
    if _ref is None:
        lib = ct.CDLL(str(REF_SO))
        lib.ref_single.argtypes = [ct.c_int, _P, ct.c_int, ct.c_int, ct.c_int, ct.c_double, _P, ct.c_int]
        lib.ref_macd.argtypes = [_P, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, _P, _P, _P, ct.c_int]
        lib.ref_bbands.argtypes = [_P, ct.c_int, ct.c_int, ct.c_int, ct.c_double, ct.c_double, _P, _P, _P, ct.c_int]
        lib.ref_hlc.argtypes = [ct.c_int, _P, _P, _P, ct.c_int, ct.c_int, ct.c_int, ct.c_int, _P, _P, ct.c_int]
        lib.ref_states.argtypes = [ct.c_int, _P, _P, _P, _P, ct.c_int, ct.c_int, ct.c_int, ct.c_int, _P, ct.c_int]
        lib.ref_cdl.argtypes = [ct.c_int, _P, _P, _P, _P, ct.c_int, ct.c_int, _P, ct.c_int]
        lib.ref_price.argtypes = [ct.c_int, _P, _P, _P, ct.c_int, ct.c_int, ct.c_int, _P, ct.c_int]
        _ref = lib
    return _ref


_REF_SINGLE = {"sma": 0, "ema": 1, "wma": 2, "rsi": 3, "stddev": 4, "var": 5,
               "linearreg": 6, "dema": 7, "tema": 8, "t3": 9, "roc": 10, "rma": 11, "rocp": 12}
_REF_STATES = {"obv": 0, "ad": 1, "mfi": 2, "adosc": 3, "natr": 4}
_REF_PRICE = {"medprice": 0, "typprice": 1, "midprice": 2, "ibs": 3, "marketfi": 4, "qstick": 5}
REF_FAMILIES = (tuple(_REF_SINGLE) + ("macd", "bbands", "atr", "trange", "stoch") + tuple(_REF_STATES)
                + tuple(_REF_PRICE))


def ref_run(name: str, data: dict, threads: int = 0, **params):
    """Run the reference's own CPU code for ``name`` (see REF_FAMILIES)."""
    lib = _load_ref()
    c = _f4(data["close"]) if "close" in data else None
    shape = (c if c is not None else _f4(data["high"])).shape
    S, T = shape
    if name in _REF_SINGLE:
        out = np.empty(shape, np.float64)
        rc = lib.ref_single(_REF_SINGLE[name], c.ctypes.data, S, T, int(params.get("period", 0)),
                            float(params.get("vfactor", params.get("nbdev", 0.0))),
                            out.ctypes.data, threads)
        if name == "stddev" and float(params.get("nbdev", 1.0)) != 1.0:
            out = out * float(params["nbdev"])
        return (out,) if rc == 0 else None
    if name == "macd":
        outs = [np.empty(shape, np.float64) for _ in range(3)]
        rc = lib.ref_macd(c.ctypes.data, S, T, params["fast"], params["slow"], params["signal"],
                          *(o.ctypes.data for o in outs), threads)
        return tuple(outs) if rc == 0 else None
    if name == "bbands":
        outs = [np.empty(shape, np.float64) for _ in range(3)]
        rc = lib.ref_bbands(c.ctypes.data, S, T, params["period"], float(params["up"]),
                            float(params["dn"]), *(o.ctypes.data for o in outs), threads)
        return tuple(outs) if rc == 0 else None
    h, l = _f4(data.get("high", c)), _f4(data.get("low", c))
    if name == "qstick":
        h, l = _f4(data["open"]), c
    if name in _REF_PRICE:
        out = np.empty(shape, np.float64)
        third = _f4(data["volume"]) if name == "marketfi" else c
        rc = lib.ref_price(_REF_PRICE[name], h.ctypes.data, l.ctypes.data,
                           third.ctypes.data if third is not None else None, S, T,
                           int(params.get("period", 0)), out.ctypes.data, threads)
        return (out,) if rc == 0 else None
    if name in ("atr", "trange", "stoch"):
        fam = {"atr": 0, "trange": 1, "stoch": 2}[name]
        o0, o1 = np.empty(shape, np.float64), np.empty(shape, np.float64)
        p = params.get("period", params.get("k", 0))
        q = params.get("d", 0)
        rc = lib.ref_hlc(fam, h.ctypes.data, l.ctypes.data, c.ctypes.data, S, T, p, q,
                         o0.ctypes.data, o1.ctypes.data, threads)
        if rc != 0:
            return None
        return (o0, o1) if name == "stoch" else (o0,)
    if name in _REF_STATES:
        v = _f4(data["volume"]) if "volume" in data else None
        out = np.empty(shape, np.float32)
        p = params.get("period", params.get("fast", 0))
        q = params.get("slow", 0)
        lib.ref_states(_REF_STATES[name], h.ctypes.data, l.ctypes.data, c.ctypes.data,
                       v.ctypes.data if v is not None else None, S, T, p, q, out.ctypes.data, threads)
        return (out,)
    raise KeyError(name)


def ref_cdl(k: int, o, h, l, c, threads: int = 0):
    lib = _load_ref()
    o, h, l, c = (_f4(a) for a in (o, h, l, c))
    S, T = o.shape
    out = np.empty(o.shape, dtype=np.int32)
    rc = lib.ref_cdl(k, o.ctypes.data, h.ctypes.data, l.ctypes.data, c.ctypes.data, S, T,
                     out.ctypes.data, threads)
    if rc != 0:
        raise ValueError(k)
    return out


def host_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
