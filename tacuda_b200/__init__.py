"""tacuda_b200: B200-native (sm_100a) batched technical indicators behind
TACUDA's C ABI.

The product is the C-ABI shared library ``libtacuda_b200.so`` next to this
file (built by ``python -m tacuda_b200.build``). This module is a thin ctypes
front-end mirroring the reference's Python binding
(bindings/python/tacuda/__init__.py:792-940): ``sma_batch``, ``ema_batch``,
``rsi_batch``, ``atr_batch``, ``macd_batch``, ``bbands_batch`` and
``stochastic_batch`` take NumPy ``(numSeries, seriesLen)`` matrices, call the
host batch entry points and raise ``RuntimeError`` with the library's last
error on failure. ``tacuda_b200.torch_api`` adds the torch-tensor (device
pointer + current stream) wrappers and the autograd functions.

There is no CPU fallback: importing this module without the built library
raises.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path
from typing import Any, Tuple

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libtacuda_b200.so"

CT_STATUS = {
    0: "CT_STATUS_SUCCESS", 1: "CT_STATUS_ALLOC_FAILED", 2: "CT_STATUS_COPY_FAILED",
    3: "CT_STATUS_KERNEL_FAILED", 4: "CT_STATUS_INVALID_ARGUMENT", 5: "CT_STATUS_DEVICE_ERROR",
    6: "CT_STATUS_UNSUPPORTED",
}

# ctB200Family / ctB200Plane (include/tacuda.h)
FAMILIES = ("sma", "ema", "wma", "rsi", "macd", "atr", "natr", "trange", "adx", "dx", "bbands", "stoch",
            "cci", "obv", "ad", "adosc", "mfi", "willr", "sum", "min", "max", "stddev", "var", "linearreg",
            "correl", "dema", "tema", "t3", "cdl", "roc", "rma", "medprice", "typprice", "midprice",
            "rocp", "rocr", "rocr100", "momentum", "avgprice", "wclprice", "midpoint",
            "rolling_mean", "rolling_max", "rolling_min", "rolling_std", "ibs", "marketfi", "qstick",
            "aroon", "aroonosc")
FAMILY_ID = {n: i for i, n in enumerate(FAMILIES)}
PLANES = ("open", "high", "low", "close", "volume", "aux")
PLANE_ID = {n: i for i, n in enumerate(PLANES)}
OUTPUTS = {"macd": 3, "bbands": 3, "stoch": 2, "aroon": 2}

_P = ct.c_void_p
_I = ct.c_int
_F = ct.c_float


class ctB200Series(ct.Structure):
    _fields_ = [("planes", _P * 6), ("offsets", _P), ("seriesLen", ct.c_int64), ("numSeries", _I)]


class ctB200Job(ct.Structure):
    _fields_ = [("family", _I), ("params", _I * 3), ("fparams", ct.c_double * 2), ("inputs", _I * 4),
                ("outputs", _P * 3), ("cdl_mask", ct.c_uint64), ("cdl_stride", ct.c_int64),
                ("cdl_int32", _I), ("precision", _I)]


class ctB200AlphaParams(ct.Structure):
    _fields_ = [("emaPeriod", _I), ("fastPeriod", _I), ("slowPeriod", _I), ("signalPeriod", _I),
                ("rsiPeriod", _I)]


def _load() -> ct.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"tacuda_b200 native library missing: {LIB_PATH} "
                          "(build it with `python -m tacuda_b200.build`)")
    lib = ct.CDLL(str(LIB_PATH))
    lib.ct_get_last_error.restype = ct.c_char_p
    lib.ct_status_string.restype = ct.c_char_p
    lib.ct_version.restype = ct.c_char_p
    lib.ct_b200_cdl_name.restype = ct.c_char_p
    lib.ct_b200_cdl_name.argtypes = [_I]
    lib.ct_b200_cdl_lookback.argtypes = [_I]
    lib.ct_b200_launch_count.restype = ct.c_ulonglong
    lib.ct_b200_take_device_error.argtypes = [ct.POINTER(_I)]
    lib.ct_b200_fused_batch_d.argtypes = [ct.POINTER(ctB200Series), ct.POINTER(ctB200Job), _I, _P]
    lib.ct_b200_fused_batch.argtypes = [ct.POINTER(ctB200Series), ct.POINTER(ctB200Job), _I, _P]
    lib.ct_b200_plan_create.argtypes = [ct.POINTER(ctB200Job), _I, _P, _I, ct.c_int64, ct.POINTER(_P)]
    lib.ct_b200_plan_execute.argtypes = [_P, ct.POINTER(ctB200Series), ct.POINTER(ctB200Job), _I, _P]
    lib.ct_b200_plan_autotune.argtypes = [_P, ct.POINTER(ctB200Series), ct.POINTER(ctB200Job), _I, _P]
    lib.ct_b200_plan_describe.argtypes = [_P, ct.POINTER(_I), ct.POINTER(_I), ct.POINTER(_I), ct.POINTER(_I)]
    lib.ct_b200_plan_destroy.argtypes = [_P]
    lib.ct_b200_plan_candidates.argtypes = [_P, _I, _P, _P, _P, _P]
    lib.ct_b200_plan_candidates.restype = _I
    lib.ct_b200_plan_describe_rows.argtypes = [_P, ct.POINTER(_I), ct.POINTER(_I)]
    lib.ct_b200_plan_candidates_rows.argtypes = [_P, _I, _P, _P]
    lib.ct_b200_plan_candidates_rows.restype = _I
    lib.ct_b200_cdl_batch_d.argtypes = [_P, _P, _P, _P, _P, _I, _I, ct.c_uint64, _P]
    lib.ct_b200_alpha_checkpoint_doubles.argtypes = [_I]
    lib.ct_b200_alpha_checkpoint_doubles.restype = ct.c_longlong
    lib.ct_b200_alpha_forward_d.argtypes = [_P, _P, _I, _I, ct.POINTER(ctB200AlphaParams)] + [_P] * 7
    lib.ct_b200_alpha_backward_d.argtypes = [_P, _P, _I, _I, ct.POINTER(ctB200AlphaParams)] + [_P] * 9
    return lib


_lib = None


def get_lib() -> ct.CDLL:
    """The loaded native library (loaded on first use; raises if missing)."""
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def __getattr__(name: str):
    if name == "lib":
        return get_lib()
    raise AttributeError(name)


def version() -> str:
    return get_lib().ct_version().decode()


def status_string(rc: int) -> str:
    return get_lib().ct_status_string(int(rc)).decode()


def get_last_error() -> str:
    return (get_lib().ct_get_last_error() or b"").decode()


def call_status(rc: int, func_name: str) -> None:
    """Raise like the reference binding (bindings/python/tacuda/__init__.py:643-645)."""
    if rc != 0:
        raise RuntimeError(f"{func_name} failed with code {rc} ({status_string(rc)}): {get_last_error()}")


def cdl_names() -> list[str]:
    return [get_lib().ct_b200_cdl_name(k).decode() for k in range(get_lib().ct_b200_cdl_count())]


def cdl_lookback(k: int) -> int:
    return int(get_lib().ct_b200_cdl_lookback(k))


def launch_count() -> int:
    return int(get_lib().ct_b200_launch_count())


def take_device_error() -> int:
    """Read and clear the current device's error word (bit 0: a bounded wait
    of an engine ran out since the last read); ct_b200_take_device_error."""
    flags = ct.c_int(0)
    call_status(get_lib().ct_b200_take_device_error(ct.byref(flags)), "ct_b200_take_device_error")
    return int(flags.value)


def stream_arg(value: Any) -> ct.c_void_p:
    if value is None:
        return ct.c_void_p(0)
    if isinstance(value, ct.c_void_p):
        return value
    if isinstance(value, bool) or not isinstance(value, int):
        raise TypeError("stream must be None, an int handle or ctypes.c_void_p")
    return ct.c_void_p(value)


def _mat(a: Any) -> np.ndarray:
    m = np.asarray(a, dtype=np.float32)
    if m.ndim != 2:
        raise ValueError("batch input must be a 2D array (numSeries, seriesLen)")
    return np.ascontiguousarray(m)


def _ptr(a: np.ndarray) -> ct.c_void_p:
    return ct.c_void_p(a.ctypes.data)


def _same(*ms: np.ndarray) -> None:
    for m in ms[1:]:
        if m.shape != ms[0].shape:
            raise ValueError("input matrices must have the same shape")


# --- host batch API, names and arguments as the reference binding ------------

def sma_batch(inputs: Any, period: int, max_concurrency: int = 0, stream: Any = None) -> np.ndarray:
    a = _mat(inputs); out = np.zeros_like(a)
    call_status(get_lib().ct_sma_batch(_ptr(a), _ptr(out), _I(a.shape[1]), _I(a.shape[0]), _I(int(period)),
                                 _I(int(max_concurrency)), stream_arg(stream)), "ct_sma_batch")
    return out


def ema_batch(inputs: Any, period: int, max_concurrency: int = 0, stream: Any = None) -> np.ndarray:
    a = _mat(inputs); out = np.zeros_like(a)
    call_status(get_lib().ct_ema_batch(_ptr(a), _ptr(out), _I(a.shape[1]), _I(a.shape[0]), _I(int(period)),
                                 _I(int(max_concurrency)), stream_arg(stream)), "ct_ema_batch")
    return out


def rsi_batch(inputs: Any, period: int, max_concurrency: int = 0, stream: Any = None) -> np.ndarray:
    a = _mat(inputs); out = np.zeros_like(a)
    call_status(get_lib().ct_rsi_batch(_ptr(a), _ptr(out), _I(a.shape[1]), _I(a.shape[0]), _I(int(period)),
                                 _I(int(max_concurrency)), stream_arg(stream)), "ct_rsi_batch")
    return out


def atr_batch(high: Any, low: Any, close: Any, period: int, initial: float = 0.0, max_concurrency: int = 0,
              stream: Any = None) -> np.ndarray:
    h, l, c = _mat(high), _mat(low), _mat(close); _same(h, l, c)
    out = np.zeros_like(h)
    call_status(get_lib().ct_atr_batch(_ptr(h), _ptr(l), _ptr(c), _ptr(out), _I(h.shape[1]), _I(h.shape[0]),
                                 _I(int(period)), _F(float(initial)), _I(int(max_concurrency)),
                                 stream_arg(stream)), "ct_atr_batch")
    return out


def macd_batch(inputs: Any, fastPeriod: int = 12, slowPeriod: int = 26, signalPeriod: int = 9, type: int = 1,
               max_concurrency: int = 0, stream: Any = None) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    a = _mat(inputs); m, s, h = np.zeros_like(a), np.zeros_like(a), np.zeros_like(a)
    call_status(get_lib().ct_macd_batch(_ptr(a), _ptr(m), _ptr(s), _ptr(h), _I(a.shape[1]), _I(a.shape[0]),
                                  _I(int(fastPeriod)), _I(int(slowPeriod)), _I(int(signalPeriod)), _I(int(type)),
                                  _I(int(max_concurrency)), stream_arg(stream)), "ct_macd_batch")
    return m, s, h


def bbands_batch(inputs: Any, period: int, upperMul: float = 2.0, lowerMul: float = 2.0, max_concurrency: int = 0,
                 stream: Any = None) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    a = _mat(inputs); up, mid, lo = np.zeros_like(a), np.zeros_like(a), np.zeros_like(a)
    call_status(get_lib().ct_bbands_batch(_ptr(a), _ptr(up), _ptr(mid), _ptr(lo), _I(a.shape[1]), _I(a.shape[0]),
                                    _I(int(period)), _F(float(upperMul)), _F(float(lowerMul)),
                                    _I(int(max_concurrency)), stream_arg(stream)), "ct_bbands_batch")
    return up, mid, lo


def stochastic_batch(high: Any, low: Any, close: Any, kPeriod: int = 14, dPeriod: int = 3,
                     max_concurrency: int = 0, stream: Any = None) -> Tuple[np.ndarray, np.ndarray]:
    h, l, c = _mat(high), _mat(low), _mat(close); _same(h, l, c)
    k, d = np.zeros_like(h), np.zeros_like(h)
    call_status(get_lib().ct_stochastic_batch(_ptr(h), _ptr(l), _ptr(c), _ptr(k), _ptr(d), _I(h.shape[1]),
                                        _I(h.shape[0]), _I(int(kPeriod)), _I(int(dPeriod)),
                                        _I(int(max_concurrency)), stream_arg(stream)), "ct_stochastic_batch")
    return k, d


# --- fused jobs ----------------------------------------------------------------

PRECISIONS = {"fp64": 0, "fp32": 1, "fp32c": 2, "fp32/fp64carry": 3}


def make_job(family: str, params=(), fparams=(), outputs=(), inputs=None, cdl_mask: int = 0,
             cdl_stride: int = 0, cdl_int32: bool = False, precision="fp64") -> ctB200Job:
    j = ctB200Job()
    j.family = FAMILY_ID[family]
    for i, v in enumerate(params):
        j.params[i] = int(v)
    for i, v in enumerate(fparams):
        j.fparams[i] = float(v)
    if inputs is None:
        j.inputs[0] = -1
    else:
        for i, v in enumerate(inputs):
            j.inputs[i] = PLANE_ID[v] if isinstance(v, str) else int(v)
    for i, p in enumerate(outputs):
        j.outputs[i] = int(p)
    j.cdl_mask = int(cdl_mask)
    j.cdl_stride = int(cdl_stride)
    j.cdl_int32 = 1 if cdl_int32 else 0
    j.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    return j


def make_series(planes: dict, numSeries: int, seriesLen: int = 0, offsets: int = 0) -> ctB200Series:
    s = ctB200Series()
    for name, ptr in planes.items():
        s.planes[PLANE_ID[name]] = int(ptr) if ptr else None
    s.offsets = int(offsets) if offsets else None
    s.seriesLen = int(seriesLen)
    s.numSeries = int(numSeries)
    return s


def job_array(jobs):
    return (ctB200Job * len(jobs))(*jobs)


class Plan:
    """Reusable schedule for a (possibly ragged) batch: ct_b200_plan_*."""

    def __init__(self, jobs, numSeries: int, seriesLen: int = 0, host_offsets: np.ndarray | None = None):
        self._jobs = job_array(jobs)
        self._n = len(jobs)
        self.handle = ct.c_void_p()
        off = None
        if host_offsets is not None:
            self._off = np.ascontiguousarray(host_offsets, dtype=np.int64)
            off = ct.c_void_p(self._off.ctypes.data)
        call_status(get_lib().ct_b200_plan_create(self._jobs, self._n, off, int(numSeries), int(seriesLen),
                                            ct.byref(self.handle)), "ct_b200_plan_create")

    def execute(self, series: ctB200Series, jobs, stream: Any = None) -> None:
        arr = job_array(jobs)
        call_status(get_lib().ct_b200_plan_execute(self.handle, ct.byref(series), arr, len(jobs), stream_arg(stream)),
                    "ct_b200_plan_execute")

    def autotune(self, series: ctB200Series, jobs, stream: Any = None) -> None:
        arr = job_array(jobs)
        call_status(get_lib().ct_b200_plan_autotune(self.handle, ct.byref(series), arr, len(jobs), stream_arg(stream)),
                    "ct_b200_plan_autotune")

    def describe(self) -> dict:
        m, k, w, b = _I(), _I(), _I(), _I()
        call_status(get_lib().ct_b200_plan_describe(self.handle, ct.byref(m), ct.byref(k), ct.byref(w),
                                                    ct.byref(b)), "ct_b200_plan_describe")
        d = {"mode": m.value, "bars_per_lane": k.value, "warps_per_block": w.value, "max_blocks": b.value}
        if m.value == 1:
            p, g = _I(), _I()
            call_status(get_lib().ct_b200_plan_describe_rows(self.handle, ct.byref(p), ct.byref(g)),
                        "ct_b200_plan_describe_rows")
            d.update(parts=p.value, groups=g.value)  # 0: the library's default for the job set
        return d

    ENGINES = {0: "warp-scan", 1: "row-parallel", 2: "look-back"}

    def candidates(self) -> list[dict]:
        """Launch shapes the last autotune() timed, with milliseconds per launch."""
        lib = get_lib()
        n = lib.ct_b200_plan_candidates(self.handle, 0, None, None, None, None)
        if n <= 0:
            return []
        m, k, w = (np.zeros(n, np.int32) for _ in range(3))
        ms = np.zeros(n, np.float32)
        lib.ct_b200_plan_candidates(self.handle, n, m.ctypes.data, k.ctypes.data, w.ctypes.data, ms.ctypes.data)
        p, g = np.zeros(n, np.int32), np.zeros(n, np.int32)
        lib.ct_b200_plan_candidates_rows(self.handle, n, p.ctypes.data, g.ctypes.data)
        out = []
        for i in range(n):
            c = {"engine": self.ENGINES.get(int(m[i]), str(int(m[i])))}
            if int(m[i]) == 1:
                c.update(parts=int(p[i]), groups=int(g[i]))
            else:
                c.update(bars_per_lane=int(k[i]), warps_per_block=int(w[i]))
            c["ms"] = float(ms[i])
            out.append(c)
        return out

    def close(self) -> None:
        if self.handle:
            get_lib().ct_b200_plan_destroy(self.handle)
            self.handle = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fused_batch_d(series: ctB200Series, jobs, stream: Any = None) -> None:
    arr = job_array(jobs)
    call_status(get_lib().ct_b200_fused_batch_d(ct.byref(series), arr, len(jobs), stream_arg(stream)),
                "ct_b200_fused_batch_d")


def fused_batch(series: ctB200Series, jobs, stream: Any = None) -> None:
    arr = job_array(jobs)
    call_status(get_lib().ct_b200_fused_batch(ct.byref(series), arr, len(jobs), stream_arg(stream)),
                "ct_b200_fused_batch")
