"""CPU: the C-ABI library loads and exports exactly what include/tacuda.h
declares; argument validation needs no GPU."""
import ctypes as ct
import re
from pathlib import Path

import pytest

import tacuda_b200 as tb

ROOT = Path(__file__).resolve().parents[1]
HEADER = (ROOT / "include" / "tacuda.h").read_text()
DECLARED = sorted(set(re.findall(r"CTAPI_EXPORT\s+[\w\s\*]+?\b(ct_\w+)\s*\(", HEADER)))


def test_header_declares_reference_surface():
    # the reference batch entry points of the hot path are all declared
    for fam in ("sma", "ema", "wma", "rsi", "macd", "atr", "natr", "adx", "dx", "bbands", "stochastic", "cci",
                "obv", "ad", "adosc", "mfi", "willr", "sum", "min", "max", "stddev", "var", "linearreg", "correl",
                "dema", "tema", "t3", "trange"):
        assert f"ct_{fam}_batch_d" in DECLARED
        assert f"ct_{fam}_d" in DECLARED
    assert sum(1 for s in DECLARED if s.startswith("ct_cdl_") and s.endswith("_batch_d")) == 63
    assert len(DECLARED) > 200


@pytest.mark.parametrize("sym", DECLARED)
def test_every_declared_symbol_is_exported(sym):
    assert hasattr(tb.get_lib(), sym), sym


def test_status_strings_and_version():
    assert tb.status_string(0) == "success"
    assert tb.status_string(4) == "invalid argument"
    assert tb.version().startswith("0.9.3")
    assert len(tb.cdl_names()) == 63 and tb.cdl_names()[0] == "doji"
    assert [tb.cdl_lookback(k) for k in (0, 1, 3, 22, 31, 62)] == [10, 11, 1, 2, 5, 2]


def test_invalid_arguments_need_no_gpu():
    lib = tb.get_lib()
    P, I = ct.c_void_p, ct.c_int
    # null pointers and bad sizes are rejected before any CUDA call
    assert lib.ct_sma_batch_d(P(0), P(0), I(10), I(2), I(3), I(0), P(0)) == 4
    assert "null pointer or invalid size" in tb.get_last_error()
    fake = P(0x1000)
    assert lib.ct_sma_batch_d(fake, fake, I(0), I(2), I(3), I(0), P(0)) == 4
    assert lib.ct_sma_batch_d(fake, fake, I(10), I(-1), I(3), I(0), P(0)) == 4
    assert lib.ct_rsi_batch_d(fake, fake, I(10), I(2), I(0), I(0), P(0)) == 4
    assert "invalid period" in tb.get_last_error()
    assert lib.ct_macd_batch_d(fake, fake, fake, fake, I(10), I(2), I(12), I(26), I(9), I(0), I(0), P(0)) == 6
    assert lib.ct_stochastic_batch_d(fake, fake, fake, fake, fake, I(10), I(2), I(14), I(0), I(0), P(0)) == 4
    assert lib.ct_cdl_doji_batch_d(P(0), fake, fake, fake, fake, I(10), I(2), I(0), P(0)) == 4


def test_error_state_is_thread_local():
    import threading
    lib = tb.get_lib()
    P, I = ct.c_void_p, ct.c_int
    assert lib.ct_sma_batch_d(P(0), P(0), I(10), I(2), I(3), I(0), P(0)) == 4
    seen = []
    t = threading.Thread(target=lambda: seen.append(tb.get_last_error()))
    t.start(); t.join()
    assert seen == [""] and tb.get_last_error() != ""


def test_fused_job_validation():
    s = tb.make_series({"close": 0x1000}, 4, 100)
    with pytest.raises(RuntimeError, match="invalid period"):
        tb.fused_batch_d(s, [tb.make_job("sma", (0,), (), [0x2000])])
    with pytest.raises(RuntimeError, match="null input"):
        tb.fused_batch_d(s, [tb.make_job("atr", (14,), (), [0x2000])])
    with pytest.raises(RuntimeError, match="bad candle mask"):
        tb.fused_batch_d(tb.make_series({k: 0x1000 for k in ("open", "high", "low", "close")}, 4, 100),
                         [tb.make_job("cdl", (), (), [0x2000], cdl_mask=0)])


def test_appended_families_validate_like_the_reference():
    lib = tb.get_lib()
    P, I = ct.c_void_p, ct.c_int
    fake = P(0x1000)
    # ROC.cu / Momentum.cu / MIDPRICE.cu / MIDPOINT.cu: period <= 0 is invalid
    for name in ("roc", "rocp", "rocr", "rocr100", "momentum", "change", "rma", "midpoint"):
        assert getattr(lib, f"ct_{name}_batch_d")(fake, fake, I(10), I(2), I(0), I(0), P(0)) == 4, name
        assert "invalid period" in tb.get_last_error()
    assert lib.ct_midprice_batch_d(fake, fake, fake, I(10), I(2), I(-3), I(0), P(0)) == 4
    # Aroon.cu throws on period <= 0; the reference's ct_aroon_d turns every
    # exception into KERNEL_FAILED, its ct_aroonosc_d classifies it as invalid
    assert lib.ct_aroon_batch_d(fake, fake, fake, fake, I(10), I(2), I(0), I(0), P(0)) == 3
    assert lib.ct_aroonosc_batch_d(fake, fake, fake, I(10), I(2), I(0), I(0), P(0)) == 4
    # TA_RMA's period range ends at 100000
    assert lib.ct_rma_batch_d(fake, fake, I(10), I(2), I(100001), I(0), P(0)) == 4
    # staged windows end at 4096 bars
    assert lib.ct_roc_batch_d(fake, fake, I(10), I(2), I(4097), I(0), P(0)) == 6
    # ClubPack.cu:409-413: a rolling period above the row length is invalid
    for name in ("rolling_mean", "rolling_max", "rolling_min", "rolling_std"):
        assert getattr(lib, f"ct_{name}_batch_d")(fake, fake, I(10), I(2), I(11), I(0), P(0)) == 4, name
        assert getattr(lib, f"ct_{name}_d")(fake, fake, I(10), I(11), P(0)) == 4, name
    # null pointers, as for every entry
    assert lib.ct_medprice_batch_d(P(0), fake, fake, I(10), I(2), I(0), P(0)) == 4
    assert lib.ct_avgprice_batch_d(fake, fake, P(0), fake, fake, I(10), I(2), I(0), P(0)) == 4
    assert lib.ct_typprice_d(fake, fake, fake, P(0), I(10), P(0)) == 4
    assert lib.ct_wclprice_batch_d(fake, fake, fake, fake, I(0), I(2), I(0), P(0)) == 4
