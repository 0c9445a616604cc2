// Test infrastructure only: a C-ABI bridge over the reference's own CPU code,
// compiled from the reference tree where it lies (see oracle/Makefile). It is
// used to pin the project's oracle (oracle/ta_oracle.c) and to time the
// reference's CPU path in bench.py. Nothing in the product links it.
//
// What it wraps, by reference path:
//   * src/compat/Talib08Formulas.h (+ talib08_formulas.inc): the vendored
//     TA-Lib 0.8.3 C (commit 62021c1d, third_party/ta_lib_0_8_3/PROVENANCE.json)
//     in FP64: TA_SMA, TA_EMA, TA_WMA, TA_RSI, TA_MACD, TA_ATR, TA_BBANDS,
//     TA_STOCH, TA_STDDEV, TA_VAR, TA_LINEARREG, TA_DEMA, TA_TEMA, TA_T3,
//     TA_TRANGE, TA_ROC, TA_ROCP, TA_RMA, TA_MEDPRICE, TA_TYPPRICE,
//     TA_MIDPRICE, TA_IBS, TA_MARKETFI, TA_QSTICK.
//   * include/utils/StreamStates.h: ObvState, AdState, precise::MfiState,
//     precise::AdoscState, precise::NatrState (the fused batch arithmetic).
//   * include/utils/CandleUtils.h: the cdl_*_talib pattern decisions.
// Families with no CPU code in the reference (ADX, DX, CCI, WILLR, CORREL,
// SUM, MIN, MAX) are not here; the oracle port covers them.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <limits>
#include <omp.h>

#define __host__
#define __device__
#define __forceinline__ inline
#include <src/compat/Talib08Formulas.h>
#include <include/utils/StreamStates.h>
#include <include/utils/CandleUtils.h>
#include "ref_candles.inc"

using namespace tacuda::talib08::ref;
namespace ss = tacuda::streaming;

namespace {
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

struct Row {
  std::vector<double> buf[5];
  std::vector<double> out[3];
  std::vector<unsigned char> arena;
  explicit Row(int T) {
    for (auto& b : buf) b.resize(T);
    for (auto& o : out) o.resize(T);
    arena.resize(static_cast<size_t>(T) * 64 + (1 << 20));
  }
  Arena make_arena() { return Arena{arena.data(), arena.size()}; }
};

inline void load(std::vector<double>& dst, const float* src, int T) {
  for (int t = 0; t < T; ++t) dst[t] = static_cast<double>(src[t]);
}

// Scatter a TA-Lib result (outBegIdx, outNB) into a full row with NaN warm-up.
inline void scatter(double* dst, const double* src, int T, int beg, int nb) {
  for (int t = 0; t < T; ++t) dst[t] = kNaN;
  for (int k = 0; k < nb; ++k) dst[beg + k] = src[k];
}

template <class F>
void rows(int S, int threads, F&& body) {
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
  for (int s = 0; s < S; ++s) body(s);
}
}  // namespace

extern "C" {

int ref_threads(void) { return omp_get_max_threads(); }

// One-input, one-output TA-Lib families: 0 SMA, 1 EMA, 2 WMA, 3 RSI,
// 4 STDDEV(nbdev=1), 5 VAR(nbdev=1), 6 LINEARREG, 7 DEMA, 8 TEMA, 9 T3(v=fparam),
// 10 ROC, 11 RMA, 12 ROCP.
int ref_single(int fam, const float* x, int S, int T, int p, double fparam,
               double* out, int threads) {
  int rc_all = 0;
  rows(S, threads, [&](int s) {
    Row r(T);
    load(r.buf[0], x + static_cast<size_t>(s) * T, T);
    Arena a = r.make_arena();
    int beg = 0, nb = 0;
    TA_RetCode rc = TA_SUCCESS;
    const double* in = r.buf[0].data();
    double* o = r.out[0].data();
    switch (fam) {
      case 0: rc = TA_SMA(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 1: rc = TA_EMA(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 2: rc = TA_WMA(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 3: rc = TA_RSI(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 4: rc = TA_STDDEV(a, 0, T - 1, in, p, 1.0, &beg, &nb, o); break;
      case 5: rc = TA_VAR(a, 0, T - 1, in, p, 1.0, &beg, &nb, o); break;
      case 6: rc = TA_LINEARREG(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 7: rc = TA_DEMA(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 8: rc = TA_TEMA(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 9: rc = TA_T3(a, 0, T - 1, in, p, fparam, &beg, &nb, o); break;
      case 10: rc = TA_ROC(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 11: rc = TA_RMA(a, 0, T - 1, in, p, &beg, &nb, o); break;
      case 12: rc = TA_ROCP(a, 0, T - 1, in, p, &beg, &nb, o); break;
      default: rc = TA_BAD_PARAM;
    }
    if (rc != TA_SUCCESS) { rc_all = static_cast<int>(rc); nb = 0; }
    scatter(out + static_cast<size_t>(s) * T, o, T, beg, nb);
  });
  return rc_all;
}

int ref_macd(const float* x, int S, int T, int fast, int slow, int signal,
             double* macd, double* sig, double* hist, int threads) {
  int rc_all = 0;
  rows(S, threads, [&](int s) {
    Row r(T);
    load(r.buf[0], x + static_cast<size_t>(s) * T, T);
    Arena a = r.make_arena();
    int beg = 0, nb = 0;
    TA_RetCode rc = TA_MACD(a, 0, T - 1, r.buf[0].data(), fast, slow, signal, &beg, &nb,
                            r.out[0].data(), r.out[1].data(), r.out[2].data());
    if (rc != TA_SUCCESS) { rc_all = static_cast<int>(rc); nb = 0; }
    const size_t o = static_cast<size_t>(s) * T;
    scatter(macd + o, r.out[0].data(), T, beg, nb);
    scatter(sig + o, r.out[1].data(), T, beg, nb);
    scatter(hist + o, r.out[2].data(), T, beg, nb);
  });
  return rc_all;
}

int ref_bbands(const float* x, int S, int T, int p, double up, double dn,
               double* upper, double* middle, double* lower, int threads) {
  int rc_all = 0;
  rows(S, threads, [&](int s) {
    Row r(T);
    load(r.buf[0], x + static_cast<size_t>(s) * T, T);
    Arena a = r.make_arena();
    int beg = 0, nb = 0;
    TA_RetCode rc = TA_BBANDS(a, 0, T - 1, r.buf[0].data(), p, up, dn, 0, &beg, &nb,
                              r.out[0].data(), r.out[1].data(), r.out[2].data());
    if (rc != TA_SUCCESS) { rc_all = static_cast<int>(rc); nb = 0; }
    const size_t o = static_cast<size_t>(s) * T;
    scatter(upper + o, r.out[0].data(), T, beg, nb);
    scatter(middle + o, r.out[1].data(), T, beg, nb);
    scatter(lower + o, r.out[2].data(), T, beg, nb);
  });
  return rc_all;
}

// HLC families: 0 ATR(p), 1 TRANGE, 2 STOCH(k=p, slowK=q, slowD=q; two outputs).
int ref_hlc(int fam, const float* h, const float* l, const float* c, int S, int T,
            int p, int q, double* out0, double* out1, int threads) {
  int rc_all = 0;
  rows(S, threads, [&](int s) {
    Row r(T);
    const size_t o = static_cast<size_t>(s) * T;
    load(r.buf[0], h + o, T); load(r.buf[1], l + o, T); load(r.buf[2], c + o, T);
    Arena a = r.make_arena();
    int beg = 0, nb = 0;
    TA_RetCode rc = TA_SUCCESS;
    switch (fam) {
      case 0: rc = TA_ATR(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), r.buf[2].data(), p,
                          &beg, &nb, r.out[0].data()); break;
      case 1: rc = TA_TRANGE(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), r.buf[2].data(),
                             &beg, &nb, r.out[0].data()); break;
      case 2: rc = TA_STOCH(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), r.buf[2].data(),
                            p, q, 0, q, 0, &beg, &nb, r.out[0].data(), r.out[1].data()); break;
      default: rc = TA_BAD_PARAM;
    }
    if (rc != TA_SUCCESS) { rc_all = static_cast<int>(rc); nb = 0; }
    scatter(out0 + o, r.out[0].data(), T, beg, nb);
    if (fam == 2 && out1) scatter(out1 + o, r.out[1].data(), T, beg, nb);
  });
  return rc_all;
}

// Price transforms and per-bar functions: 0 MEDPRICE(h,l), 1 TYPPRICE(h,l,c),
// 2 MIDPRICE(h,l; p), 3 IBS(h,l,c), 4 MARKETFI(h,l,v) (c carries v),
// 5 QSTICK(open, close; p) (h carries open, l close).
int ref_price(int fam, const float* h, const float* l, const float* c, int S, int T, int p,
              double* out, int threads) {
  int rc_all = 0;
  rows(S, threads, [&](int s) {
    Row r(T);
    const size_t o = static_cast<size_t>(s) * T;
    load(r.buf[0], h + o, T); load(r.buf[1], l + o, T);
    if (fam == 1 || fam == 3 || fam == 4) load(r.buf[2], c + o, T);
    Arena a = r.make_arena();
    int beg = 0, nb = 0;
    TA_RetCode rc = TA_SUCCESS;
    switch (fam) {
      case 0: rc = TA_MEDPRICE(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), &beg, &nb, r.out[0].data()); break;
      case 1: rc = TA_TYPPRICE(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), r.buf[2].data(), &beg, &nb,
                               r.out[0].data()); break;
      case 2: rc = TA_MIDPRICE(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), p, &beg, &nb, r.out[0].data()); break;
      case 3: rc = TA_IBS(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), r.buf[2].data(), &beg, &nb, r.out[0].data()); break;
      case 5: rc = TA_QSTICK(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), p, &beg, &nb, r.out[0].data()); break;
      case 4: rc = TA_MARKETFI(a, 0, T - 1, r.buf[0].data(), r.buf[1].data(), r.buf[2].data(), &beg, &nb,
                               r.out[0].data()); break;
      default: rc = TA_BAD_PARAM;
    }
    if (rc != TA_SUCCESS) { rc_all = static_cast<int>(rc); nb = 0; }
    scatter(out + o, r.out[0].data(), T, beg, nb);
  });
  return rc_all;
}

// StreamStates families (float outputs exactly as the reference rounds them):
// 0 OBV(close, volume), 1 AD(h,l,c,v), 2 MFI(h,l,c,v; p), 3 ADOSC(h,l,c,v; p=fast, q=slow),
// 4 NATR(h,l,c; p).
int ref_states(int fam, const float* h, const float* l, const float* c, const float* v,
               int S, int T, int p, int q, float* out, int threads) {
  rows(S, threads, [&](int s) {
    const size_t o = static_cast<size_t>(s) * T;
    std::vector<double> ring(2 * (p > 0 ? p : 1) + 2, 0.0);
    ss::ObvState obv; ss::AdState ad; ss::precise::MfiState mfi;
    ss::precise::AdoscState adosc; ss::precise::NatrState natr;
    obv.init(); ad.init();
    if (fam == 2) mfi.init(p);
    if (fam == 3) adosc.init(p, q);
    if (fam == 4) natr.init(p);
    for (int t = 0; t < T; ++t) {
      ss::StreamBar b{};
      b.close = c[o + t];
      if (h) b.high = h[o + t];
      if (l) b.low = l[o + t];
      if (v) b.volume = v[o + t];
      float y = 0.0f;
      switch (fam) {
        case 0: obv.step(nullptr, b, &y); break;
        case 1: ad.step(nullptr, b, &y); break;
        case 2: mfi.step(ring.data(), b, &y); break;
        case 3: adosc.step(nullptr, b, &y); break;
        case 4: natr.step(nullptr, b, &y); break;
        default: y = std::numeric_limits<float>::quiet_NaN();
      }
      out[o + t] = y;
    }
  });
  return 0;
}

// Candle patterns through CandleUtils.h (see ref_candles.inc for the table).
int ref_cdl(int pattern, const float* op, const float* hi, const float* lo, const float* cl,
            int S, int T, int* out, int threads) {
  if (pattern < 0 || pattern >= kRefCandleCount) return -1;
  rows(S, threads, [&](int s) {
    const size_t o = static_cast<size_t>(s) * T;
    ref_candle_row(pattern, op + o, hi + o, lo + o, cl + o, T, out + o);
  });
  return 0;
}

int ref_cdl_count(void) { return kRefCandleCount; }

}  // extern "C"
