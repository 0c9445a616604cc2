// Host-side facts about one job that every engine's launcher needs: the
// input planes it reads, the bars of history it reads before a chunk or round,
// its look-back descriptor slots and the FP64 lines the warp-scan engine keeps.
#pragma once

#include "engine.h"

namespace tb {

// Look-back descriptor slots of a job: one per first-index carry and one per
// recurrence stage, in the order the round functions address them.
inline int lb_slots(const Job& j) {
  switch (j.family) {
    case F_EMA: case F_RMA: return 2;
    case F_QSTICK: return 3;
    case F_DEMA: return 3;
    case F_TEMA: return 4;
    case F_T3: return 7;
    case F_RSI: return 2;
    case F_MACD: return 4;
    case F_ATR: case F_NATR: return 1;
    case F_ADX: return 2;
    case F_DX: return 1;
    case F_OBV: case F_AD: return 1;
    case F_ADOSC: return 3;
    case F_MIN: case F_MAX: case F_CORREL: case F_MIDPOINT: case F_IBS: case F_MARKETFI: return 1;
    default: return 0;
  }
}

inline int job_halo(const Job& j) {
  switch (j.family) {
    case F_SMA: case F_SUM: case F_WMA: case F_BBANDS: case F_STDDEV: case F_VAR:
    case F_LINEARREG: case F_MIN: case F_MAX: case F_WILLR: case F_CCI: case F_CORREL:
      return j.ip[0] - 1;
    case F_MFI: case F_ROC: case F_ROCP: case F_ROCR: case F_ROCR100: case F_MOM: return j.ip[0];
    case F_MIDPOINT: case F_RMEAN: case F_RMAX: case F_RMIN: case F_RSTD: case F_QSTICK: return j.ip[0] - 1;
    case F_MIDPRICE: return j.ip[0] - 1;
    case F_AROON: case F_AROONOSC: return j.ip[0];
    case F_STOCH: return j.ip[0] - 1 + 2 * (j.ip[1] - 1);
    case F_CDL: return 16;  // 10-bar averages anchored up to 5 bars back
    default: return 1;  // previous bar
  }
}

inline unsigned job_planes(const Job& j) {
  unsigned m = 0;
  int n = 0;
  switch (j.family) {
    case F_SMA: case F_EMA: case F_WMA: case F_RSI: case F_MACD: case F_BBANDS: case F_SUM:
    case F_MIN: case F_MAX: case F_STDDEV: case F_VAR: case F_LINEARREG: case F_DEMA:
    case F_TEMA: case F_T3: case F_ROC: case F_RMA: case F_ROCP: case F_ROCR: case F_ROCR100:
    case F_MOM: case F_MIDPOINT: case F_RMEAN: case F_RMAX: case F_RMIN: case F_RSTD:
      n = 1; break;
    case F_OBV: case F_CORREL: case F_MEDPRICE: case F_MIDPRICE: case F_QSTICK: case F_AROON: case F_AROONOSC:
      n = 2; break;
    case F_ATR: case F_NATR: case F_TRANGE: case F_ADX: case F_DX: case F_STOCH: case F_WILLR:
    case F_TYPPRICE: case F_WCLPRICE: case F_IBS: case F_MARKETFI:
      n = 3; break;
    case F_CCI: n = 3; break;
    case F_AD: case F_ADOSC: case F_MFI: case F_CDL: case F_AVGPRICE: n = 4; break;
    default: n = 0;
  }
  for (int i = 0; i < n; ++i) m |= 1u << j.in[i];
  return m;
}

inline int job_lines(const Job& j) {
  switch (j.family) {
    case F_MACD: case F_ADX: case F_DX: case F_STOCH: return 1;
    case F_ADOSC: return 2;
    case F_DEMA: return 2;
    case F_TEMA: return 3;
    case F_T3: return 4;
    default: return 0;
  }
}

}  // namespace tb
