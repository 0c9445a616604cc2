// TA-Lib's 61 candlestick pattern rules (plus the reference's legacy bullish /
// bearish engulfing split) as templates over a bar view B, which provides the
// bars before the current one (O/H/L/C(d), d bars back), their real body and
// shadows in FP64, and AVG(setting, d): TA-Lib's candle average of a setting
// anchored d bars back (include/utils/CandleUtils.h:37-63, 1466-1495).
// The candle tile kernel (candles.cuh) supplies the view.
#pragma once

#include "common.cuh"
#include "engine.h"

namespace tb {
namespace rules {

enum CdlRange { CR_BODY = 0, CR_HL = 1, CR_SHADOW = 2 };
enum CdlSet {
  BODY_LONG = 0, BODY_VERY_LONG, BODY_SHORT, BODY_DOJI, SHADOW_LONG, SHADOW_VERY_LONG, SHADOW_SHORT,
  SHADOW_VERY_SHORT, NEAR, FAR, EQUAL
};
// averaging period of each range slot (body/10, high-low/10, shadows/10,
// high-low/5)
__device__ __constant__ const int kSlotPeriod[4] = {10, 10, 10, 5};
// range slot (-1: the bar itself) and factor of each setting, as constant
// expressions: the pattern functions pass literal settings, so these fold at
// compile time.
__host__ __device__ constexpr int set_slot(int s) {
  return s <= 2 ? 0 : s == 3 ? 1 : s <= 5 ? -1 : s == 6 ? 2 : s == 7 ? 1 : 3;
}
__host__ __device__ constexpr float set_factor(int s) {
  return s == 0 ? 1.0f : s == 1 ? 3.0f : s == 2 ? 1.0f : s == 3 ? 0.1f : s == 4 ? 1.0f : s == 5 ? 2.0f
       : s == 6 ? 1.0f : s == 7 ? 0.1f : s == 8 ? 0.2f : s == 9 ? 0.6f : 0.05f;
}

constexpr int kCdlBack = 5;  // anchors r-5 .. r (HIKKAKEMOD reads NEAR at r-5)

__device__ __forceinline__ double cdl_range(int type, float o, float h, float l, float c) {
  const double od = o, hd = h, ld = l, cd = c;
  if (type == CR_BODY) return fabs(cd - od);
  if (type == CR_HL) return hd - ld;
  return (hd - fmax(od, cd)) + (fmin(od, cd) - ld);
}

#define CDL_FN(name) template <class B> __device__ __forceinline__ int name(const B& b)

CDL_FN(c_two_crows) {
  return (b.COL(2) == 1 && b.RB(2) > b.AVG(BODY_LONG, 2) && b.COL(1) == -1 && b.BGAP_UP(1, 2) && b.COL(0) == -1 &&
          b.O(0) < b.O(1) && b.O(0) > b.C(1) && b.C(0) > b.O(2) && b.C(0) < b.C(2)) ? -100 : 0;
}
CDL_FN(c_three_black_crows) {
  return (b.COL(3) == 1 && b.COL(2) == -1 && b.LS(2) < b.AVG(SHADOW_VERY_SHORT, 2) && b.COL(1) == -1 &&
          b.LS(1) < b.AVG(SHADOW_VERY_SHORT, 1) && b.COL(0) == -1 && b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
          b.O(1) < b.O(2) && b.O(1) > b.C(2) && b.O(0) < b.O(1) && b.O(0) > b.C(1) && b.H(3) > b.C(2) &&
          b.C(2) > b.C(1) && b.C(1) > b.C(0)) ? -100 : 0;
}
CDL_FN(c_three_inside) {
  if (b.RB(2) > b.AVG(BODY_LONG, 2) && b.RB(1) <= b.AVG(BODY_SHORT, 1) &&
      fmaxf(b.C(1), b.O(1)) < fmaxf(b.C(2), b.O(2)) && fminf(b.C(1), b.O(1)) > fminf(b.C(2), b.O(2)) &&
      ((b.COL(2) == 1 && b.COL(0) == -1 && b.C(0) < b.O(2)) || (b.COL(2) == -1 && b.COL(0) == 1 && b.C(0) > b.O(2))))
    return -b.COL(2) * 100;
  return 0;
}
CDL_FN(c_three_line_strike) {
  if (b.COL(3) == b.COL(2) && b.COL(2) == b.COL(1) && b.COL(0) == -b.COL(1) &&
      (double)b.O(2) >= (double)b.BOT(3) - b.AVG(NEAR, 3) && (double)b.O(2) <= (double)b.TOP(3) + b.AVG(NEAR, 3) &&
      (double)b.O(1) >= (double)b.BOT(2) - b.AVG(NEAR, 2) && (double)b.O(1) <= (double)b.TOP(2) + b.AVG(NEAR, 2) &&
      ((b.COL(1) == 1 && b.C(1) > b.C(2) && b.C(2) > b.C(3) && b.O(0) > b.C(1) && b.C(0) < b.O(3)) ||
       (b.COL(1) == -1 && b.C(1) < b.C(2) && b.C(2) < b.C(3) && b.O(0) < b.C(1) && b.C(0) > b.O(3))))
    return b.COL(1) * 100;
  return 0;
}
CDL_FN(c_three_outside) {
  if ((b.COL(1) == 1 && b.COL(2) == -1 && b.C(1) > b.O(2) && b.O(1) < b.C(2) && b.C(0) > b.C(1)) ||
      (b.COL(1) == -1 && b.COL(2) == 1 && b.O(1) > b.C(2) && b.C(1) < b.O(2) && b.C(0) < b.C(1)))
    return b.COL(1) * 100;
  return 0;
}
CDL_FN(c_three_stars_in_south) {
  return (b.COL(2) == -1 && b.COL(1) == -1 && b.COL(0) == -1 && b.RB(2) > b.AVG(BODY_LONG, 2) &&
          b.LS(2) > b.AVG(SHADOW_LONG, 2) && b.RB(1) < b.RB(2) && b.O(1) > b.C(2) && b.O(1) <= b.H(2) &&
          b.L(1) < b.C(2) && b.L(1) >= b.L(2) && b.LS(1) > b.AVG(SHADOW_VERY_SHORT, 1) &&
          b.RB(0) < b.AVG(BODY_SHORT, 0) && b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
          b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0) && b.L(0) > b.L(1) && b.H(0) < b.H(1)) ? 100 : 0;
}
CDL_FN(c_three_white_soldiers) {
  return (b.COL(2) == 1 && b.US(2) < b.AVG(SHADOW_VERY_SHORT, 2) && b.COL(1) == 1 &&
          b.US(1) < b.AVG(SHADOW_VERY_SHORT, 1) && b.COL(0) == 1 && b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
          b.C(0) > b.C(1) && b.C(1) > b.C(2) && b.O(1) > b.O(2) &&
          (double)b.O(1) <= (double)b.C(2) + b.AVG(NEAR, 2) && b.O(0) > b.O(1) &&
          (double)b.O(0) <= (double)b.C(1) + b.AVG(NEAR, 1) && b.RB(1) > b.RB(2) - b.AVG(FAR, 2) &&
          b.RB(0) > b.RB(1) - b.AVG(FAR, 1) && b.RB(0) > b.AVG(BODY_SHORT, 0)) ? 100 : 0;
}
CDL_FN(c_abandoned_baby) {
  const double pen = 0.3;
  if (b.RB(2) > b.AVG(BODY_LONG, 2) && b.RB(1) <= b.AVG(BODY_DOJI, 1) && b.RB(0) > b.AVG(BODY_SHORT, 0) &&
      ((b.COL(2) == 1 && b.COL(0) == -1 && b.C(0) < b.C(2) - b.RB(2) * pen && b.RGAP_UP(1, 2) && b.RGAP_DN(0, 1)) ||
       (b.COL(2) == -1 && b.COL(0) == 1 && b.C(0) > b.C(2) + b.RB(2) * pen && b.RGAP_DN(1, 2) && b.RGAP_UP(0, 1))))
    return b.COL(0) * 100;
  return 0;
}
CDL_FN(c_advance_block) {
  if (b.COL(2) == 1 && b.COL(1) == 1 && b.COL(0) == 1 && b.C(0) > b.C(1) && b.C(1) > b.C(2) && b.O(1) > b.O(2) &&
      b.O(1) <= b.C(2) + b.AVG(NEAR, 2) && b.O(0) > b.O(1) && b.O(0) <= b.C(1) + b.AVG(NEAR, 1) &&
      b.RB(2) > b.AVG(BODY_LONG, 2) && b.US(2) < b.AVG(SHADOW_SHORT, 2) &&
      ((b.RB(1) < b.RB(2) - b.AVG(FAR, 2) && b.RB(0) < b.RB(1) + b.AVG(NEAR, 1)) ||
       (b.RB(0) < b.RB(1) - b.AVG(FAR, 1)) ||
       (b.RB(0) < b.RB(1) && b.RB(1) < b.RB(2) &&
        (b.US(0) > b.AVG(SHADOW_SHORT, 0) || b.US(1) > b.AVG(SHADOW_SHORT, 1))) ||
       (b.RB(0) < b.RB(1) && b.US(0) > b.AVG(SHADOW_LONG, 0))))
    return -100;
  return 0;
}
CDL_FN(c_belt_hold) {
  if (b.RB(0) > b.AVG(BODY_LONG, 0) && ((b.COL(0) == 1 && b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0)) ||
                                         (b.COL(0) == -1 && b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0))))
    return b.COL(0) * 100;
  return 0;
}
CDL_FN(c_breakaway) {
  if (b.RB(4) > b.AVG(BODY_LONG, 4) && b.COL(4) == b.COL(3) && b.COL(3) == b.COL(1) && b.COL(1) == -b.COL(0) &&
      ((b.COL(4) == -1 && b.BGAP_DN(3, 4) && b.H(2) < b.H(3) && b.L(2) < b.L(3) && b.H(1) < b.H(2) &&
        b.L(1) < b.L(2) && b.C(0) > b.O(3) && b.C(0) < b.C(4)) ||
       (b.COL(4) == 1 && b.BGAP_UP(3, 4) && b.H(2) > b.H(3) && b.L(2) > b.L(3) && b.H(1) > b.H(2) &&
        b.L(1) > b.L(2) && b.C(0) < b.O(3) && b.C(0) > b.C(4))))
    return b.COL(0) * 100;
  return 0;
}
CDL_FN(c_closing_marubozu) {
  if (b.RB(0) > b.AVG(BODY_LONG, 0) && ((b.COL(0) == 1 && b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0)) ||
                                         (b.COL(0) == -1 && b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0))))
    return b.COL(0) * 100;
  return 0;
}
CDL_FN(c_conceal_baby_swallow) {
  return (b.COL(3) == -1 && b.COL(2) == -1 && b.COL(1) == -1 && b.COL(0) == -1 &&
          b.LS(3) < b.AVG(SHADOW_VERY_SHORT, 3) && b.US(3) < b.AVG(SHADOW_VERY_SHORT, 3) &&
          b.LS(2) < b.AVG(SHADOW_VERY_SHORT, 2) && b.US(2) < b.AVG(SHADOW_VERY_SHORT, 2) && b.BGAP_DN(1, 2) &&
          b.US(1) > b.AVG(SHADOW_VERY_SHORT, 1) && b.H(1) > b.C(2) && b.H(0) > b.H(1) && b.L(0) < b.L(1)) ? 100 : 0;
}
CDL_FN(c_counterattack) {
  if (b.COL(1) == -b.COL(0) && b.RB(1) > b.AVG(BODY_LONG, 1) && b.RB(0) > b.AVG(BODY_LONG, 0) &&
      b.C(0) <= b.C(1) + b.AVG(EQUAL, 1) && b.C(0) >= b.C(1) - b.AVG(EQUAL, 1))
    return b.COL(0) * 100;
  return 0;
}
CDL_FN(c_dark_cloud_cover) {
  return (b.COL(1) == 1 && b.RB(1) > b.AVG(BODY_LONG, 1) && b.COL(0) == -1 && b.O(0) > b.H(1) && b.C(0) > b.O(1) &&
          (double)b.C(0) < (double)b.C(1) - b.RB(1) * 0.5) ? -100 : 0;
}
CDL_FN(c_doji) { return b.RB(0) <= b.AVG(BODY_DOJI, 0) ? 100 : 0; }
CDL_FN(c_doji_star) {
  if (b.RB(1) > b.AVG(BODY_LONG, 1) && b.RB(0) <= b.AVG(BODY_DOJI, 0) &&
      ((b.COL(1) == 1 && b.BGAP_UP(0, 1)) || (b.COL(1) == -1 && b.BGAP_DN(0, 1))))
    return -b.COL(1) * 100;
  return 0;
}
CDL_FN(c_dragonfly_doji) {
  return (b.RB(0) <= b.AVG(BODY_DOJI, 0) && b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
          b.LS(0) > b.AVG(SHADOW_VERY_SHORT, 0)) ? 100 : 0;
}
CDL_FN(c_engulfing) {
  const bool white = b.COL(0) == 1 && b.COL(1) == -1 &&
                     ((b.C(0) >= b.O(1) && b.O(0) < b.C(1)) || (b.C(0) > b.O(1) && b.O(0) <= b.C(1)));
  const bool black = b.COL(0) == -1 && b.COL(1) == 1 &&
                     ((b.O(0) >= b.C(1) && b.C(0) < b.O(1)) || (b.O(0) > b.C(1) && b.C(0) <= b.O(1)));
  if (white || black) return (b.O(0) != b.C(1) && b.C(0) != b.O(1)) ? b.COL(0) * 100 : b.COL(0) * 80;
  return 0;
}
template <class B>
__device__ __forceinline__ bool star_shape(const B& b, bool doji_middle, bool bull) {
  const double pen = 0.3;
  const bool mid = doji_middle ? b.RB(1) <= b.AVG(BODY_DOJI, 1) : b.RB(1) <= b.AVG(BODY_SHORT, 1);
  if (bull)
    return b.RB(2) > b.AVG(BODY_LONG, 2) && b.COL(2) == -1 && mid && b.BGAP_DN(1, 2) &&
           b.RB(0) > b.AVG(BODY_SHORT, 0) && b.COL(0) == 1 && (double)b.C(0) > (double)b.C(2) + b.RB(2) * pen;
  return b.RB(2) > b.AVG(BODY_LONG, 2) && b.COL(2) == 1 && mid && b.BGAP_UP(1, 2) &&
         b.RB(0) > b.AVG(BODY_SHORT, 0) && b.COL(0) == -1 && (double)b.C(0) < (double)b.C(2) - b.RB(2) * pen;
}
CDL_FN(c_evening_doji_star) { return star_shape(b, true, false) ? -100 : 0; }
CDL_FN(c_evening_star) { return star_shape(b, false, false) ? -100 : 0; }
CDL_FN(c_morning_doji_star) { return star_shape(b, true, true) ? 100 : 0; }
CDL_FN(c_morning_star) { return star_shape(b, false, true) ? 100 : 0; }
CDL_FN(c_gap_side_side_white) {
  if (((b.BGAP_UP(1, 2) && b.BGAP_UP(0, 2)) || (b.BGAP_DN(1, 2) && b.BGAP_DN(0, 2))) && b.COL(1) == 1 &&
      b.COL(0) == 1 && b.RB(0) >= b.RB(1) - b.AVG(NEAR, 1) && b.RB(0) <= b.RB(1) + b.AVG(NEAR, 1) &&
      b.O(0) >= b.O(1) - b.AVG(EQUAL, 1) && b.O(0) <= b.O(1) + b.AVG(EQUAL, 1))
    return b.BGAP_UP(1, 2) ? 100 : -100;
  return 0;
}
CDL_FN(c_gravestone_doji) {
  return (b.RB(0) <= b.AVG(BODY_DOJI, 0) && b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
          b.US(0) > b.AVG(SHADOW_VERY_SHORT, 0)) ? 100 : 0;
}
template <class B>
__device__ __forceinline__ bool hammer_shape(const B& b) {
  return b.RB(0) < b.AVG(BODY_SHORT, 0) && b.LS(0) > b.AVG(SHADOW_LONG, 0) && b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0);
}
CDL_FN(c_hammer) {
  return (hammer_shape(b) && (double)fminf(b.C(0), b.O(0)) <= (double)b.L(1) + b.AVG(NEAR, 1)) ? 100 : 0;
}
CDL_FN(c_hanging_man) {
  return (hammer_shape(b) && (double)fminf(b.C(0), b.O(0)) >= (double)b.H(1) - b.AVG(NEAR, 1)) ? -100 : 0;
}
template <class B>
__device__ __forceinline__ int harami_common(const B& b, bool cross) {
  const bool small = cross ? b.RB(0) <= b.AVG(BODY_DOJI, 0) : b.RB(0) <= b.AVG(BODY_SHORT, 0);
  if (b.RB(1) > b.AVG(BODY_LONG, 1) && small) {
    const float hi2 = fmaxf(b.C(0), b.O(0)), lo2 = fminf(b.C(0), b.O(0));
    const float hi1 = fmaxf(b.C(1), b.O(1)), lo1 = fminf(b.C(1), b.O(1));
    if (hi2 < hi1 && lo2 > lo1) return -b.COL(1) * 100;
    if (hi2 <= hi1 && lo2 >= lo1) return -b.COL(1) * 80;
  }
  return 0;
}
CDL_FN(c_harami) { return harami_common(b, false); }
CDL_FN(c_harami_cross) { return harami_common(b, true); }
CDL_FN(c_high_wave) {
  return (b.RB(0) < b.AVG(BODY_SHORT, 0) && b.US(0) > b.AVG(SHADOW_VERY_LONG, 0) &&
          b.LS(0) > b.AVG(SHADOW_VERY_LONG, 0)) ? b.COL(0) * 100 : 0;
}
// HIKKAKE / HIKKAKEMOD: the pattern bar, or its confirmation within three bars
// (first confirming close only), CandleUtils.h:1849-1895.
template <class B>
__device__ __forceinline__ int hikkake_at(const B& b, int d) {
  if (b.H(d + 1) < b.H(d + 2) && b.L(d + 1) > b.L(d + 2) &&
      ((b.H(d) < b.H(d + 1) && b.L(d) < b.L(d + 1)) || (b.H(d) > b.H(d + 1) && b.L(d) > b.L(d + 1))))
    return b.H(d) < b.H(d + 1) ? 100 : -100;
  return 0;
}
template <class B>
__device__ __forceinline__ int hikkake_mod_at(const B& b, int d) {
  if (b.H(d + 2) < b.H(d + 3) && b.L(d + 2) > b.L(d + 3) && b.H(d + 1) < b.H(d + 2) && b.L(d + 1) > b.L(d + 2) &&
      ((b.H(d) < b.H(d + 1) && b.L(d) < b.L(d + 1) && b.C(d + 2) <= b.L(d + 2) + b.AVG(NEAR, d + 2)) ||
       (b.H(d) > b.H(d + 1) && b.L(d) > b.L(d + 1) && b.C(d + 2) >= b.H(d + 2) - b.AVG(NEAR, d + 2))))
    return b.H(d) < b.H(d + 1) ? 100 : -100;
  return 0;
}
template <class B>
__device__ __forceinline__ int hikkake_confirm(const B& b, bool modified) {
  const int pat = modified ? hikkake_mod_at(b, 0) : hikkake_at(b, 0);
  if (pat != 0) return pat;
  const long long lowest = modified ? 3 : 2;
  for (int d = 1; d <= 3 && b.t - d >= lowest; ++d) {
    const int pj = modified ? hikkake_mod_at(b, d) : hikkake_at(b, d);
    if (pj == 0) continue;
    for (int m = d - 1; m >= 0; --m) {
      const bool conf = (pj > 0 && b.C(m) > b.H(d + 1)) || (pj < 0 && b.C(m) < b.L(d + 1));
      if (conf) return m == 0 ? pj + (pj > 0 ? 100 : -100) : 0;
    }
    return 0;
  }
  return 0;
}
CDL_FN(c_hikkake) { return hikkake_confirm(b, false); }
CDL_FN(c_hikkake_mod) { return hikkake_confirm(b, true); }
CDL_FN(c_homing_pigeon) {
  return (b.COL(1) == -1 && b.COL(0) == -1 && b.RB(1) > b.AVG(BODY_LONG, 1) && b.RB(0) <= b.AVG(BODY_SHORT, 0) &&
          b.O(0) < b.O(1) && b.C(0) > b.C(1)) ? 100 : 0;
}
CDL_FN(c_identical_three_crows) {
  return (b.COL(2) == -1 && b.LS(2) < b.AVG(SHADOW_VERY_SHORT, 2) && b.COL(1) == -1 &&
          b.LS(1) < b.AVG(SHADOW_VERY_SHORT, 1) && b.COL(0) == -1 && b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
          b.C(2) > b.C(1) && b.C(1) > b.C(0) && (double)b.O(1) <= (double)b.C(2) + b.AVG(EQUAL, 2) &&
          (double)b.O(1) >= (double)b.C(2) - b.AVG(EQUAL, 2) && (double)b.O(0) <= (double)b.C(1) + b.AVG(EQUAL, 1) &&
          (double)b.O(0) >= (double)b.C(1) - b.AVG(EQUAL, 1)) ? -100 : 0;
}
CDL_FN(c_in_neck) {
  return (b.COL(1) == -1 && b.RB(1) > b.AVG(BODY_LONG, 1) && b.COL(0) == 1 && b.O(0) < b.L(1) &&
          (double)b.C(0) <= (double)b.C(1) + b.AVG(EQUAL, 1) && b.C(0) >= b.C(1)) ? -100 : 0;
}
CDL_FN(c_inverted_hammer) {
  return (b.RB(0) < b.AVG(BODY_SHORT, 0) && b.US(0) > b.AVG(SHADOW_LONG, 0) &&
          b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0) && b.BGAP_DN(0, 1)) ? 100 : 0;
}
template <class B>
__device__ __forceinline__ bool kicking_common(const B& b) {
  return b.COL(1) == -b.COL(0) && b.RB(1) > b.AVG(BODY_LONG, 1) && b.US(1) < b.AVG(SHADOW_VERY_SHORT, 1) &&
         b.LS(1) < b.AVG(SHADOW_VERY_SHORT, 1) && b.RB(0) > b.AVG(BODY_LONG, 0) &&
         b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0) && b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
         ((b.COL(1) == -1 && b.RGAP_UP(0, 1)) || (b.COL(1) == 1 && b.RGAP_DN(0, 1)));
}
CDL_FN(c_kicking) { return kicking_common(b) ? b.COL(0) * 100 : 0; }
CDL_FN(c_kicking_by_length) {
  if (!kicking_common(b)) return 0;
  return (b.RB(0) > b.RB(1) ? b.COL(0) : b.COL(1)) * 100;
}
CDL_FN(c_ladder_bottom) {
  return (b.COL(4) == -1 && b.COL(3) == -1 && b.COL(2) == -1 && b.O(4) > b.O(3) && b.O(3) > b.O(2) &&
          b.C(4) > b.C(3) && b.C(3) > b.C(2) && b.COL(1) == -1 && b.US(1) > b.AVG(SHADOW_VERY_SHORT, 1) &&
          b.COL(0) == 1 && b.O(0) > b.O(1) && b.C(0) > b.H(1)) ? 100 : 0;
}
CDL_FN(c_long_legged_doji) {
  return (b.RB(0) <= b.AVG(BODY_DOJI, 0) &&
          (b.LS(0) > b.AVG(SHADOW_LONG, 0) || b.US(0) > b.AVG(SHADOW_LONG, 0))) ? 100 : 0;
}
CDL_FN(c_long_line) {
  return (b.RB(0) > b.AVG(BODY_LONG, 0) && b.US(0) < b.AVG(SHADOW_SHORT, 0) && b.LS(0) < b.AVG(SHADOW_SHORT, 0))
             ? b.COL(0) * 100 : 0;
}
CDL_FN(c_marubozu) {
  return (b.RB(0) > b.AVG(BODY_LONG, 0) && b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
          b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0)) ? b.COL(0) * 100 : 0;
}
CDL_FN(c_matching_low) {
  return (b.COL(1) == -1 && b.COL(0) == -1 && b.C(0) <= b.C(1) + b.AVG(EQUAL, 1) &&
          b.C(0) >= b.C(1) - b.AVG(EQUAL, 1)) ? 100 : 0;
}
CDL_FN(c_mat_hold) {
  const double pen = 0.5;
  return (b.RB(4) > b.AVG(BODY_LONG, 4) && b.RB(3) < b.AVG(BODY_SHORT, 3) && b.RB(2) < b.AVG(BODY_SHORT, 2) &&
          b.RB(1) < b.AVG(BODY_SHORT, 1) && b.COL(4) == 1 && b.COL(3) == -1 && b.COL(0) == 1 && b.BGAP_UP(3, 4) &&
          b.BOT(2) < b.C(4) && b.BOT(1) < b.C(4) && b.BOT(2) > b.C(4) - b.RB(4) * pen &&
          b.BOT(1) > b.C(4) - b.RB(4) * pen && fmaxf(b.C(2), b.O(2)) < b.O(3) &&
          fmaxf(b.C(1), b.O(1)) < fmaxf(b.C(2), b.O(2)) && b.O(0) > b.C(1) &&
          b.C(0) > fmaxf(fmaxf(b.H(3), b.H(2)), b.H(1))) ? 100 : 0;
}
CDL_FN(c_on_neck) {
  return (b.COL(1) == -1 && b.RB(1) > b.AVG(BODY_LONG, 1) && b.COL(0) == 1 && b.O(0) < b.L(1) &&
          b.C(0) <= b.L(1) + b.AVG(EQUAL, 1) && b.C(0) >= b.L(1) - b.AVG(EQUAL, 1)) ? -100 : 0;
}
CDL_FN(c_piercing) {
  return (b.COL(1) == -1 && b.RB(1) > b.AVG(BODY_LONG, 1) && b.COL(0) == 1 && b.RB(0) > b.AVG(BODY_LONG, 0) &&
          b.O(0) < b.L(1) && b.C(0) < b.O(1) && (double)b.C(0) > (double)b.C(1) + b.RB(1) * 0.5) ? 100 : 0;
}
CDL_FN(c_rickshaw_man) {
  const double mid = (double)b.L(0) + ((double)b.H(0) - (double)b.L(0)) / 2.0;
  return (b.RB(0) <= b.AVG(BODY_DOJI, 0) && b.LS(0) > b.AVG(SHADOW_LONG, 0) && b.US(0) > b.AVG(SHADOW_LONG, 0) &&
          (double)b.BOT(0) <= mid + b.AVG(NEAR, 0) && (double)b.TOP(0) >= mid - b.AVG(NEAR, 0)) ? 100 : 0;
}
CDL_FN(c_rise_fall3_methods) {
  const int c4 = b.COL(4);
  return (b.RB(4) > b.AVG(BODY_LONG, 4) && b.RB(3) < b.AVG(BODY_SHORT, 3) && b.RB(2) < b.AVG(BODY_SHORT, 2) &&
          b.RB(1) < b.AVG(BODY_SHORT, 1) && b.RB(0) > b.AVG(BODY_LONG, 0) && c4 == -b.COL(3) &&
          b.COL(3) == b.COL(2) && b.COL(2) == b.COL(1) && b.COL(1) == -b.COL(0) && b.BOT(3) < b.H(4) &&
          b.TOP(3) > b.L(4) && b.BOT(2) < b.H(4) && b.TOP(2) > b.L(4) && b.BOT(1) < b.H(4) && b.TOP(1) > b.L(4) &&
          b.C(2) * c4 < b.C(3) * c4 && b.C(1) * c4 < b.C(2) * c4 && b.O(0) * c4 > b.C(1) * c4 &&
          b.C(0) * c4 > b.C(4) * c4) ? 100 * c4 : 0;
}
CDL_FN(c_separating_lines) {
  if (b.COL(1) == -b.COL(0) && b.O(0) <= b.O(1) + b.AVG(EQUAL, 1) && b.O(0) >= b.O(1) - b.AVG(EQUAL, 1) &&
      b.RB(0) > b.AVG(BODY_LONG, 0) &&
      ((b.COL(0) == 1 && b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0)) ||
       (b.COL(0) == -1 && b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0))))
    return b.COL(0) * 100;
  return 0;
}
CDL_FN(c_shooting_star) {
  return (b.RB(0) < b.AVG(BODY_SHORT, 0) && b.US(0) > b.AVG(SHADOW_LONG, 0) &&
          b.LS(0) < b.AVG(SHADOW_VERY_SHORT, 0) && b.BGAP_UP(0, 1)) ? -100 : 0;
}
CDL_FN(c_short_line) {
  return (b.RB(0) < b.AVG(BODY_SHORT, 0) && b.US(0) < b.AVG(SHADOW_SHORT, 0) && b.LS(0) < b.AVG(SHADOW_SHORT, 0))
             ? b.COL(0) * 100 : 0;
}
CDL_FN(c_spinning_top) {
  return (b.RB(0) < b.AVG(BODY_SHORT, 0) && b.US(0) > b.RB(0) && b.LS(0) > b.RB(0)) ? b.COL(0) * 100 : 0;
}
CDL_FN(c_stalled_pattern) {
  return (b.COL(2) == 1 && b.COL(1) == 1 && b.COL(0) == 1 && b.C(0) > b.C(1) && b.C(1) > b.C(2) &&
          b.RB(2) > b.AVG(BODY_LONG, 2) && b.RB(1) > b.AVG(BODY_LONG, 1) && b.US(1) < b.AVG(SHADOW_VERY_SHORT, 1) &&
          b.O(1) > b.O(2) && b.O(1) <= b.C(2) + b.AVG(NEAR, 2) && b.RB(0) < b.AVG(BODY_SHORT, 0) &&
          b.O(0) >= b.C(1) - b.RB(0) - b.AVG(NEAR, 1)) ? -100 : 0;
}
CDL_FN(c_stick_sandwich) {
  return (b.COL(2) == -1 && b.COL(1) == 1 && b.COL(0) == -1 && b.L(1) > b.C(2) &&
          (double)b.C(0) <= (double)b.C(2) + b.AVG(EQUAL, 2) &&
          (double)b.C(0) >= (double)b.C(2) - b.AVG(EQUAL, 2)) ? 100 : 0;
}
CDL_FN(c_takuri) {
  return (b.RB(0) <= b.AVG(BODY_DOJI, 0) && b.US(0) < b.AVG(SHADOW_VERY_SHORT, 0) &&
          b.LS(0) > b.AVG(SHADOW_VERY_LONG, 0)) ? 100 : 0;
}
CDL_FN(c_tasuki_gap) {
  if ((b.BGAP_UP(1, 2) && b.COL(1) == 1 && b.COL(0) == -1 && b.O(0) < b.C(1) && b.O(0) > b.O(1) &&
       b.C(0) < b.O(1) && b.C(0) > fmaxf(b.C(2), b.O(2)) && fabs(b.RB(1) - b.RB(0)) < b.AVG(NEAR, 1)) ||
      (b.BGAP_DN(1, 2) && b.COL(1) == -1 && b.COL(0) == 1 && b.O(0) < b.O(1) && b.O(0) > b.C(1) &&
       b.C(0) > b.O(1) && b.C(0) < fminf(b.C(2), b.O(2)) && fabs(b.RB(1) - b.RB(0)) < b.AVG(NEAR, 1)))
    return b.COL(1) * 100;
  return 0;
}
CDL_FN(c_thrusting) {
  return (b.COL(1) == -1 && b.RB(1) > b.AVG(BODY_LONG, 1) && b.COL(0) == 1 && b.O(0) < b.L(1) &&
          b.C(0) > b.C(1) + b.AVG(EQUAL, 1) && (double)b.C(0) <= (double)b.C(1) + b.RB(1) * 0.5) ? -100 : 0;
}
// TA-Lib keeps the doji average anchored at the first candle for all three.
CDL_FN(c_tristar) {
  const double d = b.AVG(BODY_DOJI, 2);
  if (b.RB(2) <= d && b.RB(1) <= d && b.RB(0) <= d) {
    int out = 0;
    if (b.BGAP_UP(1, 2) && fmaxf(b.O(0), b.C(0)) < fmaxf(b.O(1), b.C(1))) out = -100;
    if (b.BGAP_DN(1, 2) && fminf(b.O(0), b.C(0)) > fminf(b.O(1), b.C(1))) out = 100;
    return out;
  }
  return 0;
}
CDL_FN(c_unique_3_river) {
  return (b.RB(2) > b.AVG(BODY_LONG, 2) && b.COL(2) == -1 && b.COL(1) == -1 && b.C(1) > b.C(2) && b.O(1) <= b.O(2) &&
          b.L(1) < b.L(2) && b.RB(0) < b.AVG(BODY_SHORT, 0) && b.COL(0) == 1 && b.O(0) > b.L(1)) ? 100 : 0;
}
CDL_FN(c_upside_gap_2_crows) {
  return (b.COL(2) == 1 && b.RB(2) > b.AVG(BODY_LONG, 2) && b.COL(1) == -1 && b.RB(1) <= b.AVG(BODY_SHORT, 1) &&
          b.BGAP_UP(1, 2) && b.COL(0) == -1 && b.O(0) > b.O(1) && b.C(0) < b.C(1) && b.C(0) > b.C(2)) ? -100 : 0;
}
CDL_FN(c_xside_gap_3_methods) {
  if (b.COL(2) == b.COL(1) && b.COL(1) == -b.COL(0) && b.O(0) < fmaxf(b.C(1), b.O(1)) &&
      b.O(0) > fminf(b.C(1), b.O(1)) && b.C(0) < fmaxf(b.C(2), b.O(2)) && b.C(0) > fminf(b.C(2), b.O(2)) &&
      ((b.COL(2) == 1 && b.BGAP_UP(1, 2)) || (b.COL(2) == -1 && b.BGAP_DN(1, 2))))
    return b.COL(2) * 100;
  return 0;
}
#undef CDL_FN

// Pattern k in the order of the ct_cdl_*_batch_d declarations.
template <class B>
__device__ __forceinline__ int cdl_eval(int k, const B& b) {
  switch (k) {
    case 0: return c_doji(b);
    case 1: return c_hammer(b);
    case 2: return c_inverted_hammer(b);
    case 3: case 4: return c_engulfing(b);  // legacy bullish / bearish split
    case 5: return c_three_white_soldiers(b);
    case 6: return c_abandoned_baby(b);
    case 7: return c_advance_block(b);
    case 8: return c_belt_hold(b);
    case 9: return c_breakaway(b);
    case 10: return c_two_crows(b);
    case 11: return c_three_black_crows(b);
    case 12: return c_three_inside(b);
    case 13: return c_three_outside(b);
    case 14: return c_three_line_strike(b);
    case 15: return c_three_stars_in_south(b);
    case 16: return c_closing_marubozu(b);
    case 17: return c_conceal_baby_swallow(b);
    case 18: return c_counterattack(b);
    case 19: return c_dark_cloud_cover(b);
    case 20: return c_doji_star(b);
    case 21: return c_dragonfly_doji(b);
    case 22: return c_engulfing(b);
    case 23: return c_evening_doji_star(b);
    case 24: return c_evening_star(b);
    case 25: return c_gap_side_side_white(b);
    case 26: return c_gravestone_doji(b);
    case 27: return c_hanging_man(b);
    case 28: return c_harami(b);
    case 29: return c_harami_cross(b);
    case 30: return c_high_wave(b);
    case 31: return c_hikkake(b);
    case 32: return c_hikkake_mod(b);
    case 33: return c_homing_pigeon(b);
    case 34: return c_identical_three_crows(b);
    case 35: return c_in_neck(b);
    case 36: return c_kicking(b);
    case 37: return c_kicking_by_length(b);
    case 38: return c_ladder_bottom(b);
    case 39: return c_long_legged_doji(b);
    case 40: return c_long_line(b);
    case 41: return c_marubozu(b);
    case 42: return c_matching_low(b);
    case 43: return c_mat_hold(b);
    case 44: return c_morning_doji_star(b);
    case 45: return c_morning_star(b);
    case 46: return c_on_neck(b);
    case 47: return c_piercing(b);
    case 48: return c_rickshaw_man(b);
    case 49: return c_rise_fall3_methods(b);
    case 50: return c_separating_lines(b);
    case 51: return c_shooting_star(b);
    case 52: return c_short_line(b);
    case 53: return c_spinning_top(b);
    case 54: return c_stalled_pattern(b);
    case 55: return c_stick_sandwich(b);
    case 56: return c_takuri(b);
    case 57: return c_tasuki_gap(b);
    case 58: return c_thrusting(b);
    case 59: return c_tristar(b);
    case 60: return c_unique_3_river(b);
    case 61: return c_upside_gap_2_crows(b);
    case 62: return c_xside_gap_3_methods(b);
  }
  return 0;
}

// Warm-up lengths (bars before them are 0), order as above.
__device__ __constant__ const unsigned char kCdlLookbackDev[63] = {
    10, 11, 11, 1, 1, 12, 12, 12, 10, 14, 12, 13, 12, 3, 8, 12, 10, 13, 11, 11, 11, 10, 2, 12, 12, 7, 10, 11, 11, 11,
    10, 5, 10, 11, 12, 11, 11, 11, 14, 10, 10, 10, 6, 14, 12, 12, 11, 11, 10, 14, 11, 11, 10, 10, 12, 7, 10, 7, 11, 12,
    12, 12, 2};

}  // namespace rules
}  // namespace tb
