/* Test infrastructure only: FP64 CPU restatement of the reference's 63 candle
 * families (61 TA-Lib CDL* patterns plus the legacy bullish/bearish engulfing
 * split), used to check the CUDA candle engine. The decision rules are TA-Lib's
 * published ones as the reference states them in include/utils/CandleUtils.h
 * (settings :37-63, trailing average :1466-1495, patterns :1510-2330); each
 * family's warm-up length is its kernel's (src/indicators/<Pattern>.cu, e.g.
 * Doji.cu:19-23). Bars before the warm-up length are 0.
 *
 * Trailing averages are re-summed per call exactly as the reference does (FP64
 * sum over the `period` bars before the anchor, divided by the count, times the
 * setting factor, halved for shadow settings); comparisons mix float32 bar
 * values with FP64 averages the same way.
 */
#include "ta_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>

enum { R_BODY = 0, R_HL = 1, R_SHADOWS = 2 };
enum {
  S_BODY_LONG = 0, S_BODY_VERY_LONG, S_BODY_SHORT, S_BODY_DOJI, S_SHADOW_LONG,
  S_SHADOW_VERY_LONG, S_SHADOW_SHORT, S_SHADOW_VERY_SHORT, S_NEAR, S_FAR, S_EQUAL
};

/* TA-Lib default candle settings (CandleUtils.h:37-63). */
static const struct { int range, period; float factor; } kSetting[11] = {
  {R_BODY, 10, 1.0f}, {R_BODY, 10, 3.0f}, {R_BODY, 10, 1.0f}, {R_HL, 10, 0.1f},
  {R_BODY, 0, 1.0f},  {R_BODY, 0, 2.0f},  {R_SHADOWS, 10, 1.0f}, {R_HL, 10, 0.1f},
  {R_HL, 5, 0.2f},    {R_HL, 5, 0.6f},    {R_HL, 5, 0.05f},
};

typedef struct { const float *o, *h, *l, *c; } Bars;

static double range_of(int type, const Bars* b, int i) {
  const double o = b->o[i], h = b->h[i], l = b->l[i], c = b->c[i];
  if (type == R_BODY) return fabs(c - o);
  if (type == R_HL) return h - l;
  return (h - fmax(o, c)) + (fmin(o, c) - l);
}

/* CandleUtils.h:1466-1495: average of the setting's range over the bars before
 * `idx` (fewer at the start of the row), or the bar itself for period 0. */
static double avg(const Bars* b, int set, int idx) {
  const int type = kSetting[set].range, per = kSetting[set].period;
  const double factor = (double)kSetting[set].factor;
  const double div = type == R_SHADOWS ? 2.0 : 1.0;
  if (idx < 0) idx = 0;
  int start = idx - per;
  if (start < 0) start = 0;
  const int count = idx - start;
  if (per <= 0 || count <= 0) return factor * range_of(type, b, idx) / div;
  double sum = 0.0;
  for (int i = start; i < idx; ++i) sum += range_of(type, b, i);
  return factor * (sum / (double)count) / div;
}

#define O(i) (b->o[(i)])
#define H(i) (b->h[(i)])
#define L(i) (b->l[(i)])
#define C(i) (b->c[(i)])
#define RB(i) fabs((double)C(i) - (double)O(i))
#define US(i) ((double)H(i) - fmax((double)O(i), (double)C(i)))
#define LS(i) (fmin((double)O(i), (double)C(i)) - (double)L(i))
#define COL(i) (C(i) >= O(i) ? 1 : -1)
#define AVG(s, i) avg(b, (s), (i))
#define TOPF(i) fmaxf(O(i), C(i))
#define BOTF(i) fminf(O(i), C(i))
/* gaps between real bodies, and between full ranges */
#define BGAP_UP(a, p) (fminf(O(a), C(a)) > fmaxf(O(p), C(p)))
#define BGAP_DN(a, p) (fmaxf(O(a), C(a)) < fminf(O(p), C(p)))
#define RGAP_UP(a, p) (L(a) > H(p))
#define RGAP_DN(a, p) (H(a) < L(p))

static int p_two_crows(const Bars* b, int i) {
  return (COL(i - 2) == 1 && RB(i - 2) > AVG(S_BODY_LONG, i - 2) && COL(i - 1) == -1 &&
          BGAP_UP(i - 1, i - 2) && COL(i) == -1 && O(i) < O(i - 1) && O(i) > C(i - 1) &&
          C(i) > O(i - 2) && C(i) < C(i - 2)) ? -100 : 0;
}

static int p_three_black_crows(const Bars* b, int i) {
  return (COL(i - 3) == 1 && COL(i - 2) == -1 && LS(i - 2) < AVG(S_SHADOW_VERY_SHORT, i - 2) &&
          COL(i - 1) == -1 && LS(i - 1) < AVG(S_SHADOW_VERY_SHORT, i - 1) && COL(i) == -1 &&
          LS(i) < AVG(S_SHADOW_VERY_SHORT, i) && O(i - 1) < O(i - 2) && O(i - 1) > C(i - 2) &&
          O(i) < O(i - 1) && O(i) > C(i - 1) && H(i - 3) > C(i - 2) && C(i - 2) > C(i - 1) &&
          C(i - 1) > C(i)) ? -100 : 0;
}

static int p_three_inside(const Bars* b, int i) {
  if (RB(i - 2) > AVG(S_BODY_LONG, i - 2) && RB(i - 1) <= AVG(S_BODY_SHORT, i - 1) &&
      fmaxf(C(i - 1), O(i - 1)) < fmaxf(C(i - 2), O(i - 2)) &&
      fminf(C(i - 1), O(i - 1)) > fminf(C(i - 2), O(i - 2)) &&
      ((COL(i - 2) == 1 && COL(i) == -1 && C(i) < O(i - 2)) ||
       (COL(i - 2) == -1 && COL(i) == 1 && C(i) > O(i - 2))))
    return -COL(i - 2) * 100;
  return 0;
}

static int p_three_line_strike(const Bars* b, int i) {
  if (COL(i - 3) == COL(i - 2) && COL(i - 2) == COL(i - 1) && COL(i) == -COL(i - 1) &&
      (double)O(i - 2) >= (double)BOTF(i - 3) - AVG(S_NEAR, i - 3) &&
      (double)O(i - 2) <= (double)TOPF(i - 3) + AVG(S_NEAR, i - 3) &&
      (double)O(i - 1) >= (double)BOTF(i - 2) - AVG(S_NEAR, i - 2) &&
      (double)O(i - 1) <= (double)TOPF(i - 2) + AVG(S_NEAR, i - 2) &&
      ((COL(i - 1) == 1 && C(i - 1) > C(i - 2) && C(i - 2) > C(i - 3) && O(i) > C(i - 1) &&
        C(i) < O(i - 3)) ||
       (COL(i - 1) == -1 && C(i - 1) < C(i - 2) && C(i - 2) < C(i - 3) && O(i) < C(i - 1) &&
        C(i) > O(i - 3))))
    return COL(i - 1) * 100;
  return 0;
}

static int p_three_outside(const Bars* b, int i) {
  if ((COL(i - 1) == 1 && COL(i - 2) == -1 && C(i - 1) > O(i - 2) && O(i - 1) < C(i - 2) &&
       C(i) > C(i - 1)) ||
      (COL(i - 1) == -1 && COL(i - 2) == 1 && O(i - 1) > C(i - 2) && C(i - 1) < O(i - 2) &&
       C(i) < C(i - 1)))
    return COL(i - 1) * 100;
  return 0;
}

static int p_three_stars_in_south(const Bars* b, int i) {
  return (COL(i - 2) == -1 && COL(i - 1) == -1 && COL(i) == -1 &&
          RB(i - 2) > AVG(S_BODY_LONG, i - 2) && LS(i - 2) > AVG(S_SHADOW_LONG, i - 2) &&
          RB(i - 1) < RB(i - 2) && O(i - 1) > C(i - 2) && O(i - 1) <= H(i - 2) &&
          L(i - 1) < C(i - 2) && L(i - 1) >= L(i - 2) &&
          LS(i - 1) > AVG(S_SHADOW_VERY_SHORT, i - 1) && RB(i) < AVG(S_BODY_SHORT, i) &&
          LS(i) < AVG(S_SHADOW_VERY_SHORT, i) && US(i) < AVG(S_SHADOW_VERY_SHORT, i) &&
          L(i) > L(i - 1) && H(i) < H(i - 1)) ? 100 : 0;
}

static int p_three_white_soldiers(const Bars* b, int i) {
  return (COL(i - 2) == 1 && US(i - 2) < AVG(S_SHADOW_VERY_SHORT, i - 2) && COL(i - 1) == 1 &&
          US(i - 1) < AVG(S_SHADOW_VERY_SHORT, i - 1) && COL(i) == 1 &&
          US(i) < AVG(S_SHADOW_VERY_SHORT, i) && C(i) > C(i - 1) && C(i - 1) > C(i - 2) &&
          O(i - 1) > O(i - 2) && (double)O(i - 1) <= (double)C(i - 2) + AVG(S_NEAR, i - 2) &&
          O(i) > O(i - 1) && (double)O(i) <= (double)C(i - 1) + AVG(S_NEAR, i - 1) &&
          RB(i - 1) > RB(i - 2) - AVG(S_FAR, i - 2) && RB(i) > RB(i - 1) - AVG(S_FAR, i - 1) &&
          RB(i) > AVG(S_BODY_SHORT, i)) ? 100 : 0;
}

static int p_abandoned_baby(const Bars* b, int i) {
  const double pen = 0.3;
  if (RB(i - 2) > AVG(S_BODY_LONG, i - 2) && RB(i - 1) <= AVG(S_BODY_DOJI, i - 1) &&
      RB(i) > AVG(S_BODY_SHORT, i) &&
      ((COL(i - 2) == 1 && COL(i) == -1 && C(i) < C(i - 2) - RB(i - 2) * pen &&
        RGAP_UP(i - 1, i - 2) && RGAP_DN(i, i - 1)) ||
       (COL(i - 2) == -1 && COL(i) == 1 && C(i) > C(i - 2) + RB(i - 2) * pen &&
        RGAP_DN(i - 1, i - 2) && RGAP_UP(i, i - 1))))
    return COL(i) * 100;
  return 0;
}

static int p_advance_block(const Bars* b, int i) {
  if (COL(i - 2) == 1 && COL(i - 1) == 1 && COL(i) == 1 && C(i) > C(i - 1) &&
      C(i - 1) > C(i - 2) && O(i - 1) > O(i - 2) && O(i - 1) <= C(i - 2) + AVG(S_NEAR, i - 2) &&
      O(i) > O(i - 1) && O(i) <= C(i - 1) + AVG(S_NEAR, i - 1) &&
      RB(i - 2) > AVG(S_BODY_LONG, i - 2) && US(i - 2) < AVG(S_SHADOW_SHORT, i - 2) &&
      ((RB(i - 1) < RB(i - 2) - AVG(S_FAR, i - 2) && RB(i) < RB(i - 1) + AVG(S_NEAR, i - 1)) ||
       (RB(i) < RB(i - 1) - AVG(S_FAR, i - 1)) ||
       (RB(i) < RB(i - 1) && RB(i - 1) < RB(i - 2) &&
        (US(i) > AVG(S_SHADOW_SHORT, i) || US(i - 1) > AVG(S_SHADOW_SHORT, i - 1))) ||
       (RB(i) < RB(i - 1) && US(i) > AVG(S_SHADOW_LONG, i))))
    return -100;
  return 0;
}

static int p_belt_hold(const Bars* b, int i) {
  if (RB(i) > AVG(S_BODY_LONG, i) &&
      ((COL(i) == 1 && LS(i) < AVG(S_SHADOW_VERY_SHORT, i)) ||
       (COL(i) == -1 && US(i) < AVG(S_SHADOW_VERY_SHORT, i))))
    return COL(i) * 100;
  return 0;
}

static int p_breakaway(const Bars* b, int i) {
  if (RB(i - 4) > AVG(S_BODY_LONG, i - 4) && COL(i - 4) == COL(i - 3) && COL(i - 3) == COL(i - 1) &&
      COL(i - 1) == -COL(i) &&
      ((COL(i - 4) == -1 && BGAP_DN(i - 3, i - 4) && H(i - 2) < H(i - 3) && L(i - 2) < L(i - 3) &&
        H(i - 1) < H(i - 2) && L(i - 1) < L(i - 2) && C(i) > O(i - 3) && C(i) < C(i - 4)) ||
       (COL(i - 4) == 1 && BGAP_UP(i - 3, i - 4) && H(i - 2) > H(i - 3) && L(i - 2) > L(i - 3) &&
        H(i - 1) > H(i - 2) && L(i - 1) > L(i - 2) && C(i) < O(i - 3) && C(i) > C(i - 4))))
    return COL(i) * 100;
  return 0;
}

static int p_closing_marubozu(const Bars* b, int i) {
  if (RB(i) > AVG(S_BODY_LONG, i) &&
      ((COL(i) == 1 && US(i) < AVG(S_SHADOW_VERY_SHORT, i)) ||
       (COL(i) == -1 && LS(i) < AVG(S_SHADOW_VERY_SHORT, i))))
    return COL(i) * 100;
  return 0;
}

static int p_conceal_baby_swallow(const Bars* b, int i) {
  return (COL(i - 3) == -1 && COL(i - 2) == -1 && COL(i - 1) == -1 && COL(i) == -1 &&
          LS(i - 3) < AVG(S_SHADOW_VERY_SHORT, i - 3) && US(i - 3) < AVG(S_SHADOW_VERY_SHORT, i - 3) &&
          LS(i - 2) < AVG(S_SHADOW_VERY_SHORT, i - 2) && US(i - 2) < AVG(S_SHADOW_VERY_SHORT, i - 2) &&
          BGAP_DN(i - 1, i - 2) && US(i - 1) > AVG(S_SHADOW_VERY_SHORT, i - 1) &&
          H(i - 1) > C(i - 2) && H(i) > H(i - 1) && L(i) < L(i - 1)) ? 100 : 0;
}

static int p_counterattack(const Bars* b, int i) {
  if (COL(i - 1) == -COL(i) && RB(i - 1) > AVG(S_BODY_LONG, i - 1) && RB(i) > AVG(S_BODY_LONG, i) &&
      C(i) <= C(i - 1) + AVG(S_EQUAL, i - 1) && C(i) >= C(i - 1) - AVG(S_EQUAL, i - 1))
    return COL(i) * 100;
  return 0;
}

static int p_dark_cloud_cover(const Bars* b, int i) {
  const double pen = 0.5;
  return (COL(i - 1) == 1 && RB(i - 1) > AVG(S_BODY_LONG, i - 1) && COL(i) == -1 &&
          O(i) > H(i - 1) && C(i) > O(i - 1) &&
          (double)C(i) < (double)C(i - 1) - RB(i - 1) * pen) ? -100 : 0;
}

static int p_doji(const Bars* b, int i) { return RB(i) <= AVG(S_BODY_DOJI, i) ? 100 : 0; }

static int p_doji_star(const Bars* b, int i) {
  if (RB(i - 1) > AVG(S_BODY_LONG, i - 1) && RB(i) <= AVG(S_BODY_DOJI, i) &&
      ((COL(i - 1) == 1 && BGAP_UP(i, i - 1)) || (COL(i - 1) == -1 && BGAP_DN(i, i - 1))))
    return -COL(i - 1) * 100;
  return 0;
}

static int p_dragonfly_doji(const Bars* b, int i) {
  return (RB(i) <= AVG(S_BODY_DOJI, i) && US(i) < AVG(S_SHADOW_VERY_SHORT, i) &&
          LS(i) > AVG(S_SHADOW_VERY_SHORT, i)) ? 100 : 0;
}

/* TA-Lib ENGULFING: +-100 strict, +-80 when one body end coincides. */
static int p_engulfing(const Bars* b, int i) {
  const int white = COL(i) == 1 && COL(i - 1) == -1 &&
                    ((C(i) >= O(i - 1) && O(i) < C(i - 1)) || (C(i) > O(i - 1) && O(i) <= C(i - 1)));
  const int black = COL(i) == -1 && COL(i - 1) == 1 &&
                    ((O(i) >= C(i - 1) && C(i) < O(i - 1)) || (O(i) > C(i - 1) && C(i) <= O(i - 1)));
  if (white || black) return (O(i) != C(i - 1) && C(i) != O(i - 1)) ? COL(i) * 100 : COL(i) * 80;
  return 0;
}

static int star_common(const Bars* b, int i, int doji_middle, int bull) {
  const double pen = 0.3;
  const int mid_ok = doji_middle ? RB(i - 1) <= AVG(S_BODY_DOJI, i - 1)
                                 : RB(i - 1) <= AVG(S_BODY_SHORT, i - 1);
  if (bull)
    return RB(i - 2) > AVG(S_BODY_LONG, i - 2) && COL(i - 2) == -1 && mid_ok &&
           BGAP_DN(i - 1, i - 2) && RB(i) > AVG(S_BODY_SHORT, i) && COL(i) == 1 &&
           (double)C(i) > (double)C(i - 2) + RB(i - 2) * pen;
  return RB(i - 2) > AVG(S_BODY_LONG, i - 2) && COL(i - 2) == 1 && mid_ok &&
         BGAP_UP(i - 1, i - 2) && RB(i) > AVG(S_BODY_SHORT, i) && COL(i) == -1 &&
         (double)C(i) < (double)C(i - 2) - RB(i - 2) * pen;
}

static int p_evening_doji_star(const Bars* b, int i) { return star_common(b, i, 1, 0) ? -100 : 0; }
static int p_evening_star(const Bars* b, int i) { return star_common(b, i, 0, 0) ? -100 : 0; }
static int p_morning_doji_star(const Bars* b, int i) { return star_common(b, i, 1, 1) ? 100 : 0; }
static int p_morning_star(const Bars* b, int i) { return star_common(b, i, 0, 1) ? 100 : 0; }

static int p_gap_side_side_white(const Bars* b, int i) {
  if (((BGAP_UP(i - 1, i - 2) && BGAP_UP(i, i - 2)) || (BGAP_DN(i - 1, i - 2) && BGAP_DN(i, i - 2))) &&
      COL(i - 1) == 1 && COL(i) == 1 && RB(i) >= RB(i - 1) - AVG(S_NEAR, i - 1) &&
      RB(i) <= RB(i - 1) + AVG(S_NEAR, i - 1) && O(i) >= O(i - 1) - AVG(S_EQUAL, i - 1) &&
      O(i) <= O(i - 1) + AVG(S_EQUAL, i - 1))
    return BGAP_UP(i - 1, i - 2) ? 100 : -100;
  return 0;
}

static int p_gravestone_doji(const Bars* b, int i) {
  return (RB(i) <= AVG(S_BODY_DOJI, i) && LS(i) < AVG(S_SHADOW_VERY_SHORT, i) &&
          US(i) > AVG(S_SHADOW_VERY_SHORT, i)) ? 100 : 0;
}

static int hammer_shape(const Bars* b, int i) {
  return RB(i) < AVG(S_BODY_SHORT, i) && LS(i) > AVG(S_SHADOW_LONG, i) &&
         US(i) < AVG(S_SHADOW_VERY_SHORT, i);
}

static int p_hammer(const Bars* b, int i) {
  return (hammer_shape(b, i) && (double)fminf(C(i), O(i)) <= (double)L(i - 1) + AVG(S_NEAR, i - 1)) ? 100 : 0;
}

static int p_hanging_man(const Bars* b, int i) {
  return (hammer_shape(b, i) && (double)fminf(C(i), O(i)) >= (double)H(i - 1) - AVG(S_NEAR, i - 1)) ? -100 : 0;
}

static int harami_common(const Bars* b, int i, int cross) {
  const int small = cross ? RB(i) <= AVG(S_BODY_DOJI, i) : RB(i) <= AVG(S_BODY_SHORT, i);
  if (RB(i - 1) > AVG(S_BODY_LONG, i - 1) && small) {
    const float hi2 = fmaxf(C(i), O(i)), lo2 = fminf(C(i), O(i));
    const float hi1 = fmaxf(C(i - 1), O(i - 1)), lo1 = fminf(C(i - 1), O(i - 1));
    if (hi2 < hi1 && lo2 > lo1) return -COL(i - 1) * 100;
    if (hi2 <= hi1 && lo2 >= lo1) return -COL(i - 1) * 80;
  }
  return 0;
}

static int p_harami(const Bars* b, int i) { return harami_common(b, i, 0); }
static int p_harami_cross(const Bars* b, int i) { return harami_common(b, i, 1); }

static int p_high_wave(const Bars* b, int i) {
  return (RB(i) < AVG(S_BODY_SHORT, i) && US(i) > AVG(S_SHADOW_VERY_LONG, i) &&
          LS(i) > AVG(S_SHADOW_VERY_LONG, i)) ? COL(i) * 100 : 0;
}

/* HIKKAKE / HIKKAKEMOD: a pattern bar, or its confirmation within the next three
 * bars when no earlier bar confirmed it (CandleUtils.h:1849-1895). */
static int hikkake_at(const Bars* b, int i) {
  if (H(i - 1) < H(i - 2) && L(i - 1) > L(i - 2) &&
      ((H(i) < H(i - 1) && L(i) < L(i - 1)) || (H(i) > H(i - 1) && L(i) > L(i - 1))))
    return H(i) < H(i - 1) ? 100 : -100;
  return 0;
}

static int hikkake_mod_at(const Bars* b, int i) {
  if (H(i - 2) < H(i - 3) && L(i - 2) > L(i - 3) && H(i - 1) < H(i - 2) && L(i - 1) > L(i - 2) &&
      ((H(i) < H(i - 1) && L(i) < L(i - 1) && C(i - 2) <= L(i - 2) + AVG(S_NEAR, i - 2)) ||
       (H(i) > H(i - 1) && L(i) > L(i - 1) && C(i - 2) >= H(i - 2) - AVG(S_NEAR, i - 2))))
    return H(i) < H(i - 1) ? 100 : -100;
  return 0;
}

static int hikkake_confirm(const Bars* b, int i, int modified) {
  const int pat = modified ? hikkake_mod_at(b, i) : hikkake_at(b, i);
  if (pat != 0) return pat;
  const int lowest = modified ? 3 : 2;
  for (int j = i - 1; j >= i - 3 && j >= lowest; --j) {
    const int pj = modified ? hikkake_mod_at(b, j) : hikkake_at(b, j);
    if (pj == 0) continue;
    for (int m = j + 1; m <= i; ++m) {
      const int conf = (pj > 0 && C(m) > H(j - 1)) || (pj < 0 && C(m) < L(j - 1));
      if (conf) return m == i ? pj + (pj > 0 ? 100 : -100) : 0;
    }
    return 0;
  }
  return 0;
}

static int p_hikkake(const Bars* b, int i) { return hikkake_confirm(b, i, 0); }
static int p_hikkake_mod(const Bars* b, int i) { return hikkake_confirm(b, i, 1); }

static int p_homing_pigeon(const Bars* b, int i) {
  return (COL(i - 1) == -1 && COL(i) == -1 && RB(i - 1) > AVG(S_BODY_LONG, i - 1) &&
          RB(i) <= AVG(S_BODY_SHORT, i) && O(i) < O(i - 1) && C(i) > C(i - 1)) ? 100 : 0;
}

static int p_identical_three_crows(const Bars* b, int i) {
  return (COL(i - 2) == -1 && LS(i - 2) < AVG(S_SHADOW_VERY_SHORT, i - 2) && COL(i - 1) == -1 &&
          LS(i - 1) < AVG(S_SHADOW_VERY_SHORT, i - 1) && COL(i) == -1 &&
          LS(i) < AVG(S_SHADOW_VERY_SHORT, i) && C(i - 2) > C(i - 1) && C(i - 1) > C(i) &&
          (double)O(i - 1) <= (double)C(i - 2) + AVG(S_EQUAL, i - 2) &&
          (double)O(i - 1) >= (double)C(i - 2) - AVG(S_EQUAL, i - 2) &&
          (double)O(i) <= (double)C(i - 1) + AVG(S_EQUAL, i - 1) &&
          (double)O(i) >= (double)C(i - 1) - AVG(S_EQUAL, i - 1)) ? -100 : 0;
}

static int p_in_neck(const Bars* b, int i) {
  return (COL(i - 1) == -1 && RB(i - 1) > AVG(S_BODY_LONG, i - 1) && COL(i) == 1 && O(i) < L(i - 1) &&
          (double)C(i) <= (double)C(i - 1) + AVG(S_EQUAL, i - 1) && C(i) >= C(i - 1)) ? -100 : 0;
}

static int p_inverted_hammer(const Bars* b, int i) {
  return (RB(i) < AVG(S_BODY_SHORT, i) && US(i) > AVG(S_SHADOW_LONG, i) &&
          LS(i) < AVG(S_SHADOW_VERY_SHORT, i) && BGAP_DN(i, i - 1)) ? 100 : 0;
}

static int kicking_common(const Bars* b, int i) {
  return COL(i - 1) == -COL(i) && RB(i - 1) > AVG(S_BODY_LONG, i - 1) &&
         US(i - 1) < AVG(S_SHADOW_VERY_SHORT, i - 1) && LS(i - 1) < AVG(S_SHADOW_VERY_SHORT, i - 1) &&
         RB(i) > AVG(S_BODY_LONG, i) && US(i) < AVG(S_SHADOW_VERY_SHORT, i) &&
         LS(i) < AVG(S_SHADOW_VERY_SHORT, i) &&
         ((COL(i - 1) == -1 && RGAP_UP(i, i - 1)) || (COL(i - 1) == 1 && RGAP_DN(i, i - 1)));
}

static int p_kicking(const Bars* b, int i) { return kicking_common(b, i) ? COL(i) * 100 : 0; }

static int p_kicking_by_length(const Bars* b, int i) {
  if (!kicking_common(b, i)) return 0;
  return (RB(i) > RB(i - 1) ? COL(i) : COL(i - 1)) * 100;
}

static int p_ladder_bottom(const Bars* b, int i) {
  return (COL(i - 4) == -1 && COL(i - 3) == -1 && COL(i - 2) == -1 && O(i - 4) > O(i - 3) &&
          O(i - 3) > O(i - 2) && C(i - 4) > C(i - 3) && C(i - 3) > C(i - 2) && COL(i - 1) == -1 &&
          US(i - 1) > AVG(S_SHADOW_VERY_SHORT, i - 1) && COL(i) == 1 && O(i) > O(i - 1) &&
          C(i) > H(i - 1)) ? 100 : 0;
}

static int p_long_legged_doji(const Bars* b, int i) {
  return (RB(i) <= AVG(S_BODY_DOJI, i) &&
          (LS(i) > AVG(S_SHADOW_LONG, i) || US(i) > AVG(S_SHADOW_LONG, i))) ? 100 : 0;
}

static int p_long_line(const Bars* b, int i) {
  return (RB(i) > AVG(S_BODY_LONG, i) && US(i) < AVG(S_SHADOW_SHORT, i) &&
          LS(i) < AVG(S_SHADOW_SHORT, i)) ? COL(i) * 100 : 0;
}

static int p_marubozu(const Bars* b, int i) {
  return (RB(i) > AVG(S_BODY_LONG, i) && US(i) < AVG(S_SHADOW_VERY_SHORT, i) &&
          LS(i) < AVG(S_SHADOW_VERY_SHORT, i)) ? COL(i) * 100 : 0;
}

static int p_matching_low(const Bars* b, int i) {
  return (COL(i - 1) == -1 && COL(i) == -1 && C(i) <= C(i - 1) + AVG(S_EQUAL, i - 1) &&
          C(i) >= C(i - 1) - AVG(S_EQUAL, i - 1)) ? 100 : 0;
}

static int p_mat_hold(const Bars* b, int i) {
  const double pen = 0.5;
  return (RB(i - 4) > AVG(S_BODY_LONG, i - 4) && RB(i - 3) < AVG(S_BODY_SHORT, i - 3) &&
          RB(i - 2) < AVG(S_BODY_SHORT, i - 2) && RB(i - 1) < AVG(S_BODY_SHORT, i - 1) &&
          COL(i - 4) == 1 && COL(i - 3) == -1 && COL(i) == 1 && BGAP_UP(i - 3, i - 4) &&
          BOTF(i - 2) < C(i - 4) && BOTF(i - 1) < C(i - 4) &&
          BOTF(i - 2) > C(i - 4) - RB(i - 4) * pen && BOTF(i - 1) > C(i - 4) - RB(i - 4) * pen &&
          fmaxf(C(i - 2), O(i - 2)) < O(i - 3) && fmaxf(C(i - 1), O(i - 1)) < fmaxf(C(i - 2), O(i - 2)) &&
          O(i) > C(i - 1) && C(i) > fmaxf(fmaxf(H(i - 3), H(i - 2)), H(i - 1))) ? 100 : 0;
}

static int p_on_neck(const Bars* b, int i) {
  return (COL(i - 1) == -1 && RB(i - 1) > AVG(S_BODY_LONG, i - 1) && COL(i) == 1 && O(i) < L(i - 1) &&
          C(i) <= L(i - 1) + AVG(S_EQUAL, i - 1) && C(i) >= L(i - 1) - AVG(S_EQUAL, i - 1)) ? -100 : 0;
}

static int p_piercing(const Bars* b, int i) {
  return (COL(i - 1) == -1 && RB(i - 1) > AVG(S_BODY_LONG, i - 1) && COL(i) == 1 &&
          RB(i) > AVG(S_BODY_LONG, i) && O(i) < L(i - 1) && C(i) < O(i - 1) &&
          (double)C(i) > (double)C(i - 1) + RB(i - 1) * 0.5) ? 100 : 0;
}

static int p_rickshaw_man(const Bars* b, int i) {
  const double mid = (double)L(i) + ((double)H(i) - (double)L(i)) / 2.0;
  return (RB(i) <= AVG(S_BODY_DOJI, i) && LS(i) > AVG(S_SHADOW_LONG, i) &&
          US(i) > AVG(S_SHADOW_LONG, i) && (double)BOTF(i) <= mid + AVG(S_NEAR, i) &&
          (double)TOPF(i) >= mid - AVG(S_NEAR, i)) ? 100 : 0;
}

static int p_rise_fall3_methods(const Bars* b, int i) {
  const int c4 = COL(i - 4);
  return (RB(i - 4) > AVG(S_BODY_LONG, i - 4) && RB(i - 3) < AVG(S_BODY_SHORT, i - 3) &&
          RB(i - 2) < AVG(S_BODY_SHORT, i - 2) && RB(i - 1) < AVG(S_BODY_SHORT, i - 1) &&
          RB(i) > AVG(S_BODY_LONG, i) && c4 == -COL(i - 3) && COL(i - 3) == COL(i - 2) &&
          COL(i - 2) == COL(i - 1) && COL(i - 1) == -COL(i) &&
          BOTF(i - 3) < H(i - 4) && TOPF(i - 3) > L(i - 4) && BOTF(i - 2) < H(i - 4) &&
          TOPF(i - 2) > L(i - 4) && BOTF(i - 1) < H(i - 4) && TOPF(i - 1) > L(i - 4) &&
          C(i - 2) * c4 < C(i - 3) * c4 && C(i - 1) * c4 < C(i - 2) * c4 &&
          O(i) * c4 > C(i - 1) * c4 && C(i) * c4 > C(i - 4) * c4) ? 100 * c4 : 0;
}

static int p_separating_lines(const Bars* b, int i) {
  if (COL(i - 1) == -COL(i) && O(i) <= O(i - 1) + AVG(S_EQUAL, i - 1) &&
      O(i) >= O(i - 1) - AVG(S_EQUAL, i - 1) && RB(i) > AVG(S_BODY_LONG, i) &&
      ((COL(i) == 1 && LS(i) < AVG(S_SHADOW_VERY_SHORT, i)) ||
       (COL(i) == -1 && US(i) < AVG(S_SHADOW_VERY_SHORT, i))))
    return COL(i) * 100;
  return 0;
}

static int p_shooting_star(const Bars* b, int i) {
  return (RB(i) < AVG(S_BODY_SHORT, i) && US(i) > AVG(S_SHADOW_LONG, i) &&
          LS(i) < AVG(S_SHADOW_VERY_SHORT, i) && BGAP_UP(i, i - 1)) ? -100 : 0;
}

static int p_short_line(const Bars* b, int i) {
  return (RB(i) < AVG(S_BODY_SHORT, i) && US(i) < AVG(S_SHADOW_SHORT, i) &&
          LS(i) < AVG(S_SHADOW_SHORT, i)) ? COL(i) * 100 : 0;
}

static int p_spinning_top(const Bars* b, int i) {
  return (RB(i) < AVG(S_BODY_SHORT, i) && US(i) > RB(i) && LS(i) > RB(i)) ? COL(i) * 100 : 0;
}

static int p_stalled_pattern(const Bars* b, int i) {
  return (COL(i - 2) == 1 && COL(i - 1) == 1 && COL(i) == 1 && C(i) > C(i - 1) && C(i - 1) > C(i - 2) &&
          RB(i - 2) > AVG(S_BODY_LONG, i - 2) && RB(i - 1) > AVG(S_BODY_LONG, i - 1) &&
          US(i - 1) < AVG(S_SHADOW_VERY_SHORT, i - 1) && O(i - 1) > O(i - 2) &&
          O(i - 1) <= C(i - 2) + AVG(S_NEAR, i - 2) && RB(i) < AVG(S_BODY_SHORT, i) &&
          O(i) >= C(i - 1) - RB(i) - AVG(S_NEAR, i - 1)) ? -100 : 0;
}

static int p_stick_sandwich(const Bars* b, int i) {
  return (COL(i - 2) == -1 && COL(i - 1) == 1 && COL(i) == -1 && L(i - 1) > C(i - 2) &&
          (double)C(i) <= (double)C(i - 2) + AVG(S_EQUAL, i - 2) &&
          (double)C(i) >= (double)C(i - 2) - AVG(S_EQUAL, i - 2)) ? 100 : 0;
}

static int p_takuri(const Bars* b, int i) {
  return (RB(i) <= AVG(S_BODY_DOJI, i) && US(i) < AVG(S_SHADOW_VERY_SHORT, i) &&
          LS(i) > AVG(S_SHADOW_VERY_LONG, i)) ? 100 : 0;
}

static int p_tasuki_gap(const Bars* b, int i) {
  if ((BGAP_UP(i - 1, i - 2) && COL(i - 1) == 1 && COL(i) == -1 && O(i) < C(i - 1) && O(i) > O(i - 1) &&
       C(i) < O(i - 1) && C(i) > fmaxf(C(i - 2), O(i - 2)) &&
       fabs(RB(i - 1) - RB(i)) < AVG(S_NEAR, i - 1)) ||
      (BGAP_DN(i - 1, i - 2) && COL(i - 1) == -1 && COL(i) == 1 && O(i) < O(i - 1) && O(i) > C(i - 1) &&
       C(i) > O(i - 1) && C(i) < fminf(C(i - 2), O(i - 2)) &&
       fabs(RB(i - 1) - RB(i)) < AVG(S_NEAR, i - 1)))
    return COL(i - 1) * 100;
  return 0;
}

static int p_thrusting(const Bars* b, int i) {
  return (COL(i - 1) == -1 && RB(i - 1) > AVG(S_BODY_LONG, i - 1) && COL(i) == 1 && O(i) < L(i - 1) &&
          C(i) > C(i - 1) + AVG(S_EQUAL, i - 1) &&
          (double)C(i) <= (double)C(i - 1) + RB(i - 1) * 0.5) ? -100 : 0;
}

/* TA-Lib quirk kept by the reference: all three doji tests use the average
 * anchored at i-2. */
static int p_tristar(const Bars* b, int i) {
  const double d = AVG(S_BODY_DOJI, i - 2);
  if (RB(i - 2) <= d && RB(i - 1) <= d && RB(i) <= d) {
    int out = 0;
    if (BGAP_UP(i - 1, i - 2) && fmaxf(O(i), C(i)) < fmaxf(O(i - 1), C(i - 1))) out = -100;
    if (BGAP_DN(i - 1, i - 2) && fminf(O(i), C(i)) > fminf(O(i - 1), C(i - 1))) out = 100;
    return out;
  }
  return 0;
}

static int p_unique_3_river(const Bars* b, int i) {
  return (RB(i - 2) > AVG(S_BODY_LONG, i - 2) && COL(i - 2) == -1 && COL(i - 1) == -1 &&
          C(i - 1) > C(i - 2) && O(i - 1) <= O(i - 2) && L(i - 1) < L(i - 2) &&
          RB(i) < AVG(S_BODY_SHORT, i) && COL(i) == 1 && O(i) > L(i - 1)) ? 100 : 0;
}

static int p_upside_gap_2_crows(const Bars* b, int i) {
  return (COL(i - 2) == 1 && RB(i - 2) > AVG(S_BODY_LONG, i - 2) && COL(i - 1) == -1 &&
          RB(i - 1) <= AVG(S_BODY_SHORT, i - 1) && BGAP_UP(i - 1, i - 2) && COL(i) == -1 &&
          O(i) > O(i - 1) && C(i) < C(i - 1) && C(i) > C(i - 2)) ? -100 : 0;
}

static int p_xside_gap_3_methods(const Bars* b, int i) {
  if (COL(i - 2) == COL(i - 1) && COL(i - 1) == -COL(i) && O(i) < fmaxf(C(i - 1), O(i - 1)) &&
      O(i) > fminf(C(i - 1), O(i - 1)) && C(i) < fmaxf(C(i - 2), O(i - 2)) &&
      C(i) > fminf(C(i - 2), O(i - 2)) &&
      ((COL(i - 2) == 1 && BGAP_UP(i - 1, i - 2)) || (COL(i - 2) == -1 && BGAP_DN(i - 1, i - 2))))
    return COL(i - 2) * 100;
  return 0;
}

/* Legacy split engulfing (CandleUtils.h:233-260): same signal as ENGULFING,
 * computed in float from bar 1. */
static int p_legacy_engulfing(const Bars* b, int i) { return p_engulfing(b, i); }

typedef int (*PatternFn)(const Bars*, int);
static const struct { PatternFn fn; int lookback; } kPattern[63] = {
  {p_doji, 10}, {p_hammer, 11}, {p_inverted_hammer, 11}, {p_legacy_engulfing, 1},
  {p_legacy_engulfing, 1}, {p_three_white_soldiers, 12}, {p_abandoned_baby, 12},
  {p_advance_block, 12}, {p_belt_hold, 10}, {p_breakaway, 14}, {p_two_crows, 12},
  {p_three_black_crows, 13}, {p_three_inside, 12}, {p_three_outside, 3},
  {p_three_line_strike, 8}, {p_three_stars_in_south, 12}, {p_closing_marubozu, 10},
  {p_conceal_baby_swallow, 13}, {p_counterattack, 11}, {p_dark_cloud_cover, 11},
  {p_doji_star, 11}, {p_dragonfly_doji, 10}, {p_engulfing, 2}, {p_evening_doji_star, 12},
  {p_evening_star, 12}, {p_gap_side_side_white, 7}, {p_gravestone_doji, 10},
  {p_hanging_man, 11}, {p_harami, 11}, {p_harami_cross, 11}, {p_high_wave, 10},
  {p_hikkake, 5}, {p_hikkake_mod, 10}, {p_homing_pigeon, 11}, {p_identical_three_crows, 12},
  {p_in_neck, 11}, {p_kicking, 11}, {p_kicking_by_length, 11}, {p_ladder_bottom, 14},
  {p_long_legged_doji, 10}, {p_long_line, 10}, {p_marubozu, 10}, {p_matching_low, 6},
  {p_mat_hold, 14}, {p_morning_doji_star, 12}, {p_morning_star, 12}, {p_on_neck, 11},
  {p_piercing, 11}, {p_rickshaw_man, 10}, {p_rise_fall3_methods, 14},
  {p_separating_lines, 11}, {p_shooting_star, 11}, {p_short_line, 10}, {p_spinning_top, 10},
  {p_stalled_pattern, 12}, {p_stick_sandwich, 7}, {p_takuri, 10}, {p_tasuki_gap, 7},
  {p_thrusting, 11}, {p_tristar, 12}, {p_unique_3_river, 12}, {p_upside_gap_2_crows, 12},
  {p_xside_gap_3_methods, 2},
};

int orc_cdl_count(void) { return 63; }
int orc_cdl_lookback(int k) { return (k >= 0 && k < 63) ? kPattern[k].lookback : -1; }

int orc_cdl_ragged(int k, const float* o, const float* h, const float* l, const float* c,
                   int S, const long long* off, int* out, int threads) {
  if (k < 0 || k >= 63) return -1;
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads)
  for (int s = 0; s < S; ++s) {
    const long long base = off[s];
    const int n = (int)(off[s + 1] - base);
    Bars b = {o + base, h + base, l + base, c + base};
    int* y = out + base;
    for (int i = 0; i < n; ++i) y[i] = i >= kPattern[k].lookback ? kPattern[k].fn(&b, i) : 0;
  }
  return 0;
}

int orc_cdl(int k, const float* o, const float* h, const float* l, const float* c, int S,
            int T, int* out, int threads) {
  long long* off = (long long*)malloc(sizeof(long long) * (size_t)(S + 1));
  for (int s = 0; s <= S; ++s) off[s] = (long long)s * T;
  const int rc = orc_cdl_ragged(k, o, h, l, c, S, off, out, threads);
  free(off);
  return rc;
}
