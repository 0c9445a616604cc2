/* Test infrastructure only: the FP64 CPU restatement that the CUDA path is
 * checked against. Never linked into the product. See ta_oracle.h for the
 * pinning status of each family. Citations are reference paths with line
 * numbers; "talib08" means src/compat/talib08_formulas.inc (vendored TA-Lib
 * 0.8.3, commit 62021c1d). Warm-up outputs are NaN.
 *
 * Two reference batch conventions apply on top of TA-Lib and are restated here:
 *  - single-input recurrences (EMA, RSI, MACD, DEMA, TEMA, T3) start after the
 *    row's leading NaNs (src/api/BatchFused.cu:34-41);
 *  - window families see NaN only in the windows that contain it
 *    (docs/BATCH_API.md "Numerical contract"; BatchFused.cu:73-143 sums each
 *    window directly). For finite rows a direct FP64 window sum of float32
 *    values equals TA-Lib's running sum bit for bit, since both are exact.
 */
#include "ta_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

static const double kNaN = __builtin_nan("");

typedef struct {
  const float* in[5];
  double* out[3];
  int n;
  const int* ip;
  const double* fp;
} RowCtx;

static void fill_nan(double* o, int n) {
  for (int i = 0; i < n; ++i) o[i] = kNaN;
}

static int leading_nan(const float* x, int n) {
  int f = 0;
  while (f < n && isnan(x[f])) ++f;
  return f;
}

/* talib08:5546-5627 TA_EMA coefficient setup (beta, k, beta<0.5 adjustment). */
static void ema_coeffs(int p, double* beta, double* k) {
  double b = (double)(p - 1) / (double)(p + 1);
  double kk = 1.0 - b;
  if (b < 0.5) b = 1.0 - kk;
  *beta = b;
  *k = kk;
}

/* ---------------------------------------------------------------- windows */

/* talib08:14748-14812 TA_SMA; window-local NaN per the batch contract. */
static void row_sma(RowCtx* r) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  for (int t = p - 1; t < n; ++t) {
    double s = 0.0;
    for (int k = t - p + 1; k <= t; ++k) s += (double)x[k];
    o[t] = s / (double)p;
  }
}

/* BatchFused.cu:133-138 SUM: direct FP64 window sum. */
static void row_sum(RowCtx* r) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  for (int t = p - 1; t < n; ++t) {
    double s = 0.0;
    for (int k = t - p + 1; k <= t; ++k) s += (double)x[k];
    o[t] = s;
  }
}

/* BatchFused.cu:110-119 MIN/MAX: float extrema (fminf/fmaxf ignore NaN); a
 * window starting inside the row's leading NaN run stays NaN
 * (LeadingNaN.cuh:21-27 in_leading_nan_prefix). */
static void row_minmax(RowCtx* r, int is_max) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  const int f = leading_nan(x, n);
  for (int t = p - 1; t < n; ++t) {
    float v = x[t - p + 1];
    for (int k = t - p + 2; k <= t; ++k) v = is_max ? fmaxf(v, x[k]) : fminf(v, x[k]);
    o[t] = (t - p + 1 < f) ? kNaN : (double)v;
  }
}

/* talib08:19171-19277 TA_WMA; its running sums of float32 values are exact in
 * FP64, so the direct weighted sum below is the same number. */
static void row_wma(RowCtx* r) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  if (p == 1) { for (int t = 0; t < n; ++t) o[t] = (double)x[t]; return; }
  const double divider = (double)p * (p + 1) / 2.0;
  for (int t = p - 1; t < n; ++t) {
    double s = 0.0;
    for (int k = 0; k < p; ++k) s += (double)x[t - p + 1 + k] * (double)(k + 1);
    o[t] = s / divider;
  }
}

/* talib08:18047-18183 TA_VAR (shifted running moments with reseeding), restated
 * on one row from index `first`. out[t] for t >= first+p-1. */
static void var_core(const double* x, int n, int p, double* o) {
  fill_nan(o, n);
  if (p > n) return;
  const double inv = 1.0 / (double)p;
  int start = p - 1, trailing = 0;
  double shift = x[trailing], t1 = 0.0, t2 = 0.0, tmp;
  for (int j = trailing; j < start; ++j) { tmp = x[j] - shift; t1 += tmp; tmp *= tmp; t2 += tmp; }
  int reseed = 32 * p;
  double peak = t2;
  for (int i = start; i < n; ++i) {
    tmp = x[i] - shift; t1 += tmp; tmp *= tmp; t2 += tmp;
    peak = t2 > peak ? t2 : peak;
    double mean = t1 * inv;
    double var = t2 * inv - mean * mean;
    tmp = x[trailing] - shift; t1 -= tmp; tmp *= tmp; t2 -= tmp;
    trailing += 1;
    reseed -= 1;
    if (var < 0.000001 * (peak * inv) || reseed <= 0) {
      reseed = 32 * p;
      int ws = i - (p - 1);
      tmp = 0.0;
      for (int j = ws; j <= i; ++j) tmp += x[j];
      shift = tmp * inv;
      t1 = 0.0; t2 = 0.0;
      for (int j = ws; j <= i; ++j) { tmp = x[j] - shift; t1 += tmp; tmp *= tmp; t2 += tmp; }
      mean = t1 * inv;
      var = t2 * inv - mean * mean;
      if (var < 0.000001 * (t2 * inv)) {
        shift = x[i];
        t1 = 0.0; t2 = 0.0;
        for (int j = ws; j <= i; ++j) { tmp = x[j] - shift; t1 += tmp; tmp *= tmp; t2 += tmp; }
        mean = t1 * inv;
        var = t2 * inv - mean * mean;
      }
      peak = t2;
      if (var < 0.000000000001 * (t2 * inv)) var = 0.0;
      tmp = x[ws] - shift; t1 -= tmp; tmp *= tmp; t2 -= tmp;
    }
    o[i] = var;
  }
}

static double* to_double(const float* x, int n) {
  double* d = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) d[i] = (double)x[i];
  return d;
}

/* Apply a TA-Lib window routine to every maximal NaN-free run of the row, so a
 * NaN only affects the windows containing it (the reference's batch contract;
 * TA-Lib's running totals would carry it forward). Outputs start NaN. */
typedef void (*SegFn)(const double* x, int n, int p, double* const* o, const double* fp);

static void by_segments(const float* xf, int n, int p, double* const* outs, int nout, const double* fp, SegFn fn) {
  for (int j = 0; j < nout; ++j) fill_nan(outs[j], n);
  double* x = to_double(xf, n);
  double* tmp[3];
  for (int j = 0; j < nout; ++j) tmp[j] = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  int i = 0;
  while (i < n) {
    while (i < n && isnan(x[i])) ++i;
    int e = i;
    while (e < n && !isnan(x[e])) ++e;
    if (e - i >= p) {
      double* o[3] = {tmp[0], nout > 1 ? tmp[1] : NULL, nout > 2 ? tmp[2] : NULL};
      fn(x + i, e - i, p, o, fp);
      for (int j = 0; j < nout; ++j)
        for (int t = i + p - 1; t < e; ++t) outs[j][t] = tmp[j][t - i];
    }
    i = e;
  }
  for (int j = 0; j < nout; ++j) free(tmp[j]);
  free(x);
}

static void seg_var(const double* x, int n, int p, double* const* o, const double* fp) {
  (void)fp;
  var_core(x, n, p, o[0]);
}

/* talib08:18047 TA_VAR (nbdev ignored, as TA_STDDEV passes 1.0). */
static void row_var(RowCtx* r) {
  double* outs[1] = {r->out[0]};
  by_segments(r->in[0], r->n, r->ip[0], outs, 1, NULL, seg_var);
}

/* talib08:16046-16100 TA_STDDEV = sqrt(TA_VAR) * nbdev. */
static void row_stddev(RowCtx* r) {
  const double nb = r->fp ? r->fp[0] : 1.0;
  row_var(r);
  double* o = r->out[0];
  for (int t = 0; t < r->n; ++t)
    if (!isnan(o[t])) o[t] = nb != 1.0 ? sqrt(o[t]) * nb : sqrt(o[t]);
}

/* talib08:2068-2283 TA_BBANDS with MA type SMA: the middle band is the running
 * SMA, the deviation is the shifted-moment variance of TA_VAR's scheme with
 * 32*p reseeding; equal multipliers use add/sub, unequal ones fma. */
static void seg_bbands(const double* x, int n, int p, double* const* outs, const double* fp) {
  const double up = fp[0], dn = fp[1];
  double *ou = outs[0], *om = outs[1], *ol = outs[2];
  if (p > n) return;
  const double inv = 1.0 / (double)p;
  int lb = p - 1, trailing = 0;
  double shift = x[trailing], ma = 0.0, v1 = 0.0, v2 = 0.0, tmp, mean, var;
  for (int j = trailing; j < lb; ++j) { ma += x[j]; tmp = x[j] - shift; v1 += tmp; tmp *= tmp; v2 += tmp; }
  int reseed = 32 * p;
  double peak = v2;
  for (int i = lb; i < n; ++i) {
    ma += x[i];
    tmp = x[i] - shift; v1 += tmp; tmp *= tmp; v2 += tmp;
    peak = v2 > peak ? v2 : peak;
    mean = v1 * inv;
    var = v2 * inv - mean * mean;
    const double mid = ma / p;
    ma -= x[trailing];
    tmp = x[trailing] - shift; v1 -= tmp; tmp *= tmp; v2 -= tmp;
    trailing += 1;
    reseed -= 1;
    if (var < 0.000001 * (peak * inv) || reseed <= 0) {
      reseed = 32 * p;
      int ws = i - lb;
      tmp = 0.0;
      for (int j = ws; j <= i; ++j) tmp += x[j];
      shift = tmp * inv;
      v1 = 0.0; v2 = 0.0;
      for (int j = ws; j <= i; ++j) { tmp = x[j] - shift; v1 += tmp; tmp *= tmp; v2 += tmp; }
      mean = v1 * inv;
      var = v2 * inv - mean * mean;
      if (var < 0.000001 * (v2 * inv)) {
        shift = x[i];
        v1 = 0.0; v2 = 0.0;
        for (int j = ws; j <= i; ++j) { tmp = x[j] - shift; v1 += tmp; tmp *= tmp; v2 += tmp; }
        mean = v1 * inv;
        var = v2 * inv - mean * mean;
      }
      peak = v2;
      if (var < 0.000000000001 * (v2 * inv)) var = 0.0;
      tmp = x[ws] - shift; v1 -= tmp; tmp *= tmp; v2 -= tmp;
    }
    const double sd = var != 0.0 ? sqrt(var) : 0.0;
    om[i] = mid;
    if (up == dn) {
      const double d = sd * up;
      ou[i] = mid + d;
      ol[i] = mid - d;
    } else {
      ou[i] = fma(sd, up, mid);
      ol[i] = mid - sd * dn;
    }
  }
}

static void row_bbands(RowCtx* r) {
  double* outs[3] = {r->out[0], r->out[1], r->out[2]};
  by_segments(r->in[0], r->n, r->ip[0], outs, 3, r->fp, seg_bbands);
}

/* talib08:9087-9197 TA_LINEARREG: least-squares line over the window, value at
 * its last bar, fma(m, p-1, b). Evaluated per window directly. */
static void row_linearreg(RowCtx* r) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  const double sumX = (double)p * (p - 1) * 0.5;
  const double sumXSqr = (double)p * (p - 1) * (2 * p - 1) / 6.0;
  const double divisor = sumX * sumX - p * sumXSqr;
  for (int t = p - 1; t < n; ++t) {
    double sy = 0.0, sxy = 0.0;
    for (int i = p; i-- != 0;) {
      const double v = (double)x[t - i];
      sy += v;
      sxy += (double)i * v;
    }
    const double m = (p * sxy - sumX * sy) / divisor;
    const double b = (sy - m * sumX) / (double)p;
    o[t] = fma(m, (double)(p - 1), b);
  }
}

/* src/indicators/Correl.cu:23-75 CORREL: Pearson correlation of each window;
 * 0 when either variance or their product (<= 1e-14) vanishes, and 0 from the
 * first non-finite bar of the row onwards (findInvalidSuffix, :14-21). The
 * moments are taken about the window mean (two passes) in FP64. */
static void row_correl(RowCtx* r) {
  const float *x = r->in[0], *y = r->in[1]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  int first_bad = n;
  for (int i = 0; i < n; ++i)
    if (!isfinite(x[i]) || !isfinite(y[i])) { first_bad = i; break; }
  for (int t = p - 1; t < n; ++t) {
    if (t >= first_bad) { o[t] = 0.0; continue; }
    double mx = 0.0, my = 0.0;
    for (int k = t - p + 1; k <= t; ++k) { mx += x[k]; my += y[k]; }
    mx /= p; my /= p;
    double sxx = 0.0, syy = 0.0, sxy = 0.0;
    for (int k = t - p + 1; k <= t; ++k) {
      const double dx = (double)x[k] - mx, dy = (double)y[k] - my;
      sxx += dx * dx; syy += dy * dy; sxy += dx * dy;
    }
    const double prod = sxx * syy;
    o[t] = (sxx > 0.0 && syy > 0.0 && prod > 1e-14) ? sxy / sqrt(prod) : 0.0;
  }
}

/* src/indicators/WILLR.cu:11-30 WILLR: float window extrema, FP64 ratio times
 * -100, clamped to [-100, 0]; 0 for a zero range. */
static void row_willr(RowCtx* r) {
  const float *h = r->in[0], *l = r->in[1], *c = r->in[2];
  int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  for (int i = p - 1; i < n; ++i) {
    float hi = h[i], lo = l[i];
    for (int j = 1; j < p; ++j) {
      if (h[i - j] > hi) hi = h[i - j];
      if (l[i - j] < lo) lo = l[i - j];
    }
    const double den = (double)hi - lo;
    const double v = den == 0.0 ? 0.0 : (((double)hi - c[i]) / den) * -100.0;
    o[i] = isnan(v) ? kNaN : fmin(0.0, fmax(-100.0, v));
  }
}

/* src/indicators/CCI.cu:11-40 CCI: typical price ((h+l)+c)/3 in FP64, SMA and
 * mean absolute deviation over the window; 0 unless both numerator and mean
 * deviation are nonzero. */
static void row_cci(RowCtx* r) {
  const float *h = r->in[0], *l = r->in[1], *c = r->in[2];
  int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  for (int i = p - 1; i < n; ++i) {
    double sum = 0.0;
    for (int j = 0; j < p; ++j) sum += ((double)h[i - j] + l[i - j] + c[i - j]) / 3.0;
    const double sma = sum / p;
    double dev = 0.0;
    for (int j = 0; j < p; ++j) dev += fabs(((double)h[i - j] + l[i - j] + c[i - j]) / 3.0 - sma);
    const double md = dev / p;
    const double num = ((double)h[i] + l[i] + c[i]) / 3.0 - sma;
    o[i] = (num != 0.0 && md != 0.0) ? num / (0.015 * md) : 0.0;
  }
}

/* talib08:16115-16302 TA_STOCH with SMA slowing: fastK from window extrema with
 * TA-Lib's scaled zero-range test (1e-14), then SMA(q) twice. */
static void row_stoch(RowCtx* r) {
  const float *h = r->in[0], *l = r->in[1], *c = r->in[2];
  const int n = r->n, p = r->ip[0], q = r->ip[1];
  double *ok = r->out[0], *od = r->out[1];
  fill_nan(ok, n); fill_nan(od, n);
  const int lb = p - 1 + 2 * (q - 1);
  if (lb >= n) return;
  double* fk = (double*)malloc(sizeof(double) * (size_t)n);
  for (int t = p - 1; t < n; ++t) {
    double lo = l[t - p + 1], hi = h[t - p + 1];
    for (int k = t - p + 2; k <= t; ++k) {
      if ((double)l[k] < lo) lo = l[k];
      if ((double)h[k] > hi) hi = h[k];
    }
    const double range = hi - lo;
    fk[t] = fabs(range) <= 1e-14 * (fabs(hi) + fabs(lo)) ? 0.0 : ((double)c[t] - lo) / range * 100.0;
  }
  double* sk = (double*)malloc(sizeof(double) * (size_t)n);
  for (int t = p - 1 + q - 1; t < n; ++t) {
    double s = 0.0;
    for (int k = t - q + 1; k <= t; ++k) s += fk[k];
    sk[t] = s / (double)q;
  }
  for (int t = lb; t < n; ++t) {
    double s = 0.0;
    for (int k = t - q + 1; k <= t; ++k) s += sk[k];
    ok[t] = sk[t];
    od[t] = s / (double)q;
  }
  free(fk); free(sk);
}

/* ------------------------------------------------------------ recurrences */

/* talib08:5546-5627 TA_EMA (SMA seed, then fma(beta, prev, k*x)); period 1
 * copies the input. Starts after leading NaNs. */
static void ema_row(const float* x, int n, int p, double* o) {
  fill_nan(o, n);
  const int f = leading_nan(x, n);
  if (p == 1) { for (int t = f; t < n; ++t) o[t] = (double)x[t]; return; }
  if (n - f < p) return;
  double beta, k; ema_coeffs(p, &beta, &k);
  double s = 0.0;
  for (int t = f; t < f + p; ++t) s += (double)x[t];
  double prev = s / p;
  o[f + p - 1] = prev;
  for (int t = f + p; t < n; ++t) { prev = fma(beta, prev, k * (double)x[t]); o[t] = prev; }
}

static void row_ema(RowCtx* r) { ema_row(r->in[0], r->n, r->ip[0], r->out[0]); }

/* talib08:13996-14115 TA_RSI: invPeriod multiplies, gain/loss sums over the
 * first p changes, Wilder steps after; 50 when both are zero. A NaN change
 * makes the row NaN from there on (StreamStates.h:663, precise::RsiState).
 * Starts after leading NaNs. */
static void row_rsi(RowCtx* r) {
  const float* x = r->in[0]; const int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  const int f = leading_nan(x, n);
  if (n - f <= p) return;
  const double inv = 1.0 / (double)p;
  double prev = x[f], gain = 0.0, loss = 0.0;
  int poisoned = 0;
  int t = f + 1;
  for (int i = p; i > 0; --i, ++t) {
    const double v = x[t], d = v - prev;
    prev = v;
    if (isnan(d)) poisoned = 1;
    const double g = d > 0.0 ? d : 0.0;
    gain += g; loss += g - d;
  }
  loss *= inv; gain *= inv;
  t = f + p;
  for (;;) {
    const double tot = gain + loss;
    o[t] = poisoned ? kNaN : (tot > 0.0 ? 100.0 * (gain / tot) : 50.0);
    if (++t >= n) break;
    const double v = x[t], d = v - prev;
    prev = v;
    if (isnan(d)) poisoned = 1;
    loss *= (double)(p - 1); gain *= (double)(p - 1);
    const double g = d > 0.0 ? d : 0.0;
    gain += g; loss += g - d;
    loss *= inv; gain *= inv;
  }
}

/* talib08:9316-9505 TA_MACD: slow seed = SMA of the first `slow` bars, fast seed
 * = SMA of the `fast` bars ending at slow-1, signal seed = SMA of the first
 * `signal` MACD values; output from slow+signal-2. Reversed periods swap.
 * Starts after leading NaNs. */
static void row_macd(RowCtx* r) {
  const float* x = r->in[0]; const int n = r->n;
  int fast = r->ip[0], slow = r->ip[1];
  const int sig = r->ip[2];
  double *om = r->out[0], *os = r->out[1], *oh = r->out[2];
  fill_nan(om, n); fill_nan(os, n); fill_nan(oh, n);
  if (slow < fast) { int t = slow; slow = fast; fast = t; }
  double sb, sk, fb, fk, gb, gk;
  ema_coeffs(slow, &sb, &sk);
  ema_coeffs(fast, &fb, &fk);
  ema_coeffs(sig, &gb, &gk);
  const int f = leading_nan(x, n);
  const int start = f + slow - 1;           /* first MACD value */
  const int ready = start + sig - 1;        /* first output */
  if (ready >= n) return;
  double s = 0.0;
  for (int t = f; t < f + slow; ++t) s += (double)x[t];
  double ps = s / slow;
  double pf = 0.0;
  for (int t = start - fast + 1; t <= start; ++t) pf += (double)x[t];
  pf = pf / fast;
  double macd = pf - ps;
  double psig = macd;
  int t = start + 1;
  for (int i = sig - 1; i > 0; --i, ++t) {
    const double v = x[t];
    pf = fma(fb, pf, fk * v);
    ps = fma(sb, ps, sk * v);
    macd = pf - ps;
    psig += macd;
  }
  psig = psig / sig;
  om[ready] = macd; os[ready] = psig; oh[ready] = macd - psig;
  for (t = ready + 1; t < n; ++t) {
    const double v = x[t];
    pf = fma(fb, pf, fk * v);
    ps = fma(sb, ps, sk * v);
    macd = pf - ps;
    psig = sig == 1 ? macd : fma(gb, psig, gk * macd);
    om[t] = macd; os[t] = psig; oh[t] = macd - psig;
  }
}

/* talib08:17625-17690 TRUE_RANGE as TA-Lib computes it (greatest of three). */
static double true_range(double hi, double lo, double yc) {
  double g = hi - lo;
  const double a = fabs(yc - hi);
  if (a > g) g = a;
  const double b = fabs(yc - lo);
  if (b > g) g = b;
  return g;
}

static void row_trange(RowCtx* r) {
  const float *h = r->in[0], *l = r->in[1], *c = r->in[2];
  const int n = r->n; double* o = r->out[0];
  fill_nan(o, n);
  for (int t = 1; t < n; ++t) o[t] = true_range(h[t], l[t], c[t - 1]);
}

/* talib08:1931-2057 TA_ATR: mean of the first p true ranges (bars 1..p), then
 * fma(wBeta, prev, wAlpha*tr) with wBeta=(p-1)/p. */
static void atr_row(const float* h, const float* l, const float* c, int n, int p, double* o) {
  fill_nan(o, n);
  if (p >= n) return;
  const double wb = (double)(p - 1) / (double)p, wa = 1.0 - wb;
  double tot = 0.0;
  for (int t = 1; t <= p; ++t) tot += true_range(h[t], l[t], c[t - 1]);
  double prev = tot / p;
  o[p] = prev;
  for (int t = p + 1; t < n; ++t) {
    prev = fma(wb, prev, wa * true_range(h[t], l[t], c[t - 1]));
    o[t] = prev;
  }
}

static void row_atr(RowCtx* r) { atr_row(r->in[0], r->in[1], r->in[2], r->n, r->ip[0], r->out[0]); }

/* StreamStates.h:708-721 precise::NatrState: ATR/close*100 in FP64, 0 for a zero
 * close; period 1 is the unnormalised true range. */
static void row_natr(RowCtx* r) {
  const float* c = r->in[2]; const int n = r->n, p = r->ip[0]; double* o = r->out[0];
  atr_row(r->in[0], r->in[1], c, n, p, o);
  if (p == 1) return;
  for (int t = 0; t < n; ++t)
    if (!isnan(o[t])) o[t] = c[t] == 0.0f ? 0.0 : (o[t] / (double)c[t]) * 100.0;
}

/* DX and ADX as the reference computes them (src/indicators/DX.cu:18-52, 85-135;
 * ADX.cu:44-124; BatchShort.cu:168-230): bar 0 contributes TR = H-L and no
 * directional movement; TR/+DM/-DM are summed over bars 0..p-1 and then
 * smoothed as S = (p-1)/p*S + x; DX = 100|DI+ - DI-|/(DI+ + DI-) from bar p;
 * ADX is the mean of DX over bars p..2p-1, then ADX = (p-1)/p*ADX + DX/p.
 * Zero TR or zero DI sum give DI/DX 0. Arithmetic in FP64. */
static void dm_row(const float* h, const float* l, const float* c, int n, int p,
                   double* dx_out, double* adx_out) {
  if (dx_out) fill_nan(dx_out, n);
  if (adx_out) fill_nan(adx_out, n);
  if (p > n) return;
  const double a = ((double)p - 1.0) / (double)p;
  double tr = 0.0, pdm = 0.0, mdm = 0.0, adx = 0.0;
  for (int i = 0; i < n; ++i) {
    double plus = 0.0, minus = 0.0, range;
    if (i == 0) {
      range = (double)h[0] - (double)l[0];
    } else {
      const float up = h[i] - h[i - 1], down = l[i - 1] - l[i];
      plus = (up > 0.0f && up > down) ? up : 0.0f;
      minus = (down > 0.0f && down > up) ? down : 0.0f;
      const double hh = h[i], ll = l[i], pc = c[i - 1];
      range = fmax(hh - ll, fmax(fabs(hh - pc), fabs(ll - pc)));
    }
    if (i < p) { tr += range; pdm += plus; mdm += minus; continue; }
    tr = a * tr + range;
    pdm = a * pdm + plus;
    mdm = a * mdm + minus;
    const double dip = tr > 0.0 ? 100.0 * pdm / tr : 0.0;
    const double dim = tr > 0.0 ? 100.0 * mdm / tr : 0.0;
    const double tot = dip + dim;
    const double dx = tot > 0.0 ? 100.0 * fabs(dip - dim) / tot : 0.0;
    if (dx_out) dx_out[i] = dx;
    if (i < 2 * p) {
      adx += dx;
      if (i == 2 * p - 1) { adx /= p; if (adx_out) adx_out[i] = adx; }
    } else {
      adx = a * adx + dx / p;
      if (adx_out) adx_out[i] = adx;
    }
  }
}

static void row_dx(RowCtx* r) { dm_row(r->in[0], r->in[1], r->in[2], r->n, r->ip[0], r->out[0], NULL); }
static void row_adx(RowCtx* r) { dm_row(r->in[0], r->in[1], r->in[2], r->n, r->ip[0], NULL, r->out[0]); }

/* StreamStates.h:446-475 ObvState: bar 0 adds its raw volume, later bars the
 * volume signed by the close change; FP64 accumulator. */
static void row_obv(RowCtx* r) {
  const float *c = r->in[0], *v = r->in[1]; const int n = r->n; double* o = r->out[0];
  double acc = 0.0;
  for (int i = 0; i < n; ++i) {
    if (i == 0) acc += (double)v[0];
    else {
      const double pr = c[i], pv = c[i - 1];
      const double s = pr > pv ? 1.0 : (pr < pv ? -1.0 : 0.0);
      acc += s * (double)v[i];
    }
    o[i] = acc;
  }
}

/* StreamStates.h:481-506 AdState: ((c-l)-(h-c))/(h-l)*v, skipped for
 * non-finite bars and non-positive ranges. */
static double ad_term(double hi, double lo, double cl, double vol) {
  if (isfinite(hi) && isfinite(lo) && isfinite(cl) && isfinite(vol)) {
    const double range = hi - lo;
    if (range > 0.0) return (((cl - lo) - (hi - cl)) / range) * vol;
  }
  return 0.0;
}

static void row_ad(RowCtx* r) {
  const float *h = r->in[0], *l = r->in[1], *c = r->in[2], *v = r->in[3];
  const int n = r->n; double* o = r->out[0];
  double acc = 0.0;
  for (int i = 0; i < n; ++i) { acc += ad_term(h[i], l[i], c[i], v[i]); o[i] = acc; }
}

/* StreamStates.h:723-745 precise::AdoscState: EMA(fast) - EMA(slow) of the AD
 * line, both seeded with AD[0], k = 2/(n+1); warm-up max(fast,slow)-1. */
static void row_adosc(RowCtx* r) {
  const float *h = r->in[0], *l = r->in[1], *c = r->in[2], *v = r->in[3];
  const int n = r->n, fp = r->ip[0], sp = r->ip[1]; double* o = r->out[0];
  const int warm = (fp > sp ? fp : sp) - 1;
  const double kf = 2.0 / (fp + 1.0), ks = 2.0 / (sp + 1.0);
  double acc = 0.0, fast = 0.0, slow = 0.0;
  for (int i = 0; i < n; ++i) {
    acc += ad_term(h[i], l[i], c[i], v[i]);
    if (i == 0) fast = slow = acc;
    else {
      fast = kf * acc + (1.0 - kf) * fast;
      slow = ks * acc + (1.0 - ks) * slow;
    }
    o[i] = i < warm ? kNaN : fast - slow;
  }
}

/* StreamStates.h:749-792 precise::MfiState: typical price ((h+l)+c)/3 in FP64,
 * money flow = price*volume signed by the price change (non-finite prices give
 * no flow); positive/negative window sums over p flows; 0 when the total is
 * below 1. The sums are taken per window directly (the state's running sums
 * with re-summing differ only in rounding). */
static void row_mfi(RowCtx* r) {
  const float *h = r->in[0], *l = r->in[1], *c = r->in[2], *v = r->in[3];
  const int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  if (n < 1) return;
  double* pos = (double*)calloc((size_t)n, sizeof(double));
  double* neg = (double*)calloc((size_t)n, sizeof(double));
  double prev = ((double)h[0] + l[0] + c[0]) / 3.0;
  for (int i = 1; i < n; ++i) {
    const double price = ((double)h[i] + l[i] + c[i]) / 3.0;
    if (isfinite(price) && isfinite(prev)) {
      const double flow = price * (double)v[i];
      if (price > prev) pos[i] = flow;
      else if (price < prev) neg[i] = flow;
    }
    prev = price;
  }
  for (int i = p; i < n; ++i) {
    double ps = 0.0, ns = 0.0;
    for (int k = i - p + 1; k <= i; ++k) { ps += pos[k]; ns += neg[k]; }
    const double tot = ps + ns;
    o[i] = tot < 1.0 ? 0.0 : 100.0 * (ps / tot);
  }
  free(pos); free(neg);
}

/* talib08:4846-4945 TA_DEMA, talib08:17496-17612 TA_TEMA, talib08:17331-17481
 * TA_T3: cascades of EMAs where stage k+1 is seeded with the SMA of stage k's
 * first p values. DEMA/TEMA use TA_EMA's coefficients, T3 uses k=2/(p+1) and
 * fma(1-k, e, k*x). Starts after leading NaNs. */
static void cascade_row(const float* x, int n, int p, int stages, int t3, double v,
                        double* o) {
  fill_nan(o, n);
  const int f = leading_nan(x, n);
  const int lb = stages * (p - 1);
  if (p == 1) { for (int t = f + lb; t < n; ++t) o[t] = (double)x[t]; return; }
  if (f + lb >= n) return;
  double beta, k;
  if (t3) { k = 2.0 / (p + 1.0); beta = 1.0 - k; } else ema_coeffs(p, &beta, &k);
  double e[6] = {0, 0, 0, 0, 0, 0};
  double seed[6] = {0, 0, 0, 0, 0, 0};
  int cnt[6] = {0, 0, 0, 0, 0, 0};
  int ready[6] = {0, 0, 0, 0, 0, 0};
  double c1 = 0, c2 = 0, c3 = 0, c4 = 0;
  if (t3) {
    const double tr = v * v;
    c1 = -(tr * v);
    c2 = 3.0 * (tr - c1);
    c3 = -6.0 * tr - 3.0 * (v - c1);
    c4 = fma(3.0, tr, fma(3.0, v, 1.0) - c1);
  }
  for (int t = f; t < n; ++t) {
    double in = (double)x[t];
    int alive = 1;
    for (int s = 0; s < stages && alive; ++s) {
      if (!ready[s]) {
        seed[s] += in;
        if (++cnt[s] == p) { e[s] = seed[s] / p; ready[s] = 1; }
        else { alive = 0; break; }
      } else {
        e[s] = fma(beta, e[s], k * in);
      }
      in = e[s];
    }
    if (!alive || !ready[stages - 1]) continue;
    if (stages == 2) o[t] = 2.0 * e[0] - e[1];
    else if (stages == 3) o[t] = e[2] + (3.0 * e[0] - 3.0 * e[1]);
    else o[t] = fma(c4, e[2], fma(c3, e[3], fma(c1, e[5], c2 * e[4])));
  }
}

static void row_dema(RowCtx* r) { cascade_row(r->in[0], r->n, r->ip[0], 2, 0, 0.0, r->out[0]); }
static void row_tema(RowCtx* r) { cascade_row(r->in[0], r->n, r->ip[0], 3, 0, 0.0, r->out[0]); }
static void row_t3(RowCtx* r) { cascade_row(r->in[0], r->n, r->ip[0], 6, 1, r->fp[0], r->out[0]); }

/* ------------------------------------------------- ROC, RMA, price transforms */

/* The ROC kernels in float arithmetic (C float ops, no contraction), from bar
 * p with prev = x[t-p]; the ratios give 0 where prev == 0:
 *   0 ROC     src/indicators/ROC.cu:10-21      ((x - prev) / prev) * 100
 *   1 ROCP    src/indicators/ROCP.cu:10-20     (x - prev) / prev
 *   2 ROCR    src/indicators/ROCR.cu:10-20     x / prev
 *   3 ROCR100 src/indicators/ROCR100.cu:10-21  (x / prev) * 100
 *   4 MOM     src/indicators/Momentum.cu:10-18 x - prev */
static void roc_row(RowCtx* r, int mode) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  for (int t = p; t < n; ++t) {
    const float prev = x[t - p], curr = x[t];
    float v;
    if (mode == 4) v = curr - prev;
    else if (!(prev != 0.0f)) v = 0.0f;
    else if (mode == 0) v = ((curr - prev) / prev) * 100.0f;
    else if (mode == 1) v = (curr - prev) / prev;
    else if (mode == 2) v = curr / prev;
    else v = (curr / prev) * 100.0f;
    o[t] = (double)v;
  }
}
static void row_roc(RowCtx* r) { roc_row(r, 0); }
static void row_rocp(RowCtx* r) { roc_row(r, 1); }
static void row_rocr(RowCtx* r) { roc_row(r, 2); }
static void row_rocr100(RowCtx* r) { roc_row(r, 3); }
static void row_mom(RowCtx* r) { roc_row(r, 4); }

/* talib08:13614-13683 TA_RMA (mean of the first p, then fma(wBeta, y,
 * wAlpha * x)); the reference's TA-Lib runner starts after the row's leading
 * NaNs (src/compat/Talib08.cu:72-84). No period-1 shortcut: a NaN propagates. */
static void row_rma(RowCtx* r) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  const int f = leading_nan(x, n);
  if (n - f < p) return;
  const double wb = (double)(p - 1) / (double)p, wa = 1.0 - wb;
  double s = 0.0;
  for (int t = f; t < f + p; ++t) s += (double)x[t];
  double prev = s / p;
  o[f + p - 1] = prev;
  for (int t = f + p; t < n; ++t) { prev = fma(wb, prev, wa * (double)x[t]); o[t] = prev; }
}

/* src/indicators/MedPrice.cu:12-14: 0.5f * (h + l) in float. */
static void row_medprice(RowCtx* r) {
  for (int t = 0; t < r->n; ++t) r->out[0][t] = (double)(0.5f * (r->in[0][t] + r->in[1][t]));
}

/* src/indicators/TypPrice.cu:13-15: (h + l + c) / 3.0f in float. */
static void row_typprice(RowCtx* r) {
  for (int t = 0; t < r->n; ++t)
    r->out[0][t] = (double)((r->in[0][t] + r->in[1][t] + r->in[2][t]) / 3.0f);
}

/* src/indicators/AvgPrice.cu:16-18: (o + h + l + c) * 0.25f in float. */
static void row_avgprice(RowCtx* r) {
  for (int t = 0; t < r->n; ++t)
    r->out[0][t] = (double)((r->in[0][t] + r->in[1][t] + r->in[2][t] + r->in[3][t]) * 0.25f);
}

/* src/indicators/WclPrice.cu:14-16: (h + l + 2.0f * c) * 0.25f in float. */
static void row_wclprice(RowCtx* r) {
  for (int t = 0; t < r->n; ++t)
    r->out[0][t] = (double)((r->in[0][t] + r->in[1][t] + 2.0f * r->in[2][t]) * 0.25f);
}

/* src/indicators/MIDPOINT.cu:13-35: fmaxf / fminf over the window of one
 * plane, 0.5f * (max + min) from bar p-1; a window starting inside the row's
 * leading NaN run is NaN (LeadingNaN.cuh:22-28 in_leading_nan_prefix). */
static void row_midpoint(RowCtx* r) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  const int f = leading_nan(x, n);
  for (int t = p - 1; t < n; ++t) {
    float hi = x[t - p + 1], lo = hi;
    for (int k = t - p + 2; k <= t; ++k) { hi = fmaxf(hi, x[k]); lo = fminf(lo, x[k]); }
    o[t] = (t - p + 1 < f) ? kNaN : (double)(0.5f * (hi + lo));
  }
}

/* src/indicators/ClubPack.cu:375-407 rollingStrictKernel: NaN-strict windows
 * (any non-finite bar gives NaN), FP64 sums from the newest bar back; mode 0
 * mean, 1 max, 2 min, 3 population std sqrt(max(0, sq/p - mean^2)) with the
 * fma that nvcc's default contraction forms for sq/p - mean*mean. */
static void rolling_row(RowCtx* r, int mode) {
  const float* x = r->in[0]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  for (int t = p - 1; t < n; ++t) {
    int ok = 1;
    double sum = 0.0, sq = 0.0;
    float mx = x[t], mn = x[t];
    for (int k = 0; k < p; ++k) {
      const float v = x[t - k];
      if (!isfinite(v)) { ok = 0; break; }
      sum += v;
      sq = fma((double)v, (double)v, sq);
      mx = fmaxf(mx, v);
      mn = fminf(mn, v);
    }
    if (!ok) continue;
    if (mode == 0) o[t] = (double)(float)(sum / p);
    else if (mode == 1) o[t] = mx;
    else if (mode == 2) o[t] = mn;
    else {
      const double mean = sum / p;
      o[t] = (double)(float)sqrt(fmax(0.0, fma(-mean, mean, sq / p)));
    }
  }
}
static void row_rmean(RowCtx* r) { rolling_row(r, 0); }
static void row_rmax(RowCtx* r) { rolling_row(r, 1); }
static void row_rmin(RowCtx* r) { rolling_row(r, 2); }
static void row_rstd(RowCtx* r) { rolling_row(r, 3); }

/* The reference's TA-Lib device runner (src/compat/Talib08.cu:72-97) starts a
 * row at the first bar where no input is NaN (the last bar when none is
 * complete); TA_IBS: (c - l) / (h - l), 0.5 where h - l <= 0; TA_MARKETFI:
 * (h - l) / v, 0 where v == 0 (talib08 TA_IBS, TA_MARKETFI). */
static void talib_bar_row(RowCtx* r, int mode) {
  const float* a = r->in[0]; const float* b = r->in[1]; const float* z = r->in[2];
  int n = r->n; double* o = r->out[0];
  fill_nan(o, n);
  int f = 0;
  while (f < n - 1 && (isnan(a[f]) || isnan(b[f]) || isnan(z[f]))) ++f;
  for (int t = f; t < n; ++t) {
    double v;
    if (mode == 0) {
      const double range = (double)a[t] - (double)b[t];
      v = ((double)z[t] - (double)b[t]) / range;
      if (range <= 0.0) v = 0.5;
    } else {
      v = (double)z[t] != 0.0 ? ((double)a[t] - (double)b[t]) / (double)z[t] : 0.0;
    }
    o[t] = (double)(float)v;
  }
}
static void row_ibs(RowCtx* r) { talib_bar_row(r, 0); }
static void row_marketfi(RowCtx* r) { talib_bar_row(r, 1); }

/* talib08 TA_QSTICK (running FP64 sum of close - open, mean over p bars)
 * after the runner's start at the first bar with open and close present
 * (src/compat/Talib08.cu:72-84); a NaN difference stays in the running sum. */
static void row_qstick(RowCtx* r) {
  const float* op = r->in[0]; const float* cl = r->in[1];
  int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  int f = 0;
  while (f < n - 1 && (isnan(op[f]) || isnan(cl[f]))) ++f;
  if (n - f < p) return;
  double total = 0.0;
  int trailing = f, i = f;
  for (; i < f + p - 1; ++i) total += (double)cl[i] - (double)op[i];
  for (; i < n; ++i) {
    total += (double)cl[i] - (double)op[i];
    o[i] = (double)(float)(total / (double)p);
    total -= (double)cl[trailing] - (double)op[trailing];
    ++trailing;
  }
}

/* src/indicators/MIDPRICE.cu:11-24: fmaxf / fminf over [t-p+1, t] (NaN
 * ignored unless the whole window is NaN), 0.5f * (max + min), from bar p-1. */
static void row_midprice(RowCtx* r) {
  const float* h = r->in[0]; const float* l = r->in[1]; int n = r->n, p = r->ip[0]; double* o = r->out[0];
  fill_nan(o, n);
  for (int t = p - 1; t < n; ++t) {
    float hi = h[t - p + 1], lo = l[t - p + 1];
    for (int k = t - p + 2; k <= t; ++k) { hi = fmaxf(hi, h[k]); lo = fminf(lo, l[k]); }
    o[t] = (double)(0.5f * (hi + lo));
  }
}

/* src/indicators/Aroon.cu:11-52 and src/indicators/AroonOscillator.cu:12-40:
 * from bar t back over p bars, strict comparisons seeded with bar t itself
 * (ties keep the most recent bar, NaNs never win, a NaN at t keeps t), each
 * line 100.0f * (p - since) / (float)p in float, from bar p; the oscillator
 * is up - down in float. Outputs: AROON down then up. */
static float aroon_line_f(int p, int since) { return 100.0f * (float)(p - since) / (float)p; }

static void aroon_row(RowCtx* r, int osc) {
  const float* h = r->in[0]; const float* l = r->in[1];
  int n = r->n, p = r->ip[0];
  fill_nan(r->out[0], n);
  if (!osc) fill_nan(r->out[1], n);
  for (int t = p; t < n; ++t) {
    float mx = h[t], mn = l[t];
    int sh = 0, sl = 0;
    for (int d = 1; d <= p; ++d) {
      if (h[t - d] > mx) { mx = h[t - d]; sh = d; }
      if (l[t - d] < mn) { mn = l[t - d]; sl = d; }
    }
    const float up = aroon_line_f(p, sh), dn = aroon_line_f(p, sl);
    if (osc) {
      r->out[0][t] = (double)(up - dn);
    } else {
      r->out[0][t] = (double)dn;
      r->out[1][t] = (double)up;
    }
  }
}
static void row_aroon(RowCtx* r) { aroon_row(r, 0); }
static void row_aroonosc(RowCtx* r) { aroon_row(r, 1); }

/* --------------------------------------------------------------- dispatch */

typedef struct { int nin, nout, nip, nfp; void (*fn)(RowCtx*); int minp; } FamSpec;

static void row_min(RowCtx* r) { row_minmax(r, 0); }
static void row_max(RowCtx* r) { row_minmax(r, 1); }

static const FamSpec kFam[ORC_FAMILY_COUNT] = {
  [ORC_SMA] = {1, 1, 1, 0, row_sma, 1},      [ORC_EMA] = {1, 1, 1, 0, row_ema, 1},
  [ORC_WMA] = {1, 1, 1, 0, row_wma, 1},      [ORC_RSI] = {1, 1, 1, 0, row_rsi, 1},
  [ORC_MACD] = {1, 3, 3, 0, row_macd, 1},    [ORC_ATR] = {3, 1, 1, 0, row_atr, 1},
  [ORC_NATR] = {3, 1, 1, 0, row_natr, 1},    [ORC_TRANGE] = {3, 1, 0, 0, row_trange, 0},
  [ORC_ADX] = {3, 1, 1, 0, row_adx, 1},      [ORC_DX] = {3, 1, 1, 0, row_dx, 1},
  [ORC_BBANDS] = {1, 3, 1, 2, row_bbands, 2}, [ORC_STOCH] = {3, 2, 2, 0, row_stoch, 1},
  [ORC_CCI] = {3, 1, 1, 0, row_cci, 1},      [ORC_OBV] = {2, 1, 0, 0, row_obv, 0},
  [ORC_AD] = {4, 1, 0, 0, row_ad, 0},        [ORC_ADOSC] = {4, 1, 2, 0, row_adosc, 1},
  [ORC_MFI] = {4, 1, 1, 0, row_mfi, 1},      [ORC_WILLR] = {3, 1, 1, 0, row_willr, 1},
  [ORC_SUM] = {1, 1, 1, 0, row_sum, 1},      [ORC_MIN] = {1, 1, 1, 0, row_min, 1},
  [ORC_MAX] = {1, 1, 1, 0, row_max, 1},      [ORC_STDDEV] = {1, 1, 1, 1, row_stddev, 2},
  [ORC_VAR] = {1, 1, 1, 0, row_var, 1},      [ORC_LINEARREG] = {1, 1, 1, 0, row_linearreg, 2},
  [ORC_CORREL] = {2, 1, 1, 0, row_correl, 1}, [ORC_DEMA] = {1, 1, 1, 0, row_dema, 1},
  [ORC_TEMA] = {1, 1, 1, 0, row_tema, 1},    [ORC_T3] = {1, 1, 1, 1, row_t3, 1},
  [ORC_ROC] = {1, 1, 1, 0, row_roc, 1},      [ORC_RMA] = {1, 1, 1, 0, row_rma, 1},
  [ORC_MEDPRICE] = {2, 1, 0, 0, row_medprice, 0}, [ORC_TYPPRICE] = {3, 1, 0, 0, row_typprice, 0},
  [ORC_MIDPRICE] = {2, 1, 1, 0, row_midprice, 1},
  [ORC_ROCP] = {1, 1, 1, 0, row_rocp, 1},    [ORC_ROCR] = {1, 1, 1, 0, row_rocr, 1},
  [ORC_ROCR100] = {1, 1, 1, 0, row_rocr100, 1}, [ORC_MOM] = {1, 1, 1, 0, row_mom, 1},
  [ORC_AVGPRICE] = {4, 1, 0, 0, row_avgprice, 0}, [ORC_WCLPRICE] = {3, 1, 0, 0, row_wclprice, 0},
  [ORC_MIDPOINT] = {1, 1, 1, 0, row_midpoint, 1},
  [ORC_RMEAN] = {1, 1, 1, 0, row_rmean, 1},  [ORC_RMAX] = {1, 1, 1, 0, row_rmax, 1},
  [ORC_RMIN] = {1, 1, 1, 0, row_rmin, 1},    [ORC_RSTD] = {1, 1, 1, 0, row_rstd, 1},
  [ORC_IBS] = {3, 1, 0, 0, row_ibs, 0},      [ORC_MARKETFI] = {3, 1, 0, 0, row_marketfi, 0},
  [ORC_QSTICK] = {2, 1, 1, 0, row_qstick, 1},
  [ORC_AROON] = {2, 2, 1, 0, row_aroon, 1},  [ORC_AROONOSC] = {2, 1, 1, 0, row_aroonosc, 1},
};

static int check_params(int family, const int* ip) {
  if (family < 0 || family >= ORC_FAMILY_COUNT) return -1;
  const FamSpec* fs = &kFam[family];
  for (int i = 0; i < fs->nip; ++i)
    if (ip[i] < fs->minp && !(family == ORC_MACD && i == 2 && ip[i] >= 1)) return -1;
  return 0;
}

int orc_batch_ragged(int family, const float* const* ins, int S, const long long* off,
                     const int* ip, const double* fp, double* const* outs, int threads) {
  if (check_params(family, ip) != 0) return -1;
  const FamSpec* fs = &kFam[family];
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads)
  for (int s = 0; s < S; ++s) {
    RowCtx r;
    memset(&r, 0, sizeof(r));
    const long long b = off[s];
    r.n = (int)(off[s + 1] - b);
    r.ip = ip; r.fp = fp;
    for (int i = 0; i < fs->nin; ++i) r.in[i] = ins[i] + b;
    for (int i = 0; i < fs->nout; ++i) r.out[i] = outs[i] + b;
    if (r.n > 0) fs->fn(&r);
  }
  return 0;
}

int orc_batch(int family, const float* const* ins, int S, int T, const int* ip,
              const double* fp, double* const* outs, int threads) {
  long long* off = (long long*)malloc(sizeof(long long) * (size_t)(S + 1));
  for (int s = 0; s <= S; ++s) off[s] = (long long)s * T;
  const int rc = orc_batch_ragged(family, ins, S, off, ip, fp, outs, threads);
  free(off);
  return rc;
}
