// Precision variants of the long-window families and the EMA (job precision
// 1 = plain FP32, 2 = compensated FP32, 3 = FP32 bars with FP64 carries).
//
// They follow the FP64 round functions of families.cuh line for line (same
// lane-local origins, warm-up and NaN rules, TA-Lib operation order). The
// windows compute their per-bar terms (deviations, squares, products) in T
// and keep their running sums - the quantities carried from bar to bar - in
// A: float/float (plain), F2/F2 (compensated; products exact through the
// two-product), float/double (FP32 terms, FP64 carries). The EMA keeps its
// per-bar state in S and the carries between lanes and tiles in C. They exist
// to measure what each precision costs in error on long, level-offset rows;
// the FP64 path remains the default.
#pragma once

#include "families.cuh"
#include "reals.cuh"

namespace tb {

// Conversion between the arithmetic types (exact from float, and between F2
// and double up to F2's 48 bits).
template <class A, class T>
__device__ __forceinline__ A conv(T v) { return Real<A>::of(Real<T>::to_d(v)); }
template <>
__device__ __forceinline__ float conv<float, float>(float v) { return v; }
template <>
__device__ __forceinline__ F2 conv<F2, F2>(F2 v) { return v; }

// SMA / SUM / WMA (sum_window_round): terms in T, sums in S.
template <int K, class T, class S>
__device__ __forceinline__ void sum_window_p(const Ctx<K>& c, const Job& j, int mode) {
  using R = Real<S>;
  using RT = Real<T>;
  const int pl = j.in[0], p = j.ip[0];
  const int g0 = c.gb0();
  const int tf = g0 > p - 1 ? g0 : (int)(p - 1);
  S s = R::of(0.0), w = R::of(0.0);
  int nn = 0;
  if (tf < g0 + K && c.valid(tf)) {
    for (int i = 0; i < p; ++i) {
      const float v = c.x(pl, tf - p + 1 + i);
      if (isnan(v)) ++nn;
      else { s += R::of(v); w += conv<S>(RT::of(v) * RT::of(i + 1)); }
    }
  }
  const T tp = RT::of(p);
  const S divider = R::of((double)p * (p + 1) / 2.0), sp = R::of(p);
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= tf) {
      if (t > tf) {
        const float vin = c.x(pl, t), vout = c.x(pl, t - p);
        if (mode == 2) w -= s;
        if (isnan(vout)) --nn; else s -= R::of(vout);
        if (isnan(vin)) ++nn;
        else { s += R::of(vin); if (mode == 2) w += conv<S>(RT::of(vin) * tp); }
      }
      if (nn == 0) {
        if (mode == 0) o = (float)R::to_d(s / sp);
        else if (mode == 1) o = (float)R::to_d(s);
        else o = p == 1 ? c.x(pl, t) : (float)R::to_d(w / divider);
      }
    }
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// BBANDS / STDDEV / VAR (moment_window_round): terms in T, sums in S.
template <int K, class T, class S>
__device__ __forceinline__ void moment_window_p(const Ctx<K>& c, const Job& j, int mode) {
  using R = Real<S>;
  using RT = Real<T>;
  const int pl = j.in[0], p = j.ip[0];
  const int g0 = c.gb0();
  const int tf = g0 > p - 1 ? g0 : (int)(p - 1);
  S raw = R::of(0.0), s2 = R::of(0.0), o = R::of(0.0);
  T ot = RT::of(0.0);
  int nn = 0;
  if (tf < g0 + K && c.valid(tf)) {
    const float ov = c.x(pl, tf);
    o = R::of(isnan(ov) ? 0.0 : (double)ov);
    ot = RT::of(isnan(ov) ? 0.0 : (double)ov);
    for (int i = 0; i < p; ++i) {
      const float v = c.x(pl, tf - p + 1 + i);
      if (isnan(v)) ++nn;
      else { raw += R::of(v); const T d = RT::of(v) - ot; s2 += conv<S>(d * d); }
    }
  }
  const S inv = R::of(1.0 / (double)p), po = R::of(p) * o, sp = R::of(p);
  const S up = R::of(j.fp[0]), dn = R::of(j.fp[1]);
  const S zero = R::of(0.0);
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o0 = qnan(), o1 = qnan(), o2 = qnan();
    if (t >= tf) {
      if (t > tf) {
        const float vin = c.x(pl, t), vout = c.x(pl, t - p);
        if (isnan(vout)) --nn;
        else { raw -= R::of(vout); const T d = RT::of(vout) - ot; s2 -= conv<S>(d * d); }
        if (isnan(vin)) ++nn;
        else { raw += R::of(vin); const T d = RT::of(vin) - ot; s2 += conv<S>(d * d); }
      }
      if (nn == 0) {
        const S m1 = (raw - po) * inv;
        S var = s2 * inv - m1 * m1;
        if (!(var > zero)) var = zero;
        if (mode == 2) o0 = (float)R::to_d(var);
        else {
          const S sd = var != zero ? R::sqrt_r(var) : zero;
          if (mode == 1) o0 = (float)R::to_d(sd * up);
          else {
            const S mid = raw / sp;
            o0 = (float)R::to_d(R::fma_r(sd, up, mid));
            o2 = (float)R::to_d(mid - sd * dn);
            o1 = (float)R::to_d(mid);
          }
        }
      }
    }
    c.put(0, k, o0);
    if (mode == 0) { c.put(1, k, o1); c.put(2, k, o2); }
  }
  c.flush(0, (float*)j.out[0]);
  if (mode == 0) { c.flush(1, (float*)j.out[1]); c.flush(2, (float*)j.out[2]); }
}

// LINEARREG (linreg_round): terms in T, sums in S.
template <int K, class T, class S>
__device__ __forceinline__ void linreg_p(const Ctx<K>& c, const Job& j) {
  using R = Real<S>;
  using RT = Real<T>;
  const int pl = j.in[0], p = j.ip[0];
  const int g0 = c.gb0();
  const int tf = g0 > p - 1 ? g0 : (int)(p - 1);
  const double sumXd = (double)p * (p - 1) * 0.5;
  const double sumXSqr = (double)p * (p - 1) * (2 * p - 1) / 6.0;
  const S sumX = R::of(sumXd), divisor = R::of(sumXd * sumXd - p * sumXSqr), sp = R::of(p);
  const S pm1 = R::of(p - 1);
  S sy = R::of(0.0), sxy = R::of(0.0), o = R::of(0.0);
  T ot = RT::of(0.0);
  int nn = 0;
  if (tf < g0 + K && c.valid(tf)) {
    const float ov = c.x(pl, tf);
    o = R::of(isnan(ov) ? 0.0 : (double)ov);
    ot = RT::of(isnan(ov) ? 0.0 : (double)ov);
    for (int i = p - 1; i >= 0; --i) {
      const float v = c.x(pl, tf - i);
      if (isnan(v)) ++nn;
      else { const T d = RT::of(v) - ot; sy += conv<S>(d); sxy += conv<S>(RT::of(i) * d); }
    }
  }
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float out = qnan();
    if (t >= tf) {
      if (t > tf) {
        const float vout = c.x(pl, t - p), vin = c.x(pl, t);
        const S dout = conv<S>(isnan(vout) ? RT::of(0.0) : RT::of(vout) - ot);
        const S din = conv<S>(isnan(vin) ? RT::of(0.0) : RT::of(vin) - ot);
        sxy = sxy + sy - sp * dout;
        sy = sy - dout + din;
        nn += (isnan(vin) ? 1 : 0) - (isnan(vout) ? 1 : 0);
      }
      if (nn == 0) {
        const S m = (sp * sxy - sumX * sy) / divisor;
        const S b = (sy - m * sumX) / sp;
        out = (float)R::to_d(o + R::fma_r(m, pm1, b));
      }
    }
    c.put(0, k, out);
  }
  c.flush(0, (float*)j.out[0]);
}

// CORREL (correl_round): terms in T, sums in S.
template <int K, class T, class S>
__device__ __forceinline__ void correl_p(const Ctx<K>& c, const Job& j, Carry& cy) {
  using R = Real<S>;
  using RT = Real<T>;
  const int px = j.in[0], py = j.in[1], p = j.ip[0];
  const int g0 = c.gb0();
  int bad = cy.f;
  if (bad < 0) {
    int first = 0x7fffffff;
    for (int k = 0; k < K; ++k) {
      const int t = g0 + k;
      if (!c.valid(t)) break;
      if (!isfinite(c.x(px, t)) || !isfinite(c.x(py, t))) { first = t; break; }
    }
    first = warp_min_int(first);
    bad = first == 0x7fffffff ? -1 : first;
    if (c.lb) bad = lb_first_index(c.lbd + j.lb_slot, c.lbs, c.tile, bad, c.err, c.lane);
  }
  const int tf = g0 > p - 1 ? g0 : (int)(p - 1);
  S sx = R::of(0.0), sy = R::of(0.0), sxx = R::of(0.0), syy = R::of(0.0), sxy = R::of(0.0);
  T ox = RT::of(0.0), oy = RT::of(0.0);
  if (tf < g0 + K && c.valid(tf)) {
    const float fx = c.x(px, tf - p + 1), fy = c.x(py, tf - p + 1);
    ox = RT::of(isfinite(fx) ? (double)fx : 0.0);
    oy = RT::of(isfinite(fy) ? (double)fy : 0.0);
    for (int i = 0; i < p; ++i) {
      const T dx = RT::of(c.x(px, tf - p + 1 + i)) - ox, dy = RT::of(c.x(py, tf - p + 1 + i)) - oy;
      sx += conv<S>(dx); sy += conv<S>(dy);
      sxx += conv<S>(dx * dx); syy += conv<S>(dy * dy); sxy += conv<S>(dx * dy);
    }
  }
  const S pp = R::of(p), zero = R::of(0.0);
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= tf) {
      if (t > tf) {
        const T ax = RT::of(c.x(px, t - p)) - ox, ay = RT::of(c.x(py, t - p)) - oy;
        const T bx = RT::of(c.x(px, t)) - ox, by = RT::of(c.x(py, t)) - oy;
        sx += conv<S>(bx) - conv<S>(ax); sy += conv<S>(by) - conv<S>(ay);
        sxx += conv<S>(bx * bx) - conv<S>(ax * ax); syy += conv<S>(by * by) - conv<S>(ay * ay);
        sxy += conv<S>(bx * by) - conv<S>(ax * ay);
      }
      if (bad >= 0 && t >= bad) o = 0.0f;
      else {
        const S cov = sxy - sx * sy / pp;
        const S vx = sxx - sx * sx / pp, vy = syy - sy * sy / pp;
        const S prod = vx * vy;
        o = (vx > zero && vy > zero && prod > R::of(1e-14)) ? (float)R::to_d(cov / R::sqrt_r(prod)) : 0.0f;
      }
    }
    c.put(0, k, o);
  }
  cy.f = bad;
  c.flush(0, (float*)j.out[0]);
}

// EMA (ema_round / stage_round) with the per-bar state in S and the carries
// (lane composition, warp scan, look-back aggregates) in C.
template <int K, class S, class C>
__device__ __forceinline__ void ema_p(const Ctx<K>& c, const Job& j, Carry& cy) {
  using RS = Real<S>;
  using RC = Real<C>;
  const int pl = j.in[0], p = j.ip[0];
  const int f = resolve_start(c, cy, pl, j.lb_slot);
  const int g0 = c.gb0();
  const S beta = RS::of(j.fp[0]), kk = RS::of(j.fp[1]), sp = RS::of(p);
  const C betaC = RC::of(j.fp[0]), kC = RC::of(j.fp[1]), invC = RC::of(1.0 / p), one = RC::of(1.0);
  float xin[K];
#pragma unroll
  for (int k = 0; k < K; ++k) xin[k] = (f >= 0 && c.valid(g0 + k) && g0 + k >= f) ? c.x(pl, g0 + k) : 0.0f;
  // origin: first counted input of the round
  float o = 0.0f;
  if (f >= 0) {
    const int to = c.t0 > f ? c.t0 : f;
    if (to < c.t0 + c.L) {
      o = c.x(pl, to);
      if (!isfinite(o)) o = 0.0f;
    }
  }
  const C oC = RC::of(o);
  auto coef = [&](int r, C& a, C& w) {
    if (p == 1) { a = RC::of(0.0); w = one; }
    else if (r < p - 1) { a = one; w = one; }
    else if (r == p - 1) { a = invC; w = invC; }
    else { a = betaC; w = kC; }
  };
  auto expect = [&](int r) { return (p > 1 && r < p - 1) ? (double)(r + 1) : 1.0; };
  C A = one, B = RC::of(0.0);
  if (f >= 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int t = g0 + k;
      if (c.valid(t) && t >= f) {
        C a, w;
        coef(t - f, a, w);
        B = RC::fma_r(a, B, w * (RC::of(xin[k]) - oC));
        A = A * a;
      }
    }
  }
  // inclusive warp scan of the lane maps, then the exclusive prefix
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const C pA = shfl_up_r(A, d), pB = shfl_up_r(B, d);
    if (c.lane >= d) { B = RC::fma_r(A, pB, B); A = A * pA; }
  }
  C Ae = shfl_up_r(A, 1), Be = shfl_up_r(B, 1);
  if (c.lane == 0) { Ae = one; Be = RC::of(0.0); }
  double carry = cy.v[0];
  if (c.lb) {
    const double tA[1] = {RC::to_d(shfl_r(A, 31))};
    const double tB[1] = {RC::to_d(shfl_r(B, 31)) + (double)o * (1.0 - tA[0])};
    const double init[1] = {carry};
    double Y[1];
    lb_resolve<1>(c.lbd + j.lb_slot + 1, c.lbs, c.tile, tA, tB, init, lb_first_steady(f, p == 1 ? 0 : p, Ctx<K>::TILE),
                  Y, c.err, c.lane);
    carry = Y[0];
  }
  S y = RS::of(carry);
  if (f >= 0) {
    const int cr = c.t0 - 1 - f, cl = g0 - 1 - f;
    const C er = RC::of(cr >= 0 ? expect(cr) * (double)o : 0.0);
    const C el = RC::of(cl >= 0 ? expect(cl) * (double)o : 0.0);
    y = RS::of(RC::to_d(el + RC::fma_r(Ae, RC::of(carry) - er, Be)));
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) continue;
    float out = qnan();
    if (f >= 0 && t >= f) {
      const int r = t - f;
      const S x = RS::of(xin[k]);
      if (p == 1) y = x;
      else if (r < p - 1) y = y + x;
      else if (r == p - 1) y = (y + x) / sp;
      else y = RS::fma_r(beta, y, kk * x);
      if (r >= p - 1) out = (float)RS::to_d(y);
    }
    c.put(0, k, out);
  }
  const S tail = shfl_r(y, (c.L - 1) / K);
  cy.v[0] = RS::to_d(tail);
  if (c.lb) {
    const double Y[1] = {cy.v[0]};
    lb_publish<1>(c.lbd + j.lb_slot + 1, c.lbs, c.tile, Y, c.lane);
  }
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
}

}  // namespace tb
