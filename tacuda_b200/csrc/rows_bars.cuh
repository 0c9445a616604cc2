// Bar-parallel window jobs of the row engine. A window output depends only on
// the bars inside its window, so these jobs take the 32 bars of a chunk across
// the lanes and walk the rows of the group one at a time: every output is
// computed directly from the staged ring (its halo holds the bars before the
// chunk), lanes read consecutive shared-memory words, and each row's 32
// outputs leave as one coalesced store with no transpose stage. Having no
// state that runs along a row, a job can be split over a team of warps by
// rows (member k takes rows k, k+m, ...), which shortens the longest warp of
// the CTA; and with no running sums there is no NaN / infinity bookkeeping and
// no second code path. The price is more instructions per output than a
// running window, so the launcher sends only CCI here always (it sums its
// windows directly in any form) and WILLR / STOCH when few jobs share the CTA
// (their extremes, hence their bits, are the same in both forms).
//
// Per-warp lines hold values several windows share (typical prices, fastK /
// slowK) for the bars [t0 - 64, t0 + 32) of the current row, at index
// bar - (t0 - 64).
#pragma once

#include "rows.cuh"

namespace tb {
namespace rows {

constexpr int kBarLine = 96;  // entries of one per-warp line

// out[base + t] for the lanes whose bar exists
__device__ __forceinline__ void put_bar(float* out, long long base, long long n, int t, float v) {
  if (t < n) out[base + t] = v;
}

// WILLR (src/indicators/WILLR.cu:11-30): extremes anchored at the current bar,
// so a NaN high or low there gives NaN while earlier NaNs are skipped by the
// strict comparisons; float32 ratio times -100 clamped to [-100, 0], 0 for a
// zero range.
__device__ void b_willr(const Warp& w, const Job& j) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0];
  float* out = (float*)j.out[0];
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const int t0 = c * C, t = t0 + w.lane;
    for (int r = w.tk; r < 32; r += w.tm) {
      long long base;
      const long long n = w.row_len(r, base);
      if (t0 >= n) continue;
      const float* H = w.Xrow(c, ph, r) + w.lane;
      const float* Lo = w.Xrow(c, plo, r) + w.lane;
      float hi = H[0], lo = Lo[0];
#pragma unroll 4
      for (int i = 1; i < p; ++i) {
        const float a = H[-i], b = Lo[-i];
        hi = a > hi ? a : hi;
        lo = b < lo ? b : lo;
      }
      const float den = hi - lo;
      const float v = den == 0.0f ? 0.0f : fdiv(hi - w.Xrow(c, pc, r)[w.lane], den) * -100.0f;
      const float o = isnan(v) ? qnan() : fminf(0.0f, fmaxf(-100.0f, v));
      put_bar(out, base, n, t, t >= p - 1 ? o : qnan());
    }
    w.release(c);
  }
}

// STOCH (talib08:16115-16302, SMA slowing): fastK from the window extremes
// anchored at the window's first bar (a NaN there gives NaN, later NaNs are
// skipped), TA-Lib's zero-range test; slowK and slowD are means of the last q
// fastK / slowK values summed oldest first, all in float32.
__device__ void b_stoch(const Warp& w, const Job& j, float* line) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0], q = j.ip[1];
  const int lb = p - 1 + 2 * (q - 1);
  const float invq = 1.0f / (float)q;
  float* fk = line;             // fastK of bar t0 - 64 + i at [i]
  float* sk = line + kBarLine;  // slowK
  float* out0 = (float*)j.out[0];
  float* out1 = (float*)j.out[1];
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const int t0 = c * C, t = t0 + w.lane;
    for (int r = w.tk; r < 32; r += w.tm) {
      long long base;
      const long long n = w.row_len(r, base);
      if (t0 >= n) continue;
      const float* H = w.Xrow(c, ph, r) + w.lane;
      const float* Lo = w.Xrow(c, plo, r) + w.lane;
      const float* Cl = w.Xrow(c, pc, r) + w.lane;
      // fastK of the bars t - 64, t - 32, t that a slowD of this chunk reads
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int off = (k - 2) * C;
        if (w.lane + off < -2 * (q - 1)) continue;
        float hi = H[off - p + 1], lo = Lo[off - p + 1];
        for (int i = p - 2; i >= 0; --i) {
          const float a = H[off - i], b = Lo[off - i];
          hi = a > hi ? a : hi;
          lo = b < lo ? b : lo;
        }
        const float range = hi - lo;
        fk[w.lane + off + 64] =
            fabsf(range) <= 1e-14f * (fabsf(hi) + fabsf(lo)) ? 0.0f : fdiv(Cl[off] - lo, range) * 100.0f;
      }
      __syncwarp();
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int off = (k - 2) * C, i = w.lane + off + 64;
        if (w.lane + off < -(q - 1)) continue;
        float s = fk[i - q + 1];
        for (int m = q - 2; m >= 0; --m) s += fk[i - m];
        sk[i] = s * invq;
      }
      __syncwarp();
      const int i = w.lane + 64;
      float d = sk[i - q + 1];
      for (int m = q - 2; m >= 0; --m) d += sk[i - m];
      const bool ok = t >= lb;
      put_bar(out0, base, n, t, ok ? sk[i] : qnan());
      put_bar(out1, base, n, t, ok ? d * invq : qnan());
      __syncwarp();
    }
    w.release(c);
  }
}

// CCI (src/indicators/CCI.cu:11-40), in the reference's arithmetic: typical
// price (((double)h + l) + c) / 3.0, the window sum taken directly from the
// newest bar back, sma = sum / p, the mean absolute deviation summed in the
// same order, md = dev / p (each divide correctly rounded, as div_by gives
// them); then (tp - sma) / (0.015 md) when both are nonzero, taken in float
// (within 3 float ulp of the reference's FP64 quotient rounded to float).
// Direct sums keep a constant window's deviation exactly zero, and a
// non-finite price makes every window holding it NaN.
__device__ void b_cci(const Warp& w, const Job& j, double* line) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0];
  const double dp = (double)p, ip = 1.0 / dp, third = 1.0 / 3.0;
  float* out = (float*)j.out[0];
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const int t0 = c * C, t = t0 + w.lane;
    for (int r = w.tk; r < 32; r += w.tm) {
      long long base;
      const long long n = w.row_len(r, base);
      if (t0 >= n) continue;
      const float* H = w.Xrow(c, ph, r) + w.lane;
      const float* Lo = w.Xrow(c, plo, r) + w.lane;
      const float* Cl = w.Xrow(c, pc, r) + w.lane;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int off = (k - 2) * C;
        if (w.lane + off < -(p - 1)) continue;
        line[w.lane + off + 64] = div_by(((double)H[off] + (double)Lo[off]) + (double)Cl[off], 3.0, third);
      }
      __syncwarp();
      const double* cur = line + w.lane + 64;
      double s = 0.0;
#pragma unroll 4
      for (int i = 0; i < p; ++i) s += cur[-i];
      const double sma = div_by(s, dp, ip);
      double dev = 0.0;
#pragma unroll 4
      for (int i = 0; i < p; ++i) dev += fabs(cur[-i] - sma);
      const double md = div_by(dev, dp, ip);
      const double num = cur[0] - sma;
      const float o = (num != 0.0 && md != 0.0) ? fdiv((float)num, (float)(0.015 * md)) : 0.0f;
      put_bar(out, base, n, t, t >= p - 1 ? o : qnan());
      __syncwarp();
    }
    w.release(c);
  }
}

}  // namespace rows
}  // namespace tb
