// Series-parallel family kernels: one thread walks one series bar by bar in
// TA-Lib's own order (citations as in families.cuh); the state lives in
// registers across chunks. Window families re-derive their sums from the staged
// halo at the start of every chunk (direct FP64 sums, exact for float32 inputs)
// and slide within it, so rounding never drifts along a long series and a NaN
// only poisons the windows containing it.
#pragma once

#include "sp_engine.cuh"

namespace tb {
namespace sp {

// Per-warp driver of the chunk loop: stages chunk c (and prefetches c+1) at
// begin(c) and releases the buffer at end(c). Every warp of the CTA makes the
// same calls, so the CTA barriers inside match.
struct Driver {
  const Launch* L;
  const Layout* lay;
  unsigned char* smem;
  const long long* rows_base;  // [G*32] (-1: no series)
  const long long* rows_n;     // [G*32]
  int nchunks;
  int group;                   // this warp's group
  int lane;
  long long my_base, my_n;

  __device__ __forceinline__ float* buf(int parity) const {
    return reinterpret_cast<float*>(smem + (size_t)parity * lay->in_bytes);
  }

  __device__ void issue(int c) const {
    if (c >= nchunks) return;
    const int span = lay->H + C;
    const long long t0 = (long long)c * C;
    float* dst0 = buf(c & 1);
    const int nw = blockDim.x >> 5, w = threadIdx.x >> 5, ln = threadIdx.x & 31;
    const int tasks = lay->G * lay->nplanes * 32;  // one staged row per task
    for (int task = w; task < tasks; task += nw) {
      const int row = task & 31;
      const int gs = task >> 5;  // g * nplanes + slot
      const int slot = gs % lay->nplanes;
      const int g = gs / lay->nplanes;
      const int plane = lay->slot_plane[slot];
      const long long rb = rows_base[g * 32 + row];
      const long long n = rows_n[g * 32 + row];
      const float* src = L->plane[plane] + (rb >= 0 ? rb : 0);
      float* dst = dst0 + (size_t)task * lay->RS;
      const long long tlo = t0 - lay->H;
      for (int i = ln; i < span; i += 32) {
        const long long t = tlo + i;
        const bool ok = rb >= 0 && t >= 0 && t < n;
        cp_async4(dst + i, ok ? src + t : src, ok);
      }
    }
  }

  __device__ __forceinline__ void begin(int c) const {
    if (c == 0) { issue(0); cp_commit(); }
    issue(c + 1);
    cp_commit();
    cp_wait1();
    __syncthreads();
  }
  __device__ __forceinline__ void end(int) const { __syncthreads(); }

  __device__ __forceinline__ Row row(int c) const {
    Row rw;
    rw.t0 = (long long)c * C;
    rw.n = my_n;
    return rw;
  }
  // staged bars of this thread's row for `plane`; index r = t - t0 in [-H, C)
  __device__ __forceinline__ const float* pptr(int c, int plane) const {
    const int slot = lay->plane_slot[plane];
    return reinterpret_cast<const float*>(smem + (size_t)(c & 1) * lay->in_bytes) +
           ((size_t)(group * lay->nplanes + slot) * 32 + lane) * lay->RS + lay->H;
  }
};

// per-warp FP64 scratch line of the thread's row: [32][RS] doubles, entry for
// round-relative bar r at index r + H
struct Line {
  double* p;
  int RS, H;
  __device__ __forceinline__ double& at(int lane, int r) const { return p[(size_t)lane * RS + r + H]; }
};

#define SP_ARGS Driver& drv, const Job& j, const Stage& st, const Line& ln, int lane
#define SP_FLUSH(k) st.flush(k, (float*)j.out[k], drv.my_base, drv.my_n, rw.t0, lane)

// ---------------------------------------------------------------- windows

// SMA / SUM / WMA (mode 0/1/2)
__device__ void sp_sum_window(SP_ARGS, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  const double divider = (double)p * (p + 1) / 2.0;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    double s = 0.0, w = 0.0;
    int nn = 0;
    bool seeded = false;
    for_chunk(rw, [&](int r, long long t) {
      float o = qnan();
      if (t >= p - 1) {
        if (!seeded) {
          seeded = true;
          for (int i = 0; i < p; ++i) {
            const float v = X_pl[r - p + 1 + i];
            if (isnan(v)) ++nn;
            else { s += (double)v; w += (double)v * (double)(i + 1); }
          }
        } else {
          const float vin = X_pl[r], vout = X_pl[r - p];
          if (mode == 2) w -= s;
          if (isnan(vout)) --nn; else s -= (double)vout;
          if (isnan(vin)) ++nn;
          else { s += (double)vin; if (mode == 2) w += (double)vin * (double)p; }
        }
        if (nn == 0) {
          if (mode == 0) o = (float)(s / (double)p);
          else if (mode == 1) o = (float)s;
          else o = p == 1 ? X_pl[r] : (float)(w / divider);
        }
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// BBANDS / STDDEV / VAR (mode 0/1/2): moments of x - o about the window start
__device__ void sp_moment_window(SP_ARGS, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  const double inv = 1.0 / (double)p, up = j.fp[0], dn = j.fp[1];
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    double raw = 0.0, s2 = 0.0, o = 0.0;
    int nn = 0;
    bool seeded = false;
    for_chunk(rw, [&](int r, long long t) {
      float o0 = qnan(), o1 = qnan(), o2 = qnan();
      if (t >= p - 1) {
        if (!seeded) {
          seeded = true;
          const float ov = X_pl[r];
          o = isnan(ov) ? 0.0 : (double)ov;
          for (int i = 0; i < p; ++i) {
            const float v = X_pl[r - p + 1 + i];
            if (isnan(v)) ++nn;
            else { raw += (double)v; const double d = (double)v - o; s2 += d * d; }
          }
        } else {
          const float vin = X_pl[r], vout = X_pl[r - p];
          if (isnan(vout)) --nn;
          else { raw -= (double)vout; const double d = (double)vout - o; s2 -= d * d; }
          if (isnan(vin)) ++nn;
          else { raw += (double)vin; const double d = (double)vin - o; s2 += d * d; }
        }
        if (nn == 0) {
          const double m1 = (raw - (double)p * o) * inv;
          double var = s2 * inv - m1 * m1;
          if (!(var > 0.0)) var = 0.0;
          if (mode == 2) o0 = (float)var;
          else {
            const double sd = var != 0.0 ? sqrt(var) : 0.0;
            if (mode == 1) o0 = (float)(up != 1.0 ? sd * up : sd);
            else {
              const double mid = raw / (double)p;
              if (up == dn) { const double dv = sd * up; o0 = (float)(mid + dv); o2 = (float)(mid - dv); }
              else { o0 = (float)fma(sd, up, mid); o2 = (float)(mid - sd * dn); }
              o1 = (float)mid;
            }
          }
        }
      }
      st.put(0, lane, r, o0);
      if (mode == 0) { st.put(1, lane, r, o1); st.put(2, lane, r, o2); }
    });
    SP_FLUSH(0);
    if (mode == 0) { SP_FLUSH(1); SP_FLUSH(2); }
    drv.end(c);
  }
}

// LINEARREG: TA-Lib's sliding SumY / SumXY about a window-start origin
__device__ void sp_linreg(SP_ARGS) {
  const int pl = j.in[0], p = j.ip[0];
  const double sumX = (double)p * (p - 1) * 0.5;
  const double sumXSqr = (double)p * (p - 1) * (2 * p - 1) / 6.0;
  const double divisor = sumX * sumX - p * sumXSqr;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    double sy = 0.0, sxy = 0.0, o = 0.0;
    int nn = 0;
    bool seeded = false;
    for_chunk(rw, [&](int r, long long t) {
      float out = qnan();
      if (t >= p - 1) {
        if (!seeded) {
          seeded = true;
          const float ov = X_pl[r];
          o = isnan(ov) ? 0.0 : (double)ov;
          for (int i = p - 1; i >= 0; --i) {
            const float v = X_pl[r - i];
            if (isnan(v)) ++nn;
            else { const double d = (double)v - o; sy += d; sxy += (double)i * d; }
          }
        } else {
          const float vout = X_pl[r - p], vin = X_pl[r];
          const double dout = isnan(vout) ? 0.0 : (double)vout - o;
          const double din = isnan(vin) ? 0.0 : (double)vin - o;
          sxy = sxy + sy - (double)p * dout;
          sy = sy - dout + din;
          nn += (isnan(vin) ? 1 : 0) - (isnan(vout) ? 1 : 0);
        }
        if (nn == 0) {
          const double m = (p * sxy - sumX * sy) / divisor;
          const double b = (sy - m * sumX) / (double)p;
          out = (float)(o + fma(m, (double)(p - 1), b));
        }
      }
      st.put(0, lane, r, out);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// CORREL (Correl.cu:23-75): window moments about the window start; 0 from the
// row's first non-finite bar on.
__device__ void sp_correl(SP_ARGS) {
  const int px = j.in[0], py = j.in[1], p = j.ip[0];
  long long bad = -1;
  const double pp = (double)p;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_px = drv.pptr(c, px);
    const float* X_py = drv.pptr(c, py);
    double sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0, ox = 0, oy = 0;
    bool seeded = false;
    for_chunk(rw, [&](int r, long long t) {
      if (bad < 0 && (!isfinite(X_px[r]) || !isfinite(X_py[r]))) bad = t;
      float o = qnan();
      if (t >= p - 1) {
        if (!seeded) {
          seeded = true;
          ox = X_px[r - p + 1];
          oy = X_py[r - p + 1];
          if (!isfinite(ox)) ox = 0.0;
          if (!isfinite(oy)) oy = 0.0;
          for (int i = 0; i < p; ++i) {
            const double dx = (double)X_px[r - p + 1 + i] - ox, dy = (double)X_py[r - p + 1 + i] - oy;
            sx += dx; sy += dy; sxx += dx * dx; syy += dy * dy; sxy += dx * dy;
          }
        } else {
          const double ax = (double)X_px[r - p] - ox, ay = (double)X_py[r - p] - oy;
          const double bx = (double)X_px[r] - ox, by = (double)X_py[r] - oy;
          sx += bx - ax; sy += by - ay;
          sxx += bx * bx - ax * ax; syy += by * by - ay * ay; sxy += bx * by - ax * ay;
        }
        if (bad >= 0 && t >= bad) o = 0.0f;
        else {
          const double cov = sxy - sx * sy / pp;
          const double vx = sxx - sx * sx / pp, vy = syy - sy * sy / pp;
          const double prod = vx * vy;
          o = (vx > 0.0 && vy > 0.0 && prod > 1e-14) ? (float)(cov / sqrt(prod)) : 0.0f;
        }
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// MIN / MAX with the leading-NaN window rule
// MIN / MAX; mid: MIDPOINT = 0.5f * (max + min) (src/indicators/MIDPOINT.cu:24-34)
__device__ void sp_minmax(SP_ARGS, bool is_max, bool mid = false) {
  const int pl = j.in[0], p = j.ip[0];
  long long f = -1;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    for_chunk(rw, [&](int r, long long t) {
      if (f < 0 && !isnan(X_pl[r])) f = t;
      float o = qnan();
      if (t >= p - 1 && f >= 0 && t - p + 1 >= f) {
        if (mid) {
          float hi = X_pl[r - p + 1], lo = hi;
          for (int i = 1; i < p; ++i) {
            hi = fmaxf(hi, X_pl[r - p + 1 + i]);
            lo = fminf(lo, X_pl[r - p + 1 + i]);
          }
          o = 0.5f * (hi + lo);
        } else {
          o = X_pl[r - p + 1];
          for (int i = 1; i < p; ++i) o = is_max ? fmaxf(o, X_pl[r - p + 1 + i]) : fminf(o, X_pl[r - p + 1 + i]);
        }
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// WILLR (WILLR.cu:11-30)
__device__ void sp_willr(SP_ARGS) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0];
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pc = drv.pptr(c, pc);
    const float* X_ph = drv.pptr(c, ph);
    const float* X_plo = drv.pptr(c, plo);
    for_chunk(rw, [&](int r, long long t) {
      float o = qnan();
      if (t >= p - 1) {
        float hi = X_ph[r], lo = X_plo[r];
        float hi2 = p > 1 ? X_ph[r - 1] : hi, lo2 = p > 1 ? X_plo[r - 1] : lo;
        int i = 2;
        for (; i + 1 < p; i += 2) {
          const float h = X_ph[r - i], l = X_plo[r - i], h2 = X_ph[r - i - 1], l2 = X_plo[r - i - 1];
          if (h > hi) hi = h;
          if (l < lo) lo = l;
          if (h2 > hi2) hi2 = h2;
          if (l2 < lo2) lo2 = l2;
        }
        for (; i < p; ++i) {
          const float h = X_ph[r - i], l = X_plo[r - i];
          if (h > hi) hi = h;
          if (l < lo) lo = l;
        }
        if (hi2 > hi) hi = hi2;
        if (lo2 < lo) lo = lo2;
        const double den = (double)hi - (double)lo;
        const double v = den == 0.0 ? 0.0 : (((double)hi - (double)X_pc[r]) / den) * -100.0;
        o = isnan(v) ? qnan() : (float)fmin(0.0, fmax(-100.0, v));
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// ROC / ROCP / ROCR / ROCR100 / MOM (roc_value in families.cuh)
__device__ void sp_roc(SP_ARGS, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    for_chunk(rw, [&](int r, long long t) {
      float o = qnan();
      if (t >= p) o = roc_value(X_pl[r], X_pl[r - p], mode);
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// MEDPRICE / TYPPRICE / AVGPRICE / WCLPRICE (price_round modes in families.cuh)
__device__ void sp_price(SP_ARGS, int mode) {
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* A = drv.pptr(c, j.in[0]);
    const float* B = drv.pptr(c, j.in[1]);
    const float* C2 = mode >= 1 ? drv.pptr(c, j.in[2]) : A;
    const float* D = mode == 2 ? drv.pptr(c, j.in[3]) : A;
    for_chunk(rw, [&](int r, long long) {
      const float a = A[r], b = B[r];
      float o;
      if (mode == 0) o = 0.5f * (a + b);
      else if (mode == 1) o = (a + b + C2[r]) / 3.0f;
      else if (mode == 2) o = (a + b + C2[r] + D[r]) * 0.25f;
      else o = (a + b + 2.0f * C2[r]) * 0.25f;
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// MIDPRICE (src/indicators/MIDPRICE.cu:11-24): fmaxf / fminf window extrema
__device__ void sp_midprice(SP_ARGS) {
  const int ph = j.in[0], plo = j.in[1], p = j.ip[0];
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_ph = drv.pptr(c, ph);
    const float* X_plo = drv.pptr(c, plo);
    for_chunk(rw, [&](int r, long long t) {
      float o = qnan();
      if (t >= p - 1) {
        float hi = X_ph[r - p + 1], lo = X_plo[r - p + 1];
        for (int i = 1; i < p; ++i) {
          hi = fmaxf(hi, X_ph[r - p + 1 + i]);
          lo = fminf(lo, X_plo[r - p + 1 + i]);
        }
        o = 0.5f * (hi + lo);
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// NaN-strict rolling mean / max / min / std (rolling_round in families.cuh)
__device__ void sp_rolling(SP_ARGS, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    for_chunk(rw, [&](int r, long long t) {
      float o = qnan();
      if (t >= p - 1) {
        bool ok = true;
        double sum = 0.0, sq = 0.0;
        float mx = X_pl[r], mn = mx;
        for (int i = 0; i < p; ++i) {
          const float v = X_pl[r - i];
          if (!isfinite(v)) { ok = false; break; }
          sum += v;
          sq = fma((double)v, (double)v, sq);
          mx = fmaxf(mx, v);
          mn = fminf(mn, v);
        }
        if (ok) {
          if (mode == 0) o = (float)(sum / p);
          else if (mode == 1) o = mx;
          else if (mode == 2) o = mn;
          else {
            const double mean = sum / p;
            o = (float)sqrt(fmax(0.0, fma(-mean, mean, sq / p)));
          }
        }
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// IBS / MARKETFI (talib_bar_round in families.cuh)
__device__ void sp_talib_bar(SP_ARGS, int mode) {
  const int p0 = j.in[0], p1 = j.in[1], p2 = j.in[2];
  long long f = -1;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* A = drv.pptr(c, p0);
    const float* B = drv.pptr(c, p1);
    const float* Z = drv.pptr(c, p2);
    for_chunk(rw, [&](int r, long long t) {
      if (f < 0 && !isnan(A[r]) && !isnan(B[r]) && !isnan(Z[r])) f = t;
      float o = qnan();
      if (f >= 0 || t == rw.n - 1) {
        const double a = A[r], b = B[r], z = Z[r];
        double v;
        if (mode == 0) {
          const double range = a - b;
          v = (z - b) / range;
          if (range <= 0.0) v = 0.5;
        } else {
          v = z != 0.0 ? (a - b) / z : 0.0;
        }
        o = (float)v;
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// QSTICK (qstick_round in families.cuh)
__device__ void sp_qstick(SP_ARGS) {
  const int po = j.in[0], pc = j.in[1], p = j.ip[0];
  long long f = -1, g = -1;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* O = drv.pptr(c, po);
    const float* C2 = drv.pptr(c, pc);
    for_chunk(rw, [&](int r, long long t) {
      if (f < 0 && !isnan(O[r]) && !isnan(C2[r])) f = t;
      if (f >= 0 && g < 0 && isnan((double)C2[r] - (double)O[r])) g = t;
      float o = qnan();
      if (f >= 0 && t >= f + p - 1 && g < 0) {
        double s = 0.0;
        for (int i = r - p + 1; i <= r; ++i) s += (double)C2[i] - (double)O[i];
        o = (float)(s / (double)p);
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// STOCH (talib08:16115-16302): fastK into the warp line for the chunk and the
// 2(d-1) bars before it, then slowK / slowD as direct means.
__device__ void sp_stoch(SP_ARGS) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0], q = j.ip[1];
  const long long lb = (long long)p - 1 + 2ll * (q - 1);
  const int ext = 2 * (q - 1);
  const double invq = 1.0 / (double)q;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pc = drv.pptr(c, pc);
    const float* X_ph = drv.pptr(c, ph);
    const float* X_plo = drv.pptr(c, plo);
    const int lim = (int)min((long long)C, rw.n - rw.t0);
    for (int r = -ext; r < lim; ++r) {
      const long long t = rw.t0 + r;
      double v = 0.0;
      if (t >= p - 1) {
        double lo = X_plo[r - p + 1], hi = X_ph[r - p + 1];
        for (int i = 1; i < p; ++i) {
          const double l = X_plo[r - p + 1 + i], h = X_ph[r - p + 1 + i];
          if (l < lo) lo = l;
          if (h > hi) hi = h;
        }
        const double range = hi - lo;
        v = fabs(range) <= 1e-14 * (fabs(hi) + fabs(lo)) ? 0.0 : ((double)X_pc[r] - lo) / range * 100.0;
      }
      ln.at(lane, r) = v;
    }
    for_chunk(rw, [&](int r, long long t) {
      float o0 = qnan(), o1 = qnan();
      if (t >= lb) {
        double dsum = 0.0, k0 = 0.0;
        for (int i = 0; i < q; ++i) {
          double s = 0.0;
          for (int m = q - 1; m >= 0; --m) s += ln.at(lane, r - i - m);
          const double kv = s * invq;
          if (i == 0) k0 = kv;
          dsum += kv;
        }
        o0 = (float)k0;
        o1 = (float)(dsum * invq);
      }
      st.put(0, lane, r, o0);
      st.put(1, lane, r, o1);
    });
    SP_FLUSH(0);
    SP_FLUSH(1);
    drv.end(c);
  }
}

__device__ __forceinline__ double typ_price(const float* h, const float* l, const float* c, int r) {
  return ((double)h[r] + (double)l[r] + (double)c[r]) / 3.0;
}

// CCI (CCI.cu:11-40): typical prices of the window into the warp line
__device__ void sp_cci(SP_ARGS) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0];
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const int lim = (int)min((long long)C, rw.n - rw.t0);
    const float* Hp = drv.pptr(c, ph);
    const float* Lp = drv.pptr(c, plo);
    const float* Cp = drv.pptr(c, pc);
    for (int r = -(p - 1); r < lim; ++r) ln.at(lane, r) = typ_price(Hp, Lp, Cp, r);
    for_chunk(rw, [&](int r, long long t) {
      float o = qnan();
      if (t >= p - 1) {
        // four interleaved partial sums shorten the dependent FP64 chains
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int i = 0;
        for (; i + 3 < p; i += 4) {
          s0 += ln.at(lane, r - i); s1 += ln.at(lane, r - i - 1);
          s2 += ln.at(lane, r - i - 2); s3 += ln.at(lane, r - i - 3);
        }
        for (; i < p; ++i) s0 += ln.at(lane, r - i);
        const double sma = ((s0 + s1) + (s2 + s3)) / p;
        double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
        i = 0;
        for (; i + 3 < p; i += 4) {
          d0 += fabs(ln.at(lane, r - i) - sma); d1 += fabs(ln.at(lane, r - i - 1) - sma);
          d2 += fabs(ln.at(lane, r - i - 2) - sma); d3 += fabs(ln.at(lane, r - i - 3) - sma);
        }
        for (; i < p; ++i) d0 += fabs(ln.at(lane, r - i) - sma);
        const double md = ((d0 + d1) + (d2 + d3)) / p;
        const double num = ln.at(lane, r) - sma;
        o = (num != 0.0 && md != 0.0) ? (float)(num / (0.015 * md)) : 0.0f;
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// MFI (StreamStates.h:749-792): flows from the typical-price line, window sums
// re-derived per chunk, re-summed if they cancel below zero.
__device__ void sp_mfi(SP_ARGS) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], pv = j.in[3], p = j.ip[0];
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pv = drv.pptr(c, pv);
    const int lim = (int)min((long long)C, rw.n - rw.t0);
    const float* Hp = drv.pptr(c, ph);
    const float* Lp = drv.pptr(c, plo);
    const float* Cp = drv.pptr(c, pc);
    for (int r = -p; r < lim; ++r) ln.at(lane, r) = typ_price(Hp, Lp, Cp, r);
    auto flow = [&](int r, long long t, double& pos, double& neg) {
      pos = neg = 0.0;
      if (t < 1) return;
      const double pr = ln.at(lane, r), pp = ln.at(lane, r - 1);
      if (isfinite(pr) && isfinite(pp)) {
        const double fl = pr * (double)X_pv[r];
        if (pr > pp) pos = fl;
        else if (pr < pp) neg = fl;
      }
    };
    double ps = 0.0, ns = 0.0;
    bool seeded = false;
    for_chunk(rw, [&](int r, long long t) {
      float o = qnan();
      if (t >= p) {
        double a, b;
        if (!seeded) {
          seeded = true;
          for (int i = p - 1; i >= 0; --i) { flow(r - i, t - i, a, b); ps += a; ns += b; }
        } else {
          flow(r - p, t - p, a, b);
          ps -= a; ns -= b;
          flow(r, t, a, b);
          ps += a; ns += b;
          if (ps < 0.0 || ns < 0.0) {
            ps = ns = 0.0;
            for (int i = p - 1; i >= 0; --i) { flow(r - i, t - i, a, b); ps += a; ns += b; }
          }
        }
        const double tot = ps + ns;
        o = tot < 1.0 ? 0.0f : (float)(100.0 * (ps / tot));
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// ------------------------------------------------------------ recurrences

// EMA (talib08:5546-5627); leading NaNs skipped
__device__ void sp_ema(SP_ARGS) {
  const int pl = j.in[0], p = j.ip[0];
  const double beta = j.fp[0], kk = j.fp[1];
  const bool copy1 = j.family != F_RMA;  // TA_RMA has no period-1 copy
  double y = 0.0;
  long long cnt = -1;  // count of the current bar since the first non-NaN
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    for_chunk(rw, [&](int r, long long) {
      const double x = X_pl[r];
      float o = qnan();
      if (cnt >= 0 || !isnan(x)) {
        ++cnt;
        if (p == 1 && copy1) y = x;
        else if (cnt < p - 1) y += x;
        else if (cnt == p - 1) y = (y + x) / p;
        else y = fma(beta, y, kk * x);
        if (cnt >= p - 1) o = (float)y;
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// DEMA / TEMA / T3 cascades (talib08:4846-4945, 17496-17612, 17331-17481)
__device__ void sp_cascade(SP_ARGS, int stages) {
  const int pl = j.in[0], p = j.ip[0];
  const double beta = j.fp[0], kk = j.fp[1];
  double c1 = 0, c2 = 0, c3 = 0, c4 = 0;
  if (stages == 6) {
    const double v = j.fp[2], tr = v * v;
    c1 = -(tr * v);
    c2 = 3.0 * (tr - c1);
    c3 = -6.0 * tr - 3.0 * (v - c1);
    c4 = fma(3.0, tr, fma(3.0, v, 1.0) - c1);
  }
  double e[6] = {0, 0, 0, 0, 0, 0};
  long long cnt = -1;
  const long long lb = (long long)stages * (p - 1);
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    for_chunk(rw, [&](int r, long long) {
      const double x = X_pl[r];
      float o = qnan();
      if (cnt >= 0 || !isnan(x)) {
        ++cnt;
        double in = x;
#pragma unroll
        for (int s = 0; s < 6; ++s) {
          if (s < stages) {
            const long long rr = cnt - (long long)s * (p - 1);
            if (rr >= 0) {
              if (p == 1) e[s] = in;
              else if (rr < p - 1) e[s] += in;
              else if (rr == p - 1) e[s] = (e[s] + in) / p;
              else e[s] = fma(beta, e[s], kk * in);
            }
            in = e[s];
          }
        }
        if (cnt >= lb) {
          if (p == 1) o = (float)x;
          else if (stages == 2) o = (float)(2.0 * e[0] - e[1]);
          else if (stages == 3) o = (float)(e[2] + (3.0 * e[0] - 3.0 * e[1]));
          else o = (float)fma(c4, e[2], fma(c3, e[3], fma(c1, e[5], c2 * e[4])));
        }
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// RSI (talib08:13996-14115); NaN change poisons; leading NaNs skipped
__device__ void sp_rsi(SP_ARGS) {
  const int pl = j.in[0], p = j.ip[0];
  const double inv = 1.0 / (double)p, pm1 = (double)(p - 1);
  double gain = 0.0, loss = 0.0;
  long long cnt = -1;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    for_chunk(rw, [&](int r, long long) {
      const double x = X_pl[r];
      float o = qnan();
      if (cnt >= 0 || !isnan(x)) {
        ++cnt;
        if (cnt > 0) {
          const double d = x - (double)X_pl[r - 1];
          if (isnan(d)) { gain = loss = d; }
          else {
            const double g = d > 0.0 ? d : 0.0, l = g - d;
            if (cnt < p) { gain += g; loss += l; }
            else if (cnt == p) { gain = (gain + g) * inv; loss = (loss + l) * inv; }
            else { gain = (gain * pm1 + g) * inv; loss = (loss * pm1 + l) * inv; }
          }
        }
        if (cnt >= p) {
          const double tot = gain + loss;
          o = isnan(tot) ? qnan() : (tot > 0.0 ? (float)(100.0 * (gain / tot)) : 50.0f);
        }
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// MACD (talib08:9316-9505); leading NaNs skipped
__device__ void sp_macd(SP_ARGS) {
  const int pl = j.in[0], fast = j.ip[0], slow = j.ip[1], sig = j.ip[2];
  const double fb = j.fp[0], fk = j.fp[1], sb = j.fp[2], sk = j.fp[3];
  double gb, gk;
  talib_ema_coeffs(sig, gb, gk);
  const long long start = slow - 1, ready = start + sig - 1;
  double ps = 0.0, pf = 0.0, psig = 0.0;
  long long cnt = -1;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pl = drv.pptr(c, pl);
    for_chunk(rw, [&](int r, long long) {
      const double x = X_pl[r];
      float o0 = qnan(), o1 = qnan(), o2 = qnan();
      if (cnt >= 0 || !isnan(x)) {
        ++cnt;
        if (cnt < start) {
          ps += x;
          if (cnt >= slow - fast) pf += x;
        } else if (cnt == start) {
          ps = (ps + x) / slow;
          pf = (pf + x) / fast;
        } else {
          pf = fma(fb, pf, fk * x);
          ps = fma(sb, ps, sk * x);
        }
        if (cnt >= start) {
          const double m = pf - ps;
          if (cnt < ready) psig += m;
          else if (cnt == ready) psig = (psig + m) / sig;
          else psig = sig == 1 ? m : fma(gb, psig, gk * m);
          if (cnt >= ready) { o0 = (float)m; o1 = (float)psig; o2 = (float)(m - psig); }
        }
      }
      st.put(0, lane, r, o0);
      st.put(1, lane, r, o1);
      st.put(2, lane, r, o2);
    });
    SP_FLUSH(0);
    SP_FLUSH(1);
    SP_FLUSH(2);
    drv.end(c);
  }
}

// ATR / NATR / TRANGE (mode 0/1/2)
__device__ void sp_atr(SP_ARGS, int mode) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2];
  const int p = mode == 2 ? 1 : j.ip[0];
  const double wb = j.fp[0], wa = j.fp[1];
  double y = 0.0;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pc = drv.pptr(c, pc);
    const float* X_ph = drv.pptr(c, ph);
    const float* X_plo = drv.pptr(c, plo);
    for_chunk(rw, [&](int r, long long t) {
      float o = qnan();
      if (t >= 1) {
        const double tr = true_range((double)X_ph[r], (double)X_plo[r], (double)X_pc[r - 1]);
        if (mode == 2) o = (float)tr;
        else {
          if (t < p) y += tr;
          else if (t == p) y = (y + tr) / p;
          else y = fma(wb, y, wa * tr);
          if (t >= p) {
            if (mode == 0 || p == 1) o = (float)y;
            else {
              const double cl = X_pc[r];
              o = cl == 0.0 ? 0.0f : (float)((y / cl) * 100.0);
            }
          }
        }
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// ADX / DX (DX.cu, ADX.cu, BatchShort.cu:168-230 conventions)
__device__ void sp_adx(SP_ARGS, bool adx) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0];
  const double a = ((double)p - 1.0) / (double)p;
  double tr = 0.0, pd = 0.0, md = 0.0, av = 0.0;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_pc = drv.pptr(c, pc);
    const float* X_ph = drv.pptr(c, ph);
    const float* X_plo = drv.pptr(c, plo);
    for_chunk(rw, [&](int r, long long t) {
      double range, plus = 0.0, minus = 0.0;
      if (t == 0) {
        range = (double)X_ph[r] - (double)X_plo[r];
      } else {
        const float u = X_ph[r] - X_ph[r - 1], dw = X_plo[r - 1] - X_plo[r];
        plus = (u > 0.0f && u > dw) ? u : 0.0f;
        minus = (dw > 0.0f && dw > u) ? dw : 0.0f;
        const double hh = X_ph[r], ll = X_plo[r], yc = X_pc[r - 1];
        range = fmax(hh - ll, fmax(fabs(hh - yc), fabs(ll - yc)));
      }
      float o = qnan();
      if (t < p) { tr += range; pd += plus; md += minus; }
      else {
        tr = a * tr + range;
        pd = a * pd + plus;
        md = a * md + minus;
        const double dip = tr > 0.0 ? 100.0 * pd / tr : 0.0;
        const double dim = tr > 0.0 ? 100.0 * md / tr : 0.0;
        const double tot = dip + dim;
        const double dx = tot > 0.0 ? 100.0 * fabs(dip - dim) / tot : 0.0;
        if (!adx) o = (float)dx;
        else if (t < 2 * p - 1) av += dx;
        else if (t == 2 * p - 1) { av = (av + dx) / p; o = (float)av; }
        else { av = a * av + dx / p; o = (float)av; }
      }
      st.put(0, lane, r, o);
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

// OBV / AD / ADOSC (mode 0/1/2; StreamStates.h:446-506, 723-745)
__device__ void sp_volume(SP_ARGS, int mode) {
  double acc = 0.0, fast = 0.0, slow = 0.0;
  const int warm = mode == 2 ? (j.ip[0] > j.ip[1] ? j.ip[0] : j.ip[1]) - 1 : 0;
  const double kf = mode == 2 ? 2.0 / (j.ip[0] + 1.0) : 0.0, ks = mode == 2 ? 2.0 / (j.ip[1] + 1.0) : 0.0;
  for (int c = 0; c < drv.nchunks; ++c) {
    drv.begin(c);
    const Row rw = drv.row(c);
    const float* X_j_in_0_ = drv.pptr(c, j.in[0]);
    const float* X_j_in_1_ = drv.pptr(c, j.in[1]);
    const float* X_j_in_2_ = drv.pptr(c, j.in[2]);
    const float* X_j_in_3_ = drv.pptr(c, j.in[3]);
    for_chunk(rw, [&](int r, long long t) {
      if (mode == 0) {
        const double v = X_j_in_1_[r];
        if (t == 0) acc += v;
        else {
          const double pr = X_j_in_0_[r], pp = X_j_in_0_[r - 1];
          acc += (pr > pp ? 1.0 : (pr < pp ? -1.0 : 0.0)) * v;
        }
        st.put(0, lane, r, (float)acc);
        return;
      }
      const double hi = X_j_in_0_[r], lo = X_j_in_1_[r], cl = X_j_in_2_[r], vo = X_j_in_3_[r];
      double term = 0.0;
      if (isfinite(hi) && isfinite(lo) && isfinite(cl) && isfinite(vo)) {
        const double range = hi - lo;
        if (range > 0.0) term = (((cl - lo) - (hi - cl)) / range) * vo;
      }
      acc += term;
      if (mode == 1) { st.put(0, lane, r, (float)acc); return; }
      if (t == 0) fast = slow = acc;
      else {
        fast = kf * acc + (1.0 - kf) * fast;
        slow = ks * acc + (1.0 - ks) * slow;
      }
      st.put(0, lane, r, t < warm ? qnan() : (float)(fast - slow));
    });
    SP_FLUSH(0);
    drv.end(c);
  }
}

#undef SP_FLUSH
#undef SP_ARGS

}  // namespace sp
}  // namespace tb
