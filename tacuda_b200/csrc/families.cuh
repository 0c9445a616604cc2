// Per-round device implementations of the indicator families.
//
// A "round" is TILE = 32*K consecutive bars of one series handled by one warp
// (lane l owns K consecutive bars). Recurrences are evaluated as piecewise
// affine maps in FP64: each lane composes its K maps, a warp shuffle scan
// stitches the lanes, then every lane replays its bars with the exact TA-Lib
// arithmetic starting from its incoming state. Windows read the staged halo.
//
// Arithmetic per family follows the pinned TA-Lib 0.8.3 C
// (src/compat/talib08_formulas.inc in the reference, "talib08" below) or, for
// families the vendored set lacks, the reference kernels; the citations are on
// each round function. Outputs are float32 with NaN warm-up.
#pragma once

#include "common.cuh"
#include "engine.h"
#include "lookback.cuh"

namespace tb {

// Carry of one job between rounds of a series (kept in shared memory).
struct Carry {
  int f;  // first bar that counts (after leading NaNs), -1 = not found yet
  double v[10];
};

template <int K>
struct Ctx {
  static constexpr int TILE = 32 * K;
  static constexpr int EXT = 64;                                 // front extension of a line
  static constexpr int LINE = (TILE + EXT) + (TILE + EXT) / 16 + 1;  // padded doubles per line
  int lane;
  int n;     // row length
  int t0;    // first bar of the round
  int L;           // bars in the round
  int H;           // staged halo
  long long base;  // row offset in the planes (64-bit); bar indices within a row are int
  long long obase; // row offset in the outputs (= base except for streaming appends)
  int lo;          // first bar of the row held in the planes (0 except for appends)
  // This warp's shared memory, addressed from the kernel's extern __shared__
  // base so every access below compiles to a shared-space load or store.
  unsigned char* sm;
  int off_planes, plane_len, off_tp, off_dscr, off_stage, stage_len;
  unsigned slots;  // 4-bit staged slot of each plane
  bool has_tp;
  // look-back mode: this round is tile `tile` of a series split across warps
  bool lb;
  int tile;
  LbDesc* lbd;       // descriptors of this series' tile 0 (slot 0)
  long long lbs;     // descriptors per tile
  int* err;

  __device__ __forceinline__ const float* plane(int p) const {
    return reinterpret_cast<const float*>(sm + off_planes) + (int)((slots >> (4 * p)) & 15u) * plane_len;
  }
  __device__ __forceinline__ int gb0() const { return t0 + lane * K; }
  __device__ __forceinline__ bool valid(int t) const { return t < t0 + L; }
  __device__ __forceinline__ float x(int p, int t) const { return plane(p)[pad((t - t0) + H)]; }
  __device__ __forceinline__ double typ(int t) const {
    const int i = (t - t0) + H;
    return reinterpret_cast<const double*>(sm + off_tp)[i + (i >> 4)];
  }
  // Scratch line entry for round-relative bar idx in [-EXT, TILE).
  __device__ __forceinline__ double& eline(int ln, int idx) const {
    const int i = idx + EXT;
    return reinterpret_cast<double*>(sm + off_dscr)[ln * LINE + i + (i >> 4)];
  }
  __device__ __forceinline__ double& line(int ln, int k) const { return eline(ln, lane * K + k); }
  __device__ __forceinline__ float* stage(int j) const {
    return reinterpret_cast<float*>(sm + off_stage) + j * stage_len;
  }
  __device__ __forceinline__ void put(int j, int k, float v) const { stage(j)[pad(lane * K + k)] = v; }

  // Coalesced copy of staged output j to out[base + t0 .. + L).
  __device__ __forceinline__ void flush(int j, float* out) const {
    __syncwarp();
    float* dst = out + obase + t0;
    const float* src = stage(j);
    for (int i = lane; i < L; i += 32) dst[i] = src[pad(i)];
    __syncwarp();
  }
};

// First bar from which a single-input recurrence counts: the first non-NaN bar
// of the row (src/api/BatchFused.cu:34-41 skips a leading NaN run). Resolved
// once per series; warp-uniform. -1 while the row is all NaN so far.
template <int K>
__device__ __forceinline__ int resolve_start(const Ctx<K>& c, const Carry& cy, int plane, int slot = -1) {
  if (!c.lb && cy.f >= 0) return cy.f;
  int first = 0x7fffffff;
  for (int k = 0; k < K; ++k) {
    const int t = c.gb0() + k;
    if (c.valid(t) && !isnan(c.x(plane, t))) { first = t; break; }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) first = min(first, __shfl_xor_sync(kFull, first, d));
  const int local = first == 0x7fffffff ? -1 : first;
  if (c.lb) return lb_first_index(c.lbd + slot, c.lbs, c.tile, local, c.err, c.lane);
  return local;
}

// Value held after the last valid bar of the round (exact replay state).
template <int K>
__device__ __forceinline__ double round_tail(const Ctx<K>& c, double v) {
  return __shfl_sync(kFull, v, (c.L - 1) / K);
}

// ----------------------------------------------------------------- EMA core

// Recurrence stages are piecewise affine: bar with count c maps the state y to
// a(c)*y + w(c)*x + (terms independent of x). The warp scan composes these maps
// in coordinates shifted by E(c)*o, the state the stage would hold after count
// c if every input equalled the origin o (a level stage: E = o once seeded,
// (r+1)*o while summing its seed). The shifted map is y' = a*y + w*(x - o), so
// a constant series composes to exactly zero offset and every lane starts from
// the exact level; otherwise the shift only improves the carries' rounding.
// The lanes then replay their bars with TA-Lib's own arithmetic.

// One EMA stage in TA-Lib order (talib08:5546-5627): inputs counted from
// `start` are summed, the mean of the first p seeds the average at count
// start+p-1, later bars apply y = fma(beta, y, k*x). Period 1 copies.
struct EmaStage {
  int p, start;
  double beta, k, inv;
  // period 1 copies the input (TA_EMA); RMA clears it and keeps the general
  // steps, so a NaN propagates through fma(0, y, x) as in TA_RMA
  bool copy1 = true;
  __device__ __forceinline__ void coef(int cnt, double& a, double& w) const {
    if (cnt < start) { a = 1.0; w = 0.0; return; }
    if (p == 1 && copy1) { a = 0.0; w = 1.0; return; }
    const int r = cnt - start;
    if (r < p - 1) { a = 1.0; w = 1.0; }
    else if (r == p - 1) { a = inv; w = inv; }
    else { a = beta; w = k; }
  }
  // E(cnt) / o after the bar with count cnt
  __device__ __forceinline__ double expect(int cnt) const {
    if (cnt < start) return 0.0;
    const int r = cnt - start;
    return (p > 1 && r < p - 1) ? (double)(r + 1) : 1.0;
  }
  __device__ __forceinline__ double step(int cnt, double y, double x) const {
    if (cnt < start) return y;
    if (p == 1 && copy1) return x;
    const int r = cnt - start;
    if (r < p - 1) return y + x;
    if (r == p - 1) return (y + x) / p;
    return fma(beta, y, k * x);
  }
  __device__ __forceinline__ bool ready(int cnt) const { return cnt >= start + p - 1; }
  // first count whose map is the constant steady one
  __device__ __forceinline__ int steady_from() const { return p == 1 && copy1 ? 0 : start + p; }
};

// Scan one stage over the round. in(t, k) gives the FP64 input of the lane's
// k-th bar; sink(k, cnt, y) receives the state after it (cnt = -1 before the
// series starts). Returns the state after the round.
template <int K, class Stage, class In, class Sink>
__device__ __forceinline__ double stage_round(const Ctx<K>& c, int f, const Stage& st,
                                              double carry, In in, Sink sink, int slot = -1) {
  const int g0 = c.gb0();
  // inputs of the lane's bars, evaluated once and kept in registers
  double xin[K];
#pragma unroll
  for (int k = 0; k < K; ++k) xin[k] = (f >= 0 && c.valid(g0 + k) && g0 + k >= f) ? in(g0 + k, k) : 0.0;
  // origin: input of the first counted bar of the round (warp-uniform)
  double o = 0.0;
  if (f >= 0) {
    const int to = c.t0 > f ? c.t0 : f;
    if (to < c.t0 + c.L) {
      const int lo = (to - c.t0) / K, ko = (to - c.t0) % K;
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (k == ko) v = xin[k];
      o = __shfl_sync(kFull, v, lo);
      if (!isfinite(o)) o = 0.0;
    }
  }
  double A = 1.0, B = 0.0;
  if (f >= 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int t = g0 + k;
      if (c.valid(t) && t >= f) {
        double a, w;
        st.coef(t - f, a, w);
        B = fma(a, B, w * (xin[k] - o));
        A *= a;
      }
    }
  }
  warp_scan_affine(A, B, c.lane);
  const double Ae = shfl_excl(A, 1.0, c.lane), Be = shfl_excl(B, 0.0, c.lane);
  if (c.lb && slot >= 0) {
    // aggregate of the tile in absolute coordinates (meaningful when the tile
    // starts past warm-up, where E = 1 before and after every bar)
    const double tA[1] = {__shfl_sync(kFull, A, 31)};
    const double tB[1] = {__shfl_sync(kFull, B, 31) + o * (1.0 - tA[0])};
    const double init[1] = {carry};
    double Y[1];
    lb_resolve<1>(c.lbd + slot, c.lbs, c.tile, tA, tB, init, lb_first_steady(f, st.steady_from(), Ctx<K>::TILE), Y,
                  c.err, c.lane);
    carry = Y[0];
  }
  double y = carry;
  if (f >= 0) {
    const int cr = c.t0 - 1 - f, cl = g0 - 1 - f;
    const double er = cr >= 0 ? st.expect(cr) * o : 0.0;
    const double el = cl >= 0 ? st.expect(cl) * o : 0.0;
    y = el + fma(Ae, carry - er, Be);
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (c.valid(t)) {
      if (f < 0 || t < f) sink(k, -1, y);
      else {
        y = st.step(t - f, y, xin[k]);
        sink(k, t - f, y);
      }
    }
  }
  const double tail = round_tail(c, y);
  if (c.lb && slot >= 0) {
    const double Y[1] = {tail};
    lb_publish<1>(c.lbd + slot, c.lbs, c.tile, Y, c.lane);
  }
  return tail;
}

// EMA(p): talib08:5546-5627 TA_EMA; leading NaNs skipped (BatchFused.cu:34-41).
// fp[0] = beta, fp[1] = k (host-precomputed TA-Lib coefficients).
// RMA(p) is the same stage (talib08:13614-13683 TA_RMA: mean seed, then
// fma(wBeta, y, wAlpha*x)) with wBeta = (p-1)/p, wAlpha = 1 - wBeta and no
// period-1 copy; the reference's TA-Lib runner skips the row's leading NaNs
// the same way (src/compat/Talib08.cu:72-84).
template <int K>
__device__ __forceinline__ void ema_round(const Ctx<K>& c, const Job& j, Carry& cy) {
  const int pl = j.in[0];
  const int f = resolve_start(c, cy, pl, j.lb_slot);
  const EmaStage st{j.ip[0], 0, j.fp[0], j.fp[1], 1.0 / j.ip[0], j.family != F_RMA};
  cy.v[0] = stage_round(
      c, f, st, cy.v[0], [&](int t, int) { return (double)c.x(pl, t); },
      [&](int k, int cnt, double v) { c.put(0, k, (cnt >= 0 && st.ready(cnt)) ? (float)v : qnan()); },
      j.lb_slot + 1);
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
}

// DEMA / TEMA / T3: cascades of EMA stages, stage s seeded with the mean of the
// first p values of stage s-1 (talib08:4846-4945 DEMA, 17496-17612 TEMA,
// 17331-17481 T3). DEMA/TEMA use TA_EMA's coefficients, T3 k=2/(p+1) with
// fma(1-k, e, k*x) and the GD combination; fp[0]=beta fp[1]=k, fp[2]=vfactor.
// Scratch lines: 0 = running stage value, 1.. = stage values kept for the
// combination (DEMA: e1; TEMA: e1 e2; T3: e3 e4 e5).
template <int K>
__device__ __forceinline__ void cascade_round(const Ctx<K>& c, const Job& j, Carry& cy, int stages) {
  const int pl = j.in[0];
  const int f = resolve_start(c, cy, pl, j.lb_slot);
  const int p = j.ip[0];
  const double beta = j.fp[0], kk = j.fp[1];
  double c1 = 0, c2 = 0, c3 = 0, c4 = 0;
  if (stages == 6) {
    const double v = j.fp[2], tr = v * v;
    c1 = -(tr * v);
    c2 = 3.0 * (tr - c1);
    c3 = -6.0 * tr - 3.0 * (v - c1);
    c4 = fma(3.0, tr, fma(3.0, v, 1.0) - c1);
  }
  const int lb = stages * (p - 1);
  for (int s = 0; s < stages; ++s) {
    const EmaStage st{p, s * (p - 1), beta, kk, 1.0 / p};
    const bool last = s == stages - 1;
    int keep = -1;  // kept line storing this stage's value
    if (stages == 2 && s == 0) keep = 1;
    if (stages == 3 && s < 2) keep = 1 + s;
    if (stages == 6 && s >= 2 && s <= 4) keep = s - 1;
    cy.v[s] = stage_round(
        c, f, st, cy.v[s],
        [&](int t, int k) { return s == 0 ? (double)c.x(pl, t) : c.line(0, k); },
        [&](int k, int cnt, double v) {
          c.line(0, k) = v;
          if (keep >= 0) c.line(keep, k) = v;
          if (last) {
            float o = qnan();
            if (cnt >= lb) {
              if (p == 1) o = (float)v;
              else if (stages == 2) o = (float)(2.0 * c.line(1, k) - v);
              else if (stages == 3) o = (float)(v + (3.0 * c.line(1, k) - 3.0 * c.line(2, k)));
              else o = (float)fma(c4, c.line(1, k), fma(c3, c.line(2, k), fma(c1, v, c2 * c.line(3, k))));
            }
            c.put(0, k, o);
          }
        },
        j.lb_slot + 1 + s);
    __syncwarp();
  }
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
}

// ----------------------------------------------------------------- RSI

// RSI(p): talib08:13996-14115 TA_RSI. Gains and losses of the first p changes
// are summed and multiplied by 1/p; afterwards g = (g*(p-1) + gain)/p via the
// same multiply by 1/p; 100*g/(g+l), 50 when both are zero. A NaN change makes
// the row NaN from there on (StreamStates.h:663). Leading NaNs skipped.
template <int K>
__device__ __forceinline__ void rsi_round(const Ctx<K>& c, const Job& j, Carry& cy) {
  const int pl = j.in[0];
  const int f = resolve_start(c, cy, pl, j.lb_slot);
  const int p = j.ip[0];
  const double inv = 1.0 / (double)p, pm1 = (double)(p - 1);
  const double steady = pm1 * inv;
  double A = 1.0, B[2] = {0.0, 0.0};
  const int g0 = c.gb0();
  double gk[K], lk[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    gk[k] = lk[k] = 0.0;
    if (f >= 0 && c.valid(t) && t - f > 0) {
      const double d = (double)c.x(pl, t) - (double)c.x(pl, t - 1);
      if (isnan(d)) { gk[k] = lk[k] = d; }
      else { gk[k] = d > 0.0 ? d : 0.0; lk[k] = gk[k] - d; }
    }
  }
  if (f >= 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int t = g0 + k;
      const int cnt = t - f;
      if (c.valid(t) && cnt > 0) {
        double g = gk[k], l = lk[k], a;
        if (cnt < p) a = 1.0;
        else if (cnt == p) { a = inv; g *= inv; l *= inv; }
        else { a = steady; g *= inv; l *= inv; }
        B[0] = fma(a, B[0], g);
        B[1] = fma(a, B[1], l);
        A *= a;
      }
    }
  }
  warp_scan_affine_shared<2>(A, B, c.lane);
  const double Ae = shfl_excl(A, 1.0, c.lane);
  const double Be0 = shfl_excl(B[0], 0.0, c.lane), Be1 = shfl_excl(B[1], 0.0, c.lane);
  if (c.lb) {
    const double a31 = __shfl_sync(kFull, A, 31);
    const double tA[2] = {a31, a31};
    const double tB[2] = {__shfl_sync(kFull, B[0], 31), __shfl_sync(kFull, B[1], 31)};
    const double init[2] = {cy.v[0], cy.v[1]};
    double Y[2];
    lb_resolve<2>(c.lbd + j.lb_slot + 1, c.lbs, c.tile, tA, tB, init, lb_first_steady(f, p + 1, Ctx<K>::TILE), Y,
                  c.err, c.lane);
    cy.v[0] = Y[0];
    cy.v[1] = Y[1];
  }
  double gain = fma(Ae, cy.v[0], Be0);
  double loss = fma(Ae, cy.v[1], Be1);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) continue;
    const int cnt = f < 0 ? -1 : t - f;
    if (cnt > 0) {
      const double g = gk[k], l = lk[k];
      if (isnan(g)) { gain = loss = g; }
      else if (cnt < p) { gain += g; loss += l; }
      else if (cnt == p) { gain = (gain + g) * inv; loss = (loss + l) * inv; }
      else {
        gain = (gain * pm1 + g) * inv;
        loss = (loss * pm1 + l) * inv;
      }
    }
    float o = qnan();
    if (cnt >= p) {
      const double tot = gain + loss;
      o = isnan(tot) ? qnan() : (tot > 0.0 ? (float)(100.0 * (gain / tot)) : 50.0f);
    }
    c.put(0, k, o);
  }
  cy.v[0] = round_tail(c, gain);
  cy.v[1] = round_tail(c, loss);
  if (c.lb) {
    const double Y[2] = {cy.v[0], cy.v[1]};
    lb_publish<2>(c.lbd + j.lb_slot + 1, c.lbs, c.tile, Y, c.lane);
  }
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
}

// ----------------------------------------------------------------- MACD

// Signal line of MACD: accumulate the MACD values from `start`, seed with their
// mean at `ready`, then fma(gb, y, gk*m); signal period 1 copies.
struct SigStage {
  int sig;
  int start, ready;
  double gb, gk, inv;
  __device__ __forceinline__ void coef(int cnt, double& a, double& w) const {
    if (cnt < start) { a = 1.0; w = 0.0; }
    else if (cnt < ready) { a = 1.0; w = 1.0; }
    else if (cnt == ready) { a = inv; w = inv; }
    else if (sig == 1) { a = 0.0; w = 1.0; }
    else { a = gb; w = gk; }
  }
  __device__ __forceinline__ double expect(int cnt) const {
    if (cnt < start) return 0.0;
    if (cnt < ready) return (double)(cnt - start + 1);
    return 1.0;
  }
  __device__ __forceinline__ int steady_from() const { return (int)ready + 1; }
  __device__ __forceinline__ double step(int cnt, double y, double m) const {
    if (cnt < start) return y;
    if (cnt < ready) return y + m;
    if (cnt == ready) return (y + m) / sig;
    return sig == 1 ? m : fma(gb, y, gk * m);
  }
};

// MACD(fast, slow, signal): talib08:9316-9505 TA_MACD. The slow average is
// seeded with the mean of the first `slow` bars, the fast one with the mean of
// the `fast` bars ending at the same bar (slow-1); both then fma(beta, y, k*x).
// The signal line runs over the FP64 MACD values; outputs from slow+signal-2.
// Reversed periods are swapped on the host; fp = [fast beta, fast k, slow
// beta, slow k]. Leading NaNs skipped. Scratch line 0 carries the slow line,
// then the MACD line.
template <int K>
__device__ __forceinline__ void macd_round(const Ctx<K>& c, const Job& j, Carry& cy) {
  const int pl = j.in[0];
  const int f = resolve_start(c, cy, pl, j.lb_slot);
  const int fast = j.ip[0], slow = j.ip[1], sig = j.ip[2];
  const EmaStage slowSt{slow, 0, j.fp[2], j.fp[3], 1.0 / slow};
  const EmaStage fastSt{fast, slow - fast, j.fp[0], j.fp[1], 1.0 / fast};
  double gb, gk;
  talib_ema_coeffs(sig, gb, gk);
  const int start = slow - 1, ready = start + sig - 1;
  auto px = [&](int t, int) { return (double)c.x(pl, t); };
  cy.v[1] = stage_round(c, f, slowSt, cy.v[1], px, [&](int k, int, double y) { c.line(0, k) = y; }, j.lb_slot + 1);
  cy.v[0] = stage_round(c, f, fastSt, cy.v[0], px, [&](int k, int cnt, double y) {
    c.line(0, k) = cnt >= start ? y - c.line(0, k) : 0.0;
  }, j.lb_slot + 2);
  const SigStage sst{sig, start, ready, gb, gk, 1.0 / sig};
  cy.v[2] = stage_round(
      c, f, sst, cy.v[2], [&](int, int k) { return c.line(0, k); },
      [&](int k, int cnt, double s) {
        const bool ok = cnt >= ready;
        const double m = c.line(0, k);
        c.put(0, k, ok ? (float)m : qnan());
        c.put(1, k, ok ? (float)s : qnan());
        c.put(2, k, ok ? (float)(m - s) : qnan());
      },
      j.lb_slot + 3);
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
  c.flush(1, (float*)j.out[1]);
  c.flush(2, (float*)j.out[2]);
}

// ----------------------------------------------------------------- ATR family

// Wilder average of the true range as TA_ATR computes it: bars 1..p are summed
// and divided by p at bar p, later bars apply fma(wb, y, wa*tr).
struct AtrStage {
  int p;
  double wb, wa, inv;
  __device__ __forceinline__ void coef(int t, double& a, double& w) const {
    if (t < 1) { a = 1.0; w = 0.0; }
    else if (t < p) { a = 1.0; w = 1.0; }
    else if (t == p) { a = inv; w = inv; }
    else { a = wb; w = wa; }
  }
  __device__ __forceinline__ double expect(int t) const {
    if (t < 1) return 0.0;
    return t < p ? (double)t : 1.0;
  }
  __device__ __forceinline__ int steady_from() const { return p + 1; }
  __device__ __forceinline__ double step(int t, double y, double r) const {
    if (t < 1) return y;
    if (t < p) return y + r;
    if (t == p) return (y + r) / p;
    return fma(wb, y, wa * r);
  }
};

// ATR(p): talib08:1931-2057 TA_ATR (first output at bar p); wb = (p-1)/p and
// wa = 1-wb in fp[0..1]. NATR (StreamStates.h:708-721): 100*ATR/close in FP64,
// 0 for a zero close; period 1 keeps the unnormalised true range. TRANGE:
// true range from bar 1 (talib08:17625-17690). mode: 0 ATR, 1 NATR, 2 TRANGE.
template <int K>
__device__ __forceinline__ void atr_round(const Ctx<K>& c, const Job& j, Carry& cy, int mode) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2];
  auto tr = [&](int t, int) {
    return t < 1 ? 0.0 : true_range((double)c.x(ph, t), (double)c.x(plo, t), (double)c.x(pc, t - 1));
  };
  const int g0 = c.gb0();
  if (mode == 2) {
    for (int k = 0; k < K; ++k) {
      const int t = g0 + k;
      if (!c.valid(t)) break;
      c.put(0, k, t >= 1 ? (float)tr(t, k) : qnan());
    }
    c.flush(0, (float*)j.out[0]);
    return;
  }
  const int p = j.ip[0];
  const AtrStage st{p, j.fp[0], j.fp[1], 1.0 / p};
  cy.v[0] = stage_round(c, 0, st, cy.v[0], tr, [&](int k, int t, double y) {
    float o = qnan();
    if (t >= p) {
      if (mode == 0 || p == 1) o = (float)y;
      else {
        const double cl = c.x(pc, t);
        o = cl == 0.0 ? 0.0f : (float)((y / cl) * 100.0);
      }
    }
    c.put(0, k, o);
  }, j.lb_slot);
  c.flush(0, (float*)j.out[0]);
}

// ----------------------------------------------------------------- ADX / DX

// ADX(p) / DX(p) as the reference computes them (src/indicators/DX.cu:18-52,
// 85-135; ADX.cu:44-124; BatchShort.cu:168-230): bar 0 contributes TR = H-L and
// no movement; TR, +DM, -DM are summed over bars 0..p-1, then S = a*S + x with
// a = (p-1)/p; DX = 100|DI+ - DI-|/(DI+ + DI-) from bar p (0 when TR or the DI
// sum is 0); ADX is the mean of DX over bars p..2p-1, then a*ADX + DX/p.
// The reference keeps DI/DX in float; this path keeps them in FP64.
template <int K>
__device__ __forceinline__ void adx_round(const Ctx<K>& c, const Job& j, Carry& cy, bool adx) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2];
  const int p = j.ip[0];
  const double a = ((double)p - 1.0) / (double)p;
  auto moves = [&](int t, double& r, double& pl, double& mi) {
    if (t == 0) {
      r = (double)c.x(ph, 0) - (double)c.x(plo, 0);
      pl = mi = 0.0;
      return;
    }
    const float up = c.x(ph, t) - c.x(ph, t - 1), dn = c.x(plo, t - 1) - c.x(plo, t);
    pl = (up > 0.0f && up > dn) ? up : 0.0f;
    mi = (dn > 0.0f && dn > up) ? dn : 0.0f;
    const double hh = c.x(ph, t), ll = c.x(plo, t), yc = c.x(pc, t - 1);
    r = fmax(hh - ll, fmax(fabs(hh - yc), fabs(ll - yc)));
  };
  const int g0 = c.gb0();
  double rk[K];
  float pk[K], mk[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    rk[k] = 0.0; pk[k] = mk[k] = 0.0f;
    if (c.valid(g0 + k)) {
      double pl, mi;
      moves(g0 + k, rk[k], pl, mi);
      pk[k] = (float)pl; mk[k] = (float)mi;
    }
  }
  double A = 1.0, B[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (c.valid(t)) {
      const double m = t < p ? 1.0 : a;
      B[0] = fma(m, B[0], rk[k]);
      B[1] = fma(m, B[1], (double)pk[k]);
      B[2] = fma(m, B[2], (double)mk[k]);
      A *= m;
    }
  }
  warp_scan_affine_shared<3>(A, B, c.lane);
  const double Ae = shfl_excl(A, 1.0, c.lane);
  const double Be0 = shfl_excl(B[0], 0.0, c.lane), Be1 = shfl_excl(B[1], 0.0, c.lane),
               Be2 = shfl_excl(B[2], 0.0, c.lane);
  if (c.lb) {
    const double a31 = __shfl_sync(kFull, A, 31);
    const double tA[3] = {a31, a31, a31};
    const double tB[3] = {__shfl_sync(kFull, B[0], 31), __shfl_sync(kFull, B[1], 31), __shfl_sync(kFull, B[2], 31)};
    const double init[3] = {cy.v[0], cy.v[1], cy.v[2]};
    double Y[3];
    lb_resolve<3>(c.lbd + j.lb_slot, c.lbs, c.tile, tA, tB, init, lb_first_steady(0, p, Ctx<K>::TILE), Y, c.err,
                  c.lane);
    cy.v[0] = Y[0]; cy.v[1] = Y[1]; cy.v[2] = Y[2];
  }
  double tr = fma(Ae, cy.v[0], Be0);
  double pd = fma(Ae, cy.v[1], Be1);
  double md = fma(Ae, cy.v[2], Be2);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) continue;
    const double r = rk[k], pl = pk[k], mi = mk[k];
    double dx = 0.0;
    if (t < p) { tr += r; pd += pl; md += mi; }
    else {
      tr = a * tr + r;
      pd = a * pd + pl;
      md = a * md + mi;
      const double rtr = tr > 0.0 ? 100.0 / tr : 0.0;
      const double dip = pd * rtr;
      const double dim = md * rtr;
      const double tot = dip + dim;
      dx = tot > 0.0 ? 100.0 * fabs(dip - dim) / tot : 0.0;
    }
    c.line(0, k) = dx;
    if (!adx) c.put(0, k, t >= p ? (float)dx : qnan());
  }
  cy.v[0] = round_tail(c, tr);
  cy.v[1] = round_tail(c, pd);
  cy.v[2] = round_tail(c, md);
  if (c.lb) {
    const double Y[3] = {cy.v[0], cy.v[1], cy.v[2]};
    lb_publish<3>(c.lbd + j.lb_slot, c.lbs, c.tile, Y, c.lane);
  }
  if (adx) {
    struct AdxStage {
      int p; double a, inv;
      __device__ __forceinline__ void coef(int t, double& m, double& w) const {
        if (t < p) { m = 1.0; w = 0.0; }
        else if (t < 2 * p - 1) { m = 1.0; w = 1.0; }
        else if (t == 2 * p - 1) { m = inv; w = inv; }
        else { m = a; w = inv; }
      }
      __device__ __forceinline__ double expect(int t) const {
        if (t < p) return 0.0;
        return t < 2 * p - 1 ? (double)(t - p + 1) : 1.0;
      }
      __device__ __forceinline__ int steady_from() const { return 2 * p; }
      __device__ __forceinline__ double step(int t, double y, double dx) const {
        if (t < p) return y;
        if (t < 2 * p - 1) return y + dx;
        if (t == 2 * p - 1) return (y + dx) / p;
        return a * y + dx / p;
      }
    } st{p, a, 1.0 / p};
    cy.v[3] = stage_round(
        c, 0, st, cy.v[3], [&](int, int k) { return c.line(0, k); },
        [&](int k, int t, double y) { c.put(0, k, t >= 2 * p - 1 ? (float)y : qnan()); }, j.lb_slot + 1);
  }
  c.flush(0, (float*)j.out[0]);
}

// ----------------------------------------------------------------- volume

// OBV (StreamStates.h:446-475): bar 0 adds its volume, later bars the volume
// signed by the close change; FP64 running sum (exact for float32 volumes).
// AD (:481-506): ((c-l)-(h-c))/(h-l)*v, skipped for non-finite bars and
// non-positive ranges. ADOSC (:723-745): EMA(fast) - EMA(slow) of the AD line,
// both seeded with AD[0], k = 2/(n+1), warm-up max(fast, slow)-1.
// mode: 0 OBV (in: close, volume), 1 AD, 2 ADOSC (in: h, l, c, v).
template <int K>
__device__ __forceinline__ void volume_round(const Ctx<K>& c, const Job& j, Carry& cy, int mode) {
  const int g0 = c.gb0();
  auto term = [&](int t) -> double {
    if (mode == 0) {
      const int pc = j.in[0], pv = j.in[1];
      const double v = c.x(pv, t);
      if (t == 0) return v;
      const double pr = c.x(pc, t), pp = c.x(pc, t - 1);
      const double s = pr > pp ? 1.0 : (pr < pp ? -1.0 : 0.0);
      return s * v;
    }
    const double hi = c.x(j.in[0], t), lo = c.x(j.in[1], t), cl = c.x(j.in[2], t), vo = c.x(j.in[3], t);
    if (isfinite(hi) && isfinite(lo) && isfinite(cl) && isfinite(vo)) {
      const double range = hi - lo;
      if (range > 0.0) return (((cl - lo) - (hi - cl)) / range) * vo;
    }
    return 0.0;
  };
  double tm[K];
  double B = 0.0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    tm[k] = c.valid(g0 + k) ? term(g0 + k) : 0.0;
    B += tm[k];
  }
  // prefix sum (all multipliers are 1)
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double u = __shfl_up_sync(kFull, B, d);
    if (c.lane >= d) B += u;
  }
  if (c.lb) {
    const double tA[1] = {1.0};
    const double tB[1] = {__shfl_sync(kFull, B, 31)};
    const double init[1] = {cy.v[0]};
    double Y[1];
    lb_resolve<1>(c.lbd + j.lb_slot, c.lbs, c.tile, tA, tB, init, 0, Y, c.err, c.lane);
    cy.v[0] = Y[0];
  }
  double acc = cy.v[0] + shfl_excl(B, 0.0, c.lane);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!c.valid(g0 + k)) continue;
    acc += tm[k];
    if (mode < 2) c.put(0, k, (float)acc);
    else c.line(0, k) = acc;
  }
  cy.v[0] = round_tail(c, acc);
  if (c.lb) {
    const double Y[1] = {cy.v[0]};
    lb_publish<1>(c.lbd + j.lb_slot, c.lbs, c.tile, Y, c.lane);
  }
  if (mode == 2) {
    const int fp_ = j.ip[0], sp_ = j.ip[1];
    const int warm = (fp_ > sp_ ? fp_ : sp_) - 1;
    struct Osc {
      double kk;
      __device__ __forceinline__ void coef(int t, double& a, double& w) const {
        if (t == 0) { a = 0.0; w = 1.0; } else { a = 1.0 - kk; w = kk; }
      }
      __device__ __forceinline__ double expect(int) const { return 1.0; }
      __device__ __forceinline__ int steady_from() const { return 1; }
      __device__ __forceinline__ double step(int t, double y, double ad) const {
        return t == 0 ? ad : kk * ad + (1.0 - kk) * y;
      }
    };
    const Osc fs{2.0 / (fp_ + 1.0)}, ss{2.0 / (sp_ + 1.0)};
    cy.v[1] = stage_round(c, 0, fs, cy.v[1], [&](int, int k) { return c.line(0, k); },
                          [&](int k, int, double y) { c.line(1, k) = y; }, j.lb_slot + 1);
    cy.v[2] = stage_round(c, 0, ss, cy.v[2], [&](int, int k) { return c.line(0, k); },
                          [&](int k, int t, double y) {
                            c.put(0, k, t >= warm ? (float)(c.line(1, k) - y) : qnan());
                          },
                          j.lb_slot + 2);
  }
  c.flush(0, (float*)j.out[0]);
}

// ----------------------------------------------------------------- windows

// Lane-local sliding windows over the staged halo: the first window of the lane
// is summed directly, later ones slide. NaN inputs only poison the windows that
// contain them (src/api/BatchFused.cu:73-143 sums every window directly);
// FP64 sums of float32 values are exact, so sliding equals direct summation.

// SMA(p) (talib08:14748-14812), SUM(p) (BatchFused.cu:133-138), WMA(p)
// (talib08:19171-19277, weights 1..p over the divider p(p+1)/2).
// mode: 0 SMA, 1 SUM, 2 WMA.
template <int K>
__device__ __forceinline__ void sum_window_round(const Ctx<K>& c, const Job& j, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  const int g0 = c.gb0();
  const int tf = g0 > p - 1 ? g0 : (int)(p - 1);
  double s = 0.0, w = 0.0;
  int nn = 0;
  if (tf < g0 + K && c.valid(tf)) {
    for (int i = 0; i < p; ++i) {
      const float v = c.x(pl, tf - p + 1 + i);
      if (isnan(v)) ++nn;
      else { s += (double)v; w += (double)v * (double)(i + 1); }
    }
  }
  const double divider = (double)p * (p + 1) / 2.0;
  // constant divisors as reciprocals: one FP64 multiply per bar instead of a
  // division (within an ulp of FP64, far below the float outputs' rounding)
  const double inv_p = 1.0 / (double)p, inv_div = 1.0 / divider;
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= tf) {
      if (t > tf) {
        const float vin = c.x(pl, t), vout = c.x(pl, t - p);
        if (mode == 2) w -= s;  // weights shift down by one (NaN-free part)
        if (isnan(vout)) --nn; else s -= (double)vout;
        if (isnan(vin)) ++nn;
        else { s += (double)vin; if (mode == 2) w += (double)vin * (double)p; }
      }
      if (nn == 0) {
        if (mode == 0) o = (float)(s * inv_p);
        else if (mode == 1) o = (float)s;
        else o = p == 1 ? c.x(pl, t) : (float)(w * inv_div);
      }
    }
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// BBANDS(p, up, dn) with an SMA middle band (talib08:2068-2283), STDDEV(p, nb)
// (talib08:16046-16100) and VAR(p) (talib08:18047-18183): population variance
// of the window from FP64 moments of x - o about a lane-local origin o (the
// sums are then exact), clamped at zero as the reference's batch path does.
// The middle band is the exact window sum divided by p, as TA-Lib's.
// mode: 0 BBANDS, 1 STDDEV, 2 VAR.
template <int K>
__device__ __forceinline__ void moment_window_round(const Ctx<K>& c, const Job& j, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  const int g0 = c.gb0();
  const int tf = g0 > p - 1 ? g0 : (int)(p - 1);
  double raw = 0.0, s2 = 0.0, o = 0.0;
  int nn = 0;
  if (tf < g0 + K && c.valid(tf)) {
    const float ov = c.x(pl, tf);
    o = isnan(ov) ? 0.0 : (double)ov;
    for (int i = 0; i < p; ++i) {
      const float v = c.x(pl, tf - p + 1 + i);
      if (isnan(v)) ++nn;
      else { raw += (double)v; const double d = (double)v - o; s2 += d * d; }
    }
  }
  const double inv = 1.0 / (double)p, po = (double)p * o;
  const double up = j.fp[0], dn = j.fp[1];
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o0 = qnan(), o1 = qnan(), o2 = qnan();
    if (t >= tf) {
      if (t > tf) {
        const float vin = c.x(pl, t), vout = c.x(pl, t - p);
        if (isnan(vout)) --nn;
        else { raw -= (double)vout; const double d = (double)vout - o; s2 -= d * d; }
        if (isnan(vin)) ++nn;
        else { raw += (double)vin; const double d = (double)vin - o; s2 += d * d; }
      }
      if (nn == 0) {
        const double m1 = (raw - po) * inv;
        double var = s2 * inv - m1 * m1;
        if (!(var > 0.0)) var = 0.0;
        if (mode == 2) o0 = (float)var;
        else {
          const double sd = var != 0.0 ? sqrt(var) : 0.0;
          if (mode == 1) o0 = (float)(up != 1.0 ? sd * up : sd);
          else {
            const double mid = raw * inv;
            if (up == dn) { const double dv = sd * up; o0 = (float)(mid + dv); o2 = (float)(mid - dv); }
            else { o0 = (float)fma(sd, up, mid); o2 = (float)(mid - sd * dn); }
            o1 = (float)mid;
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

// LINEARREG(p): talib08:9087-9197 TA_LINEARREG: least-squares line of the
// window evaluated at its last bar, fma(m, p-1, b). Sums are taken about a
// lane-local origin o (LINEARREG(o + d) = o + LINEARREG(d)) and slide as
// TA-Lib's: SumXY += SumY - p*y_out, SumY += y_in - y_out.
template <int K>
__device__ __forceinline__ void linreg_round(const Ctx<K>& c, const Job& j) {
  const int pl = j.in[0], p = j.ip[0];
  const int g0 = c.gb0();
  const int tf = g0 > p - 1 ? g0 : (int)(p - 1);
  const double sumX = (double)p * (p - 1) * 0.5;
  const double sumXSqr = (double)p * (p - 1) * (2 * p - 1) / 6.0;
  const double divisor = sumX * sumX - p * sumXSqr;
  const double inv_divisor = 1.0 / divisor, inv_p = 1.0 / (double)p;
  double sy = 0.0, sxy = 0.0, o = 0.0;
  int nn = 0;
  if (tf < g0 + K && c.valid(tf)) {
    const float ov = c.x(pl, tf);
    o = isnan(ov) ? 0.0 : (double)ov;
    for (int i = p - 1; i >= 0; --i) {
      const float v = c.x(pl, tf - i);
      if (isnan(v)) ++nn;
      else { const double d = (double)v - o; sy += d; sxy += (double)i * d; }
    }
  }
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float out = qnan();
    if (t >= tf) {
      if (t > tf) {
        const float vout = c.x(pl, t - p), vin = c.x(pl, t);
        const double dout = isnan(vout) ? 0.0 : (double)vout - o;
        const double din = isnan(vin) ? 0.0 : (double)vin - o;
        sxy = sxy + sy - (double)p * dout;
        sy = sy - dout + din;
        nn += (isnan(vin) ? 1 : 0) - (isnan(vout) ? 1 : 0);
      }
      if (nn == 0) {
        const double m = (p * sxy - sumX * sy) * inv_divisor;
        const double b = (sy - m * sumX) * inv_p;
        out = (float)(o + fma(m, (double)(p - 1), b));
      }
    }
    c.put(0, k, out);
  }
  c.flush(0, (float*)j.out[0]);
}

// Extremes of the lane's K windows [t-p+1, t], t = g0 .. g0+K-1, for p-1 >= K
// (van Herk / Gil-Werman): a suffix sweep over the p-1 bars before g0 keeps
// the extreme of [g0-p+1+k, g0-1] for each k, a prefix sweep over the lane's
// bars the extreme of [g0, g0+k]; out[k] combines the two. About 2 + p/K
// comparisons per bar instead of p. Returns whether a NaN was met: callers
// whose NaN rule depends on the comparison order then use the direct window.
template <int K, bool kMax>
__device__ __forceinline__ bool lane_window_ext(const Ctx<K>& c, int pl, int p, float (&out)[K]) {
  auto op = [](float run, float v) { return kMax ? (v > run ? v : run) : (v < run ? v : run); };
  const int g0 = c.gb0();
  bool nan = false;
  float run = kMax ? -INFINITY : INFINITY;
  for (int i = g0 - 1; i > g0 - p + K; --i) {
    const float v = c.x(pl, i);
    nan |= isnan(v);
    run = op(run, v);
  }
  float suf[K];
#pragma unroll
  for (int k = K - 1; k >= 0; --k) {
    const float v = c.x(pl, g0 - p + 1 + k);
    nan |= isnan(v);
    run = op(run, v);
    suf[k] = run;
  }
  float pre = kMax ? -INFINITY : INFINITY;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const float v = c.x(pl, g0 + k);
    nan |= isnan(v);
    pre = op(pre, v);
    out[k] = op(suf[k], pre);
  }
  return __any_sync(kFull, nan) ? true : false;
}

// Window extrema over [t-p+1, t] of a float plane; fmaxf/fminf ignore NaN.
template <int K>
__device__ __forceinline__ float win_max(const Ctx<K>& c, int pl, int t, int p) {
  float v = c.x(pl, t - p + 1);
  for (int i = 1; i < p; ++i) v = fmaxf(v, c.x(pl, t - p + 1 + i));
  return v;
}
template <int K>
__device__ __forceinline__ float win_min(const Ctx<K>& c, int pl, int t, int p) {
  float v = c.x(pl, t - p + 1);
  for (int i = 1; i < p; ++i) v = fminf(v, c.x(pl, t - p + 1 + i));
  return v;
}

// MIN(p) / MAX(p): BatchFused.cu:110-119 (float extrema; a window reaching
// into the row's leading NaN run stays NaN, LeadingNaN.cuh:21-27).
template <int K>
__device__ __forceinline__ void minmax_round(const Ctx<K>& c, const Job& j, Carry& cy, bool is_max) {
  const int pl = j.in[0], p = j.ip[0];
  const int f = resolve_start(c, cy, pl, j.lb_slot);
  const int g0 = c.gb0();
  float ext[K];
  const bool fast = p - 1 >= K && !(is_max ? lane_window_ext<K, true>(c, pl, p, ext)
                                           : lane_window_ext<K, false>(c, pl, p, ext));
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= p - 1) {
      o = fast ? ext[k] : (is_max ? win_max(c, pl, t, p) : win_min(c, pl, t, p));
      if (f < 0 || t - p + 1 < f) o = qnan();
    }
    c.put(0, k, o);
  }
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
}

// ROC family from bar p, the reference kernels' float arithmetic (NaN inputs
// propagate: NaN != 0), prev = x[t-p]:
//   mode 0 ROC      ((x - prev) / prev) * 100   src/indicators/ROC.cu:10-21
//   mode 1 ROCP     (x - prev) / prev           src/indicators/ROCP.cu:10-20
//   mode 2 ROCR     x / prev                    src/indicators/ROCR.cu:10-20
//   mode 3 ROCR100  (x / prev) * 100            src/indicators/ROCR100.cu:10-21
//   mode 4 MOM      x - prev                    src/indicators/Momentum.cu:10-18
// ROC* give 0 where prev == 0.
__device__ __forceinline__ float roc_value(float curr, float prev, int mode) {
  if (mode == 4) return curr - prev;
  if (!(prev != 0.0f)) return 0.0f;
  switch (mode) {
    case 0: return ((curr - prev) / prev) * 100.0f;
    case 1: return (curr - prev) / prev;
    case 2: return curr / prev;
    default: return (curr / prev) * 100.0f;
  }
}

template <int K>
__device__ __forceinline__ void roc_round(const Ctx<K>& c, const Job& j, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  const int g0 = c.gb0();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= p) {
      o = roc_value(c.x(pl, t), c.x(pl, t - p), mode);
    }
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// Price transforms, float arithmetic in the reference's order, no warm-up:
//   mode 0 MEDPRICE  0.5f * (h + l)             src/indicators/MedPrice.cu:12-14
//   mode 1 TYPPRICE  (h + l + c) / 3.0f         src/indicators/TypPrice.cu:13-15
//   mode 2 AVGPRICE  (o + h + l + c) * 0.25f    src/indicators/AvgPrice.cu:16-18
//   mode 3 WCLPRICE  (h + l + 2.0f * c) * 0.25f src/indicators/WclPrice.cu:14-16
// Inputs in[0..] are (h, l[, c]) for modes 0,1,3 and (o, h, l, c) for mode 2.
template <int K>
__device__ __forceinline__ void price_round(const Ctx<K>& c, const Job& j, int mode) {
  const int p0 = j.in[0], p1 = j.in[1], p2 = j.in[2], p3 = j.in[3];
  const int g0 = c.gb0();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    const float a = c.x(p0, t), b = c.x(p1, t);
    float o;
    if (mode == 0) o = 0.5f * (a + b);
    else if (mode == 1) o = (a + b + c.x(p2, t)) / 3.0f;
    else if (mode == 2) o = (a + b + c.x(p2, t) + c.x(p3, t)) * 0.25f;
    else o = (a + b + 2.0f * c.x(p2, t)) * 0.25f;
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// MIDPRICE(p): src/indicators/MIDPRICE.cu:11-24: fmaxf / fminf over the window
// [t-p+1, t] of high / low (NaN ignored unless the whole window is NaN), then
// 0.5f * (max + min), from bar p-1. Lane sweeps when the warp meets no NaN.
template <int K>
__device__ __forceinline__ void midprice_round(const Ctx<K>& c, const Job& j) {
  const int ph = j.in[0], plo = j.in[1], p = j.ip[0];
  const int g0 = c.gb0();
  float his[K], los[K];
  bool fast = p - 1 >= K;
  if (fast) {
    const bool n1 = lane_window_ext<K, true>(c, ph, p, his);
    const bool n2 = lane_window_ext<K, false>(c, plo, p, los);
    fast = !n1 && !n2;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= p - 1) {
      const float hi = fast ? his[k] : win_max(c, ph, t, p);
      const float lo = fast ? los[k] : win_min(c, plo, t, p);
      o = 0.5f * (hi + lo);
    }
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// AROON / AROONOSC(p) as the reference's float kernels compute them
// (src/indicators/Aroon.cu:11-52, src/indicators/AroonOscillator.cu:12-40):
// from bar t back over p bars, the latest bar holding the window's highest
// high (lowest low), found with strict comparisons seeded with bar t itself
// (so ties keep the most recent bar and NaNs are skipped, a NaN at bar t
// keeping t); up = 100.0f * (p - since) / (float)p, down alike, osc = up -
// down, from bar p. mode 0: AROON (out[0] down, out[1] up); 1: AROONOSC.

template <int K>
__device__ __forceinline__ void aroon_round(const Ctx<K>& c, const Job& j, int mode) {
  const int ph = j.in[0], plo = j.in[1], p = j.ip[0];
  const int g0 = c.gb0();
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float up = qnan(), dn = qnan();
    if (t >= p) {
      float mx = c.x(ph, t), mn = c.x(plo, t);
      int sh = 0, sl = 0;
      for (int d = 1; d <= p; ++d) {
        const float h = c.x(ph, t - d), l = c.x(plo, t - d);
        if (h > mx) { mx = h; sh = d; }
        if (l < mn) { mn = l; sl = d; }
      }
      up = aroon_line(p, sh);
      dn = aroon_line(p, sl);
    }
    if (mode == 0) {
      c.put(0, k, dn);
      c.put(1, k, up);
    } else {
      c.put(0, k, t >= p ? up - dn : qnan());
    }
  }
  c.flush(0, (float*)j.out[0]);
  if (mode == 0) c.flush(1, (float*)j.out[1]);
}

// MIDPOINT(p): src/indicators/MIDPOINT.cu:13-35: fmaxf / fminf over the
// window of one plane, 0.5f * (max + min) from bar p-1; a window starting in
// the row's leading NaN run stays NaN (LeadingNaN.cuh:22-28, as MIN/MAX).
template <int K>
__device__ __forceinline__ void midpoint_round(const Ctx<K>& c, const Job& j, Carry& cy) {
  const int pl = j.in[0], p = j.ip[0];
  const int f = resolve_start(c, cy, pl, j.lb_slot);
  const int g0 = c.gb0();
  float his[K], los[K];
  bool fast = p - 1 >= K;
  if (fast) {
    const bool n1 = lane_window_ext<K, true>(c, pl, p, his);
    const bool n2 = lane_window_ext<K, false>(c, pl, p, los);
    fast = !n1 && !n2;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= p - 1 && f >= 0 && t - p + 1 >= f) {
      const float hi = fast ? his[k] : win_max(c, pl, t, p);
      const float lo = fast ? los[k] : win_min(c, pl, t, p);
      o = 0.5f * (hi + lo);
    }
    c.put(0, k, o);
  }
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
}

// NaN-strict rolling statistics (src/indicators/ClubPack.cu:375-407): a window
// holding a NaN or an infinity gives NaN; otherwise FP64 sums accumulated from
// the newest bar back, in the reference's order. mode 0 mean (sum / p), 1 max,
// 2 min (fmaxf / fminf), 3 population standard deviation
// sqrt(max(0, sq/p - mean^2)). The reference file is compiled with FMA
// contraction on, which fuses sq/p - mean*mean into one fma; this library is
// built without contraction, so the fma is written out.
template <int K>
__device__ __forceinline__ void rolling_round(const Ctx<K>& c, const Job& j, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  const int g0 = c.gb0();
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= p - 1) {
      bool ok = true;
      double sum = 0.0, sq = 0.0;
      float mx = c.x(pl, t), mn = mx;
      for (int i = 0; i < p; ++i) {
        const float v = c.x(pl, t - i);
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
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// Per-bar TA-Lib functions run by the reference's TA-Lib 0.8.3 device runner
// (src/compat/Talib08.cu:72-97): the row starts at the first bar where no input
// is NaN (the last bar when there is none), earlier bars stay NaN; FP64, then
// rounded to float.
//   mode 0 IBS (h, l, c)       talib08 TA_IBS: (c - l) / (h - l), 0.5 where h - l <= 0
//   mode 1 MARKETFI (h, l, v)  talib08 TA_MARKETFI: (h - l) / v, 0 where v == 0
template <int K>
__device__ __forceinline__ void talib_bar_round(const Ctx<K>& c, const Job& j, Carry& cy, int mode) {
  const int p0 = j.in[0], p1 = j.in[1], p2 = j.in[2];
  // first bar of the row with every input present (warp-uniform; look-back
  // mode resolves it across tiles like the single-input start)
  int f;
  if (!c.lb && cy.f >= 0) {
    f = cy.f;
  } else {
    int first = 0x7fffffff;
    for (int k = 0; k < K; ++k) {
      const int t = c.gb0() + k;
      if (c.valid(t) && !isnan(c.x(p0, t)) && !isnan(c.x(p1, t)) && !isnan(c.x(p2, t))) { first = t; break; }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) first = min(first, __shfl_xor_sync(kFull, first, d));
    const int local = first == 0x7fffffff ? -1 : first;
    f = c.lb ? lb_first_index(c.lbd + j.lb_slot, c.lbs, c.tile, local, c.err, c.lane) : local;
  }
  const int g0 = c.gb0();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if ((f >= 0 && t >= f) || (f < 0 && t == c.n - 1)) {
      const double a = c.x(p0, t), b = c.x(p1, t), z = c.x(p2, t);
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
    c.put(0, k, o);
  }
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
}

// QSTICK(p) through the reference's TA-Lib runner (talib08 TA_QSTICK,
// src/compat/Talib08.cu:72-97): from the first bar f where open and close are
// both present, the mean of close - open over the last p bars, from bar
// f + p - 1. TA_QSTICK keeps a running FP64 sum: the first NaN difference g
// at or after f turns every later output NaN, and so does the first infinite
// difference gi once it leaves the window (inf - inf), i.e. from bar gi + p.
// The windows here are summed directly (exact for float32 inputs) and stop at
// min(g, gi + p). Scratch carries: v[0] = g + 1, v[1] = gi + 1 (0 while none
// is known).
template <int K>
__device__ __forceinline__ int qstick_first(const Ctx<K>& c, const Job& j, int f, int g0, bool inf, int slot,
                                            double& carry) {
  const int po = j.in[0], pc = j.in[1];
  if (!c.lb && carry > 0.0) return (int)carry - 1;
  int first = 0x7fffffff;
  if (f >= 0) {
    for (int k = 0; k < K; ++k) {
      const int t = g0 + k;
      if (!c.valid(t) || t < f) continue;
      const double d = (double)c.x(pc, t) - (double)c.x(po, t);
      if (inf ? isinf(d) : isnan(d)) { first = t; break; }
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) first = min(first, __shfl_xor_sync(kFull, first, d));
  const int local = first == 0x7fffffff ? -1 : first;
  const int v = c.lb ? lb_first_index(c.lbd + j.lb_slot + slot, c.lbs, c.tile, local, c.err, c.lane) : local;
  carry = v >= 0 ? (double)v + 1.0 : 0.0;
  return v;
}

template <int K>
__device__ __forceinline__ void qstick_round(const Ctx<K>& c, const Job& j, Carry& cy) {
  const int po = j.in[0], pc = j.in[1], p = j.ip[0];
  const int g0 = c.gb0();
  int f;
  if (!c.lb && cy.f >= 0) {
    f = cy.f;
  } else {
    int first = 0x7fffffff;
    for (int k = 0; k < K; ++k) {
      const int t = g0 + k;
      if (c.valid(t) && !isnan(c.x(po, t)) && !isnan(c.x(pc, t))) { first = t; break; }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) first = min(first, __shfl_xor_sync(kFull, first, d));
    const int local = first == 0x7fffffff ? -1 : first;
    f = c.lb ? lb_first_index(c.lbd + j.lb_slot, c.lbs, c.tile, local, c.err, c.lane) : local;
  }
  const int g = qstick_first(c, j, f, g0, false, 1, cy.v[0]);
  const int gi = qstick_first(c, j, f, g0, true, 2, cy.v[1]);
  const int stop = g < 0 ? (gi < 0 ? 0x7fffffff : gi + p) : (gi < 0 ? g : min(g, gi + p));
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (f >= 0 && t >= f + p - 1 && t < stop) {
      double s = 0.0;
      for (int i = t - p + 1; i <= t; ++i) s += (double)c.x(pc, i) - (double)c.x(po, i);
      o = (float)(s / (double)p);
    }
    c.put(0, k, o);
  }
  cy.f = f;
  c.flush(0, (float*)j.out[0]);
}

// WILLR(p): src/indicators/WILLR.cu:11-30: float window extrema (strict
// comparisons seeded with the current bar), ((HH - C)/(HH - LL)) * -100 in
// FP64, clamped to [-100, 0]; 0 for a zero range.
template <int K>
__device__ __forceinline__ void willr_round(const Ctx<K>& c, const Job& j) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0];
  const int g0 = c.gb0();
  float his[K], los[K];
  bool fast = p - 1 >= K;
  if (fast) {
    const bool n1 = lane_window_ext<K, true>(c, ph, p, his);
    const bool n2 = lane_window_ext<K, false>(c, plo, p, los);
    fast = !n1 && !n2;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= p - 1) {
      float hi = his[k], lo = los[k];
      if (!fast) {
        hi = c.x(ph, t);
        lo = c.x(plo, t);
        for (int i = 1; i < p; ++i) {
          const float h = c.x(ph, t - i), l = c.x(plo, t - i);
          if (h > hi) hi = h;
          if (l < lo) lo = l;
        }
      }
      const double den = (double)hi - (double)lo;
      const double v = den == 0.0 ? 0.0 : (((double)hi - (double)c.x(pc, t)) / den) * -100.0;
      o = isnan(v) ? qnan() : (float)fmin(0.0, fmax(-100.0, v));
    }
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// STOCH(k, d) with SMA slowing (talib08:16115-16302): fastK from window
// extrema with TA-Lib's scaled zero-range test, slowK = SMA_d(fastK),
// slowD = SMA_d(slowK), both from bar k-1+2(d-1). fastK of the round and of the
// 2(d-1) bars before it goes to scratch line 0, then each bar averages it.
template <int K>
__device__ __forceinline__ void stoch_round(const Ctx<K>& c, const Job& j) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2];
  const int p = j.ip[0], q = j.ip[1];
  const int lb = (int)p - 1 + 2ll * (q - 1);
  const int ext = 2 * (q - 1);
  auto fastk = [&](int t) -> double {
    if (t < p - 1) return 0.0;
    double lo = c.x(plo, t - p + 1), hi = c.x(ph, t - p + 1);
    for (int i = 1; i < p; ++i) {
      const double l = c.x(plo, t - p + 1 + i), h = c.x(ph, t - p + 1 + i);
      if (l < lo) lo = l;
      if (h > hi) hi = h;
    }
    const double range = hi - lo;
    return fabs(range) <= 1e-14 * (fabs(hi) + fabs(lo)) ? 0.0 : ((double)c.x(pc, t) - lo) / range * 100.0;
  };
  const int g0 = c.gb0();
  float his[K], los[K];
  bool fast = p - 1 >= K;
  if (fast) {
    const bool n1 = lane_window_ext<K, true>(c, ph, p, his);
    const bool n2 = lane_window_ext<K, false>(c, plo, p, los);
    fast = !n1 && !n2;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    double v;
    if (!fast || t < p - 1) {
      v = fastk(t);
    } else {
      const double lo = los[k], hi = his[k];
      const double range = hi - lo;
      v = fabs(range) <= 1e-14 * (fabs(hi) + fabs(lo)) ? 0.0 : ((double)c.x(pc, t) - lo) / range * 100.0;
    }
    c.line(0, k) = v;
  }
  for (int i = c.lane; i < ext; i += 32) c.eline(0, i - ext) = fastk(c.t0 - ext + i);
  __syncwarp();
  const double invq = 1.0 / (double)q;
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o0 = qnan(), o1 = qnan();
    if (t >= lb) {
      const int r = (int)(t - c.t0);
      double dsum = 0.0, k0 = 0.0;
      for (int i = 0; i < q; ++i) {
        double s = 0.0;
        for (int m = q - 1; m >= 0; --m) s += c.eline(0, r - i - m);
        const double kv = s * invq;
        if (i == 0) k0 = kv;
        dsum += kv;
      }
      o0 = (float)k0;
      o1 = (float)(dsum * invq);
    }
    c.put(0, k, o0);
    c.put(1, k, o1);
  }
  c.flush(0, (float*)j.out[0]);
  c.flush(1, (float*)j.out[1]);
}

// CCI(p): src/indicators/CCI.cu:11-40, in its arithmetic: typical price
// ((h+l)+c)/3.0 in FP64, sma = direct window sum / p, md = deviation sum / p
// (both summed from the newest bar back), (tp - sma)/(0.015*md) in FP64, 0
// unless both the numerator and md are nonzero.
template <int K>
__device__ __forceinline__ void cci_round(const Ctx<K>& c, const Job& j) {
  const int p = j.ip[0];
  const int g0 = c.gb0();
  const double dp = (double)p;
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= p - 1) {
      double sum = 0.0;
      for (int i = 0; i < p; ++i) sum += c.typ(t - i);
      const double sma = sum / dp;
      double dev = 0.0;
      for (int i = 0; i < p; ++i) dev += fabs(c.typ(t - i) - sma);
      const double md = dev / dp;
      const double num = c.typ(t) - sma;
      o = (num != 0.0 && md != 0.0) ? (float)(num / (0.015 * md)) : 0.0f;
    }
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// MFI(p): StreamStates.h:749-792 precise::MfiState: money flow tp*v signed by
// the typical price change (non-finite prices give no flow), positive and
// negative sums over the last p flows, 100*pos/(pos+neg), 0 when the total is
// below 1; output from bar p.
template <int K>
__device__ __forceinline__ void mfi_round(const Ctx<K>& c, const Job& j) {
  const int pv = j.in[3], p = j.ip[0];
  const int g0 = c.gb0();
  auto flow = [&](int t, double& pos, double& neg) {
    pos = neg = 0.0;
    if (t < 1) return;
    const double pr = c.typ(t), pp = c.typ(t - 1);
    if (isfinite(pr) && isfinite(pp)) {
      const double fl = pr * (double)c.x(pv, t);
      if (pr > pp) pos = fl;
      else if (pr < pp) neg = fl;
    }
  };
  const int tf = g0 > p ? g0 : (int)p;
  double ps = 0.0, ns = 0.0;
  if (tf < g0 + K && c.valid(tf)) {
    for (int i = p - 1; i >= 0; --i) {
      double a, b;
      flow(tf - i, a, b);
      ps += a; ns += b;
    }
  }
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= tf) {
      if (t > tf) {
        double a, b;
        flow(t - p, a, b);
        ps -= a; ns -= b;
        flow(t, a, b);
        ps += a; ns += b;
        if (ps < 0.0 || ns < 0.0) {  // re-sum a window that cancelled below zero
          ps = ns = 0.0;
          for (int i = p - 1; i >= 0; --i) { flow(t - i, a, b); ps += a; ns += b; }
        }
      }
      const double tot = ps + ns;
      o = tot < 1.0 ? 0.0f : (float)(100.0 * (ps / tot));
    }
    c.put(0, k, o);
  }
  c.flush(0, (float*)j.out[0]);
}

// CORREL(p): src/indicators/Correl.cu:23-75: Pearson correlation of the window
// from FP64 moments about a lane-local origin; 0 when either variance or their
// product (<= 1e-14) vanishes; 0 from the first non-finite bar of the row on
// (findInvalidSuffix, Correl.cu:14-21). Carry.f holds that first bar (-1 none).
template <int K>
__device__ __forceinline__ void correl_round(const Ctx<K>& c, const Job& j, Carry& cy) {
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
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) first = min(first, __shfl_xor_sync(kFull, first, d));
    bad = first == 0x7fffffff ? -1 : first;
    if (c.lb) bad = lb_first_index(c.lbd + j.lb_slot, c.lbs, c.tile, bad, c.err, c.lane);
  }
  const int tf = g0 > p - 1 ? g0 : (int)(p - 1);
  double sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0, ox = 0, oy = 0;
  if (tf < g0 + K && c.valid(tf)) {
    ox = c.x(px, tf - p + 1);
    oy = c.x(py, tf - p + 1);
    if (!isfinite(ox)) ox = 0.0;
    if (!isfinite(oy)) oy = 0.0;
    for (int i = 0; i < p; ++i) {
      const double dx = (double)c.x(px, tf - p + 1 + i) - ox, dy = (double)c.x(py, tf - p + 1 + i) - oy;
      sx += dx; sy += dy; sxx += dx * dx; syy += dy * dy; sxy += dx * dy;
    }
  }
  const double inv_pp = 1.0 / (double)p;
  for (int k = 0; k < K; ++k) {
    const int t = g0 + k;
    if (!c.valid(t)) break;
    float o = qnan();
    if (t >= tf) {
      if (t > tf) {
        const double ax = (double)c.x(px, t - p) - ox, ay = (double)c.x(py, t - p) - oy;
        const double bx = (double)c.x(px, t) - ox, by = (double)c.x(py, t) - oy;
        sx += bx - ax; sy += by - ay;
        sxx += bx * bx - ax * ax; syy += by * by - ay * ay; sxy += bx * by - ax * ay;
      }
      if (bad >= 0 && t >= bad) o = 0.0f;
      else {
        const double cov = sxy - sx * sy * inv_pp;
        const double vx = sxx - sx * sx * inv_pp, vy = syy - sy * sy * inv_pp;
        const double prod = vx * vy;
        o = (vx > 0.0 && vy > 0.0 && prod > 1e-14) ? (float)(cov * rsqrt(prod)) : 0.0f;
      }
    }
    c.put(0, k, o);
  }
  cy.f = bad;
  c.flush(0, (float*)j.out[0]);
}

}  // namespace tb
