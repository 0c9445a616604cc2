// Differentiable EMA / MACD / RSI with a per-series smoothing coefficient
// alpha, and their hand-written adjoint.
//
// Forward (TA-Lib's structure with alpha in place of the recurrence
// coefficient; periods fix the lookback and the seeds):
//   EMA(p):  mean of x[0..p-1] at bar p-1, then y = fma(1-a, y, a*x)
//            (talib08 TA_EMA; a = 2/(p+1) gives TA_EMA's coefficients).
//   MACD(fast, slow, signal): slow EMA with TA-Lib's 2/(slow+1); fast EMA
//            seeded with the mean of the `fast` bars ending at slow-1 and then
//            alpha (talib08 TA_MACD with alpha for the fast line); the signal
//            line over the MACD values with TA-Lib's 2/(signal+1).
//   RSI(p):  gains / losses of the first p changes summed and multiplied by
//            1/p, then g = fma(1-a, g, a*gain) (TA_RSI's Wilder step with a =
//            1/p); 100*g/(g+l), 50 when both are zero.
// The state entering every 256-bar segment (6 FP64 values: EMA, slow, fast,
// signal, gain, loss) is written as a checkpoint; no per-bar state is kept.
//
// Adjoint of L = sum_t (w_ema*EMA + w_macd*MACD + w_sig*SIGNAL + w_hist*HIST
// + w_rsi*RSI): a reverse-time affine recurrence per stage,
//   lambda_t = dL/dout_t + a(t+1) * lambda_{t+1},
// with dL/dx_t += w(t) * lambda_t through each stage's input coefficient and
// dL/dalpha += lambda_t * (x_t - y_{t-1}) over the stage's steady bars. The
// signal stage feeds dL/dMACD, which feeds the fast (+) and slow (-) lines;
// the RSI channels feed dL/dgain and dL/dloss, then dL/dx through the
// bar-to-bar change.
//
// Both passes split every series into 256-bar pieces over several lanes of a
// warp and join the lanes with segmented affine scans (see the layout note
// below). The adjoint recomputes the forward quantities of 32-bar sub-blocks
// from the checkpoints into shared memory and consumes them in reverse.
#include "adjoint.h"
#include "pool.h"
#include "families.cuh"

namespace tb {

namespace {

constexpr int kSeg = kAlphaSegment;
constexpr int kQ = 6;  // per-bar quantities kept for the reverse walk

struct Stages {
  EmaStage E, Sl, F;
  SigStage G;
  int rp, ready, slow;
  double a, b, rinv;
};

__device__ __forceinline__ Stages make_stages(const AlphaParams& P, double a) {
  double bs, ks, bg, kg;
  talib_ema_coeffs(P.slow, bs, ks);
  talib_ema_coeffs(P.signal, bg, kg);
  Stages s;
  s.a = a;
  s.b = 1.0 - a;
  s.E = EmaStage{P.ema_period, 0, s.b, a, 1.0 / P.ema_period};
  s.Sl = EmaStage{P.slow, 0, bs, ks, 1.0 / P.slow};
  s.F = EmaStage{P.fast, P.slow - P.fast, s.b, a, 1.0 / P.fast};
  s.G = SigStage{P.signal, P.slow - 1, P.slow + P.signal - 2, bg, kg, 1.0 / P.signal};
  s.rp = P.rsi_period;
  s.ready = P.slow + P.signal - 2;
  s.slow = P.slow;
  s.rinv = 1.0 / P.rsi_period;
  return s;
}

struct State {
  double e, sl, f, g, rg, rl;
};

// Per-bar forward quantities the reverse walk consumes.
struct BarQ {
  double eE;  // x_t - EMA_{t-1}
  double eF;  // x_t - fast_{t-1}
  double cG;  // d RSI_t / d gain_t
  double cL;  // d RSI_t / d loss_t
  double eG;  // gain change_t - gain_{t-1}
  double eL;  // loss change_t - loss_{t-1}
};

// One forward bar: advances the state and returns the outputs and the
// quantities of the bar. xprev is x_{t-1} (unused at t = 0).
struct BarOut {
  double ema, macd, sig, rsi;
  bool ema_ok, macd_ok, rsi_ok;
};

template <bool kGrad>
__device__ __forceinline__ BarOut step(const Stages& s, int t, double x, double xprev, State& st, BarQ& q) {
  BarOut o;
  q.eE = x - st.e;
  q.eF = x - st.f;
  st.e = s.E.step(t, st.e, x);
  st.sl = s.Sl.step(t, st.sl, x);
  st.f = s.F.step(t, st.f, x);
  const double m = t >= s.slow - 1 ? st.f - st.sl : 0.0;
  st.g = s.G.step(t, st.g, m);
  o.ema = st.e;
  o.ema_ok = s.E.ready(t);
  o.macd = m;
  o.sig = st.g;
  o.macd_ok = t >= s.ready;
  // RSI
  double u = 0.0, v = 0.0;
  if (t >= 1) {
    const double d = x - xprev;
    u = d > 0.0 ? d : 0.0;
    v = u - d;
  }
  q.eG = u - st.rg;
  q.eL = v - st.rl;
  if (t >= 1) {
    if (t < s.rp) { st.rg += u; st.rl += v; }
    else if (t == s.rp) { st.rg = (st.rg + u) * s.rinv; st.rl = (st.rl + v) * s.rinv; }
    else { st.rg = fma(s.b, st.rg, s.a * u); st.rl = fma(s.b, st.rl, s.a * v); }
  }
  o.rsi_ok = t >= s.rp;
  q.cG = q.cL = 0.0;
  o.rsi = 50.0;
  if (o.rsi_ok) {
    const double tot = st.rg + st.rl;
    if (tot > 0.0) {
      if (kGrad) {
        const double inv2 = 100.0 / (tot * tot);
        q.cG = st.rl * inv2;
        q.cL = -st.rg * inv2;
      } else {
        o.rsi = 100.0 * (st.rg / tot);
      }
    }
  }
  return o;
}

// RSI channel coefficients of bar t: y_t = a*y_{t-1} + w*change_t.
__device__ __forceinline__ void rsi_coef(const Stages& s, int t, double& a, double& w) {
  if (t < 1) { a = 1.0; w = 0.0; }
  else if (t < s.rp) { a = 1.0; w = 1.0; }
  else if (t == s.rp) { a = s.rinv; w = s.rinv; }
  else { a = s.b; w = s.a; }
}

// ---------------------------------------------------------------- layout
//
// A series is cut into 256-bar pieces (the checkpoint interval). G lanes of a
// warp work on one series (G = the next power of two >= pieces, at most 32),
// lane li on pieces [li*ppl, (li+1)*ppl). Recurrences cross lanes through
// segmented warp scans of affine maps: inclusive with __shfl_up (forward in
// time) for the forward pass, with __shfl_down (backward in time) for the
// adjoint. A warp holds 32/G series.

struct SegLane {
  int sid, li, t0, t1, p0, p1;
  bool live;
};

__device__ __forceinline__ SegLane seg_lane(const AlphaLaunch& L, int G, int ppl) {
  SegLane g;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int sidx = gw * (32 / G) + lane / G;
  g.live = sidx < L.S;
  g.sid = g.live ? sidx : 0;
  g.li = lane % G;
  const int nseg = (L.T + kSeg - 1) / kSeg;
  g.p0 = min(nseg, g.li * ppl);
  g.p1 = min(nseg, (g.li + 1) * ppl);
  if (!g.live) g.p1 = g.p0;
  g.t0 = min(L.T, g.p0 * kSeg);
  g.t1 = min(L.T, g.p1 * kSeg);
  return g;
}

// Segmented inclusive scans of maps y -> A*y + B (NC channels sharing A).
template <int NC>
__device__ __forceinline__ void scan_up(double& A, double (&B)[NC], int li, int G) {
  for (int d = 1; d < G; d <<= 1) {
    const double pA = __shfl_up_sync(kFull, A, d, G);
    double pB[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) pB[c] = __shfl_up_sync(kFull, B[c], d, G);
    if (li >= d) {
#pragma unroll
      for (int c = 0; c < NC; ++c) B[c] = fma(A, pB[c], B[c]);
      A *= pA;
    }
  }
}
template <int NC>
__device__ __forceinline__ void scan_down(double& A, double (&B)[NC], int li, int G) {
  for (int d = 1; d < G; d <<= 1) {
    const double nA = __shfl_down_sync(kFull, A, d, G);
    double nB[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) nB[c] = __shfl_down_sync(kFull, B[c], d, G);
    if (li + d < G) {
#pragma unroll
      for (int c = 0; c < NC; ++c) B[c] = fma(A, nB[c], B[c]);
      A *= nA;
    }
  }
}

// Coefficient a(t) of each stage (the multiplier of the previous state).
__device__ __forceinline__ double coef_a(const EmaStage& st, int t) {
  double a, w;
  st.coef(t, a, w);
  return a;
}
__device__ __forceinline__ double coef_a(const SigStage& st, int t) {
  double a, w;
  st.coef(t, a, w);
  return a;
}

__device__ __forceinline__ void rsi_moves(int t, double x, double xprev, double& u, double& v) {
  u = v = 0.0;
  if (t >= 1) {
    const double d = x - xprev;
    u = d > 0.0 ? d : 0.0;
    v = u - d;
  }
}

__device__ __forceinline__ void rsi_step(const Stages& s, int t, double u, double v, double& g, double& l) {
  if (t < 1) return;
  if (t < s.rp) { g += u; l += v; }
  else if (t == s.rp) { g = (g + u) * s.rinv; l = (l + v) * s.rinv; }
  else { g = fma(s.b, g, s.a * u); l = fma(s.b, l, s.a * v); }
}

__global__ void __launch_bounds__(128) alpha_forward_kernel(AlphaLaunch L, int G, int ppl) {
  const SegLane g = seg_lane(L, G, ppl);
  const Stages s = make_stages(L.P, g.live ? (double)L.alpha[g.sid] : 0.5);
  const long long base = (long long)g.sid * L.T;
  const int nseg = (L.T + kSeg - 1) / kSeg;
  double* ck = L.ckpt + (long long)g.sid * nseg * 6;
  const float nan = qnan();
  // pass 1: maps of the EMA, slow, fast and RSI stages over the lane's bars
  double AE = 1.0, BE[1] = {0.0}, AS = 1.0, BS[1] = {0.0}, AF = 1.0, BF[1] = {0.0}, AR = 1.0, BR[2] = {0.0, 0.0};
  double xprev = g.t0 > 0 ? (double)L.x[base + g.t0 - 1] : 0.0;
  for (int t = g.t0; t < g.t1; ++t) {
    const double x = L.x[base + t];
    double a, w;
    s.E.coef(t, a, w);  BE[0] = fma(a, BE[0], w * x); AE *= a;
    s.Sl.coef(t, a, w); BS[0] = fma(a, BS[0], w * x); AS *= a;
    s.F.coef(t, a, w);  BF[0] = fma(a, BF[0], w * x); AF *= a;
    double u, v;
    rsi_moves(t, x, xprev, u, v);
    rsi_coef(s, t, a, w);
    BR[0] = fma(a, BR[0], w * u);
    BR[1] = fma(a, BR[1], w * v);
    AR *= a;
    xprev = x;
  }
  scan_up<1>(AE, BE, g.li, G);
  scan_up<1>(AS, BS, g.li, G);
  scan_up<1>(AF, BF, g.li, G);
  scan_up<2>(AR, BR, g.li, G);
  // every stage starts the series from state 0: the incoming state is the
  // exclusive prefix's offset
  State st;
  st.e = __shfl_up_sync(kFull, BE[0], 1, G);
  st.sl = __shfl_up_sync(kFull, BS[0], 1, G);
  st.f = __shfl_up_sync(kFull, BF[0], 1, G);
  st.rg = __shfl_up_sync(kFull, BR[0], 1, G);
  st.rl = __shfl_up_sync(kFull, BR[1], 1, G);
  if (g.li == 0) st.e = st.sl = st.f = st.rg = st.rl = 0.0;
  const State in = st;
  // pass 2: replay EMA and RSI (outputs), compose the signal stage
  double AG = 1.0, BG[1] = {0.0};
  xprev = g.t0 > 0 ? (double)L.x[base + g.t0 - 1] : 0.0;
  for (int t = g.t0; t < g.t1; ++t) {
    if (t % kSeg == 0) {
      double* c = ck + (t / kSeg) * 6;
      c[0] = st.e; c[4] = st.rg; c[5] = st.rl;
    }
    const double x = L.x[base + t];
    st.e = s.E.step(t, st.e, x);
    st.sl = s.Sl.step(t, st.sl, x);
    st.f = s.F.step(t, st.f, x);
    const double m = t >= s.slow - 1 ? st.f - st.sl : 0.0;
    double a, w;
    s.G.coef(t, a, w);
    BG[0] = fma(a, BG[0], w * m);
    AG *= a;
    double u, v;
    rsi_moves(t, x, xprev, u, v);
    rsi_step(s, t, u, v, st.rg, st.rl);
    xprev = x;
    if (L.ema) L.ema[base + t] = s.E.ready(t) ? (float)st.e : nan;
    if (L.rsi) {
      float o = nan;
      if (t >= s.rp) {
        const double tot = st.rg + st.rl;
        o = tot > 0.0 ? (float)(100.0 * (st.rg / tot)) : 50.0f;
      }
      L.rsi[base + t] = o;
    }
  }
  scan_up<1>(AG, BG, g.li, G);
  double sig = __shfl_up_sync(kFull, BG[0], 1, G);
  if (g.li == 0) sig = 0.0;
  // pass 3: replay the MACD lines (outputs), checkpoint the slow, fast, signal states
  st.sl = in.sl;
  st.f = in.f;
  st.g = sig;
  for (int t = g.t0; t < g.t1; ++t) {
    if (t % kSeg == 0) {
      double* c = ck + (t / kSeg) * 6;
      c[1] = st.sl; c[2] = st.f; c[3] = st.g;
    }
    const double x = L.x[base + t];
    st.sl = s.Sl.step(t, st.sl, x);
    st.f = s.F.step(t, st.f, x);
    const double m = t >= s.slow - 1 ? st.f - st.sl : 0.0;
    st.g = s.G.step(t, st.g, m);
    const bool ok = t >= s.ready;
    if (L.macd) L.macd[base + t] = ok ? (float)m : nan;
    if (L.sig) L.sig[base + t] = ok ? (float)st.g : nan;
    if (L.hist) L.hist[base + t] = ok ? (float)(m - st.g) : nan;
  }
}

// ---------------------------------------------------------------- adjoint

constexpr int kSub = 16;                 // bars per recomputed sub-block
constexpr int kSubs = kSeg / kSub;       // sub-blocks per piece
constexpr int kAdjWarps = 4;             // warps per block of the adjoint kernel

struct AdjSmem {
  float q[kSub][kQ][32];    // per-bar forward quantities of the current sub-block
};

__device__ __forceinline__ double wv(const float* w, long long i) { return w ? (double)w[i] : 0.0; }

// Walk the lane's bars backwards, sub-block by sub-block, recomputing each
// sub-block's forward quantities from the state saved at its start (sub
// checkpoints written by the adjoint's first phase). body(t, q) is called for
// t = t1-1 down to t0 with q the bar's quantities.
template <class Body>
__device__ __forceinline__ void reverse_walk(const AlphaLaunch& L, const Stages& s, const SegLane& g,
                                             long long base, const double* sub, AdjSmem& sm, Body body) {
  const int lane = threadIdx.x & 31;
  for (int b0 = ((g.t1 - 1) / kSub) * kSub; b0 >= g.t0 && g.t1 > g.t0; b0 -= kSub) {
    const int b1 = min(g.t1, b0 + kSub);
    const double* c = sub + (long long)(b0 / kSub) * 6;
    State st{c[0], c[1], c[2], c[3], c[4], c[5]};
    double xp = b0 > 0 ? (double)L.x[base + b0 - 1] : 0.0;
    for (int t = b0; t < b1; ++t) {
      const double x = L.x[base + t];
      BarQ q;
      step<true>(s, t, x, xp, st, q);
      xp = x;
      const int k = t - b0;
      sm.q[k][0][lane] = (float)q.eE; sm.q[k][1][lane] = (float)q.eF; sm.q[k][2][lane] = (float)q.cG;
      sm.q[k][3][lane] = (float)q.cL; sm.q[k][4][lane] = (float)q.eG; sm.q[k][5][lane] = (float)q.eL;
    }
    for (int t = b1 - 1; t >= b0; --t) {
      const int k = t - b0;
      BarQ q;
      q.eE = sm.q[k][0][lane]; q.eF = sm.q[k][1][lane]; q.cG = sm.q[k][2][lane];
      q.cL = sm.q[k][3][lane]; q.eG = sm.q[k][4][lane]; q.eL = sm.q[k][5][lane];
      body(t, q);
    }
  }
}

__global__ void __launch_bounds__(32 * kAdjWarps) alpha_backward_kernel(AlphaLaunch L, int G, int ppl,
                                                                        double* subck) {
  __shared__ AdjSmem smem[kAdjWarps];
  AdjSmem& sm = smem[threadIdx.x >> 5];
  const SegLane g = seg_lane(L, G, ppl);
  const Stages s = make_stages(L.P, g.live ? (double)L.alpha[g.sid] : 0.5);
  const long long base = (long long)g.sid * L.T;
  const int nseg = (L.T + kSeg - 1) / kSeg;
  const double* ck = L.ckpt + (long long)g.sid * nseg * 6;
  // the state entering every kSub-bar sub-block of the series (6 doubles each)
  double* sub = subck + (long long)g.sid * nseg * kSubs * 6;
  // phase 1: lane maps of the reverse recurrences that need no other adjoint:
  // lambda_t = o_t + a(t+1) lambda_{t+1}, composed forwards as
  // lambda_t0 = P * lambda_t1 + sum_t P_t o_t with P_t = prod a(t0+1 .. t)
  double PE = 1.0, BE[1] = {0.0}, PG = 1.0, BG[1] = {0.0}, PR = 1.0, BR[2] = {0.0, 0.0};
  for (int piece = g.p0; piece < g.p1; ++piece) {
    const int pt0 = piece * kSeg, pt1 = min(L.T, pt0 + kSeg);
    State st{ck[piece * 6 + 0], ck[piece * 6 + 1], ck[piece * 6 + 2], ck[piece * 6 + 3], ck[piece * 6 + 4],
             ck[piece * 6 + 5]};
    double xprev = pt0 > 0 ? (double)L.x[base + pt0 - 1] : 0.0;
    for (int t = pt0; t < pt1; ++t) {
      if (t % kSub == 0) {
        double* c = sub + (long long)(t / kSub) * 6;
        c[0] = st.e; c[1] = st.sl; c[2] = st.f; c[3] = st.g; c[4] = st.rg; c[5] = st.rl;
      }
      const long long gi = base + t;
      const double x = L.x[gi];
      BarQ q;
      step<true>(s, t, x, xprev, st, q);
      xprev = x;
      const bool ok = t >= s.ready;
      const double oE = s.E.ready(t) ? wv(L.w_ema, gi) : 0.0;
      const double oG = ok ? wv(L.w_sig, gi) - wv(L.w_hist, gi) : 0.0;
      const double wr = t >= s.rp ? wv(L.w_rsi, gi) : 0.0;
      BE[0] = fma(PE, oE, BE[0]);
      BG[0] = fma(PG, oG, BG[0]);
      BR[0] = fma(PR, wr * q.cG, BR[0]);
      BR[1] = fma(PR, wr * q.cL, BR[1]);
      double a, w;
      PE *= coef_a(s.E, t + 1);
      PG *= coef_a(s.G, t + 1);
      rsi_coef(s, t + 1, a, w);
      PR *= a;
    }
  }
  scan_down<1>(PE, BE, g.li, G);
  scan_down<1>(PG, BG, g.li, G);
  scan_down<2>(PR, BR, g.li, G);
  // adjoints at the next lane's first bar (0 past the series end)
  const bool last = g.li == G - 1;
  double lE = __shfl_down_sync(kFull, BE[0], 1, G), lG = __shfl_down_sync(kFull, BG[0], 1, G);
  double lRG = __shfl_down_sync(kFull, BR[0], 1, G), lRL = __shfl_down_sync(kFull, BR[1], 1, G);
  if (last) lE = lG = lRG = lRL = 0.0;
  double a1, w1;
  rsi_coef(s, g.t1, a1, w1);
  const double cE0 = coef_a(s.E, g.t1) * lE, cG0 = coef_a(s.G, g.t1) * lG;
  const double cRG0 = a1 * lRG, cRL0 = a1 * lRL;
  // phase 2: walk back over the signal adjoint alone (it needs no forward
  // state) to compose the fast and slow lines' maps, which take dL/dMACD
  double AFr = 1.0, BFr[1] = {0.0}, ASr = 1.0, BSr[1] = {0.0};
  {
    double cG = cG0;
    for (int t = g.t1 - 1; t >= g.t0; --t) {
      const long long gi = base + t;
      double a, w;
      const bool ok = t >= s.ready;
      const double wh = ok ? wv(L.w_hist, gi) : 0.0;
      const double lg = (ok ? wv(L.w_sig, gi) - wh : 0.0) + cG;
      s.G.coef(t, a, w);
      const double mu = (ok ? wv(L.w_macd, gi) + wh : 0.0) + w * lg;
      cG = a * lg;
      const double mm = t >= s.slow - 1 ? mu : 0.0;
      const double aF = coef_a(s.F, t + 1), aS = coef_a(s.Sl, t + 1);
      BFr[0] = fma(aF, BFr[0], mm);
      AFr *= aF;
      BSr[0] = fma(aS, BSr[0], -mm);
      ASr *= aS;
    }
  }
  // the change term the lane's first bar owes the previous lane's last bar,
  // from the RSI adjoints at that bar (the suffix scan's inclusive offsets)
  double pend_out = 0.0;
  if (g.t1 > g.t0 && g.t0 >= 1) {
    double a, w;
    rsi_coef(s, g.t0, a, w);
    const double d = (double)L.x[base + g.t0] - (double)L.x[base + g.t0 - 1];
    pend_out = d > 0.0 ? -(w * BR[0]) : (d < 0.0 ? w * BR[1] : 0.0);
  }
  scan_down<1>(AFr, BFr, g.li, G);
  scan_down<1>(ASr, BSr, g.li, G);
  double lF = __shfl_down_sync(kFull, BFr[0], 1, G), lS = __shfl_down_sync(kFull, BSr[0], 1, G);
  double pend_in = __shfl_down_sync(kFull, pend_out, 1, G);
  if (last) lF = lS = pend_in = 0.0;
  // phase 3: the full reverse walk with every adjoint known at the lane's end
  double cE = cE0, cG = cG0, cRG = cRG0, cRL = cRL0;
  double cF = coef_a(s.F, g.t1) * lF, cS = coef_a(s.Sl, g.t1) * lS;
  double pend = pend_in, dalpha = 0.0;
  reverse_walk(L, s, g, base, sub, sm, [&](int t, const BarQ& q) {
    const long long gi = base + t;
    double a, w, dx = pend;
    const double lE2 = (s.E.ready(t) ? wv(L.w_ema, gi) : 0.0) + cE;
    s.E.coef(t, a, w);
    dx += w * lE2;
    if (t >= s.E.p) dalpha += lE2 * q.eE;
    cE = a * lE2;
    const bool ok = t >= s.ready;
    const double wh = ok ? wv(L.w_hist, gi) : 0.0;
    const double lg = (ok ? wv(L.w_sig, gi) - wh : 0.0) + cG;
    s.G.coef(t, a, w);
    const double mu = (ok ? wv(L.w_macd, gi) + wh : 0.0) + w * lg;
    cG = a * lg;
    const double mm = t >= s.slow - 1 ? mu : 0.0;
    const double lf = mm + cF;
    s.F.coef(t, a, w);
    dx += w * lf;
    if (t >= s.slow) dalpha += lf * q.eF;
    cF = a * lf;
    const double ls = -mm + cS;
    s.Sl.coef(t, a, w);
    dx += w * ls;
    cS = a * ls;
    const double wr = t >= s.rp ? wv(L.w_rsi, gi) : 0.0;
    const double lrg = wr * q.cG + cRG, lrl = wr * q.cL + cRL;
    rsi_coef(s, t, a, w);
    if (t > s.rp) dalpha += lrg * q.eG + lrl * q.eL;
    cRG = a * lrg;
    cRL = a * lrl;
    double dd = 0.0;
    if (t >= 1) {
      const double d = (double)L.x[gi] - (double)L.x[gi - 1];
      if (d > 0.0) dd = w * lrg;
      else if (d < 0.0) dd = -w * lrl;
    }
    dx += dd;
    pend = -dd;
    L.dx[gi] = (float)dx;
  });
  // dL/dalpha: sum over the series' lanes in a fixed tree
  for (int d = 1; d < G; d <<= 1) {
    const double o = __shfl_down_sync(kFull, dalpha, d, G);
    if ((g.li & (2 * d - 1)) == 0 && g.li + d < G) dalpha += o;
  }
  if (g.li == 0 && g.live) L.dalpha[g.sid] = (float)dalpha;
}

void seg_geometry(int T, int& G, int& ppl) {
  const int nseg = (T + kSeg - 1) / kSeg;
  G = 1;
  while (G < nseg && G < 32) G <<= 1;
  ppl = (nseg + G - 1) / G;
}

}  // namespace

cudaError_t alpha_forward(const AlphaLaunch& L, cudaStream_t stream) {
  int G, ppl;
  seg_geometry(L.T, G, ppl);
  const long long lanes = (long long)((L.S + 32 / G - 1) / (32 / G)) * 32;
  const int threads = 128;
  const int blocks = (int)((lanes + threads - 1) / threads);
  alpha_forward_kernel<<<blocks, threads, 0, stream>>>(L, G, ppl);
  return cudaGetLastError();
}

cudaError_t alpha_backward(AlphaLaunch L, cudaStream_t stream) {
  int G, ppl;
  seg_geometry(L.T, G, ppl);
  const int nseg = (L.T + kSeg - 1) / kSeg;
  const size_t bytes = (size_t)L.S * nseg * kSubs * 6 * sizeof(double);
  double* subck = nullptr;
  cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&subck), bytes, stream);
  if (e != cudaSuccess) return e;
  const int warps = (L.S + 32 / G - 1) / (32 / G);
  alpha_backward_kernel<<<(warps + kAdjWarps - 1) / kAdjWarps, 32 * kAdjWarps, 0, stream>>>(L, G, ppl, subck);
  e = cudaGetLastError();
  const cudaError_t ef = scratch_free(subck, stream);
  return e != cudaSuccess ? e : ef;
}

}  // namespace tb
