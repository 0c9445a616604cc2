// Differentiable EMA / MACD / RSI with a per-series smoothing coefficient
// alpha, and their hand-written adjoint.
//
// Forward (one thread per series, TA-Lib's structure with alpha in place of
// the recurrence coefficient; periods fix the lookback and the seeds):
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
// bar-to-bar change. Walking the segments from the last one back, each
// segment's forward quantities are recomputed from its checkpoint into a
// per-series scratch line, then consumed in reverse.
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

__global__ void alpha_forward_kernel(AlphaLaunch L) {
  const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
  if (sidx >= L.S) return;
  const Stages s = make_stages(L.P, (double)L.alpha[sidx]);
  const long long base = (long long)sidx * L.T;
  const int nseg = (L.T + kSeg - 1) / kSeg;
  State st{0, 0, 0, 0, 0, 0};
  double xprev = 0.0;
  const float nan = qnan();
  for (int t = 0; t < L.T; ++t) {
    if (t % kSeg == 0) {
      double* c = L.ckpt + ((long long)sidx * nseg + t / kSeg) * 6;
      c[0] = st.e; c[1] = st.sl; c[2] = st.f; c[3] = st.g; c[4] = st.rg; c[5] = st.rl;
    }
    const double x = L.x[base + t];
    BarQ q;
    const BarOut o = step<false>(s, t, x, xprev, st, q);
    xprev = x;
    if (L.ema) L.ema[base + t] = o.ema_ok ? (float)o.ema : nan;
    if (L.macd) L.macd[base + t] = o.macd_ok ? (float)o.macd : nan;
    if (L.sig) L.sig[base + t] = o.macd_ok ? (float)o.sig : nan;
    if (L.hist) L.hist[base + t] = o.macd_ok ? (float)(o.macd - o.sig) : nan;
    if (L.rsi) L.rsi[base + t] = o.rsi_ok ? (float)o.rsi : nan;
  }
}

__device__ __forceinline__ double wv(const float* w, long long i) { return w ? (double)w[i] : 0.0; }

__global__ void alpha_backward_kernel(AlphaLaunch L) {
  const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
  if (sidx >= L.S) return;
  const Stages s = make_stages(L.P, (double)L.alpha[sidx]);
  const long long base = (long long)sidx * L.T;
  const int nseg = (L.T + kSeg - 1) / kSeg;
  // scratch line of this series: [bar][quantity][series] for coalesced access
  auto qat = [&](int i, int k) -> double& { return L.scratch[((long long)i * kQ + k) * L.S + sidx]; };
  // carries of the reverse recurrences: a(t+1) * lambda_{t+1}
  double cE = 0, cG = 0, cF = 0, cS = 0, cRG = 0, cRL = 0;
  double pend = 0.0;  // -dL/dchange_{t+1}, owed to x_t
  double dalpha = 0.0;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int t0 = seg * kSeg, t1 = min(L.T, t0 + kSeg);
    const double* c = L.ckpt + ((long long)sidx * nseg + seg) * 6;
    State st{c[0], c[1], c[2], c[3], c[4], c[5]};
    double xprev = t0 > 0 ? (double)L.x[base + t0 - 1] : 0.0;
    for (int t = t0; t < t1; ++t) {
      const double x = L.x[base + t];
      BarQ q;
      step<true>(s, t, x, xprev, st, q);
      xprev = x;
      const int i = t - t0;
      qat(i, 0) = q.eE; qat(i, 1) = q.eF; qat(i, 2) = q.cG;
      qat(i, 3) = q.cL; qat(i, 4) = q.eG; qat(i, 5) = q.eL;
    }
    for (int t = t1 - 1; t >= t0; --t) {
      const int i = t - t0;
      const long long gi = base + t;
      double a, w, dx = pend;
      // EMA
      const double lE = (s.E.ready(t) ? wv(L.w_ema, gi) : 0.0) + cE;
      s.E.coef(t, a, w);
      dx += w * lE;
      if (t >= s.E.p) dalpha += lE * qat(i, 0);
      cE = a * lE;
      // signal line, then dL/dMACD
      const bool ok = t >= s.ready;
      const double wh = ok ? wv(L.w_hist, gi) : 0.0;
      const double lG = (ok ? wv(L.w_sig, gi) - wh : 0.0) + cG;
      s.G.coef(t, a, w);
      const double mu = (ok ? wv(L.w_macd, gi) + wh : 0.0) + w * lG;
      cG = a * lG;
      const double mm = t >= s.slow - 1 ? mu : 0.0;
      // fast line (alpha) and slow line
      const double lF = mm + cF;
      s.F.coef(t, a, w);
      dx += w * lF;
      if (t >= s.slow) dalpha += lF * qat(i, 1);
      cF = a * lF;
      const double lS = -mm + cS;
      s.Sl.coef(t, a, w);
      dx += w * lS;
      cS = a * lS;
      // RSI: gain / loss channels, then the change x_t - x_{t-1}
      const double wr = t >= s.rp ? wv(L.w_rsi, gi) : 0.0;
      const double lRG = wr * qat(i, 2) + cRG;
      const double lRL = wr * qat(i, 3) + cRL;
      rsi_coef(s, t, a, w);
      if (t > s.rp) dalpha += lRG * qat(i, 4) + lRL * qat(i, 5);
      cRG = a * lRG;
      cRL = a * lRL;
      double dd = 0.0;
      if (t >= 1) {
        const double d = (double)L.x[gi] - (double)L.x[gi - 1];
        if (d > 0.0) dd = w * lRG;
        else if (d < 0.0) dd = -w * lRL;
      }
      dx += dd;
      pend = -dd;
      L.dx[gi] = (float)dx;
    }
  }
  L.dalpha[sidx] = (float)dalpha;
}

}  // namespace

cudaError_t alpha_forward(const AlphaLaunch& L, cudaStream_t stream) {
  const int threads = 32;
  const int blocks = (L.S + threads - 1) / threads;
  alpha_forward_kernel<<<blocks, threads, 0, stream>>>(L);
  return cudaGetLastError();
}

cudaError_t alpha_backward(AlphaLaunch L, cudaStream_t stream) {
  const size_t bytes = (size_t)kSeg * kQ * L.S * sizeof(double);
  double* scratch = nullptr;
  cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&scratch), bytes, stream);
  if (e != cudaSuccess) return e;
  L.scratch = scratch;
  const int threads = 32;
  const int blocks = (L.S + threads - 1) / threads;
  alpha_backward_kernel<<<blocks, threads, 0, stream>>>(L);
  e = cudaGetLastError();
  const cudaError_t ef = scratch_free(scratch, stream);
  return e != cudaSuccess ? e : ef;
}

}  // namespace tb
