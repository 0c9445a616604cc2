// Differentiable EMA / MACD / RSI with a per-series smoothing coefficient:
// launch descriptors shared by the C entry points and the kernels.
#pragma once

#include <cuda_runtime.h>

namespace tb {

// Bars between forward checkpoints (the state entering each segment).
constexpr int kAlphaSegment = 256;
constexpr int kAlphaStates = 6;  // EMA, slow, fast, signal, RSI gain, RSI loss

struct AlphaParams {
  int ema_period, fast, slow, signal, rsi_period;
};

struct AlphaLaunch {
  const float* x;       // closes, numSeries rows of seriesLen
  const float* alpha;   // one coefficient per series, in (0, 1)
  int T, S;
  AlphaParams P;
  // forward outputs (any may be null) and checkpoints
  float *ema, *macd, *sig, *hist, *rsi;
  double* ckpt;         // S * ceil(T / kAlphaSegment) * kAlphaStates
  // adjoint: output weights dL/d(output) (null = 0) and gradients
  const float *w_ema, *w_macd, *w_sig, *w_hist, *w_rsi;
  float* dx;            // dL/dclose, S*T
  float* dalpha;        // dL/dalpha, S
};

cudaError_t alpha_forward(const AlphaLaunch& L, cudaStream_t stream);
cudaError_t alpha_backward(AlphaLaunch L, cudaStream_t stream);

}  // namespace tb
