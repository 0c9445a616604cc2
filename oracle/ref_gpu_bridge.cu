// Test infrastructure only: a C-ABI bridge over the reference's own GPU code,
// compiled from the reference tree where it lies by oracle/Makefile (target
// refgpu) into oracle/_ref/libtaref_gpu.so. It produces reference-held outputs
// for the families whose only reference implementation is CUDA (ADX, DX, CCI,
// WILLR, CORREL; the fused SUM / MIN / MAX windows), which pin the project's
// FP64 oracle, and it times the reference's own batch kernels on the same GPU.
// Nothing in the product links it.
//
// What it calls, by reference path:
//   * src/api/BatchShort.cu launch_short_rows: the short-row kernels that
//     ct_adx_batch_d / ct_dx_batch_d / ct_correl_batch_d run when
//     short_batch_shape holds (src/api/api_batch_generated.inc:702-717, 2387-2402);
//   * src/indicators/{ADX,DX,Correl}.cu ::calculate: the per-series path of the
//     same entry points;
//   * src/indicators/{CCI,WILLR}.cu ::calculate over the flattened matrix plus
//     a NaN warm-up of p-1 bars per row: the reference's Flat rows plan for
//     ct_cci_batch_d / ct_willr_batch_d (api_batch_generated.inc:871-917,
//     src/api/api_batch.cu:76-117);
//   * src/api/BatchFused.cu FusedCall::launch: the fused per-row kernels of
//     ct_{sma,ema,rsi,atr,macd,bbands,stochastic,wma,natr,stddev,sum,min,max,
//     obv,mfi,ad,adosc}_batch_d (src/api/BatchFused.cu:178-213);
//   * the per-series ("plain", TACUDA_BATCH_FUSED=0) path of the batch entry
//     points (src/api/api_batch.cu:478-533): for every series, the indicator
//     object that the single-series ct_*_d entry constructs, calculate() on one
//     stream (src/api/api_device.cu: ct_sma_d :539, ct_ema_d, ct_wma_d, ct_rsi_d,
//     ct_atr_d :818, ct_adx_d, ct_bbands_d :1131, ct_stochastic_d :1053,
//     ct_cci_d, ct_obv_d, ct_mfi_d, ct_willr_d). MACD's ct_macd_d runs MACDEXT,
//     which needs the moving-average and TA-Lib 0.8.3 runner sources; it is not
//     bridged.
#include <cuda_runtime.h>

#include <exception>

#include "BatchFused.h"
#include "BatchShort.h"
#include <indicators/ADX.h>
#include <indicators/ATR.h>
#include <indicators/BBANDS.h>
#include <indicators/CCI.h>
#include <indicators/Correl.h>
#include <indicators/DX.h>
#include <indicators/EMA.h>
#include <indicators/MFI.h>
#include <indicators/OBV.h>
#include <indicators/RSI.h>
#include <indicators/SMA.h>
#include <indicators/Stochastic.h>
#include <indicators/WILLR.h>
#include <indicators/WMA.h>

namespace {

namespace td = tacuda::detail;

template <class F>
int guarded(F f) {
  try {
    f();
  } catch (const std::exception&) {
    return 1;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// NaN (all bits set) over the first `warm` bars of every row
void warmup_nan(float* out, int T, int S, int warm, cudaStream_t s) {
  if (warm > 0) cudaMemset2DAsync(out, (size_t)T * sizeof(float), 0xFF, (size_t)warm * sizeof(float), S, s);
}

}  // namespace

extern "C" {

// path 0: short-row kernel (the batch entry's choice for seriesLen <= 1024),
// path 1: the per-series calculate() of every row.
int refgpu_adx(const float* h, const float* l, const float* c, float* out, int T, int S, int p, int path,
               void* stream) {
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  return guarded([&] {
    if (path == 0) {
      const float* in[3] = {h, l, c};
      float* o[1] = {out};
      td::launch_short_rows(td::ShortFamily::Adx, in, 3, o, 1, T, S, td::ShortOptions{p}, s);
    } else {
      tacuda::ADX ind(p);
      for (int r = 0; r < S; ++r)
        ind.calculate(h + (size_t)r * T, l + (size_t)r * T, c + (size_t)r * T, out + (size_t)r * T, T, s);
    }
  });
}

int refgpu_dx(const float* h, const float* l, const float* c, float* out, int T, int S, int p, int path,
              void* stream) {
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  return guarded([&] {
    if (path == 0) {
      const float* in[3] = {h, l, c};
      float* o[1] = {out};
      td::launch_short_rows(td::ShortFamily::Dx, in, 3, o, 1, T, S, td::ShortOptions{p}, s);
    } else {
      tacuda::DX ind(p);
      for (int r = 0; r < S; ++r)
        ind.calculate(h + (size_t)r * T, l + (size_t)r * T, c + (size_t)r * T, out + (size_t)r * T, T, s);
    }
  });
}

int refgpu_correl(const float* x, const float* y, float* out, int T, int S, int p, int path, void* stream) {
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  return guarded([&] {
    if (path == 0) {
      const float* in[2] = {x, y};
      float* o[1] = {out};
      td::launch_short_rows(td::ShortFamily::Correl, in, 2, o, 1, T, S, td::ShortOptions{p}, s);
    } else {
      tacuda::Correl ind(p);
      for (int r = 0; r < S; ++r) ind.calculate(x + (size_t)r * T, y + (size_t)r * T, out + (size_t)r * T, T, s);
    }
  });
}

// Flat plan: one calculate() over the S*T flattened bars, then the warm-up.
int refgpu_cci(const float* h, const float* l, const float* c, float* out, int T, int S, int p, void* stream) {
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  return guarded([&] {
    tacuda::CCI(p).calculate(h, l, c, out, T * S, s);
    warmup_nan(out, T, S, p - 1, s);
  });
}

int refgpu_willr(const float* h, const float* l, const float* c, float* out, int T, int S, int p, void* stream) {
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  return guarded([&] {
    tacuda::WILLR(p).calculate(h, l, c, out, T * S, s);
    warmup_nan(out, T, S, p - 1, s);
  });
}

// FusedFamily order of src/api/BatchFused.h: None, Sma, Ema, Rsi, Atr, Macd,
// Bbands, Stochastic, Wma, Natr, Stddev, Sum, Min, Max, Obv, Mfi, Ad, Adosc.
int refgpu_fused(int family, const float* in0, const float* in1, const float* in2, const float* in3, float* out0,
                 float* out1, float* out2, int T, int S, int p, int q, int r, float up, float dn, void* stream) {
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float* in[4] = {in0, in1, in2, in3};
  float* out[3] = {out0, out1, out2};
  const td::FusedCall call = td::fused_call(static_cast<td::FusedFamily>(family), p, q, r, 1, up, dn);
  const ctStatus_t st = call.launch(in, out, T, S, s);
  return st == CT_STATUS_SUCCESS ? 0 : 10 + (int)st;
}

// Per-series path, family codes: 1 SMA, 2 EMA, 3 WMA, 4 RSI, 5 ATR, 6 ADX,
// 7 BBANDS, 8 STOCH (slowK, slowD), 9 CCI, 10 OBV (close, volume), 11 MFI,
// 12 WILLR. Inputs h, l, c, v as the family reads them; outputs o0..o2.
int refgpu_plain(int family, const float* h, const float* l, const float* c, const float* v, float* o0, float* o1,
                 float* o2, int T, int S, int p, int q, float up, float dn, void* stream) {
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  return guarded([&] {
    for (int r = 0; r < S; ++r) {
      const size_t off = (size_t)r * T;
      const float *hr = h ? h + off : nullptr, *lr = l ? l + off : nullptr, *cr = c ? c + off : nullptr;
      const float* vr = v ? v + off : nullptr;
      float *a = o0 + off, *b = o1 ? o1 + off : nullptr, *d = o2 ? o2 + off : nullptr;
      switch (family) {
        case 1: tacuda::SMA(p).calculate(cr, a, T, s); break;
        case 2: tacuda::EMA(p).calculate(cr, a, T, s); break;
        case 3: tacuda::WMA(p).calculate(cr, a, T, s); break;
        case 4: tacuda::RSI(p).calculate(cr, a, T, s); break;
        case 5: tacuda::ATR(p, 0.0f).calculate(hr, lr, cr, a, T, s); break;
        case 6: tacuda::ADX(p).calculate(hr, lr, cr, a, T, s); break;
        case 7: tacuda::BBANDS(p, up, dn).calculate(cr, a, b, d, T, s); break;
        case 8: tacuda::Stochastic(p, q).calculate(hr, lr, cr, a, b, T, s); break;
        case 9: tacuda::CCI(p).calculate(hr, lr, cr, a, T, s); break;
        case 10: tacuda::OBV().calculate(cr, vr, a, T, s); break;
        case 11: tacuda::MFI(p).calculate(hr, lr, cr, vr, a, T, s); break;
        case 12: tacuda::WILLR(p).calculate(hr, lr, cr, a, T, s); break;
        default: throw std::exception();
      }
    }
  });
}

}  // extern "C"
