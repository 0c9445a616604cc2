// extern "C" boundary of the library: the reference's batch / single-series
// entry points (same names, arguments, status codes and stream semantics as
// include/tacuda.h and include/tacuda_device.h of TACUDA 0.9.3) plus the
// append-only ct_b200_* surface. Every batch call is one launch of the fused
// engine (engine.cu) with one or more jobs.
#include <tacuda.h>

#include "adjoint.h"
#include "engine.h"
#include "pool.h"
#include "families.cuh"
#include "scheduler.h"

#include <algorithm>
#include <functional>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <mutex>
#include <vector>

namespace {

using tb::Job;
using tb::Launch;

thread_local std::string t_last_error;
std::atomic<unsigned long long> g_launches{0};

void clear_error() { t_last_error.clear(); }

ctStatus_t fail(ctStatus_t st, const std::string& msg) {
  t_last_error = msg;
  return st;
}

ctStatus_t cuda_fail(ctStatus_t st, const char* where, cudaError_t e) {
  return fail(st, std::string(where) + ": " + cudaGetErrorString(e));
}

// Minimum valid period of each family's first integer parameter.
int min_period(int family) {
  switch (family) {
    case tb::F_OBV: case tb::F_AD: case tb::F_TRANGE: case tb::F_CDL: case tb::F_MEDPRICE: case tb::F_TYPPRICE:
    case tb::F_AVGPRICE: case tb::F_WCLPRICE: case tb::F_IBS: case tb::F_MARKETFI:
      return 0;
    default: return 1;
  }
}

int default_inputs(int family, int* in) {
  switch (family) {
    case tb::F_ATR: case tb::F_NATR: case tb::F_TRANGE: case tb::F_ADX: case tb::F_DX:
    case tb::F_STOCH: case tb::F_WILLR: case tb::F_CCI: case tb::F_TYPPRICE: case tb::F_WCLPRICE: case tb::F_IBS:
      in[0] = tb::P_HIGH; in[1] = tb::P_LOW; in[2] = tb::P_CLOSE; return 3;
    case tb::F_MARKETFI: in[0] = tb::P_HIGH; in[1] = tb::P_LOW; in[2] = tb::P_VOLUME; return 3;
    case tb::F_QSTICK: in[0] = tb::P_OPEN; in[1] = tb::P_CLOSE; return 2;
    case tb::F_MEDPRICE: case tb::F_MIDPRICE: case tb::F_AROON: case tb::F_AROONOSC:
      in[0] = tb::P_HIGH; in[1] = tb::P_LOW; return 2;
    case tb::F_AD: case tb::F_ADOSC: case tb::F_MFI:
      in[0] = tb::P_HIGH; in[1] = tb::P_LOW; in[2] = tb::P_CLOSE; in[3] = tb::P_VOLUME; return 4;
    case tb::F_OBV: in[0] = tb::P_CLOSE; in[1] = tb::P_VOLUME; return 2;
    case tb::F_CORREL: in[0] = tb::P_CLOSE; in[1] = tb::P_AUX; return 2;
    case tb::F_CDL: case tb::F_AVGPRICE:
      in[0] = tb::P_OPEN; in[1] = tb::P_HIGH; in[2] = tb::P_LOW; in[3] = tb::P_CLOSE; return 4;
    default: in[0] = tb::P_CLOSE; return 1;
  }
}

int output_count(int family) {
  switch (family) {
    case tb::F_MACD: case tb::F_BBANDS: return 3;
    case tb::F_STOCH: case tb::F_AROON: return 2;
    default: return 1;
  }
}

constexpr int kMaxWindow = 4096;  // largest window period staged in shared memory

// Build an engine job from reference-style parameters; precomputes TA-Lib's
// coefficients on the host so the device uses the identical doubles.
ctStatus_t make_job(const ctB200Job& u, Job& j, const char* who) {
  std::memset(&j, 0, sizeof(j));
  j.family = u.family;
  if (u.family < 0 || u.family >= tb::F_COUNT) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": unknown family");
  for (int i = 0; i < 3; ++i) j.ip[i] = u.params[i];
  const int f = u.family;
  j.prec = u.precision;
  if (u.precision < 0 || u.precision > 3)
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": precision must be 0..3");
  if (u.precision != 0 && f != tb::F_SMA && f != tb::F_SUM && f != tb::F_WMA && f != tb::F_BBANDS &&
      f != tb::F_STDDEV && f != tb::F_VAR && f != tb::F_LINEARREG && f != tb::F_CORREL && f != tb::F_EMA)
    return fail(CT_STATUS_INVALID_ARGUMENT,
                std::string(who) + ": precision variants exist for SMA SUM WMA BBANDS STDDEV VAR LINEARREG CORREL EMA");
  const int mp = min_period(f);
  if (mp > 0 && u.params[0] < mp) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": invalid period");
  if ((f == tb::F_MACD && (u.params[1] < 1 || u.params[2] < 1)) ||
      (f == tb::F_STOCH && u.params[1] < 1) || (f == tb::F_ADOSC && u.params[1] < 1))
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": invalid period");
  switch (f) {
    case tb::F_SMA: case tb::F_SUM: case tb::F_WMA: case tb::F_BBANDS: case tb::F_STDDEV: case tb::F_VAR:
    case tb::F_LINEARREG: case tb::F_MIN: case tb::F_MAX: case tb::F_WILLR: case tb::F_CCI: case tb::F_MFI:
    case tb::F_CORREL: case tb::F_ROC: case tb::F_MIDPRICE: case tb::F_ROCP: case tb::F_ROCR: case tb::F_ROCR100:
    case tb::F_MOM: case tb::F_MIDPOINT: case tb::F_RMEAN: case tb::F_RMAX: case tb::F_RMIN: case tb::F_RSTD:
    case tb::F_QSTICK: case tb::F_AROON: case tb::F_AROONOSC:
      if (u.params[0] > kMaxWindow) return fail(CT_STATUS_UNSUPPORTED, std::string(who) + ": window period above 4096");
      break;
    case tb::F_STOCH:
      if (u.params[0] > kMaxWindow || u.params[1] > 32)
        return fail(CT_STATUS_UNSUPPORTED, std::string(who) + ": STOCH kPeriod above 4096 or dPeriod above 32");
      break;
    default: break;
  }
  double b, k;
  switch (f) {
    case tb::F_EMA: case tb::F_DEMA: case tb::F_TEMA:
      tb::talib_ema_coeffs(u.params[0], b, k);
      j.fp[0] = b; j.fp[1] = k;
      break;
    case tb::F_T3:
      k = 2.0 / (u.params[0] + 1.0);
      j.fp[0] = 1.0 - k; j.fp[1] = k; j.fp[2] = u.fparams[0];
      break;
    case tb::F_MACD: {
      int fast = u.params[0], slow = u.params[1];
      if (slow < fast) std::swap(fast, slow);  // TA-Lib swaps reversed periods
      j.ip[0] = fast; j.ip[1] = slow; j.ip[2] = u.params[2];
      tb::talib_ema_coeffs(fast, j.fp[0], j.fp[1]);
      tb::talib_ema_coeffs(slow, j.fp[2], j.fp[3]);
      break;
    }
    case tb::F_ATR: case tb::F_NATR:
      j.fp[0] = (double)(u.params[0] - 1) / (double)u.params[0];
      j.fp[1] = 1.0 - j.fp[0];
      break;
    case tb::F_RMA:
      // talib08:13614-13683 TA_RMA: wBeta, wAlpha; periods above 100000 are
      // TA-Lib's TA_BAD_PARAM, an invalid argument at the reference's boundary
      if (u.params[0] > 100000) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": invalid period");
      j.fp[0] = (double)(u.params[0] - 1) / (double)u.params[0];
      j.fp[1] = 1.0 - j.fp[0];
      break;
    case tb::F_BBANDS: j.fp[0] = u.fparams[0]; j.fp[1] = u.fparams[1]; break;
    case tb::F_STDDEV: j.fp[0] = u.fparams[0] == 0.0 ? 1.0 : u.fparams[0]; break;
    default: break;
  }
  int def[4] = {0, 0, 0, 0};
  const int nin = default_inputs(f, def);
  for (int i = 0; i < 4; ++i) j.in[i] = def[i];
  if (u.inputs[0] >= 0) {
    for (int i = 0; i < nin; ++i) {
      if (u.inputs[i] < 0 || u.inputs[i] >= tb::P_COUNT) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": bad input plane");
      j.in[i] = u.inputs[i];
    }
    if ((f == tb::F_CCI || f == tb::F_MFI) &&
        (j.in[0] != tb::P_HIGH || j.in[1] != tb::P_LOW || j.in[2] != tb::P_CLOSE))
      return fail(CT_STATUS_UNSUPPORTED, std::string(who) + ": CCI/MFI read the high/low/close planes");
  }
  const int nout = f == tb::F_CDL ? 1 : output_count(f);
  for (int i = 0; i < nout; ++i) {
    if (!u.outputs[i]) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null output");
    j.out[i] = u.outputs[i];
  }
  if (f == tb::F_CDL) {
    j.cdl_mask = u.cdl_mask;
    j.cdl_stride = u.cdl_stride;
    j.cdl_int32 = u.cdl_int32;
    if (u.cdl_mask == 0 || (u.cdl_mask >> tb::kCdlPatterns) != 0)
      return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": bad candle mask");
  }
  return CT_STATUS_SUCCESS;
}

ctStatus_t check_planes(const Launch& L, const char* who) {
  for (int j = 0; j < L.njobs; ++j) {
    const Job& jb = L.jobs[j];
    int def[4];
    const int nin = default_inputs(jb.family, def);
    for (int i = 0; i < nin; ++i)
      if (!L.plane[jb.in[i]]) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null input");
    if ((jb.family == tb::F_CCI || jb.family == tb::F_MFI) &&
        (!L.plane[tb::P_HIGH] || !L.plane[tb::P_LOW] || !L.plane[tb::P_CLOSE]))
      return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null input");
  }
  return CT_STATUS_SUCCESS;
}

// Synchronise `stream` and report a bounded wait of an engine that ran out
// meanwhile: the per-device error word is read into a pinned per-thread slot
// on the same stream, before the synchronisation, and cleared when set.
ctStatus_t sync_and_check(cudaStream_t stream, const char* who) {
  thread_local int* slot = nullptr;
  if (!slot && cudaMallocHost(reinterpret_cast<void**>(&slot), sizeof(int)) != cudaSuccess) slot = nullptr;
  int* sticky = tb::sticky_word();
  if (slot && sticky) {
    *slot = 0;
    const cudaError_t e = cudaMemcpyAsync(slot, sticky, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return cuda_fail(CT_STATUS_DEVICE_ERROR, who, e);
  }
  const cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(CT_STATUS_DEVICE_ERROR, who, e);
  if (slot && sticky && *slot != 0) {
    cudaMemset(sticky, 0, sizeof(int));
    return fail(CT_STATUS_KERNEL_FAILED,
                std::string(who) + ": a bounded wait of the engine ran out; the outputs are not valid");
  }
  return CT_STATUS_SUCCESS;
}

ctStatus_t finish(cudaStream_t stream, const char* who) {
  if (stream == 0) return sync_and_check(0, who);
  return CT_STATUS_SUCCESS;
}

ctStatus_t launch(Launch& L, long long total, long long maxlen, const tb::SchedulePlan* forced, cudaStream_t stream,
                  const char* who, tb::LaunchStats* stats = nullptr) {
  const tb::SchedulePlan plan = forced ? *forced : tb::plan_for(L, total, maxlen);
  L.max_len = maxlen;
  // test knob: one bounded wait of the launch is made to run out (see
  // Launch::stall_test); the call then reports CT_STATUS_KERNEL_FAILED
  if (const char* e = std::getenv("TACUDA_B200_TEST_STALL")) L.stall_test = std::atoi(e) != 0;
  const cudaError_t e = tb::launch_batch(L, plan, total, stream, stats);
  if (e != cudaSuccess) return cuda_fail(CT_STATUS_KERNEL_FAILED, who, e);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return CT_STATUS_SUCCESS;
}

// One-job uniform batch helper used by every reference entry point.
ctStatus_t run_single(const float* const planes[tb::P_COUNT], const ctB200Job& u, int seriesLen, int numSeries,
                      cudaStream_t stream, const char* who) {
  clear_error();
  if (seriesLen <= 0 || numSeries <= 0) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null pointer or invalid size");
  Launch L;
  std::memset(&L, 0, sizeof(L));
  for (int p = 0; p < tb::P_COUNT; ++p) L.plane[p] = planes[p];
  L.T = seriesLen;
  L.S = numSeries;
  L.njobs = 1;
  ctStatus_t st = make_job(u, L.jobs[0], who);
  if (st != CT_STATUS_SUCCESS) {
    if (st == CT_STATUS_INVALID_ARGUMENT && t_last_error.find("null output") != std::string::npos)
      t_last_error = std::string(who) + ": null pointer or invalid size";
    return st;
  }
  st = check_planes(L, who);
  if (st != CT_STATUS_SUCCESS) return fail(st, std::string(who) + ": null pointer or invalid size");
  st = launch(L, (long long)seriesLen * numSeries, seriesLen, nullptr, stream, who);
  if (st != CT_STATUS_SUCCESS) return st;
  return finish(stream, who);
}

ctB200Job job_of(int family, int p0 = 0, int p1 = 0, int p2 = 0, double f0 = 0.0, double f1 = 0.0) {
  ctB200Job u;
  std::memset(&u, 0, sizeof(u));
  u.family = family;
  u.params[0] = p0; u.params[1] = p1; u.params[2] = p2;
  u.fparams[0] = f0; u.fparams[1] = f1;
  u.inputs[0] = -1;
  return u;
}

struct Planes {
  const float* p[tb::P_COUNT] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

Planes close_only(const float* c) { Planes P; P.p[tb::P_CLOSE] = c; return P; }
Planes hlc(const float* h, const float* l, const float* c) {
  Planes P; P.p[tb::P_HIGH] = h; P.p[tb::P_LOW] = l; P.p[tb::P_CLOSE] = c; return P;
}
Planes hlcv(const float* h, const float* l, const float* c, const float* v) {
  Planes P = hlc(h, l, c); P.p[tb::P_VOLUME] = v; return P;
}
Planes ohlc(const float* o, const float* h, const float* l, const float* c) {
  Planes P = hlc(h, l, c); P.p[tb::P_OPEN] = o; return P;
}

const char* const kCdlNames[tb::kCdlPatterns] = {
#define TB_CDL(name, lb) #name,
#include "candle_list.inc"
#undef TB_CDL
};
const int kCdlLookback[tb::kCdlPatterns] = {
#define TB_CDL(name, lb) lb,
#include "candle_list.inc"
#undef TB_CDL
};

ctStatus_t run_cdl(const float* o, const float* h, const float* l, const float* c, void* out, int seriesLen,
                   int numSeries, uint64_t mask, int as_int, cudaStream_t stream, const char* who) {
  ctB200Job u = job_of(tb::F_CDL);
  u.outputs[0] = out;
  u.cdl_mask = mask;
  u.cdl_stride = as_int ? (int64_t)seriesLen * numSeries : 0;
  u.cdl_int32 = as_int;
  if (!o || !h || !l || !c || !out) {
    clear_error();
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null pointer or invalid size");
  }
  const Planes P = ohlc(o, h, l, c);
  return run_single(P.p, u, seriesLen, numSeries, stream, who);
}

int cdl_index(const char* name) {
  for (int k = 0; k < tb::kCdlPatterns; ++k)
    if (std::strcmp(kCdlNames[k], name) == 0) return k;
  return -1;
}

}  // namespace

struct ctB200Plan {
  std::vector<Job> jobs;
  int njobs = 0;
  int numSeries = 0;
  long long seriesLen = 0;
  bool ragged = false;
  long long total = 0, maxlen = 0;
  int* d_order = nullptr;
  tb::SchedulePlan sched;
  tb::LaunchStats stats;
  int device = 0;
  struct Tried {
    tb::SchedulePlan plan;
    float ms;
  };
  std::vector<Tried> tried;  // candidates of the last autotune and their times per launch
};

extern "C" {

const char* ct_status_string(ctStatus_t s) {
  switch (s) {
    case CT_STATUS_SUCCESS: return "success";
    case CT_STATUS_ALLOC_FAILED: return "allocation failed";
    case CT_STATUS_COPY_FAILED: return "copy failed";
    case CT_STATUS_KERNEL_FAILED: return "kernel failed";
    case CT_STATUS_INVALID_ARGUMENT: return "invalid argument";
    case CT_STATUS_DEVICE_ERROR: return "device error";
    case CT_STATUS_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

const char* ct_get_last_error(void) { return t_last_error.c_str(); }
const char* ct_version(void) { return "0.9.3-b200"; }
unsigned long long ct_b200_launch_count(void) { return g_launches.load(); }

ctStatus_t ct_b200_take_device_error(int* flags) {
  clear_error();
  if (!flags) return fail(CT_STATUS_INVALID_ARGUMENT, "ct_b200_take_device_error: null pointer");
  const cudaError_t e = tb::take_sticky_error(flags);
  if (e != cudaSuccess) return cuda_fail(CT_STATUS_DEVICE_ERROR, "ct_b200_take_device_error", e);
  return CT_STATUS_SUCCESS;
}

// ------------------------------------------------------------ batch API

#define TB_S1(NAME, FAM)                                                                              \
  ctStatus_t ct_##NAME##_batch_d(const float* d_inputs, float* d_outputs, int seriesLen, int numSeries, \
                                 int period, int, cudaStream_t stream) {                              \
    ctB200Job u = job_of(FAM, period);                                                                \
    u.outputs[0] = d_outputs;                                                                         \
    const Planes P = close_only(d_inputs);                                                            \
    return run_single(P.p, u, seriesLen, numSeries, stream, "ct_" #NAME "_batch_d");                  \
  }                                                                                                   \
  ctStatus_t ct_##NAME##_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream) { \
    ctB200Job u = job_of(FAM, period);                                                                \
    u.outputs[0] = d_output;                                                                          \
    const Planes P = close_only(d_input);                                                             \
    return run_single(P.p, u, size, 1, stream, "ct_" #NAME "_d");                                     \
  }

TB_S1(sma, tb::F_SMA)
TB_S1(ema, tb::F_EMA)
TB_S1(wma, tb::F_WMA)
TB_S1(rsi, tb::F_RSI)
TB_S1(dema, tb::F_DEMA)
TB_S1(tema, tb::F_TEMA)
TB_S1(stddev, tb::F_STDDEV)
TB_S1(var, tb::F_VAR)
TB_S1(sum, tb::F_SUM)
TB_S1(max, tb::F_MAX)
TB_S1(min, tb::F_MIN)
TB_S1(linearreg, tb::F_LINEARREG)
TB_S1(roc, tb::F_ROC)  // tacuda.h:1007, tacuda_device.h:174
TB_S1(rma, tb::F_RMA)  // tacuda.h:4110, tacuda_device.h:1212
TB_S1(rocp, tb::F_ROCP)  // tacuda.h:1016, tacuda_device.h:177
TB_S1(rocr, tb::F_ROCR)  // tacuda.h:1026, tacuda_device.h:180
TB_S1(rocr100, tb::F_ROCR100)  // tacuda.h:1036, tacuda_device.h:183
TB_S1(momentum, tb::F_MOM)  // tacuda.h:997, tacuda_device.h:171
TB_S1(midpoint, tb::F_MIDPOINT)  // tacuda.h:1516, tacuda_device.h:447
TB_S1(change, tb::F_MOM)  // tacuda.h:1506, tacuda_device.h:444; src/indicators/Change.cu is MOM's arithmetic
#undef TB_S1

// NaN-strict rolling statistics: a period above the row length is an invalid
// argument (src/indicators/ClubPack.cu:409-413 check_period).
#define TB_ROLL(NAME, FAM)                                                                            \
  ctStatus_t ct_##NAME##_batch_d(const float* d_inputs, float* d_outputs, int seriesLen, int numSeries, \
                                 int period, int, cudaStream_t stream) {                              \
    if (period > seriesLen && seriesLen > 0) {                                                        \
      clear_error();                                                                                  \
      return fail(CT_STATUS_INVALID_ARGUMENT, "ct_" #NAME "_batch_d: invalid period");              \
    }                                                                                                 \
    ctB200Job u = job_of(FAM, period);                                                                \
    u.outputs[0] = d_outputs;                                                                         \
    const Planes P = close_only(d_inputs);                                                            \
    return run_single(P.p, u, seriesLen, numSeries, stream, "ct_" #NAME "_batch_d");                  \
  }                                                                                                   \
  ctStatus_t ct_##NAME##_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream) { \
    if (period > size && size > 0 && d_input && d_output) {                                           \
      clear_error();                                                                                  \
      return fail(CT_STATUS_INVALID_ARGUMENT, "ct_" #NAME "_d: invalid period");                    \
    }                                                                                                 \
    ctB200Job u = job_of(FAM, period);                                                                \
    u.outputs[0] = d_output;                                                                          \
    const Planes P = close_only(d_input);                                                             \
    return run_single(P.p, u, size, 1, stream, "ct_" #NAME "_d");                                     \
  }

TB_ROLL(rolling_mean, tb::F_RMEAN)  // tacuda.h:3157, tacuda_device.h:981
TB_ROLL(rolling_max, tb::F_RMAX)    // tacuda.h:3171, tacuda_device.h:985
TB_ROLL(rolling_min, tb::F_RMIN)    // tacuda.h:3185, tacuda_device.h:988
TB_ROLL(rolling_std, tb::F_RSTD)    // tacuda.h:3199, tacuda_device.h:991
#undef TB_ROLL

#define TB_HLC(NAME, FAM)                                                                                  \
  ctStatus_t ct_##NAME##_batch_d(const float* d_highs, const float* d_lows, const float* d_closes,         \
                                 float* d_outputs, int seriesLen, int numSeries, int period, int,          \
                                 cudaStream_t stream) {                                                    \
    ctB200Job u = job_of(FAM, period);                                                                     \
    u.outputs[0] = d_outputs;                                                                              \
    const Planes P = hlc(d_highs, d_lows, d_closes);                                                       \
    return run_single(P.p, u, seriesLen, numSeries, stream, "ct_" #NAME "_batch_d");                       \
  }                                                                                                        \
  ctStatus_t ct_##NAME##_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, \
                           int size, int period, cudaStream_t stream) {                                    \
    ctB200Job u = job_of(FAM, period);                                                                     \
    u.outputs[0] = d_output;                                                                               \
    const Planes P = hlc(d_high, d_low, d_close);                                                          \
    return run_single(P.p, u, size, 1, stream, "ct_" #NAME "_d");                                          \
  }

TB_HLC(natr, tb::F_NATR)
TB_HLC(adx, tb::F_ADX)
TB_HLC(dx, tb::F_DX)
TB_HLC(willr, tb::F_WILLR)
TB_HLC(cci, tb::F_CCI)
#undef TB_HLC

ctStatus_t ct_atr_batch_d(const float* d_highs, const float* d_lows, const float* d_closes, float* d_outputs,
                          int seriesLen, int numSeries, int period, float, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_ATR, period);
  u.outputs[0] = d_outputs;
  const Planes P = hlc(d_highs, d_lows, d_closes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_atr_batch_d");
}
ctStatus_t ct_atr_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size,
                    int period, float, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_ATR, period);
  u.outputs[0] = d_output;
  const Planes P = hlc(d_high, d_low, d_close);
  return run_single(P.p, u, size, 1, stream, "ct_atr_d");
}

ctStatus_t ct_trange_batch_d(const float* d_highs, const float* d_lows, const float* d_closes, float* d_outputs,
                             int seriesLen, int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_TRANGE);
  u.outputs[0] = d_outputs;
  const Planes P = hlc(d_highs, d_lows, d_closes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_trange_batch_d");
}
ctStatus_t ct_trange_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size,
                       cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_TRANGE);
  u.outputs[0] = d_output;
  const Planes P = hlc(d_high, d_low, d_close);
  return run_single(P.p, u, size, 1, stream, "ct_trange_d");
}

static ctStatus_t macd_common(const float* in, float* m, float* s, float* h, int len, int n, int fast, int slow,
                              int signal, int maType, cudaStream_t stream, const char* who) {
  if (maType != 1) {
    clear_error();
    return fail(CT_STATUS_UNSUPPORTED, std::string(who) + ": only maType = CT_MA_EMA is implemented");
  }
  ctB200Job u = job_of(tb::F_MACD, fast, slow, signal);
  u.outputs[0] = m; u.outputs[1] = s; u.outputs[2] = h;
  const Planes P = close_only(in);
  return run_single(P.p, u, len, n, stream, who);
}
ctStatus_t ct_macd_batch_d(const float* d_inputs, float* d_macds, float* d_signals, float* d_hists, int seriesLen,
                           int numSeries, int fastPeriod, int slowPeriod, int signalPeriod, int maType, int,
                           cudaStream_t stream) {
  return macd_common(d_inputs, d_macds, d_signals, d_hists, seriesLen, numSeries, fastPeriod, slowPeriod,
                     signalPeriod, maType, stream, "ct_macd_batch_d");
}
ctStatus_t ct_macd_d(const float* d_input, float* d_macd, float* d_signal, float* d_hist, int size, int fastPeriod,
                     int slowPeriod, int signalPeriod, int maType, cudaStream_t stream) {
  return macd_common(d_input, d_macd, d_signal, d_hist, size, 1, fastPeriod, slowPeriod, signalPeriod, maType,
                     stream, "ct_macd_d");
}

ctStatus_t ct_bbands_batch_d(const float* d_inputs, float* d_uppers, float* d_middles, float* d_lowers,
                             int seriesLen, int numSeries, int period, float upperMul, float lowerMul, int,
                             cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_BBANDS, period, 0, 0, upperMul, lowerMul);
  u.outputs[0] = d_uppers; u.outputs[1] = d_middles; u.outputs[2] = d_lowers;
  const Planes P = close_only(d_inputs);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_bbands_batch_d");
}
ctStatus_t ct_bbands_d(const float* d_input, float* d_upper, float* d_middle, float* d_lower, int size, int period,
                       float nbDevUp, float nbDevDn, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_BBANDS, period, 0, 0, nbDevUp, nbDevDn);
  u.outputs[0] = d_upper; u.outputs[1] = d_middle; u.outputs[2] = d_lower;
  const Planes P = close_only(d_input);
  return run_single(P.p, u, size, 1, stream, "ct_bbands_d");
}

ctStatus_t ct_stochastic_batch_d(const float* d_highs, const float* d_lows, const float* d_closes, float* d_ks,
                                 float* d_ds, int seriesLen, int numSeries, int kPeriod, int dPeriod, int,
                                 cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_STOCH, kPeriod, dPeriod);
  u.outputs[0] = d_ks; u.outputs[1] = d_ds;
  const Planes P = hlc(d_highs, d_lows, d_closes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_stochastic_batch_d");
}
ctStatus_t ct_stochastic_d(const float* d_high, const float* d_low, const float* d_close, float* d_slowK,
                           float* d_slowD, int size, int kPeriod, int dPeriod, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_STOCH, kPeriod, dPeriod);
  u.outputs[0] = d_slowK; u.outputs[1] = d_slowD;
  const Planes P = hlc(d_high, d_low, d_close);
  return run_single(P.p, u, size, 1, stream, "ct_stochastic_d");
}

ctStatus_t ct_t3_batch_d(const float* d_inputs, float* d_outputs, int seriesLen, int numSeries, int period,
                         float vFactor, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_T3, period, 0, 0, vFactor);
  u.outputs[0] = d_outputs;
  const Planes P = close_only(d_inputs);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_t3_batch_d");
}
ctStatus_t ct_t3_d(const float* d_input, float* d_output, int size, int period, float vFactor, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_T3, period, 0, 0, vFactor);
  u.outputs[0] = d_output;
  const Planes P = close_only(d_input);
  return run_single(P.p, u, size, 1, stream, "ct_t3_d");
}

ctStatus_t ct_obv_batch_d(const float* d_closes, const float* d_volumes, float* d_outputs, int seriesLen,
                          int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_OBV);
  u.outputs[0] = d_outputs;
  Planes P = close_only(d_closes);
  P.p[tb::P_VOLUME] = d_volumes;
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_obv_batch_d");
}
ctStatus_t ct_obv_d(const float* d_close, const float* d_volume, float* d_output, int size, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_OBV);
  u.outputs[0] = d_output;
  Planes P = close_only(d_close);
  P.p[tb::P_VOLUME] = d_volume;
  return run_single(P.p, u, size, 1, stream, "ct_obv_d");
}

ctStatus_t ct_mfi_batch_d(const float* d_highs, const float* d_lows, const float* d_closes, const float* d_volumes,
                          float* d_outputs, int seriesLen, int numSeries, int period, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_MFI, period);
  u.outputs[0] = d_outputs;
  const Planes P = hlcv(d_highs, d_lows, d_closes, d_volumes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_mfi_batch_d");
}
ctStatus_t ct_mfi_d(const float* d_high, const float* d_low, const float* d_close, const float* d_volume,
                    float* d_output, int size, int period, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_MFI, period);
  u.outputs[0] = d_output;
  const Planes P = hlcv(d_high, d_low, d_close, d_volume);
  return run_single(P.p, u, size, 1, stream, "ct_mfi_d");
}

ctStatus_t ct_ad_batch_d(const float* d_highs, const float* d_lows, const float* d_closes, const float* d_volumes,
                         float* d_outputs, int seriesLen, int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_AD);
  u.outputs[0] = d_outputs;
  const Planes P = hlcv(d_highs, d_lows, d_closes, d_volumes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_ad_batch_d");
}
ctStatus_t ct_ad_d(const float* d_high, const float* d_low, const float* d_close, const float* d_volume,
                   float* d_output, int size, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_AD);
  u.outputs[0] = d_output;
  const Planes P = hlcv(d_high, d_low, d_close, d_volume);
  return run_single(P.p, u, size, 1, stream, "ct_ad_d");
}

ctStatus_t ct_adosc_batch_d(const float* d_highs, const float* d_lows, const float* d_closes,
                            const float* d_volumes, float* d_outputs, int seriesLen, int numSeries, int fastPeriod,
                            int slowPeriod, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_ADOSC, fastPeriod, slowPeriod);
  u.outputs[0] = d_outputs;
  const Planes P = hlcv(d_highs, d_lows, d_closes, d_volumes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_adosc_batch_d");
}
ctStatus_t ct_adosc_d(const float* d_high, const float* d_low, const float* d_close, const float* d_volume,
                      float* d_output, int size, int fastPeriod, int slowPeriod, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_ADOSC, fastPeriod, slowPeriod);
  u.outputs[0] = d_output;
  const Planes P = hlcv(d_high, d_low, d_close, d_volume);
  return run_single(P.p, u, size, 1, stream, "ct_adosc_d");
}

ctStatus_t ct_correl_batch_d(const float* d_xs, const float* d_ys, float* d_outputs, int seriesLen, int numSeries,
                             int period, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_CORREL, period);
  u.outputs[0] = d_outputs;
  Planes P = close_only(d_xs);
  P.p[tb::P_AUX] = d_ys;
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_correl_batch_d");
}
ctStatus_t ct_correl_d(const float* d_x, const float* d_y, float* d_output, int size, int period,
                       cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_CORREL, period);
  u.outputs[0] = d_output;
  Planes P = close_only(d_x);
  P.p[tb::P_AUX] = d_y;
  return run_single(P.p, u, size, 1, stream, "ct_correl_d");
}

// ------------------------------------------------------------ price transforms

ctStatus_t ct_medprice_batch_d(const float* d_highs, const float* d_lows, float* d_outputs, int seriesLen,
                               int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_MEDPRICE);
  u.outputs[0] = d_outputs;
  Planes P;
  P.p[tb::P_HIGH] = d_highs; P.p[tb::P_LOW] = d_lows;
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_medprice_batch_d");
}
ctStatus_t ct_medprice_d(const float* d_high, const float* d_low, float* d_output, int size, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_MEDPRICE);
  u.outputs[0] = d_output;
  Planes P;
  P.p[tb::P_HIGH] = d_high; P.p[tb::P_LOW] = d_low;
  return run_single(P.p, u, size, 1, stream, "ct_medprice_d");
}

ctStatus_t ct_typprice_batch_d(const float* d_highs, const float* d_lows, const float* d_closes, float* d_outputs,
                               int seriesLen, int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_TYPPRICE);
  u.outputs[0] = d_outputs;
  const Planes P = hlc(d_highs, d_lows, d_closes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_typprice_batch_d");
}
ctStatus_t ct_typprice_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size,
                         cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_TYPPRICE);
  u.outputs[0] = d_output;
  const Planes P = hlc(d_high, d_low, d_close);
  return run_single(P.p, u, size, 1, stream, "ct_typprice_d");
}

ctStatus_t ct_ibs_batch_d(const float* d_highs, const float* d_lows, const float* d_closes, float* d_outputs,
                          int seriesLen, int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_IBS);
  u.outputs[0] = d_outputs;
  const Planes P = hlc(d_highs, d_lows, d_closes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_ibs_batch_d");
}
ctStatus_t ct_ibs_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size,
                    cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_IBS);
  u.outputs[0] = d_output;
  const Planes P = hlc(d_high, d_low, d_close);
  return run_single(P.p, u, size, 1, stream, "ct_ibs_d");
}

ctStatus_t ct_marketfi_batch_d(const float* d_highs, const float* d_lows, const float* d_volumes, float* d_outputs,
                               int seriesLen, int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_MARKETFI);
  u.outputs[0] = d_outputs;
  Planes P;
  P.p[tb::P_HIGH] = d_highs; P.p[tb::P_LOW] = d_lows; P.p[tb::P_VOLUME] = d_volumes;
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_marketfi_batch_d");
}
ctStatus_t ct_marketfi_d(const float* d_high, const float* d_low, const float* d_volume, float* d_output, int size,
                         cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_MARKETFI);
  u.outputs[0] = d_output;
  Planes P;
  P.p[tb::P_HIGH] = d_high; P.p[tb::P_LOW] = d_low; P.p[tb::P_VOLUME] = d_volume;
  return run_single(P.p, u, size, 1, stream, "ct_marketfi_d");
}

ctStatus_t ct_qstick_batch_d(const float* d_opens, const float* d_closes, float* d_outputs, int seriesLen,
                             int numSeries, int period, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_QSTICK, period);
  u.outputs[0] = d_outputs;
  Planes P;
  P.p[tb::P_OPEN] = d_opens; P.p[tb::P_CLOSE] = d_closes;
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_qstick_batch_d");
}
ctStatus_t ct_qstick_d(const float* d_open, const float* d_close, float* d_output, int size, int period,
                       cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_QSTICK, period);
  u.outputs[0] = d_output;
  Planes P;
  P.p[tb::P_OPEN] = d_open; P.p[tb::P_CLOSE] = d_close;
  return run_single(P.p, u, size, 1, stream, "ct_qstick_d");
}

ctStatus_t ct_wclprice_batch_d(const float* d_highs, const float* d_lows, const float* d_closes, float* d_outputs,
                               int seriesLen, int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_WCLPRICE);
  u.outputs[0] = d_outputs;
  const Planes P = hlc(d_highs, d_lows, d_closes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_wclprice_batch_d");
}
ctStatus_t ct_wclprice_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size,
                         cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_WCLPRICE);
  u.outputs[0] = d_output;
  const Planes P = hlc(d_high, d_low, d_close);
  return run_single(P.p, u, size, 1, stream, "ct_wclprice_d");
}

ctStatus_t ct_avgprice_batch_d(const float* d_opens, const float* d_highs, const float* d_lows, const float* d_closes,
                               float* d_outputs, int seriesLen, int numSeries, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_AVGPRICE);
  u.outputs[0] = d_outputs;
  const Planes P = ohlc(d_opens, d_highs, d_lows, d_closes);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_avgprice_batch_d");
}
ctStatus_t ct_avgprice_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close,
                         float* d_output, int size, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_AVGPRICE);
  u.outputs[0] = d_output;
  const Planes P = ohlc(d_open, d_high, d_low, d_close);
  return run_single(P.p, u, size, 1, stream, "ct_avgprice_d");
}

ctStatus_t ct_midprice_batch_d(const float* d_highs, const float* d_lows, float* d_outputs, int seriesLen,
                               int numSeries, int period, int, cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_MIDPRICE, period);
  u.outputs[0] = d_outputs;
  Planes P;
  P.p[tb::P_HIGH] = d_highs; P.p[tb::P_LOW] = d_lows;
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_midprice_batch_d");
}
ctStatus_t ct_midprice_d(const float* d_high, const float* d_low, float* d_output, int size, int period,
                         cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_MIDPRICE, period);
  u.outputs[0] = d_output;
  Planes P;
  P.p[tb::P_HIGH] = d_high; P.p[tb::P_LOW] = d_low;
  return run_single(P.p, u, size, 1, stream, "ct_midprice_d");
}

// AROON (src/indicators/Aroon.cu:11-52 via api_device.cu:1467-1484): outputs in
// the reference's order, aroon down then aroon up. The reference's ct_aroon_d
// turns every exception, an invalid period included, into
// CT_STATUS_KERNEL_FAILED (api_device.cu:1482-1483); so does this entry.
static ctStatus_t aroon_bad_period(const char* who) {
  clear_error();
  return fail(CT_STATUS_KERNEL_FAILED, std::string(who) + ": invalid period");
}
ctStatus_t ct_aroon_batch_d(const float* d_highs, const float* d_lows, float* d_aroon_downs, float* d_aroon_ups,
                            int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream) {
  (void)maxConcurrency;
  if (period < 1 && d_highs && d_lows && d_aroon_downs && d_aroon_ups && seriesLen > 0 && numSeries > 0)
    return aroon_bad_period("ct_aroon_batch_d");
  ctB200Job u = job_of(tb::F_AROON, period);
  u.outputs[0] = d_aroon_downs;
  u.outputs[1] = d_aroon_ups;
  const Planes P = hlc(d_highs, d_lows, nullptr);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_aroon_batch_d");
}
ctStatus_t ct_aroon_d(const float* d_high, const float* d_low, float* d_aroonDown, float* d_aroonUp, int size,
                      int period, cudaStream_t stream) {
  if (period < 1 && d_high && d_low && d_aroonDown && d_aroonUp && size > 0) return aroon_bad_period("ct_aroon_d");
  ctB200Job u = job_of(tb::F_AROON, period);
  u.outputs[0] = d_aroonDown;
  u.outputs[1] = d_aroonUp;
  const Planes P = hlc(d_high, d_low, nullptr);
  return run_single(P.p, u, size, 1, stream, "ct_aroon_d");
}
// AROONOSC (src/indicators/AroonOscillator.cu:12-40 via api_device.cu:1486-1496).
ctStatus_t ct_aroonosc_batch_d(const float* d_highs, const float* d_lows, float* d_outputs, int seriesLen,
                               int numSeries, int period, int maxConcurrency, cudaStream_t stream) {
  (void)maxConcurrency;
  ctB200Job u = job_of(tb::F_AROONOSC, period);
  u.outputs[0] = d_outputs;
  const Planes P = hlc(d_highs, d_lows, nullptr);
  return run_single(P.p, u, seriesLen, numSeries, stream, "ct_aroonosc_batch_d");
}
ctStatus_t ct_aroonosc_d(const float* d_high, const float* d_low, float* d_output, int size, int period,
                         cudaStream_t stream) {
  ctB200Job u = job_of(tb::F_AROONOSC, period);
  u.outputs[0] = d_output;
  const Planes P = hlc(d_high, d_low, nullptr);
  return run_single(P.p, u, size, 1, stream, "ct_aroonosc_d");
}

// ------------------------------------------------------------ candles

#define TB_CDL(NAME, LB)                                                                                     \
  ctStatus_t ct_cdl_##NAME##_batch_d(const float* d_opens, const float* d_highs, const float* d_lows,        \
                                     const float* d_closes, float* d_outputs, int seriesLen, int numSeries,  \
                                     int, cudaStream_t stream) {                                            \
    return run_cdl(d_opens, d_highs, d_lows, d_closes, d_outputs, seriesLen, numSeries,                     \
                   1ull << cdl_index(#NAME), 0, stream, "ct_cdl_" #NAME "_batch_d");                         \
  }                                                                                                          \
  ctStatus_t ct_cdl_##NAME##_d(const float* d_open, const float* d_high, const float* d_low,                 \
                               const float* d_close, float* d_output, int size, cudaStream_t stream) {       \
    return run_cdl(d_open, d_high, d_low, d_close, d_output, size, 1, 1ull << cdl_index(#NAME), 0, stream,  \
                   "ct_cdl_" #NAME "_d");                                                                    \
  }
#include "candle_list.inc"
#undef TB_CDL

ctStatus_t ct_b200_cdl_batch_d(const float* d_opens, const float* d_highs, const float* d_lows,
                               const float* d_closes, int32_t* d_out, int seriesLen, int numSeries,
                               uint64_t patternMask, cudaStream_t stream) {
  if (patternMask == 0 || (patternMask >> tb::kCdlPatterns) != 0) {
    clear_error();
    return fail(CT_STATUS_INVALID_ARGUMENT, "ct_b200_cdl_batch_d: bad pattern mask");
  }
  return run_cdl(d_opens, d_highs, d_lows, d_closes, d_out, seriesLen, numSeries, patternMask, 1, stream,
                 "ct_b200_cdl_batch_d");
}

int ct_b200_cdl_count(void) { return tb::kCdlPatterns; }
const char* ct_b200_cdl_name(int k) { return (k >= 0 && k < tb::kCdlPatterns) ? kCdlNames[k] : nullptr; }
int ct_b200_cdl_lookback(int k) { return (k >= 0 && k < tb::kCdlPatterns) ? kCdlLookback[k] : -1; }

// ------------------------------------------------------------ fused API

static ctStatus_t build_launch(const ctB200Series* series, const ctB200Job* jobs, int numJobs, Launch& L,
                               const char* who) {
  if (!series || !jobs || numJobs <= 0 || numJobs > tb::kMaxJobs)
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null pointer or bad job count");
  if (series->numSeries <= 0 || (!series->offsets && series->seriesLen <= 0))
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": invalid size");
  std::memset(&L, 0, sizeof(L));
  for (int p = 0; p < tb::P_COUNT; ++p) L.plane[p] = series->planes[p];
  L.offsets = reinterpret_cast<const long long*>(series->offsets);
  L.T = series->seriesLen;
  L.S = series->numSeries;
  L.njobs = numJobs;
  for (int j = 0; j < numJobs; ++j) {
    const ctStatus_t st = make_job(jobs[j], L.jobs[j], who);
    if (st != CT_STATUS_SUCCESS) return st;
    if (L.jobs[j].prec != L.jobs[0].prec)
      return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": all jobs of a launch need the same precision");
  }
  return check_planes(L, who);
}

ctStatus_t ct_b200_fused_batch_d(const ctB200Series* series, const ctB200Job* jobs, int numJobs,
                                 cudaStream_t stream) {
  clear_error();
  const char* who = "ct_b200_fused_batch_d";
  Launch L;
  ctStatus_t st = build_launch(series, jobs, numJobs, L, who);
  if (st != CT_STATUS_SUCCESS) return st;
  if (L.offsets) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": ragged rows need a plan");
  st = launch(L, L.T * (long long)L.S, L.T, nullptr, stream, who);
  if (st != CT_STATUS_SUCCESS) return st;
  return finish(stream, who);
}

ctStatus_t ct_b200_fused_lookback_static_d(const ctB200Series* series, const ctB200Job* jobs, int numJobs,
                                           cudaStream_t stream) {
  clear_error();
  const char* who = "ct_b200_fused_lookback_static_d";
  Launch L;
  ctStatus_t st = build_launch(series, jobs, numJobs, L, who);
  if (st != CT_STATUS_SUCCESS) return st;
  if (L.offsets) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": uniform rows only");
  for (int j = 0; j < L.njobs; ++j) {
    if (L.jobs[j].family == tb::F_CDL)
      return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": candle jobs are not supported");
    if (L.jobs[j].prec != 0)
      return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": FP64 jobs only");
  }
  tb::SchedulePlan plan = tb::plan_for(L, L.T * (long long)L.S, L.T);
  plan.mode = 2;
  if (const char* e = std::getenv("TACUDA_B200_TEST_STALL")) L.stall_test = std::atoi(e) != 0;
  size_t need = 0;
  const cudaError_t e = tb::launch_lookback_static(L, plan, stream, &need);
  if (e == cudaErrorInvalidValue && need > tb::kStaticLookbackBytes) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "%s: batch needs %zu bytes of look-back scratch, more than the static %zu bytes",
                  who, need, (size_t)tb::kStaticLookbackBytes);
    return fail(CT_STATUS_INVALID_ARGUMENT, msg);
  }
  if (e != cudaSuccess) return cuda_fail(CT_STATUS_KERNEL_FAILED, who, e);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (stream != 0) return CT_STATUS_SUCCESS;
  // stream 0: synchronise, then read the device's error word into a stack
  // variable (the regular entries read it into a pinned per-thread slot,
  // which is allocated on a thread's first call)
  cudaError_t es = cudaStreamSynchronize(0);
  if (es != cudaSuccess) return cuda_fail(CT_STATUS_DEVICE_ERROR, who, es);
  int* sticky = tb::sticky_word();
  int flag = 0;
  if (sticky) {
    es = cudaMemcpy(&flag, sticky, sizeof(int), cudaMemcpyDeviceToHost);
    if (es != cudaSuccess) return cuda_fail(CT_STATUS_DEVICE_ERROR, who, es);
  }
  if (flag != 0) {
    cudaMemset(sticky, 0, sizeof(int));
    return fail(CT_STATUS_KERNEL_FAILED,
                std::string(who) + ": a bounded wait of the engine ran out; the outputs are not valid");
  }
  return CT_STATUS_SUCCESS;
}

// ------------------------------------------------------------ alpha API

long long ct_b200_alpha_checkpoint_doubles(int seriesLen) {
  if (seriesLen <= 0) return 0;
  return (long long)((seriesLen + tb::kAlphaSegment - 1) / tb::kAlphaSegment) * tb::kAlphaStates;
}

static ctStatus_t alpha_params(const ctB200AlphaParams* p, tb::AlphaParams& out, const char* who) {
  if (!p) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null parameters");
  out = tb::AlphaParams{p->emaPeriod, p->fastPeriod, p->slowPeriod, p->signalPeriod, p->rsiPeriod};
  if (out.ema_period < 2 || out.fast < 2 || out.slow < out.fast || out.signal < 1 || out.rsi_period < 2 ||
      out.ema_period > kMaxWindow || out.slow > kMaxWindow || out.signal > kMaxWindow || out.rsi_period > kMaxWindow)
    return fail(CT_STATUS_INVALID_ARGUMENT,
                std::string(who) + ": invalid periods (need ema>=2, 2<=fast<=slow, signal>=1, rsi>=2)");
  return CT_STATUS_SUCCESS;
}

ctStatus_t ct_b200_alpha_forward_d(const float* d_close, const float* d_alpha, int seriesLen, int numSeries,
                                   const ctB200AlphaParams* params, float* d_ema, float* d_macd, float* d_signal,
                                   float* d_hist, float* d_rsi, double* d_checkpoints, cudaStream_t stream) {
  clear_error();
  const char* who = "ct_b200_alpha_forward_d";
  if (!d_close || !d_alpha || !d_checkpoints || seriesLen <= 0 || numSeries <= 0)
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null pointer or invalid size");
  tb::AlphaLaunch L{};
  ctStatus_t st = alpha_params(params, L.P, who);
  if (st != CT_STATUS_SUCCESS) return st;
  L.x = d_close; L.alpha = d_alpha; L.T = seriesLen; L.S = numSeries;
  L.ema = d_ema; L.macd = d_macd; L.sig = d_signal; L.hist = d_hist; L.rsi = d_rsi;
  L.ckpt = d_checkpoints;
  const cudaError_t e = tb::alpha_forward(L, stream);
  if (e != cudaSuccess) return cuda_fail(CT_STATUS_KERNEL_FAILED, who, e);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return finish(stream, who);
}

ctStatus_t ct_b200_alpha_backward_d(const float* d_close, const float* d_alpha, int seriesLen, int numSeries,
                                    const ctB200AlphaParams* params, const double* d_checkpoints,
                                    const float* d_w_ema, const float* d_w_macd, const float* d_w_signal,
                                    const float* d_w_hist, const float* d_w_rsi, float* d_dclose, float* d_dalpha,
                                    cudaStream_t stream) {
  clear_error();
  const char* who = "ct_b200_alpha_backward_d";
  if (!d_close || !d_alpha || !d_checkpoints || !d_dclose || !d_dalpha || seriesLen <= 0 || numSeries <= 0)
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null pointer or invalid size");
  tb::AlphaLaunch L{};
  ctStatus_t st = alpha_params(params, L.P, who);
  if (st != CT_STATUS_SUCCESS) return st;
  L.x = d_close; L.alpha = d_alpha; L.T = seriesLen; L.S = numSeries;
  L.ckpt = const_cast<double*>(d_checkpoints);
  L.w_ema = d_w_ema; L.w_macd = d_w_macd; L.w_sig = d_w_signal; L.w_hist = d_w_hist; L.w_rsi = d_w_rsi;
  L.dx = d_dclose; L.dalpha = d_dalpha;
  const cudaError_t e = tb::alpha_backward(L, stream);
  if (e != cudaSuccess) return cuda_fail(CT_STATUS_KERNEL_FAILED, who, e);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return finish(stream, who);
}

// Auxiliary streams of the host-memory entry point (per device, created once):
// row chunks rotate over them so one chunk's copy-in, another's kernel and a
// third's copy-out overlap.
static constexpr int kPipeStreams = 8;
static std::mutex g_pipe_mutex;
static std::vector<std::vector<cudaStream_t>> g_pipe_streams;

static cudaError_t pipe_streams(cudaStream_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_pipe_mutex);
  if ((int)g_pipe_streams.size() <= dev) g_pipe_streams.resize(dev + 1);
  auto& v = g_pipe_streams[dev];
  while ((int)v.size() < kPipeStreams) {
    cudaStream_t st = nullptr;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    v.push_back(st);
  }
  for (int i = 0; i < kPipeStreams; ++i) out[i] = v[i];
  return cudaSuccess;
}

ctStatus_t ct_b200_fused_batch(const ctB200Series* hs, const ctB200Job* hjobs, int numJobs, cudaStream_t stream) {
  clear_error();
  const char* who = "ct_b200_fused_batch";
  Launch L;
  ctStatus_t st = build_launch(hs, hjobs, numJobs, L, who);
  if (st != CT_STATUS_SUCCESS) return st;
  if (L.offsets) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": ragged rows need a plan");
  const size_t n = (size_t)L.T * L.S;
  const size_t bytes = n * sizeof(float);
  bool has_cdl = false;
  for (int j = 0; j < L.njobs; ++j) has_cdl = has_cdl || L.jobs[j].family == tb::F_CDL;
  // device buffers from the stream-ordered pool
  std::vector<void*> owned;
  auto alloc = [&](size_t b) -> void* {
    void* p = nullptr;
    if (tb::scratch_alloc(&p, b, stream) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return p;
  };
  auto release = [&]() { for (void* p : owned) tb::scratch_free(p, stream); };
  const float* hplanes[tb::P_COUNT] = {};
  for (int p = 0; p < tb::P_COUNT; ++p) {
    hplanes[p] = L.plane[p];
    if (!L.plane[p]) continue;
    void* d = alloc(bytes);
    if (!d) { release(); return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed"); }
    L.plane[p] = static_cast<const float*>(d);
  }
  struct Back { float* dev; float* host; };  // one output plane, numSeries x seriesLen
  std::vector<Back> back;
  std::vector<std::pair<void*, std::pair<void*, size_t>>> cdl_back;  // whole candle buffers
  for (int j = 0; j < L.njobs; ++j) {
    Job& jb = L.jobs[j];
    if (jb.family == tb::F_CDL) {
      const size_t span = jb.cdl_stride > 0 ? (size_t)jb.cdl_stride * (tb::kCdlPatterns - 1) + n : n;
      const size_t b = span * 4;
      void* d = alloc(b);
      if (!d) { release(); return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed"); }
      cdl_back.push_back({d, {jb.out[0], b}});
      jb.out[0] = d;
      continue;
    }
    for (int o = 0; o < output_count(jb.family); ++o) {
      void* d = alloc(bytes);
      if (!d) { release(); return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed"); }
      back.push_back({static_cast<float*>(d), static_cast<float*>(jb.out[o])});
      jb.out[o] = d;
    }
  }
  // Rows in two chunks over the auxiliary streams (measured best on 4000x234:
  // 1.66 ms against 1.80 unchunked and 2.11 with 8 chunks; one chunk for small batches
  // and for candle outputs, whose pattern planes are strided).
  const size_t in_bytes_total = bytes * [&] { int c = 0; for (auto* p : hplanes) c += p != nullptr; return c; }();
  // TACUDA_B200_HOST_CHUNKS overrides the chunk count (1 = no pipelining)
  int nchunks = (has_cdl || in_bytes_total + back.size() * bytes < (8u << 20)) ? 1 : 2;
  if (const char* env = std::getenv("TACUDA_B200_HOST_CHUNKS")) {
    const int v = std::atoi(env);
    if (v >= 1 && v <= 64 && !has_cdl) nchunks = v;
  }
  if (nchunks > L.S) nchunks = L.S;
  cudaStream_t aux[kPipeStreams];
  cudaEvent_t fork = nullptr, done[kPipeStreams] = {};
  bool forked = false;
  if (nchunks > 1) {
    if (pipe_streams(aux) != cudaSuccess || cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess) {
      nchunks = 1;
    } else {
      for (int i = 0; i < kPipeStreams; ++i) cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
      cudaEventRecord(fork, stream);
      for (int i = 0; i < kPipeStreams; ++i) cudaStreamWaitEvent(aux[i], fork, 0);
      forked = true;
    }
  }
  const char* copy_err = nullptr;
  const int rows = (L.S + nchunks - 1) / nchunks;
  // every chunk runs the plan of the whole batch, so its rows get the bits the
  // device entry gives them (an engine's rows never depend on the other rows)
  const tb::SchedulePlan whole = tb::plan_for(L, (long long)L.S * L.T, L.T);
  for (int c = 0; c < nchunks && st == CT_STATUS_SUCCESS && !copy_err; ++c) {
    const int r0 = c * rows, r1 = std::min(L.S, r0 + rows);
    if (r0 >= r1) break;
    cudaStream_t cs = forked ? aux[c % kPipeStreams] : stream;
    const size_t off = (size_t)r0 * L.T, cnt = (size_t)(r1 - r0) * L.T;
    Launch Lc = L;
    for (int p = 0; p < tb::P_COUNT; ++p) {
      if (!hplanes[p]) continue;
      if (cudaMemcpyAsync(const_cast<float*>(L.plane[p]) + off, hplanes[p] + off, cnt * 4, cudaMemcpyHostToDevice,
                          cs) != cudaSuccess)
        copy_err = ": host to device copy failed";
      Lc.plane[p] = L.plane[p] + off;
    }
    if (copy_err) break;
    Lc.S = r1 - r0;
    for (int j = 0; j < Lc.njobs; ++j) {
      Job& jb = Lc.jobs[j];
      const int nout = jb.family == tb::F_CDL ? 1 : output_count(jb.family);
      for (int o = 0; o < nout; ++o) jb.out[o] = static_cast<char*>(jb.out[o]) + off * 4;
    }
    st = launch(Lc, (long long)cnt, L.T, &whole, cs, who);
    if (st != CT_STATUS_SUCCESS) break;
    for (const Back& b : back)
      if (cudaMemcpyAsync(b.host + off, b.dev + off, cnt * 4, cudaMemcpyDeviceToHost, cs) != cudaSuccess)
        copy_err = ": device to host copy failed";
  }
  if (forked) {
    for (int i = 0; i < kPipeStreams; ++i) {
      cudaEventRecord(done[i], aux[i]);
      cudaStreamWaitEvent(stream, done[i], 0);
      cudaEventDestroy(done[i]);
    }
    cudaEventDestroy(fork);
  }
  // every chunk has joined `stream`: buffers are freed after their last use
  if (st == CT_STATUS_SUCCESS && !copy_err)
    for (auto& b : cdl_back)
      if (cudaMemcpyAsync(b.second.first, b.first, b.second.second, cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        copy_err = ": device to host copy failed";
  release();
  if (st != CT_STATUS_SUCCESS) return st;
  if (copy_err) return fail(CT_STATUS_COPY_FAILED, std::string(who) + copy_err);
  return sync_and_check(stream, who);
}

// ------------------------------------------------------------ stream batches
//
// include/tacuda_stream.h:155-269 in the reference: one handle advances the
// state of numSeries series of one indicator by n bars per append, so that a
// run of appends gives the outputs of one batch call over the concatenated
// bars. Here every append runs the warp-scan engine on the GPU from the state
// the previous append left: the per-series recurrence carries (kept in device
// memory) and the last `hist` bars of every input row (the windows' halo),
// kept at the front of a double-buffered device staging matrix whose rows
// hold [hist bars | up to cap new bars].

struct ctStreamBatch {
  int family;
  Job job;            // validated job (outputs set per append)
  int S;
  long long seen;     // bars appended so far (per series)
  int hist, cap;      // history bars kept, new bars a staging row holds
  int nin, in_plane[4];
  int lookback, nout;
  float* stage[2];    // nin planes x S rows x (hist + cap)
  int cur;
  void* carry;        // S x Carry
  int dev;
  bool gpu_only;
};

namespace {
std::mutex g_stream_mutex;
std::vector<ctStreamBatch*> g_streams;  // live handles

bool stream_live(const ctStreamBatch* b) {
  std::lock_guard<std::mutex> lk(g_stream_mutex);
  for (auto* p : g_streams)
    if (p == b) return true;
  return false;
}

int stream_lookback(const Job& j) {
  switch (j.family) {
    case tb::F_SMA: case tb::F_EMA: case tb::F_WMA: case tb::F_BBANDS: return j.ip[0] - 1;
    case tb::F_RSI: case tb::F_ATR: case tb::F_NATR: return j.ip[0];
    case tb::F_MACD: return j.ip[1] + j.ip[2] - 2;
    default: return 0;  // OBV, AD
  }
}

ctStatus_t stream_create(const ctB200Job& u, int numSeries, ctStreamBatch** out, const char* who) {
  clear_error();
  if (!out) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null out parameter");
  *out = nullptr;
  if (numSeries <= 0) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": numSeries must be > 0");
  auto* b = new (std::nothrow) ctStreamBatch();
  if (!b) return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": allocation failed");
  // the job is validated now; its output pointers are placeholders that every
  // append replaces before launching
  ctB200Job v = u;
  for (int k = 0; k < 3; ++k) v.outputs[k] = reinterpret_cast<void*>(static_cast<uintptr_t>(256));
  ctStatus_t st = make_job(v, b->job, who);
  if (st != CT_STATUS_SUCCESS) { delete b; return st; }
  b->family = u.family;
  b->S = numSeries;
  b->seen = 0;
  b->nin = default_inputs(u.family, b->in_plane);
  b->nout = output_count(u.family);
  b->lookback = stream_lookback(b->job);
  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.njobs = 1;
  L.jobs[0] = b->job;
  b->hist = ((tb::max_lookback_halo(L) + 31) / 32) * 32;
  b->cap = 0;
  b->stage[0] = b->stage[1] = nullptr;
  b->cur = 0;
  b->gpu_only = true;
  if (cudaGetDevice(&b->dev) != cudaSuccess || cudaMalloc(&b->carry, sizeof(tb::Carry) * (size_t)numSeries) != cudaSuccess) {
    delete b;
    return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed");
  }
  {
    std::lock_guard<std::mutex> lk(g_stream_mutex);
    g_streams.push_back(b);
  }
  *out = b;
  return CT_STATUS_SUCCESS;
}

// Grow the staging rows to hold n new bars, keeping the history rows.
ctStatus_t stream_reserve(ctStreamBatch* b, int n, const char* who) {
  if (n <= b->cap) return CT_STATUS_SUCCESS;
  const int cap = std::max(n, 2 * b->cap);
  const size_t row = (size_t)b->hist + cap;
  const size_t bytes = row * (size_t)b->S * b->nin * sizeof(float);
  float* fresh[2] = {nullptr, nullptr};
  for (int i = 0; i < 2; ++i)
    if (cudaMalloc(&fresh[i], bytes) != cudaSuccess) {
      if (fresh[0]) cudaFree(fresh[0]);
      return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed");
    }
  if (b->stage[b->cur] && b->hist > 0) {
    const size_t old_row = (size_t)b->hist + b->cap;
    if (cudaMemcpy2D(fresh[0], row * sizeof(float), b->stage[b->cur], old_row * sizeof(float),
                     (size_t)b->hist * sizeof(float), (size_t)b->S * b->nin, cudaMemcpyDeviceToDevice) != cudaSuccess) {
      cudaFree(fresh[0]);
      cudaFree(fresh[1]);
      return fail(CT_STATUS_COPY_FAILED, std::string(who) + ": history copy failed");
    }
  }
  for (int i = 0; i < 2; ++i)
    if (b->stage[i]) cudaFree(b->stage[i]);
  b->stage[0] = fresh[0];
  b->stage[1] = fresh[1];
  b->cur = 0;
  b->cap = cap;
  return CT_STATUS_SUCCESS;
}

ctStatus_t stream_append(ctStreamBatch* b, int family, const float* const* ins, int n, float* const* outs,
                         const char* who) {
  clear_error();
  if (!stream_live(b)) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": invalid or destroyed batch handle");
  if (b->family != family)
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": batch was created for a different indicator");
  if (n <= 0) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": n must be > 0");
  for (int i = 0; i < b->nin; ++i)
    if (!ins[i]) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null input pointer");
  for (int k = 0; k < b->nout; ++k)
    if (!outs[k]) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null output pointer");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != b->dev)
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": batch belongs to another device");
  ctStatus_t st = stream_reserve(b, n, who);
  if (st != CT_STATUS_SUCCESS) return st;
  const cudaStream_t stream = 0;
  const size_t row = (size_t)b->hist + b->cap;
  const size_t plane_stride = row * b->S;
  float* cur = b->stage[b->cur];
  float* nxt = b->stage[b->cur ^ 1];
  // new bars after each row's history
  for (int i = 0; i < b->nin; ++i)
    if (cudaMemcpy2DAsync(cur + i * plane_stride + b->hist, row * sizeof(float), ins[i], (size_t)n * sizeof(float),
                          (size_t)n * sizeof(float), b->S, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return fail(CT_STATUS_COPY_FAILED, std::string(who) + ": host to device copy failed");
  float* dout = nullptr;
  const size_t out_elems = (size_t)n * b->S;
  if (tb::scratch_alloc(reinterpret_cast<void**>(&dout), out_elems * b->nout * sizeof(float), stream) != cudaSuccess)
    return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed");
  Launch L;
  std::memset(&L, 0, sizeof(L));
  for (int i = 0; i < b->nin; ++i) L.plane[b->in_plane[i]] = cur + i * plane_stride;
  L.T = n;
  L.S = b->S;
  L.njobs = 1;
  L.jobs[0] = b->job;
  for (int k = 0; k < b->nout; ++k) L.jobs[0].out[k] = dout + k * out_elems;
  L.st_carry = b->carry;
  L.st_seen = b->seen;
  L.st_hist = b->hist;
  L.st_row = (long long)row;
  tb::SchedulePlan plan = tb::plan_for(L, (long long)n * b->S, n);
  plan.mode = 0;  // rows continue from their kept carries: warp-per-series engine
  const cudaError_t e = tb::launch_batch(L, plan, (long long)n * b->S, stream, nullptr);
  if (e != cudaSuccess) {
    tb::scratch_free(dout, stream);
    return cuda_fail(CT_STATUS_KERNEL_FAILED, who, e);
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  for (int k = 0; k < b->nout; ++k)
    if (cudaMemcpyAsync(outs[k], dout + k * out_elems, out_elems * sizeof(float), cudaMemcpyDeviceToHost, stream) !=
        cudaSuccess) {
      tb::scratch_free(dout, stream);
      return fail(CT_STATUS_COPY_FAILED, std::string(who) + ": device to host copy failed");
    }
  // the last `hist` bars of every row become the next append's history
  if (b->hist > 0 &&
      cudaMemcpy2DAsync(nxt, row * sizeof(float), cur + n, row * sizeof(float), (size_t)b->hist * sizeof(float),
                        (size_t)b->S * b->nin, cudaMemcpyDeviceToDevice, stream) != cudaSuccess) {
    tb::scratch_free(dout, stream);
    return fail(CT_STATUS_COPY_FAILED, std::string(who) + ": history copy failed");
  }
  tb::scratch_free(dout, stream);
  const ctStatus_t ss = sync_and_check(stream, who);
  if (ss != CT_STATUS_SUCCESS) return ss;
  b->cur ^= 1;
  b->seen += n;
  return CT_STATUS_SUCCESS;
}

ctStatus_t stream_query(const ctStreamBatch* b, const char* who, const std::function<ctStatus_t()>& f) {
  clear_error();
  if (!stream_live(b)) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": invalid or destroyed batch handle");
  return f();
}
}  // namespace

ctStatus_t ct_stream_batch_destroy(ctStreamBatch_t* batch) {
  clear_error();
  if (!batch) return CT_STATUS_SUCCESS;
  {
    std::lock_guard<std::mutex> lk(g_stream_mutex);
    auto it = std::find(g_streams.begin(), g_streams.end(), batch);
    if (it == g_streams.end())
      return fail(CT_STATUS_INVALID_ARGUMENT, "ct_stream_batch_destroy: invalid or destroyed batch handle");
    g_streams.erase(it);
  }
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(batch->dev);
  for (auto* p : batch->stage)
    if (p) cudaFree(p);
  cudaFree(batch->carry);
  cudaSetDevice(cur);
  delete batch;
  return CT_STATUS_SUCCESS;
}

ctStatus_t ct_stream_batch_reset(ctStreamBatch_t* batch) {
  return stream_query(batch, "ct_stream_batch_reset", [&] {
    batch->seen = 0;  // the next append starts every series from the empty state
    return CT_STATUS_SUCCESS;
  });
}

ctStatus_t ct_stream_batch_lookback(const ctStreamBatch_t* batch, int* outLookback) {
  return stream_query(batch, "ct_stream_batch_lookback", [&] {
    if (!outLookback) return fail(CT_STATUS_INVALID_ARGUMENT, "ct_stream_batch_lookback: null out parameter");
    *outLookback = batch->lookback;
    return CT_STATUS_SUCCESS;
  });
}

ctStatus_t ct_stream_batch_series(const ctStreamBatch_t* batch, int* outSeries) {
  return stream_query(batch, "ct_stream_batch_series", [&] {
    if (!outSeries) return fail(CT_STATUS_INVALID_ARGUMENT, "ct_stream_batch_series: null out parameter");
    *outSeries = batch->S;
    return CT_STATUS_SUCCESS;
  });
}

ctStatus_t ct_stream_batch_outputs(const ctStreamBatch_t* batch, int* outCount) {
  return stream_query(batch, "ct_stream_batch_outputs", [&] {
    if (!outCount) return fail(CT_STATUS_INVALID_ARGUMENT, "ct_stream_batch_outputs: null out parameter");
    *outCount = batch->nout;
    return CT_STATUS_SUCCESS;
  });
}

ctStatus_t ct_stream_batch_bars(const ctStreamBatch_t* batch, long long* outBars) {
  return stream_query(batch, "ct_stream_batch_bars", [&] {
    if (!outBars) return fail(CT_STATUS_INVALID_ARGUMENT, "ct_stream_batch_bars: null out parameter");
    *outBars = batch->seen;
    return CT_STATUS_SUCCESS;
  });
}

ctStatus_t ct_stream_batch_set_exec(ctStreamBatch_t* batch, ctStreamExec_t exec) {
  return stream_query(batch, "ct_stream_batch_set_exec", [&] {
    if (exec == CT_STREAM_EXEC_AUTO || exec == CT_STREAM_EXEC_GPU) return CT_STATUS_SUCCESS;
    if (exec == CT_STREAM_EXEC_CPU)
      return fail(CT_STATUS_UNSUPPORTED, "ct_stream_batch_set_exec: this library runs every append on the GPU");
    return fail(CT_STATUS_INVALID_ARGUMENT, "ct_stream_batch_set_exec: unknown execution policy");
  });
}

#define TB_STREAM_PERIOD_CREATE(name, fam)                                                   \
  ctStatus_t ct_##name##_stream_batch_create(int period, int numSeries, ctStreamBatch_t** out) { \
    return stream_create(job_of(fam, period), numSeries, out, "ct_" #name "_stream_batch_create"); \
  }
TB_STREAM_PERIOD_CREATE(sma, tb::F_SMA)
TB_STREAM_PERIOD_CREATE(ema, tb::F_EMA)
TB_STREAM_PERIOD_CREATE(wma, tb::F_WMA)
TB_STREAM_PERIOD_CREATE(rsi, tb::F_RSI)
TB_STREAM_PERIOD_CREATE(atr, tb::F_ATR)
TB_STREAM_PERIOD_CREATE(natr, tb::F_NATR)
#undef TB_STREAM_PERIOD_CREATE

ctStatus_t ct_obv_stream_batch_create(int numSeries, ctStreamBatch_t** out) {
  return stream_create(job_of(tb::F_OBV), numSeries, out, "ct_obv_stream_batch_create");
}
ctStatus_t ct_ad_stream_batch_create(int numSeries, ctStreamBatch_t** out) {
  return stream_create(job_of(tb::F_AD), numSeries, out, "ct_ad_stream_batch_create");
}
ctStatus_t ct_macd_stream_batch_create(int fastPeriod, int slowPeriod, int signalPeriod, int numSeries,
                                       ctStreamBatch_t** out) {
  return stream_create(job_of(tb::F_MACD, fastPeriod, slowPeriod, signalPeriod), numSeries, out,
                       "ct_macd_stream_batch_create");
}
ctStatus_t ct_bbands_stream_batch_create(int period, float upperMul, float lowerMul, int numSeries,
                                         ctStreamBatch_t** out) {
  return stream_create(job_of(tb::F_BBANDS, period, 0, 0, upperMul, lowerMul), numSeries, out,
                       "ct_bbands_stream_batch_create");
}

#define TB_STREAM_CLOSE_APPEND(name, fam)                                                          \
  ctStatus_t ct_##name##_stream_batch_append(ctStreamBatch_t* batch, const float* closes, int n, float* outs) { \
    const float* in[1] = {closes};                                                                 \
    float* o[1] = {outs};                                                                          \
    return stream_append(batch, fam, in, n, o, "ct_" #name "_stream_batch_append");               \
  }
TB_STREAM_CLOSE_APPEND(sma, tb::F_SMA)
TB_STREAM_CLOSE_APPEND(ema, tb::F_EMA)
TB_STREAM_CLOSE_APPEND(wma, tb::F_WMA)
TB_STREAM_CLOSE_APPEND(rsi, tb::F_RSI)
#undef TB_STREAM_CLOSE_APPEND

ctStatus_t ct_atr_stream_batch_append(ctStreamBatch_t* batch, const float* highs, const float* lows,
                                      const float* closes, int n, float* outs) {
  const float* in[3] = {highs, lows, closes};
  float* o[1] = {outs};
  return stream_append(batch, tb::F_ATR, in, n, o, "ct_atr_stream_batch_append");
}
ctStatus_t ct_natr_stream_batch_append(ctStreamBatch_t* batch, const float* highs, const float* lows,
                                       const float* closes, int n, float* outs) {
  const float* in[3] = {highs, lows, closes};
  float* o[1] = {outs};
  return stream_append(batch, tb::F_NATR, in, n, o, "ct_natr_stream_batch_append");
}
ctStatus_t ct_obv_stream_batch_append(ctStreamBatch_t* batch, const float* closes, const float* volumes, int n,
                                      float* outs) {
  const float* in[2] = {closes, volumes};
  float* o[1] = {outs};
  return stream_append(batch, tb::F_OBV, in, n, o, "ct_obv_stream_batch_append");
}
ctStatus_t ct_ad_stream_batch_append(ctStreamBatch_t* batch, const float* highs, const float* lows,
                                     const float* closes, const float* volumes, int n, float* outs) {
  const float* in[4] = {highs, lows, closes, volumes};
  float* o[1] = {outs};
  return stream_append(batch, tb::F_AD, in, n, o, "ct_ad_stream_batch_append");
}
ctStatus_t ct_macd_stream_batch_append(ctStreamBatch_t* batch, const float* closes, int n, float* outMacd,
                                       float* outSignal, float* outHist) {
  const float* in[1] = {closes};
  float* o[3] = {outMacd, outSignal, outHist};
  return stream_append(batch, tb::F_MACD, in, n, o, "ct_macd_stream_batch_append");
}
ctStatus_t ct_bbands_stream_batch_append(ctStreamBatch_t* batch, const float* closes, int n, float* outUpper,
                                         float* outMiddle, float* outLower) {
  const float* in[1] = {closes};
  float* o[3] = {outUpper, outMiddle, outLower};
  return stream_append(batch, tb::F_BBANDS, in, n, o, "ct_bbands_stream_batch_append");
}

// ------------------------------------------------------------ plans

ctStatus_t ct_b200_plan_create(const ctB200Job* jobs, int numJobs, const int64_t* hostOffsets, int numSeries,
                               int64_t seriesLen, ctB200Plan** out) {
  clear_error();
  const char* who = "ct_b200_plan_create";
  if (!out || !jobs || numJobs <= 0 || numJobs > tb::kMaxJobs || numSeries <= 0 || (!hostOffsets && seriesLen <= 0))
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null pointer or invalid size");
  ctB200Plan* plan = new (std::nothrow) ctB200Plan();
  if (!plan) return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": out of host memory");
  plan->njobs = numJobs;
  plan->numSeries = numSeries;
  plan->seriesLen = seriesLen;
  plan->ragged = hostOffsets != nullptr;
  plan->jobs.resize(numJobs);
  for (int j = 0; j < numJobs; ++j) {
    ctB200Job u = jobs[j];
    // outputs are supplied at execution; validate shape with a placeholder
    for (int o = 0; o < 3; ++o) if (!u.outputs[o]) u.outputs[o] = reinterpret_cast<void*>(16);
    const ctStatus_t st = make_job(u, plan->jobs[j], who);
    if (st != CT_STATUS_SUCCESS) { delete plan; return st; }
  }
  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.S = numSeries;
  L.njobs = numJobs;
  for (int j = 0; j < numJobs; ++j) L.jobs[j] = plan->jobs[j];
  cudaGetDevice(&plan->device);
  if (plan->ragged) {
    std::vector<long long> len(numSeries);
    long long total = 0, mx = 0;
    for (int s = 0; s < numSeries; ++s) {
      len[s] = hostOffsets[s + 1] - hostOffsets[s];
      if (len[s] < 0) { delete plan; return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": offsets decrease"); }
      total += len[s];
      mx = std::max(mx, len[s]);
    }
    std::vector<int> order(numSeries);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return len[a] > len[b]; });
    if (cudaMalloc(&plan->d_order, sizeof(int) * numSeries) != cudaSuccess) {
      delete plan;
      return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed");
    }
    if (cudaMemcpy(plan->d_order, order.data(), sizeof(int) * numSeries, cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(plan->d_order);
      delete plan;
      return fail(CT_STATUS_COPY_FAILED, std::string(who) + ": order upload failed");
    }
    plan->total = total;
    plan->maxlen = mx;
  } else {
    plan->total = seriesLen * (long long)numSeries;
    plan->maxlen = seriesLen;
  }
  plan->sched = tb::plan_for(L, plan->total, plan->maxlen);
  *out = plan;
  return CT_STATUS_SUCCESS;
}

static ctStatus_t plan_launch(const ctB200Plan* plan, const ctB200Series* series, const ctB200Job* jobs,
                              int numJobs, const tb::SchedulePlan& sched, cudaStream_t stream, const char* who,
                              tb::LaunchStats* stats) {
  if (!plan) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null plan");
  Launch L;
  ctStatus_t st = build_launch(series, jobs, numJobs, L, who);
  if (st != CT_STATUS_SUCCESS) return st;
  if (numJobs != plan->njobs || series->numSeries != plan->numSeries || (series->offsets != nullptr) != plan->ragged ||
      (!plan->ragged && series->seriesLen != plan->seriesLen))
    return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": batch does not match the plan");
  for (int j = 0; j < numJobs; ++j) {
    const Job& a = L.jobs[j];
    const Job& b = plan->jobs[j];
    if (a.family != b.family || a.ip[0] != b.ip[0] || a.ip[1] != b.ip[1] || a.ip[2] != b.ip[2])
      return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": jobs do not match the plan");
  }
  L.order = plan->d_order;
  return launch(L, plan->total, plan->maxlen, &sched, stream, who, stats);
}

ctStatus_t ct_b200_plan_execute(const ctB200Plan* plan, const ctB200Series* series, const ctB200Job* jobs,
                                int numJobs, cudaStream_t stream) {
  clear_error();
  const char* who = "ct_b200_plan_execute";
  const ctStatus_t st = plan_launch(plan, series, jobs, numJobs, plan ? plan->sched : tb::SchedulePlan{}, stream,
                                    who, nullptr);
  if (st != CT_STATUS_SUCCESS) return st;
  return finish(stream, who);
}

ctStatus_t ct_b200_plan_autotune(ctB200Plan* plan, const ctB200Series* series, const ctB200Job* jobs, int numJobs,
                                 cudaStream_t stream) {
  clear_error();
  const char* who = "ct_b200_plan_autotune";
  if (!plan) return fail(CT_STATUS_INVALID_ARGUMENT, std::string(who) + ": null plan");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  tb::SchedulePlan bestPlan = plan->sched;
  // candidates: the row-parallel engine; the warp-scan engine over round
  // widths and block sizes; the look-back engine where its tiles fit the rows
  std::vector<tb::SchedulePlan> cands;
  // row-parallel engine: the job set whole (one row group per CTA) or split
  // into partitions with two row groups per CTA
  for (const int pg : {0x11, 0x42, 0x52, 0x62}) {
    tb::SchedulePlan cand;
    cand.mode = 1;
    cand.parts = pg >> 4;
    cand.groups = pg & 15;
    cands.push_back(cand);
  }
  for (int mode : {0, 2})
    for (int ki : {4, 8, 16}) {
      if (ki == 4 && plan->maxlen > 4096) continue;
      if (mode == 2 && plan->maxlen < 4ll * 32 * ki) continue;
      for (int wi : {4, 8, 16}) {
        tb::SchedulePlan cand;
        cand.mode = mode;
        cand.k = ki;
        cand.warps_per_block = wi;
        cands.push_back(cand);
      }
    }
  plan->tried.clear();
  for (const tb::SchedulePlan& cand : cands) {
    ctStatus_t st = plan_launch(plan, series, jobs, numJobs, cand, stream, who, nullptr);  // warm-up
    if (st != CT_STATUS_SUCCESS) continue;
    cudaEventRecord(e0, stream);
    for (int r = 0; r < 3; ++r) plan_launch(plan, series, jobs, numJobs, cand, stream, who, nullptr);
    cudaEventRecord(e1, stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) continue;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    plan->tried.push_back({cand, ms / 3.0f});
    if (ms < best) {
      best = ms;
      bestPlan = cand;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  clear_error();
  plan->sched = bestPlan;
  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.S = plan->numSeries;
  L.njobs = plan->njobs;
  for (int j = 0; j < plan->njobs; ++j) L.jobs[j] = plan->jobs[j];
  tb::remember_plan(tb::shape_key(L, plan->total, plan->maxlen), bestPlan);
  return CT_STATUS_SUCCESS;
}

ctStatus_t ct_b200_plan_describe(const ctB200Plan* plan, int* engine, int* barsPerLane, int* warpsPerBlock,
                                 int* blocks) {
  clear_error();
  if (!plan) return fail(CT_STATUS_INVALID_ARGUMENT, "ct_b200_plan_describe: null plan");
  if (engine) *engine = plan->sched.mode;
  if (barsPerLane) *barsPerLane = plan->sched.k;
  if (warpsPerBlock) *warpsPerBlock = plan->sched.warps_per_block;
  if (blocks) *blocks = plan->sched.max_blocks;
  return CT_STATUS_SUCCESS;
}

ctStatus_t ct_b200_plan_describe_rows(const ctB200Plan* plan, int* parts, int* groups) {
  clear_error();
  if (!plan) return fail(CT_STATUS_INVALID_ARGUMENT, "ct_b200_plan_describe_rows: null plan");
  if (parts) *parts = plan->sched.parts;
  if (groups) *groups = plan->sched.groups;
  return CT_STATUS_SUCCESS;
}

int ct_b200_plan_candidates_rows(const ctB200Plan* plan, int maxOut, int* parts, int* groups) {
  clear_error();
  if (!plan) return 0;
  const int n = (int)plan->tried.size();
  for (int i = 0; i < n && i < maxOut; ++i) {
    const ctB200Plan::Tried& t = plan->tried[(size_t)i];
    if (parts) parts[i] = t.plan.parts;
    if (groups) groups[i] = t.plan.groups;
  }
  return n;
}

int ct_b200_plan_candidates(const ctB200Plan* plan, int maxOut, int* engine, int* barsPerLane, int* warpsPerBlock,
                            float* ms) {
  clear_error();
  if (!plan) return 0;
  const int n = (int)plan->tried.size();
  for (int i = 0; i < n && i < maxOut; ++i) {
    const ctB200Plan::Tried& t = plan->tried[(size_t)i];
    if (engine) engine[i] = t.plan.mode;
    if (barsPerLane) barsPerLane[i] = t.plan.k;
    if (warpsPerBlock) warpsPerBlock[i] = t.plan.warps_per_block;
    if (ms) ms[i] = t.ms;
  }
  return n;
}

ctStatus_t ct_b200_plan_destroy(ctB200Plan* plan) {
  clear_error();
  if (!plan) return CT_STATUS_SUCCESS;
  if (plan->d_order) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(plan->device);
    cudaFree(plan->d_order);
    cudaSetDevice(cur);
  }
  delete plan;
  return CT_STATUS_SUCCESS;
}

// ------------------------------------------------------------ host batch API

static ctStatus_t host_run(const std::vector<const float*>& hin, const std::vector<float*>& hout, size_t n,
                           cudaStream_t stream, const char* who,
                           ctStatus_t (*dev)(const std::vector<const float*>&, const std::vector<float*>&, void*,
                                             cudaStream_t),
                           void* ctx) {
  std::vector<void*> owned;
  auto release = [&]() { for (void* p : owned) tb::scratch_free(p, stream); };
  std::vector<const float*> din;
  std::vector<float*> dout;
  for (const float* h : hin) {
    void* d = nullptr;
    if (tb::scratch_alloc(&d, n * 4, stream) != cudaSuccess) { release(); return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed"); }
    owned.push_back(d);
    if (cudaMemcpyAsync(d, h, n * 4, cudaMemcpyHostToDevice, stream) != cudaSuccess) { release(); return fail(CT_STATUS_COPY_FAILED, std::string(who) + ": copy failed"); }
    din.push_back(static_cast<const float*>(d));
  }
  for (size_t i = 0; i < hout.size(); ++i) {
    void* d = nullptr;
    if (tb::scratch_alloc(&d, n * 4, stream) != cudaSuccess) { release(); return fail(CT_STATUS_ALLOC_FAILED, std::string(who) + ": device allocation failed"); }
    owned.push_back(d);
    dout.push_back(static_cast<float*>(d));
  }
  // run on a private non-null stream view so the device call does not sync early
  ctStatus_t st = dev(din, dout, ctx, stream == 0 ? cudaStreamPerThread : stream);
  if (st != CT_STATUS_SUCCESS) { release(); return st; }
  cudaStream_t s2 = stream == 0 ? cudaStreamPerThread : stream;
  for (size_t i = 0; i < hout.size(); ++i)
    if (cudaMemcpyAsync(hout[i], dout[i], n * 4, cudaMemcpyDeviceToHost, s2) != cudaSuccess) { release(); return fail(CT_STATUS_COPY_FAILED, std::string(who) + ": copy failed"); }
  release();
  return sync_and_check(s2, who);
}

struct HostArgs { int len, n, p0, p1, p2, p3; float f0, f1; };

#define TB_HOST_S1(NAME)                                                                                   \
  ctStatus_t ct_##NAME##_batch(const float* host_inputs, float* host_outputs, int seriesLen, int numSeries, \
                               int period, int, cudaStream_t stream) {                                     \
    clear_error();                                                                                         \
    if (!host_inputs || !host_outputs || seriesLen <= 0 || numSeries <= 0)                                  \
      return fail(CT_STATUS_INVALID_ARGUMENT, "ct_" #NAME "_batch: null pointer or invalid size");          \
    HostArgs a{seriesLen, numSeries, period, 0, 0, 0, 0.f, 0.f};                                           \
    return host_run({host_inputs}, {host_outputs}, (size_t)seriesLen * numSeries, stream, "ct_" #NAME "_batch", \
                    [](const std::vector<const float*>& i, const std::vector<float*>& o, void* c, cudaStream_t s) { \
                      const HostArgs& h = *static_cast<HostArgs*>(c);                                      \
                      return ct_##NAME##_batch_d(i[0], o[0], h.len, h.n, h.p0, 0, s);                      \
                    }, &a);                                                                                \
  }
TB_HOST_S1(sma)
TB_HOST_S1(ema)
TB_HOST_S1(rsi)
#undef TB_HOST_S1

ctStatus_t ct_atr_batch(const float* h, const float* l, const float* c, float* out, int seriesLen, int numSeries,
                        int period, float, int, cudaStream_t stream) {
  clear_error();
  if (!h || !l || !c || !out || seriesLen <= 0 || numSeries <= 0)
    return fail(CT_STATUS_INVALID_ARGUMENT, "ct_atr_batch: null pointer or invalid size");
  HostArgs a{seriesLen, numSeries, period, 0, 0, 0, 0.f, 0.f};
  return host_run({h, l, c}, {out}, (size_t)seriesLen * numSeries, stream, "ct_atr_batch",
                  [](const std::vector<const float*>& i, const std::vector<float*>& o, void* x, cudaStream_t s) {
                    const HostArgs& q = *static_cast<HostArgs*>(x);
                    return ct_atr_batch_d(i[0], i[1], i[2], o[0], q.len, q.n, q.p0, 0.f, 0, s);
                  }, &a);
}

ctStatus_t ct_macd_batch(const float* in, float* m, float* sg, float* hs, int seriesLen, int numSeries, int fast,
                         int slow, int signal, int maType, int, cudaStream_t stream) {
  clear_error();
  if (!in || !m || !sg || !hs || seriesLen <= 0 || numSeries <= 0)
    return fail(CT_STATUS_INVALID_ARGUMENT, "ct_macd_batch: null pointer or invalid size");
  HostArgs a{seriesLen, numSeries, fast, slow, signal, maType, 0.f, 0.f};
  return host_run({in}, {m, sg, hs}, (size_t)seriesLen * numSeries, stream, "ct_macd_batch",
                  [](const std::vector<const float*>& i, const std::vector<float*>& o, void* x, cudaStream_t s) {
                    const HostArgs& q = *static_cast<HostArgs*>(x);
                    return ct_macd_batch_d(i[0], o[0], o[1], o[2], q.len, q.n, q.p0, q.p1, q.p2, q.p3, 0, s);
                  }, &a);
}

ctStatus_t ct_bbands_batch(const float* in, float* u, float* mid, float* lo, int seriesLen, int numSeries, int period,
                           float upperMul, float lowerMul, int, cudaStream_t stream) {
  clear_error();
  if (!in || !u || !mid || !lo || seriesLen <= 0 || numSeries <= 0)
    return fail(CT_STATUS_INVALID_ARGUMENT, "ct_bbands_batch: null pointer or invalid size");
  HostArgs a{seriesLen, numSeries, period, 0, 0, 0, upperMul, lowerMul};
  return host_run({in}, {u, mid, lo}, (size_t)seriesLen * numSeries, stream, "ct_bbands_batch",
                  [](const std::vector<const float*>& i, const std::vector<float*>& o, void* x, cudaStream_t s) {
                    const HostArgs& q = *static_cast<HostArgs*>(x);
                    return ct_bbands_batch_d(i[0], o[0], o[1], o[2], q.len, q.n, q.p0, q.f0, q.f1, 0, s);
                  }, &a);
}

ctStatus_t ct_stochastic_batch(const float* h, const float* l, const float* c, float* k, float* d, int seriesLen,
                               int numSeries, int kPeriod, int dPeriod, int, cudaStream_t stream) {
  clear_error();
  if (!h || !l || !c || !k || !d || seriesLen <= 0 || numSeries <= 0)
    return fail(CT_STATUS_INVALID_ARGUMENT, "ct_stochastic_batch: null pointer or invalid size");
  HostArgs a{seriesLen, numSeries, kPeriod, dPeriod, 0, 0, 0.f, 0.f};
  return host_run({h, l, c}, {k, d}, (size_t)seriesLen * numSeries, stream, "ct_stochastic_batch",
                  [](const std::vector<const float*>& i, const std::vector<float*>& o, void* x, cudaStream_t s) {
                    const HostArgs& q = *static_cast<HostArgs*>(x);
                    return ct_stochastic_batch_d(i[0], i[1], i[2], o[0], o[1], q.len, q.n, q.p0, q.p1, 0, s);
                  }, &a);
}

}  // extern "C"
