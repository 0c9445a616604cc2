// Launch descriptors shared by the host scheduler and the device engine.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tb {

// Indicator families the engine evaluates. Each maps to one reference batch
// entry point (ct_<family>_batch_d) except CDL, which evaluates any subset of
// the candle patterns in one pass. New families are appended after CDL so the
// public ids stay stable.
enum Family : int {
  F_SMA = 0, F_EMA, F_WMA, F_RSI, F_MACD, F_ATR, F_NATR, F_TRANGE, F_ADX, F_DX,
  F_BBANDS, F_STOCH, F_CCI, F_OBV, F_AD, F_ADOSC, F_MFI, F_WILLR, F_SUM, F_MIN,
  F_MAX, F_STDDEV, F_VAR, F_LINEARREG, F_CORREL, F_DEMA, F_TEMA, F_T3, F_CDL,
  F_ROC, F_RMA, F_MEDPRICE, F_TYPPRICE, F_MIDPRICE, F_ROCP, F_ROCR, F_ROCR100, F_MOM,
  F_AVGPRICE, F_WCLPRICE, F_MIDPOINT, F_RMEAN, F_RMAX, F_RMIN, F_RSTD, F_IBS, F_MARKETFI, F_QSTICK,
  F_AROON, F_AROONOSC,
  F_COUNT
};

// Input planes of a launch. Single-input families read in[0] of their job.
enum Plane : int { P_OPEN = 0, P_HIGH, P_LOW, P_CLOSE, P_VOLUME, P_AUX, P_COUNT };

constexpr int kMaxJobs = 24;
constexpr int kMaxOut = 3;
constexpr int kCdlPatterns = 63;

struct Job {
  int family;
  int ip[3];        // integer parameters (periods) in reference order
  double fp[4];     // real parameters and host-precomputed coefficients
  int in[4];        // plane index of each logical input
  void* out[kMaxOut];
  // CDL only: pattern k is written to out[0] + k * cdl_stride elements when bit
  // k of the mask is set; int32 when cdl_int32 else float32.
  uint64_t cdl_mask;
  long long cdl_stride;
  int cdl_int32;
  int halo;         // bars of history this job reads before a round
  int lb_slot;      // first look-back descriptor slot of this job (look-back mode)
  int prec;         // 0 FP64, 1 FP32, 2 compensated FP32, 3 FP32 with FP64 carries
};

struct LbDesc;

struct Launch {
  const float* plane[P_COUNT];
  const long long* offsets;  // ragged row starts (S+1 entries) or nullptr
  const int* order;          // processing order of series (longest first) or nullptr
  long long T;               // uniform row length when offsets == nullptr
  long long max_len;         // longest row of the batch
  int S;
  int njobs;
  int halo;                  // multiple of 32, >= every job's halo
  unsigned plane_mask;       // planes staged in shared memory
  int need_tp;               // stage the FP64 typical price ((h+l)+c)/3
  int* sched;                // [0] series counter, [1] finished warps (self-resetting)
  int total_warps;
  int* err;                  // look-back error word of this launch (0 = ok), or nullptr
  int* sticky;               // per-device error word: bit 0 set when a bounded wait ran out
  int stall_test;            // test knob: one wait of the launch is made to run out (short limit)
  // look-back mode: series split into one-round tiles taken in order
  int lb;
  unsigned long long* lb_counter;  // next tile (zeroed before the launch)
  long long lb_tiles;        // total tiles
  long long* lb_tile_start;  // ragged: first tile of each series (S+1), else nullptr
  LbDesc* lb_desc;           // lb_tiles * lb_nslots descriptors (zeroed)
  int lb_nslots;
  // streaming append: rows continue earlier appends. Bar t of row s (t counted
  // from the row's first bar ever) is at plane[s*st_row + st_hist - st_seen + t]
  // for t >= st_seen - st_hist; the T new bars start at st_seen; outputs go to
  // out[s*T + t - st_seen]; carries persist in st_carry (S x njobs). Null
  // st_carry: an ordinary batch.
  void* st_carry;
  long long st_seen, st_hist, st_row;
  Job jobs[kMaxJobs];
};

}  // namespace tb
