// Candlestick engine (bar-parallel): every selected CDL pattern of every bar.
//
// Candle decisions read at most six bars back and TA-Lib's trailing averages
// of at most ten bars before an anchor up to five bars back
// (include/utils/CandleUtils.h:37-63, 1466-1495), so a bar needs only the 16
// bars before it: rows split into independent tiles of kTileBars bars, one
// thread per bar. A block stages the tile and its halo of open/high/low/close
// with coalesced loads, computes the three FP64 ranges of every staged bar,
// then the four distinct trailing means (body/10, high-low/10, shadows/10,
// high-low/5) of every anchor, each summed oldest first and divided once as
// the reference's candle_average_d does, and finally evaluates the patterns of
// the mask, one coalesced int32 (or float) store per pattern and bar.
// Warm-up bars (before the pattern's lookback) are 0.
#pragma once

#include "engine.h"
#include "cdl_rules.cuh"

namespace tb {
namespace cdl {

constexpr int kTileBars = 256;             // bars per tile = threads per block
constexpr int kHalo = 16;                  // staged bars before the tile
constexpr int kSpan = kTileBars + kHalo;
constexpr int kAnchors = kTileBars + rules::kCdlBack;

struct TileSmem {
  float o[kSpan], h[kSpan], l[kSpan], c[kSpan];
  double rng[3][kSpan];         // body, high-low, shadows of each staged bar
  double us[kSpan], ls[kSpan];  // upper and lower shadow of each staged bar
  double mean[4][kAnchors];     // trailing mean of each table slot at anchors t0-5 ..
};

// Bar view over the staged tile with the interface the pattern functions use.
struct TileBars {
  const TileSmem* s;
  int i;        // staged index of the bar (kHalo + bar - t0)
  long long t;  // bar index within the row
  __device__ __forceinline__ float O(int d) const { return s->o[i - d]; }
  __device__ __forceinline__ float H(int d) const { return s->h[i - d]; }
  __device__ __forceinline__ float L(int d) const { return s->l[i - d]; }
  __device__ __forceinline__ float C(int d) const { return s->c[i - d]; }
  __device__ __forceinline__ double RB(int d) const { return s->rng[0][i - d]; }
  __device__ __forceinline__ double US(int d) const { return s->us[i - d]; }
  __device__ __forceinline__ double LS(int d) const { return s->ls[i - d]; }
  __device__ __forceinline__ int COL(int d) const { return C(d) >= O(d) ? 1 : -1; }
  __device__ __forceinline__ float TOP(int d) const { return fmaxf(O(d), C(d)); }
  __device__ __forceinline__ float BOT(int d) const { return fminf(O(d), C(d)); }
  __device__ __forceinline__ bool BGAP_UP(int a, int b) const { return fminf(O(a), C(a)) > fmaxf(O(b), C(b)); }
  __device__ __forceinline__ bool BGAP_DN(int a, int b) const { return fmaxf(O(a), C(a)) < fminf(O(b), C(b)); }
  __device__ __forceinline__ bool RGAP_UP(int a, int b) const { return L(a) > H(b); }
  __device__ __forceinline__ bool RGAP_DN(int a, int b) const { return H(a) < L(b); }
  // TA-Lib candle average of setting st anchored at bar t-d:
  // factor * (sum / count) / divisor, the mean precomputed per anchor.
  __device__ __forceinline__ double AVG(int st, int d) const {
    const int slot = rules::set_slot(st);
    const double factor = (double)rules::set_factor(st);
    if (slot < 0) return factor * RB(d);
    const double m = s->mean[slot][i - kHalo - d + rules::kCdlBack];
    return slot == 2 ? factor * m / 2.0 : factor * m;
  }
};

// Range type of each table slot: body, high-low, shadows, high-low.
__device__ __forceinline__ int slot_range(int slot) { return slot == 0 ? 0 : (slot == 2 ? 2 : 1); }

struct TileArgs {
  const float* plane[4];           // open, high, low, close
  const long long* offsets;        // ragged row starts or nullptr
  const int* order;                // processing order of the rows or nullptr
  long long T;
  int S;
  int njobs;
  Job jobs[kMaxJobs];              // candle jobs only
};

__global__ void __launch_bounds__(kTileBars) tile_kernel(const __grid_constant__ TileArgs A) {
  __shared__ TileSmem sm;
  const int tid = threadIdx.x;
  for (long long pass = 0;; ++pass) {
    const long long idx = pass * gridDim.x + ((pass & 1) ? (gridDim.x - 1 - blockIdx.x) : blockIdx.x);
    if (idx >= A.S) break;
    const int s = A.order ? A.order[idx] : (int)idx;
    long long base, n;
    if (A.offsets) {
      base = A.offsets[s];
      n = A.offsets[s + 1] - base;
    } else {
      base = (long long)s * A.T;
      n = A.T;
    }
    for (long long t0 = 0; t0 < n; t0 += kTileBars) {
      __syncthreads();  // previous tile's readers are done
      for (int i = tid; i < kSpan; i += kTileBars) {
        const long long t = t0 - kHalo + i;
        const bool ok = t >= 0 && t < n;
        const long long g = base + (ok ? t : 0);
        const float o = ok ? A.plane[0][g] : 0.0f, h = ok ? A.plane[1][g] : 0.0f;
        const float l = ok ? A.plane[2][g] : 0.0f, c = ok ? A.plane[3][g] : 0.0f;
        sm.o[i] = o; sm.h[i] = h; sm.l[i] = l; sm.c[i] = c;
        sm.rng[0][i] = rules::cdl_range(rules::CR_BODY, o, h, l, c);
        sm.rng[1][i] = rules::cdl_range(rules::CR_HL, o, h, l, c);
        sm.rng[2][i] = rules::cdl_range(rules::CR_SHADOW, o, h, l, c);
        sm.us[i] = (double)h - fmax((double)o, (double)c);
        sm.ls[i] = fmin((double)o, (double)c) - (double)l;
      }
      __syncthreads();
      for (int j = tid; j < 4 * kAnchors; j += kTileBars) {
        const int slot = j / kAnchors, a = j - slot * kAnchors;
        const long long ta = t0 - rules::kCdlBack + a;  // anchor bar in the row
        const int per = rules::kSlotPeriod[slot];
        const int ia = kHalo - rules::kCdlBack + a;     // staged index of the anchor
        const double* r = sm.rng[slot_range(slot)];
        double m;
        const long long start = ta - per < 0 ? 0 : ta - per;
        const long long cnt = ta - start;
        if (cnt <= 0) {
          m = ta >= 0 ? r[ia] : 0.0;
        } else {
          double sum = 0.0;
          for (long long b = start; b < ta; ++b) sum += r[ia - (int)(ta - b)];
          m = sum / (double)cnt;
        }
        sm.mean[slot][a] = m;
      }
      __syncthreads();
      const long long t = t0 + tid;
      if (t < n) {
        TileBars b{&sm, kHalo + tid, t};
        for (int jb = 0; jb < A.njobs; ++jb) {
          const Job& j = A.jobs[jb];
          uint64_t mask = j.cdl_mask;
          while (mask) {
            const int k = __ffsll((long long)mask) - 1;
            mask &= mask - 1;
            const int v = t >= rules::kCdlLookbackDev[k] ? rules::cdl_eval(k, b) : 0;
            const long long at = (long long)k * j.cdl_stride + base + t;
            if (j.cdl_int32) reinterpret_cast<int*>(j.out[0])[at] = v;
            else reinterpret_cast<float*>(j.out[0])[at] = (float)v;
          }
        }
      }
    }
  }
}

}  // namespace cdl
}  // namespace tb
