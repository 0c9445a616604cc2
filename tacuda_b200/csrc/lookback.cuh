// Decoupled look-back between the tiles of a long series.
//
// A series longer than a few rounds is split into tiles of one round each,
// handed to warps in order by an atomic counter, so a tile only ever waits for
// tiles already taken by running warps. For every recurrence stage a tile
// publishes, as soon as its bars are staged, the affine map of the whole tile
// assuming the stage is past its warm-up (AGGREGATE), and later the exact
// state after its last bar (INCLUSIVE). A tile resolves its incoming state
// from the aggregates of its predecessors back to a fixed anchor whose
// inclusive state it waits for (see lb_resolve), so results are reproducible.
// Whether a tile starts past the warm-up follows from the row's first counted
// bar f, resolved first as a "first index" carry. Every wait is bounded; a
// timeout sets the launch error word and the tile continues (results of such
// a launch are reported invalid by the synchronous entry points).
#pragma once

#include "common.cuh"

namespace tb {

struct __align__(16) LbDesc {
  int flag;   // 0 nothing, 1 aggregate, 2 inclusive
  int f;      // first-index carries: local (aggregate) / inclusive value, -1 = none
  int pad0, pad1;
  double A[3], B[3], Y[3];
};

constexpr int kLbAgg = 1, kLbInc = 2;
constexpr long long kLbSpinLimit = 1ll << 26;  // about a second of polling

__device__ __forceinline__ int lb_load_flag(const LbDesc* d) {
  return *reinterpret_cast<const volatile int*>(&d->flag);
}

__device__ __forceinline__ void lb_store_flag(LbDesc* d, int v) {
  __threadfence();
  *reinterpret_cast<volatile int*>(&d->flag) = v;
}

// Wait (bounded) until flag >= want; returns the flag or 0 on timeout.
__device__ __forceinline__ int lb_wait(const LbDesc* d, int want, int* err) {
  long long spins = 0;
  int v;
  while ((v = lb_load_flag(d)) < want) {
    if (++spins > kLbSpinLimit) {
      atomicExch(err, 1);
      return 0;
    }
    __nanosleep(32);
  }
  __threadfence();
  return v;
}

// First-index carry: the earliest bar with a property (first non-NaN input,
// first non-finite pair). local = this tile's earliest such bar or -1.
// Lane 0 performs the protocol; the result is broadcast.
__device__ __forceinline__ int lb_first_index(LbDesc* base, long long stride, int tile, int local, int* err, int lane) {
  int res = -1;
  if (lane == 0) {
    LbDesc* me = base + (long long)tile * stride;
    if (tile == 0) {
      res = local;
    } else {
      me->f = local;
      lb_store_flag(me, kLbAgg);
      int best = -1;
      int j = tile - 1;
      for (; j >= 0; --j) {
        const LbDesc* d = base + (long long)j * stride;
        const int fl = lb_wait(d, kLbAgg, err);
        if (fl == 0) break;
        const int fv = *reinterpret_cast<const volatile int*>(&d->f);
        if (fl == kLbInc) {
          if (fv >= 0) best = fv;
          break;
        }
        if (fv >= 0) best = fv;
      }
      res = best >= 0 ? best : local;
    }
    me->f = res;
    lb_store_flag(me, kLbInc);
  }
  return __shfl_sync(kFull, res, 0);
}

// Resolve the incoming state of an NC-channel stage, deterministically.
//   tA/tB:        this tile's aggregate in absolute coordinates (valid when the
//                 tile starts past warm-up), published first;
//   first_steady: first tile of the series that starts past warm-up;
//   init:         state before the series' first tile.
// The state before tile t is composed from a fixed set of predecessors: the
// aggregates of tiles stop+1 .. t-1 applied to the inclusive state of tile
// `stop`, the latest checkpoint (a multiple of kLbSpan) or the last tile still
// in warm-up, whichever is later. Lane l handles tile t-1-l and the warp
// combines the maps in a fixed tree, so the result does not depend on timing.
constexpr int kLbSpan = 32;

template <int NC>
__device__ __forceinline__ void lb_resolve(LbDesc* base, long long stride, int tile, const double (&tA)[NC],
                                           const double (&tB)[NC], const double (&init)[NC], int first_steady,
                                           double (&Y)[NC], int* err, int lane) {
  if (tile == 0) {
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) Y[ch] = init[ch];
    return;
  }
  if (lane == 0) {
    LbDesc* me = base + (long long)tile * stride;
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) { me->A[ch] = tA[ch]; me->B[ch] = tB[ch]; }
    lb_store_flag(me, kLbAgg);
  }
  const int ckpt = ((tile - 1) / kLbSpan) * kLbSpan;
  int stop = first_steady - 1 > ckpt ? first_steady - 1 : ckpt;
  if (stop > tile - 1) stop = tile - 1;
  const int j = tile - 1 - lane;
  double a[NC], b[NC];
#pragma unroll
  for (int ch = 0; ch < NC; ++ch) { a[ch] = 1.0; b[ch] = 0.0; }
  if (j >= stop) {
    const LbDesc* d = base + (long long)j * stride;
    const bool inc = j == stop;
    if (lb_wait(d, inc ? kLbInc : kLbAgg, err) != 0) {
#pragma unroll
      for (int ch = 0; ch < NC; ++ch) {
        if (inc) {
          a[ch] = 0.0;  // constant map to the inclusive state
          b[ch] = *reinterpret_cast<const volatile double*>(&d->Y[ch]);
        } else {
          a[ch] = *reinterpret_cast<const volatile double*>(&d->A[ch]);
          b[ch] = *reinterpret_cast<const volatile double*>(&d->B[ch]);
        }
      }
    }
  }
  // lane l's map is applied after lane l+1's: fold the inner maps upward
#pragma unroll
  for (int dd = 1; dd < 32; dd <<= 1) {
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) {
      const double ai = __shfl_down_sync(kFull, a[ch], dd);
      const double bi = __shfl_down_sync(kFull, b[ch], dd);
      if ((lane & (2 * dd - 1)) == 0 && lane + dd < 32) {
        b[ch] = fma(a[ch], bi, b[ch]);
        a[ch] = a[ch] * ai;
      }
    }
  }
#pragma unroll
  for (int ch = 0; ch < NC; ++ch) Y[ch] = __shfl_sync(kFull, b[ch], 0);
}

// First tile whose first bar has count >= steady_from (count = bar - f).
__device__ __forceinline__ int lb_first_steady(int f, int steady_from, int tile_bars) {
  if (f < 0) return 0x7fffffff;
  return (int)(((long long)f + steady_from + tile_bars - 1) / tile_bars);
}

// Publish the exact state after this tile.
template <int NC>
__device__ __forceinline__ void lb_publish(LbDesc* base, long long stride, int tile, const double (&Y)[NC], int lane) {
  if (lane == 0) {
    LbDesc* me = base + (long long)tile * stride;
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) me->Y[ch] = Y[ch];
    lb_store_flag(me, kLbInc);
  }
}

}  // namespace tb
