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
  int f;      // first-index carries: inclusive value (-1 = none yet)
  int gflag;  // last tile of a group of 32: 1 once its group aggregate is set
  int floc;   // first-index carries: this tile's own value (-1 = none)
  int gf;     // first-index carries: the group's earliest value (-1 = none)
  int pad;
  double A[3], B[3], Y[3];
  double GA[3], GB[3];
};

constexpr int kLbGroup = 32;
constexpr int kLbSpan = 1024;  // 32 groups

constexpr int kLbAgg = 1, kLbInc = 2;
// polls / 32 = 2^21 polls, each a sleep of at most 256 ns plus an L2 round
// trip: one to two seconds
constexpr long long kLbSpinLimit = 1ll << 26;

// The polls a wait makes before giving up: err[1] when the host set it (a test
// that makes a wait run out), else kLbSpinLimit / 32.
__device__ __forceinline__ long long lb_spin_limit(const int* err) {
  const int v = *reinterpret_cast<const volatile int*>(err + 1);
  return v > 0 ? (long long)v : (kLbSpinLimit >> 5);
}

// Flags are published with release stores and polled with acquire loads
// (GPU scope): the descriptor fields a tile writes before its flag are visible
// to every thread that reads the flag set, with no separate fence on either
// side (a full fence per wait and per publish had cost a quarter of the issue
// slots of a 100,000-bar row in membar stalls). Every publish and every read
// of the fields behind a flag is done by one thread, the one that stored or
// acquired that flag.
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.b32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int lb_load_flag(const LbDesc* d) { return ld_acquire(&d->flag); }

__device__ __forceinline__ void lb_store_flag(LbDesc* d, int v) { st_release(&d->flag, v); }

// Wait (bounded) until flag >= want; returns the flag or 0 on timeout.
__device__ __forceinline__ int lb_wait_on(const int* flag, int want, int* err) {
  long long spins = 0;
  unsigned ns = 32;
  int v;
  while ((v = ld_acquire(flag)) < want) {
    if (++spins > lb_spin_limit(err)) {
      atomicExch(err, 1);
      return 0;
    }
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  return v;
}

// Warp-uniform wait: every lane with `active` set waits until *flag >= want.
// The warp polls together with a growing back-off, so waiting lanes neither
// diverge nor flood L2 with polls. Returns false (and sets *err) on timeout.
__device__ __forceinline__ bool lb_wait_all(const int* flag, int want, bool active, int* err) {
  long long spins = 0;
  unsigned ns = 32;
  for (;;) {
    const bool ok = !active || ld_acquire(flag) >= want;
    if (__all_sync(kFull, ok)) break;
    if (++spins > lb_spin_limit(err)) {
      if (active) atomicExch(err, 1);
      return false;
    }
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  return true;
}

__device__ __forceinline__ int lb_wait(const LbDesc* d, int want, int* err) {
  long long spins = 0;
  unsigned ns = 32;
  int v;
  while ((v = lb_load_flag(d)) < want) {
    if (++spins > lb_spin_limit(err)) {
      atomicExch(err, 1);
      return 0;
    }
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  return v;
}

// The predecessors a tile combines, latest first: the tiles of its own group
// before it, then whole groups, then the tiles of the first partial group,
// then the anchor `stop`, whose inclusive value closes the range.
struct LbItems {
  int tile, stop, nTail, nGroups, nHead, headEnd, grpEnd;
  __device__ __forceinline__ LbItems(int tile_, int stop_) : tile(tile_), stop(stop_) {
    const int first = stop + 1;
    const int tg0 = (tile / kLbGroup) * kLbGroup;
    if (first >= tg0) {
      nTail = tile - first;
      nGroups = nHead = headEnd = grpEnd = 0;
    } else {
      nTail = tile - tg0;
      const int gFull = (first + kLbGroup - 1) / kLbGroup;  // first whole group
      grpEnd = tg0 / kLbGroup;                               // groups gFull .. grpEnd-1
      nGroups = grpEnd - gFull;
      headEnd = gFull * kLbGroup;                            // head tiles first .. headEnd-1
      nHead = headEnd - first;
    }
  }
  __device__ __forceinline__ int count() const { return nTail + nGroups + nHead; }
  // item r < count(): kind 0 = tile aggregate of tile idx, 1 = group aggregate
  // held by tile idx (the group's last); r == count(): kind 2 = anchor
  __device__ __forceinline__ void item(int r, int& idx, int& kind) const {
    if (r == count()) { idx = stop; kind = 2; }
    else if (r < nTail) { idx = tile - 1 - r; kind = 0; }
    else if (r >= nTail + nGroups) { idx = headEnd - 1 - (r - nTail - nGroups); kind = 0; }
    else { idx = (grpEnd - 1 - (r - nTail)) * kLbGroup + kLbGroup - 1; kind = 1; }
  }
};

// First-index carry: the earliest bar with a property (first non-NaN input,
// first non-finite pair) up to this tile; local = this tile's earliest such
// bar or -1. Bar indices grow with the tile, so the earliest is the least
// non-negative value. The tile combines its own value, its predecessors'
// values and group minima back to the latest kLbSpan checkpoint, and that
// checkpoint's inclusive value, like lb_resolve; the last tile of each group
// publishes the group's minimum.
__device__ __forceinline__ int lb_first_index(LbDesc* base, long long stride, int tile, int local, int* err, int lane) {
  LbDesc* me = base + (long long)tile * stride;
  if (tile == 0) {
    if (lane == 0) {
      me->floc = local;
      me->f = local;
      lb_store_flag(me, kLbInc);
    }
    return local;
  }
  if (lane == 0) {
    me->floc = local;
    lb_store_flag(me, kLbAgg);
  }
  auto earliest = [](int v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = min(v, __shfl_xor_sync(kFull, v, d));
    return v;
  };
  const int kNone = 0x7fffffff;
  const int g = tile / kLbGroup;
  if (tile % kLbGroup == kLbGroup - 1 && g > 0) {
    const LbDesc* d = base + (long long)(tile - lane) * stride;
    const bool ok = lb_wait_all(&d->flag, kLbAgg, lane != 0, err);
    int v = lane == 0 ? local : (ok ? *reinterpret_cast<const volatile int*>(&d->floc) : -1);
    v = earliest(v >= 0 ? v : kNone);
    if (lane == 0) {
      me->gf = v == kNone ? -1 : v;
      st_release(&me->gflag, 1);
    }
  }
  // common case first: tile 0 (resolved at once) already holds the index
  {
    const bool ok0 = lb_wait_all(&base->flag, kLbInc, lane == 0, err);
    int f0 = -1;
    if (lane == 0 && ok0) f0 = *reinterpret_cast<const volatile int*>(&base->f);
    f0 = __shfl_sync(kFull, f0, 0);
    if (f0 >= 0) {
      if (lane == 0) {
        me->f = f0;
        lb_store_flag(me, kLbInc);
      }
      return f0;
    }
  }
  const LbItems it(tile, ((tile - 1) / kLbSpan) * kLbSpan);
  int best = local >= 0 ? local : kNone;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int r = 3 * lane + k;
    const bool active = r <= it.count();
    int idx = 0, kind = 0;
    if (active) it.item(r, idx, kind);
    const LbDesc* d = base + (long long)idx * stride;
    const int* flag = kind == 1 ? &d->gflag : &d->flag;
    const int want = kind == 1 ? 1 : (kind == 2 ? kLbInc : kLbAgg);
    ok = lb_wait_all(flag, want, active && ok, err) && ok;
    if (active && ok) {
      const int v = *reinterpret_cast<const volatile int*>(kind == 0 ? &d->floc : (kind == 1 ? &d->gf : &d->f));
      if (v >= 0 && v < best) best = v;
    }
  }
  best = earliest(best);
  const int res = best == kNone ? -1 : best;
  if (lane == 0) {
    me->f = res;
    lb_store_flag(me, kLbInc);
  }
  return res;
}

// Resolve the incoming state of an NC-channel stage, deterministically.
//   tA/tB:        this tile's aggregate in absolute coordinates (valid when the
//                 tile starts past warm-up), published first;
//   first_steady: first tile of the series that starts past warm-up;
//   init:         state before the series' first tile.
// The state before tile t is composed from a fixed set of predecessors: the
// aggregates of tiles stop+1 .. t-1 applied to the inclusive state of tile
// `stop`, the latest checkpoint (a multiple of kLbSpan tiles) or the last tile
// still in warm-up, whichever is later. Whole groups of 32 tiles inside that
// range enter through their group aggregate, which the last tile of each
// steady group publishes; the rest enter tile by tile. Every lane composes up
// to three consecutive items and the warp folds the lanes in a fixed tree, so
// the result does not depend on timing. Only the checkpoints chain inclusive
// states, one hop per kLbSpan tiles.
template <int NC>
__device__ __forceinline__ void lb_compose(double (&a)[NC], double (&b)[NC], const double* A, const double* B) {
  // (a, b) := (a, b) o (A, B): the new map is applied first
#pragma unroll
  for (int ch = 0; ch < NC; ++ch) {
    b[ch] = fma(a[ch], B[ch], b[ch]);
    a[ch] = a[ch] * A[ch];
  }
}

template <int NC>
__device__ __forceinline__ void lb_fold(double (&a)[NC], double (&b)[NC], int lane) {
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
}

template <int NC>
__device__ __forceinline__ void lb_resolve(LbDesc* base, long long stride, int tile, const double (&tA)[NC],
                                           const double (&tB)[NC], const double (&init)[NC], int first_steady,
                                           double (&Y)[NC], int* err, int lane) {
  if (tile == 0) {
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) Y[ch] = init[ch];
    return;
  }
  LbDesc* me = base + (long long)tile * stride;
  if (lane == 0) {
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) { me->A[ch] = tA[ch]; me->B[ch] = tB[ch]; }
    lb_store_flag(me, kLbAgg);
  }
  double a[NC], b[NC];
  // last tile of a steady group (other than group 0): publish the group's aggregate
  const int g = tile / kLbGroup;
  if (tile % kLbGroup == kLbGroup - 1 && g > 0 && g * kLbGroup >= first_steady) {
#pragma unroll
    for (int ch = 0; ch < NC; ++ch) { a[ch] = 1.0; b[ch] = 0.0; }
    const int j = tile - lane;  // lane 0 = this tile (outermost)
    const LbDesc* d = base + (long long)j * stride;
    const bool ok = lb_wait_all(&d->flag, kLbAgg, lane != 0, err);
    if (lane == 0) {
#pragma unroll
      for (int ch = 0; ch < NC; ++ch) { a[ch] = tA[ch]; b[ch] = tB[ch]; }
    } else if (ok) {
#pragma unroll
      for (int ch = 0; ch < NC; ++ch) {
        a[ch] = *reinterpret_cast<const volatile double*>(&d->A[ch]);
        b[ch] = *reinterpret_cast<const volatile double*>(&d->B[ch]);
      }
    }
    lb_fold<NC>(a, b, lane);
    if (lane == 0) {
#pragma unroll
      for (int ch = 0; ch < NC; ++ch) { me->GA[ch] = a[ch]; me->GB[ch] = b[ch]; }
      st_release(&me->gflag, 1);
    }
  }
  const int ckpt = ((tile - 1) / kLbSpan) * kLbSpan;
  int stop = first_steady - 1 > ckpt ? first_steady - 1 : ckpt;
  if (stop > tile - 1) stop = tile - 1;
  const LbItems it(tile, stop);
  const int nItems = it.count();
#pragma unroll
  for (int ch = 0; ch < NC; ++ch) { a[ch] = 1.0; b[ch] = 0.0; }
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int r = 3 * lane + k;
    const bool active = r <= nItems;
    // the item's descriptor, the flag to wait for and the map's fields
    int idx = 0, kind = 0;  // kind: 0 tile aggregate, 1 group aggregate, 2 anchor
    if (active) it.item(r, idx, kind);
    const LbDesc* d = base + (long long)idx * stride;
    const int* flag = kind == 1 ? &d->gflag : &d->flag;
    const int want = kind == 1 ? 1 : (kind == 2 ? kLbInc : kLbAgg);
    ok = lb_wait_all(flag, want, active && ok, err) && ok;
    if (active && ok) {
      double A[NC], B[NC];
#pragma unroll
      for (int ch = 0; ch < NC; ++ch) {
        if (kind == 2) {  // the anchor: constant map to its inclusive state
          A[ch] = 0.0;
          B[ch] = *reinterpret_cast<const volatile double*>(&d->Y[ch]);
        } else if (kind == 1) {
          A[ch] = *reinterpret_cast<const volatile double*>(&d->GA[ch]);
          B[ch] = *reinterpret_cast<const volatile double*>(&d->GB[ch]);
        } else {
          A[ch] = *reinterpret_cast<const volatile double*>(&d->A[ch]);
          B[ch] = *reinterpret_cast<const volatile double*>(&d->B[ch]);
        }
      }
      lb_compose<NC>(a, b, A, B);
    }
  }
  lb_fold<NC>(a, b, lane);
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
