// Row-parallel engine: batches with many series.
//
// A CTA owns a group of 32 rows (lane = row). One producer warp streams the
// input planes the jobs read into a shared-memory ring, chunk by chunk
// (C = 32 bars), with cp.async; every other warp runs one job over the 32 rows,
// each thread walking its row bar by bar in TA-Lib's sequential order with the
// indicator state in registers. Producer and job warps meet only at mbarriers:
// "full" (the chunk landed) and "empty" (every job warp is done with a chunk,
// including its use as the halo of later chunks). A slow job never holds up a
// fast one by more than the ring depth, and no CTA-wide barrier is taken after
// the prologue.
//
// Ring layout per staged plane and row: [Hs mirror slots | NS slots] of C bars
// and one padding float (odd row stride: lane r reading its row is bank-
// conflict free). Chunk c goes to slot c % NS; the last Hs slots are also
// copied to the mirror slots in front of slot 0, so the halo of every chunk
// (up to Hs*C bars back) is contiguous in shared memory and read without
// wrap-around.
//
// Outputs go through a per-warp [nout][32][C+1] transpose buffer and leave as
// coalesced row segments.
//
// The warps of a CTA run up to 15 different families at once, so the hot code
// of all of them competes for the SM's instruction cache; the per-bar loops
// are therefore not unrolled (unrolled by 8 they measured 1.7x slower on the
// 13-indicator pass, with most issue slots lost to instruction fetch).
//
// Arithmetic: float32 for the bulk (ranges, ratios, Wilder and EMA states of
// short periods, window extrema); FP64 where the result needs it: the window
// sums of float32 inputs (exact in FP64, so a running sum equals the direct
// sum), cumulative OBV / AD, the MACD lines (fast - slow cancels), CCI's
// typical-price deviations and the long-period recurrences (error grows with
// the period). Every choice is made per job from its parameters alone, so the
// bits of a row never depend on the other rows of the batch.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "engine.h"

namespace tb {
namespace rows {

constexpr int C = 32;                 // bars per chunk
constexpr int kMaxHalo = 64;          // bars of history a job may read before a chunk
constexpr int kMaxLine = 64;          // per-lane history of the line-keeping families
constexpr int kMaxConsumers = 19;     // job warps per row group (one more warp stages the inputs)
constexpr int kMaxWarps = kMaxConsumers + 1;  // warps per CTA over all its row groups
constexpr int kMaxParts = 8;          // partitions of a job set (one per grid row)
constexpr int kFp32MaxPeriod = 32;    // recurrences up to this period keep float32 state
constexpr unsigned long long kWaitNs = 1000000000ull;  // one mbarrier wait gives up after 1 s
constexpr unsigned long long kStallWaitNs = 1000000ull;  // 1 ms under the stall test knob
constexpr unsigned kWaitPolls = 1u << 28;               // and after this many polls in any case

struct Layout {
  int nplanes;
  int slot_plane[P_COUNT];
  int plane_slot[P_COUNT];
  int Hs, NS, RS;                     // halo slots, ring slots, row stride (floats)
  int ring_off;                       // [nplanes][32][RS] floats
  int bar_off;                        // uint64 full[NS], empty[NS]
  int tab_off;                        // long long base[32], n[32]; int maxn, abort
  int nconsumers;
  int producer_warp;
  int warp_job[kMaxConsumers + 1];    // job of each warp, -1 for the producer
  int warp_team[kMaxConsumers + 1];   // member k and team size m of a bar-parallel job: k | m << 8
  unsigned long long bp_mask;         // families that run bar-parallel (1 << family)
  int stage_off[kMaxConsumers + 1];   // [nout][32][C+1] floats
  int line_off[kMaxConsumers + 1];    // per-warp history lines
  int total;
};

// A launch: the job set split into P partitions; CTAs cta0[y] .. cta0[y+1]-1
// run partition y with layout lay[y], G[y] row groups of 32 rows each.
struct Split {
  int P;
  int G[kMaxParts];
  int cta0[kMaxParts + 1];
  Layout lay[kMaxParts];
};

// ------------------------------------------------------------ primitives

__device__ __forceinline__ unsigned saddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(saddr(b)) : "memory");
}
// arrives on the barrier once this thread's earlier cp.async copies have landed
__device__ __forceinline__ void cp_async_arrive(uint64_t* b) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(saddr(b)) : "memory");
}
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr(dst)), "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
  return t;
}

// Bounded wait for the phase of `b` with parity `par`: false when the wait ran
// out (the error word is set and the CTA's abort flag raised) or another warp
// of the CTA aborted.
__device__ bool mbar_wait(uint64_t* b, unsigned par, volatile int* abort_flag, int* err, int lane,
                          unsigned long long limit_ns) {
  unsigned long long t0 = 0;
  for (unsigned i = 0; i < kWaitPolls; ++i) {
    if (mbar_try_wait(b, par)) return true;
    if ((i & 255) == 255) {
      if (*abort_flag) return false;
      const unsigned long long now = global_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > limit_ns) break;
    }
  }
  if (lane == 0) {
    if (err) atomicOr(err, 1);
    *abort_flag = 1;
  }
  return false;
}

__device__ __forceinline__ bool finitef(float v) { return fabsf(v) < __int_as_float(0x7f800000); }
__device__ __forceinline__ float finf() { return __int_as_float(0x7f800000); }

// Non-finite values inside a window: NaN, +inf and -inf counts. A window sum
// over them is NaN (any NaN, or both infinities), else +-inf.
struct Bad {
  int nan = 0, pinf = 0, ninf = 0;
  __device__ __forceinline__ void add(float v, int d) {
    if (isnan(v)) nan += d;
    else if (v > 0.0f) pinf += d;
    else ninf += d;
  }
  __device__ __forceinline__ bool any() const { return (nan | pinf | ninf) != 0; }
  __device__ __forceinline__ float value() const {
    return (nan != 0 || (pinf != 0 && ninf != 0)) ? qnan() : (pinf != 0 ? finf() : -finf());
  }
};

// --------------------------------------------------------------- driver

// a / b through the approximate reciprocal (max 1 ulp) and one rounding: the
// ratios below need the float tolerance, not IEEE division's last bit.
__device__ __forceinline__ float fdiv(float a, float b) {
  float r;
  asm("rcp.approx.f32 %0, %1;\n" : "=f"(r) : "f"(b));
  return a * r;
}
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }

// x / d correctly rounded, from y = RN(1/d), without a divide: the product
// x*y is within 1.5 ulp of the quotient, a first FMA correction brings it
// within one ulp, and then one more correction rounds it correctly
// (Markstein's theorem: P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990). Holds
// for normal operands; zeros and non-finite quotients pass through x*y, which
// is already right for them.
__device__ __forceinline__ double div_by(double x, double d, double y) {
  const double q0 = x * y;
  const double q1 = fma(fma(-q0, d, x), y, q0);
  const double q2 = fma(fma(-q1, d, x), y, q1);
  return (q0 == 0.0 || !(fabs(q0) < __longlong_as_double(0x7ff0000000000000ll))) ? q0 : q2;
}

struct Warp {
  unsigned char* smem;
  const Layout* lay;
  uint64_t* full;
  uint64_t* empty;
  const long long* tbase;
  const long long* tn;
  volatile int* abort_flag;
  int* err;
  float* stage;
  int lane, nchunks, maxn, Hs, NS, RS;
  unsigned long long wait_ns;  // limit of one wait
  long long n;     // this lane's row length
  bool uni;        // rows of the group are consecutive rows of a uniform batch
  long long T;     // their length
  long long s0T;   // element offset of the group's first row
  int nvalid;      // rows of the group that exist
  int tk, tm;      // bar-parallel jobs: this warp takes rows tk, tk + tm, ... of the group

  __device__ __forceinline__ const float* X(int c, int plane) const { return Xrow(c, plane, lane); }
  // row r's line of chunk c: [i] is bar c*C + i, i >= -Hs*C
  __device__ __forceinline__ const float* Xrow(int c, int plane, int r) const {
    const float* ring = reinterpret_cast<const float*>(smem + lay->ring_off);
    return ring + ((size_t)lay->plane_slot[plane] * 32 + r) * RS + (Hs + c % NS) * C;
  }
  // output offset and length of row r of the group (length 0 for a missing row)
  __device__ __forceinline__ long long row_len(int r, long long& base) const {
    if (uni) {
      base = s0T + (long long)r * T;
      return r < nvalid ? T : 0;
    }
    base = tbase[r];
    return base >= 0 ? tn[r] : 0;
  }
  __device__ __forceinline__ int lim(int c) const { return min(C, maxn - c * C); }
  // chunk c is this warp's share of a job split over a team by chunks
  __device__ __forceinline__ bool own(int c) const { return tm <= 1 || c % tm == tk; }
  // bars of chunk c a steady (unrolled by 8) loop covers
  __device__ __forceinline__ int lim8(int c) const { return (lim(c) + 7) & ~7; }

  __device__ __forceinline__ bool wait(int c) const {
    return mbar_wait(&full[c % NS], (unsigned)((c / NS) & 1), abort_flag, err, lane, wait_ns);
  }
  // chunk c is done: chunk c - Hs is no longer read as a halo
  __device__ __forceinline__ void release(int c) const {
    const int r = c - Hs;
    __syncwarp();
    if (r >= 0 && lane == 0) mbar_arrive(&empty[r % NS]);
  }
  __device__ __forceinline__ float* stage_row(int k) const { return stage + (k * 32 + lane) * (C + 1); }
  __device__ __forceinline__ void put(int k, int r, float v) const { stage[(k * 32 + lane) * (C + 1) + r] = v; }
  // coalesced row segments of output k for chunk c
  __device__ void flush(int k, float* out, int c) const {
    __syncwarp();
    const int t0 = c * C;
    const float* src = stage + k * 32 * (C + 1);
    if (uni) {
      if (((T | ((long long)(uintptr_t)out >> 2)) & 1) == 0) {
        // even rows in 8-byte aligned planes: half a warp per row, two bars a lane
        const int half = lane >> 4, col = (lane & 15) << 1;
        if (t0 + col < T) {
          float* p = out + s0T + half * T + t0 + col;
          const float* sp = src + half * (C + 1) + col;
#pragma unroll 4
          for (int i = half; i < nvalid; i += 2) {
            float2 v;
            v.x = sp[0];
            v.y = sp[1];
            *reinterpret_cast<float2*>(p) = v;
            p += 2 * T;
            sp += 2 * (C + 1);
          }
        }
      } else if (t0 + lane < T) {
        float* p = out + s0T + t0 + lane;
        const float* sp = src + lane;
#pragma unroll 4
        for (int i = 0; i < nvalid; ++i) {
          *p = *sp;
          p += T;
          sp += C + 1;
        }
      }
    } else {
      const long long t = t0 + lane;
      src += lane;
#pragma unroll 4
      for (int i = 0; i < 32; ++i) {
        const long long b = tbase[i];
        if (b >= 0 && t < tn[i]) out[b + t] = src[i * (C + 1)];
      }
    }
    __syncwarp();
  }
};

__device__ __forceinline__ bool all_lanes(bool v) { return __all_sync(kFull, v); }

// ------------------------------------------------------------- windows

// SMA / SUM / WMA (mode 0/1/2): running FP64 sums of the window. Sums of
// float32 values are exact in FP64, so the running sum is the direct sum of
// every window, with no drift along the row; NaN and +-inf are kept out of
// the sums and counted, so each window sees them only while it holds them.
// A chunk whose windows hold only finite values runs without that
// bookkeeping (same arithmetic); if a non-finite value shows up, the chunk is
// run again the general way from the saved sums.
// talib08:14748-14812 TA_SMA, talib08:19171-19277 TA_WMA, BatchFused.cu:133-138 SUM.
__device__ void w_sum_window(const Warp& w, const Job& j, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  const double invp = 1.0 / (double)p;
  const double invdiv = 1.0 / ((double)p * (p + 1) / 2.0);
  const double dp = (double)p;
  double s = 0.0, ws = 0.0;
  Bad bad;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    const float* Xo = X - p;
    float* st = w.stage_row(0);
    const int t0 = c * C;
    bool general = !(t0 >= p && all_lanes(!bad.any()));
    if (!general) {
      const double s_in = s, ws_in = ws;
      const int n8 = w.lim8(c);
      for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 1
        for (int u = 0; u < 8; ++u) {
          const int r = r8 + u;
          const double a = (double)X[r], b = (double)Xo[r];
          if (mode == 2) ws = fma(dp, a, ws - s);
          s = (s + a) - b;
          st[r] = mode == 0 ? (float)(s * invp) : mode == 1 ? (float)s : (p == 1 ? X[r] : (float)(ws * invdiv));
        }
      }
      if (!all_lanes(isfinite(s) && isfinite(ws))) {
        s = s_in;
        ws = ws_in;
        general = true;
      }
    }
    if (general) {
      const int lim = w.lim(c);
      for (int r = 0; r < lim; ++r) {
        const int t = t0 + r;
        const float vin = X[r];
        const bool out_bar = t >= p;
        const float vout = out_bar ? Xo[r] : 0.0f;
        const bool fi = finitef(vin), fo = finitef(vout);
        if (!(fi && fo)) {
          if (!fi) bad.add(vin, 1);
          if (!fo) bad.add(vout, -1);
        }
        const double a = fi ? (double)vin : 0.0, b = fo ? (double)vout : 0.0;
        if (mode == 2) ws = out_bar ? fma(dp, a, ws - s) : fma((double)(t + 1), a, ws);
        s = (s + a) - b;
        float o = qnan();
        if (t >= p - 1) {
          if (bad.any()) o = (mode == 2 && p == 1) ? vin : bad.value();
          else if (mode == 0) o = (float)(s * invp);
          else if (mode == 1) o = (float)s;
          else o = p == 1 ? vin : (float)(ws * invdiv);
        }
        st[r] = o;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// BBANDS / STDDEV / VAR (mode 0/1/2): moments of d = x - o about an origin o,
// the bar at each chunk's first output, where the window is summed directly
// (talib08:18047-18183 TA_VAR re-centres the same way); the variance follows
// TA-Lib's E[d^2] - E[d]^2 in FP64 and is clamped at zero; the square root and
// the bands in float32. A chunk whose windows are finite runs without NaN
// bookkeeping, with the same arithmetic. Chunks share no state, so a team of
// warps can share the job by chunks.
__device__ __forceinline__ void moment_out(int mode, double o, double s1, double s2, double inv, float up, float dn,
                                           float& o0, float& o1, float& o2) {
  const double m1 = s1 * inv;
  double var = fma(-m1, m1, s2 * inv);
  var = var > 0.0 ? var : 0.0;
  const float vf = (float)var;
  if (mode == 2) {
    o0 = vf;
    return;
  }
  const float sd = sqrtf(vf);
  if (mode == 1) {
    o0 = sd * up;
    return;
  }
  const float mid = (float)(o + m1);
  if (up == dn) {
    const float dv = sd * up;
    o0 = mid + dv;
    o2 = mid - dv;
  } else {
    o0 = fmaf(sd, up, mid);
    o2 = mid - sd * dn;
  }
  o1 = mid;
}

__device__ void w_moment_window(const Warp& w, const Job& j, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  const double inv = 1.0 / (double)p;
  const float up = (float)j.fp[0], dn = (float)j.fp[1];
  const int nout = mode == 0 ? 3 : 1;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    if (!w.own(c)) {
      w.release(c);
      continue;
    }
    const float* X = w.X(c, pl);
    const float* Xo = X - p;
    float* st0 = w.stage_row(0);
    float* st1 = w.stage_row(1);
    float* st2 = w.stage_row(2);
    const int t0 = c * C;
    bool general = t0 < p - 1;
    if (!general) {
      // seed at bar t0 (r = 0)
      const double o = (double)X[0];
      double s1 = 0.0, s2 = 0.0;
      for (int i = 0; i < p; ++i) {
        const double d = (double)X[i - p + 1] - o;
        s1 += d;
        s2 = fma(d, d, s2);
      }
      float o0 = 0.0f, o1 = 0.0f, o2 = 0.0f;
      moment_out(mode, o, s1, s2, inv, up, dn, o0, o1, o2);
      st0[0] = o0;
      if (mode == 0) { st1[0] = o1; st2[0] = o2; }
      const int n8 = w.lim8(c);
      for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 1
        for (int u = 0; u < 8; ++u) {
          const int r = r8 + u;
          if (r == 0) continue;
          const double di = (double)X[r] - o, dd = (double)Xo[r] - o;
          s1 = (s1 + di) - dd;
          s2 = fma(-dd, dd, fma(di, di, s2));
          moment_out(mode, o, s1, s2, inv, up, dn, o0, o1, o2);
          st0[r] = o0;
          if (mode == 0) { st1[r] = o1; st2[r] = o2; }
        }
      }
      if (!all_lanes(isfinite(s1) && isfinite(s2))) general = true;
    }
    if (general) {
      const int lim = w.lim(c);
      double s1 = 0.0, s2 = 0.0, o = 0.0;
      int nn = 0;
      bool seeded = false;
      for (int r = 0; r < lim; ++r) {
        const int t = t0 + r;
        float o0 = qnan(), o1 = qnan(), o2 = qnan();
        if (t >= p - 1) {
          if (!seeded) {
            seeded = true;
            const float ov = X[r];
            o = isnan(ov) ? 0.0 : (double)ov;
            s1 = s2 = 0.0;
            nn = 0;
            for (int i = 0; i < p; ++i) {
              const float v = X[r - p + 1 + i];
              if (isnan(v)) ++nn;
              else {
                const double d = (double)v - o;
                s1 += d;
                s2 = fma(d, d, s2);
              }
            }
          } else {
            const float vin = X[r], vout = Xo[r];
            const double di = isnan(vin) ? 0.0 : (double)vin - o;
            const double dd = isnan(vout) ? 0.0 : (double)vout - o;
            nn += (isnan(vin) ? 1 : 0) - (isnan(vout) ? 1 : 0);
            s1 = (s1 + di) - dd;
            s2 = fma(-dd, dd, fma(di, di, s2));
          }
          if (nn == 0) moment_out(mode, o, s1, s2, inv, up, dn, o0, o1, o2);
        }
        st0[r] = o0;
        if (mode == 0) { st1[r] = o1; st2[r] = o2; }
      }
    }
    for (int k = 0; k < nout; ++k) w.flush(k, (float*)j.out[k], c);
    w.release(c);
  }
}

// Running window extremum over p bars (van Herk / Gil-Werman): blocks of p bars
// from the row's first bar; the extremum of a window is the suffix extremum of
// its part in the previous block and the prefix extremum of its part in the
// current one. The suffixes of a block are computed once, when the next block
// starts, into a per-lane line. fmaxf / fminf skip NaN exactly as a direct
// fmaxf / fminf scan does.
template <bool kMax>
struct VanHerk {
  float* suf;  // this lane's line: suf[k * 32] for k in 0..p-1
  float pre;
  __device__ __forceinline__ static float op(float a, float b) { return kMax ? fmaxf(a, b) : fminf(a, b); }
  // block start at bar t (t >= p): suffix extrema of bars t-p .. t-1
  __device__ __forceinline__ void fill(const float* X, int r, int p) {
    float m = X[r - 1];
    suf[(p - 1) * 32] = m;
    for (int k = p - 2; k >= 0; --k) {
      m = op(m, X[r - p + k]);
      suf[k * 32] = m;
    }
  }
  // the state entering chunk-relative bar 0 (row bar t0), rebuilt from the
  // halo: the extremum of the current block's bars before t0 and the
  // suffixes of the block before it; returns t0's block position. Reads
  // back to bar t0 - pos - p (at most 2p - 1 bars).
  __device__ __forceinline__ int reseed(const float* X, long long t0, int p) {
    const int pos = (int)(t0 % p);
    if (pos > 0) {
      float m = X[-pos];
      for (int k = -pos + 1; k < 0; ++k) m = op(m, X[k]);
      pre = m;
      if (t0 - pos >= p) fill(X, -pos, p);
    }
    return pos;
  }
  // bar t at block position pos (t = k*p + pos) with value x
  __device__ __forceinline__ float step(float x, int pos, int p) {
    pre = pos == 0 ? x : op(pre, x);
    const int k = pos + 1 == p ? 0 : pos + 1;  // entry p does not exist
    const float s = op(suf[k * 32], pre);
    return pos == p - 1 ? pre : s;
  }
};

// WILLR (src/indicators/WILLR.cu:11-30): extremes anchored at the current bar
// (a NaN high or low there gives NaN, earlier NaNs are skipped), float32 ratio
// times -100 clamped to [-100, 0]; 0 for a zero range. Every chunk rebuilds its
// van Herk state from the halo (extremes are exact, so the bits do not
// change), and a team of warps can share the job by chunks.
__device__ void w_willr(const Warp& w, const Job& j, float* line, int cap) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0];
  VanHerk<true> hh{line + w.lane, 0.0f};
  VanHerk<false> ll{line + 32 * cap + w.lane, 0.0f};
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    if (!w.own(c)) {
      w.release(c);
      continue;
    }
    const float* H = w.X(c, ph);
    const float* Lo = w.X(c, plo);
    const float* Cl = w.X(c, pc);
    float* st = w.stage_row(0);
    const int t0 = c * C, n8 = w.lim8(c);
    int pos = hh.reseed(H, t0, p);
    ll.reseed(Lo, t0, p);
    for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int r = r8 + u, t = t0 + r;
        if (pos == 0 && t >= p) {
          hh.fill(H, r, p);
          ll.fill(Lo, r, p);
        }
        const float h = H[r], l = Lo[r];
        float hi = hh.step(h, pos, p);
        float lo = ll.step(l, pos, p);
        pos = pos + 1 == p ? 0 : pos + 1;
        hi = isnan(h) ? h : hi;
        lo = isnan(l) ? l : lo;
        const float den = hi - lo;
        const float v = den == 0.0f ? 0.0f : fdiv(hi - Cl[r], den) * -100.0f;
        const float o = isnan(v) ? qnan() : fminf(0.0f, fmaxf(-100.0f, v));
        st[r] = t >= p - 1 ? o : qnan();
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// fastK of chunk-relative bar r from its window directly (extremes anchored
// at the window's first bar, as the running form gives them)
__device__ __forceinline__ float stoch_fastk(const float* H, const float* Lo, const float* Cl, int r, int p) {
  float hi = H[r - p + 1], lo = Lo[r - p + 1];
  for (int i = r - p + 2; i <= r; ++i) {
    const float a = H[i], b = Lo[i];
    hi = a > hi ? a : hi;
    lo = b < lo ? b : lo;
  }
  const float range = hi - lo;
  return fabsf(range) <= 1e-14f * (fabsf(hi) + fabsf(lo)) ? 0.0f : fdiv(Cl[r] - lo, range) * 100.0f;
}

// STOCH (talib08:16115-16302, SMA slowing): fastK from the window extremes
// anchored at the window's first bar, TA-Lib's zero-range test; slowK and
// slowD are direct means of the last q fastK / slowK values, summed oldest
// first, from registers for q = Q > 0 or per-lane lines (Q = 0). Every chunk
// rebuilds its state from the halo, so a team of warps can share the job by
// chunks.
template <int Q>
__device__ void w_stoch(const Warp& w, const Job& j, float* line, int cap) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0], q = Q > 0 ? Q : j.ip[1];
  const int lb = p - 1 + 2 * (q - 1), kready = p - 1 + (q - 1);
  const int mask = cap - 1;
  const float invq = 1.0f / (float)q;
  VanHerk<true> hh{line + w.lane, 0.0f};
  VanHerk<false> ll{line + 32 * cap + w.lane, 0.0f};
  float* fkl = line + 2 * 32 * cap + w.lane;  // [(t & mask) * 32]
  float* skl = line + 3 * 32 * cap + w.lane;
  float fh[4] = {0.0f, 0.0f, 0.0f, 0.0f}, sh[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // [0] newest
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    if (!w.own(c)) {
      w.release(c);
      continue;
    }
    const float* H = w.X(c, ph);
    const float* Lo = w.X(c, plo);
    const float* Cl = w.X(c, pc);
    float* st0 = w.stage_row(0);
    float* st1 = w.stage_row(1);
    const int t0 = c * C, n8 = w.lim8(c);
    // state entering bar t0 from the halo: the van Herk blocks, and fastK /
    // slowK of the 2(q-1) / q-1 bars before t0 (window extremes are exact, so
    // the bits do not depend on where a chunk starts)
    int pos = hh.reseed(H, t0, p);
    ll.reseed(Lo, t0, p);
    if (Q > 0) {
      float fk[2 * (Q > 0 ? Q : 1)];
#pragma unroll
      for (int i = 0; i < 2 * (Q - 1); ++i) fk[i] = stoch_fastk(H, Lo, Cl, i - 2 * (Q - 1), p);  // oldest first
#pragma unroll
      for (int m = 0; m < Q - 1; ++m) {
        fh[m] = fk[2 * (Q - 1) - 1 - m];
        // slowK of bar t0-1-m: fastK of bars t0-m-q .. t0-1-m, oldest first
        const int e = 2 * (Q - 1) - 1 - m;
        float sk = fk[e - (Q - 1)];
#pragma unroll
        for (int i = e - (Q - 1) + 1; i <= e; ++i) sk += fk[i];
        sh[m] = sk * invq;
      }
    } else {
      for (int r = -2 * (q - 1); r < 0; ++r) fkl[((t0 + r) & mask) * 32] = stoch_fastk(H, Lo, Cl, r, p);
      for (int r = -(q - 1); r < 0; ++r) {
        float sk = fkl[((t0 + r - q + 1) & mask) * 32];
        for (int m = q - 2; m >= 0; --m) sk += fkl[((t0 + r - m) & mask) * 32];
        skl[((t0 + r) & mask) * 32] = sk * invq;
      }
    }
    for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int r = r8 + u, t = t0 + r;
        if (pos == 0 && t >= p) {
          hh.fill(H, r, p);
          ll.fill(Lo, r, p);
        }
        float hi = hh.step(H[r], pos, p);
        float lo = ll.step(Lo[r], pos, p);
        pos = pos + 1 == p ? 0 : pos + 1;
        const float ha = H[r - p + 1], la = Lo[r - p + 1];
        hi = isnan(ha) ? ha : hi;
        lo = isnan(la) ? la : lo;
        const float range = hi - lo;
        const float k = fabsf(range) <= 1e-14f * (fabsf(hi) + fabsf(lo)) ? 0.0f : fdiv(Cl[r] - lo, range) * 100.0f;
        float o0 = qnan(), o1 = qnan();
        if (Q > 0) {
#pragma unroll
          for (int m = 3; m > 0; --m) fh[m] = fh[m - 1];
          fh[0] = k;
          float s = fh[Q - 1];
#pragma unroll
          for (int m = Q - 2; m >= 0; --m) s += fh[m];
          const float kv = s * invq;
#pragma unroll
          for (int m = 3; m > 0; --m) sh[m] = sh[m - 1];
          sh[0] = kv;
          float d = sh[Q - 1];
#pragma unroll
          for (int m = Q - 2; m >= 0; --m) d += sh[m];
          if (t >= lb) {
            o0 = kv;
            o1 = d * invq;
          }
        } else if (t >= p - 1) {
          fkl[(t & mask) * 32] = k;
          if (t >= kready) {
            float s = 0.0f;
            for (int m = q - 1; m >= 0; --m) s += fkl[((t - m) & mask) * 32];
            const float kv = s * invq;
            skl[(t & mask) * 32] = kv;
            if (t >= lb) {
              float d = 0.0f;
              for (int m = q - 1; m >= 0; --m) d += skl[((t - m) & mask) * 32];
              o0 = kv;
              o1 = d * invq;
            }
          }
        }
        st0[r] = o0;
        st1[r] = o1;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.flush(1, (float*)j.out[1], c);
    w.release(c);
  }
}

// MFI (include/utils/StreamStates.h:749-792 precise::MfiState): flows of the
// FP64 typical price ((h+l)+c)/3.0 (correctly rounded, div_by) times volume,
// signed by the typical price's change, in a per-lane line; running positive /
// negative window sums, re-summed directly when one turns negative or a
// non-finite flow is in reach (the reference sums every window); 100 * pos /
// (pos + neg), 0 below a total of 1. Every chunk starts from sums rebuilt from
// the halo, so a chunk depends on no state of the chunk before and a team of
// warps can share the job by chunks.
__device__ void w_mfi(const Warp& w, const Job& j, double* line, int cap) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], pv = j.in[3], p = j.ip[0];
  const int mask = cap - 1;
  const double third = 1.0 / 3.0;
  double* pos_l = line + w.lane;  // [(t & mask) * 32]
  double* neg_l = line + 32 * cap + w.lane;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    if (!w.own(c)) {
      w.release(c);
      continue;
    }
    const float* H = w.X(c, ph);
    const float* Lo = w.X(c, plo);
    const float* Cl = w.X(c, pc);
    const float* V = w.X(c, pv);
    float* st = w.stage_row(0);
    const int t0 = c * C, n8 = w.lim8(c);
    // the state entering bar t0, rebuilt from the ring's halo: the flows of
    // bars t0-p .. t0-1 (from bar 0 in the first p bars), their sums taken
    // oldest first, and the previous typical price
    double ps = 0.0, ns = 0.0, prev_tp = 0.0;
    int last_bad = -(1 << 30);
    if (t0 > 0) {
      const int r0 = max(-p, -t0);
      double prev = t0 + r0 >= 1 ? div_by(((double)H[r0 - 1] + (double)Lo[r0 - 1]) + (double)Cl[r0 - 1], 3.0, third)
                                 : 0.0;
      for (int r = r0; r < 0; ++r) {
        const int t = t0 + r;
        const double tp = div_by(((double)H[r] + (double)Lo[r]) + (double)Cl[r], 3.0, third);
        const double fl = tp * (double)V[r];
        const bool ok = t >= 1 && isfinite(tp) && isfinite(prev);
        const double a = ok && tp > prev ? fl : 0.0, b = ok && tp < prev ? fl : 0.0;
        if (!isfinite(a + b)) last_bad = t;
        prev = tp;
        pos_l[(t & mask) * 32] = a;
        neg_l[(t & mask) * 32] = b;
        ps += a;
        ns += b;
      }
      prev_tp = prev;
    }
    for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 4
      for (int u = 0; u < 8; ++u) {
        const int r = r8 + u, t = t0 + r;
        const double tp = div_by(((double)H[r] + (double)Lo[r]) + (double)Cl[r], 3.0, third);
        const double fl = tp * (double)V[r];
        const bool ok = t >= 1 && isfinite(tp) && isfinite(prev_tp);
        const double a = ok && tp > prev_tp ? fl : 0.0, b = ok && tp < prev_tp ? fl : 0.0;
        if (!isfinite(a + b)) last_bad = t;
        prev_tp = tp;
        const int slot = (t & mask) * 32, g = ((t - p) & mask) * 32;
        const double ga = pos_l[g], gb = neg_l[g];
        pos_l[slot] = a;
        neg_l[slot] = b;
        float o = qnan();
        if (t >= p) {
          if (t > p) {
            ps = (ps - ga) + a;
            ns = (ns - gb) + b;
          }
          if (t == p || ps < 0.0 || ns < 0.0 || last_bad >= t - p) {
            ps = ns = 0.0;
            for (int i = p - 1; i >= 0; --i) {
              ps += pos_l[((t - i) & mask) * 32];
              ns += neg_l[((t - i) & mask) * 32];
            }
          }
          const double tot = ps + ns;
          o = tot < 1.0 ? 0.0f : 100.0f * fdiv((float)ps, (float)tot);
        }
        st[r] = o;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// ------------------------------------------------------------ recurrences

// EMA / RMA (talib08:5546-5627 TA_EMA, talib08:13614-13683 TA_RMA): SMA seed,
// then fma(beta, y, k*x); leading NaNs skipped (BatchFused.cu:34-41). Chunks
// past every lane's seed run the bare recurrence.
template <class R>
__device__ void w_ema(const Warp& w, const Job& j) {
  const int pl = j.in[0], p = j.ip[0];
  const R beta = (R)j.fp[0], kk = (R)j.fp[1];
  const bool copy = p == 1 && j.family != F_RMA;  // TA_RMA has no period-1 copy
  R y = 0;
  int cnt = -1;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    float* st = w.stage_row(0);
    if (all_lanes(cnt >= p - 1)) {
      const int n8 = w.lim8(c);
      for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 1
        for (int u = 0; u < 8; ++u) {
          const R x = (R)X[r8 + u];
          y = copy ? x : fma(beta, y, kk * x);
          st[r8 + u] = (float)y;
        }
      }
      cnt += n8;
    } else {
      const int lim = w.lim(c);
      for (int r = 0; r < lim; ++r) {
        const float xf = X[r];
        float o = qnan();
        if (cnt >= 0 || !isnan(xf)) {
          ++cnt;
          const R x = (R)xf;
          if (copy) y = x;
          else if (cnt > p - 1) y = fma(beta, y, kk * x);
          else if (cnt < p - 1) y += x;
          else y = (y + x) / (R)p;
          if (cnt >= p - 1) o = (float)y;
        }
        st[r] = o;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// RSI (talib08:13996-14115): Wilder sums of gains and losses; a NaN change
// makes the rest of the row NaN; leading NaNs skipped.
template <class R>
__device__ __forceinline__ float rsi_out(R gain, R loss) {
  const R tot = gain + loss;
  return isnan(tot) ? qnan() : (tot > (R)0 ? (float)((R)100 * fdiv(gain, tot)) : 50.0f);
}

template <class R>
__device__ void w_rsi(const Warp& w, const Job& j) {
  const int pl = j.in[0], p = j.ip[0];
  const R inv = (R)(1.0 / (double)p), pm1 = (R)(p - 1);
  R gain = 0, loss = 0;
  int cnt = -1;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    float* st = w.stage_row(0);
    if (all_lanes(cnt >= p)) {
      R xp = (R)X[-1];
      const int n8 = w.lim8(c);
      for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 1
        for (int u = 0; u < 8; ++u) {
          const R x = (R)X[r8 + u];
          const R d = x - xp;
          xp = x;
          const R g = d > (R)0 ? d : (R)0, l = g - d;
          gain = (gain * pm1 + g) * inv;
          loss = (loss * pm1 + l) * inv;
          st[r8 + u] = rsi_out(gain, loss);
        }
      }
      cnt += n8;
    } else {
      const int lim = w.lim(c);
      for (int r = 0; r < lim; ++r) {
        const float xf = X[r];
        float o = qnan();
        if (cnt >= 0 || !isnan(xf)) {
          ++cnt;
          if (cnt > 0) {
            const R d = (R)xf - (R)X[r - 1];
            const R g = d > (R)0 ? d : (R)0, l = g - d;
            if (cnt > p) {
              gain = (gain * pm1 + g) * inv;
              loss = (loss * pm1 + l) * inv;
            } else if (cnt < p) {
              gain += g;
              loss += l;
            } else {
              gain = (gain + g) * inv;
              loss = (loss + l) * inv;
            }
          }
          if (cnt >= p) o = rsi_out(gain, loss);
        }
        st[r] = o;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// MACD (talib08:9316-9505): slow seed = SMA of the first `slow` bars, fast seed
// = SMA of the `fast` bars ending there, signal seeded by the SMA of the first
// `signal` MACD values; FP64 lines (fast - slow cancels); leading NaNs skipped.
__device__ void w_macd(const Warp& w, const Job& j) {
  const int pl = j.in[0], fast = j.ip[0], slow = j.ip[1], sig = j.ip[2];
  const double fb = j.fp[0], fk = j.fp[1], sb = j.fp[2], sk = j.fp[3];
  double gb, gk;
  talib_ema_coeffs(sig, gb, gk);
  const int start = slow - 1, ready = start + sig - 1;
  double ps = 0.0, pf = 0.0, psig = 0.0;
  int cnt = -1;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    float* st0 = w.stage_row(0);
    float* st1 = w.stage_row(1);
    float* st2 = w.stage_row(2);
    if (all_lanes(cnt >= ready)) {
      const int n8 = w.lim8(c);
      for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 1
        for (int u = 0; u < 8; ++u) {
          const int r = r8 + u;
          const double x = (double)X[r];
          pf = fma(fb, pf, fk * x);
          ps = fma(sb, ps, sk * x);
          const double m = pf - ps;
          psig = sig == 1 ? m : fma(gb, psig, gk * m);
          st0[r] = (float)m;
          st1[r] = (float)psig;
          st2[r] = (float)(m - psig);
        }
      }
      cnt += n8;
    } else {
      const int lim = w.lim(c);
      for (int r = 0; r < lim; ++r) {
        const float xf = X[r];
        float o0 = qnan(), o1 = qnan(), o2 = qnan();
        if (cnt >= 0 || !isnan(xf)) {
          ++cnt;
          const double x = (double)xf;
          if (cnt > start) {
            pf = fma(fb, pf, fk * x);
            ps = fma(sb, ps, sk * x);
          } else if (cnt < start) {
            ps += x;
            if (cnt >= slow - fast) pf += x;
          } else {
            ps = (ps + x) / slow;
            pf = (pf + x) / fast;
          }
          if (cnt >= start) {
            const double m = pf - ps;
            if (cnt > ready) psig = sig == 1 ? m : fma(gb, psig, gk * m);
            else if (cnt < ready) psig += m;
            else psig = (psig + m) / sig;
            if (cnt >= ready) {
              o0 = (float)m;
              o1 = (float)psig;
              o2 = (float)(m - psig);
            }
          }
        }
        st0[r] = o0;
        st1[r] = o1;
        st2[r] = o2;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.flush(1, (float*)j.out[1], c);
    w.flush(2, (float*)j.out[2], c);
    w.release(c);
  }
}

// TA-Lib TRUE_RANGE: the greatest of H-L, |prevC-H|, |prevC-L| by strict
// comparisons in that order.
template <class R>
__device__ __forceinline__ R true_range_r(R hi, R lo, R yc) {
  R g = hi - lo;
  const R a = fabs(yc - hi);
  if (a > g) g = a;
  const R b = fabs(yc - lo);
  if (b > g) g = b;
  return g;
}

// ATR / NATR / TRANGE (mode 0/1/2): Wilder smoothing of the true range from
// bar 1, fma(wb, y, wa*tr) (talib08 TA_ATR; StreamStates.h:675-721).
template <class R>
__device__ __forceinline__ float atr_out(int mode, int p, R y, R cl) {
  if (mode == 0 || p == 1) return (float)y;
  return cl == (R)0 ? 0.0f : (float)(fdiv(y, cl) * (R)100);
}

template <class R>
__device__ void w_atr(const Warp& w, const Job& j, int mode) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2];
  const int p = mode == 2 ? 1 : j.ip[0];
  const R wb = (R)j.fp[0], wa = (R)j.fp[1];
  R y = 0;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* H = w.X(c, ph);
    const float* Lo = w.X(c, plo);
    const float* Cl = w.X(c, pc);
    float* st = w.stage_row(0);
    const int t0 = c * C;
    if (t0 > p || (mode == 2 && t0 >= 1)) {
      R cp = (R)Cl[-1];
      const int n8 = w.lim8(c);
      for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 1
        for (int u = 0; u < 8; ++u) {
          const int r = r8 + u;
          const R cl = (R)Cl[r];
          const R tr = true_range_r<R>((R)H[r], (R)Lo[r], cp);
          cp = cl;
          if (mode == 2) st[r] = (float)tr;
          else {
            y = fma(wb, y, wa * tr);
            st[r] = atr_out<R>(mode, p, y, cl);
          }
        }
      }
    } else {
      const int lim = w.lim(c);
      for (int r = 0; r < lim; ++r) {
        const int t = t0 + r;
        float o = qnan();
        if (t >= 1) {
          const R tr = true_range_r<R>((R)H[r], (R)Lo[r], (R)Cl[r - 1]);
          if (mode == 2) o = (float)tr;
          else {
            if (t > p) y = fma(wb, y, wa * tr);
            else if (t < p) y += tr;
            else y = (y + tr) / (R)p;
            if (t >= p) o = atr_out<R>(mode, p, y, (R)Cl[r]);
          }
        }
        st[r] = o;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// ADX / DX (src/indicators/DX.cu, ADX.cu; BatchShort.cu:168-230 conventions):
// Wilder sums of the true range and directional movements, DI+/DI-, DX, and
// for ADX the Wilder mean of DX seeded at 2p-1.
template <class R>
struct DmBar {
  R range, plus, minus;
};

template <class R>
__device__ __forceinline__ DmBar<R> dm_bar(float h, float l, float hp, float lp, float cp) {
  DmBar<R> b;
  const float u = h - hp, dw = lp - l;
  b.plus = (u > 0.0f && u > dw) ? (R)u : (R)0;
  b.minus = (dw > 0.0f && dw > u) ? (R)dw : (R)0;
  const R hh = (R)h, ll = (R)l, yc = (R)cp;
  b.range = fmax(hh - ll, fmax(fabs(hh - yc), fabs(ll - yc)));
  return b;
}

template <class R>
__device__ __forceinline__ R dx_of(R tr, R pd, R md) {
  const R dip = tr > (R)0 ? fdiv((R)100 * pd, tr) : (R)0;
  const R dim = tr > (R)0 ? fdiv((R)100 * md, tr) : (R)0;
  const R tot = dip + dim;
  return tot > (R)0 ? fdiv((R)100 * fabs(dip - dim), tot) : (R)0;
}

template <class R>
__device__ void w_adx(const Warp& w, const Job& j, bool adx) {
  const int ph = j.in[0], plo = j.in[1], pc = j.in[2], p = j.ip[0];
  const R a = (R)(((double)p - 1.0) / (double)p), invp = (R)(1.0 / (double)p);
  R tr = 0, pd = 0, md = 0, av = 0;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* H = w.X(c, ph);
    const float* Lo = w.X(c, plo);
    const float* Cl = w.X(c, pc);
    float* st = w.stage_row(0);
    const int t0 = c * C;
    if (t0 > (adx ? 2 * p - 1 : p)) {
      float hp = H[-1], lp = Lo[-1], cp = Cl[-1];
      const int n8 = w.lim8(c);
      for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 1
        for (int u = 0; u < 8; ++u) {
          const int r = r8 + u;
          const float h = H[r], l = Lo[r];
          const DmBar<R> b = dm_bar<R>(h, l, hp, lp, cp);
          hp = h;
          lp = l;
          cp = Cl[r];
          tr = a * tr + b.range;
          pd = a * pd + b.plus;
          md = a * md + b.minus;
          const R dx = dx_of(tr, pd, md);
          if (adx) {
            av = a * av + dx * invp;
            st[r] = (float)av;
          } else {
            st[r] = (float)dx;
          }
        }
      }
    } else {
      const int lim = w.lim(c);
      for (int r = 0; r < lim; ++r) {
        const int t = t0 + r;
        DmBar<R> b;
        if (t == 0) {
          b.range = (R)H[r] - (R)Lo[r];
          b.plus = b.minus = (R)0;
        } else {
          b = dm_bar<R>(H[r], Lo[r], H[r - 1], Lo[r - 1], Cl[r - 1]);
        }
        float o = qnan();
        if (t < p) {
          tr += b.range;
          pd += b.plus;
          md += b.minus;
        } else {
          tr = a * tr + b.range;
          pd = a * pd + b.plus;
          md = a * md + b.minus;
          const R dx = dx_of(tr, pd, md);
          if (!adx) o = (float)dx;
          else if (t > 2 * p - 1) {
            av = a * av + dx * invp;
            o = (float)av;
          } else if (t < 2 * p - 1) {
            av += dx;
          } else {
            av = (av + dx) / (R)p;
            o = (float)av;
          }
        }
        st[r] = o;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// OBV / AD / ADOSC (mode 0/1/2; StreamStates.h:446-506, 723-745): FP64
// cumulative sums; ADOSC's EMAs of AD from bar 0.
__device__ void w_volume(const Warp& w, const Job& j, int mode) {
  double acc = 0.0, fastv = 0.0, slowv = 0.0;
  const int warm = mode == 2 ? (j.ip[0] > j.ip[1] ? j.ip[0] : j.ip[1]) - 1 : 0;
  const double kf = mode == 2 ? 2.0 / (j.ip[0] + 1.0) : 0.0, ks = mode == 2 ? 2.0 / (j.ip[1] + 1.0) : 0.0;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* I0 = w.X(c, j.in[0]);
    const float* I1 = w.X(c, j.in[1]);
    const float* I2 = mode ? w.X(c, j.in[2]) : I0;
    const float* I3 = mode ? w.X(c, j.in[3]) : I0;
    float* st = w.stage_row(0);
    const int t0 = c * C;
    if (mode == 0 && t0 >= 1) {
      float pp = I0[-1];
      const int n8 = w.lim8(c);
      for (int r8 = 0; r8 < n8; r8 += 8) {
#pragma unroll 1
        for (int u = 0; u < 8; ++u) {
          const int r = r8 + u;
          const double v = (double)I1[r];
          const float pr = I0[r];
          acc += pr > pp ? v : (pr < pp ? -v : 0.0 * v);
          pp = pr;
          st[r] = (float)acc;
        }
      }
    } else {
      const int lim = w.lim(c);
      for (int r = 0; r < lim; ++r) {
        const int t = t0 + r;
        float o;
        if (mode == 0) {
          const double v = (double)I1[r];
          if (t == 0) acc += v;
          else {
            const float pr = I0[r], pp = I0[r - 1];
            acc += pr > pp ? v : (pr < pp ? -v : 0.0 * v);
          }
          o = (float)acc;
        } else {
          const double hi = I0[r], lo = I1[r], cl = I2[r], vo = I3[r];
          double term = 0.0;
          if (isfinite(hi) && isfinite(lo) && isfinite(cl) && isfinite(vo)) {
            const double range = hi - lo;
            if (range > 0.0) term = (((cl - lo) - (hi - cl)) / range) * vo;
          }
          acc += term;
          if (mode == 1) o = (float)acc;
          else {
            if (t == 0) fastv = slowv = acc;
            else {
              fastv = kf * acc + (1.0 - kf) * fastv;
              slowv = ks * acc + (1.0 - ks) * slowv;
            }
            o = t < warm ? qnan() : (float)(fastv - slowv);
          }
        }
        st[r] = o;
      }
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// ------------------------------------------------------ further families
// The families below follow the same TA-Lib / reference conventions as the
// warp-scan engine's round functions (families.cuh), one thread per row.

// DEMA / TEMA / T3 cascades (talib08:4846-4945, 17496-17612, 17331-17481):
// stage k+1 is seeded with the SMA of stage k's first p values; FP64 stages.
__device__ void w_cascade(const Warp& w, const Job& j, int stages) {
  const int pl = j.in[0], p = j.ip[0];
  const double beta = j.fp[0], kk = j.fp[1];
  double c1 = 0, c2 = 0, c3 = 0, c4 = 0;
  if (stages == 6) {
    const double v = j.fp[2], tr = v * v;
    c1 = -(tr * v);
    c2 = 3.0 * (tr - c1);
    c3 = -6.0 * tr - 3.0 * (v - c1);
    c4 = fma(3.0, tr, fma(3.0, v, 1.0) - c1);
  }
  double e[6] = {0, 0, 0, 0, 0, 0};
  int cnt = -1;
  const int lb = stages * (p - 1);
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    const int lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const double x = X[r];
      float o = qnan();
      if (cnt >= 0 || !isnan(x)) {
        ++cnt;
        double in = x;
#pragma unroll
        for (int s = 0; s < 6; ++s) {
          if (s < stages) {
            const int rr = cnt - s * (p - 1);
            if (rr >= 0) {
              if (p == 1) e[s] = in;
              else if (rr < p - 1) e[s] += in;
              else if (rr == p - 1) e[s] = (e[s] + in) / p;
              else e[s] = fma(beta, e[s], kk * in);
            }
            in = e[s];
          }
        }
        if (cnt >= lb) {
          if (p == 1) o = (float)x;
          else if (stages == 2) o = (float)(2.0 * e[0] - e[1]);
          else if (stages == 3) o = (float)(e[2] + (3.0 * e[0] - 3.0 * e[1]));
          else o = (float)fma(c4, e[2], fma(c3, e[3], fma(c1, e[5], c2 * e[4])));
        }
      }
      w.put(0, r, o);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// LINEARREG (talib08:9087-9197): TA-Lib's sliding SumY / SumXY about a
// window-start origin, re-derived directly at each chunk's first output bar.
__device__ void w_linreg(const Warp& w, const Job& j) {
  const int pl = j.in[0], p = j.ip[0];
  const double sumX = (double)p * (p - 1) * 0.5;
  const double sumXSqr = (double)p * (p - 1) * (2 * p - 1) / 6.0;
  const double divisor = sumX * sumX - p * sumXSqr;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    const int t0 = c * C, lim = w.lim(c);
    double sy = 0.0, sxy = 0.0, o = 0.0;
    int nn = 0;
    bool seeded = false;
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      float out = qnan();
      if (t >= p - 1) {
        if (!seeded) {
          seeded = true;
          const float ov = X[r];
          o = isnan(ov) ? 0.0 : (double)ov;
          for (int i = p - 1; i >= 0; --i) {
            const float v = X[r - i];
            if (isnan(v)) ++nn;
            else {
              const double d = (double)v - o;
              sy += d;
              sxy += (double)i * d;
            }
          }
        } else {
          const float vout = X[r - p], vin = X[r];
          const double dout = isnan(vout) ? 0.0 : (double)vout - o;
          const double din = isnan(vin) ? 0.0 : (double)vin - o;
          sxy = sxy + sy - (double)p * dout;
          sy = sy - dout + din;
          nn += (isnan(vin) ? 1 : 0) - (isnan(vout) ? 1 : 0);
        }
        if (nn == 0) {
          const double m = (p * sxy - sumX * sy) / divisor;
          const double b = (sy - m * sumX) / (double)p;
          out = (float)(o + fma(m, (double)(p - 1), b));
        }
      }
      w.put(0, r, out);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// CORREL (src/indicators/Correl.cu:23-75): window moments about the window
// start, re-derived at each chunk's first output bar; 0 from the row's first
// non-finite bar on.
__device__ void w_correl(const Warp& w, const Job& j) {
  const int px = j.in[0], py = j.in[1], p = j.ip[0];
  int bad = -1;
  const double pp = (double)p;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* Xx = w.X(c, px);
    const float* Xy = w.X(c, py);
    const int t0 = c * C, lim = w.lim(c);
    double sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0, ox = 0, oy = 0;
    bool seeded = false;
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      if (bad < 0 && (!isfinite(Xx[r]) || !isfinite(Xy[r]))) bad = t;
      float o = qnan();
      if (t >= p - 1) {
        if (!seeded) {
          seeded = true;
          ox = Xx[r - p + 1];
          oy = Xy[r - p + 1];
          if (!isfinite(ox)) ox = 0.0;
          if (!isfinite(oy)) oy = 0.0;
          for (int i = 0; i < p; ++i) {
            const double dx = (double)Xx[r - p + 1 + i] - ox, dy = (double)Xy[r - p + 1 + i] - oy;
            sx += dx; sy += dy; sxx += dx * dx; syy += dy * dy; sxy += dx * dy;
          }
        } else {
          const double ax = (double)Xx[r - p] - ox, ay = (double)Xy[r - p] - oy;
          const double bx = (double)Xx[r] - ox, by = (double)Xy[r] - oy;
          sx += bx - ax; sy += by - ay;
          sxx += bx * bx - ax * ax; syy += by * by - ay * ay; sxy += bx * by - ax * ay;
        }
        if (bad >= 0 && t >= bad) o = 0.0f;
        else {
          const double cov = sxy - sx * sy / pp;
          const double vx = sxx - sx * sx / pp, vy = syy - sy * sy / pp;
          const double prod = vx * vy;
          o = (vx > 0.0 && vy > 0.0 && prod > 1e-14) ? (float)(cov / sqrt(prod)) : 0.0f;
        }
      }
      w.put(0, r, o);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// MIN / MAX (BatchFused.cu:110-119): fminf / fmaxf over the window; a window
// starting inside the row's leading NaN run stays NaN. mid: MIDPOINT =
// 0.5f * (max + min) (src/indicators/MIDPOINT.cu:24-34).
__device__ void w_minmax(const Warp& w, const Job& j, bool is_max, bool mid) {
  const int pl = j.in[0], p = j.ip[0];
  int f = -1;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    const int t0 = c * C, lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      if (f < 0 && !isnan(X[r])) f = t;
      float o = qnan();
      if (t >= p - 1 && f >= 0 && t - p + 1 >= f) {
        if (mid) {
          float hi = X[r - p + 1], lo = hi;
          for (int i = 1; i < p; ++i) {
            hi = fmaxf(hi, X[r - p + 1 + i]);
            lo = fminf(lo, X[r - p + 1 + i]);
          }
          o = 0.5f * (hi + lo);
        } else {
          o = X[r - p + 1];
          for (int i = 1; i < p; ++i) o = is_max ? fmaxf(o, X[r - p + 1 + i]) : fminf(o, X[r - p + 1 + i]);
        }
      }
      w.put(0, r, o);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// ROC / ROCP / ROCR / ROCR100 / MOM: the reference's float32 kernels
// (roc_value in families.cuh), bit for bit.
__device__ __forceinline__ float roc_value_f(float curr, float prev, int mode) {
  if (mode == 4) return curr - prev;
  if (!(prev != 0.0f)) return 0.0f;
  switch (mode) {
    case 0: return ((curr - prev) / prev) * 100.0f;
    case 1: return (curr - prev) / prev;
    case 2: return curr / prev;
    default: return (curr / prev) * 100.0f;
  }
}

__device__ void w_roc(const Warp& w, const Job& j, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    const int t0 = c * C, lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      w.put(0, r, t >= p ? roc_value_f(X[r], X[r - p], mode) : qnan());
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// MEDPRICE / TYPPRICE / AVGPRICE / WCLPRICE: the reference's float32 kernels.
__device__ void w_price(const Warp& w, const Job& j, int mode) {
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* A = w.X(c, j.in[0]);
    const float* B = w.X(c, j.in[1]);
    const float* C2 = mode >= 1 ? w.X(c, j.in[2]) : A;
    const float* D = mode == 2 ? w.X(c, j.in[3]) : A;
    const int lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const float a = A[r], b = B[r];
      float o;
      if (mode == 0) o = 0.5f * (a + b);
      else if (mode == 1) o = (a + b + C2[r]) / 3.0f;
      else if (mode == 2) o = (a + b + C2[r] + D[r]) * 0.25f;
      else o = (a + b + 2.0f * C2[r]) * 0.25f;
      w.put(0, r, o);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// MIDPRICE (src/indicators/MIDPRICE.cu:11-24): fmaxf / fminf window extrema.
__device__ void w_midprice(const Warp& w, const Job& j) {
  const int ph = j.in[0], plo = j.in[1], p = j.ip[0];
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* H = w.X(c, ph);
    const float* Lo = w.X(c, plo);
    const int t0 = c * C, lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      float o = qnan();
      if (t >= p - 1) {
        float hi = H[r - p + 1], lo = Lo[r - p + 1];
        for (int i = 1; i < p; ++i) {
          hi = fmaxf(hi, H[r - p + 1 + i]);
          lo = fminf(lo, Lo[r - p + 1 + i]);
        }
        o = 0.5f * (hi + lo);
      }
      w.put(0, r, o);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// NaN-strict rolling mean / max / min / std (src/indicators/ClubPack.cu:375-407):
// any non-finite value in the window gives NaN; the std writes the reference's
// contracted fma(-mean, mean, sq / p).
__device__ void w_rolling(const Warp& w, const Job& j, int mode) {
  const int pl = j.in[0], p = j.ip[0];
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* X = w.X(c, pl);
    const int t0 = c * C, lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      float o = qnan();
      if (t >= p - 1) {
        bool ok = true;
        double sum = 0.0, sq = 0.0;
        float mx = X[r], mn = mx;
        for (int i = 0; i < p; ++i) {
          const float v = X[r - i];
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
      w.put(0, r, o);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// IBS / MARKETFI (talib_bar_round in families.cuh): the reference's TA-Lib
// runner starts a row at its first bar with no NaN input
// (src/compat/Talib08.cu:72-84); TA_IBS / TA_MARKETFI in FP64.
__device__ void w_talib_bar(const Warp& w, const Job& j, int mode) {
  const int p0 = j.in[0], p1 = j.in[1], p2 = j.in[2];
  int f = -1;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* A = w.X(c, p0);
    const float* B = w.X(c, p1);
    const float* Z = w.X(c, p2);
    const int t0 = c * C, lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      if (f < 0 && !isnan(A[r]) && !isnan(B[r]) && !isnan(Z[r])) f = t;
      float o = qnan();
      if (f >= 0 || t == w.n - 1) {
        const double a = A[r], b = B[r], z = Z[r];
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
      w.put(0, r, o);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// QSTICK (qstick_round in families.cuh): TA_QSTICK's mean of close - open from
// the runner's start bar; after a NaN difference every later output is NaN,
// and so is every output from p bars after an infinite difference (the
// running sum's inf - inf when it leaves the window).
__device__ void w_qstick(const Warp& w, const Job& j) {
  const int po = j.in[0], pc = j.in[1], p = j.ip[0];
  int f = -1;
  long long stop = 1ll << 62;
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* O = w.X(c, po);
    const float* C2 = w.X(c, pc);
    const int t0 = c * C, lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      if (f < 0 && !isnan(O[r]) && !isnan(C2[r])) f = t;
      if (f >= 0) {
        const double d = (double)C2[r] - (double)O[r];
        if (isnan(d)) stop = min(stop, (long long)t);
        else if (isinf(d)) stop = min(stop, (long long)t + p);
      }
      float o = qnan();
      if (f >= 0 && t >= f + p - 1 && t < stop) {
        double s = 0.0;
        for (int i = r - p + 1; i <= r; ++i) s += (double)C2[i] - (double)O[i];
        o = (float)(s / (double)p);
      }
      w.put(0, r, o);
    }
    w.flush(0, (float*)j.out[0], c);
    w.release(c);
  }
}

// AROON / AROONOSC (aroon_round in families.cuh): each bar scans its window
// back from itself with strict comparisons, as the reference's kernels do.
__device__ void w_aroon(const Warp& w, const Job& j, int mode) {
  const int ph = j.in[0], plo = j.in[1], p = j.ip[0];
  for (int c = 0; c < w.nchunks; ++c) {
    if (!w.wait(c)) return;
    const float* H = w.X(c, ph);
    const float* Lo = w.X(c, plo);
    const int t0 = c * C, lim = w.lim(c);
    for (int r = 0; r < lim; ++r) {
      const int t = t0 + r;
      float up = qnan(), dn = qnan();
      if (t >= p) {
        float mx = H[r], mn = Lo[r];
        int sh = 0, sl = 0;
        for (int d = 1; d <= p; ++d) {
          const float h = H[r - d], l = Lo[r - d];
          if (h > mx) { mx = h; sh = d; }
          if (l < mn) { mn = l; sl = d; }
        }
        up = aroon_line(p, sh);
        dn = aroon_line(p, sl);
      }
      if (mode == 0) {
        w.put(0, r, dn);
        w.put(1, r, up);
      } else {
        w.put(0, r, t >= p ? up - dn : qnan());
      }
    }
    w.flush(0, (float*)j.out[0], c);
    if (mode == 0) w.flush(1, (float*)j.out[1], c);
    w.release(c);
  }
}

}  // namespace rows
}  // namespace tb
