// Row-parallel engine: kernel and launcher (see rows.cuh for the design).
#include "rows.cuh"
#include "rows_bars.cuh"

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "jobs.h"
#include "scheduler.h"

namespace tb {
namespace rows {

// Jobs run bar-parallel (rows_bars.cuh), as a mask of families. CCI sums its
// windows directly in either form, so it always goes bar-parallel, where a
// team of warps shares it. WILLR and STOCH give the same bits in both forms
// (window extremes are exact); bar-parallel costs more instructions but
// splits over a team, which pays only when few jobs share the CTA. The other
// window families keep their running row-sequential form.
static_assert(F_COUNT <= 64, "bar-parallel family mask holds 64 families");
inline unsigned long long bar_parallel_mask(int njobs) {
  unsigned long long m = 1ull << F_CCI;
  if (njobs <= 4) m |= (1ull << F_WILLR) | (1ull << F_STOCH);
  return m;
}
__host__ __device__ inline bool bar_parallel(unsigned long long mask, int family) {
  return family >= 0 && family < 64 && ((mask >> family) & 1ull) != 0;
}

// Per-lane history line of a row-sequential job (entries per lane, a power of
// two; 0: none).
__host__ __device__ inline int line_entries(const Job& j) {
  int need = 0;
  switch (j.family) {
    case F_WILLR: need = j.ip[0]; break;
    case F_STOCH: need = j.ip[0] > j.ip[1] ? j.ip[0] : j.ip[1]; break;
    case F_MFI: need = j.ip[0] + 1; break;
    default: return 0;
  }
  int cap = 1;
  while (cap < need) cap <<= 1;
  return cap;
}

// Bytes of a job warp's own lines.
__host__ __device__ inline int line_bytes(const Job& j, unsigned long long bp) {
  if (bar_parallel(bp, j.family)) {
    switch (j.family) {
      case F_STOCH: return 2 * kBarLine * 4;
      case F_CCI: return kBarLine * 8;
      default: return 0;
    }
  }
  const int cap = line_entries(j);
  switch (j.family) {
    case F_WILLR: return 2 * 32 * cap * 4;
    case F_STOCH: return 4 * 32 * cap * 4;
    case F_MFI: return 2 * 32 * cap * 8;
    default: return 0;
  }
}

__host__ __device__ inline int out_count(int family) {
  return family == F_MACD || family == F_BBANDS ? 3 : (family == F_STOCH || family == F_AROON ? 2 : 1);
}

// Families of the core kernel: the indicators of the reference's fused batch
// path and the window / recurrence families around them. A launch whose jobs
// are all core families runs rows_kernel<false>, which leaves the other
// families' code out: its hot loops then sit in a smaller code image (the
// 13-indicator pass measured 8 % faster than in the kernel with every family).
__host__ __device__ inline bool core_family(int f) {
  switch (f) {
    case F_SMA: case F_SUM: case F_WMA: case F_BBANDS: case F_STDDEV: case F_VAR: case F_WILLR: case F_STOCH:
    case F_CCI: case F_MFI: case F_EMA: case F_RMA: case F_RSI: case F_MACD: case F_ATR: case F_NATR:
    case F_TRANGE: case F_ADX: case F_DX: case F_OBV: case F_AD: case F_ADOSC:
      return true;
    default:
      return false;
  }
}

template <bool kAll>
__device__ void run_job(const Warp& w, const Job& j, unsigned char* line) {
  const bool f32 = j.ip[0] <= kFp32MaxPeriod;
  switch (j.family) {
    case F_SMA: w_sum_window(w, j, 0); break;
    case F_SUM: w_sum_window(w, j, 1); break;
    case F_WMA: w_sum_window(w, j, 2); break;
    case F_BBANDS: w_moment_window(w, j, 0); break;
    case F_STDDEV: w_moment_window(w, j, 1); break;
    case F_VAR: w_moment_window(w, j, 2); break;
    case F_WILLR:
      if (bar_parallel(w.lay->bp_mask, F_WILLR)) b_willr(w, j);
      else w_willr(w, j, reinterpret_cast<float*>(line), line_entries(j));
      break;
    case F_STOCH:
      if (bar_parallel(w.lay->bp_mask, F_STOCH)) b_stoch(w, j, reinterpret_cast<float*>(line));
      else if (j.ip[1] == 3) w_stoch<3>(w, j, reinterpret_cast<float*>(line), line_entries(j));
      else w_stoch<0>(w, j, reinterpret_cast<float*>(line), line_entries(j));
      break;
    case F_CCI: b_cci(w, j, reinterpret_cast<double*>(line)); break;
    case F_MFI: w_mfi(w, j, reinterpret_cast<double*>(line), line_entries(j)); break;
    case F_EMA: case F_RMA:
      if (f32) w_ema<float>(w, j); else w_ema<double>(w, j);
      break;
    case F_RSI:
      if (f32) w_rsi<float>(w, j); else w_rsi<double>(w, j);
      break;
    case F_MACD: w_macd(w, j); break;
    case F_ATR:
      if (f32) w_atr<float>(w, j, 0); else w_atr<double>(w, j, 0);
      break;
    case F_NATR:
      if (f32) w_atr<float>(w, j, 1); else w_atr<double>(w, j, 1);
      break;
    case F_TRANGE: w_atr<float>(w, j, 2); break;
    case F_ADX:
      if (f32) w_adx<float>(w, j, true); else w_adx<double>(w, j, true);
      break;
    case F_DX: w_adx<double>(w, j, false); break;
    case F_OBV: w_volume(w, j, 0); break;
    case F_AD: w_volume(w, j, 1); break;
    case F_ADOSC: w_volume(w, j, 2); break;
    default:
      if constexpr (kAll) {
        switch (j.family) {
          case F_DEMA: w_cascade(w, j, 2); return;
          case F_TEMA: w_cascade(w, j, 3); return;
          case F_T3: w_cascade(w, j, 6); return;
          case F_LINEARREG: w_linreg(w, j); return;
          case F_CORREL: w_correl(w, j); return;
          case F_MIN: w_minmax(w, j, false, false); return;
          case F_MAX: w_minmax(w, j, true, false); return;
          case F_MIDPOINT: w_minmax(w, j, false, true); return;
          case F_ROC: w_roc(w, j, 0); return;
          case F_ROCP: w_roc(w, j, 1); return;
          case F_ROCR: w_roc(w, j, 2); return;
          case F_ROCR100: w_roc(w, j, 3); return;
          case F_MOM: w_roc(w, j, 4); return;
          case F_MEDPRICE: w_price(w, j, 0); return;
          case F_TYPPRICE: w_price(w, j, 1); return;
          case F_AVGPRICE: w_price(w, j, 2); return;
          case F_WCLPRICE: w_price(w, j, 3); return;
          case F_MIDPRICE: w_midprice(w, j); return;
          case F_RMEAN: w_rolling(w, j, 0); return;
          case F_RMAX: w_rolling(w, j, 1); return;
          case F_RMIN: w_rolling(w, j, 2); return;
          case F_RSTD: w_rolling(w, j, 3); return;
          case F_IBS: w_talib_bar(w, j, 0); return;
          case F_MARKETFI: w_talib_bar(w, j, 1); return;
          case F_QSTICK: w_qstick(w, j); return;
          case F_AROON: w_aroon(w, j, 0); return;
          case F_AROONOSC: w_aroon(w, j, 1); return;
          default: break;
        }
      }
      // unreachable: the launcher admits only the families above
      for (int c = 0; c < w.nchunks; ++c) {
        if (!w.wait(c)) return;
        w.release(c);
      }
  }
}

// Producer warp: stages chunk c of every plane for the 32 rows once the job
// warps have released the chunk that last used its slot.
__device__ void produce(const Launch& L, const Layout& lay, unsigned char* smem, uint64_t* full, uint64_t* empty,
                        const long long* tbase, const long long* tn, volatile int* abort_flag, int* err,
                        int nchunks, int lane, long long group) {
  float* ring = reinterpret_cast<float*>(smem + lay.ring_off);
  const int NS = lay.NS, Hs = lay.Hs, RS = lay.RS;
  const bool uni = !L.order && !L.offsets;
  const long long s0T = group * 32 * L.T;
  const int nvalid = (int)min(32ll, (long long)L.S - group * 32);
  const unsigned long long limit = L.stall_test ? kStallWaitNs : kWaitNs;
  for (int c = 0; c < nchunks; ++c) {
    const int s = c % NS, use = c / NS;
    if (use > 0 && !mbar_wait(&empty[s], (unsigned)((use - 1) & 1), abort_flag, err, lane, limit)) break;
    const long long t = (long long)c * C + lane;
    const bool mir = s >= NS - Hs;
    const int off = (Hs + s) * C + lane, moff = (s - (NS - Hs)) * C + lane;
    for (int q = 0; q < lay.nplanes; ++q) {
      const float* base = L.plane[lay.slot_plane[q]];
      float* dst = ring + (size_t)q * 32 * RS;
      if (uni) {
        // rows of the group are consecutive rows of T bars
        const bool in_row = t < L.T;
        const float* src = base + s0T + t;
#pragma unroll 4
        for (int i = 0; i < 32; ++i) {
          const bool ok = in_row && i < nvalid;
          const float* sp = ok ? src + (long long)i * L.T : base;
          cp_async4(dst + i * RS + off, sp, ok);
          if (mir) cp_async4(dst + i * RS + moff, sp, ok);
        }
      } else {
#pragma unroll 4
        for (int i = 0; i < 32; ++i) {
          const long long b = tbase[i];
          const bool ok = b >= 0 && t < tn[i];
          const float* sp = ok ? base + b + t : base;
          cp_async4(dst + i * RS + off, sp, ok);
          if (mir) cp_async4(dst + i * RS + moff, sp, ok);
        }
      }
    }
    // test knob: chunk 0 is never announced, so the job warps' first wait runs out
    if (!(L.stall_test && c == 0)) cp_async_arrive(&full[s]);
  }
  cp_async_wait_all();
}

// CTA x of partition y (cta0[y] <= x < cta0[y+1]) runs row groups
// (x - cta0[y])*G[y] .. +G[y]-1 of that partition's jobs; each group has its
// own warps, ring, mbarriers and tables (a block of lay.total bytes of shared
// memory), so the groups of a CTA run independently.
template <bool kAll>
__global__ void __launch_bounds__(32 * kMaxWarps, 1) rows_kernel(const __grid_constant__ Launch L, const __grid_constant__ Split sp) {
  extern __shared__ __align__(16) unsigned char smem_all[];
  int y = 0;
  while (y + 1 < sp.P && (int)blockIdx.x >= sp.cta0[y + 1]) ++y;
  const Layout& lay = sp.lay[y];
  const int G = sp.G[y];
  const int wpg = lay.nconsumers + 1;
  const int gw = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = gw / wpg, warp = gw - sub * wpg;
  const long long group = (long long)((int)blockIdx.x - sp.cta0[y]) * G + sub;
  const bool live = sub < G && group * 32 < (long long)L.S;
  unsigned char* smem = smem_all + (size_t)(live ? sub : 0) * lay.total;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + lay.bar_off);
  uint64_t* empty = full + lay.NS;
  long long* tbase = reinterpret_cast<long long*>(smem + lay.tab_off);
  long long* tn = tbase + 32;
  int* misc = reinterpret_cast<int*>(tn + 32);  // [0] longest row of the group, [1] abort
  int* err = L.sticky;
  if (live && warp == 0) {
    const long long idx = group * 32 + lane;
    long long b = -1, n = 0;
    if (idx < L.S) {
      const int s = L.order ? L.order[idx] : (int)idx;
      if (L.offsets) {
        b = L.offsets[s];
        n = L.offsets[s + 1] - b;
      } else {
        b = (long long)s * L.T;
        n = L.T;
      }
    }
    tbase[lane] = b;
    tn[lane] = n;
    const int m = warp_max_int((int)min(n, (long long)INT_MAX));
    if (lane == 0) {
      misc[0] = m;
      misc[1] = 0;
      for (int s = 0; s < lay.NS; ++s) {
        mbar_init(&full[s], 32);
        mbar_init(&empty[s], (unsigned)lay.nconsumers);
      }
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
  }
  __syncthreads();
  if (!live) return;
  const int maxn = misc[0];
  const int nchunks = (maxn + C - 1) / C;
  volatile int* abort_flag = misc + 1;
  if (warp == lay.producer_warp) {
    produce(L, lay, smem, full, empty, tbase, tn, abort_flag, err, nchunks, lane, group);
    return;
  }
  if (warp > lay.nconsumers) return;
  Warp w;
  w.smem = smem;
  w.lay = &lay;
  w.full = full;
  w.empty = empty;
  w.tbase = tbase;
  w.tn = tn;
  w.abort_flag = abort_flag;
  w.err = err;
  w.wait_ns = L.stall_test ? kStallWaitNs : kWaitNs;
  w.stage = reinterpret_cast<float*>(smem + lay.stage_off[warp]);
  w.lane = lane;
  w.nchunks = nchunks;
  w.maxn = maxn;
  w.Hs = lay.Hs;
  w.NS = lay.NS;
  w.RS = lay.RS;
  w.n = tn[lane];
  w.uni = !L.order && !L.offsets;
  w.T = L.T;
  w.s0T = group * 32 * L.T;
  w.nvalid = (int)min(32ll, (long long)L.S - group * 32);
  w.tk = lay.warp_team[warp] & 255;
  w.tm = lay.warp_team[warp] >> 8;
  run_job<kAll>(w, L.jobs[lay.warp_job[warp]], smem + lay.line_off[warp]);
}

namespace {

bool family_supported(int f) {
  switch (f) {
    case F_SMA: case F_SUM: case F_WMA: case F_BBANDS: case F_STDDEV: case F_VAR: case F_WILLR: case F_STOCH:
    case F_CCI: case F_MFI: case F_EMA: case F_RMA: case F_RSI: case F_MACD: case F_ATR: case F_NATR:
    case F_TRANGE: case F_ADX: case F_DX: case F_OBV: case F_AD: case F_ADOSC: case F_DEMA: case F_TEMA:
    case F_T3: case F_LINEARREG: case F_CORREL: case F_MIN: case F_MAX: case F_MIDPOINT: case F_ROC:
    case F_ROCP: case F_ROCR: case F_ROCR100: case F_MOM: case F_MEDPRICE: case F_TYPPRICE: case F_AVGPRICE:
    case F_WCLPRICE: case F_MIDPRICE: case F_RMEAN: case F_RMAX: case F_RMIN: case F_RSTD: case F_IBS:
    case F_MARKETFI: case F_QSTICK: case F_AROON: case F_AROONOSC:
      return true;
    default:
      return false;
  }
}

// bars of history a job reads before a chunk: one more than its lookback halo
// (the bar leaving a running window, the previous close)
int rows_halo(const Job& j) {
  int h = job_halo(j);
  // WILLR / STOCH rebuild their van Herk blocks at every chunk from up to
  // 2p - 1 bars before it
  if (j.family == F_WILLR || j.family == F_STOCH) h = std::max(h, 2 * j.ip[0] - 1);
  return h + 1;
}

// Jobs split over a team of warps by chunks: row-sequential windows whose
// chunks share no state. Like the bar-parallel WILLR / STOCH, this pays only
// when few jobs share the CTA (a single BBANDS: 53 -> 24 us, MFI: 63 -> 45 us
// at 4000 x 234); with many jobs the SM's issue rate, not one warp's chain,
// bounds the CTA, and the extra warps slowed the 13-indicator pass (181 ->
// 188 us).
inline bool chunk_team(int njobs, int family) {
  if (njobs > 4) return false;
  switch (family) {
    case F_WILLR: case F_STOCH: case F_MFI: case F_BBANDS: case F_STDDEV: case F_VAR:
      return true;
    default:
      return false;
  }
}

struct DevState {
  int sms = 0, smem_optin = 0;
  bool attr = false;
};
std::mutex g_mutex;
std::vector<DevState> g_dev;

// Relative time a job's warp needs for the rows of a CTA, from a per-warp
// timing trace of the 13-indicator pass at 4000 x 234 (microseconds a warp
// was busy, i.e. not waiting on the ring, with the other jobs beside it), for
// the warp placement and the team sizes. A team of m warps divides a job's
// figure by m.
int family_cost(const Job& j, unsigned long long bp) {
  const int p = j.ip[0];
  switch (j.family) {
    case F_CCI: return 36 * p;
    case F_MFI: return 150;
    case F_STOCH: return bar_parallel(bp, F_STOCH) ? 30 * p : 147;
    case F_WILLR: return bar_parallel(bp, F_WILLR) ? 25 * p : 143;
    case F_ADX: case F_DX: return 95;
    case F_BBANDS: return 94;
    case F_MACD: return 87;
    case F_STDDEV: case F_VAR: return 70;
    case F_RSI: return 63;
    case F_WMA: return 60;
    case F_OBV: case F_AD: return 57;
    case F_SMA: case F_SUM: return 53;
    case F_ATR: case F_NATR: return 49;
    case F_EMA: case F_RMA: return 44;
    default: return 40 + 4 * p;
  }
}

// Job warps: one per job, and spare warps up to kMaxConsumers go to the jobs
// that can be split as team members (a bar-parallel job splits its rows, a
// chunk-team job its chunks), each time to the job whose warps carry the most
// work, while that is more than the heaviest job that cannot be split. Warp w of a CTA issues from sub-partition
// w % 4: the job warps and the producer are placed longest-first on the least
// loaded sub-partition, so the heaviest warps do not share one.
void assign_warps(const Launch& L, const int* jl, int nj, Layout& lay, int budget) {
  int team[kMaxConsumers];
  int nw = nj, seq_max = 0;
  for (int j = 0; j < nj; ++j) {
    team[j] = 1;
    const Job& jb = L.jobs[jl[j]];
    if (!bar_parallel(lay.bp_mask, jb.family) && !chunk_team(nj, jb.family))
      seq_max = std::max(seq_max, family_cost(jb, lay.bp_mask));
  }
  while (nw < budget) {
    int best = -1;
    double bc = (double)seq_max;
    for (int j = 0; j < nj; ++j) {
      const Job& jb = L.jobs[jl[j]];
      const int f = jb.family;
      if (!bar_parallel(lay.bp_mask, f) && !chunk_team(nj, f)) continue;
      // a chunk team works on at most the ring's NS - Hs chunks at once
      if (!bar_parallel(lay.bp_mask, f) && team[j] >= lay.NS - lay.Hs) continue;
      const double c = (double)family_cost(jb, lay.bp_mask) / team[j];
      if (c > bc) {
        bc = c;
        best = j;
      }
    }
    if (best < 0) break;
    ++team[best];
    ++nw;
  }
  const int n = nw + 1;  // job warps + producer
  int item_job[kMaxConsumers + 1], item_k[kMaxConsumers + 1], order[kMaxConsumers + 1];
  double cost[kMaxConsumers + 1];
  int i = 0;
  for (int j = 0; j < nj; ++j)
    for (int k = 0; k < team[j]; ++k, ++i) {
      item_job[i] = j;
      item_k[i] = k;
      cost[i] = (double)family_cost(L.jobs[jl[j]], lay.bp_mask) / team[j];
    }
  item_job[i] = -1;
  item_k[i] = 0;
  cost[i] = 18.0 * lay.nplanes;
  for (int k = 0; k < n; ++k) order[k] = k;
  std::stable_sort(order, order + n, [&](int a, int b) { return cost[a] > cost[b]; });
  double load[4] = {0, 0, 0, 0};
  int used[4] = {0, 0, 0, 0};
  for (int k = 0; k < n; ++k) {
    int best = -1;
    for (int q = 0; q < 4; ++q) {
      // the warp ids of sub-partition q are q, q+4, ... below n
      if (q + 4 * used[q] >= n) continue;
      if (best < 0 || load[q] < load[best]) best = q;
    }
    const int w = best + 4 * used[best];
    ++used[best];
    const int it = order[k];
    load[best] += cost[it];
    const int jb = item_job[it];
    lay.warp_job[w] = jb < 0 ? -1 : jl[jb];
    lay.warp_team[w] = jb < 0 ? (1 << 8) : (item_k[it] | team[jb] << 8);
    if (jb < 0) lay.producer_warp = w;
  }
  lay.nconsumers = nw;
}

// The shared-memory layout and warps of one row group running jobs jl[0..nj)
// with at most `budget` job warps, within `limit` bytes: team warps are given
// up until it fits. False when even one warp per job does not fit.
bool build_layout(const Launch& L, const int* jl, int nj, int budget, int limit, int depth, bool split, Layout& lay) {
  std::memset(&lay, 0, sizeof(lay));
  unsigned mask = 0;
  int H = 1;
  for (int j = 0; j < nj; ++j) {
    mask |= job_planes(L.jobs[jl[j]]);
    H = std::max(H, rows_halo(L.jobs[jl[j]]));
  }
  int np = 0;
  for (int p = 0; p < P_COUNT; ++p) {
    lay.plane_slot[p] = (mask & (1u << p)) ? np : -1;
    if (mask & (1u << p)) lay.slot_plane[np++] = p;
  }
  lay.nplanes = np;
  lay.Hs = std::max(1, (H + C - 1) / C);
  lay.NS = lay.Hs + depth;  // depth - 1 chunks in flight ahead of the slowest job
  lay.RS = (lay.Hs + lay.NS) * C + 1;
  int off = 0;
  lay.ring_off = off;
  off += np * 32 * lay.RS * 4;
  off = (off + 15) & ~15;
  lay.bar_off = off;
  off += 2 * lay.NS * 8;
  lay.tab_off = off;
  off += 64 * 8 + 16;
  // a partition of a split job set keeps WILLR / STOCH row-sequential: the
  // bar-parallel form doubles their instructions, which pays only when they
  // have an SM's issue slots to themselves
  lay.bp_mask = split ? (1ull << F_CCI) : bar_parallel_mask(nj);
  // team members cost shared memory (a transpose stage and lines each): give
  // up spare warps until the layout fits
  const int fixed = off;
  for (int b = std::min(budget, kMaxConsumers);; --b) {
    if (b < nj) return false;
    assign_warps(L, jl, nj, lay, b);
    off = fixed;
    for (int w = 0; w <= lay.nconsumers; ++w) {
      const int jb = lay.warp_job[w];
      off = (off + 15) & ~15;
      lay.stage_off[w] = off;
      if (jb < 0) continue;
      if (!bar_parallel(lay.bp_mask, L.jobs[jb].family)) off += out_count(L.jobs[jb].family) * 32 * (C + 1) * 4;
      off = (off + 15) & ~15;
      lay.line_off[w] = off;
      off += line_bytes(L.jobs[jb], lay.bp_mask);
    }
    lay.total = (off + 127) & ~127;
    if (lay.total <= limit) return true;
  }
}

// Jobs into P partitions by the measured per-warp cost, heaviest first: onto
// the least loaded partition that already reads the job's input planes while
// it stays within 1.2x the mean load, else onto the least loaded partition (a
// partition's ring holds only the planes its jobs read).
void partition_jobs(const Launch& L, int P, int* part) {
  const unsigned long long bp = bar_parallel_mask(L.njobs);
  int order[kMaxJobs];
  double load[kMaxParts] = {}, total = 0.0;
  unsigned planes[kMaxParts] = {};
  for (int j = 0; j < L.njobs; ++j) {
    order[j] = j;
    total += family_cost(L.jobs[j], bp);
  }
  std::stable_sort(order, order + L.njobs,
                   [&](int a, int b) { return family_cost(L.jobs[a], bp) > family_cost(L.jobs[b], bp); });
  const double cap = 1.2 * total / P;
  for (int k = 0; k < L.njobs; ++k) {
    const int j = order[k];
    const unsigned m = job_planes(L.jobs[j]);
    const double c = family_cost(L.jobs[j], bp);
    int best = -1;
    for (int q = 0; q < P; ++q)
      if (planes[q] != 0 && (planes[q] & m) == m && load[q] + c <= cap && (best < 0 || load[q] < load[best])) best = q;
    if (best < 0) {
      best = 0;
      for (int q = 1; q < P; ++q)
        if (load[q] < load[best]) best = q;
    }
    part[j] = best;
    load[best] += c;
    planes[best] |= m;
  }
}

// partition_jobs, then the partitions left empty dropped; returns their number
int partition_nonempty(const Launch& L, int P, int* part) {
  partition_jobs(L, P, part);
  int id[kMaxParts], n = 0;
  for (int q = 0; q < P; ++q) {
    id[q] = -1;
    for (int j = 0; j < L.njobs; ++j)
      if (part[j] == q) {
        id[q] = n++;
        break;
      }
  }
  for (int j = 0; j < L.njobs; ++j) part[j] = id[part[j]];
  return n;
}

// The partitions, groups per CTA and per-partition layouts of a launch
// (host only). TACUDA_B200_ROWS_PARTS / TACUDA_B200_ROWS_GROUPS /
// TACUDA_B200_ROWS_DEPTH pin P, G and the ring depth (read on every call);
// none of them changes a bit of any output. False when no layout fits.
bool plan_split(const Launch& L, int parts, int groups, int smem_optin, Split& sp) {
  if (const char* v = std::getenv("TACUDA_B200_ROWS_PARTS")) parts = std::atoi(v);
  if (const char* v = std::getenv("TACUDA_B200_ROWS_GROUPS")) groups = std::atoi(v);
  // Defaults: a job set of five or more jobs is split into four partitions,
  // each CTA running up to two row groups (13-indicator pass, 4000 x 234:
  // 210 -> 124-150 us; the same jobs over 10,000 ragged rows: 11.3-12.6 ->
  // 8.4 ms). A CTA then holds the code of a few families instead of all of
  // them (instruction-cache hit rate 59 -> 86 %), and each SM works on 64 rows
  // of a partition instead of 32 rows of everything. Five or six partitions,
  // or more groups per CTA, measured within a few percent of this (six were
  // best on the ragged rows, 7.7 ms); the autotuner tries 4-6.
  if (parts <= 0) parts = L.njobs >= 5 ? 4 : 1;
  if (groups <= 0) groups = parts > 1 ? 2 : 1;
  int P = std::max(1, std::min({parts, L.njobs, kMaxParts}));
  const long long ngroups = ((long long)L.S + 31) / 32;
  const int Gmax = (int)std::max(1ll, std::min<long long>(std::min(groups, kMaxWarps / 2), ngroups));
  int part[kMaxJobs];
  P = partition_nonempty(L, P, part);
  std::memset(&sp, 0, sizeof(sp));
  sp.P = P;
  // ring depth (chunks past the halo): 4, or less when that lets G groups fit
  int dmax = 4, dmin = 2;
  if (const char* v = std::getenv("TACUDA_B200_ROWS_DEPTH")) dmax = dmin = std::max(2, std::min(4, std::atoi(v)));
  // per partition, the largest G <= Gmax that fits: job warps within the
  // CTA's warp budget and G groups within the shared memory. (Fewer groups
  // with larger teams of chained window jobs measured slower: the 13-indicator
  // pass with the MFI/STOCH/WILLR partition at one group and teams of three
  // or four took 195-200 us against 145-155 us.)
  for (int q = 0; q < P; ++q) {
    int jl[kMaxJobs], nj = 0;
    for (int j = 0; j < L.njobs; ++j)
      if (part[j] == q) jl[nj++] = j;
    int G = Gmax;
    for (;; --G) {
      if (G < 1) return false;
      bool ok = false;
      for (int depth = dmax; depth >= (G > 1 ? dmin : dmax) && !ok; --depth)
        ok = build_layout(L, jl, nj, kMaxWarps / G - 1, smem_optin / G, depth, P > 1, sp.lay[q]);
      if (ok) break;
    }
    sp.G[q] = G;
  }
  // CTAs of the partitions with the longest chains first: a CTA lasts about
  // as long as its slowest warp (a job's measured cost over its team size), so
  // the long ones start in the first wave and the short ones fill the tail
  // (13-indicator pass at 4000 x 234: 132 -> 122 us against partition order)
  double len[kMaxParts];
  int ord[kMaxParts];
  for (int q = 0; q < P; ++q) {
    len[q] = 0.0;
    ord[q] = q;
    const Layout& y = sp.lay[q];
    for (int w = 0; w <= y.nconsumers; ++w)
      if (y.warp_job[w] >= 0)
        len[q] = std::max(len[q], (double)family_cost(L.jobs[y.warp_job[w]], y.bp_mask) / (y.warp_team[w] >> 8));
  }
  std::stable_sort(ord, ord + P, [&](int a, int b) { return len[a] > len[b]; });
  Split tmp = sp;
  for (int i = 0; i < P; ++i) {
    sp.lay[i] = tmp.lay[ord[i]];
    sp.G[i] = tmp.G[ord[i]];
  }
  sp.cta0[0] = 0;
  for (int q = 0; q < P; ++q) sp.cta0[q + 1] = sp.cta0[q] + (int)((ngroups + sp.G[q] - 1) / sp.G[q]);
  return true;
}

}  // namespace

bool supports(const Launch& L, long long max_len) {
  if (L.njobs < 1 || L.njobs > kMaxConsumers || L.st_carry) return false;
  if (max_len > (1ll << 30)) return false;
  for (int j = 0; j < L.njobs; ++j) {
    const Job& jb = L.jobs[j];
    if (jb.prec != 0 || !family_supported(jb.family)) return false;
    if (rows_halo(jb) > kMaxHalo) return false;
    if (jb.family != F_CCI && line_entries(jb) > kMaxLine) return false;
  }
  return true;
}

cudaError_t launch(Launch& L, long long max_len, cudaStream_t stream, LaunchStats* stats, int parts, int groups) {
  if (!supports(L, max_len)) return cudaErrorNotSupported;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  DevState* ds;
  {
    std::lock_guard<std::mutex> lk(g_mutex);
    if ((int)g_dev.size() <= dev) g_dev.resize(dev + 1);
    ds = &g_dev[dev];
    if (ds->sms == 0) {
      cudaDeviceGetAttribute(&ds->sms, cudaDevAttrMultiProcessorCount, dev);
      cudaDeviceGetAttribute(&ds->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    }
    if (!ds->attr) {
      e = cudaFuncSetAttribute(rows_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ds->smem_optin);
      if (e != cudaSuccess) return e;
      e = cudaFuncSetAttribute(rows_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ds->smem_optin);
      if (e != cudaSuccess) return e;
      ds->attr = true;
    }
  }
  Split sp;
  if (!plan_split(L, parts, groups, ds->smem_optin, sp)) return cudaErrorNotSupported;
  int wmax = 0, smem = 0;
  for (int q = 0; q < sp.P; ++q) {
    wmax = std::max(wmax, sp.G[q] * (sp.lay[q].nconsumers + 1));
    smem = std::max(smem, sp.G[q] * sp.lay[q].total);
  }
  const dim3 grid((unsigned)sp.cta0[sp.P]);
  const int threads = 32 * wmax;
  bool all = false;
  for (int j = 0; j < L.njobs; ++j) all |= !core_family(L.jobs[j].family);
  if (all) rows_kernel<true><<<grid, threads, smem, stream>>>(L, sp);
  else rows_kernel<false><<<grid, threads, smem, stream>>>(L, sp);
  if (stats) {
    stats->blocks = (int)grid.x;
    stats->warps_per_block = wmax;
    stats->smem_per_block = smem;
    stats->k = 0;
    stats->blocks_per_sm = 1;
  }
  return cudaGetLastError();
}

}  // namespace rows
}  // namespace tb
