// Persistent fused batch engine: one launch evaluates any set of indicator
// jobs over every series of a (uniform or ragged) batch.
//
// Work split: each warp takes series in a static snake order over the caller's
// (or the host's longest-first) series order, and walks a series in rounds of
// TILE = 32*K bars. A round stages the needed input planes (plus a halo of
// earlier bars) in shared memory with coalesced loads, then runs every job on
// them; per-job recurrence state is carried between rounds in shared memory.
// Outputs are staged per warp and written back with coalesced stores, so each
// input byte is read from HBM once per launch and each output byte written once.
//
// This file is compiled twice: normally (FP64 engines for the families up to
// CDL, candles, entry-side launch logic) and with TB_PREC_TU defined, which
// builds the kernels of the precision variants (launch_prec) and the FP64
// kernels that also hold the families appended after CDL (launch_ext), so the
// two halves compile in parallel and the common job sets keep lean kernels.
#include "engine.h"
#include "pool.h"
#include "families.cuh"
#include "families_prec.cuh"
#include "scheduler.h"
#include "jobs.h"
#ifndef TB_PREC_TU
#include "candles.cuh"
#endif

#include <algorithm>
#include <type_traits>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

namespace tb {

struct SmemLayout {
  int warps;            // warps per block
  int bytes_per_warp;
  int off_tp, off_dscr, off_planes, off_stage, off_carry;
  int nlines;
  int plane_len;        // padded floats per staged plane
  int tp_len;           // padded doubles of the typical-price plane
  int stage_len;        // padded floats per staging buffer
  int plane_slot[P_COUNT];
};

// Precision variants: P = 1 plain FP32, 2 compensated FP32, 3 FP32 bars with
// FP64 carries (families_prec.cuh); other families run in FP64.
template <int K, int P>
__device__ __forceinline__ bool run_job_prec(const Ctx<K>& c, const Job& j, Carry& cy) {
  // T: per-bar terms and state, C: running sums and carries
  using T = typename std::conditional<P == 2, F2, float>::type;
  using C = typename std::conditional<P == 2, F2, typename std::conditional<P == 3, double, float>::type>::type;
  switch (j.family) {
    case F_SMA: sum_window_p<K, T, C>(c, j, 0); return true;
    case F_SUM: sum_window_p<K, T, C>(c, j, 1); return true;
    case F_WMA: sum_window_p<K, T, C>(c, j, 2); return true;
    case F_BBANDS: moment_window_p<K, T, C>(c, j, 0); return true;
    case F_STDDEV: moment_window_p<K, T, C>(c, j, 1); return true;
    case F_VAR: moment_window_p<K, T, C>(c, j, 2); return true;
    case F_LINEARREG: linreg_p<K, T, C>(c, j); return true;
    case F_CORREL: correl_p<K, T, C>(c, j, cy); return true;
    case F_EMA: ema_p<K, T, C>(c, j, cy); return true;
    default: return false;
  }
}

// Families appended after CDL (ROC ... MIDPOINT): compiled only into the P = 4
// kernels, so the kernels of the other job sets keep their code size and
// register allocation.
template <int K>
__device__ __forceinline__ void run_job_ext(const Ctx<K>& c, const Job& j, Carry& cy) {
  switch (j.family) {
    case F_ROC: roc_round(c, j, 0); break;
    case F_ROCP: roc_round(c, j, 1); break;
    case F_ROCR: roc_round(c, j, 2); break;
    case F_ROCR100: roc_round(c, j, 3); break;
    case F_MOM: roc_round(c, j, 4); break;
    case F_RMA: ema_round(c, j, cy); break;
    case F_MEDPRICE: price_round(c, j, 0); break;
    case F_TYPPRICE: price_round(c, j, 1); break;
    case F_AVGPRICE: price_round(c, j, 2); break;
    case F_WCLPRICE: price_round(c, j, 3); break;
    case F_MIDPRICE: midprice_round(c, j); break;
    case F_MIDPOINT: midpoint_round(c, j, cy); break;
    case F_RMEAN: rolling_round(c, j, 0); break;
    case F_RMAX: rolling_round(c, j, 1); break;
    case F_RMIN: rolling_round(c, j, 2); break;
    case F_RSTD: rolling_round(c, j, 3); break;
    case F_IBS: talib_bar_round(c, j, cy, 0); break;
    case F_MARKETFI: talib_bar_round(c, j, cy, 1); break;
    case F_QSTICK: qstick_round(c, j, cy); break;
    case F_AROON: aroon_round(c, j, 0); break;
    case F_AROONOSC: aroon_round(c, j, 1); break;
    default: break;
  }
}

// P = 0: FP64 families up to CDL; P = 1..3: precision variants (a precision
// launch holds only the families that have them, which the host validates);
// P = 4: FP64, all families.
template <int K, int P>
__device__ __forceinline__ void run_job(const Ctx<K>& c, const Job& j, Carry& cy) {
  if constexpr (P >= 1 && P <= 3) {
    run_job_prec<K, P>(c, j, cy);
  } else {
  switch (j.family) {
    case F_SMA: sum_window_round(c, j, 0); break;
    case F_SUM: sum_window_round(c, j, 1); break;
    case F_WMA: sum_window_round(c, j, 2); break;
    case F_EMA: ema_round(c, j, cy); break;
    case F_DEMA: cascade_round(c, j, cy, 2); break;
    case F_TEMA: cascade_round(c, j, cy, 3); break;
    case F_T3: cascade_round(c, j, cy, 6); break;
    case F_RSI: rsi_round(c, j, cy); break;
    case F_MACD: macd_round(c, j, cy); break;
    case F_ATR: atr_round(c, j, cy, 0); break;
    case F_NATR: atr_round(c, j, cy, 1); break;
    case F_TRANGE: atr_round(c, j, cy, 2); break;
    case F_ADX: adx_round(c, j, cy, true); break;
    case F_DX: adx_round(c, j, cy, false); break;
    case F_OBV: volume_round(c, j, cy, 0); break;
    case F_AD: volume_round(c, j, cy, 1); break;
    case F_ADOSC: volume_round(c, j, cy, 2); break;
    case F_BBANDS: moment_window_round(c, j, 0); break;
    case F_STDDEV: moment_window_round(c, j, 1); break;
    case F_VAR: moment_window_round(c, j, 2); break;
    case F_LINEARREG: linreg_round(c, j); break;
    case F_MIN: minmax_round(c, j, cy, false); break;
    case F_MAX: minmax_round(c, j, cy, true); break;
    case F_WILLR: willr_round(c, j); break;
    case F_STOCH: stoch_round(c, j); break;
    case F_CCI: cci_round(c, j); break;
    case F_MFI: mfi_round(c, j); break;
    case F_CORREL: correl_round(c, j, cy); break;
    default:
      if constexpr (P == 4) run_job_ext<K>(c, j, cy);
      break;
  }
  }
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}

template <int K, int P>
__global__ void __launch_bounds__(256, (K <= 8 ? 2 : 1)) batch_kernel(const __grid_constant__ Launch L, const SmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int TILE = 32 * K;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  Ctx<K> c;
  c.lane = lane;
  c.H = L.halo;
  c.sm = smem + (size_t)warp * lay.bytes_per_warp;
  c.off_planes = lay.off_planes;
  c.plane_len = lay.plane_len;
  c.off_tp = lay.off_tp;
  c.off_dscr = lay.off_dscr;
  c.off_stage = lay.off_stage;
  c.stage_len = lay.stage_len;
  c.has_tp = L.need_tp;
  unsigned slots = 0;
  for (int p = 0; p < P_COUNT; ++p)
    if (lay.plane_slot[p] >= 0) slots |= (unsigned)lay.plane_slot[p] << (4 * p);
  c.slots = slots;
  Carry* carry = reinterpret_cast<Carry*>(c.sm + lay.off_carry);
  float* planes = reinterpret_cast<float*>(c.sm + lay.off_planes);

  const int W = gridDim.x * lay.warps;
  const int gw = blockIdx.x * lay.warps + warp;
  const int span = L.halo + TILE;
  auto stage_round_inputs = [&](int t0) {
    c.t0 = t0;
    c.L = min(TILE, c.n - t0);
    // stage the input planes with asynchronous copies, all in flight at once
    // (bars outside the row read as 0; no family reads them for an output)
    const int tlo = t0 - L.halo;
    for (int p = 0; p < P_COUNT; ++p) {
      if (!(L.plane_mask & (1u << p))) continue;
      const float* src = L.plane[p] + c.base;
      float* dst = planes + lay.plane_slot[p] * lay.plane_len;
      for (int i = lane; i < span; i += 32) {
        const int t = tlo + i;
        const bool ok = t >= c.lo && t < c.n;
        cp_async4(dst + pad(i), ok ? src + t : src, ok);
      }
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
    if (L.need_tp) {
      const float* hp = c.plane(P_HIGH);
      const float* lp = c.plane(P_LOW);
      const float* cp = c.plane(P_CLOSE);
      double* tpp = reinterpret_cast<double*>(c.sm + lay.off_tp);
      for (int i = lane; i < span; i += 32)
        tpp[i + (i >> 4)] = ((double)hp[pad(i)] + (double)lp[pad(i)] + (double)cp[pad(i)]) / 3.0;
    }
    __syncwarp();
  };
  c.lo = 0;
  if (L.lb) {
    // Look-back mode: tiles of one round taken in order from a global counter;
    // the carries between tiles come from the descriptors, not shared memory.
    c.lb = true;
    c.lbs = L.lb_nslots;
    c.err = L.err;
    const long long tps = L.lb_tile_start ? 0 : (L.T + TILE - 1) / TILE;
    const long long ntiles = L.lb_tile_start ? L.lb_tile_start[L.S] : L.lb_tiles;
    for (long long pass = 0;; ++pass) {
      // tiles in order from the counter; without recurrence carries (no
      // counter) tiles are independent and assigned statically
      unsigned long long g = (unsigned long long)(pass * W + gw);
      if (L.lb_counter) {
        if (lane == 0) g = atomicAdd(L.lb_counter, 1ull);
        g = __shfl_sync(kFull, g, 0);
      }
      if ((long long)g >= ntiles) break;
      long long s, first;
      if (L.lb_tile_start) {
        long long lo = 0, hi = L.S;  // largest s with tile_start[s] <= g
        while (lo < hi) {
          const long long mid = (lo + hi + 1) >> 1;
          if (L.lb_tile_start[mid] <= (long long)g) lo = mid;
          else hi = mid - 1;
        }
        s = lo;
        first = L.lb_tile_start[s];
        c.base = L.offsets[s];
        c.n = (int)(L.offsets[s + 1] - c.base);
      } else {
        s = (long long)g / tps;
        first = s * tps;
        c.base = s * L.T;
        c.n = (int)L.T;
      }
      c.obase = c.base;
      c.tile = (int)((long long)g - first);
      c.lbd = L.lb_desc + first * L.lb_nslots;
      stage_round_inputs(c.tile * TILE);
      for (int j = 0; j < L.njobs; ++j) {
        Carry cy;
        cy.f = -1;
#pragma unroll
        for (int v = 0; v < 10; ++v) cy.v[v] = 0.0;
        run_job<K, P>(c, L.jobs[j], cy);
        __syncwarp();
      }
    }
    return;
  }
  c.lb = false;
  for (int pass = 0;; ++pass) {
    const long long idx = (long long)pass * W + ((pass & 1) ? (W - 1 - gw) : gw);
    if (idx >= L.S) break;
    const int s = L.order ? L.order[idx] : (int)idx;
    int t_start = 0;
    Carry* keep = nullptr;  // streaming: carries kept between appends
    if (L.st_carry) {
      t_start = (int)L.st_seen;
      c.base = (long long)s * L.st_row + L.st_hist - L.st_seen;
      c.obase = (long long)s * L.T - L.st_seen;
      c.n = (int)(L.st_seen + L.T);
      c.lo = (int)(L.st_seen > L.st_hist ? L.st_seen - L.st_hist : 0);
      keep = static_cast<Carry*>(L.st_carry) + (long long)s * L.njobs;
    } else if (L.offsets) {
      c.base = L.offsets[s];
      c.n = (int)(L.offsets[s + 1] - c.base);
      c.obase = c.base;
    } else {
      c.base = (long long)s * L.T;
      c.n = (int)L.T;
      c.obase = c.base;
    }
    for (int t0 = t_start; t0 < c.n; t0 += TILE) {
      stage_round_inputs(t0);
      const bool first = t0 == t_start, last = t0 + TILE >= c.n;
      for (int j = 0; j < L.njobs; ++j) {
        // a row's first round starts from the empty carry (or the one kept by
        // the previous append), its last keeps none (or hands it to the next)
        Carry cy;
        if (first && (!keep || t_start == 0)) {
          cy.f = -1;
#pragma unroll
          for (int v = 0; v < 10; ++v) cy.v[v] = 0.0;
        } else if (first) {
          cy = keep[j];
        } else {
          cy = carry[j];
        }
        run_job<K, P>(c, L.jobs[j], cy);
        if (!last) {
          __syncwarp();
          if (lane == 0) carry[j] = cy;
          __syncwarp();
        } else if (keep) {
          __syncwarp();
          if (lane == 0) keep[j] = cy;
          __syncwarp();
        }
      }
    }
  }
}

// First look-back tile of every ragged series: tile_start[s] = sum over
// earlier series of ceil(n / tile), tile_start[S] = total. One block.
static __global__ void __launch_bounds__(1024) lb_tile_start_kernel(const long long* offsets, int S, int tile,
                                                             long long* tile_start) {
  __shared__ long long part[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  const long long per = ((long long)S + nt - 1) / nt;
  const long long lo = min((long long)S, (long long)tid * per), hi = min((long long)S, lo + per);
  long long sum = 0;
  for (long long s = lo; s < hi; ++s) sum += (offsets[s + 1] - offsets[s] + tile - 1) / tile;
  part[tid] = sum;
  __syncthreads();
  if (tid == 0) {
    long long acc = 0;
    for (int i = 0; i < nt; ++i) {
      const long long v = part[i];
      part[i] = acc;
      acc += v;
    }
    tile_start[S] = acc;
  }
  __syncthreads();
  long long acc = part[tid];
  for (long long s = lo; s < hi; ++s) {
    tile_start[s] = acc;
    acc += (offsets[s + 1] - offsets[s] + tile - 1) / tile;
  }
}

// ------------------------------------------------------------------ host side

namespace {

template <int K>
SmemLayout make_layout(const Launch& L, int warps) {
  SmemLayout lay{};
  lay.warps = warps;
  constexpr int TILE = 32 * K;
  const int span = L.halo + TILE;
  int nl = 0;
  for (int j = 0; j < L.njobs; ++j) nl = std::max(nl, job_lines(L.jobs[j]));
  lay.nlines = nl;
  lay.plane_len = (padded_len(span) + 3) & ~3;
  lay.tp_len = L.need_tp ? span + span / 16 + 2 : 0;
  lay.stage_len = (padded_len(TILE) + 3) & ~3;
  int slots = 0;
  for (int p = 0; p < P_COUNT; ++p) lay.plane_slot[p] = (L.plane_mask & (1u << p)) ? slots++ : -1;
  int off = 0;
  lay.off_tp = off;
  off += lay.tp_len * 8;
  lay.off_dscr = off;
  off += nl * Ctx<K>::LINE * 8;
  lay.off_carry = off;
  off += L.njobs * (int)sizeof(Carry);
  off = (off + 15) & ~15;
  lay.off_planes = off;
  off += slots * lay.plane_len * 4;
  lay.off_stage = off;
  off += kMaxOut * lay.stage_len * 4;
  lay.bytes_per_warp = (off + 127) & ~127;
  return lay;
}

struct OccEntry { int k, warps, smem, per_sm; };

struct DeviceInfo {
  int sms = 0;
  int smem_optin = 0;
  bool attr_set[3][5] = {};
  bool sp_attr = false;
  int cdl_per_sm = 0;
  std::vector<OccEntry> occ;
};

int k_slot(int k) { return k == 4 ? 0 : (k == 8 ? 1 : 2); }

std::mutex g_mutex;
std::vector<DeviceInfo> g_dev;

DeviceInfo& device_info(int dev) {
  std::lock_guard<std::mutex> lk(g_mutex);
  if ((int)g_dev.size() <= dev) g_dev.resize(dev + 1);
  DeviceInfo& d = g_dev[dev];
  if (d.sms == 0) {
    cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  }
  return d;
}

template <int K, int P = 0>
cudaError_t launch_k(Launch& L, const SchedulePlan& plan, cudaStream_t stream, LaunchStats* stats) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  DeviceInfo& di = device_info(dev);
  int warps = plan.warps_per_block > 0 ? plan.warps_per_block : 8;
  SmemLayout lay = make_layout<K>(L, warps);
  while (warps > 1 && lay.bytes_per_warp * warps > di.smem_optin) {
    warps /= 2;
    lay = make_layout<K>(L, warps);
  }
  const size_t smem = (size_t)lay.bytes_per_warp * warps;
  if ((int)smem > di.smem_optin) return cudaErrorInvalidConfiguration;
  int per_sm = -1;
  {
    std::lock_guard<std::mutex> lk(g_mutex);
    if (!di.attr_set[k_slot(K)][P]) {
      e = cudaFuncSetAttribute(batch_kernel<K, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, di.smem_optin);
      if (e != cudaSuccess) return e;
      di.attr_set[k_slot(K)][P] = true;
    }
    for (const OccEntry& o : di.occ)
      if (o.k == K + 100 * P && o.warps == warps && o.smem == (int)smem) per_sm = o.per_sm;
    if (per_sm < 0) {
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<K, P>, warps * 32, smem);
      if (e != cudaSuccess) return e;
      di.occ.push_back({K + 100 * P, warps, (int)smem, per_sm});
    }
  }
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  long long units = L.S;
  if (L.lb) units = L.lb_tiles;
  long long want = (units + warps - 1) / warps;
  long long cap = (long long)per_sm * di.sms;
  if (plan.max_blocks > 0) cap = std::min<long long>(cap, plan.max_blocks);
  const int blocks = (int)std::max<long long>(1, std::min(want, cap));
  L.total_warps = blocks * warps;
  batch_kernel<K, P><<<blocks, warps * 32, smem, stream>>>(L, lay);
  if (stats) {
    stats->blocks = blocks;
    stats->warps_per_block = warps;
    stats->smem_per_block = (int)smem;
    stats->k = K;
    stats->blocks_per_sm = per_sm;
  }
  return cudaGetLastError();
}

}  // namespace

#ifndef TB_PREC_TU
int max_lookback_halo(const Launch& L) {
  int h = 1;
  for (int j = 0; j < L.njobs; ++j) h = std::max(h, job_halo(L.jobs[j]));
  return h;
}

// Candle jobs run on the bar-parallel tile kernel; consecutive jobs reading
// the same planes share one launch.
// The candle pass of a job set that also has indicator jobs runs beside the
// indicator engine, on a library-owned stream of the lowest priority forked
// from and joined back into the caller's stream (events, so graph capture
// sees an ordinary fork and join). The indicator engine's CTAs are launched
// first and keep their SMs; candle blocks fill the SMs the engine leaves
// idle, e.g. while the CTAs of the longest ragged rows finish.
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  std::mutex m;
};
std::mutex g_side_mutex;
std::vector<std::unique_ptr<SideStream>> g_side;

cudaError_t side_stream(SideStream** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_side_mutex);
  if ((int)g_side.size() <= dev) g_side.resize(dev + 1);
  if (!g_side[dev]) {
    std::unique_ptr<SideStream> ss(new SideStream);
    int least = 0, greatest = 0;
    e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&ss->s, cudaStreamNonBlocking, least);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss->join, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    g_side[dev] = std::move(ss);
  }
  *out = g_side[dev].get();
  return cudaSuccess;
}

// `beside`: the pass shares the GPU with another kernel, so every row gets a
// block of its own (longest rows first) and the block scheduler hands them to
// SMs as those free up; alone, the pass runs as a persistent grid.
cudaError_t launch_candles(const Launch& L, const Job* jobs, int n, cudaStream_t stream, bool beside = false) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  DeviceInfo& di = device_info(dev);
  {
    std::lock_guard<std::mutex> lk(g_mutex);
    if (di.cdl_per_sm == 0) {
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&di.cdl_per_sm, cdl::tile_kernel, cdl::kTileBars, 0);
      if (e != cudaSuccess) return e;
      if (di.cdl_per_sm < 1) return cudaErrorInvalidConfiguration;
    }
  }
  for (int a = 0; a < n;) {
    cdl::TileArgs A;
    std::memset(&A, 0, sizeof(A));
    for (int i = 0; i < 4; ++i) A.plane[i] = L.plane[jobs[a].in[i]];
    A.offsets = L.offsets;
    A.order = L.order;
    A.T = L.T;
    A.S = L.S;
    int b = a;
    while (b < n && std::memcmp(jobs[b].in, jobs[a].in, sizeof(jobs[a].in)) == 0) A.jobs[A.njobs++] = jobs[b++];
    const long long blocks = beside ? (long long)L.S : std::min<long long>(L.S, (long long)di.cdl_per_sm * di.sms);
    cdl::tile_kernel<<<(int)std::max<long long>(1, blocks), cdl::kTileBars, 0, stream>>>(A);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    a = b;
  }
  return cudaSuccess;
}

#endif  // TB_PREC_TU

// A look-back wait that ran out in this launch also sets the per-device error
// word, so that calls on any stream can report it.
static __global__ void fold_error_kernel(const int* err, int* sticky) {
  if (*err) atomicOr(sticky, 1);
}

// Test knob (Launch::stall_test): tile 0 is never taken, so the tiles that
// wait for it run out after a short limit instead of two seconds.
static cudaError_t lookback_stall(unsigned long long* counter, int* err, cudaStream_t stream) {
  static const unsigned long long one = 1;
  static const int limit = 64;
  cudaError_t e = cudaMemcpyAsync(counter, &one, sizeof(one), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(err + 1, &limit, sizeof(limit), cudaMemcpyHostToDevice, stream);
  return e;
}

template <int K, int P>
cudaError_t launch_lookback(Launch& L, const SchedulePlan& plan, long long total_bars, cudaStream_t stream,
                            LaunchStats* stats) {
  constexpr int TILE = 32 * K;
  int nslots = 0;
  for (int j = 0; j < L.njobs; ++j) {
    L.jobs[j].lb_slot = nslots;
    nslots += lb_slots(L.jobs[j]);
  }
  if (nslots == 0 && !L.offsets) {
    // windows only: independent tiles, no scratch
    L.lb = 1;
    L.lb_counter = nullptr;
    L.err = nullptr;
    L.lb_tile_start = nullptr;
    L.lb_desc = nullptr;
    L.lb_nslots = 0;
    L.lb_tiles = (long long)L.S * ((L.T + TILE - 1) / TILE);
    return launch_k<K, P>(L, plan, stream, stats);
  }
  if (nslots == 0) nslots = 1;
  // bound on the tile count (exact for uniform rows)
  const long long ntiles = L.offsets ? total_bars / TILE + L.S : (long long)L.S * ((L.T + TILE - 1) / TILE);
  const size_t head = 256;
  const size_t ts_bytes = L.offsets ? (((size_t)(L.S + 1) * 8 + 255) & ~(size_t)255) : 0;
  const size_t desc_bytes = (size_t)ntiles * nslots * sizeof(LbDesc);
  unsigned char* scratch = nullptr;
  cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&scratch), head + ts_bytes + desc_bytes, stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(scratch, 0, head + ts_bytes + desc_bytes, stream);
  if (e == cudaSuccess) {
    L.lb = 1;
    L.lb_counter = reinterpret_cast<unsigned long long*>(scratch);
    L.err = reinterpret_cast<int*>(scratch + 8);
    L.lb_tile_start = L.offsets ? reinterpret_cast<long long*>(scratch + head) : nullptr;
    L.lb_desc = reinterpret_cast<LbDesc*>(scratch + head + ts_bytes);
    L.lb_nslots = nslots;
    L.lb_tiles = ntiles;
    if (L.offsets) {
      lb_tile_start_kernel<<<1, 1024, 0, stream>>>(L.offsets, L.S, TILE, L.lb_tile_start);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && L.stall_test) e = lookback_stall(L.lb_counter, L.err, stream);
    if (e == cudaSuccess) e = launch_k<K, P>(L, plan, stream, stats);
    if (e == cudaSuccess && L.sticky) {
      fold_error_kernel<<<1, 1, 0, stream>>>(L.err, L.sticky);
      e = cudaGetLastError();
    }
  }
  const cudaError_t ef = scratch_free(scratch, stream);
  return e != cudaSuccess ? e : ef;
}

#ifdef TB_PREC_TU
// Precision variants (rounds of 512 bars): warp-scan or look-back engine.
cudaError_t launch_prec(Launch& L, const SchedulePlan& plan, long long total_bars, cudaStream_t stream,
                        LaunchStats* stats) {
  const bool lb = plan.mode == 2;
  switch (L.jobs[0].prec) {
    case 1: return lb ? launch_lookback<16, 1>(L, plan, total_bars, stream, stats) : launch_k<16, 1>(L, plan, stream, stats);
    case 2: return lb ? launch_lookback<16, 2>(L, plan, total_bars, stream, stats) : launch_k<16, 2>(L, plan, stream, stats);
    case 3: return lb ? launch_lookback<16, 3>(L, plan, total_bars, stream, stats) : launch_k<16, 3>(L, plan, stream, stats);
    default: return cudaErrorInvalidValue;
  }
}

// Job sets with a family appended after CDL: the P = 4 kernels.
cudaError_t launch_ext_k(int k, Launch& L, const SchedulePlan& plan, cudaStream_t stream, LaunchStats* stats) {
  switch (k) {
    case 4: return launch_k<4, 4>(L, plan, stream, stats);
    case 16: return launch_k<16, 4>(L, plan, stream, stats);
    default: return launch_k<8, 4>(L, plan, stream, stats);
  }
}
cudaError_t launch_ext(Launch& L, const SchedulePlan& plan, long long total_bars, cudaStream_t stream,
                       LaunchStats* stats) {
  if (plan.mode == 2) {
    switch (plan.k) {
      case 4: return launch_lookback<4, 4>(L, plan, total_bars, stream, stats);
      case 16: return launch_lookback<16, 4>(L, plan, total_bars, stream, stats);
      default: return launch_lookback<8, 4>(L, plan, total_bars, stream, stats);
    }
  }
  return launch_ext_k(plan.k, L, plan, stream, stats);
}
#else
cudaError_t launch_prec(Launch& L, const SchedulePlan& plan, long long total_bars, cudaStream_t stream,
                        LaunchStats* stats);
cudaError_t launch_ext_k(int k, Launch& L, const SchedulePlan& plan, cudaStream_t stream, LaunchStats* stats);
cudaError_t launch_ext(Launch& L, const SchedulePlan& plan, long long total_bars, cudaStream_t stream,
                       LaunchStats* stats);

bool has_ext_family(const Launch& L) {
  for (int j = 0; j < L.njobs; ++j)
    if (L.jobs[j].family > F_CDL) return true;
  return false;
}

// Per-device error word: every engine sets bit 0 when one of its bounded
// waits runs out (the look-back engine through fold_error_kernel, the
// row-parallel engine directly). Synchronous calls read and clear it after
// their synchronisation; ct_b200_take_device_error does for any caller.
__device__ int g_sticky_err;

namespace {
std::mutex g_sticky_mutex;
std::vector<int*> g_sticky_ptr;  // per device
}  // namespace

int* sticky_word() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(g_sticky_mutex);
  if ((int)g_sticky_ptr.size() <= dev) g_sticky_ptr.resize(dev + 1, nullptr);
  if (!g_sticky_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_sticky_err) != cudaSuccess) return nullptr;
    g_sticky_ptr[dev] = static_cast<int*>(p);
  }
  return g_sticky_ptr[dev];
}

cudaError_t take_sticky_error(int* value) {
  *value = 0;
  int* p = sticky_word();
  if (!p) return cudaErrorInvalidDevice;
  int v = 0;
  cudaError_t e = cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && v != 0) e = cudaMemset(p, 0, sizeof(int));
  *value = v;
  return e;
}

// Look-back scratch of the allocation-free entry point: a file-scope device
// array (one copy per device, created when the module loads there). Its
// address is taken once per device with cudaGetSymbolAddress while that device
// is current. Every launch zeroes the part it uses (tile counter, error word,
// descriptor flags) on its stream first, so calls must not overlap in time.
__device__ __align__(256) unsigned char g_static_lb_scratch[kStaticLookbackBytes];

namespace {
std::mutex g_static_mutex;
std::vector<unsigned char*> g_static_ptr;  // per device

cudaError_t static_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_static_mutex);
  if ((int)g_static_ptr.size() <= dev) g_static_ptr.resize(dev + 1, nullptr);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_lb_scratch);
    if (e != cudaSuccess) return e;
    g_static_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_static_ptr[dev];
  return cudaSuccess;
}

template <int K>
cudaError_t launch_lookback_static_k(Launch& L, const SchedulePlan& plan, cudaStream_t stream, size_t* need) {
  constexpr int TILE = 32 * K;
  int nslots = 0;
  for (int j = 0; j < L.njobs; ++j) {
    L.jobs[j].lb_slot = nslots;
    nslots += lb_slots(L.jobs[j]);
  }
  if (nslots == 0) nslots = 1;
  const long long ntiles = (long long)L.S * ((L.T + TILE - 1) / TILE);
  const size_t head = 256;
  const size_t bytes = head + (size_t)ntiles * nslots * sizeof(LbDesc);
  *need = bytes;
  if (bytes > kStaticLookbackBytes) return cudaErrorInvalidValue;
  unsigned char* scratch = nullptr;
  cudaError_t e = static_scratch(&scratch);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(scratch, 0, bytes, stream);
  if (e != cudaSuccess) return e;
  L.lb = 1;
  L.lb_counter = reinterpret_cast<unsigned long long*>(scratch);
  L.err = reinterpret_cast<int*>(scratch + 8);
  L.lb_tile_start = nullptr;
  L.lb_desc = reinterpret_cast<LbDesc*>(scratch + head);
  L.lb_nslots = nslots;
  L.lb_tiles = ntiles;
  if (L.stall_test) e = lookback_stall(L.lb_counter, L.err, stream);
  if (e != cudaSuccess) return e;
  e = has_ext_family(L) ? launch_ext_k(K, L, plan, stream, nullptr) : launch_k<K>(L, plan, stream, nullptr);
  if (e == cudaSuccess && L.sticky) {
    fold_error_kernel<<<1, 1, 0, stream>>>(L.err, L.sticky);
    e = cudaGetLastError();
  }
  return e;
}
}  // namespace

cudaError_t launch_lookback_static(Launch& L, const SchedulePlan& plan, cudaStream_t stream, size_t* need) {
  if (!L.sticky) L.sticky = sticky_word();
  unsigned mask = 0;
  int need_tp = 0;
  for (int j = 0; j < L.njobs; ++j) {
    mask |= job_planes(L.jobs[j]);
    if (L.jobs[j].family == F_CCI || L.jobs[j].family == F_MFI) need_tp = 1;
  }
  if (need_tp) mask |= (1u << P_HIGH) | (1u << P_LOW) | (1u << P_CLOSE);
  L.plane_mask = mask;
  L.need_tp = need_tp;
  L.halo = ((max_lookback_halo(L) + 31) / 32) * 32;
  switch (plan.k) {
    case 4: return launch_lookback_static_k<4>(L, plan, stream, need);
    case 16: return launch_lookback_static_k<16>(L, plan, stream, need);
    default: return launch_lookback_static_k<8>(L, plan, stream, need);
  }
}

cudaError_t launch_batch(Launch& L, const SchedulePlan& plan, long long total_bars, cudaStream_t stream,
                         LaunchStats* stats) {
  if (!L.sticky) L.sticky = sticky_word();
  unsigned mask = 0;
  int need_tp = 0;
  for (int j = 0; j < L.njobs; ++j) {
    mask |= job_planes(L.jobs[j]);
    if (L.jobs[j].family == F_CCI || L.jobs[j].family == F_MFI) need_tp = 1;
  }
  if (need_tp) mask |= (1u << P_HIGH) | (1u << P_LOW) | (1u << P_CLOSE);
  L.plane_mask = mask;
  L.need_tp = need_tp;
  const int h = max_lookback_halo(L);
  L.halo = ((h + 31) / 32) * 32;
  // candle jobs go to the bar-parallel tile kernel, the rest to the engine
  int ncdl = 0;
  Job cdl_jobs[kMaxJobs];
  for (int j = 0, k = 0; j < L.njobs; ++j) {
    if (L.jobs[j].family == F_CDL) cdl_jobs[ncdl++] = L.jobs[j];
    else L.jobs[k++] = L.jobs[j];
  }
  L.njobs -= ncdl;
  if (ncdl > 0) {
    if (L.njobs == 0) return launch_candles(L, cdl_jobs, ncdl, stream);
    SideStream* ss = nullptr;
    cudaError_t e = side_stream(&ss);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(ss->m);
    e = cudaEventRecord(ss->fork, stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ss->s, ss->fork, 0);
    if (e != cudaSuccess) return e;
    e = launch_batch(L, plan, total_bars, stream, stats);
    const cudaError_t ec = launch_candles(L, cdl_jobs, ncdl, ss->s, true);
    // the join is enqueued whatever happened, so the side stream never
    // outlives the caller's stream (or an open capture) unjoined
    cudaError_t ej = cudaEventRecord(ss->join, ss->s);
    if (ej == cudaSuccess) ej = cudaStreamWaitEvent(stream, ss->join, 0);
    return e != cudaSuccess ? e : (ec != cudaSuccess ? ec : ej);
  }
  L.lb = 0;
  // row-parallel engine; job sets it does not take (or whose layout does not
  // fit its shared memory) run on the warp-scan engine
  if (plan.mode == 1 && rows::supports(L, L.max_len)) {
    const cudaError_t e = rows::launch(L, L.max_len, stream, stats, plan.parts, plan.groups);
    if (e != cudaErrorNotSupported) return e;
  }
  if (L.njobs > 0 && L.jobs[0].prec != 0) return launch_prec(L, plan, total_bars, stream, stats);
  if (has_ext_family(L)) return launch_ext(L, plan, total_bars, stream, stats);
  if (plan.mode == 2) {
    switch (plan.k) {
      case 4: return launch_lookback<4, 0>(L, plan, total_bars, stream, stats);
      case 16: return launch_lookback<16, 0>(L, plan, total_bars, stream, stats);
      default: return launch_lookback<8, 0>(L, plan, total_bars, stream, stats);
    }
  }
  switch (plan.k) {
    case 4: return launch_k<4>(L, plan, stream, stats);
    case 16: return launch_k<16>(L, plan, stream, stats);
    default: return launch_k<8>(L, plan, stream, stats);
  }
}

#endif  // TB_PREC_TU

}  // namespace tb
