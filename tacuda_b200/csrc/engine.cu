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
#include "engine.h"
#include "families.cuh"
#include "candles.cuh"
#include "scheduler.h"

#include <algorithm>
#include <cstring>
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

template <int K>
__device__ __forceinline__ void run_job(const Ctx<K>& c, const Job& j, Carry& cy) {
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
    case F_CDL: cdl_round(c, j); break;
    default: break;
  }
}

template <int K>
__global__ void __launch_bounds__(256) batch_kernel(const __grid_constant__ Launch L, const SmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int TILE = 32 * K;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* mine = smem + (size_t)warp * lay.bytes_per_warp;

  Ctx<K> c;
  c.lane = lane;
  c.H = L.halo;
  c.tp = L.need_tp ? reinterpret_cast<double*>(mine + lay.off_tp) : nullptr;
  c.dscr = reinterpret_cast<double*>(mine + lay.off_dscr);
  for (int p = 0; p < P_COUNT; ++p)
    c.sp[p] = lay.plane_slot[p] >= 0
                  ? reinterpret_cast<float*>(mine + lay.off_planes) + lay.plane_slot[p] * lay.plane_len
                  : nullptr;
  for (int j = 0; j < kMaxOut; ++j)
    c.stage[j] = reinterpret_cast<float*>(mine + lay.off_stage) + j * lay.stage_len;
  c.istage = reinterpret_cast<int*>(c.stage[0]);
  Carry* carry = reinterpret_cast<Carry*>(mine + lay.off_carry);

  const int W = gridDim.x * lay.warps;
  const int gw = blockIdx.x * lay.warps + warp;
  const int span = L.halo + TILE;
  for (int pass = 0;; ++pass) {
    const long long idx = (long long)pass * W + ((pass & 1) ? (W - 1 - gw) : gw);
    if (idx >= L.S) break;
    const int s = L.order ? L.order[idx] : (int)idx;
    if (L.offsets) {
      c.base = L.offsets[s];
      c.n = L.offsets[s + 1] - c.base;
    } else {
      c.base = (long long)s * L.T;
      c.n = L.T;
    }
    for (int j = 0; j < L.njobs; ++j) {
      if (lane == 0) {
        carry[j].f = -1;
        for (int v = 0; v < 10; ++v) carry[j].v[v] = 0.0;
      }
    }
    __syncwarp();
    for (long long t0 = 0; t0 < c.n; t0 += TILE) {
      c.t0 = t0;
      c.L = (int)min((long long)TILE, c.n - t0);
      // stage the input planes (NaN outside the row)
      const long long tlo = t0 - L.halo;
      for (int p = 0; p < P_COUNT; ++p) {
        if (!(L.plane_mask & (1u << p))) continue;
        const float* __restrict__ src = L.plane[p] + c.base;
        float* dst = c.sp[p];
        for (int i = lane; i < span; i += 32) {
          const long long t = tlo + i;
          dst[pad(i)] = (t >= 0 && t < c.n) ? __ldg(src + t) : qnan();
        }
      }
      __syncwarp();
      if (L.need_tp) {
        const float* hp = c.sp[P_HIGH];
        const float* lp = c.sp[P_LOW];
        const float* cp = c.sp[P_CLOSE];
        for (int i = lane; i < span; i += 32)
          c.tp[i + (i >> 4)] = ((double)hp[pad(i)] + (double)lp[pad(i)] + (double)cp[pad(i)]) / 3.0;
      }
      __syncwarp();
      for (int j = 0; j < L.njobs; ++j) {
        Carry cy = carry[j];
        run_job<K>(c, L.jobs[j], cy);
        __syncwarp();
        if (lane == 0) carry[j] = cy;
        __syncwarp();
      }
    }
  }
}

// ------------------------------------------------------------------ host side

namespace {

int job_halo(const Job& j) {
  switch (j.family) {
    case F_SMA: case F_SUM: case F_WMA: case F_BBANDS: case F_STDDEV: case F_VAR:
    case F_LINEARREG: case F_MIN: case F_MAX: case F_WILLR: case F_CCI: case F_CORREL:
      return j.ip[0] - 1;
    case F_MFI: return j.ip[0];
    case F_STOCH: return j.ip[0] - 1 + 2 * (j.ip[1] - 1);
    case F_CDL: return kCdlHalo;
    default: return 1;  // previous bar
  }
}

unsigned job_planes(const Job& j) {
  unsigned m = 0;
  int n = 0;
  switch (j.family) {
    case F_SMA: case F_EMA: case F_WMA: case F_RSI: case F_MACD: case F_BBANDS: case F_SUM:
    case F_MIN: case F_MAX: case F_STDDEV: case F_VAR: case F_LINEARREG: case F_DEMA:
    case F_TEMA: case F_T3:
      n = 1; break;
    case F_OBV: case F_CORREL: n = 2; break;
    case F_ATR: case F_NATR: case F_TRANGE: case F_ADX: case F_DX: case F_STOCH: case F_WILLR:
      n = 3; break;
    case F_CCI: n = 3; break;
    case F_AD: case F_ADOSC: case F_MFI: case F_CDL: n = 4; break;
    default: n = 0;
  }
  for (int i = 0; i < n; ++i) m |= 1u << j.in[i];
  return m;
}

int job_lines(const Job& j) {
  switch (j.family) {
    case F_MACD: case F_ADX: case F_DX: case F_STOCH: return 1;
    case F_ADOSC: return 2;
    case F_DEMA: return 2;
    case F_TEMA: return 3;
    case F_T3: return 4;
    default: return 0;
  }
}

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
  bool attr_set[3] = {false, false, false};
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

template <int K>
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
    if (!di.attr_set[k_slot(K)]) {
      e = cudaFuncSetAttribute(batch_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, di.smem_optin);
      if (e != cudaSuccess) return e;
      di.attr_set[k_slot(K)] = true;
    }
    for (const OccEntry& o : di.occ)
      if (o.k == K && o.warps == warps && o.smem == (int)smem) per_sm = o.per_sm;
    if (per_sm < 0) {
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<K>, warps * 32, smem);
      if (e != cudaSuccess) return e;
      di.occ.push_back({K, warps, (int)smem, per_sm});
    }
  }
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  long long want = (L.S + warps - 1) / warps;
  long long cap = (long long)per_sm * di.sms;
  if (plan.max_blocks > 0) cap = std::min<long long>(cap, plan.max_blocks);
  const int blocks = (int)std::max<long long>(1, std::min(want, cap));
  L.total_warps = blocks * warps;
  batch_kernel<K><<<blocks, warps * 32, smem, stream>>>(L, lay);
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

int max_lookback_halo(const Launch& L) {
  int h = 1;
  for (int j = 0; j < L.njobs; ++j) h = std::max(h, job_halo(L.jobs[j]));
  return h;
}

cudaError_t launch_batch(Launch& L, const SchedulePlan& plan, cudaStream_t stream, LaunchStats* stats) {
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
  switch (plan.k) {
    case 4: return launch_k<4>(L, plan, stream, stats);
    case 16: return launch_k<16>(L, plan, stream, stats);
    default: return launch_k<8>(L, plan, stream, stats);
  }
}

}  // namespace tb
