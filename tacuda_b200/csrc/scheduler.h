// Launch planning for the batch engine: bars per lane (K), warps per block and
// grid size, chosen per batch shape and job set. Plans come from a built-in
// heuristic or from the measured autotuner cache (see scheduler.cpp).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "engine.h"

namespace tb {

struct SchedulePlan {
  int mode = 0;            // 0: warp per series (time-parallel lanes), 1: thread per series,
                           // 2: warp per tile with decoupled look-back between tiles
  int groups = 0;          // row-parallel: 32-row groups per CTA (0 = auto)
  int parts = 0;           // row-parallel: partitions of the job set, one per grid row (0 = auto)
  int k = 8;               // bars per lane; a round covers 32*k bars
  int warps_per_block = 8;
  int max_blocks = 0;      // 0 = as many as fit
};

struct LaunchStats {
  int blocks = 0, warps_per_block = 0, smem_per_block = 0, k = 0, blocks_per_sm = 0;
};

// Shape summary used as the autotuner key.
struct ShapeKey {
  int S_bucket;     // log2 of series count
  int T_bucket;     // log2 of mean length
  int Tmax_bucket;  // log2 of max length
  uint64_t jobs;    // hash of the job families and periods
  bool operator==(const ShapeKey& o) const {
    return S_bucket == o.S_bucket && T_bucket == o.T_bucket && Tmax_bucket == o.Tmax_bucket && jobs == o.jobs;
  }
};

ShapeKey shape_key(const Launch& L, long long total_bars, long long max_len);
SchedulePlan plan_for(const Launch& L, long long total_bars, long long max_len);
void remember_plan(const ShapeKey& key, const SchedulePlan& plan);

cudaError_t launch_batch(Launch& L, const SchedulePlan& plan, long long total_bars, cudaStream_t stream,
                         LaunchStats* stats);
int max_lookback_halo(const Launch& L);

// The per-device error word (bit 0: a bounded wait of an engine ran out) and
// its read-and-clear; the read synchronises with the legacy default stream.
int* sticky_word();
cudaError_t take_sticky_error(int* value);

namespace rows {
// Row-parallel engine (rows.cu): whether it takes this job set and batch, and
// its launch. Returns cudaErrorNotSupported for job sets it does not take.
bool supports(const Launch& L, long long max_len);
cudaError_t launch(Launch& L, long long max_len, cudaStream_t stream, LaunchStats* stats, int parts = 0,
                   int groups = 0);
}  // namespace rows

// Look-back launch with its scratch in a static device array of
// kStaticLookbackBytes per device (allocation-free). Uniform rows, no candle
// jobs. Returns cudaErrorInvalidValue when the scratch it needs (*need bytes)
// exceeds the array. Calls must not overlap in time.
constexpr size_t kStaticLookbackBytes = 8u << 20;
cudaError_t launch_lookback_static(Launch& L, const SchedulePlan& plan, cudaStream_t stream, size_t* need);

}  // namespace tb
