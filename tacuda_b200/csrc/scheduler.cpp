// Launch planner and autotuner cache for the batch engine.
//
// The heuristic picks the engine from the batch shape: the row-parallel engine
// when the rows are at most 4x as long as there are rows, the look-back engine
// for few long rows (K = 16 bars per lane, K = 4 for uniform rows of up to
// 2^17 bars), the warp-scan engine (K = 8) otherwise.
// Candle jobs run on their own bar-parallel kernel.
// Measured plans (ct_b200_autotune) override it; they are keyed by a coarse
// shape histogram (log2 of the series count, mean and max length) plus a hash
// of the job set, kept in memory and optionally in the file named by
// TACUDA_B200_TUNE_CACHE.
#include "scheduler.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

namespace tb {

namespace {
std::mutex g_tune_mutex;
std::vector<std::pair<ShapeKey, SchedulePlan>> g_tuned;
bool g_loaded = false;

int log2_bucket(long long v) {
  int b = 0;
  while (v > 1) { v >>= 1; ++b; }
  return b;
}

void load_cache_locked() {
  if (g_loaded) return;
  g_loaded = true;
  const char* path = std::getenv("TACUDA_B200_TUNE_CACHE");
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  ShapeKey k{};
  SchedulePlan p{};
  unsigned long long jobs = 0;
  while (std::fscanf(f, "%d %d %d %llx %d %d %d %d %d %d", &k.S_bucket, &k.T_bucket, &k.Tmax_bucket, &jobs, &p.mode,
                     &p.groups, &p.k, &p.warps_per_block, &p.max_blocks, &p.parts) == 10) {
    k.jobs = jobs;
    g_tuned.emplace_back(k, p);
  }
  std::fclose(f);
}
}  // namespace

ShapeKey shape_key(const Launch& L, long long total_bars, long long max_len) {
  ShapeKey k{};
  k.S_bucket = log2_bucket(L.S);
  k.T_bucket = log2_bucket(L.S > 0 ? total_bars / L.S : 0);
  k.Tmax_bucket = log2_bucket(max_len);
  uint64_t h = 1469598103934665603ull;
  for (int j = 0; j < L.njobs; ++j) {
    const int vals[4] = {L.jobs[j].family, L.jobs[j].ip[0], L.jobs[j].ip[1], L.jobs[j].ip[2]};
    for (int v : vals) { h ^= (uint64_t)(uint32_t)v; h *= 1099511628211ull; }
  }
  k.jobs = h;
  return k;
}

SchedulePlan plan_for(const Launch& L, long long total_bars, long long max_len) {
  const ShapeKey key = shape_key(L, total_bars, max_len);
  {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    load_cache_locked();
    for (const auto& e : g_tuned)
      if (e.first == key) return e.second;
  }
  SchedulePlan p;
  // Engine by batch shape, as the reference's dispatcher picks its fused path
  // when seriesLen <= 4 * numSeries (src/api/BatchFused.cu:158-176):
  //  * row-parallel: a CTA per 32 rows, a warp per job (lanes are the rows,
  //    each walking its bars in TA-Lib's order with no scans) or a team of
  //    warps per direct-window job (lanes are the bars of one row);
  //  * look-back: few long rows, rounds of one row on different warps chained
  //    by decoupled look-back;
  //  * warp-scan otherwise: a warp per row, a round's bars split over lanes.
  // Within an engine the round width is fixed (the look-back engine's depends
  // on the row length of a uniform batch only), so a row's bits depend on the
  // engine and its own data, never on the other rows of the batch.
  p.k = 8;
  p.warps_per_block = 8;
  p.mode = 0;
  if (max_len <= 4ll * L.S) {
    p.mode = 1;
  } else if (L.S < 1024 && max_len >= 8ll * 32 * 16) {
    p.mode = 2;
    p.k = 16;
    // One row of up to 2^17 bars per series of a uniform batch is latency-
    // bound: 128-bar tiles put 4x more warps on it (1 x 100,000 bars,
    // SMA EMA RSI MACD: 123 -> 113 us).
    const bool uniform = total_bars == max_len * (long long)L.S;
    if (uniform && max_len <= (1ll << 17)) p.k = 4;
  }
  if (const char* e = std::getenv("TACUDA_B200_MODE")) {
    if (std::strcmp(e, "sp") == 0 || std::strcmp(e, "rows") == 0) p.mode = 1;
    if (std::strcmp(e, "ws") == 0) p.mode = 0;
    if (std::strcmp(e, "lb") == 0) p.mode = 2;
  }
  // TACUDA_B200_BARS_PER_LANE=4|8|16 pins the round width (read on every call):
  // results of a row are then bit-independent of its length as well as of the
  // other rows, batch size and order.
  if (const char* e = std::getenv("TACUDA_B200_BARS_PER_LANE")) {
    const int k = std::atoi(e);
    if (k == 4 || k == 8 || k == 16) p.k = k;
  }
  return p;
}

void remember_plan(const ShapeKey& key, const SchedulePlan& plan) {
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  load_cache_locked();
  for (auto& e : g_tuned)
    if (e.first == key) { e.second = plan; return; }
  g_tuned.emplace_back(key, plan);
  if (const char* path = std::getenv("TACUDA_B200_TUNE_CACHE")) {
    if (FILE* f = std::fopen(path, "a")) {
      std::fprintf(f, "%d %d %d %llx %d %d %d %d %d %d\n", key.S_bucket, key.T_bucket, key.Tmax_bucket,
                   (unsigned long long)key.jobs, plan.mode, plan.groups, plan.k, plan.warps_per_block,
                   plan.max_blocks, plan.parts);
      std::fclose(f);
    }
  }
}

}  // namespace tb
