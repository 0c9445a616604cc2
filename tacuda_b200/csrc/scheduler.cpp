// Launch planner and autotuner cache for the batch engine.
//
// The heuristic picks the round width from the batch shape: rows of at most
// 128 bars use K = 4 bars per lane, others K = 8 (two blocks per SM), and the
// look-back engine for few long rows K = 16 (K = 4 when the batch holds fewer
// than 1024 tiles of 512 bars).
// Candle jobs run on their own bar-parallel kernel unless the series-parallel
// engine is forced (it evaluates them in the same pass).
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
  while (std::fscanf(f, "%d %d %d %llx %d %d %d %d %d", &k.S_bucket, &k.T_bucket, &k.Tmax_bucket, &jobs, &p.mode,
                     &p.groups, &p.k, &p.warps_per_block, &p.max_blocks) == 9) {
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
  const long long mean = L.S > 0 ? total_bars / L.S : 0;
  // K = 8 runs two blocks per SM and beat K = 16 on long ragged rows too
  p.k = max_len <= 128 ? 4 : 8;
  (void)mean;
  p.warps_per_block = 8;
  // A warp per series splitting each round across its lanes; when there are
  // too few series to fill the GPU and they span many rounds, rounds of one
  // series go to different warps chained by decoupled look-back (512-bar
  // rounds: fewer tiles and hops).
  p.mode = 0;
  if (L.S < 1024 && max_len >= 8ll * 32 * 16) {
    p.mode = 2;
    p.k = 16;
    // Fewer than 1024 tiles of 512 bars leave the GPU nearly idle and the
    // call latency-bound: 128-bar tiles put 4x more warps on it
    // (1 x 100,000 bars, SMA EMA RSI MACD: 123 -> 113 us).
    if (total_bars < 1024ll * 512) p.k = 4;
  }
  if (const char* e = std::getenv("TACUDA_B200_MODE")) {
    if (std::strcmp(e, "sp") == 0) p.mode = 1;
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
      std::fprintf(f, "%d %d %d %llx %d %d %d %d %d\n", key.S_bucket, key.T_bucket, key.Tmax_bucket,
                   (unsigned long long)key.jobs, plan.mode, plan.groups, plan.k, plan.warps_per_block,
                   plan.max_blocks);
      std::fclose(f);
    }
  }
}

}  // namespace tb
