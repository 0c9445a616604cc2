// Series-parallel engine: for batches with many series.
//
// A CTA owns G groups of 32 series. Per group, the input planes are staged in
// shared memory in time chunks of C bars (plus a halo of H earlier bars), row
// per series ([row][H + C + 1] floats, odd stride: thread r reading its row is
// bank-conflict free), double-buffered with cp.async so the next chunk streams
// in while the current one is evaluated. Each warp runs one job for one group:
// thread r walks series r bar by bar with the indicator state in registers, in
// exactly TA-Lib's sequential order (no scans, every bar evaluated once).
// Outputs go through a per-warp [32][C+1] transpose buffer and leave as
// coalesced 128-byte row segments.
#pragma once

#include "common.cuh"
#include "engine.h"
#include "families.cuh"

namespace tb {
namespace sp {

constexpr int C = 32;  // bars per chunk

struct Layout {
  int G, J;             // groups per CTA, jobs (warps per group)
  int H;                // halo (multiple of 32)
  int RS;               // row stride of staged planes (floats), odd
  int nplanes;
  int plane_slot[P_COUNT];
  int slot_plane[P_COUNT];
  int in_bytes;         // one buffer: G * nplanes * 32 * RS floats
  int warp_off[32];     // per-warp output transpose buffers (bytes from smem base)
  int warp_line[32];    // per-warp FP64 line (bytes) when warp_tp
  int warp_tp[32];      // 1 if the warp keeps an FP64 line (STOCH fastK, CCI/MFI typical price)
  int cdl_first;        // job index of the candle warp that fills the group table (-1: none)
  int cdl_count;        // candle warps per group
  int cdl_table_off, cdl_table_bytes;
  int total;            // dynamic smem bytes
};

// Chunk of this thread's row: bars t0 .. min(t0 + C, n) - 1.
struct Row {
  long long t0;
  long long n;
};

template <class F>
__device__ __forceinline__ void for_chunk(const Row& rw, F f) {
  const int lim = (int)min((long long)C, rw.n - rw.t0);
  for (int r = 0; r < lim; ++r) f(r, rw.t0 + r);
}

// Per-warp output transpose: out[j][lane][r]
struct Stage {
  float* buf;  // nout * 32 * (C + 1)
  __device__ __forceinline__ void put(int j, int lane, int r, float v) const { buf[(j * 32 + lane) * (C + 1) + r] = v; }
  // write rows of the group: row i of the group has length n_i (from lane i)
  __device__ __forceinline__ void flush(int j, float* out, long long base_lane, long long n_lane, long long t0,
                                        int lane) const {
    __syncwarp();
    for (int i = 0; i < 32; ++i) {
      const long long b = __shfl_sync(kFull, base_lane, i);
      const long long n = __shfl_sync(kFull, n_lane, i);
      if (b >= 0 && t0 + lane < n) out[b + t0 + lane] = buf[(j * 32 + i) * (C + 1) + lane];
    }
    __syncwarp();
  }
  __device__ __forceinline__ void flush_int(int j, int* out, long long base_lane, long long n_lane, long long t0,
                                            int lane) const {
    __syncwarp();
    const int* ib = reinterpret_cast<const int*>(buf);
    for (int i = 0; i < 32; ++i) {
      const long long b = __shfl_sync(kFull, base_lane, i);
      const long long n = __shfl_sync(kFull, n_lane, i);
      if (b >= 0 && t0 + lane < n) out[b + t0 + lane] = ib[(j * 32 + i) * (C + 1) + lane];
    }
    __syncwarp();
  }
};

__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = valid ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

}  // namespace sp
}  // namespace tb
