#include "pool.h"

#include <cstdint>
#include <mutex>
#include <vector>

namespace tb {

namespace {
std::mutex g_pool_mutex;
std::vector<cudaMemPool_t> g_pools;  // per device, created on first use

cudaError_t device_pool(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_pool_mutex);
  if ((int)g_pools.size() <= dev) g_pools.resize(dev + 1, nullptr);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return cudaSuccess;
}

bool capturing(cudaStream_t stream) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &st) != cudaSuccess) return false;
  return st != cudaStreamCaptureStatusNone;
}
}  // namespace

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t stream) {
  if (capturing(stream)) return cudaMallocAsync(p, bytes, stream);
  cudaMemPool_t pool = nullptr;
  const cudaError_t e = device_pool(&pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, bytes, pool, stream);
}

cudaError_t scratch_free(void* p, cudaStream_t stream) { return cudaFreeAsync(p, stream); }

}  // namespace tb
