// Stream-ordered scratch for the library's own temporary buffers.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace tb {

// Allocate / free `bytes` of device scratch ordered on `stream`. Outside
// stream capture the memory comes from a library-owned pool on the current
// device whose release threshold keeps freed memory mapped, so repeated calls
// reuse it instead of mapping fresh pages every time; under capture it is an
// ordinary stream-ordered allocation (a graph memory node).
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t stream);
cudaError_t scratch_free(void* p, cudaStream_t stream);

}  // namespace tb
