// Host-to-device copies of large pageable buffers (scene triangles, tree
// arrays) through pinned staging buffers filled by several host threads.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace sg {

// Copies `bytes` from host memory `src` to device memory `dst` of the current
// device, ordered after earlier work and before later work on `stream` (the
// worker streams wait for an event recorded on `stream` at entry, so `dst` may
// come from a stream-ordered allocation on `stream`). When it returns, `src` has
// been read and may be changed or freed. Buffers below 32 MB and pinned ones
// go through one cudaMemcpyAsync. Larger pageable ones are split among up to
// 8 host threads; each copies its share into two 4 MB pinned buffers in turn,
// and sends each buffer to the device with cudaMemcpyAsync on its own stream.
// `stream` then waits for those copies. The staging buffers (64 MB of pinned
// memory per device at most) are made by the first large copy and kept until
// exit. Copies to one device run one at a time.
cudaError_t upload_host(void* dst, const void* src, size_t bytes, cudaStream_t stream);

}  // namespace sg
