// Host-side helpers shared by the kernel launchers and the runtime.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dcvc {

// Number of SMs of the current device (cached per device).
int num_sms();

// Encodes a 2D tiled TMA descriptor over a row-major matrix of 16-bit elements: `inner`
// elements per row (contiguous), `outer` rows, `row_bytes` pitch.  The box is box_inner x
// box_outer elements; `swizzle_bytes` is 128, 64, 32 or 0 (no swizzle).  Out-of-range
// rows/columns read as zero and are not written.  Returns false if the driver rejects the
// arguments.
bool make_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base, uint64_t inner,
                  uint64_t outer, uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer,
                  int swizzle_bytes = 128);

}  // namespace dcvc
