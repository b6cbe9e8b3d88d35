#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dcvc {

// Fills lut[65536] on the host: the Gaussian CDF-table index for every FP16 scale bit pattern,
// with the logarithm evaluated in double precision (the CPU restatement).
void scale_index_table(uint8_t* lut);

// Fills the device table lut[65536] with the index the reference's FP16 scale_to_index computes
// on the GPU (stream.cu:77-87 in its fast-math build): the table the codecs use.
cudaError_t scale_index_table_device(uint8_t* lut, cudaStream_t s);

}  // namespace dcvc
