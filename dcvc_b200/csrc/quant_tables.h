#pragma once

#include <stdint.h>

namespace dcvc {

// Fills lut[65536]: the Gaussian CDF-table index for every FP16 scale bit pattern.
void scale_index_table(uint8_t* lut);

}  // namespace dcvc
