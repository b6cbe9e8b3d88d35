// Conversion of the C-ABI set_param arguments (named tensors as plain pointers) into a StateDict.
#pragma once

#include "net.h"

#include <stdint.h>

namespace dcvc {

// n tensors: names[i], data[i] (host or device memory per on_device[i]), shapes[4*i .. 4*i+ndims[i]),
// dtypes[i] (DCVC_F16/BF16/F32/I32/I64).  Returns kOk or a status with the message set; `fn`
// prefixes the message.
int build_state_dict(int n, const char* const* names, const void* const* data,
                     const int64_t* shapes, const int* ndims, const int* dtypes,
                     const int* on_device, StateDict* sd, const char* fn);

}  // namespace dcvc
