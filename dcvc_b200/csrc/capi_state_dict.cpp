#include "capi_state_dict.h"

#include "errors.h"

#include "../../include/dcvc_b200.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>
#include <exception>
#include <string>
#include <vector>

namespace dcvc {

namespace {

size_t dtype_size(int dt)
{
    switch (dt) {
    case DCVC_F16:
    case DCVC_BF16: return 2;
    case DCVC_F32:
    case DCVC_I32: return 4;
    case DCVC_I64: return 8;
    default: return 0;
    }
}

void to_float(int dt, const void* src, size_t n, std::vector<float>* out)
{
    out->resize(n);
    float* o = out->data();
    switch (dt) {
    case DCVC_F16: {
        const __half* s = static_cast<const __half*>(src);
        for (size_t i = 0; i < n; ++i) o[i] = __half2float(s[i]);
        break;
    }
    case DCVC_BF16: {
        const __nv_bfloat16* s = static_cast<const __nv_bfloat16*>(src);
        for (size_t i = 0; i < n; ++i) o[i] = __bfloat162float(s[i]);
        break;
    }
    case DCVC_F32: std::memcpy(o, src, n * 4); break;
    case DCVC_I32: {
        const int32_t* s = static_cast<const int32_t*>(src);
        for (size_t i = 0; i < n; ++i) o[i] = static_cast<float>(s[i]);
        break;
    }
    case DCVC_I64: {
        const int64_t* s = static_cast<const int64_t*>(src);
        for (size_t i = 0; i < n; ++i) o[i] = static_cast<float>(s[i]);
        break;
    }
    default: break;
    }
}

}  // namespace

int build_state_dict(int n, const char* const* names, const void* const* data,
                     const int64_t* shapes, const int* ndims, const int* dtypes,
                     const int* on_device, StateDict* sd, const char* fn)
{
    const std::string f(fn);
    if (n <= 0 || names == nullptr || data == nullptr || shapes == nullptr || ndims == nullptr ||
        dtypes == nullptr || on_device == nullptr) {
        set_last_error(f + ": null argument");
        return kInvalidArgument;
    }
    std::vector<uint8_t> host;
    try {
        for (int i = 0; i < n; ++i) {
            if (names[i] == nullptr || ndims[i] < 0 || ndims[i] > 4 || dtype_size(dtypes[i]) == 0) {
                set_last_error(f + ": bad entry " + std::to_string(i));
                return kInvalidArgument;
            }
            HostTensor t;
            size_t numel = 1;
            for (int d = 0; d < ndims[i]; ++d) {
                if (shapes[4 * i + d] < 0) {
                    set_last_error(f + ": negative dimension in " + names[i]);
                    return kInvalidArgument;
                }
                t.shape.push_back(shapes[4 * i + d]);
                numel *= static_cast<size_t>(shapes[4 * i + d]);
            }
            const size_t bytes = numel * dtype_size(dtypes[i]);
            const void* src = data[i];
            if (numel > 0 && src == nullptr) {
                set_last_error(f + ": null data for " + names[i]);
                return kInvalidArgument;
            }
            if (on_device[i] && numel > 0) {
                host.resize(bytes);
                cudaError_t e = cudaMemcpy(host.data(), data[i], bytes, cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) {
                    return cuda_status(e, (f + ": reading a device tensor").c_str());
                }
                src = host.data();
            }
            to_float(dtypes[i], src, numel, &t.data);
            (*sd)[names[i]] = std::move(t);
        }
    } catch (const std::exception& e) {
        set_last_error(f + ": " + e.what());
        return kOutOfMemory;
    }
    return kOk;
}

}  // namespace dcvc
