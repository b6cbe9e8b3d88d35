// extern "C" entry points of the low-delay (LD) codec runtime (declared in include/dcvc_b200.h).
#include "capi_state_dict.h"
#include "errors.h"
#include "ld_codec.h"

#include "../../include/dcvc_b200.h"

#include <exception>

using namespace dcvc;

namespace {

struct LdHandle {
    LdCodec codec;
    std::vector<uint8_t> bytes;
};

int fail(int status, const std::string& msg)
{
    set_last_error(msg);
    return status;
}

}  // namespace

extern "C" {

int dcvc_ld_create(void** handle)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_ld_create: null output");
    }
    if (device_error_word() == nullptr) {
        return fail(kCudaError, "dcvc_ld_create: no usable CUDA device");
    }
    try {
        *handle = new LdHandle();
    } catch (const std::exception& e) {
        return fail(kOutOfMemory, std::string("dcvc_ld_create: ") + e.what());
    }
    return kOk;
}

int dcvc_ld_destroy(void* handle)
{
    delete static_cast<LdHandle*>(handle);
    return kOk;
}

int dcvc_ld_set_param(void* handle, int n, const char* const* names, const void* const* data,
                       const int64_t* shapes, const int* ndims, const int* dtypes,
                       const int* on_device, float skip_threshold)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_ld_set_param: null handle");
    }
    StateDict sd;
    const int st = build_state_dict(n, names, data, shapes, ndims, dtypes, on_device, &sd,
                                    "dcvc_ld_set_param");
    if (st != kOk) {
        return st;
    }
    return static_cast<LdHandle*>(handle)->codec.set_param(sd, skip_threshold);
}

int dcvc_ld_add_ref_feature(void* handle, const void* frame, int height, int width,
                             int apply_adaptor, void* stream)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_ld_add_ref_feature: null handle");
    }
    return static_cast<LdHandle*>(handle)->codec.add_ref_feature(
        static_cast<const __half*>(frame), height, width, apply_adaptor != 0,
        static_cast<cudaStream_t>(stream));
}

int dcvc_ld_compress(void* handle, const void* x, int height, int width, int qp, int reset,
                      int pad_b, int pad_r, void* stream, const uint8_t** bytes, size_t* nbytes,
                      int* ec_parallel)
{
    if (handle == nullptr || bytes == nullptr || nbytes == nullptr || ec_parallel == nullptr) {
        return fail(kInvalidArgument, "dcvc_ld_compress: null argument");
    }
    LdHandle* h = static_cast<LdHandle*>(handle);
    int st = h->codec.compress(static_cast<const __half*>(x), height, width, qp, reset != 0, pad_b,
                               pad_r, static_cast<cudaStream_t>(stream), &h->bytes, ec_parallel);
    if (st != kOk) {
        return st;
    }
    *bytes = h->bytes.data();
    *nbytes = h->bytes.size();
    return kOk;
}

int dcvc_ld_decompress(void* handle, const uint8_t* bytes, size_t nbytes, int qp, int height,
                       int width, int ec_parallel, int reset, void* stream, void** frame)
{
    if (handle == nullptr || frame == nullptr) {
        return fail(kInvalidArgument, "dcvc_ld_decompress: null argument");
    }
    const __half* f = nullptr;
    int st = static_cast<LdHandle*>(handle)->codec.decompress(
        bytes, nbytes, qp, height, width, ec_parallel, reset != 0, static_cast<cudaStream_t>(stream), &f);
    if (st == kOk) {
        *frame = const_cast<__half*>(f);
    }
    return st;
}

int dcvc_ld_buffer(void* handle, const char* name, const void** ptr, int* rows, int* cols,
                    int* ld)
{
    if (handle == nullptr || name == nullptr || ptr == nullptr || rows == nullptr ||
        cols == nullptr || ld == nullptr) {
        return fail(kInvalidArgument, "dcvc_ld_buffer: null argument");
    }
    return static_cast<LdHandle*>(handle)->codec.buffer(name, ptr, rows, cols, ld);
}

int dcvc_ld_stats(void* handle, int* symbols, int* kernels, size_t* device_bytes)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_ld_stats: null handle");
    }
    const LdCodec& c = static_cast<LdHandle*>(handle)->codec;
    if (symbols) *symbols = c.last_symbol_count();
    if (kernels) *kernels = c.last_kernel_count();
    if (device_bytes) *device_bytes = c.device_bytes();
    return kOk;
}

}  // extern "C"
