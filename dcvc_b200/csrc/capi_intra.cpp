// extern "C" entry points of the intra (DMCI) codec runtime (declared in include/dcvc_b200.h).
#include "capi_state_dict.h"
#include "errors.h"
#include "intra_codec.h"

#include "../../include/dcvc_b200.h"

#include <exception>

using namespace dcvc;

namespace {

struct IntraHandle {
    IntraCodec codec;
    std::vector<uint8_t> bytes;
};

int fail(int status, const std::string& msg)
{
    set_last_error(msg);
    return status;
}

}  // namespace

extern "C" {

int dcvc_intra_create(void** handle)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_intra_create: null output");
    }
    if (device_error_word() == nullptr) {
        return fail(kCudaError, "dcvc_intra_create: no usable CUDA device");
    }
    try {
        *handle = new IntraHandle();
    } catch (const std::exception& e) {
        return fail(kOutOfMemory, std::string("dcvc_intra_create: ") + e.what());
    }
    return kOk;
}

int dcvc_intra_destroy(void* handle)
{
    delete static_cast<IntraHandle*>(handle);
    return kOk;
}

int dcvc_intra_set_param(void* handle, int n, const char* const* names, const void* const* data,
                         const int64_t* shapes, const int* ndims, const int* dtypes,
                         const int* on_device, float skip_threshold)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_intra_set_param: null handle");
    }
    StateDict sd;
    const int st = build_state_dict(n, names, data, shapes, ndims, dtypes, on_device, &sd,
                                    "dcvc_intra_set_param");
    if (st != kOk) {
        return st;
    }
    return static_cast<IntraHandle*>(handle)->codec.set_param(sd, skip_threshold);
}

int dcvc_intra_compress(void* handle, const void* x, int height, int width, int qp, int pad_b,
                        int pad_r, void* stream, const uint8_t** bytes, size_t* nbytes,
                        int* ec_parallel, void** x_hat)
{
    if (handle == nullptr || bytes == nullptr || nbytes == nullptr || ec_parallel == nullptr ||
        x_hat == nullptr) {
        return fail(kInvalidArgument, "dcvc_intra_compress: null argument");
    }
    IntraHandle* h = static_cast<IntraHandle*>(handle);
    const __half* xh = nullptr;
    int st = h->codec.compress(static_cast<const __half*>(x), height, width, qp, pad_b, pad_r,
                               static_cast<cudaStream_t>(stream), &h->bytes, ec_parallel, &xh);
    if (st != kOk) {
        return st;
    }
    *bytes = h->bytes.data();
    *nbytes = h->bytes.size();
    *x_hat = const_cast<__half*>(xh);
    return kOk;
}

int dcvc_intra_decompress(void* handle, const uint8_t* bytes, size_t nbytes, int qp, int height,
                          int width, int ec_parallel, void* stream, void** x_hat)
{
    if (handle == nullptr || x_hat == nullptr) {
        return fail(kInvalidArgument, "dcvc_intra_decompress: null argument");
    }
    const __half* xh = nullptr;
    int st = static_cast<IntraHandle*>(handle)->codec.decompress(
        bytes, nbytes, qp, height, width, ec_parallel, static_cast<cudaStream_t>(stream), &xh);
    if (st == kOk) {
        *x_hat = const_cast<__half*>(xh);
    }
    return st;
}

int dcvc_intra_buffer(void* handle, const char* name, const void** ptr, int* rows, int* cols,
                      int* ld)
{
    if (handle == nullptr || name == nullptr || ptr == nullptr || rows == nullptr ||
        cols == nullptr || ld == nullptr) {
        return fail(kInvalidArgument, "dcvc_intra_buffer: null argument");
    }
    return static_cast<IntraHandle*>(handle)->codec.buffer(name, ptr, rows, cols, ld);
}

int dcvc_intra_stats(void* handle, int* symbols, int* kernels, size_t* device_bytes)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_intra_stats: null handle");
    }
    const IntraCodec& c = static_cast<IntraHandle*>(handle)->codec;
    if (symbols) *symbols = c.last_symbol_count();
    if (kernels) *kernels = c.last_kernel_count();
    if (device_bytes) *device_bytes = c.device_bytes();
    return kOk;
}

}  // extern "C"
