// extern "C" entry points of the HT-S codec runtime (declared in include/dcvc_b200.h).
#include "capi_state_dict.h"
#include "errors.h"
#include "hts_codec.h"

#include "../../include/dcvc_b200.h"

#include <exception>

using namespace dcvc;

namespace {

struct HtsHandle {
    HtsCodec codec;
    std::vector<uint8_t> bytes;
    std::vector<std::vector<uint8_t>> batch_bytes;  // per stream of the last compress_batch
    std::vector<const uint8_t*> batch_ptrs;
    std::vector<size_t> batch_sizes;
};

int fail(int status, const std::string& msg)
{
    set_last_error(msg);
    return status;
}

}  // namespace

extern "C" {

int dcvc_hts_create(void** handle)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_create: null output");
    }
    if (device_error_word() == nullptr) {
        return fail(kCudaError, "dcvc_hts_create: no usable CUDA device");
    }
    try {
        *handle = new HtsHandle();
    } catch (const std::exception& e) {
        return fail(kOutOfMemory, std::string("dcvc_hts_create: ") + e.what());
    }
    return kOk;
}

int dcvc_hts_destroy(void* handle)
{
    delete static_cast<HtsHandle*>(handle);
    return kOk;
}

int dcvc_hts_set_param(void* handle, int n, const char* const* names, const void* const* data,
                       const int64_t* shapes, const int* ndims, const int* dtypes,
                       const int* on_device, float skip_threshold)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_set_param: null handle");
    }
    StateDict sd;
    const int st = build_state_dict(n, names, data, shapes, ndims, dtypes, on_device, &sd,
                                    "dcvc_hts_set_param");
    if (st != kOk) {
        return st;
    }
    return static_cast<HtsHandle*>(handle)->codec.set_param(sd, skip_threshold);
}

int dcvc_hts_add_ref_feature(void* handle, const void* frame, int height, int width,
                             int apply_adaptor, void* stream)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_add_ref_feature: null handle");
    }
    return static_cast<HtsHandle*>(handle)->codec.add_ref_feature(
        static_cast<const __half*>(frame), height, width, apply_adaptor != 0,
        static_cast<cudaStream_t>(stream));
}

int dcvc_hts_compress(void* handle, const void* x, int height, int width, int qp, int reset,
                      int pad_b, int pad_r, void* stream, const uint8_t** bytes, size_t* nbytes,
                      int* ec_parallel)
{
    if (handle == nullptr || bytes == nullptr || nbytes == nullptr || ec_parallel == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_compress: null argument");
    }
    HtsHandle* h = static_cast<HtsHandle*>(handle);
    int st = h->codec.compress(static_cast<const __half*>(x), height, width, qp, reset != 0, pad_b,
                               pad_r, static_cast<cudaStream_t>(stream), &h->bytes, ec_parallel);
    if (st != kOk) {
        return st;
    }
    *bytes = h->bytes.data();
    *nbytes = h->bytes.size();
    return kOk;
}

int dcvc_hts_decompress(void* handle, const uint8_t* bytes, size_t nbytes, int qp, int height,
                        int width, int ec_parallel, int reset, void* stream, void** frames)
{
    if (handle == nullptr || frames == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_decompress: null argument");
    }
    const __half* f[HtsCodec::kFrames] = {nullptr};
    int st = static_cast<HtsHandle*>(handle)->codec.decompress(
        bytes, nbytes, qp, height, width, ec_parallel, reset != 0, static_cast<cudaStream_t>(stream), f);
    if (st == kOk) {
        for (int i = 0; i < HtsCodec::kFrames; ++i) {
            frames[i] = const_cast<__half*>(f[i]);
        }
    }
    return st;
}

int dcvc_hts_buffer(void* handle, const char* name, const void** ptr, int* rows, int* cols,
                    int* ld)
{
    if (handle == nullptr || name == nullptr || ptr == nullptr || rows == nullptr ||
        cols == nullptr || ld == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_buffer: null argument");
    }
    return static_cast<HtsHandle*>(handle)->codec.buffer(name, ptr, rows, cols, ld);
}

int dcvc_hts_set_precision(void* handle, int precision)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_set_precision: null handle");
    }
    return static_cast<HtsHandle*>(handle)->codec.set_precision(precision);
}

int dcvc_hts_buffer_dtype(void* handle, const char* name, int* dtype)
{
    if (handle == nullptr || name == nullptr || dtype == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_buffer_dtype: null argument");
    }
    const void* p = nullptr;
    int rows = 0, cols = 0, ld = 0;
    return static_cast<HtsHandle*>(handle)->codec.buffer(name, &p, &rows, &cols, &ld, dtype);
}

int dcvc_hts_add_ref_features(void* handle, const void* const* frames, int n, int height,
                              int width, int apply_adaptor, void* stream)
{
    if (handle == nullptr || frames == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_add_ref_features: null argument");
    }
    return static_cast<HtsHandle*>(handle)->codec.add_ref_features(
        reinterpret_cast<const __half* const*>(frames), n, height, width, apply_adaptor != 0,
        static_cast<cudaStream_t>(stream));
}

int dcvc_hts_compress_batch(void* handle, const void* const* xs, int n, int height, int width,
                            const int* qps, int reset, int pad_b, int pad_r, void* stream,
                            const uint8_t* const** bytes, const size_t** nbytes, int* ec_parallel)
{
    if (handle == nullptr || xs == nullptr || bytes == nullptr || nbytes == nullptr ||
        ec_parallel == nullptr || n < 1) {
        return fail(kInvalidArgument, "dcvc_hts_compress_batch: null argument");
    }
    HtsHandle* h = static_cast<HtsHandle*>(handle);
    h->batch_bytes.assign(n, {});
    int st = h->codec.compress_batch(reinterpret_cast<const __half* const*>(xs), n, height, width,
                                     qps, reset != 0, pad_b, pad_r,
                                     static_cast<cudaStream_t>(stream), h->batch_bytes.data(),
                                     ec_parallel);
    if (st != kOk) {
        return st;
    }
    h->batch_ptrs.resize(n);
    h->batch_sizes.resize(n);
    for (int k = 0; k < n; ++k) {
        h->batch_ptrs[k] = h->batch_bytes[k].data();
        h->batch_sizes[k] = h->batch_bytes[k].size();
    }
    *bytes = h->batch_ptrs.data();
    *nbytes = h->batch_sizes.data();
    return kOk;
}

int dcvc_hts_decompress_batch(void* handle, const uint8_t* const* bytes, const size_t* nbytes,
                              const int* qps, const int* ec_parallel, int n, int height, int width,
                              int reset, void* stream, void** frames)
{
    if (handle == nullptr || frames == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_decompress_batch: null argument");
    }
    const __half* f[HtsCodec::kFrames] = {nullptr};
    int st = static_cast<HtsHandle*>(handle)->codec.decompress_batch(
        bytes, nbytes, qps, ec_parallel, n, height, width, reset != 0,
        static_cast<cudaStream_t>(stream), f);
    if (st == kOk) {
        for (int i = 0; i < HtsCodec::kFrames; ++i) {
            frames[i] = const_cast<__half*>(f[i]);
        }
    }
    return st;
}

int dcvc_hts_share_params(void* handle, void* source)
{
    if (handle == nullptr || source == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_share_params: null handle");
    }
    return static_cast<HtsHandle*>(handle)->codec.share_params(static_cast<HtsHandle*>(source)->codec);
}

int dcvc_hts_state_bytes(void* handle, size_t* bytes)
{
    if (handle == nullptr || bytes == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_state_bytes: null argument");
    }
    *bytes = static_cast<HtsHandle*>(handle)->codec.state_bytes();
    return kOk;
}

int dcvc_hts_export_state(void* handle, void* dst, void* stream, int* flags)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_export_state: null handle");
    }
    return static_cast<HtsHandle*>(handle)->codec.export_state(dst, static_cast<cudaStream_t>(stream),
                                                               flags);
}

int dcvc_hts_import_state(void* handle, const void* src, int flags, void* stream)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_import_state: null handle");
    }
    return static_cast<HtsHandle*>(handle)->codec.import_state(src, flags,
                                                               static_cast<cudaStream_t>(stream));
}

int dcvc_hts_recon_branches(int n)
{
    if (n != 1 && n != 2 && n != 4) {
        return fail(kInvalidArgument, "dcvc_hts_recon_branches: 1, 2 or 4");
    }
    HtsCodec::set_recon_branches(n);
    return kOk;
}

int dcvc_hts_set_timing(void* handle, int enable)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_set_timing: null handle");
    }
    static_cast<HtsHandle*>(handle)->codec.set_timing(enable != 0);
    return kOk;
}

int dcvc_hts_timing(void* handle, float* out, int cap, int* count)
{
    if (handle == nullptr || out == nullptr || cap < 0) {
        return fail(kInvalidArgument, "dcvc_hts_timing: null handle or output");
    }
    const int n = static_cast<HtsHandle*>(handle)->codec.timing(out, cap);
    if (count) *count = n;
    return kOk;
}

int dcvc_hts_stats(void* handle, int* symbols, int* kernels, size_t* device_bytes)
{
    if (handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_hts_stats: null handle");
    }
    const HtsCodec& c = static_cast<HtsHandle*>(handle)->codec;
    if (symbols) *symbols = c.last_symbol_count();
    if (kernels) *kernels = c.last_kernel_count();
    if (device_bytes) *device_bytes = c.device_bytes();
    return kOk;
}

}  // extern "C"
