// extern "C" entry points of the host rANS coder (declared in include/dcvc_b200.h).
#include "errors.h"
#include "rans_coder.h"
#include "rans_gpu.cuh"

#include "../../include/dcvc_b200.h"

#include <cstring>
#include <exception>
#include <memory>

using namespace dcvc;

namespace {

struct RansHandle {
    RansTables tables;
    RansEncoderSession enc;
    RansDecoderSession dec;
    std::vector<uint8_t> encoded;
    bool enc_open = false;
};

RansHandle* as_handle(void* h) { return static_cast<RansHandle*>(h); }

struct GpuRansHandle {
    RansGpuTables tables;
    void* storage = nullptr;
};

int fail(int status, const std::string& msg)
{
    set_last_error(msg);
    return status;
}

}  // namespace

extern "C" {

int dcvc_pmf_to_quantized_cdf(const float* pmf, int n, uint32_t* cdf_out)
{
    if (pmf == nullptr || cdf_out == nullptr || n < 1) {
        return fail(kInvalidArgument, "dcvc_pmf_to_quantized_cdf: bad arguments");
    }
    std::vector<uint32_t> cdf = pmf_to_quantized_cdf(pmf, n);
    if (cdf.empty()) {
        return fail(kInvalidArgument, "dcvc_pmf_to_quantized_cdf: pmf has no mass to quantise");
    }
    std::memcpy(cdf_out, cdf.data(), cdf.size() * sizeof(uint32_t));
    return kOk;
}

int dcvc_rans_create(void** out)
{
    if (out == nullptr) {
        return fail(kInvalidArgument, "dcvc_rans_create: null output");
    }
    try {
        *out = new RansHandle();
    } catch (const std::exception& e) {
        return fail(kOutOfMemory, std::string("dcvc_rans_create: ") + e.what());
    }
    return kOk;
}

int dcvc_rans_destroy(void* h)
{
    delete as_handle(h);
    return kOk;
}

int dcvc_rans_set_cdf(void* h, int index, const int32_t* cdf, const int32_t* lengths, int count,
                      int stride)
{
    if (h == nullptr || cdf == nullptr || lengths == nullptr) {
        return fail(kInvalidArgument, "dcvc_rans_set_cdf: null argument");
    }
    std::string err;
    if (!as_handle(h)->tables.set(index, cdf, lengths, count, stride, &err)) {
        return fail(kInvalidArgument, "dcvc_rans_set_cdf: " + err);
    }
    return kOk;
}

int dcvc_rans_encode_begin(void* h, int ec_parallel)
{
    if (h == nullptr || ec_parallel < 1 || ec_parallel > kMaxEcParallel) {
        return fail(kInvalidArgument, "dcvc_rans_encode_begin: ec_parallel must be in [1, 8]");
    }
    as_handle(h)->enc.reset(ec_parallel);
    as_handle(h)->enc_open = true;
    return kOk;
}

int dcvc_rans_encode_y(void* h, const int16_t* sym, int n)
{
    if (h == nullptr || !as_handle(h)->enc_open || n < 0 || (n > 0 && sym == nullptr)) {
        return fail(kInvalidArgument, "dcvc_rans_encode_y: bad arguments or no open payload");
    }
    as_handle(h)->enc.add_y(sym, n, true);
    return kOk;
}

int dcvc_rans_encode_z(void* h, const int8_t* sym, int n, int cdf_offset, int ch)
{
    if (h == nullptr || !as_handle(h)->enc_open || n < 0 || (n > 0 && sym == nullptr) || ch < 1) {
        return fail(kInvalidArgument, "dcvc_rans_encode_z: bad arguments or no open payload");
    }
    as_handle(h)->enc.add_z(sym, n, cdf_offset, ch, true);
    return kOk;
}

int dcvc_rans_encode_finish(void* h, const uint8_t** data, size_t* size)
{
    if (h == nullptr || data == nullptr || size == nullptr || !as_handle(h)->enc_open) {
        return fail(kInvalidArgument, "dcvc_rans_encode_finish: bad arguments or no open payload");
    }
    RansHandle* r = as_handle(h);
    std::string err;
    r->enc_open = false;
    if (!r->enc.finish(r->tables, &r->encoded, &err)) {
        return fail(r->enc.fault() ? kInternal : kInvalidArgument, "dcvc_rans_encode_finish: " + err);
    }
    *data = r->encoded.data();
    *size = r->encoded.size();
    return kOk;
}

int dcvc_rans_decode_begin(void* h, const uint8_t* data, size_t size, int ec_parallel)
{
    if (h == nullptr || size > 0x7fffffff) {
        return fail(kInvalidArgument, "dcvc_rans_decode_begin: bad arguments");
    }
    std::string err;
    if (!as_handle(h)->dec.begin(data, static_cast<int>(size), ec_parallel, &err)) {
        return fail(as_handle(h)->dec.fault() ? kInternal : kCorruptStream,
                    "dcvc_rans_decode_begin: " + err);
    }
    return kOk;
}

int dcvc_rans_decode_z(void* h, int n, int cdf_offset, int ch, int8_t* out)
{
    if (h == nullptr || (n > 0 && out == nullptr)) {
        return fail(kInvalidArgument, "dcvc_rans_decode_z: bad arguments");
    }
    std::string err;
    RansHandle* r = as_handle(h);
    if (!r->dec.decode_z(r->tables, n, cdf_offset, ch, out, &err)) {
        return fail(r->dec.fault() ? kInternal : kCorruptStream, "dcvc_rans_decode_z: " + err);
    }
    return kOk;
}

int dcvc_rans_decode_y(void* h, const uint8_t* idx, int n, int8_t* out)
{
    if (h == nullptr || (n > 0 && (out == nullptr || idx == nullptr))) {
        return fail(kInvalidArgument, "dcvc_rans_decode_y: bad arguments");
    }
    std::string err;
    RansHandle* r = as_handle(h);
    if (!r->dec.decode_y(r->tables, idx, n, out, &err)) {
        return fail(r->dec.fault() ? kInternal : kCorruptStream, "dcvc_rans_decode_y: " + err);
    }
    return kOk;
}

int dcvc_rans_inject_task_fault(int sub_stream)
{
    rans_inject_task_fault(sub_stream);
    return kOk;
}

int dcvc_ec_parallel_for(int symbol_count) { return ec_parallel_for(symbol_count); }

int dcvc_rans_gpu_create(void* rans_handle, void** gpu_handle)
{
    if (rans_handle == nullptr || gpu_handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_rans_gpu_create: null argument");
    }
    RansHandle* r = as_handle(rans_handle);
    if (!r->tables.ready()) {
        return fail(kNotReady, "dcvc_rans_gpu_create: both CDF table sets must be set first");
    }
    GpuRansHandle* g = nullptr;
    try {
        g = new GpuRansHandle();
    } catch (const std::exception& e) {
        return fail(kOutOfMemory, std::string("dcvc_rans_gpu_create: ") + e.what());
    }
    const cudaError_t e = rans_gpu_upload(r->tables, &g->tables, &g->storage);
    if (e != cudaSuccess) {
        delete g;
        return cuda_status(e, "dcvc_rans_gpu_create");
    }
    *gpu_handle = g;
    return kOk;
}

int dcvc_rans_gpu_destroy(void* gpu_handle)
{
    GpuRansHandle* g = static_cast<GpuRansHandle*>(gpu_handle);
    if (g != nullptr) {
        cudaFree(g->storage);
        delete g;
    }
    return kOk;
}

size_t dcvc_rans_gpu_scratch_bytes(int n_y, int n_z, int ecp)
{
    return rans_gpu_scratch_bytes(n_y, n_z, ecp);
}

int dcvc_rans_gpu_encode(void* gpu_handle, const dcvc_rans_gpu_enc_job* jobs, int njobs,
                         void* stream)
{
    if (gpu_handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_rans_gpu_encode: null handle");
    }
    const cudaError_t e = launch_rans_gpu_encode(static_cast<GpuRansHandle*>(gpu_handle)->tables,
                                                 jobs, njobs, static_cast<cudaStream_t>(stream));
    if (e == cudaErrorInvalidValue) {
        return fail(kInvalidArgument, "dcvc_rans_gpu_encode: bad job (1..64 jobs, ec_parallel "
                                      "1..8, z tables in range, non-null buffers)");
    }
    return cuda_status(e, "dcvc_rans_gpu_encode");
}

int dcvc_rans_gpu_decode(void* gpu_handle, const dcvc_rans_gpu_dec_job* jobs, int njobs,
                         void* stream)
{
    if (gpu_handle == nullptr) {
        return fail(kInvalidArgument, "dcvc_rans_gpu_decode: null handle");
    }
    const cudaError_t e = launch_rans_gpu_decode(static_cast<GpuRansHandle*>(gpu_handle)->tables,
                                                 jobs, njobs, static_cast<cudaStream_t>(stream));
    if (e == cudaErrorInvalidValue) {
        return fail(kInvalidArgument, "dcvc_rans_gpu_decode: bad job (1..64 jobs, ec_parallel "
                                      "1..8, z tables in range, non-null buffers)");
    }
    return cuda_status(e, "dcvc_rans_gpu_decode");
}

}  // extern "C"
