// rANS coding on the GPU in the MLCodec container format, byte-identical with the host coder
// (rans_coder.h; the reference's src/cpp/py_rans/rans.cpp, py_rans.cpp).  The format fixes the
// parallelism: a payload holds at most 8 sub-streams, each a sequential rANS chain, so one thread
// codes one sub-stream and one warp one payload; many payloads (independent video streams) are
// coded by one launch.  Symbols, indexes, payloads and decoded values stay in device memory.
#pragma once

#include "dcvc_b200.h"
#include "rans_coder.h"

#include <cuda_runtime.h>
#include <stdint.h>

namespace dcvc {

constexpr int kRansGpuMaxJobs = 64;

// Device copies of a RansTables (table set 0 = z, 1 = y).
struct RansGpuTables {
    const uint32_t* enc[2] = {nullptr, nullptr};   // [count * stride]: start | freq << 16
    const int32_t* cdf[2] = {nullptr, nullptr};    // [count * stride]
    const int32_t* maxv[2] = {nullptr, nullptr};   // [count]
    int count[2] = {0, 0};
    int stride[2] = {0, 0};
};

// One payload to encode (the y segment then the z segment, as RansEncoderSession::add_y/add_z)
// and one payload to decode (z first, then the y symbols with their table indexes); the plain-C
// job structs of the public header (dcvc_rans_gpu_enc_job / dcvc_rans_gpu_dec_job).
using RansGpuEncJob = dcvc_rans_gpu_enc_job;
using RansGpuDecJob = dcvc_rans_gpu_dec_job;

enum RansGpuStatus {
    kRansGpuOk = 0,
    kRansGpuBadIndex = 1,      // a y symbol or index names a table past the set
    kRansGpuOverflow = 2,      // a sub-stream or the container outgrew its buffer
    kRansGpuBadHeader = 3,     // inconsistent sub-stream offsets
    kRansGpuOverrun = 4,       // a sub-stream ran past its bytes (truncated or corrupt)
    kRansGpuZeroFreq = 5,      // a symbol has zero probability in its table
};

// Scratch bytes an encode job needs (every sub-stream's worst case, 4 bytes per symbol + 16).
size_t rans_gpu_scratch_bytes(int n_y, int n_z, int ecp);

// Uploads both table sets (RansTables::ready() must hold) into `arena`-style device memory owned
// by the caller through *storage (freed with cudaFree).
cudaError_t rans_gpu_upload(const RansTables& t, RansGpuTables* out, void** storage);

cudaError_t launch_rans_gpu_encode(const RansGpuTables& t, const RansGpuEncJob* jobs, int njobs,
                                   cudaStream_t s);
cudaError_t launch_rans_gpu_decode(const RansGpuTables& t, const RansGpuDecJob* jobs, int njobs,
                                   cudaStream_t s);

}  // namespace dcvc
