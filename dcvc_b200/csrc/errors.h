// Error reporting shared by the C-ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace dcvc {

// Status codes returned by every extern "C" entry point.
enum Status : int {
    kOk = 0,
    kInvalidArgument = 1,
    kCudaError = 2,
    kDeviceTimeout = 3,   // a kernel's bounded wait gave up (device error word set)
    kOutOfMemory = 4,
    kCorruptStream = 5,   // rANS payload inconsistent with its container header
    kNotReady = 6,        // a submit/wait call made out of order
    kHostTimeout = 7,     // a host-side wait on a worker thread gave up
    kInternal = 8,
};

// Thread-local message of the last failing call on this thread.
void set_last_error(const std::string& msg);
const char* last_error();

// Converts a CUDA status into a Status, recording a message.
int cuda_status(cudaError_t e, const char* where);

// Per-device word that kernels set when a bounded wait gives up (allocated on first use).
int* device_error_word();

}  // namespace dcvc
