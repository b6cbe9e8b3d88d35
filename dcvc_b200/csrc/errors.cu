#include "errors.h"

#include <mutex>

namespace dcvc {

namespace {
thread_local std::string g_last_error;
std::mutex g_err_mutex;
int* g_err_word[64] = {nullptr};
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

const char* last_error() { return g_last_error.c_str(); }

int cuda_status(cudaError_t e, const char* where)
{
    if (e == cudaSuccess) {
        return kOk;
    }
    set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorInvalidValue) {
        return kInvalidArgument;
    }
    if (e == cudaErrorMemoryAllocation) {
        return kOutOfMemory;
    }
    return kCudaError;
}

int* device_error_word()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_err_mutex);
    if (g_err_word[dev] == nullptr) {
        int* p = nullptr;
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) {
            return nullptr;
        }
        cudaMemset(p, 0, sizeof(int));
        cudaDeviceSynchronize();
        g_err_word[dev] = p;
    }
    return g_err_word[dev];
}

}  // namespace dcvc
