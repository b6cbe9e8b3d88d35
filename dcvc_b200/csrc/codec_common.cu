#include "codec_common.h"

#include "elementwise.cuh"

#include "errors.h"

#include <string>

namespace dcvc {

void PhaseGraphs::clear()
{
    for (Slot& g : slots_) {
        if (g.exec != nullptr) {
            cudaGraphExecDestroy(g.exec);
        }
        g = Slot{};
    }
}

int PhaseGraphs::run(int slot, cudaStream_t s, int* err_word,
                     const std::function<void(Launch&)>& body, int* kernels)
{
    if (slot < 0 || slot >= static_cast<int>(slots_.size())) {
        set_last_error("internal: bad phase slot");
        return kInternal;
    }
    Slot& g = slots_[slot];
    if (g.exec != nullptr) {
        *kernels += g.kernels;
        return cuda_status(cudaGraphLaunch(g.exec, s), "cudaGraphLaunch");
    }
    Launch L{s, err_word};
    auto body_and_publish = [&]() {
        body(L);
        if (err_slot_dev_ != nullptr && err_word != nullptr) {
            L.note(launch_copy_counted(err_word, err_slot_dev_, sizeof(int), nullptr, 1, nullptr, s));
        }
    };
    if (!g.ran_eager) {
        body_and_publish();
        g.ran_eager = true;
        g.kernels = L.kernels;
        *kernels += L.kernels;
        return L.first != cudaSuccess ? cuda_status(L.first, "phase launch") : kOk;
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        return cuda_status(e, "cudaStreamBeginCapture");
    }
    body_and_publish();
    e = cudaStreamEndCapture(s, &graph);
    if (L.first != cudaSuccess || e != cudaSuccess) {
        if (graph != nullptr) {
            cudaGraphDestroy(graph);
        }
        cudaGetLastError();
        return cuda_status(L.first != cudaSuccess ? L.first : e, "graph capture");
    }
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        g.exec = nullptr;
        return cuda_status(e, "cudaGraphInstantiate");
    }
    *kernels += g.kernels;
    return cuda_status(cudaGraphLaunch(g.exec, s), "cudaGraphLaunch");
}

int load_cdf_tables(const StateDict& sd, RansTables* tables, int z_count, int y_count)
{
    auto table = [&](const char* cdf_name, const char* len_name, int index) -> bool {
        auto a = sd.find(cdf_name), b = sd.find(len_name);
        if (a == sd.end() || b == sd.end() || a->second.shape.size() != 2) {
            set_last_error(std::string("set_param: missing or malformed ") + cdf_name);
            return false;
        }
        const int count = static_cast<int>(a->second.shape[0]);
        const int stride = static_cast<int>(a->second.shape[1]);
        if (b->second.numel() != count) {
            set_last_error(std::string("set_param: ") + len_name + " does not match its table");
            return false;
        }
        std::vector<int32_t> cdf(a->second.data.size()), len(count);
        for (size_t i = 0; i < cdf.size(); ++i) cdf[i] = static_cast<int32_t>(a->second.data[i]);
        for (int i = 0; i < count; ++i) len[i] = static_cast<int32_t>(b->second.data[i]);
        std::string err;
        if (!tables->set(index, cdf.data(), len.data(), count, stride, &err)) {
            set_last_error("set_param: " + err);
            return false;
        }
        return true;
    };
    if (!table("bit_estimator_z.quantized_cdf", "bit_estimator_z.cdf_length", 0) ||
        !table("gaussian_encoder.quantized_cdf", "gaussian_encoder.cdf_length", 1)) {
        return kInvalidArgument;
    }
    if (tables->z().count != z_count || tables->y().count != y_count) {
        set_last_error("set_param: expected " + std::to_string(z_count) +
                       " bit-estimator tables and " + std::to_string(y_count) + " Gaussian tables");
        return kInvalidArgument;
    }
    return kOk;
}

int check_device_error_word(int* err_word, ErrorSlot& slot, const char* where)
{
    if (err_word == nullptr || slot.host == nullptr) {
        return kOk;
    }
    const int code = *static_cast<volatile int*>(slot.host);
    if (code != 0) {
        cudaMemset(err_word, 0, sizeof(int));
        *static_cast<volatile int*>(slot.host) = 0;
        set_last_error(std::string(where) + ": a kernel's bounded wait gave up (device error " +
                       std::to_string(code) + ")");
        return kDeviceTimeout;
    }
    return kOk;
}

bool ErrorSlot::alloc()
{
    void *h = nullptr, *d = nullptr;
    if (!alloc_mapped(sizeof(int), &h, &d)) {
        return false;
    }
    host = static_cast<int*>(h);
    dev = static_cast<int*>(d);
    *host = 0;
    return true;
}

void ErrorSlot::release()
{
    if (host != nullptr) {
        cudaFreeHost(host);
    }
    host = nullptr;
    dev = nullptr;
}

bool alloc_mapped(size_t bytes, void** host, void** dev)
{
    *host = nullptr;
    *dev = nullptr;
    if (cudaHostAlloc(host, bytes, cudaHostAllocMapped) != cudaSuccess) {
        cudaGetLastError();
        *host = nullptr;
        return false;
    }
    if (cudaHostGetDevicePointer(dev, *host, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeHost(*host);
        *host = nullptr;
        *dev = nullptr;
        return false;
    }
    return true;
}

}  // namespace dcvc
