#include "codec_common.h"

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
    if (!g.ran_eager) {
        body(L);
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
    body(L);
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

int check_device_error_word(int* err_word, const char* where)
{
    int code = 0;
    if (err_word == nullptr) {
        return kOk;
    }
    if (cudaMemcpy(&code, err_word, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        return cuda_status(cudaGetLastError(), where);
    }
    if (code != 0) {
        cudaMemset(err_word, 0, sizeof(int));
        set_last_error(std::string(where) + ": a kernel's bounded wait gave up (device error " +
                       std::to_string(code) + ")");
        return kDeviceTimeout;
    }
    return kOk;
}

}  // namespace dcvc
