// Pieces shared by the codec runtimes (the HT-S video codec and the intra codec): per-phase CUDA
// graphs, CDF-table loading from a state dict and the device error word check.  They play the
// part of the reference's DMCCommon (src/layers/extensions/inference/dmc_common.cpp:10-134).
#pragma once

#include "net.h"
#include "rans_coder.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <chrono>
#include <functional>
#include <vector>

namespace dcvc {

// An NVTX range over a scope (phase graph launches, host entropy coding), visible to profilers
// that attach an NVTX tool; without one the calls do nothing.
class NvtxRange {
public:
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

using Clock = std::chrono::steady_clock;
inline float ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<float, std::milli>(b - a).count();
}

// One CUDA graph per phase slot.  The first run of a slot is eager (it initialises every
// kernel's attributes and validates the launches), the second is captured into a graph, later
// runs replay it (DMCCommon::run / capture_cuda_graph, dmc_common.cpp:85-134).
class PhaseGraphs {
public:
    explicit PhaseGraphs(int slots) : slots_(slots) {}
    PhaseGraphs(const PhaseGraphs&) = delete;
    PhaseGraphs& operator=(const PhaseGraphs&) = delete;
    ~PhaseGraphs() { clear(); }
    void clear();
    // Enqueues phase `slot` on s; adds the phase's kernel count to *kernels.  Every phase ends by
    // publishing the device error word into the mapped host slot set with set_error_slot, so
    // that the host can check it after an event on s without a synchronous copy.
    int run(int slot, cudaStream_t s, int* err_word, const std::function<void(Launch&)>& body,
            int* kernels);
    void set_error_slot(int* slot_dev) { err_slot_dev_ = slot_dev; }

private:
    struct Slot {
        cudaGraphExec_t exec = nullptr;
        bool ran_eager = false;
        int kernels = 0;
    };
    std::vector<Slot> slots_;
    int* err_slot_dev_ = nullptr;
};

// A mapped pinned host int that phase graphs copy the device error word into.
struct ErrorSlot {
    int* host = nullptr;
    int* dev = nullptr;
    bool alloc();
    void release();
};

// Loads "bit_estimator_z.{quantized_cdf,cdf_length}" (table set 0) and
// "gaussian_encoder.{quantized_cdf,cdf_length}" (table set 1) and checks their counts.
int load_cdf_tables(const StateDict& sd, RansTables* tables, int z_count, int y_count);

// Pinned host memory mapped into the device address space (cudaHostAllocMapped): *host for the
// CPU, *dev for kernels.  Returns false (and leaves both null) when the allocation fails.
bool alloc_mapped(size_t bytes, void** host, void** dev);

// Checks the error word as the last phase graph published it into `slot` (and clears both the
// slot and the device word); kDeviceTimeout if a kernel's bounded wait gave up.  The caller must
// have waited for an event recorded after that phase.
int check_device_error_word(int* err_word, ErrorSlot& slot, const char* where);

}  // namespace dcvc
