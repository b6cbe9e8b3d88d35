// Runtime tile-width autotuner for the 1x1-conv GEMM family (gemm_sm100.cu).
//
// The reference picks a CUTLASS configuration per layer shape from compile-time tables filled
// offline per GPU (HINT_MAP_* in cutlass/conv1x1_bias.cu:8 and its siblings, looked up by
// launch_cutlass_helper, cutlass/cutlass_kernel.h:232-250, with a default hint for shapes not
// in the table).  Here the choice is the N tile width of the tcgen05 kernel (256, 128 or 64),
// measured at run time: gemm_autotune() times every valid width for one shape on scratch
// operands with CUDA events and records the fastest in a process-wide table keyed by (dtype,
// epilogue, M, N, K, sub_w); gemm_sm100 consults the table whenever the caller leaves the width
// to the library, and falls back to gemm_pick_bn's rule for untuned shapes.  The tile width
// never changes an output bit (every output element is one accumulator column reduced over K in
// the same order), so tuning affects speed only.
//
// Tuning allocates and frees device memory and synchronises the stream, so it never runs while
// the stream is being captured into a graph: the codecs tune a shape on the first, eager
// execution of a phase (when enabled) and their captured graphs use the recorded widths.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "gemm_sm100.cuh"

namespace dcvc {

cudaError_t gemm_sm100(int dtype, const void* A, int lda, const void* W, const GemmParams& p,
                       int epi, int bn, cudaStream_t stream);

namespace {

// A tuned width belongs to one device: a process that runs codecs on several GPUs (one chunk
// server per device) tunes and looks up per device ordinal.
struct TuneKey {
    int dev, dtype, epi, M, N, K, sub_w;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(dev, dtype, epi, M, N, K, sub_w) <
               std::tie(o.dev, o.dtype, o.epi, o.M, o.N, o.K, o.sub_w);
    }
};

int current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return dev;
}

struct TuneEntry {
    int bn;
    float us;
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tuned;
std::atomic<size_t> g_tuned_count{0};  // lets untuned processes skip the lock
std::atomic<int> g_enabled{-1};  // -1: not read from the environment yet

constexpr int kTuneReps = 5;

bool epi_has_res(int e) { return e == kEpiBiasRes || e == kEpiBiasResQ || e == kEpiBiasRes2; }

// Device scratch for one tuning run, freed on every path.
struct Scratch {
    void* p[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    ~Scratch()
    {
        for (void* q : p) {
            if (q != nullptr) {
                cudaFree(q);
            }
        }
    }
    cudaError_t get(int i, size_t bytes, cudaStream_t s)
    {
        cudaError_t e = cudaMalloc(&p[i], bytes == 0 ? 256 : bytes);
        if (e == cudaSuccess) {
            e = cudaMemsetAsync(p[i], 0, bytes == 0 ? 256 : bytes, s);
        }
        return e;
    }
};

}  // namespace

bool gemm_autotune_enabled()
{
    int v = g_enabled.load(std::memory_order_relaxed);
    if (v < 0) {
        const char* env = std::getenv("DCVC_GEMM_AUTOTUNE");
        v = (env != nullptr && std::strcmp(env, "0") != 0 && env[0] != '\0') ? 1 : 0;
        int expected = -1;
        g_enabled.compare_exchange_strong(expected, v);
        v = g_enabled.load(std::memory_order_relaxed);
    }
    return v == 1;
}

void gemm_autotune_set_enabled(bool on) { g_enabled.store(on ? 1 : 0); }

int gemm_tuned_bn(int dtype, int epi, int M, int N, int K, int sub_w)
{
    if (g_tuned_count.load(std::memory_order_acquire) == 0) {
        return 0;
    }
    const int dev = current_device();
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(TuneKey{dev, dtype, epi, M, N, K, sub_w});
    return it == g_tuned.end() ? 0 : it->second.bn;
}

void gemm_tuning_clear()
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned.clear();
    g_tuned_count.store(0, std::memory_order_release);
}

// Times every valid N tile width of one shape and records the fastest.  p supplies the shape
// (M, N, K, sub_w, sub_cout) only; the operands are zero-filled scratch buffers.  Returns
// cudaErrorInvalidValue for shapes no width supports and cudaErrorStreamCaptureUnsupported while
// `stream` is capturing.
cudaError_t gemm_autotune(int dtype, int epi, const GemmParams& shape, cudaStream_t stream,
                          int* best_bn, float* best_us)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(stream, &cs);
    if (e != cudaSuccess) {
        return e;
    }
    if (cs != cudaStreamCaptureStatusNone) {
        return cudaErrorStreamCaptureUnsupported;
    }
    const int M = shape.M, N = shape.N, K = shape.K;
    if (M <= 0 || N <= 0 || K <= 0) {
        return cudaErrorInvalidValue;
    }
    int cands[4];
    int nc = 0;
    for (int bn : {256, 128, 64}) {
        if (N % bn != 0 || (epi == kEpiQuad && bn != 256) ||
            (epi == kEpiSubpel && (shape.sub_cout <= 0 || shape.sub_cout % bn != 0))) {
            continue;
        }
        cands[nc++] = bn;
    }
    if (gemm_stream_eligible(epi, M, N, K)) {
        cands[nc++] = kBlockNStream;  // the streaming form of the residual epilogues
    }
    if (nc == 0) {
        return cudaErrorInvalidValue;
    }
    const size_t el = 2;  // f16 / bf16
    const int nout = epi == kEpiQuad ? N / 4 : (epi == kEpiSubpel ? shape.sub_cout : N);
    const size_t out_rows = epi == kEpiSubpel ? 4 * static_cast<size_t>(M) : static_cast<size_t>(M);
    Scratch s;
    GemmParams p = shape;
    if ((e = s.get(0, static_cast<size_t>(M) * K * el, stream)) != cudaSuccess ||
        (e = s.get(1, static_cast<size_t>(N) * K * el, stream)) != cudaSuccess ||
        (e = s.get(2, static_cast<size_t>(N) * sizeof(float), stream)) != cudaSuccess ||
        (e = s.get(3, out_rows * nout * el, stream)) != cudaSuccess) {
        return e;
    }
    p.bias = epi == kEpiSubpel ? nullptr : static_cast<const float*>(s.p[2]);
    p.out = s.p[3];
    p.ldo = nout;
    p.res = p.res2 = p.qscale = nullptr;
    p.ldr = p.ldr2 = 0;
    if (epi_has_res(epi)) {
        if ((e = s.get(4, static_cast<size_t>(M) * N * el, stream)) != cudaSuccess) {
            return e;
        }
        p.res = s.p[4];
        p.ldr = N;
        if (epi == kEpiBiasRes2) {
            p.res2 = s.p[4];  // read twice: the timing needs the traffic, not distinct values
            p.ldr2 = N;
        }
    }
    if (epi == kEpiBiasResQ || epi == kEpiBiasQ) {
        if ((e = s.get(5, static_cast<size_t>(N) * el, stream)) != cudaSuccess) {
            return e;
        }
        p.qscale = s.p[5];
    }
    cudaEvent_t ev[2];
    if ((e = cudaEventCreate(&ev[0])) != cudaSuccess) {
        return e;
    }
    if ((e = cudaEventCreate(&ev[1])) != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        return e;
    }
    int best = 0;
    float best_t = 0.f;
    for (int i = 0; i < nc && e == cudaSuccess; ++i) {
        e = gemm_sm100(dtype, s.p[0], K, s.p[1], p, epi, cands[i], stream);  // warm-up
        if (e == cudaErrorInvalidValue) {
            e = cudaSuccess;  // this width does not support the shape (e.g. alignment)
            continue;
        }
        for (int r = 0; r < kTuneReps && e == cudaSuccess; ++r) {
            if (r == 0) {
                e = cudaEventRecord(ev[0], stream);
            }
            if (e == cudaSuccess) {
                e = gemm_sm100(dtype, s.p[0], K, s.p[1], p, epi, cands[i], stream);
            }
        }
        if (e == cudaSuccess) {
            e = cudaEventRecord(ev[1], stream);
        }
        if (e == cudaSuccess) {
            e = cudaEventSynchronize(ev[1]);
        }
        float ms = 0.f;
        if (e == cudaSuccess) {
            e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
        }
        const float us = ms * 1e3f / kTuneReps;
        if (e == cudaSuccess && (best == 0 || us < best_t)) {
            best = cands[i];
            best_t = us;
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (e != cudaSuccess) {
        return e;
    }
    if (best == 0) {
        return cudaErrorInvalidValue;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[TuneKey{current_device(), dtype, epi, M, N, K, epi == kEpiSubpel ? shape.sub_w : 0}] =
            TuneEntry{best, best_t};
        g_tuned_count.store(g_tuned.size(), std::memory_order_release);
    }
    if (best_bn != nullptr) {
        *best_bn = best;
    }
    if (best_us != nullptr) {
        *best_us = best_t;
    }
    return cudaSuccess;
}

// The codecs' hook: the tuned width of this shape, tuning it first when tuning is enabled, the
// shape is new and the stream is not capturing; 0 (the library's rule) otherwise.
int gemm_bn_for(int dtype, int epi, const GemmParams& p, cudaStream_t stream)
{
    const int sub_w = epi == kEpiSubpel ? p.sub_w : 0;
    const int bn = gemm_tuned_bn(dtype, epi, p.M, p.N, p.K, sub_w);
    if (bn != 0 || !gemm_autotune_enabled()) {
        return bn;
    }
    int best = 0;
    if (gemm_autotune(dtype, epi, p, stream, &best, nullptr) != cudaSuccess) {
        cudaGetLastError();  // an untunable shape keeps the library's rule
        return 0;
    }
    return best;
}

}  // namespace dcvc
