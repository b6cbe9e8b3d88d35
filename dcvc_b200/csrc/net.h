// Network building blocks of the codec runtime: parameter containers, weight preparation from a
// state dict, and launch sequences for the reference's layer proxies
// (src/layers/extensions/inference/layers_proxy.cpp).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

namespace dcvc {

// Owns device allocations; released together.
class DeviceArena {
public:
    DeviceArena() = default;
    DeviceArena(const DeviceArena&) = delete;
    DeviceArena& operator=(const DeviceArena&) = delete;
    ~DeviceArena() { clear(); }
    void* alloc(size_t bytes);  // nullptr on failure
    template <typename T>
    T* alloc_n(size_t n)
    {
        return static_cast<T*>(alloc(n * sizeof(T)));
    }
    void clear();
    size_t bytes() const { return bytes_; }

private:
    std::vector<void*> blocks_;
    size_t bytes_ = 0;
};

// Host copy of one state-dict entry, converted to float.
struct HostTensor {
    std::vector<int64_t> shape;
    std::vector<float> data;
    int64_t numel() const
    {
        int64_t n = 1;
        for (auto s : shape) n *= s;
        return n;
    }
};
using StateDict = std::map<std::string, HostTensor>;

// 1x1 convolution: w [cout, cin] (K-major, in the activation format `dtype`: 0 FP16, 1 BF16),
// b [cout] (FP32, may be null).  The layer reads and writes activations of its own format.
struct Lin {
    const __half* w = nullptr;
    const float* b = nullptr;
    int cin = 0, cout = 0;
    int dtype = 0;
};

// DepthConvBlock (layers.py:128-159; layers_proxy.cpp:71-206).
struct Dcb {
    bool adaptor = false;
    Lin ad;
    Lin dc1;
    const float* dw = nullptr;  // [9][cdc] FP32
    Lin dc2;                    // bias with the depthwise bias folded in
    Lin ffn1;                   // [4*cffn, C], rows 4c+k as in the reference
    Lin ffn2;
    int C = 0, cdc = 0, cffn = 0, cin = 0;
    bool shortcut = false;      // out += block input (layers.py:155-158)
    int dtype = 0;              // activation format of the whole block (0 FP16, 1 BF16)
    // FP8 form (BF16 blocks only): ffn.0 (the quad GEMM) on E4M3 operands.  ffn1_w8 [4*cffn, C]
    // E4M3 rows quantised with their own scale, ffn1_ws = row scale * kFp8ActScale.
    const uint8_t* ffn1_w8 = nullptr;
    const float* ffn1_ws = nullptr;
};

// Quantisation scale of the activations fed to the FP8 GEMMs: x_q = E4M3(x / kFp8ActScale).
// DepthConvBlock intermediates of the calibrated models stay well inside E4M3's range (+-448).
constexpr float kFp8ActScale = 1.0f;

// ResidualBlockWithStride2: pixel_unshuffle(2) + 1x1 (K permuted to (dy, dx, c)) + DCB (with the
// block shortcut when the model keeps the reference's default, layers.py:176-188).
struct DownBlock {
    Lin down;
    Dcb dcb;
};

// ResidualBlockUpsample: 1x1 (optionally biased) with rows permuted to (dy, dx, c) + shuffle
// store + DCB.
struct UpBlock {
    Lin up;
    Dcb dcb;
};

// Builds device parameters from a state dict.  Errors are reported through `ok`/`err`.
class ParamBuilder {
public:
    ParamBuilder(const StateDict& sd, DeviceArena& arena) : sd_(sd), arena_(arena) {}
    bool has(const std::string& name) const { return sd_.count(name) != 0; }
    // activation format of the layers built from here on (0 FP16, 1 BF16); half_rows tables
    // stay FP16.  fp8 (with dtype 1): DepthConvBlocks also get E4M3 copies of their ffn.0
    // weights for the FP8 quad GEMM.
    void set_dtype(int dtype, bool fp8 = false)
    {
        dtype_ = dtype;
        fp8_ = fp8 && dtype == 1;
    }
    // a [rows, cols] table of the state dict as BF16 (per-channel factors of BF16 layers)
    const __half* bf16_rows(const std::string& name, int* rows, int* cols);
    Lin lin(const std::string& prefix, bool bias = true);
    Dcb dcb(const std::string& prefix, bool shortcut = false);
    DownBlock down(const std::string& prefix, bool shortcut = false);
    UpBlock up(const std::string& prefix, bool shortcut = false);
    // SubpelConv2x (layers.py:92-103): prefix + "conv.0.{weight,bias}", 1x1 or 3x3 (K in
    // (ky, kx, c) order), rows and bias permuted to (dy, dx, c)
    Lin subpel(const std::string& prefix);
    Lin conv3x3s2(const std::string& prefix);  // weight K permuted to (ky, kx, c)
    const __half* half_rows(const std::string& name, int* rows, int* cols);
    bool ok() const { return err_.empty(); }
    const std::string& error() const { return err_; }

private:
    const HostTensor* get(const std::string& name, size_t ndim_min = 1);
    const __half* upload_half(const std::vector<float>& v);
    const __half* upload_act(const std::vector<float>& v, int dtype);  // FP16 or BF16 bits
    const float* upload_float(const std::vector<float>& v);
    void fail(const std::string& m)
    {
        if (err_.empty()) err_ = m;
    }

    const StateDict& sd_;
    DeviceArena& arena_;
    std::string err_;
    int dtype_ = 0;
    bool fp8_ = false;
};

// Per-level scratch for DCB execution.
struct Scratch {
    __half* t0 = nullptr;  // adaptor output
    __half* t1 = nullptr;  // dc.0 output
    __half* t2 = nullptr;  // depthwise output
    __half* t3 = nullptr;  // dc output (+ residual)
    __half* t4 = nullptr;  // ffn chunk-add output
    uint8_t* t5 = nullptr; // E4M3 copy of t3 (FP8 form only)
};

struct Launch {
    cudaStream_t s;
    int* err_word;
    cudaError_t first = cudaSuccess;
    int kernels = 0;  // kernels enqueued through this context
    void note(cudaError_t e, int n = 1)
    {
        kernels += n;
        if (first == cudaSuccess && e != cudaSuccess) first = e;
    }
};

// out[M, cout] (pitch ldo) = epilogue(x[M, cin] (pitch ldx) . lin).  q_rows > 0: the rows are
// images of q_rows rows each and q holds one row of factors per image.
void gemm(Launch& L, const Lin& lin, int epi, const __half* x, int ldx, int M, __half* out,
          int ldo, const __half* res = nullptr, int ldr = 0, const __half* q = nullptr,
          int sub_w = 0, const __half* res2 = nullptr, int ldr2 = 0, int q_rows = 0);

// DepthConvBlockProxy::forward (layers_proxy.cpp:71-101).  `out` may alias `x` unless the block
// has a shortcut (its last GEMM then reads the block input as a second residual).  A packed
// batch passes H = images * img_h rows of stacked images (img_h = 0: one image) and, with a
// per-image q, one row of factors per image.
void run_dcb(Launch& L, const Dcb& d, const __half* x, int ldx, int H, int W, __half* out, int ldo,
             Scratch& s, const __half* q = nullptr, int img_h = 0);

}  // namespace dcvc
