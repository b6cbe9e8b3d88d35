// Fused ConvFFN of a DepthConvBlock for sm_100a (ffn.0 quad GEMM + ffn.2 residual GEMM in one
// kernel, the quad output kept in shared memory); see ffn_sm100.cu.
#pragma once

#include "common.cuh"

#include <cuda.h>

namespace dcvc {

struct FfnParams {
    int M;               // pixels
    int C;               // block channels: ffn.0 K, ffn.2 N (a multiple of 256)
    int cffn;            // ffn.2 K = quad outputs (128 or 256); ffn.0 N = 4 cffn
    const float* b1;     // [4 cffn] fp32
    const float* b2;     // [C] fp32
    const void* qscale;  // [C] FP16 multiplier (conv1x1_bias_shortcut_with_quant) or null
    void* out;           // [M, C] rows, pitch ldo
    int ldo;
    int* err;            // device error word
    int block_n;         // accumulator columns per item, 128 or 256 (0: the library's choice)
};

// Whether ffn_sm100 handles a block with these channel counts (n1 = ffn.0 output channels), and
// whether it is faster there than the two separate GEMMs (the codecs use it only then).
bool ffn_sm100_supported(int C, int cffn, int n1);
bool ffn_sm100_preferred(int C, int cffn, int n1);

// out = (quad(x . W1^T + b1) . W2^T + b2 + x) [* qscale] for x [M, C] FP16 (pitch ldx), W1 [4 cffn,
// C], W2 [C, cffn] dense FP16.  cudaErrorInvalidValue for unsupported shapes or alignments.
cudaError_t ffn_sm100(const void* x, int ldx, const void* w1, const void* w2, const FfnParams& p,
                      cudaStream_t stream);

}  // namespace dcvc
