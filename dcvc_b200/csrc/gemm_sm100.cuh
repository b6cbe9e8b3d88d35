// 1x1-convolution GEMM family for sm_100a: D[M,N] = epilogue(A[M,K] . W[N,K]^T).
//
// A is an NHWC activation (rows = pixels, K = input channels, row pitch lda), W the conv weight
// [C_out, C_in] (K-major).  Both operands are staged by TMA (128-byte swizzle) into a multi-stage
// shared-memory ring; one thread issues tcgen05.mma (M=128, N=BN, K=16) into a double-buffered
// FP32 accumulator in tensor memory; four epilogue warps drain it with tcgen05.ld, apply the
// fused epilogue and store FP16/BF16.  The kernel is persistent (one CTA per SM, static tile
// striding) so the epilogue of one tile overlaps the main loop of the next.
//
// Reference operators covered (src/layers/extensions/inference/def_cutlass.h:10-34):
//   conv1x1_bias, conv1x1_bias_wsilu, conv1x1_bias_shortcut, conv1x1_bias_shortcut2,
//   conv1x1_bias_shortcut_with_quant, conv1x1_bias_with_quant, conv1x1_bias_wsilu_chunk_add
//   (the "quad GEMM"), and the 2x2 stride-2 transposed conv (transposed_conv.cu) as a GEMM with
//   a pixel-shuffle store.
#pragma once

#include "common.cuh"

namespace dcvc {

enum GemmEpilogue : int {
    kEpiBias = 0,         // out = acc + b
    kEpiBiasWsilu = 1,    // out = wsilu(acc + b)
    kEpiBiasRes = 2,      // out = acc + b + r
    kEpiBiasResQ = 3,     // out = (acc + b + r) * q[n]
    kEpiBiasRes2 = 4,     // out = acc + b + r + r2
    kEpiQuad = 5,         // out[n/4] = sum_{k<4} wsilu(acc[n+k] + b[n+k])
    kEpiSubpel = 6,       // out[(2h+dy, 2w+dx), c] = acc  (columns ordered (dy, dx, c))
    kEpiBiasQ = 7,        // out = (acc + b) * q[n]
};

// block_n value selecting the streaming form of the residual epilogues (gemm_stream_sm100.cu):
// 128-wide channel slices with W resident in shared memory, contiguous row ranges per CTA.
constexpr int kBlockNStream = -1;
// block_n value selecting the CTA-pair form (cta_group::2, 256 x 256 tiles over two SMs, each
// staging half of the W tile) of the bias, WSiLU and quad epilogues with 16-bit operands.
constexpr int kBlockNPair = -2;

struct GemmParams {
    int M, N, K;
    const float* bias;   // [N] fp32 (may be null for kEpiSubpel)
    const void* res;     // residual rows, pitch ldr (elements)
    int ldr;
    const void* res2;
    int ldr2;
    const void* qscale;  // [N] per-output-channel multiplier (same dtype as the activations)
    void* out;           // output rows, pitch ldo (elements)
    int ldo;
    int sub_w;           // kEpiSubpel: width of the input grid (rows are h * sub_w + w)
    int sub_cout;        // kEpiSubpel: output channels per sub-pixel position
    int* err;            // device error word
    // FP8 form (dtype 2): per-output-channel FP32 factor applied to the accumulator before the
    // bias, the product of the weight row's and the activation's quantisation scales
    const float* wscale = nullptr;
    // Bounded-wait limit of the progress waits in SM clock cycles (0: about one second), and a
    // failure-detection test switch: the producer issues no loads, so the MMA and epilogue waits
    // run out, the kernel records DCVC_DEVICE_TIMEOUT in the error word and returns.  Set only
    // through gemm_inject_stall.
    long long wait_limit = 0;
    int stall_test = 0;
    // q_rows > 0: the M rows are images of q_rows rows stacked on each other and qscale holds one
    // row of N factors per image (per-stream QPs of a packed batch); 0: one row for all
    int q_rows = 0;
    // Streaming residual form only: also store E4M3(round_T(out) * out8_inv_scale) to out8 (bytes,
    // pitch ldo8), the operand of the FP8 GEMM that reads this output next
    void* out8 = nullptr;
    int ldo8 = 0;
    float out8_inv_scale = 1.f;
    // Streaming residual form only (kEpiBiasRes): A is the depthwise 3x3 convolution (zero
    // padding, no bias, FP32 sums in the order ky, kx) of the given A over a dw_h x dw_w pixel
    // grid (dw_h * dw_w = M rows, images of dw_img_h rows stacked), weights [9][K] FP32
    const float* dw_weight = nullptr;
    int dw_h = 0;
    int dw_w = 0;
    int dw_img_h = 0;
};

// The next `launches` GEMM launches of this process run with stall_test set and the given wait
// limit (failure-detection tests; launches <= 0 cancels).
void gemm_inject_stall(int launches, long long wait_limit_cycles);
// Applies a pending injection to a launch's parameters (used by the GEMM launchers).
GemmParams gemm_apply_injection(const GemmParams& p);

// dtype of gemm_sm100 / dcvc_conv1x1 for E4M3 operands with FP32 accumulation and BF16 output.
constexpr int kDtypeF8 = 2;

// The streaming form: residual epilogues (kEpiBiasRes, kEpiBiasResQ) with K <= 256, bias and
// WSiLU epilogues with K <= 512, N a multiple of 128.  Bitwise the same outputs as gemm_sm100 at
// any tile width.
bool gemm_stream_eligible(int epi, int M, int N, int K);
// Which epilogues the library's own choice (block_n = 0, no tuned width) may give the streaming
// form: 0 none, 1 the residual epilogues (default), 2 also bias and WSiLU; explicit block_n values
// are not affected.
void gemm_set_stream_form(int form);
bool gemm_stream_form_enabled();
// Whether the codecs compute the depthwise 3x3 inside the streaming residual GEMM (default off:
// measured slower than the two launches, see the kernel file).
void gemm_set_dw_fusion(bool on);
// Whether the library's own choice gives the quad GEMM the CTA-pair form (default off).
void gemm_set_pair_form(bool on);
bool gemm_dw_fusion_enabled();
cudaError_t gemm_stream_sm100(int dtype, const void* A, int lda, const void* W, const GemmParams& p,
                              int epi, cudaStream_t stream);

}  // namespace dcvc
