/*
 * dcvc_b200 C ABI.
 *
 * Plain pointers and sizes only.  Every function returns 0 (DCVC_OK) or a DCVC_* status; the
 * message of the last failure on the calling thread is available from dcvc_last_error().
 * Device pointers are CUDA global memory of the current device; `stream` is a cudaStream_t
 * (NULL = legacy default stream).  Activations are NHWC ("channels last"): a tensor of C
 * channels over an H x W grid is H*W rows of C contiguous elements; `ld*` is the row pitch in
 * elements (>= C) so channel slices of concatenation buffers can be passed directly.
 *
 * Each declaration names the reference interface it replaces (paths inside the reference
 * project).
 */
#ifndef DCVC_B200_H
#define DCVC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DCVC_ABI_VERSION 1

/* status codes */
#define DCVC_OK 0
#define DCVC_INVALID_ARGUMENT 1
#define DCVC_CUDA_ERROR 2
#define DCVC_DEVICE_TIMEOUT 3
#define DCVC_OUT_OF_MEMORY 4
#define DCVC_CORRUPT_STREAM 5
#define DCVC_NOT_READY 6
#define DCVC_HOST_TIMEOUT 7
#define DCVC_INTERNAL 8

/* element types */
#define DCVC_F16 0
#define DCVC_BF16 1
#define DCVC_F32 2
#define DCVC_I32 3
#define DCVC_I64 4

/* precision forms of the HT-S codec (dcvc_hts_set_precision) */
#define DCVC_PRECISION_F16 0
#define DCVC_PRECISION_BF16 1
#define DCVC_PRECISION_FP8 2

/* block_n of dcvc_conv1x1 selecting the streaming form of the residual epilogues */
#define DCVC_BLOCK_N_STREAM (-1)
/* block_n of dcvc_conv1x1 selecting the CTA-pair form of the bias, WSiLU and quad epilogues
 * (cta_group::2: two SMs share each 256 x 256 tile, each staging half of its W rows; 16-bit) */
#define DCVC_BLOCK_N_PAIR (-2)

/* 1x1-conv GEMM epilogues (dcvc_conv1x1) */
#define DCVC_EPI_BIAS 0        /* conv1x1_bias                       */
#define DCVC_EPI_BIAS_WSILU 1  /* conv1x1_bias_wsilu                 */
#define DCVC_EPI_BIAS_RES 2    /* conv1x1_bias_shortcut              */
#define DCVC_EPI_BIAS_RES_Q 3  /* conv1x1_bias_shortcut_with_quant   */
#define DCVC_EPI_BIAS_RES2 4   /* conv1x1_bias_shortcut2             */
#define DCVC_EPI_QUAD 5        /* conv1x1_bias_wsilu_chunk_add       */
#define DCVC_EPI_SUBPEL 6      /* transposed_conv (2x2, stride 2)    */
#define DCVC_EPI_BIAS_Q 7      /* conv1x1_bias_with_quant            */

/* ------------------------------------------------------------------ library */

const char* dcvc_last_error(void);
int dcvc_abi_version(void);
/* Reads (and optionally clears) the device error word that kernels set when one of their
 * bounded waits gave up.  *code = 0 means no error.  Synchronises the device. */
int dcvc_device_error(int* code, int clear);
/* Synchronises `stream`, then returns DCVC_DEVICE_TIMEOUT (and clears the word) if a kernel's
 * bounded wait gave up, else DCVC_OK.  The reference has no bounded waits (its proxy can wait
 * for ever, dmc_hts_proxy.cpp:579); no counterpart there. */
int dcvc_check_device_errors(void* stream);
/* Failure-detection test hook: the next `launches` GEMM launches (dcvc_conv1x1 and the codecs'
 * GEMMs) issue no operand loads and give their progress waits a limit of wait_limit_cycles SM
 * clocks, so the waits run out: the kernel records the timeout in the device error word, drains
 * only the copies it issued, frees its tensor memory and returns, and the GPU stays usable.
 * launches <= 0 cancels.  No counterpart in the reference. */
int dcvc_gemm_inject_stall(int launches, long long wait_limit_cycles);

/* ------------------------------------------------------------------ kernels */

/* out[M, N] = epilogue(a[M, K] . w[N, K]^T)
 * Replaces conv1x1_bias / _wsilu / _shortcut / _shortcut2 / _shortcut_with_quant /
 * _with_quant / _wsilu_chunk_add (src/layers/extensions/inference/def_cutlass.h:10-34,
 * cutlass/conv1x1_kernel.h:158-435) and transposed_conv (cutlass/transposed_conv_kernel.h:22-86,
 * as a GEMM whose weight rows are ordered (dy, dx, c) and whose epilogue stores the
 * pixel-shuffled result).
 *   bias   : fp32 [N] (unused for DCVC_EPI_SUBPEL)
 *   res    : residual rows, pitch ldr (BIAS_RES, BIAS_RES_Q, BIAS_RES2)
 *   res2   : second residual, pitch ldr2 (BIAS_RES2)
 *   qscale : per-output-channel multiplier [N], activation dtype (BIAS_RES_Q, BIAS_Q)
 *   out    : [M, N] rows (QUAD: [M, N/4]; SUBPEL: [(2H)(2W), sub_cout]) with pitch ldo
 *   sub_w, sub_cout : SUBPEL input width and output channels (N = 4 * sub_cout)
 *   block_n: N tile 256 / 128 / 64 of the tiled kernel, DCVC_BLOCK_N_STREAM for the streaming
 *            form of BIAS_RES / BIAS_RES_Q (K <= 256, N a multiple of 128: W slice resident in
 *            shared memory, contiguous row ranges per CTA), 0 = choose; every choice gives the
 *            same output bits.  K must be a multiple of 64, lda/ldr/ldo multiples of 8. */
int dcvc_conv1x1(int dtype, int epilogue, int M, int N, int K, const void* a, int lda,
                 const void* w, const float* bias, const void* res, int ldr, const void* res2,
                 int ldr2, const void* qscale, void* out, int ldo, int sub_w, int sub_cout,
                 int block_n, void* stream);
/* Which GEMMs the library's own tile choice (block_n = 0 without a tuned width, and the codecs)
 * gives the streaming form: 0 none, 1 the residual epilogues at K <= 256 (the default), 2 also
 * the bias and WSiLU epilogues at K <= 512.  Output bits are the same either way.  No counterpart
 * in the reference. */
int dcvc_gemm_stream_form(int enable);
/* Whether the library's own tile choice (and the codecs) gives the quad GEMM the CTA-pair form
 * (DCVC_BLOCK_N_PAIR): 1 or 0 (the default).  No counterpart in the reference. */
int dcvc_gemm_pair_form(int enable);
/* The FP8 form of dcvc_conv1x1 for the epilogues BIAS, BIAS_WSILU and QUAD: a [M, K] and
 * w [N, K] are E4M3 bytes (lda a multiple of 16, K of 128), the tcgen05 MMA is kind::f8f6f4
 * with FP32 accumulation, and the epilogue computes acc * wscale[n] + bias[n] (wscale: FP32
 * per output channel, the product of the activation's and the weight row's quantisation
 * scales) before the activation; out is BF16.  No counterpart in the reference (its GEMMs are
 * FP16, cutlass/conv1x1_kernel.h:37-41). */
int dcvc_conv1x1_f8(int epilogue, int M, int N, int K, const void* a, int lda, const void* w,
                    const float* wscale, const float* bias, void* out, int ldo, int block_n,
                    void* stream);
/* dst[m, c] = E4M3(src[m, c] * inv_scale), saturating at +-448: src FP16 or BF16 (src_dtype
 * DCVC_F16 / DCVC_BF16) with pitch lds, dst bytes with pitch ldd (C and both pitches multiples
 * of 8).  The A operand of dcvc_conv1x1_f8; no counterpart in the reference. */
int dcvc_quantize_fp8(const void* src, int src_dtype, int lds, float inv_scale, void* dst, int ldd,
                      int M, int C, void* stream);

/* Runtime autotuner of the dcvc_conv1x1 tile width.  Replaces the reference's compile-time
 * per-shape configuration tables (HINT_MAP_* in src/layers/extensions/inference/cutlass/
 * conv1x1_bias.cu:8 and its siblings, looked up by launch_cutlass_helper, cutlass_kernel.h:232-250).
 * dcvc_gemm_autotune times every valid N tile (256, 128, 64) of one shape (M, N, K, epilogue;
 * sub_w / sub_cout for SUBPEL) on zero-filled scratch operands on `stream`, which must not be
 * capturing, and records the fastest in a process-wide table; *block_n and *us (either may be
 * NULL) receive the choice and its time per launch.  dcvc_conv1x1 with block_n = 0 and the
 * codecs use a recorded width for their shape, else the library's rule.  The tile width changes
 * no output bit.  dcvc_gemm_autotune_enable(1) (or DCVC_GEMM_AUTOTUNE=1 in the environment) makes
 * the codecs tune every new shape on the first, eager run of a phase, before its graph is
 * captured.  dcvc_gemm_tuned reports the recorded width (0 = none); dcvc_gemm_tuning_clear
 * empties the table. */
int dcvc_gemm_autotune(int dtype, int epilogue, int M, int N, int K, int sub_w, int sub_cout,
                       void* stream, int* block_n, float* us);
int dcvc_gemm_autotune_enable(int on);
int dcvc_gemm_tuned(int dtype, int epilogue, int M, int N, int K, int sub_w, int* block_n);
int dcvc_gemm_tuning_clear(void);

/* The ConvFFN half of a DepthConvBlock in one kernel (layers_proxy.cpp:95-101: the
 * conv1x1_bias_wsilu_chunk_add quad GEMM followed by conv1x1_bias_shortcut[_with_quant]):
 * out = (quad(x . w1^T + b1) . w2^T + b2 + x) [* qscale], with the quad output kept on chip.
 * x, out [M, C] FP16 (pitches ldx, ldo), w1 [4 cffn, C] (rows 4c+k), w2 [C, cffn], b1 / b2 FP32,
 * qscale [C] FP16 or NULL.  C a multiple of 256, cffn 128 or 256; block_n = accumulator columns
 * per work item, 128 or 256 (0 = choose).  Bit-identical with the two dcvc_conv1x1 calls
 * (DCVC_EPI_QUAD, then DCVC_EPI_BIAS_RES / _RES_Q). */
int dcvc_conv_ffn(int M, int C, int cffn, const void* x, int ldx, const void* w1, const float* b1,
                  const void* w2, const float* b2, const void* qscale, void* out, int ldo,
                  int block_n, void* stream);

/* Depthwise 3x3, pad 1, no bias, FP32 accumulation: x, out [H*W, C] FP16 (pitches ldx, ldo),
 * w FP32 [9][C] tap-major.  Replaces d3x3 (src/layers/extensions/inference/cutlass/
 * d3x3_kernel.h:104-166, d3x3.cu). */
int dcvc_dwconv3x3(const void* x, int H, int W, int C, int ldx, const float* w, void* out, int ldo,
                   void* stream);
/* dcvc_dwconv3x3 for FP16 or BF16 (dtype) over images of img_h rows stacked along H (a tap in
 * the image above or below reads zero; img_h = 0: one image).  No counterpart in the reference
 * (FP16 only there, one image per launch). */
int dcvc_dwconv3x3_ex(int dtype, const void* x, int H, int W, int img_h, int C, int ldx, const float* w,
                      void* out, int ldo, void* stream);
/* out[M, N] = dw(x)[M, K] . w[N, K]^T + bias + res with M = H * W: the DepthConvBlock's depthwise
 * 3x3 and the conv1x1_bias_shortcut after it (src/layers/extensions/inference/layers_proxy.cpp:81-82,
 * d3x3 then conv1x1_bias_shortcut) as one launch of the streaming residual GEMM, whose operand
 * producer computes the depthwise 3x3 on the CUDA cores; its output never goes to memory.  dw is
 * dcvc_dwconv3x3_ex (x [H*W, K] pitch ldx, dw_weight FP32 [9][K], images of img_h rows, 0: one)
 * and the result is bitwise that of dcvc_dwconv3x3_ex followed by dcvc_conv1x1 with
 * DCVC_EPI_BIAS_RES.  dtype DCVC_F16 or DCVC_BF16; K a multiple of 64 up to 256, N of 128; w, res,
 * out with pitches K, ldr, ldo.  No counterpart in the reference (two launches there). */
int dcvc_dw3x3_conv1x1_res(int dtype, int H, int W, int img_h, const void* x, int ldx,
                           const float* dw_weight, int K, const void* w, int N, const float* bias,
                           const void* res, int ldr, void* out, int ldo, void* stream);
/* Whether the codecs run each DepthConvBlock's depthwise 3x3 inside the residual GEMM that follows
 * it (1; needs the streaming form) or as a launch of its own (0, the default: at 1080p the fused
 * launch takes 114.7 us against 32.2 us for the two launches).  Output bits are the same either
 * way.  No counterpart in the reference. */
int dcvc_dw_fusion(int enable);

/* Layout kernels (FP16, NHWC rows with pitches in elements). */
/* pad_and_unshuffle_8 / pixel_unshuffle(8) (elementwise/cat_and_pad.cu:7-51, shuffle.cu:134-185):
 * out[h8, w8, c*64 + dy*8 + dx] = x[min(8 h8 + dy, H-1), min(8 w8 + dx, W-1), c]. */
int dcvc_pad_unshuffle8(const void* x, int H, int W, int C, int ldx, int pad_b, int pad_r,
                        void* out, int ldo, void* stream);
/* pixel_shuffle_8 with clamp to [-0.5, 0.5] (shuffle.cu:40-131); out [8 H8, 8 W8, C] dense. */
int dcvc_shuffle8_clamp(const void* in, int H8, int W8, int C, int ldi, void* out, void* stream);
/* pixel_unshuffle(2) with channels in (dy, dx, c) order, the A operand of the stride-2 1x1
 * conv of ResidualBlockWithStride2 (layers_proxy.cpp:234-267). */
int dcvc_space_to_depth2(const void* x, int H, int W, int C, int ldx, void* out, void* stream);
/* 3x3 stride-2 pad-1 patches in (ky, kx, c) order, the A operand of conv_bias with kernel 3
 * (cutlass/conv_kernel.h:22-89). */
int dcvc_im2col3x3s2(const void* x, int H, int W, int C, int ldx, void* out, void* stream);

/* YUV 4:2:0 planar (I420) I/O on the device.  get_src_frame for YUV input (test_video.py:69-123,
 * ycbcr420_to_444_np transforms.py:69-80): planes = `frames` (1..8) I420 frames back to back
 * (uint8, even H and W); out [H, W] pixels with pitch ldo >= 3 frames,
 * out[p * ldo + 3 f + c] = FP16(FP16(sample / 255) - 0.5), chroma nearest-neighbour up-sampled. */
int dcvc_yuv420_to_input(const void* planes, int frames, int H, int W, void* out, int ldo,
                         void* stream);
/* The decoded-frame writer of test_video.py:355-362 (yuv_444_to_420, transforms.py:83-90): frames
 * = host array of nframes (1..8) device pointers to FP16 [Hp, Wp, 3] pictures (pixel pitch ldp),
 * cropped to H x W; planes receives their I420 planes back to back: Y = round(clamp(FP16(
 * FP16(x + 0.5) * 255), 0, 255)), U / V = trunc of the same on the 2x2 average. */
int dcvc_frames_to_yuv420(const void* const* frames, int nframes, int H, int W, int Wp, int ldp,
                          void* planes, void* stream);
/* replicate_pad / slice (cat_and_pad.cu:53-110). */
int dcvc_replicate_pad(const void* x, int H, int W, int C, int ldx, int pad_b, int pad_r, void* out,
                       void* stream);
int dcvc_crop(const void* x, int Wx, int ldx, int H, int W, int C, void* out, int ldo, void* stream);

/* Latent kernels (elementwise/stream.cu). */
/* round_z :862-894: z_hat = clamp(round(z), -64, 63) as FP16 and int8. */
int dcvc_round_z(const void* z, int n, void* z_hat, int8_t* z_i8, void* stream);
/* int8_to_dtype :454-482. */
int dcvc_int8_to_half(const int8_t* x, int n, void* out, void* stream);
/* multiply_with_broadcast :484-546: out[m, c] = x[m, c] * q[c]. */
int dcvc_mul_channel(const void* x, int M, int C, int ldx, const void* q, void* out, int ldo,
                     void* stream);
/* divide_with_clamp_inplace :422-452: y *= rcp(max(q, 0.5)). */
int dcvc_div_clamp(void* y, int M, int C, int ldy, const void* q, int ldq, void* stream);
/* process_with_mask_no_scale[_add_inplace][_add_and_multiply_inplace] :548-683 for checkerboard
 * phase 0..3; mode 0 writes, 1 accumulates, 2 accumulates and scales y_hat by max(q_dec, 0.5). */
int dcvc_quantize_phase(int phase, int mode, const void* y, int ldy, const void* scales, int lds,
                        const void* means, int ldm, const void* q_dec, int ldd, float thr, void* y_q,
                        int ldq, void* y_hat, int ldh, int H, int W, int C, void* stream);
/* restore_y[_and_add_inplace][_and_add_multiply_inplace] :685-760. */
int dcvc_restore_phase(int phase, int mode, const void* y_q, int ldq, const void* means, int ldm,
                       const void* q_dec, int ldd, void* y_hat, int ldh, int H, int W, int C,
                       void* stream);
/* build_index_enc / build_index_dec :89-173 (encode != 0: sym = (q << 8) + idx, else idx), with
 * cond = scale > thr, NHWC symbol order; lut from dcvc_scale_index_table on the device. */
int dcvc_build_index(int encode, const void* y_q, int ldq, const void* scales, int lds, float thr,
                     const uint8_t* lut, int M, int C, int16_t* sym, uint8_t* idx, uint8_t* cond,
                     void* stream);
/* conditional_index_part1 :175-338: order-preserving compaction of src (1- or 2-byte
 * elements) under cond; block_counts needs dcvc_compact_blocks(n) ints; *total (device) gets
 * the kept count. */
int dcvc_compact_blocks(int n);
int dcvc_compact(const void* src, int elem_bytes, const uint8_t* cond, int n, int* block_counts,
                 void* dst, int* total, void* stream);
/* Allocation-free dcvc_compact, for callers that cannot allocate device memory (a caller whose
 * device memory is pre-partitioned by its own allocator, or that cannot take cudaMalloc's implicit
 * synchronisation on its path): same inputs and outputs, no block_counts argument.  No counterpart
 * in the reference.  The block counts live in a 16 KB array inside the library (every GPU that
 * loads the library holds it until exit), so n <= 33,554,432 (4096 blocks of 8192); larger n is
 * rejected with DCVC_INVALID_ARGUMENT.  The first call on a device looks up the array's device
 * address and must not be made during stream capture.  All calls share the array: calls whose
 * kernels may overlap on the GPU race and must be ordered by the caller.  Allocates nothing. */
int dcvc_compact_noalloc(const void* src, int elem_bytes, const uint8_t* cond, int n, void* dst,
                         int* total, void* stream);
/* conditional_recover_with_type_conversion :359-420, with the block counts of dcvc_compact. */
int dcvc_recover(const int8_t* dec, const uint8_t* cond, const int* block_counts, int n, void* out,
                 void* stream);

/* The 65536-entry table mapping the FP16 bits of a Gaussian scale to its CDF table index, as
 * scale_to_index evaluates it in FP16 (src/layers/extensions/inference/elementwise/
 * stream.cu:77-87 with the constants of def_const.h:6-12), computed on the host with the
 * logarithm in double precision (a CPU restatement; needs no GPU). */
int dcvc_scale_index_table(uint8_t* lut);
/* The same table evaluated on the device exactly as the reference's kernel does in its
 * fast-math build (float max/min, the fast-math logarithm, FP16 roundings of the difference and
 * the product, round-down to uint8): lut is a device buffer of 65536 bytes.  The codecs use this
 * table.  Replaces the scale_to_index helper of stream.cu:77-87 (with to_uint8,
 * common_cu.h:181-184). */
int dcvc_scale_index_table_device(uint8_t* lut, void* stream);

/* ------------------------------------------------------------------ rANS coder (host) */

/* pmf -> 16-bit quantised CDF, writes n + 1 entries.
 * Replaces pmf_to_quantized_cdf (src/cpp/py_rans/py_rans.h:17, py_rans.cpp:35-94). */
int dcvc_pmf_to_quantized_cdf(const float* pmf, int n, uint32_t* cdf_out);

/* ec_parallel for a symbol count: clamp(count / 32768, 1, 8)
 * (src/layers/extensions/inference/dmc_common.cpp:31-35). */
int dcvc_ec_parallel_for(int symbol_count);

/* Failure-path testing of the host coder: the next coder task of sub-stream `sub_stream` (0 .. 7)
 * throws inside its worker thread, as a failed allocation there would.  The call that ran it
 * (dcvc_rans_encode_finish / dcvc_rans_decode_*, or a codec's compress / decompress) returns
 * DCVC_INTERNAL with the message, every other task of the call still completes, and the coder
 * stays usable.  The reference terminates the process in that case (a worker exception,
 * rans.cpp:209-222 under py_rans.cpp:104-135).  -1 cancels a pending injection. */
int dcvc_rans_inject_task_fault(int sub_stream);

/* A coder handle owns two CDF table sets (index 0: z / bit estimator, index 1: y / Gaussian),
 * one payload being encoded and one being decoded.  Not thread-safe; one handle per thread.
 * Replaces RansEncoder / RansDecoder (src/cpp/py_rans/py_rans.h:21-76, bind.cpp:14-40); the
 * bytes are identical to the reference coder's for the same symbols, tables and ec_parallel. */
int dcvc_rans_create(void** handle);
int dcvc_rans_destroy(void* handle);
/* cdf: [count, stride] int32, lengths: [count] (RansEncoder::set_cdf, py_rans.cpp:262-303) */
int dcvc_rans_set_cdf(void* handle, int index, const int32_t* cdf, const int32_t* lengths,
                      int count, int stride);
/* reset + set_entropy_coder_parallel (py_rans.cpp:251-260, 305-309) */
int dcvc_rans_encode_begin(void* handle, int ec_parallel);
/* encode_y: combined symbols (value << 8) + table index (py_rans.cpp:104-124) */
int dcvc_rans_encode_y(void* handle, const int16_t* sym, int n);
/* encode_z: table (i % ch) + cdf_offset (py_rans.cpp:126-146) */
int dcvc_rans_encode_z(void* handle, const int8_t* sym, int n, int cdf_offset, int ch);
/* flush + get_encoded_stream (py_rans.cpp:148-249); *data stays valid until the next call on
 * the handle */
int dcvc_rans_encode_finish(void* handle, const uint8_t** data, size_t* size);
/* set_entropy_coder_parallel + set_stream (py_rans.cpp:412-492) */
int dcvc_rans_decode_begin(void* handle, const uint8_t* data, size_t size, int ec_parallel);
/* decode_z / decode_y + get_decoded_tensor_cpp (py_rans.cpp:314-366); segments are decoded in
 * the reverse order of encoding.  DCVC_CORRUPT_STREAM if a sub-stream runs out of bytes. */
int dcvc_rans_decode_z(void* handle, int n, int cdf_offset, int ch, int8_t* out);
int dcvc_rans_decode_y(void* handle, const uint8_t* idx, int n, int8_t* out);

/* The same coder on the GPU (no reference counterpart: the reference codes on CPU threads,
 * py_rans.cpp:96-102, 305-312).  Bytes are identical with dcvc_rans_* for the same symbols and
 * ec_parallel; the container fixes the parallelism at one thread per sub-stream, so a launch codes
 * up to 64 payloads (independent streams) with one warp each.  All pointers in a job are device
 * pointers; status receives 0 or 1 (table index out of range), 2 (buffer overflow), 3 (bad
 * container header), 4 (truncated or corrupt sub-stream), 5 (a symbol with zero probability in
 * its table). */
typedef struct {
    const int16_t* y;   /* y symbols, (value << 8) + table index */
    int n_y;
    const int8_t* z;    /* z symbols, table (i % z_ch) + z_offset */
    int n_z;
    int z_offset;
    int z_ch;
    int ecp;            /* ec_parallel, 1..8 */
    uint8_t* scratch;   /* dcvc_rans_gpu_scratch_bytes(n_y, n_z, ecp) bytes */
    uint8_t* out;       /* the payload (container) */
    int out_cap;
    int* out_size;
    int* status;
} dcvc_rans_gpu_enc_job;
typedef struct {
    const uint8_t* data; /* the payload */
    int size;
    int ecp;
    int n_z;
    int z_offset;
    int z_ch;
    int8_t* z_out;
    const uint8_t* y_idx; /* y table index per y symbol */
    int n_y;
    int8_t* y_out;
    int* status;
} dcvc_rans_gpu_dec_job;
/* A device copy of the tables of a dcvc_rans handle (both table sets must be set). */
int dcvc_rans_gpu_create(void* rans_handle, void** gpu_handle);
int dcvc_rans_gpu_destroy(void* gpu_handle);
size_t dcvc_rans_gpu_scratch_bytes(int n_y, int n_z, int ecp);
int dcvc_rans_gpu_encode(void* gpu_handle, const dcvc_rans_gpu_enc_job* jobs, int njobs,
                         void* stream);
int dcvc_rans_gpu_decode(void* gpu_handle, const dcvc_rans_gpu_dec_job* jobs, int njobs,
                         void* stream);

/* ------------------------------------------------------------------ HT-S chunk codec */

/* One handle = one video stream (its temporal context lives on the device inside the handle),
 * the counterpart of DMCHTSProxy (src/layers/extensions/inference/dmc_hts_proxy.h:215-355,
 * bind.cpp:26-31).  A handle is not re-entrant: one call at a time.  Work is ordered after the
 * work already queued on `stream` and the caller's stream waits for the call's GPU work. */
int dcvc_hts_create(void** handle);
int dcvc_hts_destroy(void* handle);
/* set_param(state_dict, skip_threshold) (dmc_hts_proxy.cpp:712-762): n named tensors of the
 * DMC state dict plus gaussian_encoder.{quantized_cdf,cdf_length} and
 * bit_estimator_z.{quantized_cdf,cdf_length}.  shapes: n x 4 int64 (first ndims[i] used);
 * dtypes: DCVC_F16/BF16/F32/I32/I64; on_device[i] != 0 if data[i] is device memory. */
int dcvc_hts_set_param(void* handle, int n, const char* const* names, const void* const* data,
                       const int64_t* shapes, const int* ndims, const int* dtypes,
                       const int* on_device, float skip_threshold);
/* add_ref_feature_from_frame (dmc_hts_proxy.cpp:492-502): frame = [height, width, 3] FP16
 * (a [1, 3, H, W] channels-last tensor), height and width multiples of 16.  Sizes the
 * per-resolution buffers. */
int dcvc_hts_add_ref_feature(void* handle, const void* frame, int height, int width,
                             int apply_adaptor, void* stream);
/* compress (dmc_hts_proxy.cpp:504-585): x = [height, width, 24] FP16 (8 frames, channels
 * last); height + pad_b, width + pad_r must equal the reference frame size.  On success *bytes
 * (valid until the next call on the handle) holds the MLCodec rANS payload and *ec_parallel
 * its sub-stream count. */
int dcvc_hts_compress(void* handle, const void* x, int height, int width, int qp, int reset,
                      int pad_b, int pad_r, void* stream, const uint8_t** bytes, size_t* nbytes,
                      int* ec_parallel);
/* decompress (dmc_hts_proxy.cpp:587-710): height/width are the picture size of the stream.
 * frames receives 8 device pointers to [Hp, Wp, 3] FP16 reconstructions in [-0.5, 0.5], owned
 * by the handle and overwritten by the next call.  DCVC_CORRUPT_STREAM for a payload that does
 * not decode. */
int dcvc_hts_decompress(void* handle, const uint8_t* bytes, size_t nbytes, int qp, int height,
                        int width, int ec_parallel, int reset, void* stream, void** frames);
/* Read-only view of a per-stream device buffer (16-bit rows x cols, pitch ld; FP16 unless
 * dcvc_hts_buffer_dtype says BF16): "y_hat", "y_q", "memory", "ctx", "feature_p", "common",
 * "feature_i".  For inspection and tests; no counterpart in the reference. */
int dcvc_hts_buffer(void* handle, const char* name, const void** ptr, int* rows, int* cols,
                    int* ld);
/* symbols coded by the last call, kernels it enqueued, device bytes held by the handle */
int dcvc_hts_stats(void* handle, int* symbols, int* kernels, size_t* device_bytes);
/* Phase timing (off by default; enabling it adds two events per phase graph).  After a call,
 * dcvc_hts_timing writes up to `cap` values in milliseconds, -1 for a part the last call did not
 * run, and their number to *count: the device time of the phase graphs enc_analysis, enc_update,
 * enc_update (reset), dec_temporal, dec_temporal (memory), dec_hyper, dec_context,
 * dec_synthesis, then the host's time waiting for enc_analysis, rANS-encoding, decoding z,
 * waiting for dec_hyper and decoding y.  Every phase graph and host coding step is also an NVTX
 * range.  No counterpart in the reference. */
int dcvc_hts_set_timing(void* handle, int enable);
/* How many concurrent branches (1, 2 -- the default -- or 4) the 8-frame recon head of a decoded
 * chunk runs in, for HT-S codecs whose resolution is set after the call: with 2, frames 4..7 run
 * on a second stream (a parallel chain of the phase graph) with their own scratch buffers (about
 * 250 MB more at 1080p), and a 1080p chunk codes 1.2 % faster; 4 was measured slower than 2.
 * Outputs are the same in every case.  No counterpart in the reference. */
int dcvc_hts_recon_branches(int n);
int dcvc_hts_timing(void* handle, float* out, int cap, int* count);
/* Precision form of the analysis and synthesis transforms (encoder, decoder, recon head, feature
 * adaptors and extractor): DCVC_PRECISION_F16 (the reference's form, the default) or
 * DCVC_PRECISION_BF16 (BF16 activations and weights, FP32 accumulation) or DCVC_PRECISION_FP8 (the
 * BF16 form with every transform DepthConvBlock's quad GEMM, ffn.0, on E4M3 operands: weight rows
 * quantised with per-output-channel FP32 scales, activations by dcvc_quantize_fp8, FP32
 * accumulation, dcvc_conv1x1_f8).  The entropy-parameter
 * path stays FP16 with the same kernels on both sides, so symbols and CDF indexes round-trip
 * exactly in every form.  Takes effect at the next dcvc_hts_set_param; encoder and decoder
 * handles must use the same form.  No counterpart in the reference (FP16 only there,
 * test_video.py:25-27). */
int dcvc_hts_set_precision(void* handle, int precision);
/* The 16-bit format (DCVC_F16 or DCVC_BF16) of a buffer named as in dcvc_hts_buffer. */
int dcvc_hts_buffer_dtype(void* handle, const char* name, int* dtype);
/* handle takes the prepared parameters of source (set_param done there, same device) without a
 * copy: both read the same device buffers, which live until the last handle using them is
 * destroyed or re-parameterised.  The reference keeps one weight copy per proxy
 * (dmc_hts_proxy.cpp:712-762); no counterpart there. */
int dcvc_hts_share_params(void* handle, void* source);
/* Packed batches of n streams of one resolution (1 <= n <= 64): one handle holds the temporal
 * context of all n streams and runs every layer of the network as one launch over the n images
 * stacked along the rows; each stream has its own QP and its own payload (its bytes equal a
 * single-stream handle's on the same inputs).  add_ref_features seeds (and sizes) the n
 * streams from n frames [Hp, Wp, 3]; compress_batch takes n inputs [H, W, 24] and n QPs and
 * returns n payloads (pointer and size arrays owned by the handle, valid until its next call)
 * and n ec_parallel values; decompress_batch takes n payloads and returns 8 frames, each
 * [n * Hp, Wp, 3] FP16 with stream k in rows k * Hp .. (k + 1) * Hp - 1.  One reset flag covers
 * the batch.  The reference codes one stream per proxy call (dmc_hts_proxy.cpp:504-710); no
 * counterpart there. */
int dcvc_hts_add_ref_features(void* handle, const void* const* frames, int n, int height,
                              int width, int apply_adaptor, void* stream);
int dcvc_hts_compress_batch(void* handle, const void* const* xs, int n, int height, int width,
                            const int* qps, int reset, int pad_b, int pad_r, void* stream,
                            const uint8_t* const** bytes, const size_t** nbytes, int* ec_parallel);
int dcvc_hts_decompress_batch(void* handle, const uint8_t* const* bytes, const size_t* nbytes,
                              const int* qps, const int* ec_parallel, int n, int height, int width,
                              int reset, void* stream, void** frames);
/* A stream's temporal context outside the handle: its size in bytes at the handle's current
 * resolution (0 before the first add_ref_feature), and device-to-device copies of it on
 * `stream` (export also returns a flags word that import takes back); the handle's own work is
 * ordered after the copies.  A chunk server keeps one exported state per stream and runs each
 * chunk on any free handle of that resolution: import, compress or decompress, export.  The
 * layout is private to this build and valid only between handles of the same resolution and
 * precision form.  The reference keeps the context inside the proxy (dmc_hts_proxy.h:314-326);
 * no counterpart there. */
int dcvc_hts_state_bytes(void* handle, size_t* bytes);
int dcvc_hts_export_state(void* handle, void* dst, void* stream, int* flags);
int dcvc_hts_import_state(void* handle, const void* src, int flags, void* stream);

/* ------------------------------------------------------------------ HT-L chunk codec */

/* The counterpart of DMCHTLProxy (src/layers/extensions/inference/dmc_htl_proxy.h, bind.cpp:
 * 19-24), with the same arguments, ownership and stream rules as the dcvc_hts_* functions:
 * set_param (dmc_htl_proxy.cpp:917-967), add_ref_feature_from_frame (:583-593), compress
 * (:595-716; the payload holds the four checkerboard steps' y symbols in the order 3, 2, 1, 0,
 * then z), decompress (:718-915). */
int dcvc_htl_create(void** handle);
int dcvc_htl_destroy(void* handle);
int dcvc_htl_set_param(void* handle, int n, const char* const* names, const void* const* data,
                       const int64_t* shapes, const int* ndims, const int* dtypes,
                       const int* on_device, float skip_threshold);
int dcvc_htl_add_ref_feature(void* handle, const void* frame, int height, int width,
                             int apply_adaptor, void* stream);
int dcvc_htl_compress(void* handle, const void* x, int height, int width, int qp, int reset,
                      int pad_b, int pad_r, void* stream, const uint8_t** bytes, size_t* nbytes,
                      int* ec_parallel);
int dcvc_htl_decompress(void* handle, const uint8_t* bytes, size_t nbytes, int qp, int height,
                        int width, int ec_parallel, int reset, void* stream, void** frames);
/* Read-only view of a per-stream device buffer, as dcvc_hts_buffer; no counterpart in the
 * reference. */
int dcvc_htl_buffer(void* handle, const char* name, const void** ptr, int* rows, int* cols,
                    int* ld);
int dcvc_htl_stats(void* handle, int* symbols, int* kernels, size_t* device_bytes);

/* ------------------------------------------------------------------ low-delay (LD) codec */

/* The counterpart of DMCLDProxy (src/layers/extensions/inference/dmc_ld_proxy.h, bind.cpp:
 * 33-38), one frame per call, with the same arguments, ownership and stream rules as the
 * dcvc_hts_* functions: set_param (dmc_ld_proxy.cpp:595-637), add_ref_feature_from_frame
 * (:407-418), compress (:420-485; x = [height, width, 3] FP16, the payload holds the y symbols of
 * both checkerboard phases as one segment, then z), decompress (:487-593; *frame receives one
 * device frame [Hp, Wp, 3] FP16 owned by the handle, valid until the next call on it). */
int dcvc_ld_create(void** handle);
int dcvc_ld_destroy(void* handle);
int dcvc_ld_set_param(void* handle, int n, const char* const* names, const void* const* data,
                      const int64_t* shapes, const int* ndims, const int* dtypes,
                      const int* on_device, float skip_threshold);
int dcvc_ld_add_ref_feature(void* handle, const void* frame, int height, int width,
                            int apply_adaptor, void* stream);
int dcvc_ld_compress(void* handle, const void* x, int height, int width, int qp, int reset,
                     int pad_b, int pad_r, void* stream, const uint8_t** bytes, size_t* nbytes,
                     int* ec_parallel);
int dcvc_ld_decompress(void* handle, const uint8_t* bytes, size_t nbytes, int qp, int height,
                       int width, int ec_parallel, int reset, void* stream, void** frame);
/* Read-only view of a per-stream device buffer, as dcvc_hts_buffer ("temporal" adds the
 * temporal-prior parameters); no counterpart in the reference. */
int dcvc_ld_buffer(void* handle, const char* name, const void** ptr, int* rows, int* cols,
                   int* ld);
int dcvc_ld_stats(void* handle, int* symbols, int* kernels, size_t* device_bytes);

/* ------------------------------------------------------------------ intra (DMCI) codec */

/* One handle = one intra coder, the counterpart of DMCIProxy
 * (src/layers/extensions/inference/dmci_proxy.h:132-230, bind.cpp:13-17).  Same threading and
 * stream rules as the HT-S handle. */
int dcvc_intra_create(void** handle);
int dcvc_intra_destroy(void* handle);
/* set_param(state_dict, skip_threshold) (dmci_proxy.cpp:604-646): the DMCI state dict plus the
 * four CDF entries, passed as for dcvc_hts_set_param. */
int dcvc_intra_set_param(void* handle, int n, const char* const* names, const void* const* data,
                         const int64_t* shapes, const int* ndims, const int* dtypes,
                         const int* on_device, float skip_threshold);
/* compress(x, qp, padding_b, padding_r) (dmci_proxy.cpp:296-421): x = [height, width, 3] FP16
 * (a [1, 3, H, W] channels-last tensor); height + pad_b and width + pad_r multiples of 16.  On
 * success *bytes (valid until the next call on the handle) holds the rANS payload (the four
 * checkerboard steps' y symbols in the order 3, 2, 1, 0, then z), *ec_parallel its sub-stream
 * count and *x_hat a device pointer to the [height + pad_b, width + pad_r, 3] FP16
 * reconstruction, owned by the handle and overwritten by the next call. */
int dcvc_intra_compress(void* handle, const void* x, int height, int width, int qp, int pad_b,
                        int pad_r, void* stream, const uint8_t** bytes, size_t* nbytes,
                        int* ec_parallel, void** x_hat);
/* decompress(bit_stream, qp, height, width, ec_parallel) (dmci_proxy.cpp:423-602): *x_hat as
 * for compress, at the picture size rounded up to multiples of 16.  DCVC_CORRUPT_STREAM for a
 * payload that does not decode. */
int dcvc_intra_decompress(void* handle, const uint8_t* bytes, size_t nbytes, int qp, int height,
                          int width, int ec_parallel, void* stream, void** x_hat);
/* Read-only view of a device buffer: "y_hat", "y_q", "params", "z_hat".  No counterpart in the
 * reference. */
int dcvc_intra_buffer(void* handle, const char* name, const void** ptr, int* rows, int* cols,
                      int* ld);
int dcvc_intra_stats(void* handle, int* symbols, int* kernels, size_t* device_bytes);

#ifdef __cplusplus
}
#endif

#endif /* DCVC_B200_H */
