// Elementwise, layout and quantisation kernels (NHWC, FP16) and their launchers.  The layout and
// depthwise kernels that the analysis / synthesis transforms use also take BF16 activations
// (dtype 1; dtype 0 is FP16); the quantisation and entropy-parameter kernels are FP16 only.
//
// Arithmetic follows the reference's FP16 kernels op for op (src/layers/extensions/inference/
// elementwise/stream.cu, cat_and_pad.cu, shuffle.cu): every FP16 op is computed in FP32 and
// rounded once to FP16, which is what at::Half arithmetic does, so a NumPy float16
// restatement reproduces the outputs bit for bit.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dcvc {

// Four-phase checkerboard masks of the spatial prior (src/models/common_model.py:175-195,
// dmc_hts_proxy.cpp:869-890): in phase p, channel quarter q is coded at the 2x2 position
// (h%2)*2 + (w%2) == q ^ kMaskPerm[p].
__host__ __device__ __forceinline__ int mask_position(int phase, int quarter)
{
    const int perm[4] = {0, 3, 2, 1};
    return quarter ^ perm[phase];
}

// pad_and_unshuffle_8 (cat_and_pad.cu:7-51) / pixel_unshuffle by 8 (shuffle.cu:134-185):
// out[h8, w8, c*64 + dy*8 + dx] = x[min(8h8+dy, H-1), min(8w8+dx, W-1), c].
// out_dtype 1 writes the same values as BF16 (the input is FP16).
cudaError_t launch_pad_unshuffle8(const __half* x, int H, int W, int C, int ldx, int pad_b,
                                  int pad_r, __half* out, int ldo, cudaStream_t s,
                                  int out_dtype = 0);

// dst[m, c] = E4M3(src[m, c] * inv_scale) (bytes), saturating to +-448; src FP16 (0) or BF16 (1);
// C % 8 == 0, ldd % 8 == 0.  The A operand of the FP8 GEMM form.
cudaError_t launch_quantize_fp8(const __half* src, int src_dtype, int lds, float inv_scale,
                                uint8_t* dst, int ldd, int M, int C, cudaStream_t s);

// dst[m, c] = src[m, c] converted between FP16 (0) and BF16 (1), rounded to nearest; C % 8 == 0.
cudaError_t launch_convert(const __half* src, int src_dtype, int lds, __half* dst, int dst_dtype,
                           int ldd, int M, int C, cudaStream_t s);

// pixel_shuffle_8 with clamp to [-0.5, 0.5] (shuffle.cu:40-131):
// out[y, x, c] = clamp(in[y/8, x/8, c*64 + (y%8)*8 + x%8]).  out is [8*H8, 8*W8, C] dense.
// in_dtype 1: BF16 input, clamped in FP32 and rounded once to the FP16 output.
cudaError_t launch_shuffle8_clamp(const __half* in, int H8, int W8, int C, int ldi, __half* out,
                                  cudaStream_t s, int in_dtype = 0);

// out[(h, w), (dy*2 + dx)*C + c] = x[2h+dy, 2w+dx, c]   (pixel_unshuffle(2) with the channel
// order permuted to (dy, dx, c); the stride-2 conv weight is permuted to match).
cudaError_t launch_space_to_depth2(const __half* x, int H, int W, int C, int ldx, __half* out,
                                   cudaStream_t s);

// out[(ho, wo), (ky*3 + kx)*C + c] = x[2ho+ky-1, 2wo+kx-1, c] (zero outside): the patches of a
// 3x3 stride-2 pad-1 convolution (conv_bias with kernel 3, conv_kernel.h:22-89).
cudaError_t launch_im2col3x3s2(const __half* x, int H, int W, int C, int ldx, __half* out,
                               cudaStream_t s);

// out[(h, w), (ky*3 + kx)*C + c] = x[h+ky-1, w+kx-1, c] (zero outside): the patches of a 3x3
// stride-1 pad-1 convolution (conv2d of the biased sub-pixel up-sampling, layers_proxy.cpp:269-276).
cudaError_t launch_im2col3x3s1(const __half* x, int H, int W, int C, int ldx, __half* out,
                               cudaStream_t s);

// replicate_pad (cat_and_pad.cu:53-84): out [H+pb, W+pr, C] dense.
cudaError_t launch_replicate_pad(const __half* x, int H, int W, int C, int ldx, int pad_b,
                                 int pad_r, __half* out, cudaStream_t s);

// slice (cat_and_pad.cu:86-110): out[h, w, :] = x[h, w, :] for h < H, w < W; x has width Wx.
cudaError_t launch_crop(const __half* x, int Wx, int ldx, int H, int W, int C, __half* out,
                        int ldo, cudaStream_t s);

// round_z (stream.cu:862-894): z_hat = clamp(round(z), -64, 63) as FP16 and int8.
cudaError_t launch_round_z(const __half* z, int n, __half* z_hat, int8_t* z_i8, cudaStream_t s);

// int8_to_dtype (stream.cu:454-482).
cudaError_t launch_int8_to_half(const int8_t* x, int n, __half* out, cudaStream_t s);

// multiply_with_broadcast (stream.cu:484-546): out[m, c] = x[m, c] * q[c].
// in_dtype 1: x is BF16 (q and out stay FP16; one rounding of the FP32 product).
// q_rows > 0: the M rows are images of q_rows rows each, image k scaled by q row k (q [n, C]).
cudaError_t launch_mul_channel(const __half* x, int M, int C, int ldx, const __half* q,
                               __half* out, int ldo, cudaStream_t s, int in_dtype = 0,
                               int q_rows = 0);

// divide_with_clamp_inplace (stream.cu:422-452): y <- y * rcp(max(q, 0.5)), the reciprocal
// rounded from FP32 1/q.
cudaError_t launch_div_clamp(__half* y, int M, int C, int ldy, const __half* q, int ldq,
                             cudaStream_t s);

// process_with_mask_no_scale[_add_inplace][_add_and_multiply_inplace] (stream.cu:548-683) for
// mask phase `phase` on an H x W grid (img_h > 0: images of img_h rows stacked vertically, each
// with its own mask rows).  mode 0: write y_q / y_hat; 1: accumulate;
// 2: accumulate and scale y_hat by max(q_dec, 0.5); 3: accumulate and scale y_hat by q_dec
// (add_and_multiply_broadcast, stream.cu:8-37: with ldd = 0, q_dec is one row of C scales).
// groups = 4: the 4-phase masks; groups = 2: the 2-phase checkerboard of the LD model
// (phase p codes channel half g where h + w + g + p is even).
cudaError_t launch_quantize_phase(int phase, int mode, const __half* y, int ldy,
                                  const __half* scales, int lds, const __half* means, int ldm,
                                  const __half* q_dec, int ldd, __half thr, __half* y_q,
                                  int ldq, __half* y_hat, int ldh, int H, int W, int C,
                                  cudaStream_t s, int groups = 4, int img_h = 0);

// restore_y[_and_add_inplace][_and_add_multiply_inplace] (stream.cu:685-760).
cudaError_t launch_restore_phase(int phase, int mode, const __half* y_q, int ldq,
                                 const __half* means, int ldm, const __half* q_dec, int ldd,
                                 __half* y_hat, int ldh, int H, int W, int C, cudaStream_t s,
                                 int groups = 4, int img_h = 0);

// build_index_enc (stream.cu:126-173): sym[m*C + c] = (q << 8) + idx, cond = scale > thr, in
// NHWC symbol order.  idx comes from the 65536-entry table `lut` indexed by the FP16 bits of the
// scale (see scale_index_table in quant_tables.cpp).
cudaError_t launch_build_index_enc(const __half* y_q, int ldq, const __half* scales, int lds,
                                   __half thr, const uint8_t* lut, int M, int C, int16_t* sym,
                                   uint8_t* cond, cudaStream_t s);

// build_index_dec (stream.cu:89-124).
cudaError_t launch_build_index_dec(const __half* scales, int lds, __half thr,
                                   const uint8_t* lut, int M, int C, uint8_t* idx, uint8_t* cond,
                                   cudaStream_t s);

// The intra model's per-step index building over the active quarter of mask phase `phase`
// (single_part_for_writing_4x / single_part_for_reading_4x + build_index_enc/dec,
// stream.cu:89-173, 896-962): outputs [H*W, C/4] in NHWC order of the quarter-width part.
cudaError_t launch_build_index_enc_4x(int phase, const __half* y_q, int ldq,
                                      const __half* scales, int lds, __half thr,
                                      const uint8_t* lut, int H, int W, int C, int16_t* sym,
                                      uint8_t* cond, cudaStream_t s);
cudaError_t launch_build_index_dec_4x(int phase, const __half* scales, int lds, __half thr,
                                      const uint8_t* lut, int H, int W, int C, uint8_t* idx,
                                      uint8_t* cond, cudaStream_t s);

// restore_y_4x* (stream.cu:757-860): part is the dense [H*W, C/4] FP16 step values; mode 0
// writes y_hat, 1 accumulates, 2 accumulates and multiplies by max(q, 0.5), 3 accumulates and
// multiplies by q; q is [H*W, C] with pitch ldq (0: one row of C scales for every pixel).
cudaError_t launch_restore_4x(int phase, int mode, const __half* part, const __half* means,
                              int ldm, const __half* q, int ldq, __half* y_hat, int ldh, int H,
                              int W, int C, cudaStream_t s);

// Order-preserving compaction of `src` (elem_bytes 1 or 2) under `cond` (conditional_index_part1,
// stream.cu:175-338).  block_counts needs compact_blocks(n) ints; *total (device) receives the
// number of kept elements.
int compact_blocks(int n);
// Host-side validation shared by the compaction launchers (no CUDA call): n > 0, elem_bytes 1 or
// 2, non-null pointers, cond 8-byte aligned, 2-byte elements 2-byte aligned, counters 4-byte
// aligned.  block_counts is checked only when the launcher takes one.
bool compact_args_ok(const void* src, int elem_bytes, const uint8_t* cond, int n, const void* dst,
                     const int* total, bool needs_block_counts, const int* block_counts);
cudaError_t launch_compact(const void* src, int elem_bytes, const uint8_t* cond, int n,
                           int* block_counts, void* dst, int* total, cudaStream_t s);

// Copies n = min(*count, max_elems) elements of elem_bytes each (n = max_elems when count is
// null) from src to dst, either of which may be mapped pinned host memory, and stores n in
// *count_out when it is non-null.  The codecs move their symbols, indexes and decoded values
// between the device and the host with it inside the phase graphs, on the SMs, so that a
// transfer is never queued behind another phase's kernels.
cudaError_t launch_copy_counted(const void* src, void* dst, int elem_bytes, const int* count,
                                int max_elems, int* count_out, cudaStream_t s);

// Allocation-free variant of launch_compact: the block counts live in a file-scope device array
// (n <= compact_noalloc_max_elements()); see elementwise.cu for the sharing rules.
int compact_noalloc_max_elements();
cudaError_t launch_compact_noalloc(const void* src, int elem_bytes, const uint8_t* cond, int n,
                                   void* dst, int* total, cudaStream_t s);

// conditional_recover_with_type_conversion (stream.cu:359-420): out[i] = cond[i] ? dec[rank(i)]
// : 0, using the block counts written by launch_compact over the same cond.
cudaError_t launch_recover(const int8_t* dec, const uint8_t* cond, const int* block_counts, int n,
                           __half* out, cudaStream_t s);

// Depthwise 3x3, pad 1, no bias (d3x3, cutlass/d3x3_kernel.h:104-166): FP32 accumulation in the
// order ky, kx.  w is FP32 [9][C] (tap-major).
// img_h (0: H): the H rows hold images of img_h rows stacked vertically, each padded on its own.
cudaError_t launch_dwconv3x3(const __half* x, int H, int W, int C, int ldx, const float* w,
                             __half* out, int ldo, cudaStream_t s, int dtype = 0, int img_h = 0);

}  // namespace dcvc
