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
 *   block_n: N tile (0 = choose); K must be a multiple of 64, lda/ldr/ldo multiples of 8. */
int dcvc_conv1x1(int dtype, int epilogue, int M, int N, int K, const void* a, int lda,
                 const void* w, const float* bias, const void* res, int ldr, const void* res2,
                 int ldr2, const void* qscale, void* out, int ldo, int sub_w, int sub_cout,
                 int block_n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DCVC_B200_H */
