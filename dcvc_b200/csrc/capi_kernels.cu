// extern "C" kernel-level entry points (declared in include/dcvc_b200.h).
#include "errors.h"
#include "elementwise.cuh"
#include "ffn_sm100.cuh"
#include "gemm_sm100.cuh"
#include "quant_tables.h"

#include "../../include/dcvc_b200.h"

namespace dcvc {
cudaError_t gemm_autotune(int dtype, int epi, const GemmParams& shape, cudaStream_t stream,
                          int* best_bn, float* best_us);
void gemm_autotune_set_enabled(bool on);
int gemm_tuned_bn(int dtype, int epi, int M, int N, int K, int sub_w);
void gemm_tuning_clear();
cudaError_t gemm_sm100(int dtype, const void* A, int lda, const void* W, const GemmParams& p,
                       int epi, int bn, cudaStream_t stream);
}

using namespace dcvc;

extern "C" {

const char* dcvc_last_error(void) { return last_error(); }

int dcvc_abi_version(void) { return DCVC_ABI_VERSION; }

int dcvc_device_error(int* code, int clear)
{
    if (code == nullptr) {
        set_last_error("dcvc_device_error: null code pointer");
        return kInvalidArgument;
    }
    int* w = device_error_word();
    if (w == nullptr) {
        set_last_error("dcvc_device_error: no device error word");
        return kCudaError;
    }
    int st = cuda_status(cudaMemcpy(code, w, sizeof(int), cudaMemcpyDeviceToHost), "dcvc_device_error");
    if (st == kOk && clear) {
        st = cuda_status(cudaMemset(w, 0, sizeof(int)), "dcvc_device_error");
    }
    return st;
}

int dcvc_check_device_errors(void* stream)
{
    int* w = device_error_word();
    if (w == nullptr) {
        set_last_error("dcvc_check_device_errors: no device error word");
        return kCudaError;
    }
    int st = cuda_status(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)),
                         "dcvc_check_device_errors");
    if (st != kOk) {
        return st;
    }
    int code = 0;
    st = cuda_status(cudaMemcpy(&code, w, sizeof(int), cudaMemcpyDeviceToHost), "dcvc_check_device_errors");
    if (st != kOk) {
        return st;
    }
    if (code != 0) {
        cudaMemset(w, 0, sizeof(int));
        set_last_error("a kernel's bounded wait gave up (device error " + std::to_string(code) + ")");
        return kDeviceTimeout;
    }
    return kOk;
}

int dcvc_gemm_stream_form(int enable)
{
    gemm_set_stream_form(enable);
    return kOk;
}

int dcvc_gemm_pair_form(int enable)
{
    gemm_set_pair_form(enable != 0);
    return kOk;
}

int dcvc_dw_fusion(int enable)
{
    gemm_set_dw_fusion(enable != 0);
    return kOk;
}

int dcvc_gemm_inject_stall(int launches, long long wait_limit_cycles)
{
    if (launches > 0 && wait_limit_cycles <= 0) {
        set_last_error("dcvc_gemm_inject_stall: the wait limit must be positive");
        return kInvalidArgument;
    }
    gemm_inject_stall(launches, wait_limit_cycles);
    return kOk;
}

int dcvc_scale_index_table(uint8_t* lut)
{
    if (lut == nullptr) {
        set_last_error("dcvc_scale_index_table: null output");
        return kInvalidArgument;
    }
    scale_index_table(lut);
    return kOk;
}

int dcvc_conv1x1_f8(int epilogue, int M, int N, int K, const void* a, int lda, const void* w,
                    const float* wscale, const float* bias, void* out, int ldo, int block_n,
                    void* stream)
{
    GemmParams p{};
    p.M = M;
    p.N = N;
    p.K = K;
    p.bias = bias;
    p.wscale = wscale;
    p.out = out;
    p.ldo = ldo;
    p.err = device_error_word();
    cudaError_t e = gemm_sm100(kDtypeF8, a, lda, w, p, epilogue, block_n, static_cast<cudaStream_t>(stream));
    if (e == cudaErrorInvalidValue) {
        set_last_error("dcvc_conv1x1_f8: unsupported shape, pitch, alignment or epilogue");
        return kInvalidArgument;
    }
    return cuda_status(e, "dcvc_conv1x1_f8");
}

int dcvc_quantize_fp8(const void* src, int src_dtype, int lds, float inv_scale, void* dst, int ldd,
                      int M, int C, void* stream)
{
    cudaError_t e = launch_quantize_fp8(static_cast<const __half*>(src), src_dtype, lds, inv_scale,
                                        static_cast<uint8_t*>(dst), ldd, M, C,
                                        static_cast<cudaStream_t>(stream));
    if (e == cudaErrorInvalidValue) {
        set_last_error("dcvc_quantize_fp8: unsupported size, pitch, alignment or dtype");
        return kInvalidArgument;
    }
    return cuda_status(e, "dcvc_quantize_fp8");
}

int dcvc_scale_index_table_device(uint8_t* lut, void* stream)
{
    if (lut == nullptr) {
        set_last_error("dcvc_scale_index_table_device: null output");
        return kInvalidArgument;
    }
    return cuda_status(scale_index_table_device(lut, static_cast<cudaStream_t>(stream)),
                       "dcvc_scale_index_table_device");
}

int dcvc_conv1x1(int dtype, int epilogue, int M, int N, int K, const void* a, int lda,
                 const void* w, const float* bias, const void* res, int ldr, const void* res2,
                 int ldr2, const void* qscale, void* out, int ldo, int sub_w, int sub_cout,
                 int block_n, void* stream)
{
    if (dtype != DCVC_F16 && dtype != DCVC_BF16) {
        set_last_error("dcvc_conv1x1: dtype must be f16 or bf16");
        return kInvalidArgument;
    }
    GemmParams p{};
    p.M = M;
    p.N = N;
    p.K = K;
    p.bias = bias;
    p.res = res;
    p.ldr = ldr;
    p.res2 = res2;
    p.ldr2 = ldr2;
    p.qscale = qscale;
    p.out = out;
    p.ldo = ldo;
    p.sub_w = sub_w;
    p.sub_cout = sub_cout;
    p.err = device_error_word();
    cudaError_t e = gemm_sm100(dtype, a, lda, w, p, epilogue, block_n,
                               static_cast<cudaStream_t>(stream));
    if (e == cudaErrorInvalidValue) {
        set_last_error("dcvc_conv1x1: unsupported shape, pitch, alignment or epilogue");
        return kInvalidArgument;
    }
    return cuda_status(e, "dcvc_conv1x1");
}

int dcvc_gemm_autotune(int dtype, int epilogue, int M, int N, int K, int sub_w, int sub_cout,
                       void* stream, int* block_n, float* us)
{
    if (dtype != DCVC_F16 && dtype != DCVC_BF16) {
        set_last_error("dcvc_gemm_autotune: dtype must be f16 or bf16");
        return kInvalidArgument;
    }
    GemmParams p{};
    p.M = M;
    p.N = N;
    p.K = K;
    p.sub_w = sub_w;
    p.sub_cout = sub_cout;
    p.err = device_error_word();
    cudaError_t e = gemm_autotune(dtype, epilogue, p, static_cast<cudaStream_t>(stream), block_n, us);
    if (e == cudaErrorInvalidValue) {
        set_last_error("dcvc_gemm_autotune: no tile width supports this shape and epilogue");
        return kInvalidArgument;
    }
    if (e == cudaErrorStreamCaptureUnsupported) {
        set_last_error("dcvc_gemm_autotune: the stream is being captured");
        return kInvalidArgument;
    }
    return cuda_status(e, "dcvc_gemm_autotune");
}

int dcvc_gemm_autotune_enable(int on)
{
    gemm_autotune_set_enabled(on != 0);
    return kOk;
}

int dcvc_gemm_tuned(int dtype, int epilogue, int M, int N, int K, int sub_w, int* block_n)
{
    if (block_n == nullptr) {
        set_last_error("dcvc_gemm_tuned: null output");
        return kInvalidArgument;
    }
    *block_n = gemm_tuned_bn(dtype, epilogue, M, N, K, epilogue == kEpiSubpel ? sub_w : 0);
    return kOk;
}

int dcvc_gemm_tuning_clear(void)
{
    gemm_tuning_clear();
    return kOk;
}

int dcvc_conv_ffn(int M, int C, int cffn, const void* x, int ldx, const void* w1, const float* b1,
                  const void* w2, const float* b2, const void* qscale, void* out, int ldo,
                  int block_n, void* stream)
{
    FfnParams p{};
    p.M = M;
    p.C = C;
    p.cffn = cffn;
    p.b1 = b1;
    p.b2 = b2;
    p.qscale = qscale;
    p.out = out;
    p.ldo = ldo;
    p.err = device_error_word();
    p.block_n = block_n;
    cudaError_t e = ffn_sm100(x, ldx, w1, w2, p, static_cast<cudaStream_t>(stream));
    if (e == cudaErrorInvalidValue) {
        set_last_error("dcvc_conv_ffn: C must be a multiple of 256 and cffn 128 or 256, block_n "
                       "0, 128 or 256, pitches multiples of 8 elements, pointers 16-byte aligned");
        return kInvalidArgument;
    }
    return cuda_status(e, "dcvc_conv_ffn");
}

int dcvc_dwconv3x3(const void* x, int H, int W, int C, int ldx, const float* w, void* out, int ldo,
                   void* stream)
{
    if (x == nullptr || w == nullptr || out == nullptr || H <= 0 || W <= 0) {
        set_last_error("dcvc_dwconv3x3: bad arguments");
        return kInvalidArgument;
    }
    cudaError_t e = launch_dwconv3x3(static_cast<const __half*>(x), H, W, C, ldx, w,
                                     static_cast<__half*>(out), ldo, static_cast<cudaStream_t>(stream));
    if (e == cudaErrorInvalidValue) {
        set_last_error("dcvc_dwconv3x3: C, pitches and pointers must be multiples of 8 elements / 16 bytes");
        return kInvalidArgument;
    }
    return cuda_status(e, "dcvc_dwconv3x3");
}

int dcvc_dwconv3x3_ex(int dtype, const void* x, int H, int W, int img_h, int C, int ldx, const float* w,
                      void* out, int ldo, void* stream)
{
    if ((dtype != DCVC_F16 && dtype != DCVC_BF16) || x == nullptr || w == nullptr || out == nullptr ||
        H <= 0 || W <= 0 || img_h < 0) {
        set_last_error("dcvc_dwconv3x3_ex: bad arguments");
        return kInvalidArgument;
    }
    cudaError_t e = launch_dwconv3x3(static_cast<const __half*>(x), H, W, C, ldx, w, static_cast<__half*>(out),
                                     ldo, static_cast<cudaStream_t>(stream), dtype, img_h);
    if (e == cudaErrorInvalidValue) {
        set_last_error("dcvc_dwconv3x3_ex: C, pitches and pointers must be multiples of 8 elements / 16 bytes, "
                       "img_h must divide H");
        return kInvalidArgument;
    }
    return cuda_status(e, "dcvc_dwconv3x3_ex");
}

int dcvc_dw3x3_conv1x1_res(int dtype, int H, int W, int img_h, const void* x, int ldx,
                           const float* dw_weight, int K, const void* w, int N, const float* bias,
                           const void* res, int ldr, void* out, int ldo, void* stream)
{
    if ((dtype != DCVC_F16 && dtype != DCVC_BF16) || x == nullptr || dw_weight == nullptr || w == nullptr ||
        bias == nullptr || res == nullptr || out == nullptr || H <= 0 || W <= 0 || img_h < 0 ||
        static_cast<long long>(H) * W > (1LL << 30)) {
        set_last_error("dcvc_dw3x3_conv1x1_res: bad arguments");
        return kInvalidArgument;
    }
    GemmParams p{};
    p.M = H * W;
    p.N = N;
    p.K = K;
    p.bias = bias;
    p.res = res;
    p.ldr = ldr;
    p.out = out;
    p.ldo = ldo;
    p.err = device_error_word();
    p.dw_weight = dw_weight;
    p.dw_h = H;
    p.dw_w = W;
    p.dw_img_h = img_h > 0 ? img_h : H;
    cudaError_t e = gemm_sm100(dtype, x, ldx, w, p, kEpiBiasRes, kBlockNStream, static_cast<cudaStream_t>(stream));
    if (e == cudaErrorInvalidValue) {
        set_last_error("dcvc_dw3x3_conv1x1_res: unsupported shape, pitch or alignment (K a multiple of 64 "
                       "up to 256, N of 128, img_h dividing H)");
        return kInvalidArgument;
    }
    return cuda_status(e, "dcvc_dw3x3_conv1x1_res");
}

}  // extern "C"
