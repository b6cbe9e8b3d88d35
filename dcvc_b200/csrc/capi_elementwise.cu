// extern "C" wrappers of the elementwise, layout and quantisation kernels (include/dcvc_b200.h).
#include "elementwise.cuh"
#include "errors.h"
#include "yuv.cuh"

#include "../../include/dcvc_b200.h"

using namespace dcvc;

namespace {

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }
inline const __half* CH(const void* p) { return static_cast<const __half*>(p); }
inline __half* MH(void* p) { return static_cast<__half*>(p); }

int wrap(cudaError_t e, const char* where)
{
    if (e == cudaErrorInvalidValue) {
        set_last_error(std::string(where) + ": unsupported size, pitch or alignment");
        return kInvalidArgument;
    }
    return cuda_status(e, where);
}

}  // namespace

extern "C" {

int dcvc_pad_unshuffle8(const void* x, int H, int W, int C, int ldx, int pad_b, int pad_r,
                        void* out, int ldo, void* stream)
{
    return wrap(launch_pad_unshuffle8(CH(x), H, W, C, ldx, pad_b, pad_r, MH(out), ldo, S(stream)),
                "dcvc_pad_unshuffle8");
}

int dcvc_shuffle8_clamp(const void* in, int H8, int W8, int C, int ldi, void* out, void* stream)
{
    return wrap(launch_shuffle8_clamp(CH(in), H8, W8, C, ldi, MH(out), S(stream)), "dcvc_shuffle8_clamp");
}

int dcvc_space_to_depth2(const void* x, int H, int W, int C, int ldx, void* out, void* stream)
{
    return wrap(launch_space_to_depth2(CH(x), H, W, C, ldx, MH(out), S(stream)), "dcvc_space_to_depth2");
}

int dcvc_im2col3x3s2(const void* x, int H, int W, int C, int ldx, void* out, void* stream)
{
    return wrap(launch_im2col3x3s2(CH(x), H, W, C, ldx, MH(out), S(stream)), "dcvc_im2col3x3s2");
}

int dcvc_replicate_pad(const void* x, int H, int W, int C, int ldx, int pad_b, int pad_r, void* out,
                       void* stream)
{
    return wrap(launch_replicate_pad(CH(x), H, W, C, ldx, pad_b, pad_r, MH(out), S(stream)),
                "dcvc_replicate_pad");
}

int dcvc_crop(const void* x, int Wx, int ldx, int H, int W, int C, void* out, int ldo, void* stream)
{
    return wrap(launch_crop(CH(x), Wx, ldx, H, W, C, MH(out), ldo, S(stream)), "dcvc_crop");
}

int dcvc_round_z(const void* z, int n, void* z_hat, int8_t* z_i8, void* stream)
{
    return wrap(launch_round_z(CH(z), n, MH(z_hat), z_i8, S(stream)), "dcvc_round_z");
}

int dcvc_int8_to_half(const int8_t* x, int n, void* out, void* stream)
{
    return wrap(launch_int8_to_half(x, n, MH(out), S(stream)), "dcvc_int8_to_half");
}

int dcvc_mul_channel(const void* x, int M, int C, int ldx, const void* q, void* out, int ldo,
                     void* stream)
{
    return wrap(launch_mul_channel(CH(x), M, C, ldx, CH(q), MH(out), ldo, S(stream)), "dcvc_mul_channel");
}

int dcvc_div_clamp(void* y, int M, int C, int ldy, const void* q, int ldq, void* stream)
{
    return wrap(launch_div_clamp(MH(y), M, C, ldy, CH(q), ldq, S(stream)), "dcvc_div_clamp");
}

int dcvc_quantize_phase(int phase, int mode, const void* y, int ldy, const void* scales, int lds,
                        const void* means, int ldm, const void* q_dec, int ldd, float thr, void* y_q,
                        int ldq, void* y_hat, int ldh, int H, int W, int C, void* stream)
{
    return wrap(launch_quantize_phase(phase, mode, CH(y), ldy, CH(scales), lds, CH(means), ldm,
                                      CH(q_dec), ldd, __float2half_rn(thr), MH(y_q), ldq, MH(y_hat),
                                      ldh, H, W, C, S(stream)),
                "dcvc_quantize_phase");
}

int dcvc_restore_phase(int phase, int mode, const void* y_q, int ldq, const void* means, int ldm,
                       const void* q_dec, int ldd, void* y_hat, int ldh, int H, int W, int C,
                       void* stream)
{
    return wrap(launch_restore_phase(phase, mode, CH(y_q), ldq, CH(means), ldm, CH(q_dec), ldd,
                                     MH(y_hat), ldh, H, W, C, S(stream)),
                "dcvc_restore_phase");
}

int dcvc_build_index(int encode, const void* y_q, int ldq, const void* scales, int lds, float thr,
                     const uint8_t* lut, int M, int C, int16_t* sym, uint8_t* idx, uint8_t* cond,
                     void* stream)
{
    if (encode) {
        return wrap(launch_build_index_enc(CH(y_q), ldq, CH(scales), lds, __float2half_rn(thr), lut,
                                           M, C, sym, cond, S(stream)),
                    "dcvc_build_index");
    }
    return wrap(launch_build_index_dec(CH(scales), lds, __float2half_rn(thr), lut, M, C, idx, cond,
                                       S(stream)),
                "dcvc_build_index");
}

int dcvc_compact_blocks(int n) { return compact_blocks(n); }

int dcvc_compact(const void* src, int elem_bytes, const uint8_t* cond, int n, int* block_counts,
                 void* dst, int* total, void* stream)
{
    return wrap(launch_compact(src, elem_bytes, cond, n, block_counts, dst, total, S(stream)),
                "dcvc_compact");
}

int dcvc_compact_noalloc(const void* src, int elem_bytes, const uint8_t* cond, int n, void* dst,
                         int* total, void* stream)
{
    if (n > compact_noalloc_max_elements()) {
        set_last_error("dcvc_compact_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                       std::to_string(compact_noalloc_max_elements()) +
                       " elements of the built-in scratch; use dcvc_compact with a caller buffer");
        return kInvalidArgument;
    }
    return wrap(launch_compact_noalloc(src, elem_bytes, cond, n, dst, total, S(stream)),
                "dcvc_compact_noalloc");
}

int dcvc_recover(const int8_t* dec, const uint8_t* cond, const int* block_counts, int n, void* out,
                 void* stream)
{
    return wrap(launch_recover(dec, cond, block_counts, n, MH(out), S(stream)), "dcvc_recover");
}

int dcvc_yuv420_to_input(const void* planes, int frames, int H, int W, void* out, int ldo,
                         void* stream)
{
    return wrap(launch_yuv420_to_input(static_cast<const uint8_t*>(planes), frames, H, W, MH(out),
                                       ldo, S(stream)),
                "dcvc_yuv420_to_input");
}

int dcvc_frames_to_yuv420(const void* const* frames, int nframes, int H, int W, int Wp, int ldp,
                          void* planes, void* stream)
{
    return wrap(launch_frames_to_yuv420(reinterpret_cast<const __half* const*>(frames), nframes, H,
                                        W, Wp, ldp, static_cast<uint8_t*>(planes), S(stream)),
                "dcvc_frames_to_yuv420");
}

}  // extern "C"
