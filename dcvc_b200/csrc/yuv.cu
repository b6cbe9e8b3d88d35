#include "yuv.cuh"

#include "common.cuh"
#include "host_util.h"

namespace dcvc {

namespace {

constexpr int kYuvThreads = 256;

struct FramePtrs {
    const __half* p[kYuvMaxFrames];
};

__device__ __forceinline__ __half sample_to_input(uint32_t v)
{
    // x.half() / 255.0 (PyTorch: FP32 product with the FP32 reciprocal, rounded to FP16; equal
    // to the rounded quotient for all 256 sample values), then - 0.5 rounded to FP16
    const __half a = __float2half_rn(static_cast<float>(v) * (1.0f / 255.0f));
    return __float2half_rn(__half2float(a) - 0.5f);
}

__global__ void __launch_bounds__(kYuvThreads) yuv420_to_input_kernel(
    const uint8_t* __restrict__ src, int frames, int H, int W, __half* __restrict__ out, int ldo,
    bool vec)
{
    griddep_launch_dependents();
    griddep_wait();
    const long long npix = static_cast<long long>(H) * W;
    const long long csz = npix / 4;
    const long long fsz = npix + 2 * csz;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < npix;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int h = static_cast<int>(i / W);
        const int w = static_cast<int>(i - static_cast<long long>(h) * W);
        const long long ci = static_cast<long long>(h >> 1) * (W >> 1) + (w >> 1);
        __align__(16) __half vals[3 * kYuvMaxFrames];
#pragma unroll
        for (int f = 0; f < kYuvMaxFrames; ++f) {
            if (f < frames) {
                const uint8_t* fr = src + f * fsz;
                vals[3 * f + 0] = sample_to_input(__ldg(fr + i));
                vals[3 * f + 1] = sample_to_input(__ldg(fr + npix + ci));
                vals[3 * f + 2] = sample_to_input(__ldg(fr + npix + csz + ci));
            }
        }
        __half* o = out + i * ldo;
        if (vec) {  // 3 * frames == 24, 16-byte aligned rows
            uint4* o4 = reinterpret_cast<uint4*>(o);
            const uint4* v4 = reinterpret_cast<const uint4*>(vals);
            o4[0] = v4[0];
            o4[1] = v4[1];
            o4[2] = v4[2];
        } else {
            for (int c = 0; c < 3 * frames; ++c) {
                o[c] = vals[c];
            }
        }
    }
}

__device__ __forceinline__ float plus_half(__half x)
{
    return __half2float(__float2half_rn(__half2float(x) + 0.5f));
}

__device__ __forceinline__ float scaled_clamped(float x)
{
    // FP16(x * 255) clamped to [0, 255]
    const float t = __half2float(__float2half_rn(x * 255.0f));
    return fminf(fmaxf(t, 0.0f), 255.0f);
}

__global__ void __launch_bounds__(kYuvThreads) frames_to_yuv420_kernel(
    FramePtrs frames, int H, int W, int Wp, int ldp, uint8_t* __restrict__ dst)
{
    griddep_launch_dependents();
    griddep_wait();
    const int f = blockIdx.y;
    const int Hc = H >> 1, Wc = W >> 1;
    const long long nc = static_cast<long long>(Hc) * Wc;
    const long long npix = static_cast<long long>(H) * W;
    const __half* x = frames.p[f];
    uint8_t* fr = dst + f * (npix + 2 * nc);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < nc;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int ci = static_cast<int>(i / Wc);
        const int cj = static_cast<int>(i - static_cast<long long>(ci) * Wc);
        float su = 0.0f, sv = 0.0f;
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int h = 2 * ci + dy, w = 2 * cj + dx;
                const __half* px = x + (static_cast<long long>(h) * Wp + w) * ldp;
                const float yv = scaled_clamped(plus_half(px[0]));
                fr[static_cast<long long>(h) * W + w] = static_cast<uint8_t>(rintf(yv));
                su += plus_half(px[1]);  // FP32 sum in row-major order, as avg_pool2d
                sv += plus_half(px[2]);
            }
        }
        const float u = scaled_clamped(__half2float(__float2half_rn(su / 4.0f)));
        const float v = scaled_clamped(__half2float(__float2half_rn(sv / 4.0f)));
        fr[npix + i] = static_cast<uint8_t>(u);  // .byte() truncates
        fr[npix + nc + i] = static_cast<uint8_t>(v);
    }
}

int yuv_grid(long long work)
{
    const long long b = (work + kYuvThreads - 1) / kYuvThreads;
    const long long cap = 8LL * num_sms();
    return static_cast<int>(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

cudaError_t launch_yuv420_to_input(const uint8_t* src, int frames, int H, int W, __half* out,
                                   int ldo, cudaStream_t s)
{
    if (src == nullptr || out == nullptr || frames < 1 || frames > kYuvMaxFrames || H <= 0 ||
        W <= 0 || H % 2 || W % 2 || ldo < 3 * frames) {
        return cudaErrorInvalidValue;
    }
    const bool vec = frames == kYuvMaxFrames && ldo % 8 == 0 &&
                     (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    return launch_pdl(yuv420_to_input_kernel, dim3(yuv_grid(static_cast<long long>(H) * W)),
                      dim3(kYuvThreads), 0, s, src, frames, H, W, out, ldo, vec);
}

cudaError_t launch_frames_to_yuv420(const __half* const* frames, int nframes, int H, int W, int Wp,
                                    int ldp, uint8_t* dst, cudaStream_t s)
{
    if (frames == nullptr || dst == nullptr || nframes < 1 || nframes > kYuvMaxFrames || H <= 0 ||
        W <= 0 || H % 2 || W % 2 || Wp < W || ldp < 3) {
        return cudaErrorInvalidValue;
    }
    FramePtrs fp{};
    for (int i = 0; i < nframes; ++i) {
        if (frames[i] == nullptr) {
            return cudaErrorInvalidValue;
        }
        fp.p[i] = frames[i];
    }
    const long long nc = static_cast<long long>(H / 2) * (W / 2);
    return launch_pdl(frames_to_yuv420_kernel, dim3(yuv_grid(nc), nframes), dim3(kYuvThreads), 0,
                      s, fp, H, W, Wp, ldp, dst);
}

}  // namespace dcvc
