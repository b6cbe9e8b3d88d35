// Lookup tables of the quantisation path.
#include "quant_tables.h"

#include <cuda_fp16.h>

#include <cmath>

namespace dcvc {

namespace {

float round_to_half(float x) { return __half2float(__float2half_rn(x)); }

}  // namespace

// Scale -> Gaussian CDF index, as the reference's scale_to_index (stream.cu:77-87 with the
// constants of def_const.h:6-12) evaluates it in FP16:
//   s = min(max(s, 0.11), 16); t = log(s) - LOG_SCALE_MIN; idx = floor(t * LOG_SCALE_STEP_RECIP)
// with every intermediate rounded to FP16.  log is the natural logarithm evaluated in double
// precision and rounded to FP32 and then FP16.  A NaN scale behaves like the minimum scale (as
// FP16 max does).  Entries are clamped to [0, 127] so every index names one of the 128 tables.
void scale_index_table(uint8_t* lut)
{
    const float smin = round_to_half(0.11f);
    const float smax = round_to_half(16.f);
    const float log_min = round_to_half(-2.2073f);
    const float step_recip = round_to_half(1.f / ((2.7726f - (-2.2073f)) / (128 - 1)));
    for (int h = 0; h < 65536; ++h) {
        __half_raw raw;
        raw.x = static_cast<unsigned short>(h);
        float s = __half2float(__half(raw));
        s = std::isnan(s) ? smin : (s > smin ? s : smin);
        s = s < smax ? s : smax;
        const float t = round_to_half(static_cast<float>(std::log(static_cast<double>(s))));
        const float u = round_to_half(t - log_min);
        const float v = round_to_half(u * step_recip);
        float f = std::floor(v);
        f = f < 0.f ? 0.f : (f > 127.f ? 127.f : f);
        lut[h] = static_cast<uint8_t>(f);
    }
}

namespace {

// One thread per FP16 bit pattern.  The reference evaluates scale_to_index on at::Half values in a
// build with --use_fast_math (src/layers/extensions/inference/setup.py nvcc flags):
//   scale = max(scale, scale_min); scale = min(scale, scale_max)   -> float max/min, exact in FP16
//   scale = log(scale) - log_scale_min    -> float log (the fast-math logarithm, __logf), float
//                                            subtraction, one rounding to FP16 on assignment
//   scale = scale * log_step_recip        -> at::Half product: FP32 product rounded to FP16
//   index = __half2uint_rd(scale)         -> to_uint8 (common_cu.h:181-184)
// with the constants of def_const.h:6-12 converted to FP16 as the kernel arguments are.  Entries
// are clamped to [0, 127] (a scale at the minimum gives a slightly negative index there, which
// only skipped symbols ever carry, since the skip threshold 0.15 lies above the minimum 0.11).
__global__ void scale_index_table_kernel(uint8_t* __restrict__ lut)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 65536) {
        return;
    }
    const float smin = __half2float(__float2half_rn(0.11f));
    const float smax = __half2float(__float2half_rn(16.f));
    const float log_min = __half2float(__float2half_rn(-2.2073f));
    const float step_recip = __half2float(__float2half_rn(1.f / ((2.7726f - (-2.2073f)) / (128 - 1))));
    __half_raw raw;
    raw.x = static_cast<unsigned short>(h);
    float s = __half2float(__half(raw));
    s = fmaxf(s, smin);  // NaN -> smin, as max(float, float) gives
    s = fminf(s, smax);
    const __half u = __float2half_rn(__logf(s) - log_min);
    const __half v = __float2half_rn(__half2float(u) * step_recip);
    const unsigned idx = __half2uint_rd(v);
    lut[h] = static_cast<uint8_t>(idx > 127u ? 127u : idx);
}

}  // namespace

cudaError_t scale_index_table_device(uint8_t* lut, cudaStream_t s)
{
    if (lut == nullptr) {
        return cudaErrorInvalidValue;
    }
    scale_index_table_kernel<<<65536 / 256, 256, 0, s>>>(lut);
    return cudaGetLastError();
}

}  // namespace dcvc
