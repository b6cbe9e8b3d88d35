#include "elementwise.cuh"

#include "common.cuh"
#include "host_util.h"

#include <cuda_fp8.h>

#include <algorithm>
#include <mutex>

namespace dcvc {

namespace {

constexpr int kThreads = 256;

inline int grid_for(long long work, int threads = kThreads)
{
    long long g = (work + threads - 1) / threads;
    long long cap = static_cast<long long>(num_sms()) * 16;
    if (g > cap) {
        g = cap;
    }
    return g < 1 ? 1 : static_cast<int>(g);
}

// FP16 ops as at::Half does them: FP32 op, one rounding to FP16.
__device__ __forceinline__ float h2f(__half h) { return __half2float(h); }
__device__ __forceinline__ __half f2h(float f) { return __float2half_rn(f); }
__device__ __forceinline__ __half hadd(__half a, __half b) { return f2h(__fadd_rn(h2f(a), h2f(b))); }
__device__ __forceinline__ __half hsub(__half a, __half b) { return f2h(__fsub_rn(h2f(a), h2f(b))); }
__device__ __forceinline__ __half hmul(__half a, __half b) { return f2h(__fmul_rn(h2f(a), h2f(b))); }
__device__ __forceinline__ __half hzero() { return __ushort_as_half(0); }

struct alignas(16) Vec8h {
    __half v[8];
};

__device__ __forceinline__ Vec8h ld8(const __half* p) { return *reinterpret_cast<const Vec8h*>(p); }
__device__ __forceinline__ void st8(__half* p, const Vec8h& v) { *reinterpret_cast<Vec8h*>(p) = v; }

// ------------------------------------------------------------------------------ layout

// 16-bit activation formats: FP16 (0) or BF16 (1); conversions round to nearest.
template <int DT>
struct Act;
template <>
struct Act<0> {
    using T = __half;
    static __device__ __forceinline__ float2 to2(uint32_t u)
    {
        return __half22float2(*reinterpret_cast<const __half2*>(&u));
    }
    static __device__ __forceinline__ uint32_t from2(float a, float b)
    {
        __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<uint32_t*>(&h);
    }
    static __device__ __forceinline__ float to(uint16_t u) { return __half2float(__ushort_as_half(u)); }
    static __device__ __forceinline__ uint16_t from(float f) { return __half_as_ushort(__float2half_rn(f)); }
};
template <>
struct Act<1> {
    using T = __nv_bfloat16;
    static __device__ __forceinline__ float2 to2(uint32_t u)
    {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u));
    }
    static __device__ __forceinline__ uint32_t from2(float a, float b)
    {
        __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<uint32_t*>(&h);
    }
    static __device__ __forceinline__ float to(uint16_t u) { return __bfloat162float(__ushort_as_bfloat16(u)); }
    static __device__ __forceinline__ uint16_t from(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }
};

template <int ODT>
__global__ void pad_unshuffle8_kernel(const __half* __restrict__ x, int H, int W, int C, int ldx,
                                      int H8, int W8, __half* __restrict__ out, int ldo)
{
    griddep_launch_dependents();
    griddep_wait();
    // one thread = 8 output channels c*64 + dy*8 + [0, 8) of one output pixel
    const long long vec_per_pix = static_cast<long long>(C) * 8;
    const long long total = static_cast<long long>(H8) * W8 * vec_per_pix;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long pix = i / vec_per_pix;
        const int v = static_cast<int>(i - pix * vec_per_pix);
        const int c = v >> 3;
        const int dy = v & 7;
        const int h8 = static_cast<int>(pix / W8);
        const int w8 = static_cast<int>(pix - static_cast<long long>(h8) * W8);
        const int sh = min(h8 * 8 + dy, H - 1);
        Vec8h o;
#pragma unroll
        for (int dx = 0; dx < 8; ++dx) {
            const int sw = min(w8 * 8 + dx, W - 1);
            o.v[dx] = x[(static_cast<long long>(sh) * W + sw) * ldx + c];
            if constexpr (ODT == 1) {  // the same values as BF16
                o.v[dx] = __ushort_as_half(Act<1>::from(__half2float(o.v[dx])));
            }
        }
        st8(out + pix * ldo + c * 64 + dy * 8, o);
    }
}

template <int IDT>
__global__ void shuffle8_clamp_kernel(const __half* __restrict__ in, int H8, int W8, int C, int ldi,
                                      __half* __restrict__ out)
{
    griddep_launch_dependents();
    griddep_wait();
    const int Wp = W8 * 8;
    const long long total = static_cast<long long>(H8) * 8 * Wp;
    const __half lo = __float2half_rn(-0.5f);
    const __half hi = __float2half_rn(0.5f);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(i / Wp);
        const int xx = static_cast<int>(i - static_cast<long long>(y) * Wp);
        const __half* src = in + (static_cast<long long>(y >> 3) * W8 + (xx >> 3)) * ldi +
                            (y & 7) * 8 + (xx & 7);
        for (int c = 0; c < C; ++c) {
            __half v = src[c * 64];
            if constexpr (IDT == 1) {  // BF16 input: clamp in FP32, one rounding to FP16
                const float f = Act<1>::to(__half_as_ushort(v));
                v = __float2half_rn(fminf(fmaxf(f, -0.5f), 0.5f));
            } else {
                v = __hmax(v, lo);
                v = __hmin(v, hi);
            }
            out[i * C + c] = v;
        }
    }
}

// The same for C = 3 (the reconstructions) with vector accesses: one thread per output row and group
// of 8 output pixels (one input pixel), three 16-byte loads (one per channel, the row's 8 values)
// and three 16-byte stores of the 8 interleaved pixels; the clamp is the same per element.
template <int IDT>
__global__ void shuffle8_clamp3_kernel(const __half* __restrict__ in, int H8, int W8, int ldi,
                                       __half* __restrict__ out)
{
    griddep_launch_dependents();
    griddep_wait();
    const long long groups = static_cast<long long>(H8) * 8 * W8;
    const __half lo = __float2half_rn(-0.5f);
    const __half hi = __float2half_rn(0.5f);
    for (long long g = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; g < groups;
         g += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(g / W8);
        const int w8 = static_cast<int>(g - static_cast<long long>(y) * W8);
        const __half* src = in + (static_cast<long long>(y >> 3) * W8 + w8) * ldi + (y & 7) * 8;
        Vec8h u[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            u[c] = ld8(src + c * 64);
        }
        Vec8h o[3];
#pragma unroll
        for (int dx = 0; dx < 8; ++dx) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                __half v = u[c].v[dx];
                if constexpr (IDT == 1) {  // BF16 input: clamp in FP32, one rounding to FP16
                    const float f = Act<1>::to(__half_as_ushort(v));
                    v = __float2half_rn(fminf(fmaxf(f, -0.5f), 0.5f));
                } else {
                    v = __hmax(v, lo);
                    v = __hmin(v, hi);
                }
                const int k = dx * 3 + c;  // pixel dx, channel c of the 24 outputs
                o[k >> 3].v[k & 7] = v;
            }
        }
        __half* dst = out + (static_cast<long long>(y) * W8 + w8) * 24;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            st8(dst + 8 * j, o[j]);
        }
    }
}

__global__ void space_to_depth2_kernel(const __half* __restrict__ x, int H, int W, int C, int ldx,
                                       __half* __restrict__ out)
{
    griddep_launch_dependents();
    griddep_wait();
    const int Ho = H / 2, Wo = W / 2;
    const int vecs = C / 8;
    const long long total = static_cast<long long>(Ho) * Wo * 4 * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long pix = i / (4 * vecs);
        const int r = static_cast<int>(i - pix * 4 * vecs);
        const int sub = r / vecs;
        const int v = r - sub * vecs;
        const int ho = static_cast<int>(pix / Wo);
        const int wo = static_cast<int>(pix - static_cast<long long>(ho) * Wo);
        const int h = 2 * ho + (sub >> 1);
        const int w = 2 * wo + (sub & 1);
        st8(out + pix * (4LL * C) + sub * C + v * 8,
            ld8(x + (static_cast<long long>(h) * W + w) * ldx + v * 8));
    }
}

template <int S>
__global__ void im2col3x3_kernel(const __half* __restrict__ x, int H, int W, int C, int ldx,
                                 __half* __restrict__ out)
{
    griddep_launch_dependents();
    griddep_wait();
    const int Ho = H / S, Wo = W / S;
    const int vecs = C / 8;
    const long long total = static_cast<long long>(Ho) * Wo * 9 * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long pix = i / (9 * vecs);
        const int r = static_cast<int>(i - pix * 9 * vecs);
        const int tap = r / vecs;
        const int v = r - tap * vecs;
        const int ho = static_cast<int>(pix / Wo);
        const int wo = static_cast<int>(pix - static_cast<long long>(ho) * Wo);
        const int h = S * ho + tap / 3 - 1;
        const int w = S * wo + tap % 3 - 1;
        Vec8h o;
        if (h >= 0 && h < H && w >= 0 && w < W) {
            o = ld8(x + (static_cast<long long>(h) * W + w) * ldx + v * 8);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                o.v[j] = hzero();
            }
        }
        st8(out + pix * (9LL * C) + tap * C + v * 8, o);
    }
}

__global__ void replicate_pad_kernel(const __half* __restrict__ x, int H, int W, int C, int ldx,
                                     int Hp, int Wp, __half* __restrict__ out)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(Hp) * Wp * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long pix = i / vecs;
        const int v = static_cast<int>(i - pix * vecs);
        const int h = static_cast<int>(pix / Wp);
        const int w = static_cast<int>(pix - static_cast<long long>(h) * Wp);
        const int sh = min(h, H - 1), sw = min(w, W - 1);
        st8(out + pix * C + v * 8, ld8(x + (static_cast<long long>(sh) * W + sw) * ldx + v * 8));
    }
}

__global__ void crop_kernel(const __half* __restrict__ x, int Wx, int ldx, int H, int W, int C,
                            __half* __restrict__ out, int ldo)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(H) * W * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long pix = i / vecs;
        const int v = static_cast<int>(i - pix * vecs);
        const int h = static_cast<int>(pix / W);
        const int w = static_cast<int>(pix - static_cast<long long>(h) * W);
        st8(out + pix * ldo + v * 8, ld8(x + (static_cast<long long>(h) * Wx + w) * ldx + v * 8));
    }
}

// ------------------------------------------------------------------------------ latents

__global__ void round_z_kernel(const __half* __restrict__ z, int n, __half* __restrict__ z_hat,
                               int8_t* __restrict__ z_i8)
{
    griddep_launch_dependents();
    griddep_wait();
    const __half lo = __float2half_rn(-64.f), hi = __float2half_rn(63.f);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        __half v = f2h(roundf(h2f(z[i])));
        v = __hmax(v, lo);
        v = __hmin(v, hi);
        z_hat[i] = v;
        z_i8[i] = static_cast<int8_t>(static_cast<int>(h2f(v)));
    }
}

__global__ void int8_to_half_kernel(const int8_t* __restrict__ x, int n, __half* __restrict__ out)
{
    griddep_launch_dependents();
    griddep_wait();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[i] = f2h(static_cast<float>(x[i]));
    }
}

template <int IDT>
__global__ void mul_channel_kernel(const __half* __restrict__ x, int M, int C, int ldx,
                                   const __half* __restrict__ q, __half* __restrict__ out, int ldo,
                                   int q_rows)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(M) * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        Vec8h a = ld8(x + m * ldx + v * 8);
        // q_rows > 0: stacked images, each with its own row of C factors
        const Vec8h b = ld8(q + (q_rows > 0 ? (m / q_rows) * C : 0) + v * 8);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            // a BF16 input value is exact in FP32; the product is rounded once to FP16
            const float av = IDT == 1 ? Act<1>::to(__half_as_ushort(a.v[j])) : h2f(a.v[j]);
            a.v[j] = f2h(__fmul_rn(av, h2f(b.v[j])));
        }
        st8(out + m * ldo + v * 8, a);
    }
}

__global__ void div_clamp_kernel(__half* __restrict__ y, int M, int C, int ldy,
                                 const __half* __restrict__ q, int ldq)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(M) * vecs;
    const __half half_ = __float2half_rn(0.5f);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        Vec8h a = ld8(y + m * ldy + v * 8);
        const Vec8h b = ld8(q + m * ldq + v * 8);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const __half qc = __hmax(b.v[j], half_);
            const __half r = f2h(__fdiv_rn(1.0f, h2f(qc)));
            a.v[j] = hmul(a.v[j], r);
        }
        st8(y + m * ldy + v * 8, a);
    }
}

// ------------------------------------------------------------------------------ quantisation

// Whether channel vector v (of `vecs`) at (h, w) is coded in mask phase `phase`: the 4-phase masks
// (get_mask_4x, common_model.py:175-195) or, with groups == 2, the 2-phase checkerboard
// (get_mask_2x, common_model.py:157-172: channel half g at the positions with h + w + g + phase
// even).
__device__ __forceinline__ bool mask_on(int groups, int phase, int h, int w, int v, int vecs)
{
    if (groups == 2) {
        return ((h + w + v / (vecs / 2) + phase) & 1) == 0;
    }
    return ((h & 1) * 2 + (w & 1)) == mask_position(phase, v / (vecs / 4));
}

template <int MODE>
__global__ void quantize_phase_kernel(int groups, int phase, const __half* __restrict__ y, int ldy,
                                      const __half* __restrict__ scales, int lds,
                                      const __half* __restrict__ means, int ldm,
                                      const __half* __restrict__ q_dec, int ldd, __half thr,
                                      __half* __restrict__ y_q, int ldq, __half* __restrict__ y_hat,
                                      int ldh, int H, int W, int C, int img_h)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(H) * W * vecs;
    const __half qmin = __float2half_rn(-128.f), qmax = __float2half_rn(127.f);
    const __half half_ = __float2half_rn(0.5f);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        const int h = static_cast<int>(m / W);
        const int w = static_cast<int>(m - static_cast<long long>(h) * W);
        // stacked images: the mask follows each image's own row parity
        const bool on = mask_on(groups, phase, h % img_h, w, v, vecs);
        const Vec8h yy = ld8(y + m * ldy + v * 8);
        const Vec8h ss = ld8(scales + m * lds + v * 8);
        const Vec8h mm = ld8(means + m * ldm + v * 8);
        Vec8h oq, oh, pq, ph, qd;
        if (MODE >= 1) {
            pq = ld8(y_q + m * ldq + v * 8);
            ph = ld8(y_hat + m * ldh + v * 8);
        }
        if (MODE >= 2) {
            qd = ld8(q_dec + m * ldd + v * 8);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const __half s_hat = on ? ss.v[j] : hzero();
            const __half m_hat = on ? mm.v[j] : hzero();
            __half res = hsub(yy.v[j], m_hat);
            res = on ? res : hzero();
            __half q = f2h(roundf(h2f(res)));
            q = __hgt(s_hat, thr) ? q : hzero();
            q = __hmax(__hmin(q, qmax), qmin);
            __half yh = hadd(q, m_hat);
            if (MODE == 0) {
                oq.v[j] = q;
                oh.v[j] = yh;
            } else {
                oq.v[j] = hadd(pq.v[j], q);
                yh = hadd(yh, ph.v[j]);
                if (MODE == 2) {
                    yh = hmul(yh, __hmax(qd.v[j], half_));
                } else if (MODE == 3) {
                    yh = hmul(yh, qd.v[j]);
                }
                oh.v[j] = yh;
            }
        }
        st8(y_q + m * ldq + v * 8, oq);
        st8(y_hat + m * ldh + v * 8, oh);
    }
}

template <int MODE>
__global__ void restore_phase_kernel(int groups, int phase, const __half* __restrict__ y_q, int ldq,
                                     const __half* __restrict__ means, int ldm,
                                     const __half* __restrict__ q_dec, int ldd,
                                     __half* __restrict__ y_hat, int ldh, int H, int W, int C,
                                     int img_h)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(H) * W * vecs;
    const __half half_ = __float2half_rn(0.5f);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        const int h = static_cast<int>(m / W);
        const int w = static_cast<int>(m - static_cast<long long>(h) * W);
        const bool on = mask_on(groups, phase, h % img_h, w, v, vecs);
        const Vec8h qq = ld8(y_q + m * ldq + v * 8);
        const Vec8h mm = ld8(means + m * ldm + v * 8);
        Vec8h prev, qd, o;
        if (MODE >= 1) {
            prev = ld8(y_hat + m * ldh + v * 8);
        }
        if (MODE == 2) {
            qd = ld8(q_dec + m * ldd + v * 8);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            __half t = hadd(qq.v[j], mm.v[j]);
            t = on ? t : hzero();
            if (MODE >= 1) {
                t = hadd(t, prev.v[j]);
            }
            if (MODE == 2) {
                t = hmul(t, __hmax(qd.v[j], half_));
            }
            o.v[j] = t;
        }
        st8(y_hat + m * ldh + v * 8, o);
    }
}

template <bool ENC>
__global__ void build_index_kernel(const __half* __restrict__ y_q, int ldq,
                                   const __half* __restrict__ scales, int lds, __half thr,
                                   const uint8_t* __restrict__ lut, int M, int C,
                                   int16_t* __restrict__ sym, uint8_t* __restrict__ idx_out,
                                   uint8_t* __restrict__ cond)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(M) * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        const Vec8h ss = ld8(scales + m * lds + v * 8);
        const long long n = m * C + v * 8;
        uint8_t cnd[8];
        uint8_t ix[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            ix[j] = __ldg(lut + __half_as_ushort(ss.v[j]));
            cnd[j] = __hgt(ss.v[j], thr) ? 1 : 0;
        }
        *reinterpret_cast<uint2*>(cond + n) =
            make_uint2(cnd[0] | (cnd[1] << 8) | (cnd[2] << 16) | (cnd[3] << 24),
                       cnd[4] | (cnd[5] << 8) | (cnd[6] << 16) | (cnd[7] << 24));
        if (ENC) {
            const Vec8h qq = ld8(y_q + m * ldq + v * 8);
            int16_t o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int qv = __half2int_rd(qq.v[j]);
                o[j] = static_cast<int16_t>(qv * 256 + ix[j]);
            }
            *reinterpret_cast<uint4*>(sym + n) = *reinterpret_cast<uint4*>(o);
        } else {
            *reinterpret_cast<uint2*>(idx_out + n) =
                make_uint2(ix[0] | (ix[1] << 8) | (ix[2] << 16) | (ix[3] << 24),
                           ix[4] | (ix[5] << 8) | (ix[6] << 16) | (ix[7] << 24));
        }
    }
}

// The active quarter of the channels at each 2x2 position in mask phase `phase`.
__device__ __forceinline__ int active_quarter(int phase, int h, int w)
{
    return ((h & 1) * 2 + (w & 1)) ^ mask_position(phase, 0);
}

// build_index_enc/dec over the active quarter of a mask phase (single_part_for_writing_4x /
// single_part_for_reading_4x + build_index_*, stream.cu:89-173, 896-962): for every pixel m and
// channel c of the quarter-width part (C/4 channels), scale = the masked quarters summed in FP16,
// ((s0*m0 + s1*m1) + s2*m2) + s3*m3, and y_q = the active quarter's value (the other quarters
// of the running y_q hold zeros at this pixel); output in NHWC order of the part (m * C/4 + c).
template <bool ENC>
__global__ void build_index_4x_kernel(int phase, const __half* __restrict__ y_q, int ldq,
                                      const __half* __restrict__ scales, int lds, __half thr,
                                      const uint8_t* __restrict__ lut, int H, int W, int C,
                                      int16_t* __restrict__ sym, uint8_t* __restrict__ idx_out,
                                      uint8_t* __restrict__ cond)
{
    griddep_launch_dependents();
    griddep_wait();
    const int Cq = C / 4;
    const int vecs = Cq / 8;
    const long long total = static_cast<long long>(H) * W * vecs;
    const __half one = __float2half_rn(1.f);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        const int h = static_cast<int>(m / W);
        const int w = static_cast<int>(m - static_cast<long long>(h) * W);
        const int qa = active_quarter(phase, h, w);
        Vec8h ss[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ss[q] = ld8(scales + m * lds + q * Cq + v * 8);
        }
        const long long n = m * Cq + v * 8;
        uint8_t cnd[8];
        uint8_t ix[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            __half acc = hmul(ss[0].v[j], qa == 0 ? one : hzero());
#pragma unroll
            for (int q = 1; q < 4; ++q) {
                acc = hadd(acc, hmul(ss[q].v[j], qa == q ? one : hzero()));
            }
            ix[j] = __ldg(lut + __half_as_ushort(acc));
            cnd[j] = __hgt(acc, thr) ? 1 : 0;
        }
        *reinterpret_cast<uint2*>(cond + n) =
            make_uint2(cnd[0] | (cnd[1] << 8) | (cnd[2] << 16) | (cnd[3] << 24),
                       cnd[4] | (cnd[5] << 8) | (cnd[6] << 16) | (cnd[7] << 24));
        if (ENC) {
            const Vec8h qq = ld8(y_q + m * ldq + qa * Cq + v * 8);
            int16_t o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int qv = __half2int_rd(qq.v[j]);
                o[j] = static_cast<int16_t>(qv * 256 + ix[j]);
            }
            *reinterpret_cast<uint4*>(sym + n) = *reinterpret_cast<uint4*>(o);
        } else {
            *reinterpret_cast<uint2*>(idx_out + n) =
                make_uint2(ix[0] | (ix[1] << 8) | (ix[2] << 16) | (ix[3] << 24),
                           ix[4] | (ix[5] << 8) | (ix[6] << 16) | (ix[7] << 24));
        }
    }
}

// restore_y_4x[_and_add_inplace] / restore_y_4x_add_and_multiply_broadcast (stream.cu:757-860)
// and add_and_multiply_with_clamp_min_inplace (stream.cu:40-76): t = part[m, c % (C/4)] + means[m, c] on
// the phase's active quarter, 0 elsewhere; MODE 0: y_hat = t; 1: y_hat = y_hat + t;
// 2: y_hat = (y_hat + t) * max(q[m, c], 0.5); 3: y_hat = (y_hat + t) * q[m, c] (ldq = 0: one row).
template <int MODE>
__global__ void restore_4x_kernel(int phase, const __half* __restrict__ part,
                                  const __half* __restrict__ means, int ldm,
                                  const __half* __restrict__ q, int ldq, __half* __restrict__ y_hat,
                                  int ldh, int H, int W, int C)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const int quarter_vecs = vecs / 4;
    const long long total = static_cast<long long>(H) * W * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        const int h = static_cast<int>(m / W);
        const int w = static_cast<int>(m - static_cast<long long>(h) * W);
        const bool on = ((h & 1) * 2 + (w & 1)) == mask_position(phase, v / quarter_vecs);
        const Vec8h pp = ld8(part + m * (C / 4) + (v % quarter_vecs) * 8);
        const Vec8h mm = ld8(means + m * ldm + v * 8);
        Vec8h prev, qd, o;
        if (MODE >= 1) {
            prev = ld8(y_hat + m * ldh + v * 8);
        }
        if (MODE >= 2) {
            qd = ld8(q + m * ldq + v * 8);
        }
        const __half half_ = __float2half_rn(0.5f);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            __half t = on ? hadd(pp.v[j], mm.v[j]) : hzero();
            if (MODE >= 1) {
                t = hadd(prev.v[j], t);
            }
            if (MODE == 2) {
                t = hmul(t, __hmax(qd.v[j], half_));
            } else if (MODE == 3) {
                t = hmul(t, qd.v[j]);
            }
            o.v[j] = t;
        }
        st8(y_hat + m * ldh + v * 8, o);
    }
}

// ------------------------------------------------------------------------------ compaction

constexpr int kCompactThreads = 1024;
constexpr int kCompactPer = 8;
constexpr int kCompactBlock = kCompactThreads * kCompactPer;

__device__ __forceinline__ int load_cond8(const uint8_t* cond, int base, int n, uint8_t (&c)[8])
{
    int cnt = 0;
    if (base + 8 <= n) {
        const uint2 u = *reinterpret_cast<const uint2*>(cond + base);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            c[j] = (u.x >> (8 * j)) & 0xff;
            c[4 + j] = (u.y >> (8 * j)) & 0xff;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c[j] = (base + j < n) ? cond[base + j] : 0;
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        cnt += c[j] != 0;
    }
    return cnt;
}

// Exclusive scan of one int per thread over a 1024-thread block; returns the block total.
__device__ __forceinline__ int block_exclusive_scan(int x, int* warp_sums, int& excl)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) {
            incl += t;
        }
    }
    if (lane == 31) {
        warp_sums[warp] = incl;
    }
    __syncthreads();
    if (warp == 0) {
        int ws = warp_sums[lane];
        int wi = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) {
                wi += t;
            }
        }
        warp_sums[lane] = wi - ws;  // exclusive per warp
        if (lane == 31) {
            warp_sums[32] = wi;
        }
    }
    __syncthreads();
    excl = warp_sums[warp] + incl - x;
    return warp_sums[32];
}

__global__ void __launch_bounds__(kCompactThreads) compact_count_kernel(const uint8_t* __restrict__ cond,
                                                                        int n, int* __restrict__ counts)
{
    griddep_launch_dependents();
    griddep_wait();
    __shared__ int ws[33];
    uint8_t c[8];
    const int base = blockIdx.x * kCompactBlock + threadIdx.x * kCompactPer;
    const int cnt = load_cond8(cond, base, n, c);
    int excl;
    const int tot = block_exclusive_scan(cnt, ws, excl);
    if (threadIdx.x == 0) {
        counts[blockIdx.x] = tot;
    }
}

// Sum of counts[0, b) by one warp; the caller's warp 0 broadcasts it through shared memory.
__device__ __forceinline__ int prefix_of_blocks(const int* counts, int b)
{
    int s = 0;
    for (int i = threadIdx.x & 31; i < b; i += 32) {
        s += counts[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;
}

template <typename T>
__global__ void __launch_bounds__(kCompactThreads)
    compact_scatter_kernel(const T* __restrict__ src, const uint8_t* __restrict__ cond, int n,
                           const int* __restrict__ counts, T* __restrict__ dst,
                           int* __restrict__ total)
{
    griddep_launch_dependents();
    griddep_wait();
    __shared__ int ws[33];
    __shared__ int block_off;
    if (threadIdx.x < 32) {
        const int s = prefix_of_blocks(counts, blockIdx.x);
        if (threadIdx.x == 0) {
            block_off = s;
            if (blockIdx.x == gridDim.x - 1) {
                *total = s + counts[blockIdx.x];
            }
        }
    }
    uint8_t c[8];
    const int base = blockIdx.x * kCompactBlock + threadIdx.x * kCompactPer;
    const int cnt = load_cond8(cond, base, n, c);
    int excl;
    block_exclusive_scan(cnt, ws, excl);  // contains __syncthreads, publishes block_off
    int pos = block_off + excl;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (c[j]) {
            dst[pos++] = src[base + j];
        }
    }
}

__global__ void __launch_bounds__(kCompactThreads)
    recover_kernel(const int8_t* __restrict__ dec, const uint8_t* __restrict__ cond,
                   const int* __restrict__ counts, int n, __half* __restrict__ out)
{
    griddep_launch_dependents();
    griddep_wait();
    __shared__ int ws[33];
    __shared__ int block_off;
    if (threadIdx.x < 32) {
        const int s = prefix_of_blocks(counts, blockIdx.x);
        if (threadIdx.x == 0) {
            block_off = s;
        }
    }
    uint8_t c[8];
    const int base = blockIdx.x * kCompactBlock + threadIdx.x * kCompactPer;
    const int cnt = load_cond8(cond, base, n, c);
    int excl;
    block_exclusive_scan(cnt, ws, excl);
    int pos = block_off + excl;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (base + j < n) {
            out[base + j] = c[j] ? f2h(static_cast<float>(dec[pos++])) : hzero();
        }
    }
}

// ------------------------------------------------------------------------------ depthwise

// Tiled depthwise 3x3: one CTA computes a kDwTH x kDwTW pixel tile for 64 channels.  The
// (kDwTH+2) x (kDwTW+2) halo tile is staged in shared memory by 16-byte asynchronous copies
// (cp.async, zero-filled outside the image), so all of a thread's loads are in flight at once.
// Each thread then owns one channel pair of kDwRows adjacent tile rows and slides a
// (kDwRows + 2) x 3 window of FP32 values along them: per column kDwRows + 2 four-byte shared
// loads feed all of its rows' outputs.
constexpr int kDwTH = 8;
constexpr int kDwTW = 32;
constexpr int kDwCV = 8;  // channel vectors (of 8 halves) per CTA = 64 channels
constexpr int kDwRows = 2;  // output rows per thread (1: 15.2 us, 2: 13.8 us, 4: 17.6 us at 1080p)
constexpr int kDwThreads = 32 * (kDwTH / kDwRows);  // 32 channel pairs x row groups
static_assert(kDwTH % kDwRows == 0, "row groups tile the CTA rows");

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src, int src_bytes)
{
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gmem_src),
                 "r"(src_bytes)
                 : "memory");
}

// CUT: the H rows hold images of img_h rows stacked on top of each other; a tap that reaches
// into the image above or below reads zero, as the padding of each image alone would.
template <int DT, bool CUT>
__global__ void __launch_bounds__(kDwThreads) dwconv3x3_kernel(const __half* __restrict__ x, int H,
                                                               int W, int C, int ldx,
                                                               const float* __restrict__ wt,
                                                               __half* __restrict__ out, int ldo,
                                                               int img_h)
{
    griddep_launch_dependents();
    griddep_wait();
    __shared__ Vec8h tile[kDwTH + 2][kDwTW + 2][kDwCV];
    const int c0 = blockIdx.x * kDwCV;  // first channel vector
    const int h0 = blockIdx.y * kDwTH;
    const int w0 = blockIdx.z * kDwTW;
    const int cvecs = C / 8;
    const int nv = min(kDwCV, cvecs - c0);
    constexpr int kLoads = (kDwTH + 2) * (kDwTW + 2) * kDwCV;
#pragma unroll 4
    for (int i = threadIdx.x; i < kLoads; i += kDwThreads) {
        const int v = i % kDwCV;
        const int pix = i / kDwCV;
        const int tx = pix % (kDwTW + 2);
        const int ty = pix / (kDwTW + 2);
        const int h = h0 + ty - 1, w = w0 + tx - 1;
        const bool in = v < nv && h >= 0 && h < H && w >= 0 && w < W;
        // out-of-image elements read 0 bytes from a valid address and are zero-filled
        const __half* src = in ? x + (static_cast<long long>(h) * W + w) * ldx + (c0 + v) * 8 : x;
        cp_async16(&tile[ty][tx][v], src, in ? 16 : 0);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    const int cp = threadIdx.x & 31;              // channel pair within the CTA's 64 channels
    const int ty = kDwRows * (threadIdx.x >> 5);  // first of the thread's tile rows
    const int ch = c0 * 8 + 2 * cp;         // first of the pair's two channels
    const bool live = 2 * cp < nv * 8;
    float2 wp[9];  // the pair's two weights per tap
    if (live) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            wp[k] = __ldg(reinterpret_cast<const float2*>(wt + k * C + ch));
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const int ha = h0 + ty;  // the thread's output rows: ha .. ha + kDwRows - 1
    if (!live || ha >= H) {
        return;
    }
    const uint32_t* t2 = reinterpret_cast<const uint32_t*>(&tile[0][0][0]);
    auto at = [&](int r, int c) { return Act<DT>::to2(t2[(r * (kDwTW + 2) + c) * (4 * kDwCV) + cp]); };
    bool cut_up[kDwRows], cut_dn[kDwRows];  // the row above / below output row o is another image's
#pragma unroll
    for (int o = 0; o < kDwRows; ++o) {
        cut_up[o] = CUT && (ha + o) % img_h == 0;
        cut_dn[o] = CUT && (ha + o + 1) % img_h == 0;
    }
    float2 win[kDwRows + 2][3];  // window rows ty .. ty + kDwRows + 1 (image rows ha - 1 ..)
#pragma unroll
    for (int r = 0; r < kDwRows + 2; ++r) {
        win[r][0] = at(ty + r, 0);
        win[r][1] = at(ty + r, 1);
    }
    __half* orow = out + static_cast<long long>(ha) * W * ldo + ch;
    const long long next_row = static_cast<long long>(W) * ldo;
#pragma unroll
    for (int tx = 0; tx < kDwTW; ++tx) {
#pragma unroll
        for (int r = 0; r < kDwRows + 2; ++r) {
            win[r][2] = at(ty + r, tx + 2);
        }
        // FP32 accumulation in the order ky, kx (d3x3_kernel.h:104-166); one packed FP32 FMA per
        // tap for the channel pair (each lane rounds as a scalar fmaf would)
        float2 acc[kDwRows];
#pragma unroll
        for (int o = 0; o < kDwRows; ++o) {
            acc[o] = make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
#pragma unroll
                for (int o = 0; o < kDwRows; ++o) {
                    float2 v = win[ky + o][kx];
                    if (CUT && ((ky == 0 && cut_up[o]) || (ky == 2 && cut_dn[o]))) {
                        v = make_float2(0.f, 0.f);
                    }
                    acc[o] = __ffma2_rn(v, wp[ky * 3 + kx], acc[o]);
                }
            }
        }
        const int w = w0 + tx;
        if (w < W) {
            __half* op = orow + static_cast<long long>(w) * ldo;
#pragma unroll
            for (int o = 0; o < kDwRows; ++o) {
                if (ha + o < H) {
                    *reinterpret_cast<uint32_t*>(op + o * next_row) = Act<DT>::from2(acc[o].x, acc[o].y);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kDwRows + 2; ++r) {
            win[r][0] = win[r][1];
            win[r][1] = win[r][2];
        }
    }
}

// dst[m, c] = src[m, c] converted between the 16-bit activation formats (round to nearest).
template <int SDT, int DDT>
__global__ void convert_kernel(const __half* __restrict__ src, int lds, __half* __restrict__ dst,
                               int ldd, int M, int C)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(M) * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        const uint4 a = *reinterpret_cast<const uint4*>(src + m * lds + v * 8);
        const float2 f0 = Act<SDT>::to2(a.x), f1 = Act<SDT>::to2(a.y);
        const float2 f2 = Act<SDT>::to2(a.z), f3 = Act<SDT>::to2(a.w);
        *reinterpret_cast<uint4*>(dst + m * ldd + v * 8) =
            make_uint4(Act<DDT>::from2(f0.x, f0.y), Act<DDT>::from2(f1.x, f1.y),
                       Act<DDT>::from2(f2.x, f2.y), Act<DDT>::from2(f3.x, f3.y));
    }
}

// dst[m, c] = E4M3(src[m, c] * inv_scale), saturating to +-448 (NaN stays NaN).
template <int SDT>
__global__ void quantize_fp8_kernel(const __half* __restrict__ src, int lds, float inv_scale,
                                    uint8_t* __restrict__ dst, int ldd, int M, int C)
{
    griddep_launch_dependents();
    griddep_wait();
    const int vecs = C / 8;
    const long long total = static_cast<long long>(M) * vecs;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / vecs;
        const int v = static_cast<int>(i - m * vecs);
        const uint4 a = *reinterpret_cast<const uint4*>(src + m * lds + v * 8);
        const uint32_t w[4] = {a.x, a.y, a.z, a.w};
        uint32_t o[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float2 f0 = Act<SDT>::to2(w[2 * j]);
            const float2 f1 = Act<SDT>::to2(w[2 * j + 1]);
            const __nv_fp8x2_storage_t lo = __nv_cvt_float2_to_fp8x2(
                make_float2(f0.x * inv_scale, f0.y * inv_scale), __NV_SATFINITE, __NV_E4M3);
            const __nv_fp8x2_storage_t hi = __nv_cvt_float2_to_fp8x2(
                make_float2(f1.x * inv_scale, f1.y * inv_scale), __NV_SATFINITE, __NV_E4M3);
            o[j] = static_cast<uint32_t>(lo) | (static_cast<uint32_t>(hi) << 16);
        }
        *reinterpret_cast<uint2*>(dst + m * ldd + v * 8) = make_uint2(o[0], o[1]);
    }
}

inline bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace

cudaError_t launch_quantize_fp8(const __half* src, int src_dtype, int lds, float inv_scale,
                                uint8_t* dst, int ldd, int M, int C, cudaStream_t s)
{
    if (M <= 0 || C % 8 || lds % 8 || ldd % 8 || !al16(src) ||
        (reinterpret_cast<uintptr_t>(dst) & 7) || (src_dtype != 0 && src_dtype != 1)) {
        return cudaErrorInvalidValue;
    }
    const dim3 g(grid_for(static_cast<long long>(M) * (C / 8)));
    if (src_dtype == 1) {
        launch_pdl(quantize_fp8_kernel<1>, g, dim3(kThreads), 0, s, src, lds, inv_scale, dst, ldd, M, C);
    } else {
        launch_pdl(quantize_fp8_kernel<0>, g, dim3(kThreads), 0, s, src, lds, inv_scale, dst, ldd, M, C);
    }
    return cudaGetLastError();
}

cudaError_t launch_pad_unshuffle8(const __half* x, int H, int W, int C, int ldx, int pad_b,
                                  int pad_r, __half* out, int ldo, cudaStream_t s, int out_dtype)
{
    if (H <= 0 || W <= 0 || (H + pad_b) % 8 || (W + pad_r) % 8 || pad_b < 0 || pad_r < 0 ||
        ldo % 8 || !al16(out) || (out_dtype != 0 && out_dtype != 1)) {
        return cudaErrorInvalidValue;
    }
    const int H8 = (H + pad_b) / 8, W8 = (W + pad_r) / 8;
    const dim3 g(grid_for(static_cast<long long>(H8) * W8 * C * 8));
    if (out_dtype == 1) {
        launch_pdl(pad_unshuffle8_kernel<1>, g, dim3(kThreads), 0, s, x, H, W, C, ldx, H8, W8, out, ldo);
    } else {
        launch_pdl(pad_unshuffle8_kernel<0>, g, dim3(kThreads), 0, s, x, H, W, C, ldx, H8, W8, out, ldo);
    }
    return cudaGetLastError();
}

cudaError_t launch_convert(const __half* src, int src_dtype, int lds, __half* dst, int dst_dtype,
                           int ldd, int M, int C, cudaStream_t s)
{
    if (M <= 0 || C % 8 || lds % 8 || ldd % 8 || !al16(src) || !al16(dst) ||
        (src_dtype != 0 && src_dtype != 1) || (dst_dtype != 0 && dst_dtype != 1)) {
        return cudaErrorInvalidValue;
    }
    const dim3 g(grid_for(static_cast<long long>(M) * (C / 8)));
    if (src_dtype == 0 && dst_dtype == 1) {
        launch_pdl(convert_kernel<0, 1>, g, dim3(kThreads), 0, s, src, lds, dst, ldd, M, C);
    } else if (src_dtype == 1 && dst_dtype == 0) {
        launch_pdl(convert_kernel<1, 0>, g, dim3(kThreads), 0, s, src, lds, dst, ldd, M, C);
    } else if (src_dtype == 0) {
        launch_pdl(convert_kernel<0, 0>, g, dim3(kThreads), 0, s, src, lds, dst, ldd, M, C);
    } else {
        launch_pdl(convert_kernel<1, 1>, g, dim3(kThreads), 0, s, src, lds, dst, ldd, M, C);
    }
    return cudaGetLastError();
}

cudaError_t launch_shuffle8_clamp(const __half* in, int H8, int W8, int C, int ldi, __half* out,
                                  cudaStream_t s, int in_dtype)
{
    if (H8 <= 0 || W8 <= 0 || C <= 0 || (in_dtype != 0 && in_dtype != 1)) {
        return cudaErrorInvalidValue;
    }
    if (C == 3 && ldi % 8 == 0 && ldi >= 192 && al16(in) && al16(out)) {
        const dim3 g3(grid_for(8LL * H8 * W8));
        if (in_dtype == 1) {
            launch_pdl(shuffle8_clamp3_kernel<1>, g3, dim3(kThreads), 0, s, in, H8, W8, ldi, out);
        } else {
            launch_pdl(shuffle8_clamp3_kernel<0>, g3, dim3(kThreads), 0, s, in, H8, W8, ldi, out);
        }
        return cudaGetLastError();
    }
    const dim3 g(grid_for(64LL * H8 * W8));
    if (in_dtype == 1) {
        launch_pdl(shuffle8_clamp_kernel<1>, g, dim3(kThreads), 0, s, in, H8, W8, C, ldi, out);
    } else {
        launch_pdl(shuffle8_clamp_kernel<0>, g, dim3(kThreads), 0, s, in, H8, W8, C, ldi, out);
    }
    return cudaGetLastError();
}

cudaError_t launch_space_to_depth2(const __half* x, int H, int W, int C, int ldx, __half* out,
                                   cudaStream_t s)
{
    if (H % 2 || W % 2 || C % 8 || ldx % 8 || !al16(x) || !al16(out)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(space_to_depth2_kernel, dim3(grid_for(static_cast<long long>(H / 2) * (W / 2) * C / 2)), dim3(kThreads), 0, s, x, H, W, C, ldx, out);
    return cudaGetLastError();
}

cudaError_t launch_im2col3x3s2(const __half* x, int H, int W, int C, int ldx, __half* out,
                               cudaStream_t s)
{
    if (H % 2 || W % 2 || C % 8 || ldx % 8 || !al16(x) || !al16(out)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(im2col3x3_kernel<2>, dim3(grid_for(static_cast<long long>(H / 2) * (W / 2) * 9 * (C / 8))), dim3(kThreads), 0, s, x, H, W, C, ldx, out);
    return cudaGetLastError();
}

cudaError_t launch_im2col3x3s1(const __half* x, int H, int W, int C, int ldx, __half* out,
                               cudaStream_t s)
{
    if (H <= 0 || W <= 0 || C % 8 || ldx % 8 || !al16(x) || !al16(out)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(im2col3x3_kernel<1>, dim3(grid_for(static_cast<long long>(H) * W * 9 * (C / 8))),
               dim3(kThreads), 0, s, x, H, W, C, ldx, out);
    return cudaGetLastError();
}

cudaError_t launch_replicate_pad(const __half* x, int H, int W, int C, int ldx, int pad_b,
                                 int pad_r, __half* out, cudaStream_t s)
{
    if (C % 8 || ldx % 8 || pad_b < 0 || pad_r < 0 || !al16(x) || !al16(out)) {
        return cudaErrorInvalidValue;
    }
    const int Hp = H + pad_b, Wp = W + pad_r;
    launch_pdl(replicate_pad_kernel, dim3(grid_for(static_cast<long long>(Hp) * Wp * (C / 8))), dim3(kThreads), 0, s, 
        x, H, W, C, ldx, Hp, Wp, out);
    return cudaGetLastError();
}

cudaError_t launch_crop(const __half* x, int Wx, int ldx, int H, int W, int C, __half* out,
                        int ldo, cudaStream_t s)
{
    if (C % 8 || ldx % 8 || ldo % 8 || W > Wx || !al16(x) || !al16(out)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(crop_kernel, dim3(grid_for(static_cast<long long>(H) * W * (C / 8))), dim3(kThreads), 0, s, 
        x, Wx, ldx, H, W, C, out, ldo);
    return cudaGetLastError();
}

cudaError_t launch_round_z(const __half* z, int n, __half* z_hat, int8_t* z_i8, cudaStream_t s)
{
    if (n <= 0) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(round_z_kernel, dim3(grid_for(n)), dim3(kThreads), 0, s, z, n, z_hat, z_i8);
    return cudaGetLastError();
}

cudaError_t launch_int8_to_half(const int8_t* x, int n, __half* out, cudaStream_t s)
{
    if (n <= 0) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(int8_to_half_kernel, dim3(grid_for(n)), dim3(kThreads), 0, s, x, n, out);
    return cudaGetLastError();
}

cudaError_t launch_mul_channel(const __half* x, int M, int C, int ldx, const __half* q,
                               __half* out, int ldo, cudaStream_t s, int in_dtype, int q_rows)
{
    if (C % 8 || ldx % 8 || ldo % 8 || !al16(x) || !al16(q) || !al16(out) ||
        (in_dtype != 0 && in_dtype != 1)) {
        return cudaErrorInvalidValue;
    }
    const dim3 g(grid_for(static_cast<long long>(M) * (C / 8)));
    if (in_dtype == 1) {
        launch_pdl(mul_channel_kernel<1>, g, dim3(kThreads), 0, s, x, M, C, ldx, q, out, ldo, q_rows);
    } else {
        launch_pdl(mul_channel_kernel<0>, g, dim3(kThreads), 0, s, x, M, C, ldx, q, out, ldo, q_rows);
    }
    return cudaGetLastError();
}

cudaError_t launch_div_clamp(__half* y, int M, int C, int ldy, const __half* q, int ldq,
                             cudaStream_t s)
{
    if (C % 8 || ldy % 8 || ldq % 8 || !al16(y) || !al16(q)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(div_clamp_kernel, dim3(grid_for(static_cast<long long>(M) * (C / 8))), dim3(kThreads), 0, s, y, M, C,
                                                                                          ldy, q, ldq);
    return cudaGetLastError();
}

cudaError_t launch_quantize_phase(int phase, int mode, const __half* y, int ldy,
                                  const __half* scales, int lds, const __half* means, int ldm,
                                  const __half* q_dec, int ldd, __half thr, __half* y_q,
                                  int ldq, __half* y_hat, int ldh, int H, int W, int C,
                                  cudaStream_t s, int groups, int img_h)
{
    img_h = img_h > 0 ? img_h : H;
    if (H % img_h) {
        return cudaErrorInvalidValue;
    }
    if ((groups != 2 && groups != 4) || phase < 0 || phase >= groups || C % (8 * groups) || (mode >= 2 && q_dec == nullptr) || mode < 0 ||
        mode > 3) {
        return cudaErrorInvalidValue;
    }
    const int g = grid_for(static_cast<long long>(H) * W * (C / 8));
    if (mode == 3) {
        launch_pdl(quantize_phase_kernel<3>, dim3(g), dim3(kThreads), 0, s, groups, phase, y, ldy, scales,
                   lds, means, ldm, q_dec, ldd, thr, y_q, ldq, y_hat, ldh, H, W, C, img_h);
    } else if (mode == 0) {
        launch_pdl(quantize_phase_kernel<0>, dim3(g), dim3(kThreads), 0, s, groups, phase, y, ldy, scales, lds, means, ldm,
                                                        q_dec, ldd, thr, y_q, ldq, y_hat, ldh, H,
                                                        W, C, img_h);
    } else if (mode == 1) {
        launch_pdl(quantize_phase_kernel<1>, dim3(g), dim3(kThreads), 0, s, groups, phase, y, ldy, scales, lds, means, ldm,
                                                        q_dec, ldd, thr, y_q, ldq, y_hat, ldh, H,
                                                        W, C, img_h);
    } else {
        launch_pdl(quantize_phase_kernel<2>, dim3(g), dim3(kThreads), 0, s, groups, phase, y, ldy, scales, lds, means, ldm,
                                                        q_dec, ldd, thr, y_q, ldq, y_hat, ldh, H,
                                                        W, C, img_h);
    }
    return cudaGetLastError();
}

cudaError_t launch_restore_phase(int phase, int mode, const __half* y_q, int ldq,
                                 const __half* means, int ldm, const __half* q_dec, int ldd,
                                 __half* y_hat, int ldh, int H, int W, int C, cudaStream_t s,
                                 int groups, int img_h)
{
    img_h = img_h > 0 ? img_h : H;
    if (H % img_h) {
        return cudaErrorInvalidValue;
    }
    if ((groups != 2 && groups != 4) || phase < 0 || phase >= groups || C % (8 * groups) || (mode == 2 && q_dec == nullptr) || mode < 0 ||
        mode > 2) {
        return cudaErrorInvalidValue;
    }
    const int g = grid_for(static_cast<long long>(H) * W * (C / 8));
    if (mode == 0) {
        launch_pdl(restore_phase_kernel<0>, dim3(g), dim3(kThreads), 0, s, groups, phase, y_q, ldq, means, ldm, q_dec, ldd,
                                                       y_hat, ldh, H, W, C, img_h);
    } else if (mode == 1) {
        launch_pdl(restore_phase_kernel<1>, dim3(g), dim3(kThreads), 0, s, groups, phase, y_q, ldq, means, ldm, q_dec, ldd,
                                                       y_hat, ldh, H, W, C, img_h);
    } else {
        launch_pdl(restore_phase_kernel<2>, dim3(g), dim3(kThreads), 0, s, groups, phase, y_q, ldq, means, ldm, q_dec, ldd,
                                                       y_hat, ldh, H, W, C, img_h);
    }
    return cudaGetLastError();
}

cudaError_t launch_build_index_enc(const __half* y_q, int ldq, const __half* scales, int lds,
                                   __half thr, const uint8_t* lut, int M, int C, int16_t* sym,
                                   uint8_t* cond, cudaStream_t s)
{
    if (C % 8 || !al16(sym) || (reinterpret_cast<uintptr_t>(cond) & 7)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(build_index_kernel<true>, dim3(grid_for(static_cast<long long>(M) * (C / 8))), dim3(kThreads), 0, s, 
        y_q, ldq, scales, lds, thr, lut, M, C, sym, nullptr, cond);
    return cudaGetLastError();
}

cudaError_t launch_build_index_dec(const __half* scales, int lds, __half thr,
                                   const uint8_t* lut, int M, int C, uint8_t* idx, uint8_t* cond,
                                   cudaStream_t s)
{
    if (C % 8 || (reinterpret_cast<uintptr_t>(idx) & 7) || (reinterpret_cast<uintptr_t>(cond) & 7)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(build_index_kernel<false>, dim3(grid_for(static_cast<long long>(M) * (C / 8))), dim3(kThreads), 0, s, 
        nullptr, 0, scales, lds, thr, lut, M, C, nullptr, idx, cond);
    return cudaGetLastError();
}

cudaError_t launch_build_index_enc_4x(int phase, const __half* y_q, int ldq,
                                      const __half* scales, int lds, __half thr,
                                      const uint8_t* lut, int H, int W, int C, int16_t* sym,
                                      uint8_t* cond, cudaStream_t s)
{
    if (phase < 0 || phase > 3 || C % 32 || ldq % 8 || lds % 8 || !al16(sym) ||
        (reinterpret_cast<uintptr_t>(cond) & 7)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(build_index_4x_kernel<true>, dim3(grid_for(static_cast<long long>(H) * W * (C / 32))),
               dim3(kThreads), 0, s, phase, y_q, ldq, scales, lds, thr, lut, H, W, C, sym, nullptr,
               cond);
    return cudaGetLastError();
}

cudaError_t launch_build_index_dec_4x(int phase, const __half* scales, int lds, __half thr,
                                      const uint8_t* lut, int H, int W, int C, uint8_t* idx,
                                      uint8_t* cond, cudaStream_t s)
{
    if (phase < 0 || phase > 3 || C % 32 || lds % 8 || (reinterpret_cast<uintptr_t>(idx) & 7) ||
        (reinterpret_cast<uintptr_t>(cond) & 7)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(build_index_4x_kernel<false>, dim3(grid_for(static_cast<long long>(H) * W * (C / 32))),
               dim3(kThreads), 0, s, phase, nullptr, 0, scales, lds, thr, lut, H, W, C, nullptr,
               idx, cond);
    return cudaGetLastError();
}

cudaError_t launch_restore_4x(int phase, int mode, const __half* part, const __half* means,
                              int ldm, const __half* q, int ldq, __half* y_hat, int ldh, int H,
                              int W, int C, cudaStream_t s)
{
    if (phase < 0 || phase > 3 || C % 32 || ldm % 8 || ldh % 8 || ldq % 8 || !al16(part) ||
        mode < 0 || mode > 3 || (mode >= 2 && q == nullptr)) {
        return cudaErrorInvalidValue;
    }
    const int g = grid_for(static_cast<long long>(H) * W * (C / 8));
    if (mode == 0) {
        launch_pdl(restore_4x_kernel<0>, dim3(g), dim3(kThreads), 0, s, phase, part, means, ldm, q,
                   ldq, y_hat, ldh, H, W, C);
    } else if (mode == 1) {
        launch_pdl(restore_4x_kernel<1>, dim3(g), dim3(kThreads), 0, s, phase, part, means, ldm, q,
                   ldq, y_hat, ldh, H, W, C);
    } else if (mode == 2) {
        launch_pdl(restore_4x_kernel<2>, dim3(g), dim3(kThreads), 0, s, phase, part, means, ldm, q,
                   ldq, y_hat, ldh, H, W, C);
    } else {
        launch_pdl(restore_4x_kernel<3>, dim3(g), dim3(kThreads), 0, s, phase, part, means, ldm, q,
                   ldq, y_hat, ldh, H, W, C);
    }
    return cudaGetLastError();
}

int compact_blocks(int n) { return (n + kCompactBlock - 1) / kCompactBlock; }

bool compact_args_ok(const void* src, int elem_bytes, const uint8_t* cond, int n, const void* dst,
                     const int* total, bool needs_block_counts, const int* block_counts)
{
    if (n <= 0 || (elem_bytes != 1 && elem_bytes != 2)) {
        return false;
    }
    if (src == nullptr || dst == nullptr || cond == nullptr || total == nullptr ||
        (needs_block_counts && block_counts == nullptr)) {
        return false;
    }
    // cond is read 8 bytes at a time; 2-byte elements are read and written as int16
    const uintptr_t c = reinterpret_cast<uintptr_t>(cond);
    const uintptr_t e = reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst);
    const uintptr_t t = reinterpret_cast<uintptr_t>(total) |
                        reinterpret_cast<uintptr_t>(needs_block_counts ? block_counts : nullptr);
    return (c & 7) == 0 && (elem_bytes == 1 || (e & 1) == 0) && (t & 3) == 0;
}

cudaError_t launch_compact(const void* src, int elem_bytes, const uint8_t* cond, int n,
                           int* block_counts, void* dst, int* total, cudaStream_t s)
{
    if (!compact_args_ok(src, elem_bytes, cond, n, dst, total, true, block_counts)) {
        return cudaErrorInvalidValue;
    }
    const int nb = compact_blocks(n);
    launch_pdl(compact_count_kernel, dim3(nb), dim3(kCompactThreads), 0, s, cond, n, block_counts);
    if (elem_bytes == 1) {
        launch_pdl(compact_scatter_kernel<uint8_t>, dim3(nb), dim3(kCompactThreads), 0, s, 
            static_cast<const uint8_t*>(src), cond, n, block_counts, static_cast<uint8_t*>(dst),
            total);
    } else {
        launch_pdl(compact_scatter_kernel<int16_t>, dim3(nb), dim3(kCompactThreads), 0, s, 
            static_cast<const int16_t*>(src), cond, n, block_counts, static_cast<int16_t*>(dst),
            total);
    }
    return cudaGetLastError();
}

cudaError_t launch_recover(const int8_t* dec, const uint8_t* cond, const int* block_counts, int n,
                           __half* out, cudaStream_t s)
{
    if (n <= 0 || dec == nullptr || out == nullptr || block_counts == nullptr || cond == nullptr ||
        (reinterpret_cast<uintptr_t>(cond) & 7) || (reinterpret_cast<uintptr_t>(out) & 1) ||
        (reinterpret_cast<uintptr_t>(block_counts) & 3)) {
        return cudaErrorInvalidValue;
    }
    launch_pdl(recover_kernel, dim3(compact_blocks(n)), dim3(kCompactThreads), 0, s, dec, cond, block_counts, n, out);
    return cudaGetLastError();
}

cudaError_t launch_dwconv3x3(const __half* x, int H, int W, int C, int ldx, const float* w,
                             __half* out, int ldo, cudaStream_t s, int dtype, int img_h)
{
    img_h = img_h > 0 ? img_h : H;
    if (C % 8 || ldx % 8 || ldo % 8 || !al16(x) || !al16(out) || !al16(w) ||
        (dtype != 0 && dtype != 1) || H % img_h) {
        return cudaErrorInvalidValue;
    }
    const dim3 grid((C / 8 + kDwCV - 1) / kDwCV, (H + kDwTH - 1) / kDwTH, (W + kDwTW - 1) / kDwTW);
    const bool cut = img_h < H;
    if (dtype == 1) {
        if (cut) {
            launch_pdl(dwconv3x3_kernel<1, true>, grid, dim3(kDwThreads), 0, s, x, H, W, C, ldx, w, out, ldo, img_h);
        } else {
            launch_pdl(dwconv3x3_kernel<1, false>, grid, dim3(kDwThreads), 0, s, x, H, W, C, ldx, w, out, ldo, img_h);
        }
    } else {
        if (cut) {
            launch_pdl(dwconv3x3_kernel<0, true>, grid, dim3(kDwThreads), 0, s, x, H, W, C, ldx, w, out, ldo, img_h);
        } else {
            launch_pdl(dwconv3x3_kernel<0, false>, grid, dim3(kDwThreads), 0, s, x, H, W, C, ldx, w, out, ldo, img_h);
        }
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------ counted copy

namespace {

constexpr int kCopyThreads = 256;

__global__ void __launch_bounds__(kCopyThreads) copy_counted_kernel(
    const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int elem_bytes,
    const int* __restrict__ count, int max_elems, int* __restrict__ count_out, bool vec)
{
    griddep_launch_dependents();
    griddep_wait();
    int n = max_elems;
    if (count != nullptr) {
        n = min(max(*count, 0), max_elems);
    }
    if (count_out != nullptr && blockIdx.x == 0 && threadIdx.x == 0) {
        *count_out = n;
    }
    const long long bytes = static_cast<long long>(n) * elem_bytes;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    const long long t0 = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    long long done = 0;
    if (vec) {
        const long long nv = bytes / 16;
        const uint4* s4 = reinterpret_cast<const uint4*>(src);
        uint4* d4 = reinterpret_cast<uint4*>(dst);
        for (long long i = t0; i < nv; i += stride) {
            d4[i] = s4[i];
        }
        done = nv * 16;
    }
    for (long long i = done + t0; i < bytes; i += stride) {
        dst[i] = src[i];
    }
}

}  // namespace

cudaError_t launch_copy_counted(const void* src, void* dst, int elem_bytes, const int* count,
                                int max_elems, int* count_out, cudaStream_t s)
{
    if (src == nullptr || dst == nullptr || elem_bytes < 1 || elem_bytes > 8 || max_elems < 0) {
        return cudaErrorInvalidValue;
    }
    const bool vec = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0;
    const long long bytes = static_cast<long long>(max_elems) * elem_bytes;
    const long long want = (bytes / 16 + kCopyThreads - 1) / kCopyThreads;
    const int blocks = static_cast<int>(std::max(1LL, std::min(want, 4LL * num_sms())));
    launch_pdl(copy_counted_kernel, dim3(blocks), dim3(kCopyThreads), 0, s,
               static_cast<const uint8_t*>(src), static_cast<uint8_t*>(dst), elem_bytes, count,
               max_elems, count_out, vec);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------ no-alloc compaction
//
// Allocation-free variant of launch_compact for callers that cannot allocate device memory.  The
// per-block counts live in this file-scope device array instead of a caller buffer: 16 KB, enough
// for kCompactNoAllocMaxBlocks blocks of 8192 elements (n <= 33,554,432).  Every GPU that loads the
// library holds the array until the process exits.  All calls share it and it keeps the last
// call's contents; each call's count kernel writes every entry its scatter kernel reads, so
// nothing needs clearing, but two calls whose kernels overlap on the GPU (different streams, no
// ordering) race on it.

constexpr int kCompactNoAllocMaxBlocks = 4096;
static __device__ __align__(256) int g_compact_block_counts[kCompactNoAllocMaxBlocks];

int compact_noalloc_max_elements() { return kCompactNoAllocMaxBlocks * kCompactBlock; }

// The host cannot use g_compact_block_counts as a device address: its device address is looked
// up once per device (with that device current) and cached together with the context it belongs
// to.  The lookup happens on the first call on each device, so that first call must not be made
// while a stream is being captured.  If the device's context is destroyed and re-created (an
// embedding caller's cudaDeviceReset), the next call sees a different current context and looks
// the address up again instead of using the stale one.
static void* current_context()
{
    using GetCtxFn = int (*)(void**);
    static GetCtxFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<GetCtxFn>(p);
        }
    });
    void* ctx = nullptr;
    if (fn == nullptr || fn(&ctx) != 0) {
        return nullptr;
    }
    return ctx;
}

static int* compact_noalloc_scratch(cudaError_t* err)
{
    static std::mutex mu;
    static int* addr[64] = {nullptr};
    static void* ctx_of[64] = {nullptr};
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) {
        return nullptr;
    }
    if (dev < 0 || dev >= 64) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    void* ctx = current_context();
    if (addr[dev] == nullptr || ctx == nullptr || ctx != ctx_of[dev]) {
        void* p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_compact_block_counts);
        if (*err != cudaSuccess) {
            return nullptr;
        }
        addr[dev] = static_cast<int*>(p);
        // the symbol lookup makes the device's primary context current if none was
        ctx_of[dev] = ctx != nullptr ? ctx : current_context();
    }
    return addr[dev];
}

cudaError_t launch_compact_noalloc(const void* src, int elem_bytes, const uint8_t* cond, int n,
                                   void* dst, int* total, cudaStream_t s)
{
    if (n > compact_noalloc_max_elements() ||
        !compact_args_ok(src, elem_bytes, cond, n, dst, total, false, nullptr)) {
        return cudaErrorInvalidValue;
    }
    cudaError_t err = cudaSuccess;
    int* counts = compact_noalloc_scratch(&err);
    if (counts == nullptr) {
        return err;
    }
    const int nb = compact_blocks(n);
    compact_count_kernel<<<nb, kCompactThreads, 0, s>>>(cond, n, counts);
    if (elem_bytes == 1) {
        compact_scatter_kernel<uint8_t><<<nb, kCompactThreads, 0, s>>>(
            static_cast<const uint8_t*>(src), cond, n, counts, static_cast<uint8_t*>(dst), total);
    } else {
        compact_scatter_kernel<int16_t><<<nb, kCompactThreads, 0, s>>>(
            static_cast<const int16_t*>(src), cond, n, counts, static_cast<int16_t*>(dst), total);
    }
    return cudaGetLastError();
}

}  // namespace dcvc
