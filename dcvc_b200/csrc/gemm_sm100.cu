// tcgen05/TMEM persistent GEMM with fused 1x1-conv epilogues (see gemm_sm100.cuh).
#include "gemm_sm100.cuh"
#include "host_util.h"

#include <mutex>

namespace dcvc {

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;  // one 128-byte swizzle atom of 16-bit elements
constexpr int kThreads = 192;
// ~1 s at 2 GHz; a correct kernel never waits this long.
constexpr long long kWaitLimit = 2000000000LL;

template <typename T>
struct Pack2;
template <>
struct Pack2<__half> {
    static __device__ __forceinline__ uint32_t pack(float a, float b)
    {
        __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<uint32_t*>(&h);
    }
    static __device__ __forceinline__ float2 unpack(uint32_t u)
    {
        __half2 h = *reinterpret_cast<__half2*>(&u);
        return __half22float2(h);
    }
    static constexpr int kFormat = 0;
};
template <>
struct Pack2<__nv_bfloat16> {
    static __device__ __forceinline__ uint32_t pack(float a, float b)
    {
        __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<uint32_t*>(&h);
    }
    static __device__ __forceinline__ float2 unpack(uint32_t u)
    {
        __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&u);
        return __bfloat1622float2(h);
    }
    static constexpr int kFormat = 1;
};

template <int BN>
struct GemmSmem {
    static constexpr int kStages = BN >= 256 ? 4 : (BN >= 128 ? 6 : 8);
    static constexpr int kABytes = kBM * kBK * 2;
    static constexpr int kBBytes = BN * kBK * 2;
    static constexpr int kStageBytes = kABytes + kBBytes;
    static constexpr int kBarOffset = kStages * kStageBytes;
    // full[S], empty[S], tfull[2], tempty[2], drain, tmem slot, abort flag
    static constexpr int kBytes = kBarOffset + (2 * kStages + 5) * 8 + 16 + 1024;
    static constexpr int kTmemCols = 2 * BN;
};

template <typename T, int BN, int EPI>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_sm100_kernel(const __grid_constant__ CUtensorMap tmA,
                      const __grid_constant__ CUtensorMap tmB, const GemmParams p)
{
    using S = GemmSmem<BN>;
    constexpr int kStages = S::kStages;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem =
        reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::kBarOffset);
    uint64_t* empty = full + kStages;
    uint64_t* tfull = empty + kStages;
    uint64_t* tempty = tfull + 2;
    uint64_t* drain = tempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int num_m = (p.M + kBM - 1) / kBM;
    const int num_n = p.N / BN;
    const int num_tiles = num_m * num_n;
    const int kblocks = p.K / kBK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, S::kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int issued = 0;
            for (int tile = blockIdx.x; tile < num_tiles && !*abort_flag; tile += gridDim.x) {
                const int m0 = (tile % num_m) * kBM;
                const int n0 = (tile / num_m) * BN;
                for (int kb = 0; kb < kblocks; ++kb) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimit)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmProducerTimeout);
                        break;
                    }
                    mbar_arrive_expect_tx(&full[stage], S::kStageBytes);
                    uint8_t* sa = smem + stage * S::kStageBytes;
                    tma_load_2d(sa, &tmA, &full[stage], kb * kBK, m0);
                    tma_load_2d(sa + S::kABytes, &tmB, &full[stage], kb * kBK, n0);
                    ++issued;
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            if (*abort_flag) {
                // Let the copies this thread issued land before the CTA winds down.
                int n = issued < kStages ? issued : kStages;
                for (int i = 0; i < n; ++i) {
                    if (--stage < 0) {
                        stage = kStages - 1;
                        phase ^= 1;
                    }
                    mbar_wait_bounded(&full[stage], phase, kWaitLimit / 16);
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = make_idesc_f16(kBM, BN, Pack2<T>::kFormat);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            bool issued_any = false;
            for (int tile = blockIdx.x; tile < num_tiles && !*abort_flag; tile += gridDim.x) {
                if (!mbar_wait_bounded(&tempty[acc], acc_phase ^ 1, kWaitLimit)) {
                    *abort_flag = 1;
                    report_error(p.err, kErrGemmMmaTimeout);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + static_cast<uint32_t>(acc * BN);
                for (int kb = 0; kb < kblocks; ++kb) {
                    if (!mbar_wait_bounded(&full[stage], phase, kWaitLimit)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmMmaTimeout);
                        break;
                    }
                    tc_fence_after();
                    const uint8_t* sa = smem + stage * S::kStageBytes;
                    const uint64_t adesc = make_sw128_kmajor_desc(smem_u32(sa));
                    const uint64_t bdesc = make_sw128_kmajor_desc(smem_u32(sa + S::kABytes));
#pragma unroll
                    for (int k = 0; k < kBK / 16; ++k) {
                        // +32 bytes per K=16 step inside the swizzle atom (descriptor units of 16 B)
                        tc_mma_f16(d, adesc + 2 * k, bdesc + 2 * k, idesc, (kb | k) != 0 ? 1u : 0u);
                    }
                    issued_any = true;
                    tc_commit(&empty[stage]);
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                if (*abort_flag) {
                    break;
                }
                tc_commit(&tfull[acc]);
                acc ^= 1;
                if (acc == 0) {
                    acc_phase ^= 1;
                }
            }
            if (*abort_flag && issued_any) {
                // Drain this thread's outstanding MMAs before the columns are released.
                tc_commit(drain);
                mbar_wait_bounded(drain, 0, kWaitLimit / 16);
            }
        }
    } else {
        // ------------------------------------------------------------ epilogue warps (2..5)
        const int quad = warp & 3;  // TMEM lane quadrant this warp may access
        const int row = quad * 32 + lane;
        int acc = 0;
        uint32_t acc_phase = 0;
        using P = Pack2<T>;
        for (int tile = blockIdx.x; tile < num_tiles && !*abort_flag; tile += gridDim.x) {
            const int m0 = (tile % num_m) * kBM;
            const int n0 = (tile / num_m) * BN;
            if (!mbar_wait_bounded(&tfull[acc], acc_phase, kWaitLimit)) {
                *abort_flag = 1;
                report_error(p.err, kErrGemmEpilogueTimeout);
                break;
            }
            tc_fence_after();
            const int m = m0 + row;
            const bool live = m < p.M;
#pragma unroll 1
            for (int c = 0; c < BN / 32; ++c) {
                uint32_t r[32];
                tmem_ld_32x32b_x32(
                    tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + acc * BN + c * 32, r);
                tc_wait_ld();
                const int nc = n0 + c * 32;
                float v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    v[j] = __uint_as_float(r[j]);
                }
                if constexpr (EPI != kEpiSubpel) {
                    const float4* b4 = reinterpret_cast<const float4*>(p.bias + nc);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const float4 b = __ldg(b4 + j);
                        v[4 * j + 0] += b.x;
                        v[4 * j + 1] += b.y;
                        v[4 * j + 2] += b.z;
                        v[4 * j + 3] += b.w;
                    }
                }
                if constexpr (EPI == kEpiQuad) {
                    uint32_t o[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        float s0 = wsilu(v[8 * i + 0]) + wsilu(v[8 * i + 1]) + wsilu(v[8 * i + 2]) +
                                   wsilu(v[8 * i + 3]);
                        float s1 = wsilu(v[8 * i + 4]) + wsilu(v[8 * i + 5]) + wsilu(v[8 * i + 6]) +
                                   wsilu(v[8 * i + 7]);
                        o[i] = P::pack(s0, s1);
                    }
                    if (live) {
                        T* dst = reinterpret_cast<T*>(p.out) + static_cast<size_t>(m) * p.ldo + nc / 4;
                        *reinterpret_cast<uint4*>(dst) = make_uint4(o[0], o[1], o[2], o[3]);
                    }
                    continue;
                }
                if constexpr (EPI == kEpiBiasWsilu) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        v[j] = wsilu(v[j]);
                    }
                }
                if constexpr (EPI == kEpiBiasRes || EPI == kEpiBiasResQ || EPI == kEpiBiasRes2) {
                    if (live) {
                        const uint4* rs = reinterpret_cast<const uint4*>(
                            reinterpret_cast<const T*>(p.res) + static_cast<size_t>(m) * p.ldr + nc);
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const uint4 u = rs[j];
                            const float2 a = P::unpack(u.x), b = P::unpack(u.y),
                                         cc = P::unpack(u.z), d = P::unpack(u.w);
                            v[8 * j + 0] += a.x;
                            v[8 * j + 1] += a.y;
                            v[8 * j + 2] += b.x;
                            v[8 * j + 3] += b.y;
                            v[8 * j + 4] += cc.x;
                            v[8 * j + 5] += cc.y;
                            v[8 * j + 6] += d.x;
                            v[8 * j + 7] += d.y;
                        }
                    }
                }
                if constexpr (EPI == kEpiBiasRes2) {
                    if (live) {
                        const uint4* rs = reinterpret_cast<const uint4*>(
                            reinterpret_cast<const T*>(p.res2) + static_cast<size_t>(m) * p.ldr2 + nc);
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const uint4 u = rs[j];
                            const float2 a = P::unpack(u.x), b = P::unpack(u.y),
                                         cc = P::unpack(u.z), d = P::unpack(u.w);
                            v[8 * j + 0] += a.x;
                            v[8 * j + 1] += a.y;
                            v[8 * j + 2] += b.x;
                            v[8 * j + 3] += b.y;
                            v[8 * j + 4] += cc.x;
                            v[8 * j + 5] += cc.y;
                            v[8 * j + 6] += d.x;
                            v[8 * j + 7] += d.y;
                        }
                    }
                }
                if constexpr (EPI == kEpiBiasResQ || EPI == kEpiBiasQ) {
                    const uint4* qs =
                        reinterpret_cast<const uint4*>(reinterpret_cast<const T*>(p.qscale) + nc);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const uint4 u = __ldg(qs + j);
                        const float2 a = P::unpack(u.x), b = P::unpack(u.y), cc = P::unpack(u.z),
                                     d = P::unpack(u.w);
                        v[8 * j + 0] *= a.x;
                        v[8 * j + 1] *= a.y;
                        v[8 * j + 2] *= b.x;
                        v[8 * j + 3] *= b.y;
                        v[8 * j + 4] *= cc.x;
                        v[8 * j + 5] *= cc.y;
                        v[8 * j + 6] *= d.x;
                        v[8 * j + 7] *= d.y;
                    }
                }
                if (live) {
                    T* dst;
                    if constexpr (EPI == kEpiSubpel) {
                        const int sub = nc / p.sub_cout;  // dy * 2 + dx
                        const int ch = nc - sub * p.sub_cout;
                        const int h = m / p.sub_w;
                        const int w = m - h * p.sub_w;
                        const size_t orow = static_cast<size_t>(2 * h + (sub >> 1)) * (2 * p.sub_w) +
                                            (2 * w + (sub & 1));
                        dst = reinterpret_cast<T*>(p.out) + orow * p.ldo + ch;
                    } else {
                        dst = reinterpret_cast<T*>(p.out) + static_cast<size_t>(m) * p.ldo + nc;
                    }
                    uint4* d4 = reinterpret_cast<uint4*>(dst);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        d4[j] = make_uint4(P::pack(v[8 * j + 0], v[8 * j + 1]),
                                           P::pack(v[8 * j + 2], v[8 * j + 3]),
                                           P::pack(v[8 * j + 4], v[8 * j + 5]),
                                           P::pack(v[8 * j + 6], v[8 * j + 7]));
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&tempty[acc]);
            }
            acc ^= 1;
            if (acc == 0) {
                acc_phase ^= 1;
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, S::kTmemCols);
    }
}

template <typename T, int BN, int EPI>
cudaError_t launch_one(const CUtensorMap& ta, const CUtensorMap& tb, const GemmParams& p,
                       cudaStream_t stream)
{
    using S = GemmSmem<BN>;
    auto kernel = gemm_sm100_kernel<T, BN, EPI>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&] {
        attr_err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kBytes);
    });
    if (attr_err != cudaSuccess) {
        return attr_err;
    }
    const int num_tiles = ((p.M + kBM - 1) / kBM) * (p.N / BN);
    const int grid = num_tiles < num_sms() ? num_tiles : num_sms();
    kernel<<<grid, kThreads, S::kBytes, stream>>>(ta, tb, p);
    return cudaGetLastError();
}

template <typename T, int BN>
cudaError_t dispatch_epi(int epi, const CUtensorMap& ta, const CUtensorMap& tb,
                         const GemmParams& p, cudaStream_t s)
{
    switch (epi) {
    case kEpiBias: return launch_one<T, BN, kEpiBias>(ta, tb, p, s);
    case kEpiBiasWsilu: return launch_one<T, BN, kEpiBiasWsilu>(ta, tb, p, s);
    case kEpiBiasRes: return launch_one<T, BN, kEpiBiasRes>(ta, tb, p, s);
    case kEpiBiasResQ: return launch_one<T, BN, kEpiBiasResQ>(ta, tb, p, s);
    case kEpiBiasRes2: return launch_one<T, BN, kEpiBiasRes2>(ta, tb, p, s);
    case kEpiQuad: return launch_one<T, BN, kEpiQuad>(ta, tb, p, s);
    case kEpiSubpel: return launch_one<T, BN, kEpiSubpel>(ta, tb, p, s);
    case kEpiBiasQ: return launch_one<T, BN, kEpiBiasQ>(ta, tb, p, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int gemm_pick_bn(int N, int epi, int sub_cout)
{
    int lim = (epi == kEpiSubpel) ? sub_cout : N;
    if (N % 256 == 0 && lim % 256 == 0) {
        return 256;
    }
    if (N % 128 == 0 && lim % 128 == 0) {
        return 128;
    }
    if (N % 64 == 0 && lim % 64 == 0) {
        return 64;
    }
    return 0;
}

// Host launcher.  A: [M, K] with row pitch lda (elements); W: [N, K] dense.  dtype 0 = f16,
// 1 = bf16.  Returns cudaSuccess or an error (shape/alignment problems -> cudaErrorInvalidValue).
cudaError_t gemm_sm100(int dtype, const void* A, int lda, const void* W, const GemmParams& p,
                       int epi, int bn, cudaStream_t stream)
{
    if (p.M <= 0 || p.N <= 0 || p.K <= 0 || p.K % kBK != 0 || lda % 8 != 0 ||
        (reinterpret_cast<uintptr_t>(A) & 15) != 0 || (reinterpret_cast<uintptr_t>(W) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(p.out) & 15) != 0 || p.ldo % 8 != 0) {
        return cudaErrorInvalidValue;
    }
    if (bn == 0) {
        bn = gemm_pick_bn(p.N, epi, p.sub_cout);
    }
    if (bn == 0 || p.N % bn != 0) {
        return cudaErrorInvalidValue;
    }
    if (epi != kEpiSubpel && p.bias == nullptr) {
        return cudaErrorInvalidValue;
    }
    if ((epi == kEpiBiasRes || epi == kEpiBiasResQ || epi == kEpiBiasRes2) &&
        (p.res == nullptr || p.ldr % 8 != 0)) {
        return cudaErrorInvalidValue;
    }
    if (epi == kEpiBiasRes2 && (p.res2 == nullptr || p.ldr2 % 8 != 0)) {
        return cudaErrorInvalidValue;
    }
    if ((epi == kEpiBiasResQ || epi == kEpiBiasQ) && p.qscale == nullptr) {
        return cudaErrorInvalidValue;
    }
    if (epi == kEpiQuad && (p.N % 4 != 0)) {
        return cudaErrorInvalidValue;
    }
    if (epi == kEpiSubpel && (p.sub_w <= 0 || p.sub_cout % bn != 0 || p.N != 4 * p.sub_cout ||
                              p.M % p.sub_w != 0)) {
        return cudaErrorInvalidValue;
    }
    const CUtensorMapDataType dt =
        dtype == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    CUtensorMap ta, tb;
    if (!make_tmap_2d(&ta, dt, A, p.K, p.M, static_cast<uint64_t>(lda) * 2, kBK, kBM) ||
        !make_tmap_2d(&tb, dt, W, p.K, p.N, static_cast<uint64_t>(p.K) * 2, kBK, bn)) {
        return cudaErrorInvalidValue;
    }
    if (dtype == 0) {
        switch (bn) {
        case 256: return dispatch_epi<__half, 256>(epi, ta, tb, p, stream);
        case 128: return dispatch_epi<__half, 128>(epi, ta, tb, p, stream);
        case 64: return dispatch_epi<__half, 64>(epi, ta, tb, p, stream);
        }
    } else {
        switch (bn) {
        case 256: return dispatch_epi<__nv_bfloat16, 256>(epi, ta, tb, p, stream);
        case 128: return dispatch_epi<__nv_bfloat16, 128>(epi, ta, tb, p, stream);
        case 64: return dispatch_epi<__nv_bfloat16, 64>(epi, ta, tb, p, stream);
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace dcvc
