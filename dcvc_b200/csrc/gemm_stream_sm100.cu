// Streaming form of the residual 1x1-conv GEMMs for sm_100a (conv1x1_bias_shortcut and
// conv1x1_bias_shortcut_with_quant; def_cutlass.h:10-34), for K <= 256.
//
// At K = 256 these GEMMs are bound by HBM: per output pixel they read 2*K bytes of A, 2*N of
// residual and write 2*N, against N*K MACs.  The tiled persistent kernel (gemm_sm100.cu) streams
// A and W through the same operand ring and re-reads W for every tile, and its residual ring is
// one tile deep, so a tile's epilogue waits a full memory latency for its residual.  This form
// is laid out for streaming instead:
//   * every CTA owns one 128-wide slice of the output channels and a contiguous range of rows
//     (a multiple of 32 rows, balanced over the CTAs of its slice), so all CTAs move the same
//     number of bytes; the last 128-row tile of a range may be partial (its extra rows are
//     computed and never stored);
//   * the CTA's W slice (128 x K) is loaded once and stays in shared memory, so the operand ring
//     carries only A (16 KB per stage, six stages);
//   * sixteen epilogue warps (four per TMEM lane quadrant, 32 columns each) keep a two-tile-deep
//     ring of residual boxes in flight, so a tile's residual lands while earlier tiles compute;
//   * the result is written over the residual in its slot and stored by TMA.
// Depthwise form (p.dw_weight set): A is the depthwise 3x3 convolution of the given input,
// computed in the kernel (DepthConvBlock: d3x3 followed by conv1x1_bias_shortcut,
// layers_proxy.cpp:81-82).  Four producer warps compute each 128-row x 64-channel A stage on the
// CUDA cores from three TMA-staged bands of input rows (the pixel row above, the row itself and
// the row below, 66 pixels each per 64-pixel half) and write it in the MMA's 128-byte-swizzled
// operand layout; the depthwise output never goes to memory.  The products are summed in FP32 in
// the order ky, kx and rounded once to the activation type, as the standalone depthwise kernel
// does, so A, and every output bit, equal those of the two-launch form.  Measured at 1080p (M =
// 32640, K = 256, N = 512) it is slower than the two launches (114.7 us against 14.3 + 18.3 us):
// each of the four channel slices recomputes the depthwise values of its rows, and with two band
// sets in shared memory the producers wait for every band's L2 latency.  The codecs therefore use
// it only when asked to (gemm_set_dw_fusion).
// One thread issues tcgen05.mma (M = 128, N = 128, K = 16) into a double-buffered FP32 TMEM
// accumulator.  Per output element the products are summed in the same order as in the tiled
// kernel and the epilogue applies bias, residual(s) and x q in the same order, so the outputs
// are bitwise those of gemm_sm100 at any tile width.
#include "gemm_sm100.cuh"
#include "host_util.h"

#include <cuda_fp8.h>

#include <cstring>
#include <mutex>

namespace dcvc {

namespace {

constexpr int kSBM = 128;                   // rows per MMA tile
constexpr int kSBN = 128;                   // output channels per CTA
constexpr int kSBK = 64;                    // one 128-byte swizzle atom of 16-bit elements
constexpr int kSMaxK = 256;                 // residual epilogues: W slice 128 x 256 x 2 B = 64 KB
constexpr int kSMaxKPlain = 512;            // bias / WSiLU epilogues: W slice up to 128 KB
constexpr int kSEpiWarps = 16;
constexpr int kSCols = kSBN / 4;            // accumulator columns per epilogue warp (32)
constexpr int kSBoxBytes = 32 * kSCols * 2; // 32 rows x 32 columns of 16-bit values: 2 KB
// residual ring depth per warp, in tiles, and A stages of the residual epilogues (compile-time
// overrides exist for tuning builds; the library uses the defaults)
#ifndef DCVC_STREAM_RES_SLOTS
#define DCVC_STREAM_RES_SLOTS 2
#endif
#ifndef DCVC_STREAM_STAGES
#define DCVC_STREAM_STAGES 6
#endif
constexpr int kSResSlots = DCVC_STREAM_RES_SLOTS;
constexpr int kSStages = DCVC_STREAM_STAGES;
constexpr int kSStagesPlain = 4;            // bias / WSiLU: a W slice twice as large leaves four

__host__ __device__ constexpr bool stream_has_res(int epi) { return epi == kEpiBiasRes || epi == kEpiBiasResQ; }
constexpr int kSABytes = kSBM * kSBK * 2;   // 16 KB
constexpr long long kSWaitLimit = 2000000000LL;  // ~1 s at 2 GHz; a correct kernel never waits this long
// depthwise form
constexpr int kDwProdWarps = 4;
constexpr int kDwStages = 2;                        // A stages: the producers, not the MMA, set the pace
constexpr int kDwSubPx = 64;                        // output pixels per producer step (half a stage)
constexpr int kDwPxPerWarp = kDwSubPx / kDwProdWarps;  // 16 consecutive pixels per warp
constexpr int kDwBandRows = kDwSubPx + 2;           // input pixels per band: one more on each side
constexpr int kDwBandBytes = kDwBandRows * kSBK * 2;  // 8448
constexpr int kDwHaloBytes = 3 * kDwBandBytes;      // rows above, at and below: 25344

template <int EPI, bool DW>
struct StreamCfg {
    static constexpr int kProdWarps = DW ? kDwProdWarps : 1;
    static constexpr int kMmaWarp = kProdWarps;
    static constexpr int kThreads = 32 * (kProdWarps + 1 + kSEpiWarps);
    static constexpr bool kRes = stream_has_res(EPI);
    static constexpr int kStages = DW ? kDwStages : (kRes ? kSStages : kSStagesPlain);
    // residual epilogues: a ring of residual boxes per warp; others: one output staging box
    static constexpr int kResSlots = kRes ? kSResSlots : 1;
    static constexpr int kMaxK = kRes ? kSMaxK : kSMaxKPlain;
    static constexpr int kSlotBytes = kSBoxBytes;
    static constexpr int kBOffset = 0;                                   // resident W slice
    static constexpr int kBBytes = kSBN * kMaxK * 2;                     // 64 / 128 KB
    static constexpr int kAOffset = kBOffset + kBBytes;
    static constexpr int kHaloOffset = kAOffset + kStages * kSABytes;    // two band sets (DW)
    static constexpr int kHaloBytes = DW ? (2 * kDwHaloBytes + 1023) / 1024 * 1024 : 0;
    static constexpr int kEpiOffset = kHaloOffset + kHaloBytes;
    static constexpr int kEpiBytes = kSEpiWarps * kResSlots * kSlotBytes;
    static constexpr int kBarOffset = kEpiOffset + kEpiBytes;
    static constexpr int kBarBytes = 512;
    // DW: each epilogue warp's 32 bias values (registers are short with four producer warps)
    static constexpr int kBiasOffset = kBarOffset + kBarBytes;
    static constexpr int kBiasBytes = DW ? kSEpiWarps * kSCols * 4 : 0;
    static constexpr int kBytes = kBiasOffset + kBiasBytes + 1024;
    static_assert(kBytes <= 232448, "shared memory budget exceeded");
    static_assert(kEpiOffset % 1024 == 0 && kHaloOffset % 1024 == 0, "TMA destinations stay aligned");
};

template <typename T>
struct SPack2;
template <>
struct SPack2<__half> {
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
struct SPack2<__nv_bfloat16> {
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

// Byte offset of 16-byte chunk j (0..3) of row r in a 64-byte-row box written with SWIZZLE_64B.
__device__ __forceinline__ int sw64_off(int r, int j) { return r * 64 + ((j ^ ((r >> 1) & 3)) << 4); }

// Rows [r0, r1) of the CTA `idx` of `G` CTAs sharing one channel slice: 32-row groups split as
// evenly as possible.
__device__ __forceinline__ void cta_rows(int M, int idx, int G, int* r0, int* r1)
{
    const int groups = (M + 31) / 32;
    const int g0 = static_cast<int>((static_cast<long long>(groups) * idx) / G);
    const int g1 = static_cast<int>((static_cast<long long>(groups) * (idx + 1)) / G);
    *r0 = g0 * 32;
    *r1 = g1 * 32 < M ? g1 * 32 : M;
}

template <typename T, int EPI, bool DW>
__global__ void __launch_bounds__(StreamCfg<EPI, DW>::kThreads, 1)
    gemm_stream_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                       const __grid_constant__ CUtensorMap tmO, const __grid_constant__ CUtensorMap tmR,
                       const GemmParams p, int ctas_per_slice)
{
    using C = StreamCfg<EPI, DW>;
    constexpr int kStages = C::kStages;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem =
        reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::kBarOffset);
    uint64_t* empty = full + kStages;
    uint64_t* bfull = empty + kStages;
    uint64_t* tfull = bfull + 1;
    uint64_t* tempty = tfull + 2;
    uint64_t* drain = tempty + 2;
    uint64_t* resbar = drain + 1;  // [kSEpiWarps][kSResSlots]
    uint64_t* hfull = resbar + kSEpiWarps * kSResSlots;  // DW: band sets landed / read
    uint64_t* hempty = hfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(hempty + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int slice = blockIdx.x / ctas_per_slice;
    const int n0 = slice * kSBN;
    int r0, r1;
    cta_rows(p.M, blockIdx.x % ctas_per_slice, ctas_per_slice, &r0, &r1);
    const int ntiles = r1 > r0 ? (r1 - r0 + kSBM - 1) / kSBM : 0;
    const int kblocks = p.K / kSBK;
    // progress waits give up after `lim` cycles; the drains after an abort keep the full limit
    const long long lim = p.wait_limit > 0 ? p.wait_limit : kSWaitLimit;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            // DW: one arrival per producer warp once its rows of the stage are written
            mbar_init(&full[s], DW ? kDwProdWarps : 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&hfull[b], 1);
            mbar_init(&hempty[b], kDwProdWarps);
        }
        mbar_init(bfull, 1);
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], kSEpiWarps);
        }
        mbar_init(drain, 1);
        for (int w = 0; w < kSEpiWarps * kSResSlots; ++w) {
            mbar_init(&resbar[w], 1);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
    }
    if (warp == C::kMmaWarp) {
        tmem_alloc(tmem_slot, 2 * kSBN);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    griddep_launch_dependents();
    griddep_wait();

    if (DW && warp < C::kProdWarps) {
        // ------------------------------------------------------------ depthwise producers
        // Step v fills half `v & 1` (64 rows) of the A stage of unit u = v >> 1 = (tile
        // u / kblocks, K block u % kblocks) from band set v & 1; each warp computes 16
        // consecutive pixels, each lane one channel pair, sliding a 3 x 3 window of FP32 pairs.
        using P = SPack2<T>;
        const int subs = 2 * ntiles * kblocks;
        const bool issuer = warp == 0 && lane == 0;
        uint32_t halo_pending = 0;
        int halo_last0 = 0, halo_last1 = 0;  // the last step issued into band set 0 / 1
        auto issue_halo = [&](int v) {
            const int u = v >> 1;
            const int t = u / kblocks;
            const int kb = u - t * kblocks;
            const int first = r0 + t * kSBM + (v & 1) * kDwSubPx;  // first output pixel
            uint8_t* hb = smem + C::kHaloOffset + (v & 1) * kDwHaloBytes;
            mbar_arrive_expect_tx(&hfull[v & 1], kDwHaloBytes);
            for (int b = 0; b < 3; ++b) {
                // band b: input pixels first - 1 + (b - 1) * W .. + 65; rows outside the
                // image (negative or past M) read as zero
                tma_load_2d(hb + b * kDwBandBytes, &tmA, &hfull[v & 1], kb * kSBK,
                            first - 1 + (b - 1) * p.dw_w);
            }
            halo_pending |= 1u << (v & 1);
            if (v & 1) {
                halo_last1 = v;
            } else {
                halo_last0 = v;
            }
        };
        if (ntiles > 0 && !p.stall_test) {
            if (issuer) {
                mbar_arrive_expect_tx(bfull, static_cast<uint32_t>(kblocks * kSBN * kSBK * 2));
                for (int kb = 0; kb < kblocks; ++kb) {
                    tma_load_2d(smem + C::kBOffset + kb * kSBN * 128, &tmB, bfull, kb * kSBK, n0);
                }
                issue_halo(0);
                if (subs > 1) {
                    issue_halo(1);
                }
            }
            const int W8 = p.dw_w;
            const int img_h = p.dw_img_h;
            const float2* wt2 = reinterpret_cast<const float2*>(p.dw_weight);
            float2 wp[9];
            for (int v = 0; v < subs; ++v) {
                if (__any_sync(0xffffffffu, *abort_flag != 0)) {
                    break;  // one decision for the whole warp
                }
                const int u = v >> 1;
                const int ph = v & 1;
                const int t = u / kblocks;
                const int kb = u - t * kblocks;
                const int s = u % kStages;
                uint8_t* stage = smem + C::kAOffset + s * kSABytes;
                // every wait's outcome is made warp-uniform, so the warp leaves the loop together
                if (ph == 0) {
                    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&empty[s], ((u / kStages) & 1) ^ 1, lim))) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmProducerTimeout);
                        break;
                    }
                    // the weights [9][K] of this lane's channel pair in K block kb
#pragma unroll
                    for (int k = 0; k < 9; ++k) {
                        wp[k] = __ldg(wt2 + k * (p.K >> 1) + kb * (kSBK / 2) + lane);
                    }
                }
                if (!__all_sync(0xffffffffu, mbar_wait_bounded(&hfull[v & 1], (v >> 1) & 1, lim))) {
                    *abort_flag = 1;
                    report_error(p.err, kErrGemmProducerTimeout);
                    break;
                }
                if (issuer) {
                    halo_pending &= ~(1u << (v & 1));
                }
                const uint32_t* band =
                    reinterpret_cast<const uint32_t*>(smem + C::kHaloOffset + (v & 1) * kDwHaloBytes);
                constexpr int kBandWords = kDwBandBytes / 4;
                const int l0 = warp * kDwPxPerWarp;  // first pixel of this warp within the half
                const int px0 = r0 + t * kSBM + ph * kDwSubPx + l0;
                const int h0 = px0 / W8;
                int w = px0 - h0 * W8;  // column of the current pixel
                int hm = h0 % img_h;    // its row within its image
                float2 win[3][3];       // [band][column - 1 .. + 1]
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    win[b][0] = P::unpack(band[b * kBandWords + l0 * 32 + lane]);
                    win[b][1] = P::unpack(band[b * kBandWords + (l0 + 1) * 32 + lane]);
                }
#pragma unroll
                for (int j = 0; j < kDwPxPerWarp; ++j) {
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        win[b][2] = P::unpack(band[b * kBandWords + (l0 + j + 2) * 32 + lane]);
                    }
                    // taps outside the pixel's image are zero, as in the standalone kernel's
                    // zero-filled halo; FP32 accumulation in the order ky, kx
                    const bool ok_y[3] = {hm != 0, true, hm != img_h - 1};
                    const bool ok_x[3] = {w != 0, true, w != W8 - 1};
                    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                    for (int ky = 0; ky < 3; ++ky) {
#pragma unroll
                        for (int kx = 0; kx < 3; ++kx) {
                            const float2 x = (ok_y[ky] && ok_x[kx]) ? win[ky][kx] : make_float2(0.f, 0.f);
                            acc = __ffma2_rn(x, wp[ky * 3 + kx], acc);
                        }
                    }
                    // row r of the stage, channel pair `lane`: 16-byte chunk lane / 4, swizzled
                    // with the row as TMA's 128-byte swizzle would place it
                    const int r = ph * kDwSubPx + l0 + j;
                    *reinterpret_cast<uint32_t*>(stage + r * 128 + ((((lane >> 2) ^ (r & 7))) << 4) +
                                                 (lane & 3) * 4) = P::pack(acc.x, acc.y);
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        win[b][0] = win[b][1];
                        win[b][1] = win[b][2];
                    }
                    if (++w == W8) {
                        w = 0;
                        if (++hm == img_h) {
                            hm = 0;
                        }
                    }
                }
                // the stage is read by the tensor cores (async proxy)
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&hempty[v & 1]);
                    if (ph == 1) {
                        mbar_arrive(&full[s]);
                    }
                }
                if (issuer && v + 2 < subs) {
                    // the band set is free once every producer warp has read it
                    if (!mbar_wait_bounded(&hempty[v & 1], (v >> 1) & 1, lim)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmProducerTimeout);
                    } else {
                        issue_halo(v + 2);
                    }
                }
                __syncwarp();
            }
            if (issuer && *abort_flag) {
                // let this thread's copies land before the CTA winds down
                mbar_wait_bounded(bfull, 0, kSWaitLimit / 16);
                for (int b = 0; b < 2; ++b) {
                    if (halo_pending & (1u << b)) {
                        mbar_wait_bounded(&hfull[b], ((b ? halo_last1 : halo_last0) >> 1) & 1, kSWaitLimit / 16);
                    }
                }
            }
        }
    } else if (!DW && warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0 && ntiles > 0 && !p.stall_test) {
            // the W slice once: kblocks boxes of 128 rows x 64 K
            mbar_arrive_expect_tx(bfull, static_cast<uint32_t>(kblocks * kSBN * kSBK * 2));
            for (int kb = 0; kb < kblocks; ++kb) {
                tma_load_2d(smem + C::kBOffset + kb * kSBN * 128, &tmB, bfull, kb * kSBK, n0);
            }
            int stage = 0;
            uint32_t phase = 0;
            int issued = 0;
            for (int t = 0; t < ntiles && !*abort_flag; ++t) {
                const int m0 = r0 + t * kSBM;
                for (int kb = 0; kb < kblocks; ++kb) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, lim)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmProducerTimeout);
                        break;
                    }
                    mbar_arrive_expect_tx(&full[stage], kSABytes);
                    tma_load_2d(smem + C::kAOffset + stage * kSABytes, &tmA, &full[stage], kb * kSBK, m0);
                    ++issued;
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            if (*abort_flag) {
                // let this thread's copies land before the CTA winds down
                mbar_wait_bounded(bfull, 0, kSWaitLimit / 16);
                int n = issued < kStages ? issued : kStages;
                for (int i = 0; i < n; ++i) {
                    if (--stage < 0) {
                        stage = kStages - 1;
                        phase ^= 1;
                    }
                    mbar_wait_bounded(&full[stage], phase, kSWaitLimit / 16);
                }
            }
        }
    } else if (warp == C::kMmaWarp) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0 && ntiles > 0) {
            const uint32_t idesc = make_idesc_f16(kSBM, kSBN, SPack2<T>::kFormat);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            bool issued_any = false;
            if (!mbar_wait_bounded(bfull, 0, lim)) {
                *abort_flag = 1;
                report_error(p.err, kErrGemmMmaTimeout);
            }
            tc_fence_after();
            for (int t = 0; t < ntiles && !*abort_flag; ++t) {
                if (!mbar_wait_bounded(&tempty[acc], acc_phase ^ 1, lim)) {
                    *abort_flag = 1;
                    report_error(p.err, kErrGemmMmaTimeout);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + static_cast<uint32_t>(acc * kSBN);
                for (int kb = 0; kb < kblocks; ++kb) {
                    if (!mbar_wait_bounded(&full[stage], phase, lim)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmMmaTimeout);
                        break;
                    }
                    tc_fence_after();
                    const uint64_t adesc =
                        make_sw128_kmajor_desc(smem_u32(smem + C::kAOffset + stage * kSABytes));
                    const uint64_t bdesc =
                        make_sw128_kmajor_desc(smem_u32(smem + C::kBOffset + kb * kSBN * 128));
#pragma unroll
                    for (int k = 0; k < kSBK / 16; ++k) {
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
                tc_commit(drain);
                mbar_wait_bounded(drain, 0, kSWaitLimit / 16);
            }
        }
    } else {
        // ------------------------------------------------------------ epilogue warps
        using P = SPack2<T>;
        const int ew = warp - (C::kMmaWarp + 1);
        const int quad = warp & 3;        // TMEM lane quadrant this warp may access
        const int part = ew >> 2;         // which 32 of the CTA's 128 columns
        const int ncol = n0 + part * kSCols;
        uint8_t* wbuf = smem + C::kEpiOffset + ew * C::kResSlots * C::kSlotBytes;
        uint64_t* rbar = &resbar[ew * kSResSlots];
        uint32_t res_phase = 0;
        uint32_t res_pending = 0;
        if (lane == 0) {
            tma_prefetch_desc(&tmO);
            tma_prefetch_desc(&tmR);
        }
        // residual box of this warp for tile t into slot s (rows past the range: nothing)
        auto issue_res = [&](int t, int s) {
            if (!C::kRes || t >= ntiles) {
                return;
            }
            const int row0 = r0 + t * kSBM + quad * 32;
            if (row0 >= r1) {
                return;
            }
            mbar_arrive_expect_tx(&rbar[s], kSBoxBytes);
            tma_load_2d(wbuf + s * C::kSlotBytes, &tmR, &rbar[s], ncol, row0);
            res_pending |= 1u << s;
        };
        if (lane == 0) {
            for (int s = 0; s < C::kResSlots; ++s) {
                issue_res(s, s);
            }
        }
        // the bias of this warp's 32 columns, fixed for the whole range: in registers, or (DW,
        // where four producer warps leave fewer registers per thread) in shared memory
        float4 bb[DW ? 1 : 8];
        const float4* bs4 = nullptr;
        if constexpr (DW) {
            float* bs = reinterpret_cast<float*>(smem + C::kBiasOffset) + ew * kSCols;
            bs[lane] = __ldg(p.bias + ncol + lane);
            __syncwarp();
            bs4 = reinterpret_cast<const float4*>(bs);
        } else {
            const float4* b4 = reinterpret_cast<const float4*>(p.bias + ncol);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                bb[j] = __ldg(b4 + j);
            }
        }
        int acc = 0;
        uint32_t acc_phase = 0;
        for (int t = 0; t < ntiles && !*abort_flag; ++t) {
            const int slot = t % C::kResSlots;
            const int row0 = r0 + t * kSBM + quad * 32;
            const bool rows_live = row0 < r1;
            uint8_t* buf = wbuf + slot * C::kSlotBytes;
            if (!mbar_wait_bounded(&tfull[acc], acc_phase, lim)) {
                *abort_flag = 1;
                report_error(p.err, kErrGemmEpilogueTimeout);
                break;
            }
            tc_fence_after();
            if (C::kRes && rows_live) {
                if (!mbar_wait_bounded(&rbar[slot], (res_phase >> slot) & 1u, lim)) {
                    *abort_flag = 1;
                    report_error(p.err, kErrGemmEpilogueTimeout);
                } else {
                    res_pending &= ~(1u << slot);
                }
                res_phase ^= 1u << slot;
            }
            uint32_t r[32];
            tmem_ld_32x32b_x32(tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + acc * kSBN +
                                   part * kSCols,
                               r);
            tc_wait_ld();
            // the accumulator buffer is free once its columns are in registers
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&tempty[acc]);
            }
            acc ^= 1;
            if (acc == 0) {
                acc_phase ^= 1;
            }
            if (rows_live && !*abort_flag) {
                float2 v[16];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float4 b;
                    if constexpr (DW) {
                        b = bs4[j];
                    } else {
                        b = bb[j];
                    }
                    v[2 * j] = __fadd2_rn(make_float2(__uint_as_float(r[4 * j + 0]), __uint_as_float(r[4 * j + 1])),
                                          make_float2(b.x, b.y));
                    v[2 * j + 1] = __fadd2_rn(make_float2(__uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3])),
                                              make_float2(b.z, b.w));
                }
                if constexpr (C::kRes) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const uint4 u = *reinterpret_cast<const uint4*>(buf + sw64_off(lane, j));
                        v[4 * j + 0] = __fadd2_rn(v[4 * j + 0], P::unpack(u.x));
                        v[4 * j + 1] = __fadd2_rn(v[4 * j + 1], P::unpack(u.y));
                        v[4 * j + 2] = __fadd2_rn(v[4 * j + 2], P::unpack(u.z));
                        v[4 * j + 3] = __fadd2_rn(v[4 * j + 3], P::unpack(u.w));
                    }
                }
                if constexpr (EPI == kEpiBiasWsilu) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        v[j] = wsilu2(v[j]);
                    }
                }
                if constexpr (EPI == kEpiBiasResQ) {
                    // this lane's row picks its image's factors in a packed batch
                    const int qm = min(row0 + lane, p.M - 1);
                    const size_t qrow = p.q_rows > 0 ? static_cast<size_t>(qm / p.q_rows) * p.N : 0;
                    const uint4* qs = reinterpret_cast<const uint4*>(
                        reinterpret_cast<const T*>(p.qscale) + qrow + ncol);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const uint4 u = __ldg(qs + j);
                        v[4 * j + 0] = __fmul2_rn(v[4 * j + 0], P::unpack(u.x));
                        v[4 * j + 1] = __fmul2_rn(v[4 * j + 1], P::unpack(u.y));
                        v[4 * j + 2] = __fmul2_rn(v[4 * j + 2], P::unpack(u.z));
                        v[4 * j + 3] = __fmul2_rn(v[4 * j + 3], P::unpack(u.w));
                    }
                }
                uint32_t pk[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    pk[j] = P::pack(v[j].x, v[j].y);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    *reinterpret_cast<uint4*>(buf + sw64_off(lane, j)) =
                        make_uint4(pk[4 * j + 0], pk[4 * j + 1], pk[4 * j + 2], pk[4 * j + 3]);
                }
                if (p.out8 != nullptr && row0 + lane < p.M) {
                    // the E4M3 copy of the stored (rounded) values, as a separate quantisation of
                    // this output would produce it: 32 bytes of this lane's row
                    uint32_t q8[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const float2 a = P::unpack(pk[2 * j]), b = P::unpack(pk[2 * j + 1]);
                        const uint32_t lo = __nv_cvt_float2_to_fp8x2(
                            make_float2(a.x * p.out8_inv_scale, a.y * p.out8_inv_scale), __NV_SATFINITE, __NV_E4M3);
                        const uint32_t hi = __nv_cvt_float2_to_fp8x2(
                            make_float2(b.x * p.out8_inv_scale, b.y * p.out8_inv_scale), __NV_SATFINITE, __NV_E4M3);
                        q8[j] = lo | (hi << 16);
                    }
                    uint4* d8 = reinterpret_cast<uint4*>(static_cast<uint8_t*>(p.out8) +
                                                         static_cast<size_t>(row0 + lane) * p.ldo8 + ncol);
                    d8[0] = make_uint4(q8[0], q8[1], q8[2], q8[3]);
                    d8[1] = make_uint4(q8[4], q8[5], q8[6], q8[7]);
                }
                fence_proxy_async_smem();
            }
            __syncwarp();
            if (lane == 0) {
                if (rows_live && !*abort_flag) {
                    tma_store_2d(&tmO, buf, ncol, row0);
                    bulk_commit();
                }
                if (!*abort_flag) {
                    bulk_wait_read0();  // the store has read the slot: refill or reuse it
                    issue_res(t + C::kResSlots, slot);
                }
            }
            __syncwarp();
        }
        if (lane == 0) {
            // after an abort, let this warp's residual loads land before the CTA winds down
            for (int s = 0; s < C::kResSlots; ++s) {
                if (res_pending & (1u << s)) {
                    mbar_wait_bounded(&rbar[s], (res_phase >> s) & 1u, kSWaitLimit / 16);
                }
            }
            bulk_wait_read0();
        }
        __syncwarp();
    }

    tc_fence_before();
    __syncthreads();
    if (warp == C::kMmaWarp) {
        tc_fence_after();
        tmem_dealloc(tmem_base, 2 * kSBN);
    }
}

template <typename T, int EPI, bool DW>
cudaError_t launch_stream(const CUtensorMap* maps, const GemmParams& p, cudaStream_t stream)
{
    using C = StreamCfg<EPI, DW>;
    auto kernel = gemm_stream_kernel<T, EPI, DW>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&] {
        attr_err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, C::kBytes);
    });
    if (attr_err != cudaSuccess) {
        return attr_err;
    }
    const int slices = p.N / kSBN;
    // CTAs per channel slice: the SMs shared out, but no more than one per 32-row group
    int per = num_sms() / slices;
    const int groups = (p.M + 31) / 32;
    per = per < groups ? per : groups;
    per = per < 1 ? 1 : per;
    return launch_pdl(kernel, dim3(slices * per), dim3(C::kThreads), C::kBytes, stream, maps[0], maps[1],
                      maps[2], maps[3], p, per);
}

}  // namespace

bool gemm_stream_eligible(int epi, int M, int N, int K)
{
    const bool res = stream_has_res(epi);
    if (!res && epi != kEpiBias && epi != kEpiBiasWsilu) {
        return false;
    }
    return M > 0 && N % kSBN == 0 && K % kSBK == 0 && K <= (res ? kSMaxK : kSMaxKPlain) &&
           N / kSBN <= num_sms();
}

// Host launcher of the streaming form; same operands and checks as gemm_sm100 (A [M, K] with
// pitch lda, W [N, K] dense, outputs/residuals with their pitches).
cudaError_t gemm_stream_sm100(int dtype, const void* A, int lda, const void* W, const GemmParams& p,
                              int epi, cudaStream_t stream)
{
    const bool res = stream_has_res(epi);
    if (!gemm_stream_eligible(epi, p.M, p.N, p.K) || lda % 8 != 0 || p.ldo % 8 != 0 ||
        (reinterpret_cast<uintptr_t>(A) & 15) != 0 || (reinterpret_cast<uintptr_t>(W) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(p.out) & 15) != 0 || p.bias == nullptr) {
        return cudaErrorInvalidValue;
    }
    if (res && (p.res == nullptr || p.ldr % 8 != 0 || (reinterpret_cast<uintptr_t>(p.res) & 15) != 0)) {
        return cudaErrorInvalidValue;
    }
    if (!res && p.out8 != nullptr) {
        return cudaErrorInvalidValue;  // the E4M3 side output belongs to the residual epilogues
    }
    if (epi == kEpiBiasResQ && p.qscale == nullptr) {
        return cudaErrorInvalidValue;
    }
    if (p.out8 != nullptr && (p.ldo8 % 16 != 0 || (reinterpret_cast<uintptr_t>(p.out8) & 15) != 0)) {
        return cudaErrorInvalidValue;
    }
    const bool dw = p.dw_weight != nullptr;
    if (dw && (epi != kEpiBiasRes || p.dw_w < 1 || p.dw_h < 1 ||
               static_cast<long long>(p.dw_h) * p.dw_w != p.M || p.dw_img_h < 1 || p.dw_h % p.dw_img_h != 0 ||
               (reinterpret_cast<uintptr_t>(p.dw_weight) & 15) != 0)) {
        return cudaErrorInvalidValue;
    }
    const CUtensorMapDataType dt = dtype == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    CUtensorMap maps[4];
    std::memset(maps, 0, sizeof(maps));
    // A: 128-row operand boxes, or (depthwise form) unswizzled 66-pixel bands of the input
    if (!(dw ? make_tmap_2d(&maps[0], dt, A, p.K, p.M, static_cast<uint64_t>(lda) * 2, kSBK, kDwBandRows, 0)
             : make_tmap_2d(&maps[0], dt, A, p.K, p.M, static_cast<uint64_t>(lda) * 2, kSBK, kSBM, 128)) ||
        !make_tmap_2d(&maps[1], dt, W, p.K, p.N, static_cast<uint64_t>(p.K) * 2, kSBK, kSBN, 128) ||
        !make_tmap_2d(&maps[2], dt, p.out, p.N, p.M, static_cast<uint64_t>(p.ldo) * 2, kSCols, 32, 64) ||
        (res && !make_tmap_2d(&maps[3], dt, p.res, p.N, p.M, static_cast<uint64_t>(p.ldr) * 2, kSCols, 32, 64))) {
        return cudaErrorInvalidValue;
    }
    if (!res) {
        maps[3] = maps[2];  // no residual: the kernel never reads this map
    }
    if (dw) {
        return dtype == 0 ? launch_stream<__half, kEpiBiasRes, true>(maps, p, stream)
                          : launch_stream<__nv_bfloat16, kEpiBiasRes, true>(maps, p, stream);
    }
    if (dtype == 0) {
        switch (epi) {
        case kEpiBias: return launch_stream<__half, kEpiBias, false>(maps, p, stream);
        case kEpiBiasWsilu: return launch_stream<__half, kEpiBiasWsilu, false>(maps, p, stream);
        case kEpiBiasRes: return launch_stream<__half, kEpiBiasRes, false>(maps, p, stream);
        case kEpiBiasResQ: return launch_stream<__half, kEpiBiasResQ, false>(maps, p, stream);
        }
    } else {
        switch (epi) {
        case kEpiBias: return launch_stream<__nv_bfloat16, kEpiBias, false>(maps, p, stream);
        case kEpiBiasWsilu: return launch_stream<__nv_bfloat16, kEpiBiasWsilu, false>(maps, p, stream);
        case kEpiBiasRes: return launch_stream<__nv_bfloat16, kEpiBiasRes, false>(maps, p, stream);
        case kEpiBiasResQ: return launch_stream<__nv_bfloat16, kEpiBiasResQ, false>(maps, p, stream);
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace dcvc
