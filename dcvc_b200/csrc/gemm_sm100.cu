// tcgen05/TMEM persistent GEMM with fused 1x1-conv epilogues (see gemm_sm100.cuh).
#include "gemm_sm100.cuh"
#include "host_util.h"

#include <atomic>
#include <cstring>
#include <mutex>

namespace dcvc {

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;  // one 128-byte swizzle atom of 16-bit elements
constexpr int kMaxEpiWarps = 16;
// ~1 s at 2 GHz; a correct kernel never waits this long.
constexpr long long kWaitLimit = 2000000000LL;
constexpr int kSmemLimit = 232448;  // 227 KB per block on sm_100

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

__host__ __device__ constexpr bool epi_has_res(int e) { return e == kEpiBiasRes || e == kEpiBiasResQ || e == kEpiBiasRes2; }
__host__ __device__ constexpr bool epi_has_q(int e) { return e == kEpiBiasResQ || e == kEpiBiasQ; }

// Epilogue warps: 16 (four per TMEM lane quadrant, each owning a quarter of the BN accumulator
// columns) for the residual epilogues with BN >= 128, whose per-tile epilogue (residual load,
// add, store) is longer than the tile's main loop (K = 256); 8 (two per quadrant, half the
// columns each) otherwise, which leaves shared memory for a deeper operand pipeline.
__host__ __device__ constexpr int epi_warps(int bn, int epi)
{
    return (epi_has_res(epi) && bn >= 128) ? 16 : 8;
}
// Accumulator columns per epilogue warp, and output columns of one store box (32 rows high).
__host__ __device__ constexpr int epi_cols(int bn, int epi) { return bn / (epi_warps(bn, epi) / 4); }
__host__ __device__ constexpr int out_box_cols(int bn, int epi)
{
    return epi == kEpiQuad ? epi_cols(bn, epi) / 4 : (epi_cols(bn, epi) < 64 ? epi_cols(bn, epi) : 64);
}

// PAIR: the CTA is one of a cluster pair computing 256-row tiles with cta_group::2; it stages
// half of the B tile (BN / 2 rows).
template <int BN, int EPI, bool PAIR = false>
struct GemmCfg {
    static constexpr int kEpiWarps = epi_warps(BN, EPI);
    static constexpr int kThreads = 64 + 32 * kEpiWarps;  // producer warp, MMA warp, epilogue warps
    static constexpr int kCols = epi_cols(BN, EPI);             // accumulator columns per warp
    static constexpr int kOutW = out_box_cols(BN, EPI);         // output columns per store box
    static constexpr int kAccPerBox = EPI == kEpiQuad ? 4 * kOutW : kOutW;
    static constexpr int kBoxes = kCols / kAccPerBox;
    static constexpr int kBoxBytes = kOutW * 32 * 2;            // 4 KB (64 cols) or 2 KB (32 cols)
    static constexpr int kRowBytes = kOutW * 2;                 // 128 (SW128) or 64 (SW64)
    static constexpr int kResBufs = EPI == kEpiBiasRes2 ? 2 : (epi_has_res(EPI) ? 1 : 0);
    // Residual boxes in flight per warp: a ring of kResSlots box slots filled in (tile, box)
    // order, so a tile's residual streams in while its accumulator is still being computed.  The
    // result is written over the residual in its slot and stored from there; epilogues without a
    // residual stage their output in one buffer of their own.
    static constexpr int kResSlots = kResBufs == 1 ? (kBoxes < 2 ? kBoxes : 2) : (kResBufs == 2 ? 1 : 0);
    static constexpr int kWarpStage = 4096 * (kResBufs == 0 ? 1 : kResBufs * kResSlots);
    static constexpr int kEpiBytes = kEpiWarps * kWarpStage;
    static constexpr int kABytes = kBM * kBK * 2;
    static constexpr int kBBytes = (PAIR ? BN / 2 : BN) * kBK * 2;
    static constexpr int kStageBytes = kABytes + kBBytes;
    static constexpr int kBarBytes = 512;
    static constexpr int kStagesFit = (kSmemLimit - 1024 - kEpiBytes - kBarBytes) / kStageBytes;
    static constexpr int kStages = kStagesFit > 8 ? 8 : kStagesFit;
    static constexpr int kEpiOffset = kStages * kStageBytes;
    static constexpr int kBarOffset = kEpiOffset + kEpiBytes;
    static constexpr int kBytes = kBarOffset + kBarBytes + 1024;
    static constexpr int kTmemCols = 2 * BN;
    static_assert(kStages >= 2, "shared memory too small for two pipeline stages");
    static_assert(kBytes <= kSmemLimit, "shared memory budget exceeded");
    static_assert(EPI == kEpiSubpel || kBoxes * kAccPerBox == kCols, "box tiling");
    static_assert(EPI == kEpiSubpel || kOutW * 2 == 128 || kOutW * 2 == 64, "staging row width");
    static_assert(kEpiWarps <= kMaxEpiWarps, "epilogue warps");
    static_assert(kResSlots <= 2, "residual ring");
};

// Byte offset of the 16-byte chunk j of row r inside a swizzled staging box (the layout TMA
// uses for SWIZZLE_128B with 128-byte rows and SWIZZLE_64B with 64-byte rows).
template <int ROWB>
__device__ __forceinline__ int stage_off(int r, int j)
{
    if constexpr (ROWB == 128) {
        return r * 128 + ((j ^ (r & 7)) << 4);
    } else {
        return r * 64 + ((j ^ ((r >> 1) & 3)) << 4);
    }
}

// F8: E4M3 operands (kind::f8f6f4, 128 elements per 128-byte K block) with the accumulator scaled
// per output channel by p.wscale before the bias; T is then the BF16 output type.
//
// PAIR: launched as clusters of two CTAs.  The pair computes 256 x BN tiles: CTA rank r stages rows
// 128 r .. 128 r + 127 of the A tile and rows (BN / 2) r .. of the B tile, its TMA loads count on
// the even CTA's full barrier, the even CTA issues tcgen05.mma.cta_group::2 (M = 256) and commits
// to the empty and accumulator-full barriers of both CTAs, and each CTA's epilogue drains its own
// 128 accumulator rows and arrives on the even CTA's accumulator-empty barrier.
template <typename T, int BN, int EPI, bool F8 = false, bool PAIR = false>
__global__ void __launch_bounds__(GemmCfg<BN, EPI, PAIR>::kThreads, 1)
    gemm_sm100_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const __grid_constant__ CUtensorMap tmO, const __grid_constant__ CUtensorMap tmR,
                      const __grid_constant__ CUtensorMap tmR2, const GemmParams p)
{
    static_assert(!(PAIR && F8), "the pair form is built for 16-bit operands");
    constexpr int kKElems = F8 ? 128 : kBK;  // K elements per 128-byte K block
    // progress waits give up after `lim` cycles; the drains after an abort keep the full limit
    const long long lim = p.wait_limit > 0 ? p.wait_limit : kWaitLimit;
    using C = GemmCfg<BN, EPI, PAIR>;
    constexpr int kTileM = PAIR ? 2 * kBM : kBM;
    constexpr int kStages = C::kStages;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem =
        reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::kBarOffset);
    uint64_t* empty = full + kStages;
    uint64_t* tfull = empty + kStages;
    uint64_t* tempty = tfull + 2;
    uint64_t* drain = tempty + 2;
    uint64_t* resbar = drain + 1;  // [kEpiWarps][2]: one barrier per residual ring slot
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(resbar + 2 * C::kEpiWarps);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int num_m = (p.M + kTileM - 1) / kTileM;
    const int num_n = p.N / BN;
    const int num_tiles = num_m * num_n;
    const int kblocks = p.K / kKElems;
    // work units: CTAs, or (PAIR) CTA pairs; rank 0 is the pair's MMA issuer
    const uint32_t rank = PAIR ? cluster_cta_rank() : 0;
    const int unit = PAIR ? static_cast<int>(blockIdx.x >> 1) : static_cast<int>(blockIdx.x);
    const int units = PAIR ? static_cast<int>(gridDim.x >> 1) : static_cast<int>(gridDim.x);
    const int row_off = PAIR ? static_cast<int>(rank) * kBM : 0;  // this CTA's rows in the tile

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            // PAIR: both CTAs' epilogue warps release the even CTA's accumulator
            mbar_init(&tempty[b], PAIR ? 2 * C::kEpiWarps : C::kEpiWarps);
        }
        mbar_init(drain, 1);
        for (int w = 0; w < 2 * C::kEpiWarps; ++w) {
            mbar_init(&resbar[w], 1);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
    }
    if (warp == 1) {
        if constexpr (PAIR) {
            tmem_alloc_pair(tmem_slot, C::kTmemCols);
            tmem_relinquish_pair();
        } else {
            tmem_alloc(tmem_slot, C::kTmemCols);
            tmem_relinquish();
        }
    }
    tc_fence_before();
    __syncthreads();
    if constexpr (PAIR) {
        cluster_sync();  // the peer's barriers are initialised before any copy or arrive reaches them
    }
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    // setup above overlaps the predecessor's tail; its outputs are read only after this
    griddep_launch_dependents();
    griddep_wait();

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0 && !p.stall_test) {
            int stage = 0;
            uint32_t phase = 0;
            int issued = 0;
            for (int tile = unit; tile < num_tiles && !*abort_flag; tile += units) {
                const int m0 = (tile % num_m) * kTileM + row_off;
                const int n0 = (tile / num_m) * BN;
                for (int kb = 0; kb < kblocks; ++kb) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, lim)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmProducerTimeout);
                        break;
                    }
                    uint8_t* sa = smem + stage * C::kStageBytes;
                    if constexpr (PAIR) {
                        // the even CTA's barrier counts both CTAs' bytes
                        if (rank == 0) {
                            mbar_arrive_expect_tx(&full[stage], 2 * C::kStageBytes);
                        }
                        const uint32_t fb = cluster_map(&full[stage], 0);
                        tma_load_2d_pair(sa, &tmA, fb, kb * kKElems, m0);
                        tma_load_2d_pair(sa + C::kABytes, &tmB, fb, kb * kKElems,
                                         n0 + static_cast<int>(rank) * (BN / 2));
                    } else {
                        mbar_arrive_expect_tx(&full[stage], C::kStageBytes);
                        tma_load_2d(sa, &tmA, &full[stage], kb * kKElems, m0);
                        tma_load_2d(sa + C::kABytes, &tmB, &full[stage], kb * kKElems, n0);
                    }
                    ++issued;
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            if (*abort_flag && (!PAIR || rank == 0)) {
                // Let the copies this thread issued land before the CTA winds down (PAIR: the
                // even CTA's barriers count the peer's copies too; the odd CTA cannot observe its
                // own copies, so after an abort it relies on the even CTA's drain, which waits
                // (bounded) for both CTAs' bytes of each stage it issued, and on the cluster
                // barrier before either CTA exits.  A stage that only the odd CTA issued before
                // the abort is not waited for; under the stall injection neither CTA issues any.)
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
        if (lane == 0 && (!PAIR || rank == 0)) {
            // format 0 is F16 for kind::f16 and E4M3 for kind::f8f6f4
            const uint32_t idesc = make_idesc_f16(kTileM, BN, F8 ? 0 : Pack2<T>::kFormat);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            bool issued_any = false;
            for (int tile = unit; tile < num_tiles && !*abort_flag; tile += units) {
                if (!mbar_wait_bounded(&tempty[acc], acc_phase ^ 1, lim)) {
                    *abort_flag = 1;
                    report_error(p.err, kErrGemmMmaTimeout);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + static_cast<uint32_t>(acc * BN);
                for (int kb = 0; kb < kblocks; ++kb) {
                    if (!mbar_wait_bounded(&full[stage], phase, lim)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmMmaTimeout);
                        break;
                    }
                    tc_fence_after();
                    const uint8_t* sa = smem + stage * C::kStageBytes;
                    const uint64_t adesc = make_sw128_kmajor_desc(smem_u32(sa));
                    const uint64_t bdesc = make_sw128_kmajor_desc(smem_u32(sa + C::kABytes));
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        // +32 bytes per instruction inside the swizzle atom (descriptor units of
                        // 16 B): K = 16 16-bit or K = 32 8-bit elements
                        if constexpr (F8) {
                            tc_mma_f8(d, adesc + 2 * k, bdesc + 2 * k, idesc, (kb | k) != 0 ? 1u : 0u);
                        } else if constexpr (PAIR) {
                            tc_mma_f16_pair(d, adesc + 2 * k, bdesc + 2 * k, idesc, (kb | k) != 0 ? 1u : 0u);
                        } else {
                            tc_mma_f16(d, adesc + 2 * k, bdesc + 2 * k, idesc, (kb | k) != 0 ? 1u : 0u);
                        }
                    }
                    issued_any = true;
                    if constexpr (PAIR) {
                        tc_commit_pair_both(&empty[stage]);  // frees the stage in both CTAs
                    } else {
                        tc_commit(&empty[stage]);
                    }
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                if (*abort_flag) {
                    break;
                }
                if constexpr (PAIR) {
                    tc_commit_pair_both(&tfull[acc]);
                } else {
                    tc_commit(&tfull[acc]);
                }
                acc ^= 1;
                if (acc == 0) {
                    acc_phase ^= 1;
                }
            }
            if (*abort_flag && issued_any) {
                // Drain this thread's outstanding MMAs before the columns are released.
                if constexpr (PAIR) {
                    tc_commit_pair_local(drain);
                } else {
                    tc_commit(drain);
                }
                mbar_wait_bounded(drain, 0, kWaitLimit / 16);
            }
        }
    } else {
        // ------------------------------------------------------------ epilogue warps
        using P = Pack2<T>;
        const int ew = warp - 2;                  // epilogue warp index
        const int quad = warp & 3;                // TMEM lane quadrant this warp may access
        const int half = ew >> 2;                 // which column part of the BN columns
        uint8_t* wbuf = smem + C::kEpiOffset + ew * C::kWarpStage;
        // residual ring slot s: res at wbuf + 4096 * s * kResBufs, res2 right after it
        auto res_slot = [&](int s) { return wbuf + 4096 * s * C::kResBufs; };
        uint64_t* rbar = &resbar[2 * ew];
        uint32_t res_phase = 0;    // phase bit per ring slot
        uint32_t res_pending = 0;  // ring slots with a load in flight
        int acc = 0;
        uint32_t acc_phase = 0;
        if (EPI != kEpiSubpel && lane == 0) {
            tma_prefetch_desc(&tmO);
        }
        // Issues the residual load of box `b` of this CTA's `k`-th tile into ring slot `s`
        // (lane 0; nothing for tiles past the end or rows past M).
        auto issue_res = [&](int k, int b, int s) {
            const int t = unit + k * units;
            if (t >= num_tiles) {
                return;
            }
            const int r0 = (t % num_m) * kTileM + row_off + quad * 32;
            if (r0 >= p.M) {
                return;
            }
            const int col = (t / num_m) * BN + half * C::kCols + b * C::kAccPerBox;
            mbar_arrive_expect_tx(&rbar[s], C::kBoxBytes * C::kResBufs);
            tma_load_2d(res_slot(s), &tmR, &rbar[s], col, r0);
            if constexpr (EPI == kEpiBiasRes2) {
                tma_load_2d(res_slot(s) + 4096, &tmR2, &rbar[s], col, r0);
            }
            res_pending |= 1u << s;
        };
        if constexpr (epi_has_res(EPI)) {
            if (lane == 0) {
                for (int i = 0; i < C::kResSlots; ++i) {
                    issue_res(i / C::kBoxes, i % C::kBoxes, i);
                }
            }
        }
        int item = 0;  // (tile, box) sequence number of this warp
        for (int tile = unit, k = 0; tile < num_tiles && !*abort_flag; tile += units, ++k) {
            const int m0 = (tile % num_m) * kTileM + row_off;
            const int n0 = (tile / num_m) * BN;
            const int row0 = m0 + quad * 32;        // first row owned by this warp
            const bool rows_live = row0 < p.M;
            const int nacc0 = n0 + half * C::kCols;  // first accumulator column of this warp
            if (!mbar_wait_bounded(&tfull[acc], acc_phase, lim)) {
                *abort_flag = 1;
                report_error(p.err, kErrGemmEpilogueTimeout);
                break;
            }
            tc_fence_after();
            const uint32_t tbase = tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + acc * BN +
                                   half * C::kCols;
            if constexpr (EPI == kEpiSubpel) {
                // direct stores: the shuffled rows of one box are not contiguous in memory
                const int m = row0 + lane;
                const bool live = m < p.M;
#pragma unroll 1
                for (int c = 0; c < C::kCols / 32; ++c) {
                    uint32_t r[32];
                    tmem_ld_32x32b_x32(tbase + c * 32, r);
                    tc_wait_ld();
                    if (live) {
                        const int nc = nacc0 + c * 32;
                        const int sub = nc / p.sub_cout;  // dy * 2 + dx
                        const int ch = nc - sub * p.sub_cout;
                        const int h = m / p.sub_w;
                        const int w = m - h * p.sub_w;
                        const size_t orow = static_cast<size_t>(2 * h + (sub >> 1)) * (2 * p.sub_w) +
                                            (2 * w + (sub & 1));
                        uint4* d4 = reinterpret_cast<uint4*>(reinterpret_cast<T*>(p.out) + orow * p.ldo + ch);
                        float v[32];
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            v[j] = __uint_as_float(r[j]);
                        }
                        if (p.bias != nullptr) {  // the biased form (SubpelConv2x with a bias)
                            const float4* b4 = reinterpret_cast<const float4*>(p.bias + nc);
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                const float4 bb = __ldg(b4 + j);
                                v[4 * j + 0] += bb.x;
                                v[4 * j + 1] += bb.y;
                                v[4 * j + 2] += bb.z;
                                v[4 * j + 3] += bb.w;
                            }
                        }
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            d4[j] = make_uint4(P::pack(v[8 * j + 0], v[8 * j + 1]),
                                               P::pack(v[8 * j + 2], v[8 * j + 3]),
                                               P::pack(v[8 * j + 4], v[8 * j + 5]),
                                               P::pack(v[8 * j + 6], v[8 * j + 7]));
                        }
                    }
                }
            } else {
#pragma unroll 1
                for (int b = 0; b < C::kBoxes; ++b, ++item) {
                    const int ncol = nacc0 + b * C::kAccPerBox;  // first accumulator column of box
                    const int slot = C::kResSlots > 1 ? item % C::kResSlots : 0;
                    const uint8_t* res_buf = res_slot(slot);
                    const uint8_t* res2_buf = res_buf + 4096;
                    // the result replaces the residual in its slot; without a residual the
                    // warp's own buffer stages it
                    uint8_t* out_buf = epi_has_res(EPI) ? res_slot(slot) : wbuf;
                    if constexpr (epi_has_res(EPI)) {
                        if (rows_live) {
                            if (!mbar_wait_bounded(&rbar[slot], (res_phase >> slot) & 1u, lim)) {
                                *abort_flag = 1;
                                report_error(p.err, kErrGemmEpilogueTimeout);
                            } else {
                                res_pending &= ~(1u << slot);
                            }
                            res_phase ^= 1u << slot;
                        }
                    }
                    // the previous box's store must have read the staging buffer (a residual slot
                    // was already waited for before its refill)
                    if (!epi_has_res(EPI) && lane == 0) {
                        bulk_wait_read0();
                    }
                    __syncwarp();
#pragma unroll 1
                    for (int c = 0; c < C::kAccPerBox / 32; ++c) {
                        const int nc = ncol + c * 32;
                        // the bias loads are issued before the TMEM load so that their latencies
                        // overlap (not in the x q epilogues, which have no registers to spare)
                        constexpr bool kHoist = !epi_has_q(EPI);
                        const float4* b4 = reinterpret_cast<const float4*>(p.bias + nc);
                        float4 bb[8];
                        if constexpr (kHoist) {
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                bb[j] = __ldg(b4 + j);
                            }
                        }
                        uint32_t r[32];
                        tmem_ld_32x32b_x32(tbase + b * C::kAccPerBox + c * 32, r);
                        tc_wait_ld();
                        // Column pairs in packed f32x2 arithmetic: every operation rounds each
                        // lane to nearest on its own, in the same order as the scalar form, so
                        // the outputs are bitwise unchanged and the FP32 instructions halve.
                        float2 v[16];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const float4 bj = kHoist ? bb[j] : __ldg(b4 + j);
                            const float2 a0 = make_float2(__uint_as_float(r[4 * j + 0]), __uint_as_float(r[4 * j + 1]));
                            const float2 a1 = make_float2(__uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3]));
                            if constexpr (F8) {
                                // dequantise: acc * (activation scale * weight row scale) + bias
                                const float4 sj = __ldg(reinterpret_cast<const float4*>(p.wscale + nc) + j);
                                v[2 * j] = __ffma2_rn(a0, make_float2(sj.x, sj.y), make_float2(bj.x, bj.y));
                                v[2 * j + 1] = __ffma2_rn(a1, make_float2(sj.z, sj.w), make_float2(bj.z, bj.w));
                            } else {
                                v[2 * j] = __fadd2_rn(a0, make_float2(bj.x, bj.y));
                                v[2 * j + 1] = __fadd2_rn(a1, make_float2(bj.z, bj.w));
                            }
                        }
                        if constexpr (EPI == kEpiQuad) {
                            uint32_t o[4];
#pragma unroll
                            for (int i = 0; i < 4; ++i) {
                                const float2 w0 = wsilu2(v[4 * i + 0]), w1 = wsilu2(v[4 * i + 1]);
                                const float2 w2 = wsilu2(v[4 * i + 2]), w3 = wsilu2(v[4 * i + 3]);
                                const float s0 = w0.x + w0.y + w1.x + w1.y;
                                const float s1 = w2.x + w2.y + w3.x + w3.y;
                                o[i] = P::pack(s0, s1);
                            }
                            *reinterpret_cast<uint4*>(out_buf + stage_off<C::kRowBytes>(lane, c)) =
                                make_uint4(o[0], o[1], o[2], o[3]);
                            continue;
                        }
                        if constexpr (EPI == kEpiBiasWsilu) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                v[j] = wsilu2(v[j]);
                            }
                        }
                        if constexpr (epi_has_res(EPI)) {
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const uint4 u = *reinterpret_cast<const uint4*>(
                                    res_buf + stage_off<C::kRowBytes>(lane, c * 4 + j));
                                v[4 * j + 0] = __fadd2_rn(v[4 * j + 0], P::unpack(u.x));
                                v[4 * j + 1] = __fadd2_rn(v[4 * j + 1], P::unpack(u.y));
                                v[4 * j + 2] = __fadd2_rn(v[4 * j + 2], P::unpack(u.z));
                                v[4 * j + 3] = __fadd2_rn(v[4 * j + 3], P::unpack(u.w));
                            }
                        }
                        if constexpr (EPI == kEpiBiasRes2) {
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const uint4 u = *reinterpret_cast<const uint4*>(
                                    res2_buf + stage_off<C::kRowBytes>(lane, c * 4 + j));
                                v[4 * j + 0] = __fadd2_rn(v[4 * j + 0], P::unpack(u.x));
                                v[4 * j + 1] = __fadd2_rn(v[4 * j + 1], P::unpack(u.y));
                                v[4 * j + 2] = __fadd2_rn(v[4 * j + 2], P::unpack(u.z));
                                v[4 * j + 3] = __fadd2_rn(v[4 * j + 3], P::unpack(u.w));
                            }
                        }
                        if constexpr (epi_has_q(EPI)) {
                            // this lane's row picks its image's factors in a packed batch
                            const int qm = min(row0 + lane, p.M - 1);
                            const size_t qrow = p.q_rows > 0 ? static_cast<size_t>(qm / p.q_rows) * p.N : 0;
                            const uint4* qs = reinterpret_cast<const uint4*>(
                                reinterpret_cast<const T*>(p.qscale) + qrow + nc);
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const uint4 u = __ldg(qs + j);
                                v[4 * j + 0] = __fmul2_rn(v[4 * j + 0], P::unpack(u.x));
                                v[4 * j + 1] = __fmul2_rn(v[4 * j + 1], P::unpack(u.y));
                                v[4 * j + 2] = __fmul2_rn(v[4 * j + 2], P::unpack(u.z));
                                v[4 * j + 3] = __fmul2_rn(v[4 * j + 3], P::unpack(u.w));
                            }
                        }
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            *reinterpret_cast<uint4*>(out_buf + stage_off<C::kRowBytes>(lane, c * 4 + j)) =
                                make_uint4(P::pack(v[4 * j + 0].x, v[4 * j + 0].y),
                                           P::pack(v[4 * j + 1].x, v[4 * j + 1].y),
                                           P::pack(v[4 * j + 2].x, v[4 * j + 2].y),
                                           P::pack(v[4 * j + 3].x, v[4 * j + 3].y));
                        }
                    }
                    fence_proxy_async_smem();
                    __syncwarp();
                    if (lane == 0 && rows_live) {
                        const int ocol = EPI == kEpiQuad ? ncol / 4 : ncol;
                        tma_store_2d(&tmO, out_buf, ocol, row0);
                        bulk_commit();
                    }
                    if constexpr (epi_has_res(EPI)) {
                        // every lane has read this box's residual: refill the slot with the box
                        // kResSlots items ahead (possibly in this CTA's next tile)
                        if (lane == 0 && !*abort_flag) {
                            bulk_wait_read0();  // the store has read the slot
                            const int nxt = item + C::kResSlots;
                            issue_res(nxt / C::kBoxes, nxt % C::kBoxes, slot);
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                if (PAIR && rank != 0) {
                    mbar_arrive_remote(cluster_map(&tempty[acc], 0));  // the even CTA's barrier
                } else {
                    mbar_arrive(&tempty[acc]);
                }
            }
            acc ^= 1;
            if (acc == 0) {
                acc_phase ^= 1;
            }
        }
        if constexpr (epi_has_res(EPI)) {
            // after an abort, let this warp's residual loads land before the CTA winds down
            if (lane == 0) {
                for (int s = 0; s < C::kResSlots; ++s) {
                    if (res_pending & (1u << s)) {
                        mbar_wait_bounded(&rbar[s], (res_phase >> s) & 1u, kWaitLimit / 16);
                    }
                }
            }
        }
        // the staging buffers must have been read before the CTA's shared memory is released;
        // the global writes themselves complete with the grid
        if (EPI != kEpiSubpel && lane == 0) {
            bulk_wait_read0();
        }
        __syncwarp();
    }

    tc_fence_before();
    __syncthreads();
    if constexpr (PAIR) {
        // both CTAs are done with the pair's accumulators and with each other's barriers
        cluster_sync();
    }
    if (warp == 1) {
        tc_fence_after();
        if constexpr (PAIR) {
            tmem_dealloc_pair(tmem_base, C::kTmemCols);
        } else {
            tmem_dealloc(tmem_base, C::kTmemCols);
        }
    }
}

struct Maps {
    CUtensorMap a, b, o, r, r2;
};

template <typename T, int BN, int EPI, bool F8 = false, bool PAIR = false>
cudaError_t launch_one(const Maps& m, const GemmParams& p, cudaStream_t stream)
{
    using C = GemmCfg<BN, EPI, PAIR>;
    auto kernel = gemm_sm100_kernel<T, BN, EPI, F8, PAIR>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&] {
        attr_err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, C::kBytes);
    });
    if (attr_err != cudaSuccess) {
        return attr_err;
    }
    if constexpr (PAIR) {
        // one cluster of two CTAs per pair of SMs, at most one per 256-row tile
        const int num_tiles = ((p.M + 2 * kBM - 1) / (2 * kBM)) * (p.N / BN);
        int pairs = num_sms() / 2;
        pairs = num_tiles < pairs ? num_tiles : pairs;
        return launch_pdl_cluster(kernel, dim3(2 * pairs), dim3(C::kThreads), C::kBytes, stream, 2, m.a, m.b, m.o,
                                  m.r, m.r2, p);
    } else {
        const int num_tiles = ((p.M + kBM - 1) / kBM) * (p.N / BN);
        const int grid = num_tiles < num_sms() ? num_tiles : num_sms();
        return launch_pdl(kernel, dim3(grid), dim3(C::kThreads), C::kBytes, stream, m.a, m.b, m.o, m.r, m.r2, p);
    }
}

template <typename T, int BN>
cudaError_t dispatch_epi(int epi, const Maps& m, const GemmParams& p, cudaStream_t s)
{
    switch (epi) {
    case kEpiBias: return launch_one<T, BN, kEpiBias>(m, p, s);
    case kEpiBiasWsilu: return launch_one<T, BN, kEpiBiasWsilu>(m, p, s);
    case kEpiBiasRes: return launch_one<T, BN, kEpiBiasRes>(m, p, s);
    case kEpiBiasResQ: return launch_one<T, BN, kEpiBiasResQ>(m, p, s);
    case kEpiBiasRes2: return launch_one<T, BN, kEpiBiasRes2>(m, p, s);
    case kEpiQuad:
        if constexpr (BN == 256) {
            return launch_one<T, BN, kEpiQuad>(m, p, s);
        }
        return cudaErrorInvalidValue;
    case kEpiSubpel: return launch_one<T, BN, kEpiSubpel>(m, p, s);
    case kEpiBiasQ: return launch_one<T, BN, kEpiBiasQ>(m, p, s);
    default: return cudaErrorInvalidValue;
    }
}

// The FP8 form serves the DepthConvBlock GEMMs without a residual.
template <int BN>
cudaError_t dispatch_epi_f8(int epi, const Maps& m, const GemmParams& p, cudaStream_t s)
{
    switch (epi) {
    case kEpiBias: return launch_one<__nv_bfloat16, BN, kEpiBias, true>(m, p, s);
    case kEpiBiasWsilu: return launch_one<__nv_bfloat16, BN, kEpiBiasWsilu, true>(m, p, s);
    case kEpiQuad:
        if constexpr (BN == 256) {
            return launch_one<__nv_bfloat16, BN, kEpiQuad, true>(m, p, s);
        }
        return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int gemm_tuned_bn(int dtype, int epi, int M, int N, int K, int sub_w);

namespace {
std::atomic<int> g_stream_form{1};
std::atomic<int> g_dw_fusion{0};
std::atomic<int> g_pair_form{0};
}  // namespace

void gemm_set_pair_form(bool on) { g_pair_form.store(on ? 1 : 0); }

void gemm_set_stream_form(int form) { g_stream_form.store(form < 0 ? 0 : (form > 2 ? 2 : form)); }
bool gemm_stream_form_enabled() { return g_stream_form.load(std::memory_order_relaxed) != 0; }
void gemm_set_dw_fusion(bool on) { g_dw_fusion.store(on ? 1 : 0); }
bool gemm_dw_fusion_enabled() { return g_dw_fusion.load(std::memory_order_relaxed) != 0; }

int gemm_pick_bn(int M, int N, int epi, int sub_cout, int K)
{
    const int form = g_stream_form.load(std::memory_order_relaxed);
    const bool res = epi == kEpiBiasRes || epi == kEpiBiasResQ;
    if (K > 0 && (res ? form >= 1 : form >= 2) && gemm_stream_eligible(epi, M, N, K)) {
        // residual epilogues at K <= 256: the streaming form (W resident, row ranges per CTA)
        // moves the same bytes in 18.1 us where the tiled kernel takes 21.8 us (dc.3 / ffn.2 at
        // 1080p), with the same output bits; the bias / WSiLU epilogues at K <= 512 only when
        // asked for (form 2)
        return kBlockNStream;
    }
    if (epi == kEpiQuad) {
        if (N % 256 == 0 && g_pair_form.load(std::memory_order_relaxed) != 0 && num_sms() >= 2) {
            return kBlockNPair;
        }
        return N % 256 == 0 ? 256 : 0;  // the quad epilogue sums groups of 4 over BN/2 columns
    }
    int lim = (epi == kEpiSubpel) ? sub_cout : N;
    if (N % 256 == 0 && lim % 256 == 0) {
        // Small GEMMs (the y-level layers) with fewer 256-wide tiles than SMs run faster on twice
        // as many 128-wide tiles when the epilogue has no residual (dc.0 of a 512-channel block at
        // 1088 / 4 x 1920 / 4: 10.2 -> 8.1 us; the residual epilogues gain nothing).  The tile
        // width does not change any output bit.
        const long long tiles = static_cast<long long>((M + kBM - 1) / kBM) * (N / 256);
        if ((epi == kEpiBias || epi == kEpiBiasWsilu || epi == kEpiBiasQ) && tiles < num_sms()) {
            return 128;
        }
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

namespace {
std::atomic<int> g_stall_launches{0};
std::atomic<long long> g_stall_limit{0};
}  // namespace

void gemm_inject_stall(int launches, long long wait_limit_cycles)
{
    g_stall_limit.store(wait_limit_cycles);
    g_stall_launches.store(launches > 0 ? launches : 0);
}

GemmParams gemm_apply_injection(const GemmParams& p)
{
    GemmParams q = p;
    int n = g_stall_launches.load();
    while (n > 0 && !g_stall_launches.compare_exchange_weak(n, n - 1)) {
    }
    if (n > 0) {
        q.stall_test = 1;
        q.wait_limit = g_stall_limit.load();
    }
    return q;
}

// Host launcher.  A: [M, K] with row pitch lda (elements); W: [N, K] dense.  dtype 0 = f16,
// 1 = bf16, 2 = E4M3 operands with BF16 output.  Returns cudaSuccess or an error
// (shape/alignment problems -> cudaErrorInvalidValue).
cudaError_t gemm_sm100(int dtype, const void* A, int lda, const void* W, const GemmParams& p_in,
                       int epi, int bn, cudaStream_t stream)
{
    const GemmParams p = gemm_apply_injection(p_in);
    const bool f8 = dtype == kDtypeF8;
    if (dtype < 0 || dtype > kDtypeF8 || p.M <= 0 || p.N <= 0 || p.K <= 0 ||
        p.K % (f8 ? 128 : kBK) != 0 || lda % (f8 ? 16 : 8) != 0 ||
        (reinterpret_cast<uintptr_t>(A) & 15) != 0 || (reinterpret_cast<uintptr_t>(W) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(p.out) & 15) != 0 || p.ldo % 8 != 0) {
        return cudaErrorInvalidValue;
    }
    if (f8 && (p.wscale == nullptr || (reinterpret_cast<uintptr_t>(p.wscale) & 15) != 0 ||
               (epi != kEpiBias && epi != kEpiBiasWsilu && epi != kEpiQuad))) {
        return cudaErrorInvalidValue;
    }
    if (bn == 0) {
        // a width measured by the autotuner (gemm_tune.cu) for this shape, else the rule
        bn = gemm_tuned_bn(dtype, epi, p.M, p.N, p.K, epi == kEpiSubpel ? p.sub_w : 0);
        if (bn == 0) {
            bn = gemm_pick_bn(p.M, p.N, epi, p.sub_cout, p.K);
            if (bn == kBlockNPair && f8) {
                bn = 256;  // the pair form is built for 16-bit operands
            }
        }
    }
    if (bn == kBlockNStream) {
        return gemm_stream_sm100(dtype, A, lda, W, p, epi, stream);
    }
    if (p.out8 != nullptr || p.dw_weight != nullptr) {
        // the E4M3 side output and the depthwise operand exist in the streaming form only
        return cudaErrorInvalidValue;
    }
    const bool pair = bn == kBlockNPair;
    if (pair) {
        if (f8 || (epi != kEpiBias && epi != kEpiBiasWsilu && epi != kEpiQuad) || num_sms() < 2) {
            return cudaErrorInvalidValue;
        }
        bn = 256;
    }
    if (bn <= 0 || p.N % bn != 0) {
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
    if (epi == kEpiQuad && (bn != 256 || p.N % 256 != 0)) {
        return cudaErrorInvalidValue;
    }
    if (epi == kEpiSubpel && (p.sub_w <= 0 || p.sub_cout % bn != 0 || p.N != 4 * p.sub_cout ||
                              p.M % p.sub_w != 0)) {
        return cudaErrorInvalidValue;
    }
    // operands: 16-bit, or E4M3 bytes (staged as unsigned bytes); outputs/residuals: FP16, or
    // BF16 for the BF16 and FP8 forms
    const CUtensorMapDataType dt =
        dtype == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const CUtensorMapDataType dop = f8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : dt;
    const int esz = f8 ? 1 : 2;
    const int kbox = f8 ? 128 : kBK;
    Maps m;
    std::memset(&m, 0, sizeof(m));
    if (!make_tmap_2d(&m.a, dop, A, p.K, p.M, static_cast<uint64_t>(lda) * esz, kbox, kBM, 128) ||
        !make_tmap_2d(&m.b, dop, W, p.K, p.N, static_cast<uint64_t>(p.K) * esz, kbox, pair ? bn / 2 : bn, 128)) {
        return cudaErrorInvalidValue;
    }
    if (epi != kEpiSubpel) {
        const int ow = out_box_cols(bn, epi);
        const int sw = ow * 2;  // staging row bytes = swizzle span
        const int nout = epi == kEpiQuad ? p.N / 4 : p.N;
        if (!make_tmap_2d(&m.o, dt, p.out, nout, p.M, static_cast<uint64_t>(p.ldo) * 2, ow, 32, sw)) {
            return cudaErrorInvalidValue;
        }
        if (epi == kEpiBiasRes || epi == kEpiBiasResQ || epi == kEpiBiasRes2) {
            if (!make_tmap_2d(&m.r, dt, p.res, p.N, p.M, static_cast<uint64_t>(p.ldr) * 2, ow, 32, sw)) {
                return cudaErrorInvalidValue;
            }
        }
        if (epi == kEpiBiasRes2 &&
            !make_tmap_2d(&m.r2, dt, p.res2, p.N, p.M, static_cast<uint64_t>(p.ldr2) * 2, ow, 32, sw)) {
            return cudaErrorInvalidValue;
        }
    }
    if (pair) {
        switch (epi) {
        case kEpiBias:
            return dtype == 0 ? launch_one<__half, 256, kEpiBias, false, true>(m, p, stream)
                              : launch_one<__nv_bfloat16, 256, kEpiBias, false, true>(m, p, stream);
        case kEpiBiasWsilu:
            return dtype == 0 ? launch_one<__half, 256, kEpiBiasWsilu, false, true>(m, p, stream)
                              : launch_one<__nv_bfloat16, 256, kEpiBiasWsilu, false, true>(m, p, stream);
        case kEpiQuad:
            return dtype == 0 ? launch_one<__half, 256, kEpiQuad, false, true>(m, p, stream)
                              : launch_one<__nv_bfloat16, 256, kEpiQuad, false, true>(m, p, stream);
        }
        return cudaErrorInvalidValue;
    }
    if (f8) {
        switch (bn) {
        case 256: return dispatch_epi_f8<256>(epi, m, p, stream);
        case 128: return dispatch_epi_f8<128>(epi, m, p, stream);
        }
    } else if (dtype == 0) {
        switch (bn) {
        case 256: return dispatch_epi<__half, 256>(epi, m, p, stream);
        case 128: return dispatch_epi<__half, 128>(epi, m, p, stream);
        case 64: return dispatch_epi<__half, 64>(epi, m, p, stream);
        }
    } else {
        switch (bn) {
        case 256: return dispatch_epi<__nv_bfloat16, 256>(epi, m, p, stream);
        case 128: return dispatch_epi<__nv_bfloat16, 128>(epi, m, p, stream);
        case 64: return dispatch_epi<__nv_bfloat16, 64>(epi, m, p, stream);
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace dcvc
