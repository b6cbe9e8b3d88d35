// Fused ConvFFN of a DepthConvBlock (layers.py:115-125, layers_proxy.cpp:95-101) on tcgen05:
//
//   q   = sum_{k<4} WSiLU(x . W1[4c+k]^T + b1[4c+k])      (conv1x1_bias_wsilu_chunk_add)
//   out = (q . W2^T + b2 + x) [* qscale]                   (conv1x1_bias_shortcut[_with_quant])
//
// in one persistent kernel.  Per 128-row tile the quad items (256 ffn.0 columns each) write their
// 64 quad outputs straight into shared memory, laid out as one 128-byte-swizzled K block of the
// second GEMM's A operand; the ffn.2 items then read that block with tcgen05.mma and finish with
// the residual epilogue.  The quad output never goes to global memory and the block's two GEMM
// launches become one.  The arithmetic is that of the two separate GEMMs (gemm_sm100.cu): the
// same FP32 accumulation order, the quad output rounded to FP16 before the second GEMM, the same
// epilogues, so the result is bit-identical.
#include "ffn_sm100.cuh"

#include "host_util.h"

#include <cstring>
#include <mutex>

namespace dcvc {

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr int kEpiWarps = 8;     // two per TMEM lane quadrant, each owning half the columns
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr long long kWaitLimit = 2000000000LL;  // ~1 s at 2 GHz
constexpr int kSmemLimit = 232448;

// QB: K blocks of q (cffn / 64); BN: accumulator columns per item (256 or 128), the same for the
// quad items (BN ffn.0 columns -> BN / 4 quad outputs) and the output items (BN ffn.2 columns).
template <int QB, int BN>
struct FfnCfg {
    static constexpr int kABytes = kBM * kBK * 2;          // 16 KB: one K block of A (or of q)
    static constexpr int kBBytes = BN * kBK * 2;           // one K block of BN W1 or W2 rows
    static constexpr int kStageBytes = kABytes + kBBytes;
    static constexpr int kQBytes = QB * kABytes;           // one q buffer: QB K blocks
    static constexpr int kCols = BN / 2;                   // accumulator columns per epilogue warp
    static constexpr int kBoxes = kCols / 64;              // 64-column output boxes per warp
    static constexpr int kEpiBytes = kEpiWarps * kBoxes * 4096;  // residual / output boxes
    static constexpr int kBarBytes = 512;
    static constexpr int kStagesFit =
        (kSmemLimit - 1024 - 2 * kQBytes - kEpiBytes - kBarBytes) / kStageBytes;
    static constexpr int kStages = kStagesFit > 4 ? 4 : kStagesFit;
    static constexpr int kQOffset = kStages * kStageBytes;
    static constexpr int kEpiOffset = kQOffset + 2 * kQBytes;
    static constexpr int kBarOffset = kEpiOffset + kEpiBytes;
    static constexpr int kBytes = kBarOffset + kBarBytes + 1024;
    static constexpr int kTmemCols = 2 * BN;               // two accumulators
    static_assert(kStages >= 2, "shared memory too small for two pipeline stages");
    static_assert(kBytes <= kSmemLimit, "shared memory budget exceeded");
};

// Byte offset of 16-byte chunk j of row r in a 128-byte-swizzled tile (the layout TMA writes for
// SWIZZLE_128B and tcgen05 descriptors read).
__device__ __forceinline__ int sw128_off(int r, int j) { return r * 128 + ((j ^ (r & 7)) << 4); }

__device__ __forceinline__ uint32_t pack_h2(float a, float b)
{
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ float2 unpack_h2(uint32_t u)
{
    __half2 h = *reinterpret_cast<__half2*>(&u);
    return __half22float2(h);
}

template <int QB, int BN, bool HASQ>
__global__ void __launch_bounds__(kThreads, 1)
    ffn_sm100_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmW1,
                     const __grid_constant__ CUtensorMap tmW2, const __grid_constant__ CUtensorMap tmR,
                     const __grid_constant__ CUtensorMap tmO, const FfnParams p)
{
    using C = FfnCfg<QB, BN>;
    constexpr int kStages = C::kStages;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem =
        reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* qbuf = smem + C::kQOffset;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::kBarOffset);
    uint64_t* empty = full + kStages;
    uint64_t* tfull = empty + kStages;
    uint64_t* tempty = tfull + 2;
    uint64_t* qfull = tempty + 2;    // [2]: all quad items of a tile have written its q buffer
    uint64_t* qempty = qfull + 2;    // [2]: the ffn.2 MMAs of a tile have read its q buffer
    uint64_t* drain = qempty + 2;
    uint64_t* resbar = drain + 1;    // [kEpiWarps][C::kBoxes]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(resbar + C::kBoxes * kEpiWarps);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int num_m = (p.M + kBM - 1) / kBM;
    const int nq = 4 * QB * kBK / BN; // quad items per tile (BN / 4 quad outputs each)
    const int nr = p.C / BN;          // output items per tile
    const int kx = p.C / kBK;         // K blocks of x
    // This CTA's tiles are blockIdx.x + j * gridDim.x, j < ntiles.  Work runs in rounds: round j
    // holds the quad items of tile j (while j < ntiles), then the output items of tile j - 1
    // (from j = 1), so a tile's output items overlap the next tile's quad items; tile j uses q
    // buffer j % 2.  The three roles walk the same rounds.
    const int ntiles = blockIdx.x < num_m ? (num_m - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], kEpiWarps);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&qfull[b], kEpiWarps);
            mbar_init(&qempty[b], 1);
        }
        mbar_init(drain, 1);
        for (int w = 0; w < C::kBoxes * kEpiWarps; ++w) {
            mbar_init(&resbar[w], 1);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        tma_prefetch_desc(&tmX);
        tma_prefetch_desc(&tmW1);
        tma_prefetch_desc(&tmW2);
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, C::kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    griddep_launch_dependents();
    griddep_wait();

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int issued = 0;
            for (int j = 0; j <= ntiles && !*abort_flag; ++j) {
                for (int it = 0; it < nq + nr && !*abort_flag; ++it) {
                    const bool quad = it < nq;
                    if (quad ? j == ntiles : j == 0) {
                        continue;
                    }
                    const int m0 = (blockIdx.x + j * gridDim.x) * kBM;  // quad items only
                    const int kbs = quad ? kx : QB;
                    for (int kb = 0; kb < kbs; ++kb) {
                        if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimit)) {
                            *abort_flag = 1;
                            report_error(p.err, kErrGemmProducerTimeout);
                            break;
                        }
                        uint8_t* sa = smem + stage * C::kStageBytes;
                        if (quad) {
                            mbar_arrive_expect_tx(&full[stage], C::kStageBytes);
                            tma_load_2d(sa, &tmX, &full[stage], kb * kBK, m0);
                            tma_load_2d(sa + C::kABytes, &tmW1, &full[stage], kb * kBK, it * BN);
                        } else {
                            mbar_arrive_expect_tx(&full[stage], C::kBBytes);
                            tma_load_2d(sa + C::kABytes, &tmW2, &full[stage], kb * kBK,
                                        (it - nq) * BN);
                        }
                        ++issued;
                        if (++stage == kStages) {
                            stage = 0;
                            phase ^= 1;
                        }
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
            const uint32_t idesc = make_idesc_f16(kBM, BN, 0);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            bool issued_any = false;
            for (int j = 0; j <= ntiles && !*abort_flag; ++j) {
                for (int it = 0; it < nq + nr && !*abort_flag; ++it) {
                    const bool quad = it < nq;
                    if (quad ? j == ntiles : j == 0) {
                        continue;
                    }
                    const int jt = quad ? j : j - 1;  // the item's tile
                    const uint8_t* qb = qbuf + (jt & 1) * C::kQBytes;
                    if (it == nq) {
                        // q of tile jt is complete in shared memory
                        if (!mbar_wait_bounded(&qfull[jt & 1], (jt >> 1) & 1, kWaitLimit)) {
                            *abort_flag = 1;
                            report_error(p.err, kErrGemmMmaTimeout);
                            break;
                        }
                        tc_fence_after();
                    }
                    if (!mbar_wait_bounded(&tempty[acc], acc_phase ^ 1, kWaitLimit)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmMmaTimeout);
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem_base + static_cast<uint32_t>(acc * BN);
                    const int kbs = quad ? kx : QB;
                    for (int kb = 0; kb < kbs; ++kb) {
                        if (!mbar_wait_bounded(&full[stage], phase, kWaitLimit)) {
                            *abort_flag = 1;
                            report_error(p.err, kErrGemmMmaTimeout);
                            break;
                        }
                        tc_fence_after();
                        const uint8_t* sa = smem + stage * C::kStageBytes;
                        const uint8_t* a = quad ? sa : qb + kb * C::kABytes;
                        const uint64_t adesc = make_sw128_kmajor_desc(smem_u32(a));
                        const uint64_t bdesc = make_sw128_kmajor_desc(smem_u32(sa + C::kABytes));
#pragma unroll
                        for (int kk = 0; kk < kBK / 16; ++kk) {
                            tc_mma_f16(d, adesc + 2 * kk, bdesc + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
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
                if (*abort_flag) {
                    break;
                }
                if (j >= 1) {
                    // tile j - 1's q buffer may be reused once its ffn.2 MMAs complete
                    tc_commit(&qempty[(j - 1) & 1]);
                }
            }
            if (*abort_flag && issued_any) {
                tc_commit(drain);
                mbar_wait_bounded(drain, 0, kWaitLimit / 16);
            }
        }
    } else {
        // ------------------------------------------------------------ epilogue warps
        const int ew = warp - 2;
        const int quad_lanes = warp & 3;          // TMEM lane quadrant this warp may access
        const int half = ew >> 2;                 // which half of the item's 256 columns
        uint8_t* wbuf = smem + C::kEpiOffset + ew * C::kBoxes * 4096;  // box b at wbuf + 4096 b
        uint64_t* rbar = &resbar[C::kBoxes * ew];
        uint32_t res_phase = 0;
        bool res_pending = false;
        int acc = 0;
        uint32_t acc_phase = 0;
        if (lane == 0) {
            tma_prefetch_desc(&tmO);
            tma_prefetch_desc(&tmR);
        }
        const int r = quad_lanes * 32 + lane;        // this lane's row inside a tile
        for (int j = 0; j <= ntiles && !*abort_flag; ++j) {
            for (int it = 0; it < nq + nr && !*abort_flag; ++it) {
                const bool quad = it < nq;
                if (quad ? j == ntiles : j == 0) {
                    continue;
                }
                const int jt = quad ? j : j - 1;        // the item's tile
                const int row0 = (blockIdx.x + jt * gridDim.x) * kBM + quad_lanes * 32;
                const bool rows_live = row0 < p.M;
                uint8_t* qb = qbuf + (jt & 1) * C::kQBytes;
                if (quad && it == 0 && jt >= 2) {
                    // tile jt - 2's ffn.2 MMAs must have read this q buffer before it is reused
                    if (!mbar_wait_bounded(&qempty[jt & 1], ((jt >> 1) - 1) & 1, kWaitLimit)) {
                        *abort_flag = 1;
                        report_error(p.err, kErrGemmEpilogueTimeout);
                        break;
                    }
                }
                const int ncol0 = (it - nq) * BN + half * C::kCols;
                if (!quad && rows_live && lane == 0) {
                    // the residual (x) of both boxes, in flight while the accumulator finishes
                    bulk_wait_read0();  // the previous item's stores have read the buffers
                    for (int b = 0; b < C::kBoxes; ++b) {
                        mbar_arrive_expect_tx(&rbar[b], 4096);
                        tma_load_2d(wbuf + 4096 * b, &tmR, &rbar[b], ncol0 + b * 64, row0);
                    }
                    res_pending = true;
                }
                if (!mbar_wait_bounded(&tfull[acc], acc_phase, kWaitLimit)) {
                    *abort_flag = 1;
                    report_error(p.err, kErrGemmEpilogueTimeout);
                    break;
                }
                tc_fence_after();
                const uint32_t tbase = tmem_base + (static_cast<uint32_t>(quad_lanes * 32) << 16) +
                                       acc * BN + half * C::kCols;
                if (quad) {
                    // kCols accumulator columns -> kCols / 4 quad outputs of this row, written as
                    // 16-byte chunks (8 outputs) into q: quad output j lives in K block j / 64,
                    // chunk (j % 64) / 8
                    const int q0 = (it * BN + half * C::kCols) / 4;  // first quad output
                    uint8_t* qblk = qb + (q0 / 64) * C::kABytes;
#pragma unroll 1
                    for (int c = 0; c < C::kCols / 32; ++c) {
                        const int nc = it * BN + half * C::kCols + c * 32;
                        const float4* b4 = reinterpret_cast<const float4*>(p.b1 + nc);
                        float4 bb[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            bb[j] = __ldg(b4 + j);
                        }
                        uint32_t rr[32];
                        tmem_ld_32x32b_x32(tbase + c * 32, rr);
                        tc_wait_ld();
                        float v[32];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            v[4 * j + 0] = __uint_as_float(rr[4 * j + 0]) + bb[j].x;
                            v[4 * j + 1] = __uint_as_float(rr[4 * j + 1]) + bb[j].y;
                            v[4 * j + 2] = __uint_as_float(rr[4 * j + 2]) + bb[j].z;
                            v[4 * j + 3] = __uint_as_float(rr[4 * j + 3]) + bb[j].w;
                        }
                        uint32_t o[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const float s0 = wsilu(v[8 * i + 0]) + wsilu(v[8 * i + 1]) +
                                             wsilu(v[8 * i + 2]) + wsilu(v[8 * i + 3]);
                            const float s1 = wsilu(v[8 * i + 4]) + wsilu(v[8 * i + 5]) +
                                             wsilu(v[8 * i + 6]) + wsilu(v[8 * i + 7]);
                            o[i] = pack_h2(s0, s1);
                        }
                        *reinterpret_cast<uint4*>(qblk + sw128_off(r, (q0 % 64) / 8 + c)) =
                            make_uint4(o[0], o[1], o[2], o[3]);
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) {
                        mbar_arrive(&tempty[acc]);
                    }
                    if (it == nq - 1) {
                        // q complete for this warp's rows: visible to the tensor cores
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0) {
                            mbar_arrive(&qfull[jt & 1]);
                        }
                    }
                } else {
                    // ffn.2 output: 128 columns per warp in two 64-column boxes; the result is
                    // written over the box's residual and stored from there
#pragma unroll 1
                    for (int b = 0; b < C::kBoxes; ++b) {
                        const int ncol = ncol0 + b * 64;
                        uint8_t* box = wbuf + 4096 * b;
                        if (rows_live) {
                            if (!mbar_wait_bounded(&rbar[b], res_phase, kWaitLimit)) {
                                *abort_flag = 1;
                                report_error(p.err, kErrGemmEpilogueTimeout);
                            }
                        }
                        __syncwarp();
#pragma unroll 1
                        for (int c = 0; c < 2; ++c) {
                            const int nc = ncol + c * 32;
                            const float4* b4 = reinterpret_cast<const float4*>(p.b2 + nc);
                            float4 bb[8];
                            if constexpr (!HASQ) {
#pragma unroll
                                for (int j = 0; j < 8; ++j) {
                                    bb[j] = __ldg(b4 + j);
                                }
                            }
                            uint32_t rr[32];
                            tmem_ld_32x32b_x32(tbase + b * 64 + c * 32, rr);
                            tc_wait_ld();
                            float v[32];
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                const float4 bj = HASQ ? __ldg(b4 + j) : bb[j];
                                v[4 * j + 0] = __uint_as_float(rr[4 * j + 0]) + bj.x;
                                v[4 * j + 1] = __uint_as_float(rr[4 * j + 1]) + bj.y;
                                v[4 * j + 2] = __uint_as_float(rr[4 * j + 2]) + bj.z;
                                v[4 * j + 3] = __uint_as_float(rr[4 * j + 3]) + bj.w;
                            }
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const uint4 u = *reinterpret_cast<const uint4*>(
                                    box + sw128_off(lane, c * 4 + j));
                                const float2 a = unpack_h2(u.x), bq = unpack_h2(u.y),
                                             cc = unpack_h2(u.z), dd = unpack_h2(u.w);
                                v[8 * j + 0] += a.x;
                                v[8 * j + 1] += a.y;
                                v[8 * j + 2] += bq.x;
                                v[8 * j + 3] += bq.y;
                                v[8 * j + 4] += cc.x;
                                v[8 * j + 5] += cc.y;
                                v[8 * j + 6] += dd.x;
                                v[8 * j + 7] += dd.y;
                            }
                            if constexpr (HASQ) {
                                const uint4* qs = reinterpret_cast<const uint4*>(
                                    reinterpret_cast<const __half*>(p.qscale) + nc);
#pragma unroll
                                for (int j = 0; j < 4; ++j) {
                                    const uint4 u = __ldg(qs + j);
                                    const float2 a = unpack_h2(u.x), bq = unpack_h2(u.y),
                                                 cc = unpack_h2(u.z), dd = unpack_h2(u.w);
                                    v[8 * j + 0] *= a.x;
                                    v[8 * j + 1] *= a.y;
                                    v[8 * j + 2] *= bq.x;
                                    v[8 * j + 3] *= bq.y;
                                    v[8 * j + 4] *= cc.x;
                                    v[8 * j + 5] *= cc.y;
                                    v[8 * j + 6] *= dd.x;
                                    v[8 * j + 7] *= dd.y;
                                }
                            }
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                *reinterpret_cast<uint4*>(box + sw128_off(lane, c * 4 + j)) =
                                    make_uint4(pack_h2(v[8 * j + 0], v[8 * j + 1]),
                                               pack_h2(v[8 * j + 2], v[8 * j + 3]),
                                               pack_h2(v[8 * j + 4], v[8 * j + 5]),
                                               pack_h2(v[8 * j + 6], v[8 * j + 7]));
                            }
                        }
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0 && rows_live) {
                            tma_store_2d(&tmO, box, ncol, row0);
                            bulk_commit();
                        }
                        __syncwarp();
                    }
                    if (rows_live) {
                        res_phase ^= 1;
                        res_pending = false;
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) {
                        mbar_arrive(&tempty[acc]);
                    }
                }
                acc ^= 1;
                if (acc == 0) {
                    acc_phase ^= 1;
                }
            }
        }
        if (lane == 0) {
            if (res_pending) {
                // after an abort, let this warp's residual loads land before the CTA winds down
                for (int b = 0; b < C::kBoxes; ++b) {
                    mbar_wait_bounded(&rbar[b], res_phase, kWaitLimit / 16);
                }
            }
            bulk_wait_read0();
        }
        __syncwarp();
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, C::kTmemCols);
    }
}

template <int QB, int BN, bool HASQ>
cudaError_t launch_ffn(const CUtensorMap (&m)[5], const FfnParams& p, cudaStream_t stream)
{
    using C = FfnCfg<QB, BN>;
    auto kernel = ffn_sm100_kernel<QB, BN, HASQ>;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [&] {
        attr_err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, C::kBytes);
    });
    if (attr_err != cudaSuccess) {
        return attr_err;
    }
    const int num_m = (p.M + kBM - 1) / kBM;
    const int grid = num_m < num_sms() ? num_m : num_sms();
    return launch_pdl(kernel, dim3(grid), dim3(kThreads), C::kBytes, stream, m[0], m[1], m[2],
                      m[3], m[4], p);
}

}  // namespace

bool ffn_sm100_supported(int C, int cffn, int n1)
{
    return C > 0 && C % 256 == 0 && (cffn == 128 || cffn == 256) && n1 == 4 * cffn;
}

bool ffn_sm100_preferred(int C, int cffn, int n1)
{
    // With cffn = 256 the fused kernel is slower than the two GEMMs (88 us against 33 + 22 us for
    // a 512-channel block at 1080p): two 64 KB q buffers leave two 32 KB operand stages, and the
    // pipeline starves.  With cffn = 128 it is faster (a 256-channel block at 1080p: 22.5 us; the
    // LD codec gains 8-10 % per frame).
    return ffn_sm100_supported(C, cffn, n1) && cffn == 128;
}

cudaError_t ffn_sm100(const void* x, int ldx, const void* w1, const void* w2, const FfnParams& p,
                      cudaStream_t stream)
{
    if (p.M <= 0 || !ffn_sm100_supported(p.C, p.cffn, 4 * p.cffn) || ldx % 8 != 0 ||
        p.ldo % 8 != 0 || p.b1 == nullptr || p.b2 == nullptr || p.out == nullptr ||
        (reinterpret_cast<uintptr_t>(x) & 15) != 0 || (reinterpret_cast<uintptr_t>(w1) & 15) != 0 ||
        (reinterpret_cast<uintptr_t>(w2) & 15) != 0 || (reinterpret_cast<uintptr_t>(p.out) & 15) != 0) {
        return cudaErrorInvalidValue;
    }
    const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    CUtensorMap m[5];
    std::memset(m, 0, sizeof(m));
    const uint64_t xrow = static_cast<uint64_t>(ldx) * 2;
    const int n1 = 4 * p.cffn;
    // item width: 256 for q 128 wide; q 256 wide (two 64 KB q buffers) leaves room for 128 only
    const int bn = p.block_n != 0 ? p.block_n : (p.cffn == 128 ? 256 : 128);
    if ((bn != 128 && bn != 256) || (p.cffn == 256 && bn != 128)) {
        return cudaErrorInvalidValue;
    }
    if (!make_tmap_2d(&m[0], dt, x, p.C, p.M, xrow, kBK, kBM, 128) ||
        !make_tmap_2d(&m[1], dt, w1, p.C, n1, static_cast<uint64_t>(p.C) * 2, kBK, bn, 128) ||
        !make_tmap_2d(&m[2], dt, w2, p.cffn, p.C, static_cast<uint64_t>(p.cffn) * 2, kBK, bn, 128) ||
        !make_tmap_2d(&m[3], dt, x, p.C, p.M, xrow, 64, 32, 128) ||
        !make_tmap_2d(&m[4], dt, p.out, p.C, p.M, static_cast<uint64_t>(p.ldo) * 2, 64, 32, 128)) {
        return cudaErrorInvalidValue;
    }
    const bool q = p.qscale != nullptr;
    if (p.cffn == 128) {
        if (bn == 256) {
            return q ? launch_ffn<2, 256, true>(m, p, stream) : launch_ffn<2, 256, false>(m, p, stream);
        }
        return q ? launch_ffn<2, 128, true>(m, p, stream) : launch_ffn<2, 128, false>(m, p, stream);
    }
    return q ? launch_ffn<4, 128, true>(m, p, stream) : launch_ffn<4, 128, false>(m, p, stream);
}

}  // namespace dcvc
