// DCVC-UF HT-S chunk codec runtime: the B200 counterpart of DMCHTSProxy
// (src/layers/extensions/inference/dmc_hts_proxy.{h,cpp}).
#pragma once

#include "codec_common.h"
#include "net.h"
#include "rans_coder.h"

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

namespace dcvc {

class HtsCodec {
public:
    static constexpr int kFrames = 8;       // g_frame_delay (video_model_ht.py:16)
    static constexpr int kChSrcIntra = 192; // 3 * 8 * 8
    static constexpr int kChSrc = 1536;
    static constexpr int kChY = 256, kChZ = 128, kChD = 512, kChM = 512, kChRecon = 256;
    static constexpr int kQpNum = 64;

    // Activation format of the analysis and synthesis transforms (encoder, decoder, recon head,
    // feature adaptors and extractor): FP16 as the reference, or BF16.  The entropy-parameter
    // path (hyper encoder / decoder, temporal prior, prior fusion, spatial prior, quantisation
    // and indexes) runs in FP16 in every form, with the same kernels on the encoder and the
    // decoder side, so symbols and CDF indexes round-trip exactly in both.
    // kPrecisionFP8 is the BF16 form with the DepthConvBlocks' quad GEMMs (ffn.0, the largest
    // GEMM of every block) on E4M3 operands with per-output-channel scales.
    enum Precision : int { kPrecisionF16 = 0, kPrecisionBF16 = 1, kPrecisionFP8 = 2 };

    HtsCodec();
    ~HtsCodec();

    // Selects the precision form; takes effect at the next set_param.
    int set_precision(int precision);
    int precision() const { return precision_; }

    // set_param (dmc_hts_proxy.cpp:712-762): weights + CDF tables + skip threshold.
    int set_param(const StateDict& sd, float skip_threshold);
    // add_ref_feature_from_frame (dmc_hts_proxy.cpp:492-502): frame is [Hp, Wp, 3] FP16 on the
    // device, Hp and Wp multiples of 16.
    int add_ref_feature(const __half* frame, int Hp, int Wp, bool apply_adaptor, cudaStream_t s);
    // compress (dmc_hts_proxy.cpp:504-585): x is [H, W, 24] FP16 (8 frames x YUV, channels last)
    // with H + pad_b and W + pad_r equal to the resolution of the last add_ref_feature.
    int compress(const __half* x, int H, int W, int qp, bool reset, int pad_b, int pad_r,
                 cudaStream_t s, std::vector<uint8_t>* bytes, int* ec_parallel);
    // decompress (dmc_hts_proxy.cpp:587-710): returns 8 device frames [Hp, Wp, 3] FP16 owned by
    // the codec and overwritten by the next call.
    int decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                   bool reset, cudaStream_t s, const __half** frames);

    // Packed batches: n streams of one resolution coded together, every layer of the network one
    // launch over the n images stacked along the rows (the 1x1 GEMMs see n times the pixels; the
    // depthwise convolutions and checkerboard masks keep each image's own borders and parity; each
    // stream has its own QP rows and its own rANS payload, coded on its own host thread).  The
    // temporal state of all n streams lives in this codec; add_ref_features sizes it for n
    // streams.  One reset flag covers the batch.  Each stream's payload and reconstruction are
    // bitwise those of a single-stream codec given the same inputs.  decompress_batch returns 8
    // frames, each [n * Hp, Wp, 3] with stream k's frame in rows k * Hp ..
    static constexpr int kMaxBatch = 64;
    int add_ref_features(const __half* const* frames, int n, int Hp, int Wp, bool apply_adaptor,
                         cudaStream_t s);
    int compress_batch(const __half* const* xs, int n, int H, int W, const int* qps, bool reset,
                       int pad_b, int pad_r, cudaStream_t s, std::vector<uint8_t>* bytes,
                       int* ec_parallel);
    int decompress_batch(const uint8_t* const* bytes, const size_t* sizes, const int* qps,
                         const int* ecps, int n, int height, int width, bool reset, cudaStream_t s,
                         const __half** frames);
    int batch_size() const { return imgs_; }

    // Read-only view of an internal buffer for inspection and tests: "y_hat", "y_q", "memory",
    // "ctx", "feature_p", "common", "feature_i".  rows x cols 16-bit values with pitch ld, in the
    // format *dtype (0 FP16, 1 BF16: "memory", "ctx", "feature_p" and "feature_i" follow the
    // precision form, the others are FP16).
    int buffer(const std::string& name, const void** ptr, int* rows, int* cols, int* ld,
               int* dtype = nullptr) const;

    // Uses the prepared parameters of `other` (same device) instead of a copy of its own: every
    // parameter device buffer is shared and held until the last codec using it is destroyed or
    // re-parameterised.  The counterpart of one set_param with the same state dict.
    int share_params(const HtsCodec& other);

    // The per-stream temporal context (memory and decoded feature, ctx, the I-frame feature and
    // whether memory holds a value), so that a stream's state can live outside the codec that
    // codes it: a serving loop keeps one state per stream and runs its chunks on whichever codec
    // of that resolution is free.  export/import copy device to device on the caller's stream
    // and order the codec's own stream after the copies; the layout is private to this build.
    size_t state_bytes() const;
    int export_state(void* dst, cudaStream_t s, int* flags);
    int import_state(const void* src, int flags, cudaStream_t s);

    // Statistics of the last call, for reporting.
    int last_symbol_count() const { return last_count_; }
    size_t device_bytes() const { return (weights_ ? weights_->bytes() : 0) + acts_.bytes(); }
    size_t activation_bytes() const { return acts_.bytes(); }
    // Number of kernels the last compress/decompress enqueued (graph nodes included).
    int last_kernel_count() const { return last_kernels_; }
    // Phase timing of the following calls (off by default): CUDA events around every phase graph
    // and host clocks around the host's waits and entropy coding.  timing() fills up to `cap`
    // values (milliseconds; -1 for a phase the last compress / decompress did not run) in the
    // order of kTimingNames and returns how many it wrote.
    void set_timing(bool on);
    // Process-wide: how many concurrent branches codecs allocated after the call give the 8-frame
    // recon head of a decoded chunk (1, 2 or 4).
    static void set_recon_branches(int n);
    int timing(float* out, int cap);
    static constexpr int kTimingValues = 13;
    void begin_timing()
    {
        for (bool& u : tev_used_) {
            u = false;
        }
        for (float& h : host_ms_) {
            h = -1.f;
        }
    }

private:
    enum Phase {
        kEncAnalysis = 0,    // enc_0 (dmc_hts_proxy.cpp:516-559)
        kEncUpdate = 1,      // enc_1 (2 variants: reset)
        kDecTemporal = 3,    // dec_0 (2 variants: memory has value)
        kDecHyper = 5,       // dec_1
        kDecContext = 6,     // dec_2
        kDecSynthesis = 7,   // dec_3
        kPhaseSlots = 8,
    };

    int allocate(int Hp, int Wp, int imgs);
    void clear_graphs();
    int run_phase(int slot, cudaStream_t s);
    void record_phase(int slot, Launch& L);

    // phase bodies (enqueue onto L.s)
    void enc_analysis(Launch& L);
    void enc_update(Launch& L, bool reset);
    void dec_temporal(Launch& L, bool memory_has_value);
    void dec_hyper(Launch& L);
    void dec_context(Launch& L);
    void dec_synthesis(Launch& L);
    // shared pieces
    void feature_adaptor_m(Launch& L);
    void feature_adaptor_i(Launch& L, const __half* feature_i);
    void feature_extractor(Launch& L);
    // temporal prior into cat_pf_[256:768] with the given working buffers (the main ones, or the
    // side branch's in enc_analysis)
    void temporal_prior(Launch& L, __half* s2d, __half* lvl16, Scratch& sc);
    void hyper_decoder(Launch& L);
    void prior_fusion(Launch& L);
    void spatial_prior(Launch& L, int k);
    void decoder(Launch& L);
    void recon_head(Launch& L, bool all_frames);
    void set_qp(const int* qps, cudaStream_t s);  // one QP per stream of the batch

    // ---------------------------------------------------------------- parameters
    std::shared_ptr<DeviceArena> weights_;  // shared by codecs that share_params
    bool ready_ = false;
    int precision_ = kPrecisionF16;  // requested form
    int act_ = 0;                    // activation format of the transforms as set up (0 / 1)
    bool fp8_ = false;               // FP8 quad GEMMs in the transforms (as set up)
    float skip_threshold_ = 0.f;
    __half skip_thr_half_;
    const __half* q_enc_tab_ = nullptr;   // [64][512]
    const __half* q_dec_tab_ = nullptr;
    const __half* q_feat_tab_ = nullptr;
    uint8_t* scale_lut_ = nullptr;         // [65536]
    Dcb encoder_[6];
    Lin enc_down_;
    Dcb hyper_enc0_;
    DownBlock hyper_enc1_, hyper_enc2_;
    UpBlock hyper_dec0_, hyper_dec1_;
    Dcb hyper_dec2_;
    DownBlock temporal_;
    Dcb prior_fusion_[3];
    Lin prior_fusion_out_;
    Lin reduction_;
    Dcb sp_adaptor_[3];
    Dcb spatial_prior_[3];
    Lin spatial_prior_out_;
    UpBlock dec_up_;   // only .up is used (decoder.up), the DCB chain is decoder_[]
    Lin dec_up_lin_;
    Dcb decoder_[7];
    Dcb fa_i_[4];
    Dcb fa_m_[6];
    Dcb fe_[5];
    Dcb rh_common_[4];
    Dcb rh_frame_[8][3];
    Lin rh_head_[8];
    RansTables tables_;

    // ---------------------------------------------------------------- resolution state
    DeviceArena acts_;
    int Hp_ = 0, Wp_ = 0, H8_ = 0, W8_ = 0, H16_ = 0, W16_ = 0, H16p_ = 0, W16p_ = 0;
    int M8_ = 0, M16_ = 0, M16p_ = 0, M32_ = 0, M64_ = 0;  // rows over all images of the batch
    int y_num_ = 0, z_num_ = 0;
    // packed batch: images, their rows stacked (TH*), rows of one image (m*), latents of one image
    int imgs_ = 0;
    int TH8_ = 0, TH16_ = 0, TH16p_ = 0, TH32_ = 0, TH64_ = 0;
    int m8_ = 0, m16_ = 0, m16p_ = 0;
    int ny_ = 0, nz_ = 0;
    __half *cat_enc_ = nullptr, *cat_fam_ = nullptr, *feature_i_ = nullptr, *temporal_in_ = nullptr;
    __half *y_ = nullptr, *y_pad_ = nullptr, *cat_pf_ = nullptr, *hyper_pad_ = nullptr;
    __half *common_ = nullptr, *cat_spa_ = nullptr, *means_ = nullptr, *y_q_ = nullptr;
    __half *z_ = nullptr, *z_hat_ = nullptr, *col_ = nullptr, *s2d_ = nullptr;
    __half *lvl8_a_ = nullptr, *lvl8_b_ = nullptr, *lvl16_a_ = nullptr, *lvl32_a_ = nullptr;
    __half *lvl64_a_ = nullptr, *head_ = nullptr;
    __half *y_act_ = nullptr, *yhat_act_ = nullptr;  // y and y_hat in the BF16 form's format
    __half *q_enc_ = nullptr, *q_dec_ = nullptr, *q_feat_ = nullptr;  // active QP rows
    __half* x_hat_[kFrames] = {nullptr};
    int8_t* z_i8_ = nullptr;
    int16_t *sym_ = nullptr, *sym_c_ = nullptr;
    uint8_t *idx_ = nullptr, *idx_c_ = nullptr, *cond_ = nullptr;
    int8_t* y_dec_ = nullptr;
    int* block_counts_ = nullptr;
    int* count_dev_ = nullptr;
    Scratch scratch_;
    // the further branches of a decoded chunk's recon head (branch b > 0 on side_[b - 1] with
    // its own buffers, concurrently with branch 0 on main_; allocated at allocation time)
    static constexpr int kMaxReconBranches = 4;
    int recon_branches_ = 1;
    __half *rb_a_[kMaxReconBranches] = {}, *rb_b_[kMaxReconBranches] = {}, *rb_head_[kMaxReconBranches] = {};
    Scratch rb_scratch_[kMaxReconBranches];
    // enc_analysis runs the temporal prior as a side branch, concurrently with the encoder
    __half *s2d_t_ = nullptr, *lvl16_t_ = nullptr;
    Scratch scratch_t_;
    // pinned host staging
    int* count_host_ = nullptr;
    int16_t* sym_host_ = nullptr;
    uint8_t* idx_host_ = nullptr;
    int8_t* ydec_host_ = nullptr;
    int8_t* z_host_ = nullptr;
    // device addresses of the mapped host buffers above: the phase graphs move symbols, indexes,
    // decoded values and their counts through them (launch_copy_counted)
    int* count_hdev_ = nullptr;
    int16_t* sym_hdev_ = nullptr;
    uint8_t* idx_hdev_ = nullptr;
    int8_t* ydec_hdev_ = nullptr;
    int8_t* z_hdev_ = nullptr;
    bool memory_has_value_ = false;

    PhaseGraphs graphs_{kPhaseSlots};
    cudaStream_t main_ = nullptr;   // compute stream (graphs run here)
    cudaStream_t side_[kMaxReconBranches - 1] = {};  // the recon head's further branches
    cudaEvent_t ev_fork_ = nullptr, ev_join_[kMaxReconBranches - 1] = {};
    cudaEvent_t ev_in_ = nullptr, ev_phase_ = nullptr, ev_out_ = nullptr;
    cudaEvent_t ev_state_ = nullptr;  // state copies on a caller's stream, waited for by main_
    // phase timing (set_timing): events before / after each phase slot, host intervals
    bool timing_ = false;
    cudaEvent_t tev_[8][2] = {};
    bool tev_used_[8] = {};
    float host_ms_[5] = {-1.f, -1.f, -1.f, -1.f, -1.f};
    int* err_word_ = nullptr;
    ErrorSlot err_slot_;  // the error word as the phase graphs publish it
    int last_count_ = 0;
    int last_kernels_ = 0;
    int dev_ = 0;
};

}  // namespace dcvc
