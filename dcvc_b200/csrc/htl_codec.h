// DCVC-UF HT-L chunk codec runtime: the B200 counterpart of DMCHTLProxy
// (src/layers/extensions/inference/dmc_htl_proxy.{h,cpp}).  The HT-S temporal dataflow with the
// HT-L modules (plain DepthConvBlocks, biased 3x3 sub-pixel decoder up-sampling, shortcut
// resampling blocks, per-frame recon heads) and 4-step entropy coding whose steps 1-3 take their
// scales from the spatial prior.
#pragma once

#include "codec_common.h"
#include "net.h"
#include "rans_coder.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace dcvc {

class HtlCodec {
public:
    static constexpr int kFrames = 8;
    static constexpr int kChSrcIntra = 192;
    static constexpr int kChSrc = 1536;
    static constexpr int kChY = 256, kChZ = 128, kChD = 512, kChM = 512, kChRecon = 256;
    static constexpr int kQpNum = 64;
    static constexpr int kSteps = 4;

    HtlCodec();
    ~HtlCodec();

    // set_param (dmc_htl_proxy.cpp:917-967).
    int set_param(const StateDict& sd, float skip_threshold);
    // add_ref_feature_from_frame (dmc_htl_proxy.cpp:583-593): frame [Hp, Wp, 3] FP16.
    int add_ref_feature(const __half* frame, int Hp, int Wp, bool apply_adaptor, cudaStream_t s);
    // compress (dmc_htl_proxy.cpp:595-716): x [H, W, 24] FP16.
    int compress(const __half* x, int H, int W, int qp, bool reset, int pad_b, int pad_r,
                 cudaStream_t s, std::vector<uint8_t>* bytes, int* ec_parallel);
    // decompress (dmc_htl_proxy.cpp:718-915): 8 device frames [Hp, Wp, 3] FP16 owned by the codec.
    int decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                   bool reset, cudaStream_t s, const __half** frames);

    // "y_hat", "y_q", "memory", "ctx", "feature_p", "common", "feature_i".
    int buffer(const std::string& name, const void** ptr, int* rows, int* cols, int* ld) const;

    int last_symbol_count() const { return last_count_; }
    size_t device_bytes() const { return weights_.bytes() + acts_.bytes(); }
    int last_kernel_count() const { return last_kernels_; }

private:
    enum Phase {
        kEncAnalysis = 0,   // lambda_enc_0 (dmc_htl_proxy.cpp:607-689)
        kEncUpdate = 1,     // lambda_enc_1 (:702-706), 2 variants: reset
        kDecTemporal = 3,   // lambda_dec_0 (:742-747), 2 variants: memory has value
        kDecHyper = 5,      // lambda_dec_1 (:765-783)
        kDecStep = 6,       // lambda_dec_2..4 (:803-876), slots 6, 7, 8
        kDecFinal = 9,      // lambda_dec_5 (:896-908)
        kPhaseSlots = 10,
    };

    int allocate(int Hp, int Wp);
    int run_phase(int slot, cudaStream_t s);
    void record_phase(int slot, Launch& L);
    void set_qp(int qp, cudaStream_t s);

    void enc_analysis(Launch& L);
    void enc_update(Launch& L, bool reset);
    void dec_temporal(Launch& L, bool memory_has_value);
    void dec_hyper(Launch& L);
    void dec_step(Launch& L, int k);
    void dec_final(Launch& L);
    void feature_adaptor_m(Launch& L);
    void feature_adaptor_i(Launch& L, const __half* feature_i);
    void feature_extractor(Launch& L);
    void temporal_prior(Launch& L);
    void hyper_prior(Launch& L);     // hyper decoder, prior fusion, reduction
    void spatial_prior(Launch& L, int k);
    void decoder(Launch& L);
    void recon_head(Launch& L, bool all_frames);
    void compact_step(Launch& L, int k, bool enc);

    // ---------------------------------------------------------------- parameters
    DeviceArena weights_;
    bool ready_ = false;
    __half skip_thr_half_;
    const __half* q_enc_tab_ = nullptr;
    const __half* q_dec_tab_ = nullptr;
    const __half* q_feat_tab_ = nullptr;
    uint8_t* scale_lut_ = nullptr;
    Dcb encoder_[7];
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
    Lin dec_up_;        // 3x3 sub-pixel conv with bias
    Dcb decoder_[11];
    Dcb fa_i_[3];
    Dcb fa_m_[10];
    Dcb fe_[2];
    Dcb rh_[kFrames][5];
    Lin rh_head_[kFrames];
    RansTables tables_;

    // ---------------------------------------------------------------- resolution state
    DeviceArena acts_;
    int Hp_ = 0, Wp_ = 0, H8_ = 0, W8_ = 0, H16_ = 0, W16_ = 0, H16p_ = 0, W16p_ = 0;
    int M8_ = 0, M16_ = 0, M16p_ = 0, M32_ = 0, M64_ = 0;
    int part_num_ = 0, z_num_ = 0;
    __half *cat_enc_ = nullptr, *cat_fam_ = nullptr, *feature_i_ = nullptr, *temporal_in_ = nullptr;
    __half *y_ = nullptr, *y_pad_ = nullptr, *cat_pf_ = nullptr, *hyper_pad_ = nullptr;
    __half *common_ = nullptr, *cat_spa_ = nullptr, *sp_out_ = nullptr, *y_q_ = nullptr;
    __half *part_ = nullptr, *z_ = nullptr, *z_hat_ = nullptr, *col_ = nullptr, *s2d_ = nullptr;
    __half *lvl8_a_ = nullptr, *lvl16_a_ = nullptr, *lvl16_b_ = nullptr, *lvl32_a_ = nullptr;
    __half *lvl32_b_ = nullptr, *lvl64_a_ = nullptr, *head_ = nullptr;
    __half *q_enc_ = nullptr, *q_dec_ = nullptr, *q_feat_ = nullptr;
    __half* x_hat_[kFrames] = {nullptr};
    int8_t* z_i8_ = nullptr;
    int16_t *sym_ = nullptr, *sym_c_ = nullptr;
    uint8_t *idx_ = nullptr, *idx_c_ = nullptr, *cond_ = nullptr;
    int8_t* y_dec_ = nullptr;
    int* block_counts_ = nullptr;
    int* count_dev_ = nullptr;
    Scratch scratch_;
    int* count_host_ = nullptr;
    int16_t* sym_host_ = nullptr;
    uint8_t* idx_host_ = nullptr;
    int8_t* ydec_host_ = nullptr;
    int8_t* z_host_ = nullptr;
    bool memory_has_value_ = false;

    PhaseGraphs graphs_{kPhaseSlots};
    cudaStream_t main_ = nullptr;
    cudaStream_t copy_ = nullptr;
    cudaEvent_t ev_in_ = nullptr, ev_phase_ = nullptr, ev_copy_ = nullptr, ev_out_ = nullptr;
    int* err_word_ = nullptr;
    ErrorSlot err_slot_;  // the error word as the phase graphs publish it
    int last_count_ = 0;
    int last_kernels_ = 0;
    int dev_ = 0;
};

}  // namespace dcvc
