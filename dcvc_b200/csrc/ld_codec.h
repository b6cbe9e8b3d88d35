// DCVC-UF low-delay (LD) frame codec runtime: the B200 counterpart of DMCLDProxy
// (src/layers/extensions/inference/dmc_ld_proxy.{h,cpp}).  One frame per call, the temporal
// memory and temporal-prior parameters kept on the device, 2-phase checkerboard coding with a
// means-only spatial prior.
#pragma once

#include "codec_common.h"
#include "net.h"
#include "rans_coder.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace dcvc {

class LdCodec {
public:
    static constexpr int kChSrc = 192;  // 3 * 8 * 8, one frame
    static constexpr int kChY = 128, kChZ = 128, kChD = 256, kChM = 256;
    static constexpr int kQpNum = 64;

    LdCodec();
    ~LdCodec();

    // set_param (dmc_ld_proxy.cpp:595-637).
    int set_param(const StateDict& sd, float skip_threshold);
    // add_ref_feature_from_frame (dmc_ld_proxy.cpp:407-418): frame [Hp, Wp, 3] FP16.
    int add_ref_feature(const __half* frame, int Hp, int Wp, bool apply_adaptor, cudaStream_t s);
    // compress (dmc_ld_proxy.cpp:420-485): x [H, W, 3] FP16.
    int compress(const __half* x, int H, int W, int qp, bool reset, int pad_b, int pad_r,
                 cudaStream_t s, std::vector<uint8_t>* bytes, int* ec_parallel);
    // decompress (dmc_ld_proxy.cpp:487-566): one device frame [Hp, Wp, 3] FP16 owned by the codec.
    int decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                   bool reset, cudaStream_t s, const __half** frame);

    // "y_hat", "y_q", "memory", "ctx", "feature_p", "common", "feature_i", "temporal".
    int buffer(const std::string& name, const void** ptr, int* rows, int* cols, int* ld) const;

    int last_symbol_count() const { return last_count_; }
    size_t device_bytes() const { return weights_.bytes() + acts_.bytes(); }
    int last_kernel_count() const { return last_kernels_; }

private:
    enum Phase {
        kEncAnalysis = 0,   // lambda_enc_0 (dmc_ld_proxy.cpp:432-457)
        kEncUpdate = 1,     // lambda_enc_1 (:470-475), 2 variants: reset
        kDecTemporal = 3,   // lambda_dec_0 (:510-514), 2 variants: memory has value
        kDecHyper = 5,      // lambda_dec_1 (:532-547)
        kDecContext = 6,    // lambda_dec_2 (:560)
        kDecSynthesis = 7,  // lambda_dec_3 (:576-586)
        kPhaseSlots = 8,
    };

    int allocate(int Hp, int Wp);
    int run_phase(int slot, cudaStream_t s);
    void record_phase(int slot, Launch& L);
    void set_qp(int qp, cudaStream_t s);

    void enc_analysis(Launch& L);
    void enc_update(Launch& L, bool reset);
    void dec_temporal(Launch& L, bool memory_has_value);
    void dec_hyper(Launch& L);
    void dec_synthesis(Launch& L);
    void feature_adaptor_m(Launch& L);
    void feature_adaptor_i(Launch& L);
    void feature_extractor(Launch& L);
    void temporal_prior(Launch& L);
    void entropy_params(Launch& L);  // hyper decoder, temporal x q_feature, prior fusion
    void spatial_prior(Launch& L);
    void decoder(Launch& L);
    void recon_head(Launch& L, bool shuffle);

    // ---------------------------------------------------------------- parameters
    DeviceArena weights_;
    bool ready_ = false;
    __half skip_thr_half_;
    const __half* q_enc_tab_ = nullptr;   // [64][256]
    const __half* q_dec_tab_ = nullptr;   // [64][256]
    const __half* q_feat_tab_ = nullptr;  // [64][256]
    uint8_t* scale_lut_ = nullptr;
    Dcb encoder_[3];
    Lin enc_down_;
    Dcb hyper_enc0_;
    DownBlock hyper_enc1_, hyper_enc2_;
    UpBlock hyper_dec0_, hyper_dec1_;
    Dcb hyper_dec2_;
    DownBlock temporal_enc_;
    Dcb prior_fusion_[3];
    Lin prior_fusion_out_;
    Dcb spatial_prior_[2];
    Lin spatial_prior_out_;
    Lin dec_up_;
    Dcb decoder_[3];
    Lin dec_conv2_;
    Dcb fa_i_[4];
    Dcb fa_m_[4];
    Dcb fe_[5];
    Dcb rh_[3];
    Lin rh_head_;
    RansTables tables_;

    // ---------------------------------------------------------------- resolution state
    DeviceArena acts_;
    int Hp_ = 0, Wp_ = 0, H8_ = 0, W8_ = 0, H16_ = 0, W16_ = 0, H16p_ = 0, W16p_ = 0;
    int M8_ = 0, M16_ = 0, M16p_ = 0, M32_ = 0, M64_ = 0;
    int y_num_ = 0, z_num_ = 0;
    // cat_enc [M8, 512]: [64:256] the unshuffled frame, [256:512] ctx; the decoder's up-sampling
    // output overwrites [0:256] so that [0:512] is cat(up, ctx)
    __half *cat_enc_ = nullptr, *cat_fam_ = nullptr, *feature_i_ = nullptr;
    __half *y_ = nullptr, *y_pad_ = nullptr, *temporal_params_ = nullptr, *cat_pf_ = nullptr;
    __half *hyper_pad_ = nullptr, *cat_sp_ = nullptr, *means1_ = nullptr, *y_q_ = nullptr;
    __half *z_ = nullptr, *z_hat_ = nullptr, *col_ = nullptr, *s2d_ = nullptr;
    __half *lvl8_a_ = nullptr, *lvl16_a_ = nullptr, *lvl32_a_ = nullptr, *lvl64_a_ = nullptr;
    __half *q_enc_ = nullptr, *q_dec_ = nullptr, *q_feat_ = nullptr;
    __half* x_hat_ = nullptr;
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
    // device addresses of the mapped host buffers above: the phase graphs move symbols, indexes,
    // decoded values and their counts through them (launch_copy_counted)
    int* count_hdev_ = nullptr;
    int16_t* sym_hdev_ = nullptr;
    uint8_t* idx_hdev_ = nullptr;
    int8_t* ydec_hdev_ = nullptr;
    int8_t* z_hdev_ = nullptr;
    bool memory_has_value_ = false;

    PhaseGraphs graphs_{kPhaseSlots};
    cudaStream_t main_ = nullptr;
    cudaEvent_t ev_in_ = nullptr, ev_phase_ = nullptr, ev_out_ = nullptr;
    int* err_word_ = nullptr;
    ErrorSlot err_slot_;  // the error word as the phase graphs publish it
    int last_count_ = 0;
    int last_kernels_ = 0;
    int dev_ = 0;
};

}  // namespace dcvc
