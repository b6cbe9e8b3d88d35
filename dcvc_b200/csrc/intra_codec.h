// Intra (DMCI) frame codec runtime: the B200 counterpart of DMCIProxy
// (src/layers/extensions/inference/dmci_proxy.{h,cpp}).
#pragma once

#include "codec_common.h"
#include "net.h"
#include "rans_coder.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace dcvc {

class IntraCodec {
public:
    static constexpr int kChSrc = 192;  // 3 * 8 * 8 (image_model.py:11-14)
    static constexpr int kChEnc = 384;
    static constexpr int kChY = 256, kChZ = 128;
    static constexpr int kQpNum = 64;
    static constexpr int kSteps = 4;    // checkerboard coding steps

    IntraCodec();
    ~IntraCodec();

    // set_param (dmci_proxy.cpp:604-646): weights + CDF tables + skip threshold.
    int set_param(const StateDict& sd, float skip_threshold);
    // compress (dmci_proxy.cpp:296-421): x is [H, W, 3] FP16 channels-last on the device,
    // H + pad_b and W + pad_r multiples of 16.  *x_hat receives the reconstruction
    // [H + pad_b, W + pad_r, 3] FP16, owned by the codec and overwritten by the next call.
    int compress(const __half* x, int H, int W, int qp, int pad_b, int pad_r, cudaStream_t s,
                 std::vector<uint8_t>* bytes, int* ec_parallel, const __half** x_hat);
    // decompress (dmci_proxy.cpp:423-602): height/width are the picture size of the stream.
    int decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                   cudaStream_t s, const __half** x_hat);

    // Read-only view of an internal buffer: "y_hat", "y_q", "params", "z_hat".
    int buffer(const std::string& name, const void** ptr, int* rows, int* cols, int* ld) const;

    int last_symbol_count() const { return last_count_; }
    size_t device_bytes() const { return weights_.bytes() + acts_.bytes(); }
    int last_kernel_count() const { return last_kernels_; }

private:
    enum Phase {
        kEncAnalysis = 0,   // lambda_enc_0 (dmci_proxy.cpp:308-396)
        kEncSynthesis = 1,  // lambda_enc_1 (:408-411)
        kDecHyper = 2,      // lambda_dec_0 (:461-480)
        kDecStep = 3,       // lambda_dec_1..3 (:497-572), slots 3, 4, 5
        kDecFinal = 6,      // lambda_dec_4 (:589-598)
        kPhaseSlots = 7,
    };

    int allocate(int Hp, int Wp);
    int run_phase(int slot, cudaStream_t s);
    void record_phase(int slot, Launch& L);
    void set_qp(int qp, cudaStream_t s);

    // phase bodies
    void enc_analysis(Launch& L);
    void dec_hyper(Launch& L);
    void dec_step(Launch& L, int k);  // restores step k - 1, builds step k's indexes
    void dec_final(Launch& L);
    // network pieces
    void hyper_prior(Launch& L);      // z_hat -> params (cropped), reduction
    void spatial_prior(Launch& L, int k);
    void decoder(Launch& L);
    void compact_step(Launch& L, int k, bool enc);

    // ---------------------------------------------------------------- parameters
    DeviceArena weights_;
    bool ready_ = false;
    __half skip_thr_half_;
    const __half* q_enc_tab_ = nullptr;    // [64][384]
    const __half* q_dec_tab_ = nullptr;    // [64][384]
    const __half* q_y_enc_tab_ = nullptr;  // [64][256]
    const __half* q_y_dec_tab_ = nullptr;  // [64][256]
    uint8_t* scale_lut_ = nullptr;         // [65536]
    Dcb enc1_;
    Dcb enc2_[6];
    Lin enc_down_;
    Dcb hyper_enc0_;
    DownBlock hyper_enc1_, hyper_enc2_;
    UpBlock hyper_dec0_, hyper_dec1_;
    Dcb hyper_dec2_;
    Dcb prior_fusion_[3];
    Lin prior_fusion_out_;
    Lin reduction_;
    Dcb sp_adaptor_[3];
    Dcb spatial_prior_[3];
    Lin spatial_prior_out_;
    UpBlock dec_up_;
    Dcb dec1_[12];
    Dcb dec2_;
    RansTables tables_;

    // ---------------------------------------------------------------- resolution state
    DeviceArena acts_;
    int Hp_ = 0, Wp_ = 0, H8_ = 0, W8_ = 0, H16_ = 0, W16_ = 0, H16p_ = 0, W16p_ = 0;
    int M8_ = 0, M16_ = 0, M16p_ = 0, M32_ = 0, M64_ = 0;
    int part_num_ = 0, z_num_ = 0;   // symbols per step (M16 * 64), z symbols
    __half *unshuf_ = nullptr, *lvl8_a_ = nullptr, *lvl8_b_ = nullptr, *col_ = nullptr;
    __half *y_ = nullptr, *y_pad_ = nullptr, *y_s_ = nullptr, *y_q_ = nullptr;
    __half *lvl16_a_ = nullptr, *lvl16_b_ = nullptr, *lvl32_a_ = nullptr, *lvl32_b_ = nullptr;
    __half *lvl64_a_ = nullptr, *s2d_ = nullptr, *z_ = nullptr, *z_hat_ = nullptr;
    __half *params_pad_ = nullptr, *params_ = nullptr, *cat_sp_ = nullptr, *sp_out_ = nullptr;
    __half *part_ = nullptr, *head_ = nullptr, *x_hat_ = nullptr;
    __half *q_enc_ = nullptr, *q_dec_ = nullptr, *q_y_enc_ = nullptr, *q_y_dec_ = nullptr;
    int8_t* z_i8_ = nullptr;
    int16_t *sym_ = nullptr, *sym_c_ = nullptr;   // sym_c_: kSteps compacted parts
    uint8_t *idx_ = nullptr, *idx_c_ = nullptr, *cond_ = nullptr;
    int8_t* y_dec_ = nullptr;
    int* block_counts_ = nullptr;
    int* count_dev_ = nullptr;                    // [kSteps]
    Scratch scratch_;
    // pinned host staging
    int* count_host_ = nullptr;                   // [kSteps]
    int16_t* sym_host_ = nullptr;                 // kSteps * part_num_
    uint8_t* idx_host_ = nullptr;
    int8_t* ydec_host_ = nullptr;
    int8_t* z_host_ = nullptr;

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
