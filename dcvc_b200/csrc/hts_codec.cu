#include "hts_codec.h"

#include "elementwise.cuh"
#include "errors.h"
#include "gemm_sm100.cuh"
#include "quant_tables.h"

#include <algorithm>
#include <cstring>
#include <type_traits>

namespace dcvc {

namespace {

constexpr int kMaskPhases = 4;

inline int ceil_to(int v, int m) { return (v + m - 1) / m * m; }

std::string num(const char* prefix, int i, const char* suffix = ".")
{
    return std::string(prefix) + std::to_string(i) + suffix;
}

}  // namespace

HtsCodec::HtsCodec()
{
    cudaGetDevice(&dev_);
    cudaStreamCreateWithFlags(&main_, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&ev_in_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_phase_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_out_, cudaEventDisableTiming);
    err_word_ = device_error_word();
    if (err_slot_.alloc()) {
        graphs_.set_error_slot(err_slot_.dev);
    }
}

HtsCodec::~HtsCodec()
{
    cudaSetDevice(dev_);
    if (main_ != nullptr) {
        cudaStreamSynchronize(main_);
    }
    clear_graphs();
    cudaFreeHost(count_host_);
    cudaFreeHost(sym_host_);
    cudaFreeHost(idx_host_);
    cudaFreeHost(ydec_host_);
    cudaFreeHost(z_host_);
    cudaEventDestroy(ev_in_);
    cudaEventDestroy(ev_phase_);
    cudaEventDestroy(ev_out_);
    cudaStreamDestroy(main_);
    err_slot_.release();
}

void HtsCodec::clear_graphs() { graphs_.clear(); }

int HtsCodec::set_precision(int precision)
{
    if (precision != kPrecisionF16 && precision != kPrecisionBF16 && precision != kPrecisionFP8) {
        set_last_error("set_precision: precision must be 0 (FP16), 1 (BF16) or 2 (FP8)");
        return kInvalidArgument;
    }
    precision_ = precision;
    return kOk;
}

int HtsCodec::set_param(const StateDict& sd, float skip_threshold)
{
    if (main_ != nullptr) {
        cudaStreamSynchronize(main_);
    }
    clear_graphs();
    ready_ = false;
    weights_.clear();
    ParamBuilder B(sd, weights_);
    // the analysis / synthesis transforms in the precision form's format, the entropy-parameter
    // path in FP16; q_encoder / q_decoder scale outputs of the transforms, q_feature the input
    // of the temporal prior
    const int act = precision_ == kPrecisionF16 ? 0 : 1;
    const bool f8 = precision_ == kPrecisionFP8;
    act_ = act;
    fp8_ = f8;
    int r = 0, c = 0;
    q_enc_tab_ = act ? B.bf16_rows("q_encoder", &r, &c) : B.half_rows("q_encoder", &r, &c);
    if (B.ok() && (r != kQpNum || c != kChD)) {
        set_last_error("set_param: q_encoder must be [64, 512]");
        return kInvalidArgument;
    }
    q_dec_tab_ = act ? B.bf16_rows("q_decoder", &r, &c) : B.half_rows("q_decoder", &r, &c);
    q_feat_tab_ = B.half_rows("q_feature", &r, &c);
    B.set_dtype(act, f8);
    for (int i = 0; i < 6; ++i) {
        encoder_[i] = B.dcb(num("encoder.conv1.", i));
    }
    enc_down_ = B.conv3x3s2("encoder.down.");
    B.set_dtype(0);
    hyper_enc0_ = B.dcb("hyper_encoder.conv.0.");
    hyper_enc1_ = B.down("hyper_encoder.conv.1.");
    hyper_enc2_ = B.down("hyper_encoder.conv.2.");
    hyper_dec0_ = B.up("hyper_decoder.conv.0.");
    hyper_dec1_ = B.up("hyper_decoder.conv.1.");
    hyper_dec2_ = B.dcb("hyper_decoder.conv.2.");
    temporal_ = B.down("temporal_prior_encoder.conv.");
    for (int i = 0; i < 3; ++i) {
        prior_fusion_[i] = B.dcb(num("y_prior_fusion.conv.", i));
        sp_adaptor_[i] = B.dcb(num("y_spatial_prior_adaptor_", i + 1));
        spatial_prior_[i] = B.dcb(num("y_spatial_prior.conv.", i));
    }
    prior_fusion_out_ = B.lin("y_prior_fusion.conv.3.");
    reduction_ = B.lin("y_spatial_prior_reduction.");
    spatial_prior_out_ = B.lin("y_spatial_prior.conv.3.");
    B.set_dtype(act, f8);
    dec_up_lin_ = B.subpel("decoder.up.");
    for (int i = 0; i < 7; ++i) {
        decoder_[i] = B.dcb(num("decoder.conv1.", i));
    }
    for (int i = 0; i < 4; ++i) {
        fa_i_[i] = B.dcb(num("feature_adaptor_i.conv.", i));
        rh_common_[i] = B.dcb(num("recon_head.conv1.", i, ".0."));
    }
    for (int i = 0; i < 6; ++i) {
        fa_m_[i] = B.dcb(num("feature_adaptor_m.conv.", i));
    }
    for (int i = 0; i < 5; ++i) {
        fe_[i] = B.dcb(num("feature_extractor.conv.", i));
    }
    for (int i = 0; i < kFrames; ++i) {
        for (int j = 0; j < 3; ++j) {
            rh_frame_[i][j] = B.dcb(num("recon_head.conv2.", i, ".") + std::to_string(j) + ".");
        }
        rh_head_[i] = B.lin(num("recon_head.conv2.", i, ".3."));
    }
    B.set_dtype(0);
    if (!B.ok()) {
        set_last_error("set_param: " + B.error());
        weights_.clear();
        return kInvalidArgument;
    }
    // structural checks of the HT-S layout (video_model_ht.py:17-23)
    const bool shapes_ok =
        encoder_[0].cin == kChSrc + kChD && encoder_[0].C == kChD && enc_down_.cout == kChY &&
        enc_down_.cin == 9 * kChD && hyper_enc2_.down.cout == kChZ && hyper_dec0_.up.cin == kChZ &&
        temporal_.down.cin == 4 * kChD && temporal_.down.cout == 2 * kChY &&
        prior_fusion_[0].C == 3 * kChY && prior_fusion_out_.cout == 3 * kChY &&
        reduction_.cin == 3 * kChY && reduction_.cout == kChY && sp_adaptor_[0].C == 2 * kChY &&
        spatial_prior_out_.cout == kChY && dec_up_lin_.cin == kChY && dec_up_lin_.cout == 4 * kChD &&
        decoder_[0].cin == 2 * kChD && fa_i_[0].cin == kChSrcIntra && fa_m_[0].cin == kChM + kChD &&
        fe_[0].C == kChD && rh_head_[0].cout == kChSrcIntra && rh_head_[0].cin == kChRecon;
    if (!shapes_ok) {
        set_last_error("set_param: state dict is not an HT-S (DMC, ModelStructure.HTS) model");
        weights_.clear();
        return kInvalidArgument;
    }
    // CDF tables (set_param, dmc_hts_proxy.cpp:748-761)
    if (load_cdf_tables(sd, &tables_, kQpNum * kChZ, 128) != kOk) {
        weights_.clear();
        return kInvalidArgument;
    }
    // the scale -> CDF index table, evaluated on the device as the reference's FP16
    // scale_to_index computes it
    scale_lut_ = weights_.alloc_n<uint8_t>(65536);
    if (scale_lut_ == nullptr || scale_index_table_device(scale_lut_, 0) != cudaSuccess ||
        cudaStreamSynchronize(0) != cudaSuccess) {
        set_last_error("set_param: could not build the scale-index table");
        return kOutOfMemory;
    }
    skip_threshold_ = skip_threshold;
    skip_thr_half_ = __float2half_rn(skip_threshold);
    ready_ = true;
    return kOk;
}

int HtsCodec::allocate(int Hp, int Wp)
{
    if (Hp == Hp_ && Wp == Wp_) {
        return kOk;
    }
    if (Hp <= 0 || Wp <= 0 || Hp % 16 || Wp % 16) {
        set_last_error("frame height and width must be positive multiples of 16");
        return kInvalidArgument;
    }
    cudaStreamSynchronize(main_);
    clear_graphs();
    acts_.clear();
    cudaFreeHost(count_host_);
    cudaFreeHost(sym_host_);
    cudaFreeHost(idx_host_);
    cudaFreeHost(ydec_host_);
    cudaFreeHost(z_host_);
    count_host_ = nullptr;
    sym_host_ = nullptr;
    idx_host_ = nullptr;
    ydec_host_ = nullptr;
    z_host_ = nullptr;
    count_hdev_ = nullptr;
    sym_hdev_ = nullptr;
    idx_hdev_ = nullptr;
    ydec_hdev_ = nullptr;
    z_hdev_ = nullptr;
    Hp_ = Wp_ = 0;

    const int H8 = Hp / 8, W8 = Wp / 8;
    const int H16 = H8 / 2, W16 = W8 / 2;
    const int H16p = ceil_to(H16, 4), W16p = ceil_to(W16, 4);
    H8_ = H8;
    W8_ = W8;
    H16_ = H16;
    W16_ = W16;
    H16p_ = H16p;
    W16p_ = W16p;
    M8_ = H8 * W8;
    M16_ = H16 * W16;
    M16p_ = H16p * W16p;
    M32_ = (H16p / 2) * (W16p / 2);
    M64_ = (H16p / 4) * (W16p / 4);
    y_num_ = M16_ * kChY;
    z_num_ = M64_ * kChZ;
    const bool pad = (H16p != H16) || (W16p != W16);

    bool ok = true;
    auto H = [&](size_t n) {
        __half* p = acts_.alloc_n<__half>(n);
        ok = ok && p != nullptr;
        return p;
    };
    const size_t M8 = M8_, M16 = M16_, M16p = M16p_, M32 = M32_, M64 = M64_;
    cat_enc_ = H(M8 * 2048);
    cat_fam_ = H(M8 * 1024);
    feature_i_ = H(M8 * kChSrcIntra);
    temporal_in_ = H(M8 * kChD);
    y_ = H(M16 * kChY);
    y_pad_ = pad ? H(M16p * kChY) : y_;
    cat_pf_ = H(M16 * 3 * kChY);
    hyper_pad_ = pad ? H(M16p * kChY) : nullptr;
    common_ = H(M16 * 3 * kChY);
    cat_spa_ = H(M16 * 2 * kChY);
    means_ = H(M16 * kChY);
    y_q_ = H(M16 * kChY);
    z_ = H(M64 * kChZ);
    z_hat_ = H(M64 * kChZ);
    col_ = H(M16 * 9 * kChD);
    s2d_ = H(std::max({M16 * 4 * kChD, M32 * 4 * kChY, M64 * 4 * kChY}));
    lvl8_a_ = H(M8 * kChD);
    lvl8_b_ = H(M8 * kChD);
    lvl16_a_ = H(M16p * 3 * kChY);
    lvl32_a_ = H(M32 * kChY);
    lvl64_a_ = H(M64 * kChZ);
    head_ = H(M8 * kChSrcIntra);
    y_act_ = act_ ? H(M16 * kChY) : nullptr;
    yhat_act_ = act_ ? H(M16 * kChY) : nullptr;
    q_enc_ = H(kChD);
    q_dec_ = H(kChD);
    q_feat_ = H(kChD);
    for (int i = 0; i < kFrames; ++i) {
        x_hat_[i] = H(static_cast<size_t>(Hp) * Wp * 3);
    }
    const size_t S = std::max(M8 * kChD, M16p * 3 * kChY);
    scratch_.t0 = H(S);
    scratch_.t1 = H(S);
    scratch_.t2 = H(S);
    scratch_.t3 = H(S);
    scratch_.t4 = H(S);
    scratch_.t5 = fp8_ ? acts_.alloc_n<uint8_t>(M8 * kChD) : nullptr;
    ok = ok && (!fp8_ || scratch_.t5 != nullptr);
    z_i8_ = acts_.alloc_n<int8_t>(z_num_);
    sym_ = acts_.alloc_n<int16_t>(y_num_);
    sym_c_ = acts_.alloc_n<int16_t>(y_num_);
    idx_ = acts_.alloc_n<uint8_t>(y_num_);
    idx_c_ = acts_.alloc_n<uint8_t>(y_num_);
    cond_ = acts_.alloc_n<uint8_t>(y_num_);
    y_dec_ = acts_.alloc_n<int8_t>(y_num_);
    block_counts_ = acts_.alloc_n<int>(compact_blocks(y_num_));
    count_dev_ = acts_.alloc_n<int>(1);
    ok = ok && z_i8_ && sym_ && sym_c_ && idx_ && idx_c_ && cond_ && y_dec_ && block_counts_ &&
         count_dev_;
    auto mapped = [&](size_t bytes, auto** host, auto** dev) {
        void *h = nullptr, *d = nullptr;
        ok = ok && alloc_mapped(bytes, &h, &d);
        *host = static_cast<std::remove_reference_t<decltype(**host)>*>(h);
        *dev = static_cast<std::remove_reference_t<decltype(**dev)>*>(d);
    };
    mapped(sizeof(int) * 2, &count_host_, &count_hdev_);
    mapped(sizeof(int16_t) * y_num_, &sym_host_, &sym_hdev_);
    mapped(y_num_, &idx_host_, &idx_hdev_);
    mapped(y_num_, &ydec_host_, &ydec_hdev_);
    mapped(z_num_, &z_host_, &z_hdev_);
    if (!ok) {
        cudaGetLastError();
        acts_.clear();
        set_last_error("out of device or pinned host memory for this resolution");
        return kOutOfMemory;
    }
    // zero the concatenation buffers once so no stale NaN can leak through unused lanes
    cudaMemsetAsync(cat_enc_, 0, M8 * 2048 * 2, main_);
    cudaMemsetAsync(cat_fam_, 0, M8 * 1024 * 2, main_);
    cudaMemsetAsync(cat_pf_, 0, M16 * 3 * kChY * 2, main_);
    cudaMemsetAsync(cat_spa_, 0, M16 * 2 * kChY * 2, main_);
    if (cudaStreamSynchronize(main_) != cudaSuccess) {
        return cuda_status(cudaGetLastError(), "allocate");
    }
    Hp_ = Hp;
    Wp_ = Wp;
    memory_has_value_ = false;
    return kOk;
}

void HtsCodec::set_qp(int qp, cudaStream_t s)
{
    cudaMemcpyAsync(q_enc_, q_enc_tab_ + static_cast<size_t>(qp) * kChD, kChD * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_dec_, q_dec_tab_ + static_cast<size_t>(qp) * kChD, kChD * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_feat_, q_feat_tab_ + static_cast<size_t>(qp) * kChD, kChD * 2,
                    cudaMemcpyDeviceToDevice, s);
}

// ------------------------------------------------------------------------------ network pieces

void HtsCodec::feature_adaptor_m(Launch& L)
{
    // memory = FA_m(cat(memory, feature_p))   (dmc_hts_proxy.cpp:845-851)
    run_dcb(L, fa_m_[0], cat_fam_, 1024, H8_, W8_, lvl8_a_, kChM, scratch_);
    for (int i = 1; i < 5; ++i) {
        run_dcb(L, fa_m_[i], lvl8_a_, kChM, H8_, W8_, lvl8_a_, kChM, scratch_);
    }
    run_dcb(L, fa_m_[5], lvl8_a_, kChM, H8_, W8_, cat_fam_, 1024, scratch_);
}

void HtsCodec::feature_adaptor_i(Launch& L, const __half* fi)
{
    run_dcb(L, fa_i_[0], fi, kChSrcIntra, H8_, W8_, lvl8_a_, kChM, scratch_);
    for (int i = 1; i < 3; ++i) {
        run_dcb(L, fa_i_[i], lvl8_a_, kChM, H8_, W8_, lvl8_a_, kChM, scratch_);
    }
    run_dcb(L, fa_i_[3], lvl8_a_, kChM, H8_, W8_, cat_fam_, 1024, scratch_);
}

void HtsCodec::feature_extractor(Launch& L)
{
    // ctx = FE(memory); ctx lives in cat_enc[1536:2048]
    __half* ctx = cat_enc_ + kChSrc;
    run_dcb(L, fe_[0], cat_fam_, 1024, H8_, W8_, ctx, 2048, scratch_);
    for (int i = 1; i < 5; ++i) {
        run_dcb(L, fe_[i], ctx, 2048, H8_, W8_, ctx, 2048, scratch_);
    }
}

void HtsCodec::temporal_prior(Launch& L)
{
    // temporal_params = RBWS2(memory * q_feature) -> cat_pf[256:768]
    L.note(launch_mul_channel(cat_fam_, M8_, kChM, 1024, q_feat_, temporal_in_, kChM, L.s, act_));
    L.note(launch_space_to_depth2(temporal_in_, H8_, W8_, kChM, kChM, s2d_, L.s));
    gemm(L, temporal_.down, kEpiBias, s2d_, 4 * kChM, M16_, lvl16_a_, 2 * kChY);
    run_dcb(L, temporal_.dcb, lvl16_a_, 2 * kChY, H16_, W16_, cat_pf_ + kChY, 3 * kChY, scratch_);
}

void HtsCodec::hyper_decoder(Launch& L)
{
    const int H64 = H16p_ / 4, W64 = W16p_ / 4, H32 = H16p_ / 2, W32 = W16p_ / 2;
    gemm(L, hyper_dec0_.up, kEpiSubpel, z_hat_, kChZ, M64_, lvl32_a_, kChY, nullptr, 0, nullptr, W64);
    run_dcb(L, hyper_dec0_.dcb, lvl32_a_, kChY, H32, W32, lvl32_a_, kChY, scratch_);
    gemm(L, hyper_dec1_.up, kEpiSubpel, lvl32_a_, kChY, M32_, lvl16_a_, kChY, nullptr, 0, nullptr, W32);
    run_dcb(L, hyper_dec1_.dcb, lvl16_a_, kChY, H16p_, W16p_, lvl16_a_, kChY, scratch_);
    if (hyper_pad_ != nullptr) {
        run_dcb(L, hyper_dec2_, lvl16_a_, kChY, H16p_, W16p_, hyper_pad_, kChY, scratch_);
        L.note(launch_crop(hyper_pad_, W16p_, kChY, H16_, W16_, kChY, cat_pf_, 3 * kChY, L.s));
    } else {
        run_dcb(L, hyper_dec2_, lvl16_a_, kChY, H16_, W16_, cat_pf_, 3 * kChY, scratch_);
    }
}

void HtsCodec::prior_fusion(Launch& L)
{
    const int C = 3 * kChY;
    run_dcb(L, prior_fusion_[0], cat_pf_, C, H16_, W16_, lvl16_a_, C, scratch_);
    run_dcb(L, prior_fusion_[1], lvl16_a_, C, H16_, W16_, lvl16_a_, C, scratch_);
    run_dcb(L, prior_fusion_[2], lvl16_a_, C, H16_, W16_, lvl16_a_, C, scratch_);
    gemm(L, prior_fusion_out_, kEpiBias, lvl16_a_, C, M16_, common_, C);
}

void HtsCodec::spatial_prior(Launch& L, int k)
{
    const int C = 2 * kChY;
    run_dcb(L, sp_adaptor_[k], cat_spa_, C, H16_, W16_, lvl16_a_, C, scratch_);
    for (int i = 0; i < 3; ++i) {
        run_dcb(L, spatial_prior_[i], lvl16_a_, C, H16_, W16_, lvl16_a_, C, scratch_);
    }
    gemm(L, spatial_prior_out_, kEpiBias, lvl16_a_, C, M16_, means_, kChY);
}

void HtsCodec::decoder(Launch& L)
{
    // up: y_hat (cat_spa[0:256]) -> cat_enc[1024:1536]; DCBs on cat_enc[1024:2048]
    const __half* yh = cat_spa_;
    int ldyh = 2 * kChY;
    if (act_) {  // the BF16 form: y_hat (FP16, exact symbols + means) converted once
        L.note(launch_convert(cat_spa_, 0, 2 * kChY, yhat_act_, 1, kChY, M16_, kChY, L.s));
        yh = yhat_act_;
        ldyh = kChY;
    }
    gemm(L, dec_up_lin_, kEpiSubpel, yh, ldyh, M16_, cat_enc_ + 1024, 2048, nullptr, 0, nullptr,
         W16_);
    run_dcb(L, decoder_[0], cat_enc_ + 1024, 2048, H8_, W8_, lvl8_a_, kChD, scratch_);
    for (int i = 1; i < 6; ++i) {
        run_dcb(L, decoder_[i], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    }
    run_dcb(L, decoder_[6], lvl8_a_, kChD, H8_, W8_, cat_fam_ + kChM, 1024, scratch_, q_dec_);
}

void HtsCodec::recon_head(Launch& L, bool all_frames)
{
    const __half* feature_p = cat_fam_ + kChM;
    const int first = all_frames ? 0 : kFrames - 1;
    for (int i = first; i < kFrames; ++i) {
        if (i % 2 == 0 || !all_frames) {
            run_dcb(L, rh_common_[i / 2], feature_p, 1024, H8_, W8_, lvl8_b_, kChD, scratch_);
        }
        run_dcb(L, rh_frame_[i][0], lvl8_b_, kChD, H8_, W8_, lvl8_a_, kChRecon, scratch_);
        run_dcb(L, rh_frame_[i][1], lvl8_a_, kChRecon, H8_, W8_, lvl8_a_, kChRecon, scratch_);
        run_dcb(L, rh_frame_[i][2], lvl8_a_, kChRecon, H8_, W8_, lvl8_a_, kChRecon, scratch_);
        __half* out = (i == kFrames - 1) ? feature_i_ : head_;
        gemm(L, rh_head_[i], kEpiBias, lvl8_a_, kChRecon, M8_, out, kChSrcIntra);
        if (all_frames) {
            L.note(launch_shuffle8_clamp(out, H8_, W8_, 3, kChSrcIntra, x_hat_[i], L.s, act_));
        }
    }
}

// ------------------------------------------------------------------------------ phases

void HtsCodec::enc_analysis(Launch& L)
{
    const int H32 = H16p_ / 2, W32 = W16p_ / 2, H64 = H16p_ / 4, W64 = W16p_ / 4;
    // encoder (dmc_hts_proxy.cpp:67-78)
    run_dcb(L, encoder_[0], cat_enc_, 2048, H8_, W8_, lvl8_a_, kChD, scratch_);
    for (int i = 1; i < 5; ++i) {
        run_dcb(L, encoder_[i], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    }
    run_dcb(L, encoder_[5], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_, q_enc_);
    L.note(launch_im2col3x3s2(lvl8_a_, H8_, W8_, kChD, kChD, col_, L.s));
    if (act_) {  // the BF16 form: y to FP16 for the entropy-parameter path
        gemm(L, enc_down_, kEpiBias, col_, 9 * kChD, M16_, y_act_, kChY);
        L.note(launch_convert(y_act_, 1, kChY, y_, 0, kChY, M16_, kChY, L.s));
    } else {
        gemm(L, enc_down_, kEpiBias, col_, 9 * kChD, M16_, y_, kChY);
    }
    if (y_pad_ != y_) {
        L.note(launch_replicate_pad(y_, H16_, W16_, kChY, kChY, H16p_ - H16_, W16p_ - W16_, y_pad_, L.s));
    }
    // hyper encoder
    run_dcb(L, hyper_enc0_, y_pad_, kChY, H16p_, W16p_, lvl16_a_, kChY, scratch_);
    L.note(launch_space_to_depth2(lvl16_a_, H16p_, W16p_, kChY, kChY, s2d_, L.s));
    gemm(L, hyper_enc1_.down, kEpiBias, s2d_, 4 * kChY, M32_, lvl32_a_, kChY);
    run_dcb(L, hyper_enc1_.dcb, lvl32_a_, kChY, H32, W32, lvl32_a_, kChY, scratch_);
    L.note(launch_space_to_depth2(lvl32_a_, H32, W32, kChY, kChY, s2d_, L.s));
    gemm(L, hyper_enc2_.down, kEpiBias, s2d_, 4 * kChY, M64_, lvl64_a_, kChZ);
    run_dcb(L, hyper_enc2_.dcb, lvl64_a_, kChZ, H64, W64, z_, kChZ, scratch_);
    L.note(launch_round_z(z_, z_num_, z_hat_, z_i8_, L.s));
    temporal_prior(L);
    hyper_decoder(L);
    prior_fusion(L);
    // entropy parameters: q_dec | scales | means in common_ (chunk_tensors_3)
    const __half* q_dec = common_;
    const __half* scales = common_ + kChY;
    const __half* means0 = common_ + 2 * kChY;
    const int ldc = 3 * kChY;
    L.note(launch_div_clamp(y_, M16_, kChY, kChY, q_dec, ldc, L.s));
    gemm(L, reduction_, kEpiBias, common_, ldc, M16_, cat_spa_ + kChY, 2 * kChY);
    L.note(launch_quantize_phase(0, 0, y_, kChY, scales, ldc, means0, ldc, nullptr, 0,
                                 skip_thr_half_, y_q_, kChY, cat_spa_, 2 * kChY, H16_, W16_, kChY,
                                 L.s));
    for (int k = 1; k < kMaskPhases; ++k) {
        spatial_prior(L, k - 1);
        L.note(launch_quantize_phase(k, k == kMaskPhases - 1 ? 2 : 1, y_, kChY, scales, ldc,
                                     means_, kChY, q_dec, ldc, skip_thr_half_, y_q_, kChY,
                                     cat_spa_, 2 * kChY, H16_, W16_, kChY, L.s));
    }
    L.note(launch_build_index_enc(y_q_, kChY, scales, ldc, skip_thr_half_, scale_lut_, M16_, kChY,
                                  sym_, cond_, L.s));
    L.note(launch_compact(sym_, 2, cond_, y_num_, block_counts_, sym_c_, count_dev_, L.s), 2);
    // the symbols, their count and z to the mapped host buffers
    L.note(launch_copy_counted(sym_c_, sym_hdev_, 2, count_dev_, y_num_, count_hdev_, L.s));
    L.note(launch_copy_counted(z_i8_, z_hdev_, 1, nullptr, z_num_, nullptr, L.s));
}

void HtsCodec::enc_update(Launch& L, bool reset)
{
    decoder(L);
    if (reset) {
        recon_head(L, false);  // forward_reset writes head 7 into feature_i
        feature_adaptor_i(L, feature_i_);
    } else {
        feature_adaptor_m(L);
    }
    feature_extractor(L);
}

void HtsCodec::dec_temporal(Launch& L, bool memory_has_value)
{
    if (memory_has_value) {
        feature_adaptor_m(L);
    } else {
        feature_adaptor_i(L, feature_i_);
    }
    temporal_prior(L);
}

void HtsCodec::dec_hyper(Launch& L)
{
    L.note(launch_int8_to_half(z_hdev_, z_num_, z_hat_, L.s));  // z as decoded on the host
    hyper_decoder(L);
    prior_fusion(L);
    L.note(launch_build_index_dec(common_ + kChY, 3 * kChY, skip_thr_half_, scale_lut_, M16_, kChY,
                                  idx_, cond_, L.s));
    L.note(launch_compact(idx_, 1, cond_, y_num_, block_counts_, idx_c_, count_dev_, L.s), 2);
    L.note(launch_copy_counted(idx_c_, idx_hdev_, 1, count_dev_, y_num_, count_hdev_, L.s));
}

void HtsCodec::dec_context(Launch& L) { feature_extractor(L); }

void HtsCodec::dec_synthesis(Launch& L)
{
    const __half* q_dec = common_;
    const __half* means0 = common_ + 2 * kChY;
    const int ldc = 3 * kChY;
    L.note(launch_copy_counted(ydec_hdev_, y_dec_, 1, count_dev_, y_num_, nullptr, L.s));
    L.note(launch_recover(y_dec_, cond_, block_counts_, y_num_, y_q_, L.s));
    L.note(launch_restore_phase(0, 0, y_q_, kChY, means0, ldc, nullptr, 0, cat_spa_, 2 * kChY,
                                H16_, W16_, kChY, L.s));
    gemm(L, reduction_, kEpiBias, common_, ldc, M16_, cat_spa_ + kChY, 2 * kChY);
    for (int k = 1; k < kMaskPhases; ++k) {
        spatial_prior(L, k - 1);
        L.note(launch_restore_phase(k, k == kMaskPhases - 1 ? 2 : 1, y_q_, kChY, means_, kChY,
                                    q_dec, ldc, cat_spa_, 2 * kChY, H16_, W16_, kChY, L.s));
    }
    decoder(L);
    recon_head(L, true);
}

// ------------------------------------------------------------------------------ graphs

void HtsCodec::record_phase(int slot, Launch& L)
{
    switch (slot) {
    case kEncAnalysis: enc_analysis(L); break;
    case kEncUpdate: enc_update(L, false); break;
    case kEncUpdate + 1: enc_update(L, true); break;
    case kDecTemporal: dec_temporal(L, false); break;
    case kDecTemporal + 1: dec_temporal(L, true); break;
    case kDecHyper: dec_hyper(L); break;
    case kDecContext: dec_context(L); break;
    case kDecSynthesis: dec_synthesis(L); break;
    default: break;
    }
}

int HtsCodec::run_phase(int slot, cudaStream_t s)
{
    return graphs_.run(slot, s, err_word_, [&](Launch& L) { record_phase(slot, L); },
                       &last_kernels_);
}

int HtsCodec::buffer(const std::string& name, const void** ptr, int* rows, int* cols,
                     int* ld, int* dtype) const
{
    if (Hp_ == 0) {
        set_last_error("buffer: no resolution allocated yet");
        return kNotReady;
    }
    struct Entry {
        const char* n;
        const __half* p;
        int rows, cols, ld, dtype;
    };
    const Entry e[] = {
        {"y_hat", cat_spa_, M16_, kChY, 2 * kChY, 0},
        {"y_q", y_q_, M16_, kChY, kChY, 0},
        {"memory", cat_fam_, M8_, kChM, 1024, act_},
        {"feature_p", cat_fam_ + kChM, M8_, kChD, 1024, act_},
        {"ctx", cat_enc_ + kChSrc, M8_, kChD, 2048, act_},
        {"common", common_, M16_, 3 * kChY, 3 * kChY, 0},
        {"feature_i", feature_i_, M8_, kChSrcIntra, kChSrcIntra, act_},
    };
    for (const Entry& x : e) {
        if (name == x.n) {
            *ptr = x.p;
            *rows = x.rows;
            *cols = x.cols;
            *ld = x.ld;
            if (dtype != nullptr) {
                *dtype = x.dtype;
            }
            return kOk;
        }
    }
    set_last_error("buffer: unknown buffer '" + name + "'");
    return kInvalidArgument;
}

// ------------------------------------------------------------------------------ public calls

int HtsCodec::add_ref_feature(const __half* frame, int Hp, int Wp, bool apply_adaptor,
                              cudaStream_t caller)
{
    if (!ready_) {
        set_last_error("add_ref_feature_from_frame: set_param has not been called");
        return kNotReady;
    }
    if (frame == nullptr) {
        set_last_error("add_ref_feature_from_frame: null frame");
        return kInvalidArgument;
    }
    int st = allocate(Hp, Wp);
    if (st != kOk) {
        return st;
    }
    last_kernels_ = 0;
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    Launch L{main_, err_word_};
    L.note(launch_pad_unshuffle8(frame, Hp, Wp, 3, 3, 0, 0, feature_i_, kChSrcIntra, main_, act_));
    if (apply_adaptor) {
        feature_adaptor_i(L, feature_i_);
        feature_extractor(L);
    }
    memory_has_value_ = apply_adaptor;
    last_kernels_ += L.kernels;
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    return cuda_status(L.first, "add_ref_feature_from_frame");
}

int HtsCodec::compress(const __half* x, int H, int W, int qp, bool reset, int pad_b, int pad_r,
                       cudaStream_t caller, std::vector<uint8_t>* bytes, int* ec_parallel)
{
    if (!ready_ || Hp_ == 0) {
        set_last_error("compress: set_param and add_ref_feature_from_frame must come first");
        return kNotReady;
    }
    if (x == nullptr || qp < 0 || qp >= kQpNum || pad_b < 0 || pad_r < 0 || H + pad_b != Hp_ ||
        W + pad_r != Wp_) {
        set_last_error("compress: bad input pointer, qp or size (input + padding must equal the "
                       "reference frame size)");
        return kInvalidArgument;
    }
    last_kernels_ = 0;
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    set_qp(qp, main_);
    Launch L{main_, err_word_};
    L.note(launch_pad_unshuffle8(x, H, W, 24, 24, pad_b, pad_r, cat_enc_, 2048, main_, act_));
    last_kernels_ += L.kernels;
    int st = cuda_status(L.first, "compress: pad_and_unshuffle_8");
    if (st == kOk) st = run_phase(kEncAnalysis, main_);
    if (st == kOk) st = cuda_status(cudaEventRecord(ev_phase_, main_), "compress");
    if (st == kOk) st = run_phase(kEncUpdate + (reset ? 1 : 0), main_);
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    if (st != kOk) {
        return st;
    }
    // symbols to the host while enc_update runs (worker, dmc_hts_proxy.cpp:778-793)
    if (cudaEventSynchronize(ev_phase_) != cudaSuccess) {
        return cuda_status(cudaGetLastError(), "compress: analysis");
    }
    st = check_device_error_word(err_word_, err_slot_, "compress");
    if (st != kOk) {
        return st;
    }
    const int count = *count_host_;
    if (count < 0 || count > y_num_) {
        set_last_error("compress: symbol count out of range");
        return kInternal;
    }
    const int ecp = ec_parallel_for(count);
    RansEncoderSession enc;
    enc.reset(ecp);
    enc.add_y(sym_host_, count, false);
    enc.add_z(z_host_, z_num_, qp * kChZ, kChZ, false);
    std::string err;
    if (!enc.finish(tables_, bytes, &err)) {
        set_last_error("compress: " + err);
        return kInternal;
    }
    *ec_parallel = ecp;
    last_count_ = count;
    return kOk;
}

int HtsCodec::decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                         bool reset, cudaStream_t caller, const __half** frames)
{
    if (!ready_ || Hp_ == 0) {
        set_last_error("decompress: set_param and add_ref_feature_from_frame must come first");
        return kNotReady;
    }
    if (qp < 0 || qp >= kQpNum || ecp < 1 || ecp > kMaxEcParallel || n > 0x7fffffff ||
        (n > 0 && bytes == nullptr) || height <= 0 || width <= 0 ||
        (height + 63) / 64 != H16p_ / 4 || (width + 63) / 64 != W16p_ / 4 ||
        ceil_to(height, 16) != Hp_ || ceil_to(width, 16) != Wp_) {
        set_last_error("decompress: bad qp, ec_parallel, stream or picture size (the size must "
                       "match the reference frame)");
        return kInvalidArgument;
    }
    last_kernels_ = 0;
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    set_qp(qp, main_);
    int st = run_phase(kDecTemporal + (memory_has_value_ ? 1 : 0), main_);
    // z on the CPU while the temporal branch runs (dmc_hts_proxy.cpp:794-804)
    RansDecoderSession dec;
    std::string err;
    if (st == kOk && (!dec.begin(bytes, static_cast<int>(n), ecp, &err) ||
                      !dec.decode_z(tables_, z_num_, qp * kChZ, kChZ, z_host_, &err))) {
        set_last_error("decompress: " + err);
        st = dec.fault() ? kInternal : kCorruptStream;
    }
    if (st == kOk) {
        st = run_phase(kDecHyper, main_);
    }
    if (st == kOk) st = cuda_status(cudaEventRecord(ev_phase_, main_), "decompress");
    if (st == kOk) st = run_phase(kDecContext, main_);
    if (st == kOk) {
        if (cudaEventSynchronize(ev_phase_) != cudaSuccess) {
            st = cuda_status(cudaGetLastError(), "decompress: hyper prior");
        }
    }
    if (st == kOk) st = check_device_error_word(err_word_, err_slot_, "decompress");
    int count = 0;
    if (st == kOk) {
        count = *count_host_;
        if (count < 0 || count > y_num_) {
            set_last_error("decompress: symbol count out of range");
            st = kInternal;
        }
    }
    // y on the CPU while the feature extractor runs (dmc_hts_proxy.cpp:805-823)
    if (st == kOk && !dec.decode_y(tables_, idx_host_, count, ydec_host_, &err)) {
        set_last_error("decompress: " + err);
        st = dec.fault() ? kInternal : kCorruptStream;
    }
    if (st == kOk) {
        st = run_phase(kDecSynthesis, main_);
    }
    if (st == kOk) {
        memory_has_value_ = !reset;
        for (int i = 0; i < kFrames; ++i) {
            frames[i] = x_hat_[i];
        }
        last_count_ = count;
    }
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    return st;
}

}  // namespace dcvc
