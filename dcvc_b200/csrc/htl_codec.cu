#include "htl_codec.h"

#include "elementwise.cuh"
#include "errors.h"
#include "gemm_sm100.cuh"
#include "quant_tables.h"

#include <algorithm>
#include <cstring>

namespace dcvc {

namespace {

inline int ceil_to(int v, int m) { return (v + m - 1) / m * m; }

std::string num(const char* prefix, int i, const char* suffix = ".")
{
    return std::string(prefix) + std::to_string(i) + suffix;
}

}  // namespace

HtlCodec::HtlCodec()
{
    cudaGetDevice(&dev_);
    cudaStreamCreateWithFlags(&main_, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&ev_in_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_phase_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_copy_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_out_, cudaEventDisableTiming);
    err_word_ = device_error_word();
    if (err_slot_.alloc()) {
        graphs_.set_error_slot(err_slot_.dev);
    }
}

HtlCodec::~HtlCodec()
{
    cudaSetDevice(dev_);
    if (main_ != nullptr) {
        cudaStreamSynchronize(main_);
    }
    if (copy_ != nullptr) {
        cudaStreamSynchronize(copy_);
    }
    graphs_.clear();
    cudaFreeHost(count_host_);
    cudaFreeHost(sym_host_);
    cudaFreeHost(idx_host_);
    cudaFreeHost(ydec_host_);
    cudaFreeHost(z_host_);
    cudaEventDestroy(ev_in_);
    cudaEventDestroy(ev_phase_);
    cudaEventDestroy(ev_copy_);
    cudaEventDestroy(ev_out_);
    cudaStreamDestroy(main_);
    cudaStreamDestroy(copy_);
    err_slot_.release();
}

int HtlCodec::set_param(const StateDict& sd, float skip_threshold)
{
    if (main_ != nullptr) {
        cudaStreamSynchronize(main_);
    }
    graphs_.clear();
    ready_ = false;
    weights_.clear();
    ParamBuilder B(sd, weights_);
    int r[3] = {0}, c[3] = {0};
    q_enc_tab_ = B.half_rows("q_encoder", &r[0], &c[0]);
    q_dec_tab_ = B.half_rows("q_decoder", &r[1], &c[1]);
    q_feat_tab_ = B.half_rows("q_feature", &r[2], &c[2]);
    // DMC(ModelStructure.HTL) layout (video_model_ht.py:24-351, is_hts False); resampling blocks
    // keep their default shortcut (DMCHTLHyper*/TemporalPriorEncoderProxy::set_param,
    // dmc_htl_proxy.cpp:275-308, 471-474)
    for (int i = 0; i < 7; ++i) {
        encoder_[i] = B.dcb(num("encoder.conv1.", i));
    }
    enc_down_ = B.conv3x3s2("encoder.down.");
    hyper_enc0_ = B.dcb("hyper_encoder.conv.0.");
    hyper_enc1_ = B.down("hyper_encoder.conv.1.", true);
    hyper_enc2_ = B.down("hyper_encoder.conv.2.", true);
    hyper_dec0_ = B.up("hyper_decoder.conv.0.", true);
    hyper_dec1_ = B.up("hyper_decoder.conv.1.", true);
    hyper_dec2_ = B.dcb("hyper_decoder.conv.2.");
    temporal_ = B.down("temporal_prior_encoder.conv.", true);
    for (int i = 0; i < 3; ++i) {
        prior_fusion_[i] = B.dcb(num("y_prior_fusion.conv.", i));
        sp_adaptor_[i] = B.dcb(num("y_spatial_prior_adaptor_", i + 1));
        spatial_prior_[i] = B.dcb(num("y_spatial_prior.conv.", i));
    }
    prior_fusion_out_ = B.lin("y_prior_fusion.conv.3.");
    reduction_ = B.lin("y_spatial_prior_reduction.");
    spatial_prior_out_ = B.lin("y_spatial_prior.conv.3.");
    dec_up_ = B.subpel("decoder.up.");
    for (int i = 0; i < 11; ++i) {
        decoder_[i] = B.dcb(num("decoder.conv1.", i));
    }
    for (int i = 0; i < 3; ++i) {
        fa_i_[i] = B.dcb(num("feature_adaptor_i.conv.", i));
    }
    for (int i = 0; i < 10; ++i) {
        fa_m_[i] = B.dcb(num("feature_adaptor_m.conv.", i));
    }
    for (int i = 0; i < 2; ++i) {
        fe_[i] = B.dcb(num("feature_extractor.conv.", i));
    }
    for (int i = 0; i < kFrames; ++i) {
        for (int j = 0; j < 5; ++j) {
            rh_[i][j] = B.dcb(num("recon_head.conv.", i, ".") + std::to_string(j) + ".");
        }
        rh_head_[i] = B.lin(num("recon_head.conv.", i, ".5."));
    }
    if (!B.ok()) {
        set_last_error("set_param: " + B.error());
        weights_.clear();
        return kInvalidArgument;
    }
    const bool shapes_ok =
        r[0] == kQpNum && c[0] == kChD && r[1] == kQpNum && c[1] == kChD && r[2] == kQpNum &&
        c[2] == kChD && encoder_[0].cin == kChSrc + kChD && encoder_[0].C == kChD &&
        encoder_[0].cdc == kChD && enc_down_.cin == 9 * kChD && enc_down_.cout == kChY &&
        hyper_enc2_.down.cout == kChZ && hyper_dec0_.up.cin == kChZ &&
        hyper_dec0_.up.cout == 4 * kChY && hyper_dec0_.up.b != nullptr &&
        temporal_.down.cin == 4 * kChD && temporal_.down.cout == 2 * kChY &&
        prior_fusion_[0].C == 3 * kChY && prior_fusion_out_.cout == 3 * kChY &&
        reduction_.cin == 3 * kChY && reduction_.cout == kChY && sp_adaptor_[0].C == 2 * kChY &&
        spatial_prior_out_.cout == 2 * kChY && dec_up_.cin == 9 * kChY &&
        dec_up_.cout == 4 * kChD && dec_up_.b != nullptr && decoder_[0].cin == 2 * kChD &&
        fa_i_[0].cin == kChSrcIntra && fa_m_[0].cin == kChM + kChD && fe_[0].C == kChD &&
        rh_[0][0].C == kChRecon && rh_head_[0].cout == kChSrcIntra && rh_head_[0].cin == kChRecon;
    if (!shapes_ok) {
        set_last_error("set_param: state dict is not an HT-L (DMC, ModelStructure.HTL) model");
        weights_.clear();
        return kInvalidArgument;
    }
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
    skip_thr_half_ = __float2half_rn(skip_threshold);
    ready_ = true;
    return kOk;
}

int HtlCodec::allocate(int Hp, int Wp)
{
    if (Hp == Hp_ && Wp == Wp_) {
        return kOk;
    }
    if (Hp <= 0 || Wp <= 0 || Hp % 16 || Wp % 16) {
        set_last_error("frame height and width must be positive multiples of 16");
        return kInvalidArgument;
    }
    cudaStreamSynchronize(main_);
    cudaStreamSynchronize(copy_);
    graphs_.clear();
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
    Hp_ = Wp_ = 0;

    H8_ = Hp / 8;
    W8_ = Wp / 8;
    H16_ = H8_ / 2;
    W16_ = W8_ / 2;
    H16p_ = ceil_to(H16_, 4);
    W16p_ = ceil_to(W16_, 4);
    M8_ = H8_ * W8_;
    M16_ = H16_ * W16_;
    M16p_ = H16p_ * W16p_;
    M32_ = (H16p_ / 2) * (W16p_ / 2);
    M64_ = (H16p_ / 4) * (W16p_ / 4);
    part_num_ = M16_ * (kChY / 4);
    z_num_ = M64_ * kChZ;
    const bool pad = (H16p_ != H16_) || (W16p_ != W16_);

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
    sp_out_ = H(M16 * 2 * kChY);
    y_q_ = H(M16 * kChY);
    part_ = H(M16 * (kChY / 4));
    z_ = H(M64 * kChZ);
    z_hat_ = H(M64 * kChZ);
    col_ = H(M16 * 9 * kChD);
    s2d_ = H(std::max({M16 * 4 * kChD, M32 * 4 * kChY, M64 * 4 * kChY}));
    lvl8_a_ = H(M8 * kChD);
    lvl16_a_ = H(M16p * 3 * kChY);
    lvl16_b_ = H(M16p * kChY);
    lvl32_a_ = H(M32 * kChY);
    lvl32_b_ = H(M32 * kChY);
    lvl64_a_ = H(M64 * kChZ);
    head_ = H(M8 * kChSrcIntra);
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
    z_i8_ = acts_.alloc_n<int8_t>(z_num_);
    sym_ = acts_.alloc_n<int16_t>(part_num_);
    sym_c_ = acts_.alloc_n<int16_t>(static_cast<size_t>(kSteps) * part_num_);
    idx_ = acts_.alloc_n<uint8_t>(part_num_);
    idx_c_ = acts_.alloc_n<uint8_t>(part_num_);
    cond_ = acts_.alloc_n<uint8_t>(part_num_);
    y_dec_ = acts_.alloc_n<int8_t>(part_num_);
    block_counts_ = acts_.alloc_n<int>(compact_blocks(part_num_));
    count_dev_ = acts_.alloc_n<int>(kSteps);
    ok = ok && z_i8_ && sym_ && sym_c_ && idx_ && idx_c_ && cond_ && y_dec_ && block_counts_ &&
         count_dev_;
    ok = ok && cudaMallocHost(&count_host_, sizeof(int) * kSteps) == cudaSuccess;
    ok = ok && cudaMallocHost(&sym_host_, sizeof(int16_t) * kSteps * part_num_) == cudaSuccess;
    ok = ok && cudaMallocHost(&idx_host_, part_num_) == cudaSuccess;
    ok = ok && cudaMallocHost(&ydec_host_, part_num_) == cudaSuccess;
    ok = ok && cudaMallocHost(&z_host_, z_num_) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        acts_.clear();
        set_last_error("out of device or pinned host memory for this resolution");
        return kOutOfMemory;
    }
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

void HtlCodec::set_qp(int qp, cudaStream_t s)
{
    cudaMemcpyAsync(q_enc_, q_enc_tab_ + static_cast<size_t>(qp) * kChD, kChD * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_dec_, q_dec_tab_ + static_cast<size_t>(qp) * kChD, kChD * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_feat_, q_feat_tab_ + static_cast<size_t>(qp) * kChD, kChD * 2,
                    cudaMemcpyDeviceToDevice, s);
}

// ------------------------------------------------------------------------------ network pieces

void HtlCodec::feature_adaptor_m(Launch& L)
{
    // memory = FA_m(cat(memory, feature_p)) (dmc_htl_proxy.cpp:969-988)
    run_dcb(L, fa_m_[0], cat_fam_, 1024, H8_, W8_, lvl8_a_, kChM, scratch_);
    for (int i = 1; i < 9; ++i) {
        run_dcb(L, fa_m_[i], lvl8_a_, kChM, H8_, W8_, lvl8_a_, kChM, scratch_);
    }
    run_dcb(L, fa_m_[9], lvl8_a_, kChM, H8_, W8_, cat_fam_, 1024, scratch_);
}

void HtlCodec::feature_adaptor_i(Launch& L, const __half* fi)
{
    run_dcb(L, fa_i_[0], fi, kChSrcIntra, H8_, W8_, lvl8_a_, kChM, scratch_);
    run_dcb(L, fa_i_[1], lvl8_a_, kChM, H8_, W8_, lvl8_a_, kChM, scratch_);
    run_dcb(L, fa_i_[2], lvl8_a_, kChM, H8_, W8_, cat_fam_, 1024, scratch_);
}

void HtlCodec::feature_extractor(Launch& L)
{
    __half* ctx = cat_enc_ + kChSrc;  // ctx lives in cat_enc[1536:2048]
    run_dcb(L, fe_[0], cat_fam_, 1024, H8_, W8_, ctx, 2048, scratch_);
    run_dcb(L, fe_[1], ctx, 2048, H8_, W8_, ctx, 2048, scratch_);
}

void HtlCodec::temporal_prior(Launch& L)
{
    // temporal params = RBWS2(memory * q_feature) -> cat_pf[256:768]
    L.note(launch_mul_channel(cat_fam_, M8_, kChM, 1024, q_feat_, temporal_in_, kChM, L.s));
    L.note(launch_space_to_depth2(temporal_in_, H8_, W8_, kChM, kChM, s2d_, L.s));
    gemm(L, temporal_.down, kEpiBias, s2d_, 4 * kChM, M16_, lvl16_a_, 2 * kChY);
    run_dcb(L, temporal_.dcb, lvl16_a_, 2 * kChY, H16_, W16_, cat_pf_ + kChY, 3 * kChY, scratch_);
}

void HtlCodec::hyper_prior(Launch& L)
{
    const int H32 = H16p_ / 2, W32 = W16p_ / 2, W64 = W16p_ / 4;
    const int C3 = 3 * kChY;
    gemm(L, hyper_dec0_.up, kEpiSubpel, z_hat_, kChZ, M64_, lvl32_a_, kChY, nullptr, 0, nullptr, W64);
    run_dcb(L, hyper_dec0_.dcb, lvl32_a_, kChY, H32, W32, lvl32_b_, kChY, scratch_);
    gemm(L, hyper_dec1_.up, kEpiSubpel, lvl32_b_, kChY, M32_, lvl16_b_, kChY, nullptr, 0, nullptr, W32);
    run_dcb(L, hyper_dec1_.dcb, lvl16_b_, kChY, H16p_, W16p_, lvl16_a_, kChY, scratch_);
    if (hyper_pad_ != nullptr) {
        run_dcb(L, hyper_dec2_, lvl16_a_, kChY, H16p_, W16p_, hyper_pad_, kChY, scratch_);
        L.note(launch_crop(hyper_pad_, W16p_, kChY, H16_, W16_, kChY, cat_pf_, C3, L.s));
    } else {
        run_dcb(L, hyper_dec2_, lvl16_a_, kChY, H16_, W16_, cat_pf_, C3, scratch_);
    }
    run_dcb(L, prior_fusion_[0], cat_pf_, C3, H16_, W16_, lvl16_a_, C3, scratch_);
    run_dcb(L, prior_fusion_[1], lvl16_a_, C3, H16_, W16_, lvl16_a_, C3, scratch_);
    run_dcb(L, prior_fusion_[2], lvl16_a_, C3, H16_, W16_, lvl16_a_, C3, scratch_);
    gemm(L, prior_fusion_out_, kEpiBias, lvl16_a_, C3, M16_, common_, C3);
    gemm(L, reduction_, kEpiBias, common_, C3, M16_, cat_spa_ + kChY, 2 * kChY);
}

void HtlCodec::spatial_prior(Launch& L, int k)
{
    const int C2 = 2 * kChY;
    run_dcb(L, sp_adaptor_[k - 1], cat_spa_, C2, H16_, W16_, lvl16_a_, C2, scratch_);
    for (int i = 0; i < 3; ++i) {
        run_dcb(L, spatial_prior_[i], lvl16_a_, C2, H16_, W16_, lvl16_a_, C2, scratch_);
    }
    gemm(L, spatial_prior_out_, kEpiBias, lvl16_a_, C2, M16_, sp_out_, C2);
}

void HtlCodec::decoder(Launch& L)
{
    // up: 3x3 conv + bias + pixel_shuffle(2) of y_hat (cat_spa[0:256]) -> cat_enc[1024:1536]
    // (SubpelConv2xProxy::forward, layers_proxy.cpp:269-276); DCBs on cat_enc[1024:2048]
    L.note(launch_im2col3x3s1(cat_spa_, H16_, W16_, kChY, 2 * kChY, col_, L.s));
    gemm(L, dec_up_, kEpiSubpel, col_, 9 * kChY, M16_, cat_enc_ + 1024, 2048, nullptr, 0, nullptr,
         W16_);
    run_dcb(L, decoder_[0], cat_enc_ + 1024, 2048, H8_, W8_, lvl8_a_, kChD, scratch_);
    for (int i = 1; i < 10; ++i) {
        run_dcb(L, decoder_[i], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    }
    run_dcb(L, decoder_[10], lvl8_a_, kChD, H8_, W8_, cat_fam_ + kChM, 1024, scratch_, q_dec_);
}

void HtlCodec::recon_head(Launch& L, bool all_frames)
{
    // one head per frame from feature_p (DMCHTLReconHeadProxy, dmc_htl_proxy.cpp:347-380)
    const __half* feature_p = cat_fam_ + kChM;
    for (int i = all_frames ? 0 : kFrames - 1; i < kFrames; ++i) {
        run_dcb(L, rh_[i][0], feature_p, 1024, H8_, W8_, lvl8_a_, kChRecon, scratch_);
        for (int j = 1; j < 5; ++j) {
            run_dcb(L, rh_[i][j], lvl8_a_, kChRecon, H8_, W8_, lvl8_a_, kChRecon, scratch_);
        }
        __half* out = (i == kFrames - 1) ? feature_i_ : head_;
        gemm(L, rh_head_[i], kEpiBias, lvl8_a_, kChRecon, M8_, out, kChSrcIntra);
        if (all_frames) {
            L.note(launch_shuffle8_clamp(out, H8_, W8_, 3, kChSrcIntra, x_hat_[i], L.s));
        }
    }
}

void HtlCodec::compact_step(Launch& L, int k, bool enc)
{
    if (enc) {
        L.note(launch_compact(sym_, 2, cond_, part_num_, block_counts_,
                              sym_c_ + static_cast<size_t>(k) * part_num_, count_dev_ + k, L.s),
               2);
    } else {
        L.note(launch_compact(idx_, 1, cond_, part_num_, block_counts_, idx_c_, count_dev_, L.s), 2);
    }
}

// ------------------------------------------------------------------------------ phases

void HtlCodec::enc_analysis(Launch& L)
{
    const int H32 = H16p_ / 2, W32 = W16p_ / 2, H64 = H16p_ / 4, W64 = W16p_ / 4;
    const int C3 = 3 * kChY, C2 = 2 * kChY;
    // encoder (DMCHTLEncoderProxy::forward, dmc_htl_proxy.cpp:93-106)
    run_dcb(L, encoder_[0], cat_enc_, 2048, H8_, W8_, lvl8_a_, kChD, scratch_);
    for (int i = 1; i < 6; ++i) {
        run_dcb(L, encoder_[i], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    }
    run_dcb(L, encoder_[6], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_, q_enc_);
    L.note(launch_im2col3x3s2(lvl8_a_, H8_, W8_, kChD, kChD, col_, L.s));
    gemm(L, enc_down_, kEpiBias, col_, 9 * kChD, M16_, y_, kChY);
    if (y_pad_ != y_) {
        L.note(launch_replicate_pad(y_, H16_, W16_, kChY, kChY, H16p_ - H16_, W16p_ - W16_, y_pad_, L.s));
    }
    // hyper encoder (shortcut resampling blocks)
    run_dcb(L, hyper_enc0_, y_pad_, kChY, H16p_, W16p_, lvl16_b_, kChY, scratch_);
    L.note(launch_space_to_depth2(lvl16_b_, H16p_, W16p_, kChY, kChY, s2d_, L.s));
    gemm(L, hyper_enc1_.down, kEpiBias, s2d_, 4 * kChY, M32_, lvl32_a_, kChY);
    run_dcb(L, hyper_enc1_.dcb, lvl32_a_, kChY, H32, W32, lvl32_b_, kChY, scratch_);
    L.note(launch_space_to_depth2(lvl32_b_, H32, W32, kChY, kChY, s2d_, L.s));
    gemm(L, hyper_enc2_.down, kEpiBias, s2d_, 4 * kChY, M64_, lvl64_a_, kChZ);
    run_dcb(L, hyper_enc2_.dcb, lvl64_a_, kChZ, H64, W64, z_, kChZ, scratch_);
    L.note(launch_round_z(z_, z_num_, z_hat_, z_i8_, L.s));
    temporal_prior(L);
    hyper_prior(L);
    // y / max(q_dec, 0.5), then the four checkerboard steps (dmc_htl_proxy.cpp:620-688)
    L.note(launch_div_clamp(y_, M16_, kChY, kChY, common_, C3, L.s));
    for (int k = 0; k < kSteps; ++k) {
        const __half* scales = common_ + kChY;
        const __half* means = common_ + 2 * kChY;
        int ld = C3;
        if (k > 0) {
            spatial_prior(L, k);
            scales = sp_out_;
            means = sp_out_ + kChY;
            ld = C2;
        }
        const int mode = k == 0 ? 0 : (k == kSteps - 1 ? 2 : 1);
        L.note(launch_quantize_phase(k, mode, y_, kChY, scales, ld, means, ld, common_, C3,
                                     skip_thr_half_, y_q_, kChY, cat_spa_, C2, H16_, W16_, kChY,
                                     L.s));
        L.note(launch_build_index_enc_4x(k, y_q_, kChY, scales, ld, skip_thr_half_, scale_lut_,
                                         H16_, W16_, kChY, sym_, cond_, L.s));
        compact_step(L, k, true);
    }
    L.note(cudaMemcpyAsync(count_host_, count_dev_, sizeof(int) * kSteps, cudaMemcpyDeviceToHost,
                           L.s),
           0);
}

void HtlCodec::enc_update(Launch& L, bool reset)
{
    decoder(L);
    if (reset) {
        recon_head(L, false);  // the reset head writes frame 7's head into feature_i
        feature_adaptor_i(L, feature_i_);
    } else {
        feature_adaptor_m(L);
    }
    feature_extractor(L);
}

void HtlCodec::dec_temporal(Launch& L, bool memory_has_value)
{
    if (memory_has_value) {
        feature_adaptor_m(L);
    } else {
        feature_adaptor_i(L, feature_i_);
    }
    temporal_prior(L);
}

void HtlCodec::dec_hyper(Launch& L)
{
    L.note(launch_int8_to_half(z_i8_, z_num_, z_hat_, L.s));
    hyper_prior(L);
    feature_extractor(L);
    L.note(launch_build_index_dec_4x(0, common_ + kChY, 3 * kChY, skip_thr_half_, scale_lut_, H16_,
                                     W16_, kChY, idx_, cond_, L.s));
    compact_step(L, 0, false);
    L.note(cudaMemcpyAsync(count_host_, count_dev_, sizeof(int), cudaMemcpyDeviceToHost, L.s), 0);
}

void HtlCodec::dec_step(Launch& L, int k)
{
    const int C2 = 2 * kChY;
    const __half* means_prev = k == 1 ? common_ + 2 * kChY : sp_out_ + kChY;
    const int ldm = k == 1 ? 3 * kChY : C2;
    L.note(launch_recover(y_dec_, cond_, block_counts_, part_num_, part_, L.s));
    L.note(launch_restore_4x(k - 1, k == 1 ? 0 : 1, part_, means_prev, ldm, nullptr, 0, cat_spa_,
                             C2, H16_, W16_, kChY, L.s));
    spatial_prior(L, k);
    L.note(launch_build_index_dec_4x(k, sp_out_, C2, skip_thr_half_, scale_lut_, H16_, W16_, kChY,
                                     idx_, cond_, L.s));
    compact_step(L, k, false);
    L.note(cudaMemcpyAsync(count_host_, count_dev_, sizeof(int), cudaMemcpyDeviceToHost, L.s), 0);
}

void HtlCodec::dec_final(Launch& L)
{
    const int C2 = 2 * kChY;
    L.note(launch_recover(y_dec_, cond_, block_counts_, part_num_, part_, L.s));
    L.note(launch_restore_4x(kSteps - 1, 2, part_, sp_out_ + kChY, C2, common_, 3 * kChY, cat_spa_,
                             C2, H16_, W16_, kChY, L.s));
    decoder(L);
    recon_head(L, true);
}

void HtlCodec::record_phase(int slot, Launch& L)
{
    switch (slot) {
    case kEncAnalysis: enc_analysis(L); break;
    case kEncUpdate: enc_update(L, false); break;
    case kEncUpdate + 1: enc_update(L, true); break;
    case kDecTemporal: dec_temporal(L, false); break;
    case kDecTemporal + 1: dec_temporal(L, true); break;
    case kDecHyper: dec_hyper(L); break;
    case kDecStep:
    case kDecStep + 1:
    case kDecStep + 2: dec_step(L, slot - kDecStep + 1); break;
    case kDecFinal: dec_final(L); break;
    default: break;
    }
}

int HtlCodec::run_phase(int slot, cudaStream_t s)
{
    return graphs_.run(slot, s, err_word_, [&](Launch& L) { record_phase(slot, L); },
                       &last_kernels_);
}

int HtlCodec::buffer(const std::string& name, const void** ptr, int* rows, int* cols,
                     int* ld) const
{
    if (Hp_ == 0) {
        set_last_error("buffer: no resolution allocated yet");
        return kNotReady;
    }
    struct Entry {
        const char* n;
        const __half* p;
        int rows, cols, ld;
    };
    const Entry e[] = {
        {"y_hat", cat_spa_, M16_, kChY, 2 * kChY},
        {"y_q", y_q_, M16_, kChY, kChY},
        {"memory", cat_fam_, M8_, kChM, 1024},
        {"feature_p", cat_fam_ + kChM, M8_, kChD, 1024},
        {"ctx", cat_enc_ + kChSrc, M8_, kChD, 2048},
        {"common", common_, M16_, 3 * kChY, 3 * kChY},
        {"feature_i", feature_i_, M8_, kChSrcIntra, kChSrcIntra},
    };
    for (const Entry& x : e) {
        if (name == x.n) {
            *ptr = x.p;
            *rows = x.rows;
            *cols = x.cols;
            *ld = x.ld;
            return kOk;
        }
    }
    set_last_error("buffer: unknown buffer '" + name + "'");
    return kInvalidArgument;
}

// ------------------------------------------------------------------------------ public calls

int HtlCodec::add_ref_feature(const __half* frame, int Hp, int Wp, bool apply_adaptor,
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
    L.note(launch_pad_unshuffle8(frame, Hp, Wp, 3, 3, 0, 0, feature_i_, kChSrcIntra, main_));
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

int HtlCodec::compress(const __half* x, int H, int W, int qp, bool reset, int pad_b, int pad_r,
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
    L.note(launch_pad_unshuffle8(x, H, W, 24, 24, pad_b, pad_r, cat_enc_, 2048, main_));
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
    // the four steps' symbols and z to the host while the decoder and memory update run (worker,
    // dmc_htl_proxy.cpp:503-582)
    if (cudaEventSynchronize(ev_phase_) != cudaSuccess) {
        return cuda_status(cudaGetLastError(), "compress: analysis");
    }
    st = check_device_error_word(err_word_, err_slot_, "compress");
    if (st != kOk) {
        return st;
    }
    int counts[kSteps];
    int total = 0;
    for (int k = 0; k < kSteps; ++k) {
        counts[k] = count_host_[k];
        if (counts[k] < 0 || counts[k] > part_num_) {
            set_last_error("compress: symbol count out of range");
            return kInternal;
        }
        total += counts[k];
    }
    for (int k = 0; k < kSteps; ++k) {
        if (counts[k] > 0) {
            cudaMemcpyAsync(sym_host_ + static_cast<size_t>(k) * part_num_,
                            sym_c_ + static_cast<size_t>(k) * part_num_,
                            sizeof(int16_t) * counts[k], cudaMemcpyDeviceToHost, copy_);
        }
    }
    cudaMemcpyAsync(z_host_, z_i8_, z_num_, cudaMemcpyDeviceToHost, copy_);
    if (cudaStreamSynchronize(copy_) != cudaSuccess) {
        return cuda_status(cudaGetLastError(), "compress: symbol copy");
    }
    const int ecp = ec_parallel_for(total);
    RansEncoderSession enc;
    enc.reset(ecp);
    for (int k = kSteps - 1; k >= 0; --k) {
        enc.add_y(sym_host_ + static_cast<size_t>(k) * part_num_, counts[k], false);
    }
    enc.add_z(z_host_, z_num_, qp * kChZ, kChZ, false);
    std::string err;
    if (!enc.finish(tables_, bytes, &err)) {
        set_last_error("compress: " + err);
        return kInternal;
    }
    *ec_parallel = ecp;
    last_count_ = total;
    return kOk;
}

int HtlCodec::decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                         bool reset, cudaStream_t caller, const __half** frames)
{
    if (!ready_ || Hp_ == 0) {
        set_last_error("decompress: set_param and add_ref_feature_from_frame must come first");
        return kNotReady;
    }
    if (qp < 0 || qp >= kQpNum || ecp < 1 || ecp > kMaxEcParallel || n > 0x7fffffff ||
        (n > 0 && bytes == nullptr) || height <= 0 || width <= 0 ||
        ceil_to(height, 16) != Hp_ || ceil_to(width, 16) != Wp_) {
        set_last_error("decompress: bad qp, ec_parallel, stream or picture size (the size must "
                       "match the reference frame)");
        return kInvalidArgument;
    }
    last_kernels_ = 0;
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    cudaStreamWaitEvent(copy_, ev_in_, 0);
    set_qp(qp, main_);
    int st = run_phase(kDecTemporal + (memory_has_value_ ? 1 : 0), main_);
    // z on the CPU while the memory update runs (worker DecodeZ)
    RansDecoderSession dec;
    std::string err;
    if (st == kOk && (!dec.begin(bytes, static_cast<int>(n), ecp, &err) ||
                      !dec.decode_z(tables_, z_num_, qp * kChZ, kChZ, z_host_, &err))) {
        set_last_error("decompress: " + err);
        st = dec.fault() ? kInternal : kCorruptStream;
    }
    if (st == kOk) {
        cudaMemcpyAsync(z_i8_, z_host_, z_num_, cudaMemcpyHostToDevice, copy_);
        cudaEventRecord(ev_copy_, copy_);
        cudaStreamWaitEvent(main_, ev_copy_, 0);
        st = run_phase(kDecHyper, main_);
    }
    int total = 0;
    // one CPU round trip per step (worker DecodeY)
    for (int k = 0; k < kSteps && st == kOk; ++k) {
        st = cuda_status(cudaEventRecord(ev_phase_, main_), "decompress");
        if (st == kOk && cudaEventSynchronize(ev_phase_) != cudaSuccess) {
            st = cuda_status(cudaGetLastError(), "decompress: index building");
        }
        if (st == kOk) st = check_device_error_word(err_word_, err_slot_, "decompress");
        int count = 0;
        if (st == kOk) {
            count = *count_host_;
            if (count < 0 || count > part_num_) {
                set_last_error("decompress: symbol count out of range");
                st = kInternal;
            }
        }
        if (st == kOk && count > 0) {
            cudaMemcpyAsync(idx_host_, idx_c_, count, cudaMemcpyDeviceToHost, copy_);
            if (cudaStreamSynchronize(copy_) != cudaSuccess) {
                st = cuda_status(cudaGetLastError(), "decompress: index copy");
            }
        }
        if (st == kOk && !dec.decode_y(tables_, idx_host_, count, ydec_host_, &err)) {
            set_last_error("decompress: " + err);
            st = dec.fault() ? kInternal : kCorruptStream;
        }
        if (st == kOk) {
            if (count > 0) {
                cudaMemcpyAsync(y_dec_, ydec_host_, count, cudaMemcpyHostToDevice, copy_);
            }
            cudaEventRecord(ev_copy_, copy_);
            cudaStreamWaitEvent(main_, ev_copy_, 0);
            st = run_phase(k + 1 < kSteps ? kDecStep + k : kDecFinal, main_);
            total += count;
        }
    }
    if (st == kOk) {
        memory_has_value_ = !reset;
        for (int i = 0; i < kFrames; ++i) {
            frames[i] = x_hat_[i];
        }
        last_count_ = total;
    }
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    return st;
}

}  // namespace dcvc
