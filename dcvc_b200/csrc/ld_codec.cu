#include "ld_codec.h"

#include "elementwise.cuh"
#include "errors.h"
#include "gemm_sm100.cuh"
#include "quant_tables.h"

#include <algorithm>
#include <cstring>
#include <type_traits>

namespace dcvc {

namespace {

inline int ceil_to(int v, int m) { return (v + m - 1) / m * m; }

std::string num(const char* prefix, int i, const char* suffix = ".")
{
    return std::string(prefix) + std::to_string(i) + suffix;
}

}  // namespace

LdCodec::LdCodec()
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

LdCodec::~LdCodec()
{
    cudaSetDevice(dev_);
    if (main_ != nullptr) {
        cudaStreamSynchronize(main_);
    }
    graphs_.clear();
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

int LdCodec::set_param(const StateDict& sd, float skip_threshold)
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
    // video_model_ld.DMC layout (video_model_ld.py:24-213): dcb2 blocks, no shortcuts
    encoder_[0] = B.dcb("encoder.conv1.0.");
    encoder_[1] = B.dcb("encoder.conv1.1.");
    encoder_[2] = B.dcb("encoder.conv2.");
    enc_down_ = B.conv3x3s2("encoder.down.");
    hyper_enc0_ = B.dcb("hyper_encoder.conv.0.");
    hyper_enc1_ = B.down("hyper_encoder.conv.1.");
    hyper_enc2_ = B.down("hyper_encoder.conv.2.");
    hyper_dec0_ = B.up("hyper_decoder.conv.0.");
    hyper_dec1_ = B.up("hyper_decoder.conv.1.");
    hyper_dec2_ = B.dcb("hyper_decoder.conv.2.");
    temporal_enc_ = B.down("temporal_prior_encoder.conv.");
    for (int i = 0; i < 3; ++i) {
        prior_fusion_[i] = B.dcb(num("y_prior_fusion.conv.", i));
        decoder_[i] = B.dcb(num("decoder.conv1.", i));
        rh_[i] = B.dcb(num("recon_head.conv.", i));
    }
    prior_fusion_out_ = B.lin("y_prior_fusion.conv.3.");
    spatial_prior_[0] = B.dcb("y_spatial_prior.conv.0.");
    spatial_prior_[1] = B.dcb("y_spatial_prior.conv.1.");
    spatial_prior_out_ = B.lin("y_spatial_prior.conv.2.");
    dec_up_ = B.subpel("decoder.up.");
    dec_conv2_ = B.lin("decoder.conv2.");
    for (int i = 0; i < 4; ++i) {
        fa_i_[i] = B.dcb(num("feature_adaptor_i.conv.", i));
        fa_m_[i] = B.dcb(num("feature_adaptor_m.conv.", i));
    }
    for (int i = 0; i < 5; ++i) {
        fe_[i] = B.dcb(num("feature_extractor.conv.", i));
    }
    rh_head_ = B.lin("recon_head.head.");
    if (!B.ok()) {
        set_last_error("set_param: " + B.error());
        weights_.clear();
        return kInvalidArgument;
    }
    const bool shapes_ok =
        r[0] == kQpNum && c[0] == kChD && r[1] == kQpNum && c[1] == kChD && r[2] == kQpNum &&
        c[2] == 2 * kChY && encoder_[0].cin == kChSrc + kChM && encoder_[0].C == kChD &&
        enc_down_.cin == 9 * kChD && enc_down_.cout == kChY && hyper_enc0_.C == kChZ &&
        hyper_enc2_.down.cout == kChZ && hyper_dec0_.up.cin == kChZ &&
        hyper_dec2_.C == kChY && temporal_enc_.down.cin == 4 * kChM &&
        temporal_enc_.down.cout == 2 * kChY && prior_fusion_[0].C == 3 * kChY &&
        prior_fusion_out_.cout == 3 * kChY && spatial_prior_[0].cin == 4 * kChY &&
        spatial_prior_out_.cout == kChY && dec_up_.cin == kChY && dec_up_.cout == 4 * kChD &&
        dec_up_.b == nullptr && decoder_[0].cin == kChD + kChM && dec_conv2_.cout == kChD &&
        fa_i_[0].cin == kChSrc && fa_m_[0].cin == kChM + kChD && fe_[0].C == kChM &&
        rh_head_.cout == kChSrc;
    if (!shapes_ok) {
        set_last_error("set_param: state dict is not a low-delay (video_model_ld.DMC) model");
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

int LdCodec::allocate(int Hp, int Wp)
{
    if (Hp == Hp_ && Wp == Wp_) {
        return kOk;
    }
    if (Hp <= 0 || Wp <= 0 || Hp % 16 || Wp % 16) {
        set_last_error("frame height and width must be positive multiples of 16");
        return kInvalidArgument;
    }
    cudaStreamSynchronize(main_);
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
    count_hdev_ = nullptr;
    sym_hdev_ = nullptr;
    idx_hdev_ = nullptr;
    ydec_hdev_ = nullptr;
    z_hdev_ = nullptr;
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
    y_num_ = M16_ * kChY;
    z_num_ = M64_ * kChZ;
    const bool pad = (H16p_ != H16_) || (W16p_ != W16_);

    bool ok = true;
    auto H = [&](size_t n) {
        __half* p = acts_.alloc_n<__half>(n);
        ok = ok && p != nullptr;
        return p;
    };
    const size_t M8 = M8_, M16 = M16_, M16p = M16p_, M32 = M32_, M64 = M64_;
    cat_enc_ = H(M8 * 512);
    cat_fam_ = H(M8 * 512);
    feature_i_ = H(M8 * kChSrc);
    y_ = H(M16 * kChY);
    y_pad_ = pad ? H(M16p * kChY) : y_;
    temporal_params_ = H(M16 * 2 * kChY);
    cat_pf_ = H(M16 * 3 * kChY);
    hyper_pad_ = pad ? H(M16p * kChY) : nullptr;
    cat_sp_ = H(M16 * 4 * kChY);
    means1_ = H(M16 * kChY);
    y_q_ = H(M16 * kChY);
    z_ = H(M64 * kChZ);
    z_hat_ = H(M64 * kChZ);
    col_ = H(M16 * 9 * kChD);
    s2d_ = H(std::max({M16 * 4 * kChM, M32 * 4 * kChZ, M64 * 4 * kChZ}));
    lvl8_a_ = H(M8 * kChD);
    lvl16_a_ = H(M16p * 3 * kChY);
    lvl32_a_ = H(M32 * kChZ);
    lvl64_a_ = H(M64 * kChZ);
    q_enc_ = H(kChD);
    q_dec_ = H(kChD);
    q_feat_ = H(2 * kChY);
    x_hat_ = H(static_cast<size_t>(Hp) * Wp * 3);
    const size_t S = std::max({M8 * kChD, M16p * 3 * kChY, M16 * 4 * kChY});
    scratch_.t0 = H(S);
    scratch_.t1 = H(S);
    scratch_.t2 = H(S);
    scratch_.t3 = H(S);
    scratch_.t4 = H(S);
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
    cudaMemsetAsync(cat_enc_, 0, M8 * 512 * 2, main_);
    cudaMemsetAsync(cat_fam_, 0, M8 * 512 * 2, main_);
    cudaMemsetAsync(cat_pf_, 0, M16 * 3 * kChY * 2, main_);
    cudaMemsetAsync(cat_sp_, 0, M16 * 4 * kChY * 2, main_);
    if (cudaStreamSynchronize(main_) != cudaSuccess) {
        return cuda_status(cudaGetLastError(), "allocate");
    }
    Hp_ = Hp;
    Wp_ = Wp;
    memory_has_value_ = false;
    return kOk;
}

void LdCodec::set_qp(int qp, cudaStream_t s)
{
    cudaMemcpyAsync(q_enc_, q_enc_tab_ + static_cast<size_t>(qp) * kChD, kChD * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_dec_, q_dec_tab_ + static_cast<size_t>(qp) * kChD, kChD * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_feat_, q_feat_tab_ + static_cast<size_t>(qp) * 2 * kChY, 2 * kChY * 2,
                    cudaMemcpyDeviceToDevice, s);
}

// ------------------------------------------------------------------------------ network pieces

void LdCodec::feature_adaptor_m(Launch& L)
{
    // memory = FA_m(cat(memory, feature_p)) (dmc_ld_proxy.cpp:639-658)
    run_dcb(L, fa_m_[0], cat_fam_, 512, H8_, W8_, lvl8_a_, kChM, scratch_);
    run_dcb(L, fa_m_[1], lvl8_a_, kChM, H8_, W8_, lvl8_a_, kChM, scratch_);
    run_dcb(L, fa_m_[2], lvl8_a_, kChM, H8_, W8_, lvl8_a_, kChM, scratch_);
    run_dcb(L, fa_m_[3], lvl8_a_, kChM, H8_, W8_, cat_fam_, 512, scratch_);
}

void LdCodec::feature_adaptor_i(Launch& L)
{
    run_dcb(L, fa_i_[0], feature_i_, kChSrc, H8_, W8_, lvl8_a_, kChM, scratch_);
    run_dcb(L, fa_i_[1], lvl8_a_, kChM, H8_, W8_, lvl8_a_, kChM, scratch_);
    run_dcb(L, fa_i_[2], lvl8_a_, kChM, H8_, W8_, lvl8_a_, kChM, scratch_);
    run_dcb(L, fa_i_[3], lvl8_a_, kChM, H8_, W8_, cat_fam_, 512, scratch_);
}

void LdCodec::feature_extractor(Launch& L)
{
    __half* ctx = cat_enc_ + 256;  // ctx lives in cat_enc[256:512]
    run_dcb(L, fe_[0], cat_fam_, 512, H8_, W8_, ctx, 512, scratch_);
    for (int i = 1; i < 5; ++i) {
        run_dcb(L, fe_[i], ctx, 512, H8_, W8_, ctx, 512, scratch_);
    }
}

void LdCodec::temporal_prior(Launch& L)
{
    // temporal params = RBWS2(memory), computed right after each memory update
    L.note(launch_space_to_depth2(cat_fam_, H8_, W8_, kChM, 512, s2d_, L.s));
    gemm(L, temporal_enc_.down, kEpiBias, s2d_, 4 * kChM, M16_, lvl16_a_, 2 * kChY);
    run_dcb(L, temporal_enc_.dcb, lvl16_a_, 2 * kChY, H16_, W16_, temporal_params_, 2 * kChY, scratch_);
}

void LdCodec::entropy_params(Launch& L)
{
    const int H32 = H16p_ / 2, W32 = W16p_ / 2, W64 = W16p_ / 4;
    const int C3 = 3 * kChY;
    gemm(L, hyper_dec0_.up, kEpiSubpel, z_hat_, kChZ, M64_, lvl32_a_, kChZ, nullptr, 0, nullptr, W64);
    run_dcb(L, hyper_dec0_.dcb, lvl32_a_, kChZ, H32, W32, lvl32_a_, kChZ, scratch_);
    gemm(L, hyper_dec1_.up, kEpiSubpel, lvl32_a_, kChZ, M32_, lvl16_a_, kChZ, nullptr, 0, nullptr, W32);
    run_dcb(L, hyper_dec1_.dcb, lvl16_a_, kChZ, H16p_, W16p_, lvl16_a_, kChZ, scratch_);
    if (hyper_pad_ != nullptr) {
        run_dcb(L, hyper_dec2_, lvl16_a_, kChZ, H16p_, W16p_, hyper_pad_, kChY, scratch_);
        L.note(launch_crop(hyper_pad_, W16p_, kChY, H16_, W16_, kChY, cat_pf_, C3, L.s));
    } else {
        run_dcb(L, hyper_dec2_, lvl16_a_, kChZ, H16_, W16_, cat_pf_, C3, scratch_);
    }
    // prior fusion over cat(hyper, temporal x q_feature) (dmc_ld_proxy.cpp:440-443)
    L.note(launch_mul_channel(temporal_params_, M16_, 2 * kChY, 2 * kChY, q_feat_, cat_pf_ + kChY, C3, L.s));
    run_dcb(L, prior_fusion_[0], cat_pf_, C3, H16_, W16_, lvl16_a_, C3, scratch_);
    run_dcb(L, prior_fusion_[1], lvl16_a_, C3, H16_, W16_, lvl16_a_, C3, scratch_);
    run_dcb(L, prior_fusion_[2], lvl16_a_, C3, H16_, W16_, lvl16_a_, C3, scratch_);
    // q_dec | scales | means land in cat_sp[128:512], next to y_hat for the spatial prior
    gemm(L, prior_fusion_out_, kEpiBias, lvl16_a_, C3, M16_, cat_sp_ + kChY, 4 * kChY);
}

void LdCodec::spatial_prior(Launch& L)
{
    // means of phase 1 = SP(cat(y_hat of phase 0, common params))
    run_dcb(L, spatial_prior_[0], cat_sp_, 4 * kChY, H16_, W16_, lvl16_a_, 2 * kChY, scratch_);
    run_dcb(L, spatial_prior_[1], lvl16_a_, 2 * kChY, H16_, W16_, lvl16_a_, 2 * kChY, scratch_);
    gemm(L, spatial_prior_out_, kEpiBias, lvl16_a_, 2 * kChY, M16_, means1_, kChY);
}

void LdCodec::decoder(Launch& L)
{
    // DMCLDDecoderProxy::forward (dmc_ld_proxy.cpp:14-35): up -> cat_enc[0:256], DCBs on
    // cat(up, ctx), conv2 with bias x q_decoder -> feature_p (cat_fam[256:512])
    gemm(L, dec_up_, kEpiSubpel, cat_sp_, 4 * kChY, M16_, cat_enc_, 512, nullptr, 0, nullptr, W16_);
    run_dcb(L, decoder_[0], cat_enc_, 512, H8_, W8_, lvl8_a_, kChD, scratch_);
    run_dcb(L, decoder_[1], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    run_dcb(L, decoder_[2], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    gemm(L, dec_conv2_, kEpiBiasQ, lvl8_a_, kChD, M8_, cat_fam_ + kChM, 512, nullptr, 0, q_dec_);
}

void LdCodec::recon_head(Launch& L, bool shuffle)
{
    // DMCLDReconHeadProxy (dmc_ld_proxy.cpp:286-306): the head output is kept in feature_i for
    // a later reset
    run_dcb(L, rh_[0], cat_fam_ + kChM, 512, H8_, W8_, lvl8_a_, kChD, scratch_);
    run_dcb(L, rh_[1], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    run_dcb(L, rh_[2], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    gemm(L, rh_head_, kEpiBias, lvl8_a_, kChD, M8_, feature_i_, kChSrc);
    if (shuffle) {
        L.note(launch_shuffle8_clamp(feature_i_, H8_, W8_, 3, kChSrc, x_hat_, L.s));
    }
}

// ------------------------------------------------------------------------------ phases

void LdCodec::enc_analysis(Launch& L)
{
    const int H32 = H16p_ / 2, W32 = W16p_ / 2, H64 = H16p_ / 4, W64 = W16p_ / 4;
    const int C4 = 4 * kChY;
    // encoder (DMCLDEncoderProxy::forward, dmc_ld_proxy.cpp:61-68): input cat_enc[64:512]
    run_dcb(L, encoder_[0], cat_enc_ + 64, 512, H8_, W8_, lvl8_a_, kChD, scratch_);
    run_dcb(L, encoder_[1], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_);
    run_dcb(L, encoder_[2], lvl8_a_, kChD, H8_, W8_, lvl8_a_, kChD, scratch_, q_enc_);
    L.note(launch_im2col3x3s2(lvl8_a_, H8_, W8_, kChD, kChD, col_, L.s));
    gemm(L, enc_down_, kEpiBias, col_, 9 * kChD, M16_, y_, kChY);
    if (y_pad_ != y_) {
        L.note(launch_replicate_pad(y_, H16_, W16_, kChY, kChY, H16p_ - H16_, W16p_ - W16_, y_pad_, L.s));
    }
    run_dcb(L, hyper_enc0_, y_pad_, kChY, H16p_, W16p_, lvl16_a_, kChZ, scratch_);
    L.note(launch_space_to_depth2(lvl16_a_, H16p_, W16p_, kChZ, kChZ, s2d_, L.s));
    gemm(L, hyper_enc1_.down, kEpiBias, s2d_, 4 * kChZ, M32_, lvl32_a_, kChZ);
    run_dcb(L, hyper_enc1_.dcb, lvl32_a_, kChZ, H32, W32, lvl32_a_, kChZ, scratch_);
    L.note(launch_space_to_depth2(lvl32_a_, H32, W32, kChZ, kChZ, s2d_, L.s));
    gemm(L, hyper_enc2_.down, kEpiBias, s2d_, 4 * kChZ, M64_, lvl64_a_, kChZ);
    run_dcb(L, hyper_enc2_.dcb, lvl64_a_, kChZ, H64, W64, z_, kChZ, scratch_);
    L.note(launch_round_z(z_, z_num_, z_hat_, z_i8_, L.s));
    entropy_params(L);
    // y / max(q_dec, 0.5); 2-phase quantisation with the spatial prior between the phases
    // (dmc_ld_proxy.cpp:444-453)
    const __half* q_dec = cat_sp_ + kChY;
    const __half* scales = cat_sp_ + 2 * kChY;
    const __half* means0 = cat_sp_ + 3 * kChY;
    L.note(launch_div_clamp(y_, M16_, kChY, kChY, q_dec, C4, L.s));
    L.note(launch_quantize_phase(0, 0, y_, kChY, scales, C4, means0, C4, nullptr, 0,
                                 skip_thr_half_, y_q_, kChY, cat_sp_, C4, H16_, W16_, kChY, L.s,
                                 2));
    spatial_prior(L);
    L.note(launch_quantize_phase(1, 2, y_, kChY, scales, C4, means1_, kChY, q_dec, C4,
                                 skip_thr_half_, y_q_, kChY, cat_sp_, C4, H16_, W16_, kChY, L.s,
                                 2));
    L.note(launch_build_index_enc(y_q_, kChY, scales, C4, skip_thr_half_, scale_lut_, M16_, kChY,
                                  sym_, cond_, L.s));
    L.note(launch_compact(sym_, 2, cond_, y_num_, block_counts_, sym_c_, count_dev_, L.s), 2);
    // the symbols, their count and z to the mapped host buffers
    L.note(launch_copy_counted(sym_c_, sym_hdev_, 2, count_dev_, y_num_, count_hdev_, L.s));
    L.note(launch_copy_counted(z_i8_, z_hdev_, 1, nullptr, z_num_, nullptr, L.s));
}

void LdCodec::enc_update(Launch& L, bool reset)
{
    decoder(L);
    if (reset) {
        recon_head(L, false);  // forward_reset: the head output feeds FA_i
        feature_adaptor_i(L);
    } else {
        feature_adaptor_m(L);
    }
    feature_extractor(L);
    temporal_prior(L);
}

void LdCodec::dec_temporal(Launch& L, bool memory_has_value)
{
    if (memory_has_value) {
        feature_adaptor_m(L);
    } else {
        feature_adaptor_i(L);
    }
    temporal_prior(L);
}

void LdCodec::dec_hyper(Launch& L)
{
    L.note(launch_int8_to_half(z_hdev_, z_num_, z_hat_, L.s));  // z as decoded on the host
    entropy_params(L);
    L.note(launch_build_index_dec(cat_sp_ + 2 * kChY, 4 * kChY, skip_thr_half_, scale_lut_, M16_,
                                  kChY, idx_, cond_, L.s));
    L.note(launch_compact(idx_, 1, cond_, y_num_, block_counts_, idx_c_, count_dev_, L.s), 2);
    L.note(launch_copy_counted(idx_c_, idx_hdev_, 1, count_dev_, y_num_, count_hdev_, L.s));
}

void LdCodec::dec_synthesis(Launch& L)
{
    const int C4 = 4 * kChY;
    L.note(launch_copy_counted(ydec_hdev_, y_dec_, 1, count_dev_, y_num_, nullptr, L.s));
    L.note(launch_recover(y_dec_, cond_, block_counts_, y_num_, y_q_, L.s));
    L.note(launch_restore_phase(0, 0, y_q_, kChY, cat_sp_ + 3 * kChY, C4, nullptr, 0, cat_sp_, C4,
                                H16_, W16_, kChY, L.s, 2));
    spatial_prior(L);
    L.note(launch_restore_phase(1, 2, y_q_, kChY, means1_, kChY, cat_sp_ + kChY, C4, cat_sp_, C4,
                                H16_, W16_, kChY, L.s, 2));
    decoder(L);
    recon_head(L, true);
}

void LdCodec::record_phase(int slot, Launch& L)
{
    switch (slot) {
    case kEncAnalysis: enc_analysis(L); break;
    case kEncUpdate: enc_update(L, false); break;
    case kEncUpdate + 1: enc_update(L, true); break;
    case kDecTemporal: dec_temporal(L, false); break;
    case kDecTemporal + 1: dec_temporal(L, true); break;
    case kDecHyper: dec_hyper(L); break;
    case kDecContext: feature_extractor(L); break;
    case kDecSynthesis: dec_synthesis(L); break;
    default: break;
    }
}

int LdCodec::run_phase(int slot, cudaStream_t s)
{
    return graphs_.run(slot, s, err_word_, [&](Launch& L) { record_phase(slot, L); },
                       &last_kernels_);
}

int LdCodec::buffer(const std::string& name, const void** ptr, int* rows, int* cols,
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
        {"y_hat", cat_sp_, M16_, kChY, 4 * kChY},
        {"y_q", y_q_, M16_, kChY, kChY},
        {"memory", cat_fam_, M8_, kChM, 512},
        {"feature_p", cat_fam_ + kChM, M8_, kChD, 512},
        {"ctx", cat_enc_ + 256, M8_, kChM, 512},
        {"common", cat_sp_ + kChY, M16_, 3 * kChY, 4 * kChY},
        {"feature_i", feature_i_, M8_, kChSrc, kChSrc},
        {"temporal", temporal_params_, M16_, 2 * kChY, 2 * kChY},
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

int LdCodec::add_ref_feature(const __half* frame, int Hp, int Wp, bool apply_adaptor,
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
    L.note(launch_pad_unshuffle8(frame, Hp, Wp, 3, 3, 0, 0, feature_i_, kChSrc, main_));
    if (apply_adaptor) {
        feature_adaptor_i(L);
        feature_extractor(L);
        temporal_prior(L);
    }
    memory_has_value_ = apply_adaptor;
    last_kernels_ += L.kernels;
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    return cuda_status(L.first, "add_ref_feature_from_frame");
}

int LdCodec::compress(const __half* x, int H, int W, int qp, bool reset, int pad_b, int pad_r,
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
    L.note(launch_pad_unshuffle8(x, H, W, 3, 3, pad_b, pad_r, cat_enc_ + 64, 512, main_));
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

int LdCodec::decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                        bool reset, cudaStream_t caller, const __half** frame)
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
    set_qp(qp, main_);
    int st = run_phase(kDecTemporal + (memory_has_value_ ? 1 : 0), main_);
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
    if (st == kOk && cudaEventSynchronize(ev_phase_) != cudaSuccess) {
        st = cuda_status(cudaGetLastError(), "decompress: hyper prior");
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
    if (st == kOk && !dec.decode_y(tables_, idx_host_, count, ydec_host_, &err)) {
        set_last_error("decompress: " + err);
        st = dec.fault() ? kInternal : kCorruptStream;
    }
    if (st == kOk) {
        st = run_phase(kDecSynthesis, main_);
    }
    if (st == kOk) {
        memory_has_value_ = !reset;
        *frame = x_hat_;
        last_count_ = count;
    }
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    return st;
}

}  // namespace dcvc
