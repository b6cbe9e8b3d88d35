#include "hts_codec.h"

#include "elementwise.cuh"
#include "errors.h"
#include "gemm_sm100.cuh"
#include "quant_tables.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <type_traits>

namespace dcvc {

namespace {

constexpr int kMaskPhases = 4;

inline int ceil_to(int v, int m) { return (v + m - 1) / m * m; }

// two branches: 9.44 against 9.55 ms per 1080p chunk (dec_synthesis 3.75 against 3.99 ms), the
// second branch's kernels filling the SMs that the first branch's kernels leave idle in their tails
std::atomic<int> g_recon_branches{2};

std::string num(const char* prefix, int i, const char* suffix = ".")
{
    return std::string(prefix) + std::to_string(i) + suffix;
}

}  // namespace

void HtsCodec::set_recon_branches(int n) { g_recon_branches.store((n == 2 || n == 4) ? n : 1); }

HtsCodec::HtsCodec()
{
    cudaGetDevice(&dev_);
    cudaStreamCreateWithFlags(&main_, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming);
    for (int b = 0; b < kMaxReconBranches - 1; ++b) {
        cudaStreamCreateWithFlags(&side_[b], cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&ev_join_[b], cudaEventDisableTiming);
    }
    cudaEventCreateWithFlags(&ev_in_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_phase_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_out_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_state_, cudaEventDisableTiming);
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
    cudaEventDestroy(ev_state_);
    cudaEventDestroy(ev_fork_);
    for (int b = 0; b < kMaxReconBranches - 1; ++b) {
        cudaEventDestroy(ev_join_[b]);
        cudaStreamDestroy(side_[b]);
    }
    for (auto& e : tev_) {
        if (e[0] != nullptr) {
            cudaEventDestroy(e[0]);
            cudaEventDestroy(e[1]);
        }
    }
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
    weights_ = std::make_shared<DeviceArena>();
    ParamBuilder B(sd, *weights_);
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
        weights_.reset();
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
        weights_.reset();
        return kInvalidArgument;
    }
    // CDF tables (set_param, dmc_hts_proxy.cpp:748-761)
    if (load_cdf_tables(sd, &tables_, kQpNum * kChZ, 128) != kOk) {
        weights_.reset();
        return kInvalidArgument;
    }
    // the scale -> CDF index table, evaluated on the device as the reference's FP16
    // scale_to_index computes it
    scale_lut_ = weights_->alloc_n<uint8_t>(65536);
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

int HtsCodec::allocate(int Hp, int Wp, int imgs)
{
    if (Hp == Hp_ && Wp == Wp_ && imgs == imgs_) {
        return kOk;
    }
    if (Hp <= 0 || Wp <= 0 || Hp % 16 || Wp % 16) {
        set_last_error("frame height and width must be positive multiples of 16");
        return kInvalidArgument;
    }
    if (imgs < 1 || imgs > kMaxBatch) {
        set_last_error("a packed batch holds 1 to " + std::to_string(kMaxBatch) + " streams");
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
    imgs_ = 0;

    const int H8 = Hp / 8, W8 = Wp / 8;
    const int H16 = H8 / 2, W16 = W8 / 2;
    const int H16p = ceil_to(H16, 4), W16p = ceil_to(W16, 4);
    H8_ = H8;
    W8_ = W8;
    H16_ = H16;
    W16_ = W16;
    H16p_ = H16p;
    W16p_ = W16p;
    // per image, and stacked over the batch's images (row counts of every activation buffer)
    m8_ = H8 * W8;
    m16_ = H16 * W16;
    m16p_ = H16p * W16p;
    TH8_ = imgs * H8;
    TH16_ = imgs * H16;
    TH16p_ = imgs * H16p;
    TH32_ = imgs * (H16p / 2);
    TH64_ = imgs * (H16p / 4);
    M8_ = imgs * H8 * W8;
    M16_ = imgs * H16 * W16;
    M16p_ = imgs * H16p * W16p;
    M32_ = imgs * (H16p / 2) * (W16p / 2);
    M64_ = imgs * (H16p / 4) * (W16p / 4);
    ny_ = m16_ * kChY;
    nz_ = (H16p / 4) * (W16p / 4) * kChZ;
    y_num_ = imgs * ny_;
    z_num_ = imgs * nz_;
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
    q_enc_ = H(static_cast<size_t>(imgs) * kChD);
    q_dec_ = H(static_cast<size_t>(imgs) * kChD);
    q_feat_ = H(static_cast<size_t>(imgs) * kChD);
    for (int i = 0; i < kFrames; ++i) {
        x_hat_[i] = H(static_cast<size_t>(imgs) * Hp * Wp * 3);
    }
    const size_t S = std::max(M8 * kChD, M16p * 3 * kChY);
    scratch_.t0 = H(S);
    scratch_.t1 = H(S);
    scratch_.t2 = H(S);
    scratch_.t3 = H(S);
    scratch_.t4 = H(S);
    scratch_.t5 = fp8_ ? acts_.alloc_n<uint8_t>(M8 * kChD) : nullptr;
    ok = ok && (!fp8_ || scratch_.t5 != nullptr);
    // the temporal prior's side branch (enc_analysis): its DepthConvBlock is 512 channels wide at
    // the 1/16 scale
    s2d_t_ = H(M16 * 4 * kChM);
    lvl16_t_ = H(M16 * 2 * kChY);
    {
        const size_t St = M16 * 4 * kChY;
        scratch_t_.t0 = H(St);
        scratch_t_.t1 = H(St);
        scratch_t_.t2 = H(St);
        scratch_t_.t3 = H(St);
        scratch_t_.t4 = H(St);
        scratch_t_.t5 = nullptr;  // the entropy-parameter path stays 16-bit in every form
    }
    recon_branches_ = g_recon_branches.load();
    rb_a_[0] = lvl8_a_;
    rb_b_[0] = lvl8_b_;
    rb_head_[0] = head_;
    rb_scratch_[0] = scratch_;
    for (int b = 1; b < recon_branches_; ++b) {
        rb_a_[b] = H(M8 * kChD);
        rb_b_[b] = H(M8 * kChD);
        rb_head_[b] = H(M8 * kChSrcIntra);
        rb_scratch_[b].t0 = H(S);
        rb_scratch_[b].t1 = H(S);
        rb_scratch_[b].t2 = H(S);
        rb_scratch_[b].t3 = H(S);
        rb_scratch_[b].t4 = H(S);
        rb_scratch_[b].t5 = fp8_ ? acts_.alloc_n<uint8_t>(M8 * kChD) : nullptr;
        ok = ok && (!fp8_ || rb_scratch_[b].t5 != nullptr);
    }
    z_i8_ = acts_.alloc_n<int8_t>(z_num_);
    sym_ = acts_.alloc_n<int16_t>(y_num_);
    sym_c_ = acts_.alloc_n<int16_t>(y_num_);
    idx_ = acts_.alloc_n<uint8_t>(y_num_);
    idx_c_ = acts_.alloc_n<uint8_t>(y_num_);
    cond_ = acts_.alloc_n<uint8_t>(y_num_);
    y_dec_ = acts_.alloc_n<int8_t>(y_num_);
    block_counts_ = acts_.alloc_n<int>(static_cast<size_t>(imgs) * compact_blocks(ny_));
    count_dev_ = acts_.alloc_n<int>(imgs);
    ok = ok && z_i8_ && sym_ && sym_c_ && idx_ && idx_c_ && cond_ && y_dec_ && block_counts_ &&
         count_dev_;
    auto mapped = [&](size_t bytes, auto** host, auto** dev) {
        void *h = nullptr, *d = nullptr;
        ok = ok && alloc_mapped(bytes, &h, &d);
        *host = static_cast<std::remove_reference_t<decltype(**host)>*>(h);
        *dev = static_cast<std::remove_reference_t<decltype(**dev)>*>(d);
    };
    mapped(sizeof(int) * (imgs + 1), &count_host_, &count_hdev_);
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
    imgs_ = imgs;
    memory_has_value_ = false;
    return kOk;
}

void HtsCodec::set_qp(const int* qps, cudaStream_t s)
{
    for (int k = 0; k < imgs_; ++k) {
        const size_t src = static_cast<size_t>(qps[k]) * kChD, dst = static_cast<size_t>(k) * kChD;
        cudaMemcpyAsync(q_enc_ + dst, q_enc_tab_ + src, kChD * 2, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(q_dec_ + dst, q_dec_tab_ + src, kChD * 2, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(q_feat_ + dst, q_feat_tab_ + src, kChD * 2, cudaMemcpyDeviceToDevice, s);
    }
}

// ------------------------------------------------------------------------------ network pieces

void HtsCodec::feature_adaptor_m(Launch& L)
{
    // memory = FA_m(cat(memory, feature_p))   (dmc_hts_proxy.cpp:845-851)
    run_dcb(L, fa_m_[0], cat_fam_, 1024, TH8_, W8_, lvl8_a_, kChM, scratch_, nullptr, H8_);
    for (int i = 1; i < 5; ++i) {
        run_dcb(L, fa_m_[i], lvl8_a_, kChM, TH8_, W8_, lvl8_a_, kChM, scratch_, nullptr, H8_);
    }
    run_dcb(L, fa_m_[5], lvl8_a_, kChM, TH8_, W8_, cat_fam_, 1024, scratch_, nullptr, H8_);
}

void HtsCodec::feature_adaptor_i(Launch& L, const __half* fi)
{
    run_dcb(L, fa_i_[0], fi, kChSrcIntra, TH8_, W8_, lvl8_a_, kChM, scratch_, nullptr, H8_);
    for (int i = 1; i < 3; ++i) {
        run_dcb(L, fa_i_[i], lvl8_a_, kChM, TH8_, W8_, lvl8_a_, kChM, scratch_, nullptr, H8_);
    }
    run_dcb(L, fa_i_[3], lvl8_a_, kChM, TH8_, W8_, cat_fam_, 1024, scratch_, nullptr, H8_);
}

void HtsCodec::feature_extractor(Launch& L)
{
    // ctx = FE(memory); ctx lives in cat_enc[1536:2048]
    __half* ctx = cat_enc_ + kChSrc;
    run_dcb(L, fe_[0], cat_fam_, 1024, TH8_, W8_, ctx, 2048, scratch_, nullptr, H8_);
    for (int i = 1; i < 5; ++i) {
        run_dcb(L, fe_[i], ctx, 2048, TH8_, W8_, ctx, 2048, scratch_, nullptr, H8_);
    }
}

void HtsCodec::temporal_prior(Launch& L, __half* s2d, __half* lvl16, Scratch& sc)
{
    // temporal_params = RBWS2(memory * q_feature) -> cat_pf[256:768]
    L.note(launch_mul_channel(cat_fam_, M8_, kChM, 1024, q_feat_, temporal_in_, kChM, L.s, act_,
                              imgs_ > 1 ? m8_ : 0));
    L.note(launch_space_to_depth2(temporal_in_, TH8_, W8_, kChM, kChM, s2d, L.s));
    gemm(L, temporal_.down, kEpiBias, s2d, 4 * kChM, M16_, lvl16, 2 * kChY);
    run_dcb(L, temporal_.dcb, lvl16, 2 * kChY, TH16_, W16_, cat_pf_ + kChY, 3 * kChY, sc, nullptr, H16_);
}

void HtsCodec::hyper_decoder(Launch& L)
{
    const int H64 = H16p_ / 4, W64 = W16p_ / 4, H32 = H16p_ / 2, W32 = W16p_ / 2;
    gemm(L, hyper_dec0_.up, kEpiSubpel, z_hat_, kChZ, M64_, lvl32_a_, kChY, nullptr, 0, nullptr, W64);
    run_dcb(L, hyper_dec0_.dcb, lvl32_a_, kChY, TH32_, W32, lvl32_a_, kChY, scratch_, nullptr, H32);
    gemm(L, hyper_dec1_.up, kEpiSubpel, lvl32_a_, kChY, M32_, lvl16_a_, kChY, nullptr, 0, nullptr, W32);
    run_dcb(L, hyper_dec1_.dcb, lvl16_a_, kChY, TH16p_, W16p_, lvl16_a_, kChY, scratch_, nullptr, H16p_);
    if (hyper_pad_ != nullptr) {
        run_dcb(L, hyper_dec2_, lvl16_a_, kChY, TH16p_, W16p_, hyper_pad_, kChY, scratch_, nullptr, H16p_);
        for (int k = 0; k < imgs_; ++k) {  // each image's top-left H16 x W16 part
            L.note(launch_crop(hyper_pad_ + static_cast<size_t>(k) * m16p_ * kChY, W16p_, kChY, H16_,
                               W16_, kChY, cat_pf_ + static_cast<size_t>(k) * m16_ * 3 * kChY,
                               3 * kChY, L.s));
        }
    } else {
        run_dcb(L, hyper_dec2_, lvl16_a_, kChY, TH16_, W16_, cat_pf_, 3 * kChY, scratch_, nullptr, H16_);
    }
}

void HtsCodec::prior_fusion(Launch& L)
{
    const int C = 3 * kChY;
    run_dcb(L, prior_fusion_[0], cat_pf_, C, TH16_, W16_, lvl16_a_, C, scratch_, nullptr, H16_);
    run_dcb(L, prior_fusion_[1], lvl16_a_, C, TH16_, W16_, lvl16_a_, C, scratch_, nullptr, H16_);
    run_dcb(L, prior_fusion_[2], lvl16_a_, C, TH16_, W16_, lvl16_a_, C, scratch_, nullptr, H16_);
    gemm(L, prior_fusion_out_, kEpiBias, lvl16_a_, C, M16_, common_, C);
}

void HtsCodec::spatial_prior(Launch& L, int k)
{
    const int C = 2 * kChY;
    run_dcb(L, sp_adaptor_[k], cat_spa_, C, TH16_, W16_, lvl16_a_, C, scratch_, nullptr, H16_);
    for (int i = 0; i < 3; ++i) {
        run_dcb(L, spatial_prior_[i], lvl16_a_, C, TH16_, W16_, lvl16_a_, C, scratch_, nullptr, H16_);
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
    run_dcb(L, decoder_[0], cat_enc_ + 1024, 2048, TH8_, W8_, lvl8_a_, kChD, scratch_, nullptr, H8_);
    for (int i = 1; i < 6; ++i) {
        run_dcb(L, decoder_[i], lvl8_a_, kChD, TH8_, W8_, lvl8_a_, kChD, scratch_, nullptr, H8_);
    }
    run_dcb(L, decoder_[6], lvl8_a_, kChD, TH8_, W8_, cat_fam_ + kChM, 1024, scratch_, q_dec_, H8_);
}

void HtsCodec::recon_head(Launch& L, bool all_frames)
{
    const __half* feature_p = cat_fam_ + kChM;
    // frames [f0, f1) on launch context C with its own buffers
    auto frames = [&](Launch& C, int f0, int f1, __half* a, __half* b, __half* head, Scratch& sc) {
        for (int i = f0; i < f1; ++i) {
            if (i % 2 == 0 || !all_frames) {
                run_dcb(C, rh_common_[i / 2], feature_p, 1024, TH8_, W8_, b, kChD, sc, nullptr, H8_);
            }
            run_dcb(C, rh_frame_[i][0], b, kChD, TH8_, W8_, a, kChRecon, sc, nullptr, H8_);
            run_dcb(C, rh_frame_[i][1], a, kChRecon, TH8_, W8_, a, kChRecon, sc, nullptr, H8_);
            run_dcb(C, rh_frame_[i][2], a, kChRecon, TH8_, W8_, a, kChRecon, sc, nullptr, H8_);
            __half* out = (i == kFrames - 1) ? feature_i_ : head;
            gemm(C, rh_head_[i], kEpiBias, a, kChRecon, M8_, out, kChSrcIntra);
            if (all_frames) {
                C.note(launch_shuffle8_clamp(out, TH8_, W8_, 3, kChSrcIntra, x_hat_[i], C.s, act_));
            }
        }
    };
    if (!all_frames) {
        frames(L, kFrames - 1, kFrames, lvl8_a_, lvl8_b_, head_, scratch_);
        return;
    }
    const int nb = recon_branches_;
    if (nb <= 1) {
        frames(L, 0, kFrames, lvl8_a_, lvl8_b_, head_, scratch_);
        return;
    }
    // nb branches of kFrames / nb frames (a multiple of the 2 frames sharing a common block):
    // branch b > 0 on side_[b - 1], forked from and joined back into L.s (inside a graph capture
    // this makes parallel chains of the graph), branch 0 on L.s
    const int per = kFrames / nb;
    L.note(cudaEventRecord(ev_fork_, L.s), 0);
    for (int b = 1; b < nb; ++b) {
        L.note(cudaStreamWaitEvent(side_[b - 1], ev_fork_, 0), 0);
        Launch Lb{side_[b - 1], L.err_word};
        frames(Lb, b * per, (b + 1) * per, rb_a_[b], rb_b_[b], rb_head_[b], rb_scratch_[b]);
        Lb.note(cudaEventRecord(ev_join_[b - 1], side_[b - 1]), 0);
        L.note(Lb.first, 0);
        L.kernels += Lb.kernels;
    }
    frames(L, 0, per, lvl8_a_, lvl8_b_, head_, scratch_);
    for (int b = 1; b < nb; ++b) {
        L.note(cudaStreamWaitEvent(L.s, ev_join_[b - 1], 0), 0);
    }
}

// ------------------------------------------------------------------------------ phases

void HtsCodec::enc_analysis(Launch& L)
{
    const int H32 = H16p_ / 2, W32 = W16p_ / 2, H64 = H16p_ / 4, W64 = W16p_ / 4;
    // the temporal prior depends only on the memory of the last chunk: a side branch of the graph
    // (its own working buffers) computes it while the encoder and the hyper encoder run
    L.note(cudaEventRecord(ev_fork_, L.s), 0);
    L.note(cudaStreamWaitEvent(side_[0], ev_fork_, 0), 0);
    {
        Launch Lt{side_[0], L.err_word};
        temporal_prior(Lt, s2d_t_, lvl16_t_, scratch_t_);
        Lt.note(cudaEventRecord(ev_join_[0], side_[0]), 0);
        L.note(Lt.first, 0);
        L.kernels += Lt.kernels;
    }
    // encoder (dmc_hts_proxy.cpp:67-78)
    run_dcb(L, encoder_[0], cat_enc_, 2048, TH8_, W8_, lvl8_a_, kChD, scratch_, nullptr, H8_);
    for (int i = 1; i < 5; ++i) {
        run_dcb(L, encoder_[i], lvl8_a_, kChD, TH8_, W8_, lvl8_a_, kChD, scratch_, nullptr, H8_);
    }
    run_dcb(L, encoder_[5], lvl8_a_, kChD, TH8_, W8_, lvl8_a_, kChD, scratch_, q_enc_, H8_);
    for (int k = 0; k < imgs_; ++k) {  // each image's patches, zero outside its own border
        L.note(launch_im2col3x3s2(lvl8_a_ + static_cast<size_t>(k) * m8_ * kChD, H8_, W8_, kChD, kChD,
                                  col_ + static_cast<size_t>(k) * m16_ * 9 * kChD, L.s));
    }
    if (act_) {  // the BF16 form: y to FP16 for the entropy-parameter path
        gemm(L, enc_down_, kEpiBias, col_, 9 * kChD, M16_, y_act_, kChY);
        L.note(launch_convert(y_act_, 1, kChY, y_, 0, kChY, M16_, kChY, L.s));
    } else {
        gemm(L, enc_down_, kEpiBias, col_, 9 * kChD, M16_, y_, kChY);
    }
    if (y_pad_ != y_) {
        for (int k = 0; k < imgs_; ++k) {
            L.note(launch_replicate_pad(y_ + static_cast<size_t>(k) * m16_ * kChY, H16_, W16_, kChY,
                                        kChY, H16p_ - H16_, W16p_ - W16_,
                                        y_pad_ + static_cast<size_t>(k) * m16p_ * kChY, L.s));
        }
    }
    // hyper encoder
    run_dcb(L, hyper_enc0_, y_pad_, kChY, TH16p_, W16p_, lvl16_a_, kChY, scratch_, nullptr, H16p_);
    L.note(launch_space_to_depth2(lvl16_a_, TH16p_, W16p_, kChY, kChY, s2d_, L.s));
    gemm(L, hyper_enc1_.down, kEpiBias, s2d_, 4 * kChY, M32_, lvl32_a_, kChY);
    run_dcb(L, hyper_enc1_.dcb, lvl32_a_, kChY, TH32_, W32, lvl32_a_, kChY, scratch_, nullptr, H32);
    L.note(launch_space_to_depth2(lvl32_a_, TH32_, W32, kChY, kChY, s2d_, L.s));
    gemm(L, hyper_enc2_.down, kEpiBias, s2d_, 4 * kChY, M64_, lvl64_a_, kChZ);
    run_dcb(L, hyper_enc2_.dcb, lvl64_a_, kChZ, TH64_, W64, z_, kChZ, scratch_, nullptr, H64);
    L.note(launch_round_z(z_, z_num_, z_hat_, z_i8_, L.s));
    L.note(cudaStreamWaitEvent(L.s, ev_join_[0], 0), 0);  // the temporal prior branch
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
                                 skip_thr_half_, y_q_, kChY, cat_spa_, 2 * kChY, TH16_, W16_, kChY,
                                 L.s, 4, H16_));
    for (int k = 1; k < kMaskPhases; ++k) {
        spatial_prior(L, k - 1);
        L.note(launch_quantize_phase(k, k == kMaskPhases - 1 ? 2 : 1, y_, kChY, scales, ldc,
                                     means_, kChY, q_dec, ldc, skip_thr_half_, y_q_, kChY,
                                     cat_spa_, 2 * kChY, TH16_, W16_, kChY, L.s, 4, H16_));
    }
    L.note(launch_build_index_enc(y_q_, kChY, scales, ldc, skip_thr_half_, scale_lut_, M16_, kChY,
                                  sym_, cond_, L.s));
    // per image: the coded symbols compacted and copied with their count to the mapped host
    // buffers (each stream's symbols form its own payload)
    const int nb = compact_blocks(ny_);
    for (int k = 0; k < imgs_; ++k) {
        const size_t o = static_cast<size_t>(k) * ny_;
        L.note(launch_compact(sym_ + o, 2, cond_ + o, ny_, block_counts_ + static_cast<size_t>(k) * nb,
                              sym_c_ + o, count_dev_ + k, L.s), 2);
        L.note(launch_copy_counted(sym_c_ + o, sym_hdev_ + o, 2, count_dev_ + k, ny_, count_hdev_ + k,
                                   L.s));
    }
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
    temporal_prior(L, s2d_, lvl16_a_, scratch_);
}

void HtsCodec::dec_hyper(Launch& L)
{
    L.note(launch_int8_to_half(z_hdev_, z_num_, z_hat_, L.s));  // z as decoded on the host
    hyper_decoder(L);
    prior_fusion(L);
    L.note(launch_build_index_dec(common_ + kChY, 3 * kChY, skip_thr_half_, scale_lut_, M16_, kChY,
                                  idx_, cond_, L.s));
    const int nb = compact_blocks(ny_);
    for (int k = 0; k < imgs_; ++k) {
        const size_t o = static_cast<size_t>(k) * ny_;
        L.note(launch_compact(idx_ + o, 1, cond_ + o, ny_, block_counts_ + static_cast<size_t>(k) * nb,
                              idx_c_ + o, count_dev_ + k, L.s), 2);
        L.note(launch_copy_counted(idx_c_ + o, idx_hdev_ + o, 1, count_dev_ + k, ny_, count_hdev_ + k,
                                   L.s));
    }
}

void HtsCodec::dec_context(Launch& L) { feature_extractor(L); }

void HtsCodec::dec_synthesis(Launch& L)
{
    const __half* q_dec = common_;
    const __half* means0 = common_ + 2 * kChY;
    const int ldc = 3 * kChY;
    const int nb = compact_blocks(ny_);
    for (int k = 0; k < imgs_; ++k) {  // each stream's decoded values back into its latents
        const size_t o = static_cast<size_t>(k) * ny_;
        L.note(launch_copy_counted(ydec_hdev_ + o, y_dec_ + o, 1, count_dev_ + k, ny_, nullptr, L.s));
        L.note(launch_recover(y_dec_ + o, cond_ + o, block_counts_ + static_cast<size_t>(k) * nb, ny_,
                              y_q_ + o, L.s));
    }
    L.note(launch_restore_phase(0, 0, y_q_, kChY, means0, ldc, nullptr, 0, cat_spa_, 2 * kChY,
                                TH16_, W16_, kChY, L.s, 4, H16_));
    gemm(L, reduction_, kEpiBias, common_, ldc, M16_, cat_spa_ + kChY, 2 * kChY);
    for (int k = 1; k < kMaskPhases; ++k) {
        spatial_prior(L, k - 1);
        L.note(launch_restore_phase(k, k == kMaskPhases - 1 ? 2 : 1, y_q_, kChY, means_, kChY,
                                    q_dec, ldc, cat_spa_, 2 * kChY, TH16_, W16_, kChY, L.s, 4, H16_));
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
    static const char* const kNames[kPhaseSlots] = {"hts enc_analysis", "hts enc_update", "hts enc_update reset",
                                                    "hts dec_temporal", "hts dec_temporal memory", "hts dec_hyper",
                                                    "hts dec_context", "hts dec_synthesis"};
    NvtxRange range(kNames[slot]);
    if (timing_) {
        cudaEventRecord(tev_[slot][0], s);
    }
    const int st = graphs_.run(slot, s, err_word_, [&](Launch& L) { record_phase(slot, L); }, &last_kernels_);
    if (timing_) {
        cudaEventRecord(tev_[slot][1], s);
        tev_used_[slot] = true;
    }
    return st;
}

void HtsCodec::set_timing(bool on)
{
    cudaSetDevice(dev_);
    if (on && tev_[0][0] == nullptr) {
        for (auto& e : tev_) {
            cudaEventCreate(&e[0]);
            cudaEventCreate(&e[1]);
        }
    }
    timing_ = on && tev_[0][0] != nullptr;
}

int HtsCodec::timing(float* out, int cap)
{
    if (out == nullptr || cap <= 0) {
        return 0;
    }
    float v[kTimingValues];
    for (int i = 0; i < kPhaseSlots; ++i) {
        v[i] = -1.f;
        if (timing_ && tev_used_[i] && cudaEventSynchronize(tev_[i][1]) == cudaSuccess) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, tev_[i][0], tev_[i][1]) == cudaSuccess) {
                v[i] = ms;
            }
        }
    }
    cudaGetLastError();
    for (int i = 0; i < 5; ++i) {
        v[kPhaseSlots + i] = host_ms_[i];
    }
    const int n = cap < kTimingValues ? cap : kTimingValues;
    for (int i = 0; i < n; ++i) {
        out[i] = v[i];
    }
    return n;
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

// ------------------------------------------------------------------------------ sharing

int HtsCodec::share_params(const HtsCodec& o)
{
    if (&o == this) {
        return kOk;
    }
    if (!o.ready_) {
        set_last_error("share_params: the source codec has no parameters");
        return kNotReady;
    }
    if (o.dev_ != dev_) {
        set_last_error("share_params: the codecs live on different devices");
        return kInvalidArgument;
    }
    if (main_ != nullptr) {
        cudaStreamSynchronize(main_);
    }
    clear_graphs();
    if (Hp_ != 0 && (o.act_ != act_ || o.fp8_ != fp8_)) {
        // the arena's precision-form buffers differ: size it again on the next add_ref_feature
        acts_.clear();
        Hp_ = Wp_ = 0;
    }
    weights_ = o.weights_;
    precision_ = o.precision_;
    act_ = o.act_;
    fp8_ = o.fp8_;
    skip_threshold_ = o.skip_threshold_;
    skip_thr_half_ = o.skip_thr_half_;
    q_enc_tab_ = o.q_enc_tab_;
    q_dec_tab_ = o.q_dec_tab_;
    q_feat_tab_ = o.q_feat_tab_;
    scale_lut_ = o.scale_lut_;
    std::copy(std::begin(o.encoder_), std::end(o.encoder_), std::begin(encoder_));
    enc_down_ = o.enc_down_;
    hyper_enc0_ = o.hyper_enc0_;
    hyper_enc1_ = o.hyper_enc1_;
    hyper_enc2_ = o.hyper_enc2_;
    hyper_dec0_ = o.hyper_dec0_;
    hyper_dec1_ = o.hyper_dec1_;
    hyper_dec2_ = o.hyper_dec2_;
    temporal_ = o.temporal_;
    std::copy(std::begin(o.prior_fusion_), std::end(o.prior_fusion_), std::begin(prior_fusion_));
    prior_fusion_out_ = o.prior_fusion_out_;
    reduction_ = o.reduction_;
    std::copy(std::begin(o.sp_adaptor_), std::end(o.sp_adaptor_), std::begin(sp_adaptor_));
    std::copy(std::begin(o.spatial_prior_), std::end(o.spatial_prior_), std::begin(spatial_prior_));
    spatial_prior_out_ = o.spatial_prior_out_;
    dec_up_ = o.dec_up_;
    dec_up_lin_ = o.dec_up_lin_;
    std::copy(std::begin(o.decoder_), std::end(o.decoder_), std::begin(decoder_));
    std::copy(std::begin(o.fa_i_), std::end(o.fa_i_), std::begin(fa_i_));
    std::copy(std::begin(o.fa_m_), std::end(o.fa_m_), std::begin(fa_m_));
    std::copy(std::begin(o.fe_), std::end(o.fe_), std::begin(fe_));
    std::copy(std::begin(o.rh_common_), std::end(o.rh_common_), std::begin(rh_common_));
    for (int i = 0; i < kFrames; ++i) {
        std::copy(std::begin(o.rh_frame_[i]), std::end(o.rh_frame_[i]), std::begin(rh_frame_[i]));
    }
    std::copy(std::begin(o.rh_head_), std::end(o.rh_head_), std::begin(rh_head_));
    tables_ = o.tables_;
    ready_ = true;
    return kOk;
}

size_t HtsCodec::state_bytes() const
{
    if (Hp_ == 0) {
        return 0;
    }
    return static_cast<size_t>(M8_) * (1024 + kChD + kChSrcIntra) * 2;
}

int HtsCodec::export_state(void* dst, cudaStream_t caller, int* flags)
{
    if (Hp_ == 0 || dst == nullptr || flags == nullptr) {
        set_last_error("export_state: no resolution allocated yet, or a null argument");
        return Hp_ == 0 ? kNotReady : kInvalidArgument;
    }
    const size_t M8 = M8_;
    uint8_t* d = static_cast<uint8_t*>(dst);
    // the copies follow the codec's last call; the codec's next work follows the copies
    cudaEventRecord(ev_state_, main_);
    cudaStreamWaitEvent(caller, ev_state_, 0);
    cudaError_t e = cudaMemcpyAsync(d, cat_fam_, M8 * 1024 * 2, cudaMemcpyDeviceToDevice, caller);
    d += M8 * 1024 * 2;
    if (e == cudaSuccess) {
        e = cudaMemcpy2DAsync(d, kChD * 2, cat_enc_ + kChSrc, 2048 * 2, kChD * 2, M8,
                              cudaMemcpyDeviceToDevice, caller);
    }
    d += M8 * kChD * 2;
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(d, feature_i_, M8 * kChSrcIntra * 2, cudaMemcpyDeviceToDevice, caller);
    }
    cudaEventRecord(ev_state_, caller);
    cudaStreamWaitEvent(main_, ev_state_, 0);
    *flags = memory_has_value_ ? 1 : 0;
    return cuda_status(e, "export_state");
}

int HtsCodec::import_state(const void* src, int flags, cudaStream_t caller)
{
    if (Hp_ == 0 || src == nullptr) {
        set_last_error("import_state: no resolution allocated yet (add_ref_feature first), or a "
                       "null source");
        return Hp_ == 0 ? kNotReady : kInvalidArgument;
    }
    const size_t M8 = M8_;
    const uint8_t* s = static_cast<const uint8_t*>(src);
    cudaEventRecord(ev_state_, main_);
    cudaStreamWaitEvent(caller, ev_state_, 0);
    cudaError_t e = cudaMemcpyAsync(cat_fam_, s, M8 * 1024 * 2, cudaMemcpyDeviceToDevice, caller);
    s += M8 * 1024 * 2;
    if (e == cudaSuccess) {
        e = cudaMemcpy2DAsync(cat_enc_ + kChSrc, 2048 * 2, s, kChD * 2, kChD * 2, M8,
                              cudaMemcpyDeviceToDevice, caller);
    }
    s += M8 * kChD * 2;
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(feature_i_, s, M8 * kChSrcIntra * 2, cudaMemcpyDeviceToDevice, caller);
    }
    cudaEventRecord(ev_state_, caller);
    cudaStreamWaitEvent(main_, ev_state_, 0);
    memory_has_value_ = flags != 0;
    return cuda_status(e, "import_state");
}

// ------------------------------------------------------------------------------ public calls

int HtsCodec::add_ref_feature(const __half* frame, int Hp, int Wp, bool apply_adaptor,
                              cudaStream_t caller)
{
    return add_ref_features(&frame, 1, Hp, Wp, apply_adaptor, caller);
}

int HtsCodec::add_ref_features(const __half* const* frames, int n, int Hp, int Wp,
                               bool apply_adaptor, cudaStream_t caller)
{
    if (!ready_) {
        set_last_error("add_ref_feature_from_frame: set_param has not been called");
        return kNotReady;
    }
    if (frames == nullptr || n < 1) {
        set_last_error("add_ref_feature_from_frame: null frame");
        return kInvalidArgument;
    }
    for (int k = 0; k < n; ++k) {
        if (frames[k] == nullptr) {
            set_last_error("add_ref_feature_from_frame: null frame");
            return kInvalidArgument;
        }
    }
    int st = allocate(Hp, Wp, n);
    if (st != kOk) {
        return st;
    }
    last_kernels_ = 0;
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    Launch L{main_, err_word_};
    for (int k = 0; k < n; ++k) {
        L.note(launch_pad_unshuffle8(frames[k], Hp, Wp, 3, 3, 0, 0,
                                     feature_i_ + static_cast<size_t>(k) * m8_ * kChSrcIntra,
                                     kChSrcIntra, main_, act_));
    }
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

namespace {

// Runs fn(k) for k in [0, n): inline for one item, else on one thread per item (the items are
// independent rANS payloads of a packed batch).
template <typename F>
void for_each_stream(int n, F&& fn)
{
    if (n == 1) {
        fn(0);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(n);
    for (int k = 0; k < n; ++k) {
        th.emplace_back([&fn, k] { fn(k); });
    }
    for (auto& t : th) {
        t.join();
    }
}

}  // namespace

int HtsCodec::compress(const __half* x, int H, int W, int qp, bool reset, int pad_b, int pad_r,
                       cudaStream_t caller, std::vector<uint8_t>* bytes, int* ec_parallel)
{
    return compress_batch(&x, 1, H, W, &qp, reset, pad_b, pad_r, caller, bytes, ec_parallel);
}

int HtsCodec::compress_batch(const __half* const* xs, int n, int H, int W, const int* qps,
                             bool reset, int pad_b, int pad_r, cudaStream_t caller,
                             std::vector<uint8_t>* bytes, int* ec_parallel)
{
    if (!ready_ || Hp_ == 0) {
        set_last_error("compress: set_param and add_ref_feature_from_frame must come first");
        return kNotReady;
    }
    bool ok = xs != nullptr && qps != nullptr && bytes != nullptr && ec_parallel != nullptr &&
              n == imgs_ && pad_b >= 0 && pad_r >= 0 && H + pad_b == Hp_ && W + pad_r == Wp_;
    for (int k = 0; ok && k < n; ++k) {
        ok = xs[k] != nullptr && qps[k] >= 0 && qps[k] < kQpNum;
    }
    if (!ok) {
        set_last_error("compress: bad input pointer, qp, stream count or size (input + padding "
                       "must equal the reference frame size, one input per stream of the batch)");
        return kInvalidArgument;
    }
    last_kernels_ = 0;
    begin_timing();
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    set_qp(qps, main_);
    Launch L{main_, err_word_};
    for (int k = 0; k < n; ++k) {
        L.note(launch_pad_unshuffle8(xs[k], H, W, 24, 24, pad_b, pad_r,
                                     cat_enc_ + static_cast<size_t>(k) * m8_ * 2048, 2048, main_, act_));
    }
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
    const auto t_wait = Clock::now();
    if (cudaEventSynchronize(ev_phase_) != cudaSuccess) {
        return cuda_status(cudaGetLastError(), "compress: analysis");
    }
    const auto t_rans = Clock::now();
    host_ms_[0] = ms_between(t_wait, t_rans);
    NvtxRange range("hts rANS encode");
    st = check_device_error_word(err_word_, err_slot_, "compress");
    if (st != kOk) {
        return st;
    }
    for (int k = 0; k < n; ++k) {
        if (count_host_[k] < 0 || count_host_[k] > ny_) {
            set_last_error("compress: symbol count out of range");
            return kInternal;
        }
    }
    std::vector<std::string> errs(n);
    std::vector<char> good(n, 0);
    for_each_stream(n, [&](int k) {
        const int count = count_host_[k];
        const int ecp = ec_parallel_for(count);
        RansEncoderSession enc;
        enc.reset(ecp);
        enc.add_y(sym_host_ + static_cast<size_t>(k) * ny_, count, false);
        enc.add_z(z_host_ + static_cast<size_t>(k) * nz_, nz_, qps[k] * kChZ, kChZ, false);
        good[k] = enc.finish(tables_, &bytes[k], &errs[k]) ? 1 : 0;
        ec_parallel[k] = ecp;
    });
    host_ms_[1] = ms_between(t_rans, Clock::now());
    last_count_ = 0;
    for (int k = 0; k < n; ++k) {
        if (!good[k]) {
            set_last_error("compress: " + errs[k]);
            return kInternal;
        }
        last_count_ += count_host_[k];
    }
    return kOk;
}

int HtsCodec::decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                         bool reset, cudaStream_t caller, const __half** frames)
{
    return decompress_batch(&bytes, &n, &qp, &ecp, 1, height, width, reset, caller, frames);
}

int HtsCodec::decompress_batch(const uint8_t* const* bytes, const size_t* sizes, const int* qps,
                               const int* ecps, int n, int height, int width, bool reset,
                               cudaStream_t caller, const __half** frames)
{
    if (!ready_ || Hp_ == 0) {
        set_last_error("decompress: set_param and add_ref_feature_from_frame must come first");
        return kNotReady;
    }
    bool ok = bytes != nullptr && sizes != nullptr && qps != nullptr && ecps != nullptr &&
              frames != nullptr && n == imgs_ && height > 0 && width > 0 &&
              (height + 63) / 64 == H16p_ / 4 && (width + 63) / 64 == W16p_ / 4 &&
              ceil_to(height, 16) == Hp_ && ceil_to(width, 16) == Wp_;
    for (int k = 0; ok && k < n; ++k) {
        ok = qps[k] >= 0 && qps[k] < kQpNum && ecps[k] >= 1 && ecps[k] <= kMaxEcParallel &&
             sizes[k] <= 0x7fffffff && (sizes[k] == 0 || bytes[k] != nullptr);
    }
    if (!ok) {
        set_last_error("decompress: bad qp, ec_parallel, stream, stream count or picture size (the "
                       "size must match the reference frame)");
        return kInvalidArgument;
    }
    last_kernels_ = 0;
    begin_timing();
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    set_qp(qps, main_);
    int st = run_phase(kDecTemporal + (memory_has_value_ ? 1 : 0), main_);
    auto t0 = Clock::now();
    // z on the CPU while the temporal branch runs (dmc_hts_proxy.cpp:794-804)
    std::vector<RansDecoderSession> dec(n);
    std::vector<std::string> errs(n);
    std::vector<int> res(n, kOk);
    if (st == kOk) {
        NvtxRange range("hts rANS decode z");
        for_each_stream(n, [&](int k) {
            if (!dec[k].begin(bytes[k], static_cast<int>(sizes[k]), ecps[k], &errs[k]) ||
                !dec[k].decode_z(tables_, nz_, qps[k] * kChZ, kChZ,
                                 z_host_ + static_cast<size_t>(k) * nz_, &errs[k])) {
                res[k] = dec[k].fault() ? kInternal : kCorruptStream;
            }
        });
        for (int k = 0; k < n && st == kOk; ++k) {
            if (res[k] != kOk) {
                set_last_error("decompress: " + errs[k]);
                st = res[k];
            }
        }
    }
    host_ms_[2] = ms_between(t0, Clock::now());
    if (st == kOk) {
        st = run_phase(kDecHyper, main_);
    }
    if (st == kOk) st = cuda_status(cudaEventRecord(ev_phase_, main_), "decompress");
    if (st == kOk) st = run_phase(kDecContext, main_);
    t0 = Clock::now();
    if (st == kOk) {
        if (cudaEventSynchronize(ev_phase_) != cudaSuccess) {
            st = cuda_status(cudaGetLastError(), "decompress: hyper prior");
        }
    }
    host_ms_[3] = ms_between(t0, Clock::now());
    t0 = Clock::now();
    if (st == kOk) st = check_device_error_word(err_word_, err_slot_, "decompress");
    for (int k = 0; k < n && st == kOk; ++k) {
        if (count_host_[k] < 0 || count_host_[k] > ny_) {
            set_last_error("decompress: symbol count out of range");
            st = kInternal;
        }
    }
    // y on the CPU while the feature extractor runs (dmc_hts_proxy.cpp:805-823)
    if (st == kOk) {
        NvtxRange range("hts rANS decode y");
        for_each_stream(n, [&](int k) {
            const size_t o = static_cast<size_t>(k) * ny_;
            if (!dec[k].decode_y(tables_, idx_host_ + o, count_host_[k], ydec_host_ + o, &errs[k])) {
                res[k] = dec[k].fault() ? kInternal : kCorruptStream;
            }
        });
        for (int k = 0; k < n && st == kOk; ++k) {
            if (res[k] != kOk) {
                set_last_error("decompress: " + errs[k]);
                st = res[k];
            }
        }
    }
    host_ms_[4] = ms_between(t0, Clock::now());
    if (st == kOk) {
        st = run_phase(kDecSynthesis, main_);
    }
    if (st == kOk) {
        memory_has_value_ = !reset;
        for (int i = 0; i < kFrames; ++i) {
            frames[i] = x_hat_[i];
        }
        last_count_ = 0;
        for (int k = 0; k < n; ++k) {
            last_count_ += count_host_[k];
        }
    }
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    return st;
}

}  // namespace dcvc
