#include "intra_codec.h"

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

IntraCodec::IntraCodec()
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

IntraCodec::~IntraCodec()
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

int IntraCodec::set_param(const StateDict& sd, float skip_threshold)
{
    if (main_ != nullptr) {
        cudaStreamSynchronize(main_);
    }
    graphs_.clear();
    ready_ = false;
    weights_.clear();
    ParamBuilder B(sd, weights_);
    int r[4] = {0}, c[4] = {0};
    q_enc_tab_ = B.half_rows("q_scale_enc", &r[0], &c[0]);
    q_dec_tab_ = B.half_rows("q_scale_dec", &r[1], &c[1]);
    q_y_enc_tab_ = B.half_rows("q_scale_y_enc", &r[2], &c[2]);
    q_y_dec_tab_ = B.half_rows("q_scale_y_dec", &r[3], &c[3]);
    // DMCI module layout (image_model.py:21-147); the resampling blocks keep the default
    // shortcut (DMCIHyperDecoderProxy / DMCIHyperEncoderProxy::set_param, dmci_proxy.cpp:166-199,
    // DMCIDecoderProxy::set_param :74-90)
    enc1_ = B.dcb("enc.enc_1.");
    for (int i = 0; i < 6; ++i) {
        enc2_[i] = B.dcb(num("enc.enc_2.", i));
    }
    enc_down_ = B.conv3x3s2("enc.enc_2.6.");
    hyper_enc0_ = B.dcb("hyper_enc.conv.0.");
    hyper_enc1_ = B.down("hyper_enc.conv.1.", true);
    hyper_enc2_ = B.down("hyper_enc.conv.2.", true);
    hyper_dec0_ = B.up("hyper_dec.conv.0.", true);
    hyper_dec1_ = B.up("hyper_dec.conv.1.", true);
    hyper_dec2_ = B.dcb("hyper_dec.conv.2.");
    for (int i = 0; i < 3; ++i) {
        prior_fusion_[i] = B.dcb(num("y_prior_fusion.conv.", i));
        sp_adaptor_[i] = B.dcb(num("y_spatial_prior_adaptor_", i + 1));
        spatial_prior_[i] = B.dcb(num("y_spatial_prior.conv.", i));
    }
    prior_fusion_out_ = B.lin("y_prior_fusion.conv.3.");
    reduction_ = B.lin("y_spatial_prior_reduction.");
    spatial_prior_out_ = B.lin("y_spatial_prior.conv.3.");
    dec_up_ = B.up("dec.dec_1.0.", true);
    for (int i = 0; i < 12; ++i) {
        dec1_[i] = B.dcb(num("dec.dec_1.", i + 1));
    }
    dec2_ = B.dcb("dec.dec_2.");
    if (!B.ok()) {
        set_last_error("set_param: " + B.error());
        weights_.clear();
        return kInvalidArgument;
    }
    const bool shapes_ok =
        r[0] == kQpNum && c[0] == kChEnc && r[1] == kQpNum && c[1] == kChEnc && r[2] == kQpNum &&
        c[2] == kChY && r[3] == kQpNum && c[3] == kChY && enc1_.cin == kChSrc &&
        enc1_.C == kChEnc && enc2_[0].C == kChEnc && enc_down_.cin == 9 * kChEnc &&
        enc_down_.cout == kChY && hyper_enc0_.cin == kChY && hyper_enc0_.C == kChZ &&
        hyper_enc1_.down.cin == 4 * kChZ && hyper_enc2_.down.cout == kChZ &&
        hyper_dec0_.up.cin == kChZ && hyper_dec0_.up.cout == 4 * kChZ &&
        hyper_dec1_.up.cout == 4 * kChZ && hyper_dec2_.cin == kChZ && hyper_dec2_.C == kChY &&
        prior_fusion_[0].cin == kChY && prior_fusion_[0].C == 2 * kChY &&
        prior_fusion_out_.cout == 2 * kChY && reduction_.cin == 2 * kChY &&
        reduction_.cout == kChY && sp_adaptor_[0].C == 2 * kChY &&
        spatial_prior_out_.cout == 2 * kChY && dec_up_.up.cin == kChY &&
        dec_up_.up.cout == 4 * kChEnc && dec1_[0].C == kChEnc && dec2_.cin == kChEnc &&
        dec2_.C == kChSrc;
    if (!shapes_ok) {
        set_last_error("set_param: state dict is not an intra (DMCI) model");
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

int IntraCodec::allocate(int Hp, int Wp)
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

    // pre_allocate_tensors (dmci_proxy.cpp:701-802)
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
    unshuf_ = H(M8 * kChSrc);
    lvl8_a_ = H(M8 * kChEnc);
    lvl8_b_ = H(M8 * kChEnc);
    head_ = H(M8 * kChSrc);
    col_ = H(M16 * 9 * kChEnc);
    y_ = H(M16 * kChY);
    y_pad_ = pad ? H(M16p * kChY) : y_;
    y_s_ = H(M16 * kChY);
    y_q_ = H(M16 * kChY);
    lvl16_a_ = H(M16p * 2 * kChY);
    lvl16_b_ = H(M16p * 2 * kChY);
    params_ = H(M16 * 2 * kChY);
    params_pad_ = pad ? H(M16p * 2 * kChY) : params_;
    cat_sp_ = H(M16 * 2 * kChY);
    sp_out_ = H(M16 * 2 * kChY);
    part_ = H(M16 * (kChY / 4));
    lvl32_a_ = H(M32 * kChZ);
    lvl32_b_ = H(M32 * kChZ);
    lvl64_a_ = H(M64 * kChZ);
    s2d_ = H(std::max(M32, M64) * 4 * kChZ);
    z_ = H(M64 * kChZ);
    z_hat_ = H(M64 * kChZ);
    x_hat_ = H(static_cast<size_t>(Hp) * Wp * 3);
    q_enc_ = H(kChEnc);
    q_dec_ = H(kChEnc);
    q_y_enc_ = H(kChY);
    q_y_dec_ = H(kChY);
    const size_t S = std::max({M8 * kChEnc, M16p * 2 * kChY, M32 * 4 * kChZ});
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
    cudaMemsetAsync(cat_sp_, 0, M16 * 2 * kChY * 2, main_);
    if (cudaStreamSynchronize(main_) != cudaSuccess) {
        return cuda_status(cudaGetLastError(), "allocate");
    }
    Hp_ = Hp;
    Wp_ = Wp;
    return kOk;
}

void IntraCodec::set_qp(int qp, cudaStream_t s)
{
    cudaMemcpyAsync(q_enc_, q_enc_tab_ + static_cast<size_t>(qp) * kChEnc, kChEnc * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_dec_, q_dec_tab_ + static_cast<size_t>(qp) * kChEnc, kChEnc * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_y_enc_, q_y_enc_tab_ + static_cast<size_t>(qp) * kChY, kChY * 2,
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q_y_dec_, q_y_dec_tab_ + static_cast<size_t>(qp) * kChY, kChY * 2,
                    cudaMemcpyDeviceToDevice, s);
}

// ------------------------------------------------------------------------------ network pieces

void IntraCodec::hyper_prior(Launch& L)
{
    // hyper decoder -> prior fusion (at the 4-aligned size) -> crop -> reduction
    // (lambda_enc_0 / lambda_dec_0, dmci_proxy.cpp:314-332, 463-473)
    const int H32 = H16p_ / 2, W32 = W16p_ / 2, W64 = W16p_ / 4;
    const int C2 = 2 * kChY;
    gemm(L, hyper_dec0_.up, kEpiSubpel, z_hat_, kChZ, M64_, lvl32_a_, kChZ, nullptr, 0, nullptr, W64);
    run_dcb(L, hyper_dec0_.dcb, lvl32_a_, kChZ, H32, W32, lvl32_b_, kChZ, scratch_);
    gemm(L, hyper_dec1_.up, kEpiSubpel, lvl32_b_, kChZ, M32_, lvl16_a_, kChZ, nullptr, 0, nullptr, W32);
    run_dcb(L, hyper_dec1_.dcb, lvl16_a_, kChZ, H16p_, W16p_, lvl16_b_, kChZ, scratch_);
    run_dcb(L, hyper_dec2_, lvl16_b_, kChZ, H16p_, W16p_, lvl16_a_, kChY, scratch_);
    run_dcb(L, prior_fusion_[0], lvl16_a_, kChY, H16p_, W16p_, lvl16_b_, C2, scratch_);
    run_dcb(L, prior_fusion_[1], lvl16_b_, C2, H16p_, W16p_, lvl16_b_, C2, scratch_);
    run_dcb(L, prior_fusion_[2], lvl16_b_, C2, H16p_, W16p_, lvl16_b_, C2, scratch_);
    gemm(L, prior_fusion_out_, kEpiBias, lvl16_b_, C2, M16p_, params_pad_, C2);
    if (params_pad_ != params_) {
        L.note(launch_crop(params_pad_, W16p_, C2, H16_, W16_, C2, params_, C2, L.s));
    }
    gemm(L, reduction_, kEpiBias, params_, C2, M16_, cat_sp_ + kChY, C2);
}

void IntraCodec::spatial_prior(Launch& L, int k)
{
    // adaptor_k(cat(y_hat so far, reduced)) -> spatial prior -> [scales | means]
    const int C2 = 2 * kChY;
    run_dcb(L, sp_adaptor_[k - 1], cat_sp_, C2, H16_, W16_, lvl16_a_, C2, scratch_);
    for (int i = 0; i < 3; ++i) {
        run_dcb(L, spatial_prior_[i], lvl16_a_, C2, H16_, W16_, lvl16_a_, C2, scratch_);
    }
    gemm(L, spatial_prior_out_, kEpiBias, lvl16_a_, C2, M16_, sp_out_, C2);
}

void IntraCodec::decoder(Launch& L)
{
    // DMCIDecoderProxy::forward (dmci_proxy.cpp:14-33): y_hat lives in cat_sp_[:, 0:256]
    gemm(L, dec_up_.up, kEpiSubpel, cat_sp_, 2 * kChY, M16_, lvl8_a_, kChEnc, nullptr, 0, nullptr,
         W16_);
    run_dcb(L, dec_up_.dcb, lvl8_a_, kChEnc, H8_, W8_, lvl8_b_, kChEnc, scratch_);
    for (int i = 0; i < 11; ++i) {
        run_dcb(L, dec1_[i], lvl8_b_, kChEnc, H8_, W8_, lvl8_b_, kChEnc, scratch_);
    }
    run_dcb(L, dec1_[11], lvl8_b_, kChEnc, H8_, W8_, lvl8_b_, kChEnc, scratch_, q_dec_);
    run_dcb(L, dec2_, lvl8_b_, kChEnc, H8_, W8_, head_, kChSrc, scratch_);
    L.note(launch_shuffle8_clamp(head_, H8_, W8_, 3, kChSrc, x_hat_, L.s));
}

void IntraCodec::compact_step(Launch& L, int k, bool enc)
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

void IntraCodec::enc_analysis(Launch& L)
{
    const int H32 = H16p_ / 2, W32 = W16p_ / 2, H64 = H16p_ / 4, W64 = W16p_ / 4;
    const int C2 = 2 * kChY;
    // DMCIEncoderProxy::forward (dmci_proxy.cpp:92-105): enc_1 then x q_scale_enc
    run_dcb(L, enc1_, unshuf_, kChSrc, H8_, W8_, lvl8_a_, kChEnc, scratch_, q_enc_);
    for (int i = 0; i < 6; ++i) {
        run_dcb(L, enc2_[i], lvl8_a_, kChEnc, H8_, W8_, lvl8_a_, kChEnc, scratch_);
    }
    L.note(launch_im2col3x3s2(lvl8_a_, H8_, W8_, kChEnc, kChEnc, col_, L.s));
    gemm(L, enc_down_, kEpiBias, col_, 9 * kChEnc, M16_, y_, kChY);
    if (y_pad_ != y_) {
        L.note(launch_replicate_pad(y_, H16_, W16_, kChY, kChY, H16p_ - H16_, W16p_ - W16_, y_pad_,
                                    L.s));
    }
    // hyper encoder -> z_hat
    run_dcb(L, hyper_enc0_, y_pad_, kChY, H16p_, W16p_, lvl16_a_, kChZ, scratch_);
    L.note(launch_space_to_depth2(lvl16_a_, H16p_, W16p_, kChZ, kChZ, s2d_, L.s));
    gemm(L, hyper_enc1_.down, kEpiBias, s2d_, 4 * kChZ, M32_, lvl32_a_, kChZ);
    run_dcb(L, hyper_enc1_.dcb, lvl32_a_, kChZ, H32, W32, lvl32_b_, kChZ, scratch_);
    L.note(launch_space_to_depth2(lvl32_b_, H32, W32, kChZ, kChZ, s2d_, L.s));
    gemm(L, hyper_enc2_.down, kEpiBias, s2d_, 4 * kChZ, M64_, lvl64_a_, kChZ);
    run_dcb(L, hyper_enc2_.dcb, lvl64_a_, kChZ, H64, W64, z_, kChZ, scratch_);
    L.note(launch_round_z(z_, z_num_, z_hat_, z_i8_, L.s));
    hyper_prior(L);
    // y * q_scale_y_enc, then the four checkerboard steps (dmci_proxy.cpp:326-396)
    L.note(launch_mul_channel(y_, M16_, kChY, kChY, q_y_enc_, y_s_, kChY, L.s));
    for (int k = 0; k < kSteps; ++k) {
        const __half* prm = params_;
        if (k > 0) {
            spatial_prior(L, k);
            prm = sp_out_;
        }
        const int mode = k == 0 ? 0 : (k == kSteps - 1 ? 3 : 1);
        L.note(launch_quantize_phase(k, mode, y_s_, kChY, prm, C2, prm + kChY, C2, q_y_dec_, 0,
                                     skip_thr_half_, y_q_, kChY, cat_sp_, C2, H16_, W16_, kChY,
                                     L.s));
        L.note(launch_build_index_enc_4x(k, y_q_, kChY, prm, C2, skip_thr_half_, scale_lut_, H16_,
                                         W16_, kChY, sym_, cond_, L.s));
        compact_step(L, k, true);
    }
    L.note(cudaMemcpyAsync(count_host_, count_dev_, sizeof(int) * kSteps, cudaMemcpyDeviceToHost,
                           L.s),
           0);
}

void IntraCodec::dec_hyper(Launch& L)
{
    L.note(launch_int8_to_half(z_i8_, z_num_, z_hat_, L.s));
    hyper_prior(L);
    L.note(launch_build_index_dec_4x(0, params_, 2 * kChY, skip_thr_half_, scale_lut_, H16_, W16_,
                                     kChY, idx_, cond_, L.s));
    compact_step(L, 0, false);
    L.note(cudaMemcpyAsync(count_host_, count_dev_, sizeof(int), cudaMemcpyDeviceToHost, L.s), 0);
}

void IntraCodec::dec_step(Launch& L, int k)
{
    const int C2 = 2 * kChY;
    const __half* means_prev = (k == 1 ? params_ : sp_out_) + kChY;
    L.note(launch_recover(y_dec_, cond_, block_counts_, part_num_, part_, L.s));
    L.note(launch_restore_4x(k - 1, k == 1 ? 0 : 1, part_, means_prev, C2, nullptr, 0, cat_sp_,
                             C2, H16_, W16_, kChY, L.s));
    spatial_prior(L, k);
    L.note(launch_build_index_dec_4x(k, sp_out_, C2, skip_thr_half_, scale_lut_, H16_, W16_, kChY,
                                     idx_, cond_, L.s));
    compact_step(L, k, false);
    L.note(cudaMemcpyAsync(count_host_, count_dev_, sizeof(int), cudaMemcpyDeviceToHost, L.s), 0);
}

void IntraCodec::dec_final(Launch& L)
{
    const int C2 = 2 * kChY;
    L.note(launch_recover(y_dec_, cond_, block_counts_, part_num_, part_, L.s));
    L.note(launch_restore_4x(kSteps - 1, 3, part_, sp_out_ + kChY, C2, q_y_dec_, 0, cat_sp_, C2,
                             H16_, W16_, kChY, L.s));
    decoder(L);
}

void IntraCodec::record_phase(int slot, Launch& L)
{
    switch (slot) {
    case kEncAnalysis: enc_analysis(L); break;
    case kEncSynthesis: decoder(L); break;
    case kDecHyper: dec_hyper(L); break;
    case kDecStep:
    case kDecStep + 1:
    case kDecStep + 2: dec_step(L, slot - kDecStep + 1); break;
    case kDecFinal: dec_final(L); break;
    default: break;
    }
}

int IntraCodec::run_phase(int slot, cudaStream_t s)
{
    return graphs_.run(slot, s, err_word_, [&](Launch& L) { record_phase(slot, L); },
                       &last_kernels_);
}

int IntraCodec::buffer(const std::string& name, const void** ptr, int* rows, int* cols,
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
        {"y_hat", cat_sp_, M16_, kChY, 2 * kChY},
        {"y_q", y_q_, M16_, kChY, kChY},
        {"params", params_, M16_, 2 * kChY, 2 * kChY},
        {"z_hat", z_hat_, M64_, kChZ, kChZ},
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

int IntraCodec::compress(const __half* x, int H, int W, int qp, int pad_b, int pad_r,
                         cudaStream_t caller, std::vector<uint8_t>* bytes, int* ec_parallel,
                         const __half** x_hat)
{
    if (!ready_) {
        set_last_error("compress: set_param has not been called");
        return kNotReady;
    }
    if (x == nullptr || qp < 0 || qp >= kQpNum || H <= 0 || W <= 0 || pad_b < 0 || pad_r < 0 ||
        (H + pad_b) % 16 || (W + pad_r) % 16) {
        set_last_error("compress: bad input pointer, qp, size or padding (the padded size must "
                       "be a multiple of 16)");
        return kInvalidArgument;
    }
    int st = allocate(H + pad_b, W + pad_r);
    if (st != kOk) {
        return st;
    }
    last_kernels_ = 0;
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    set_qp(qp, main_);
    // the input pointer is not part of the graphs (dmci_proxy.cpp:303-305)
    Launch L{main_, err_word_};
    L.note(launch_pad_unshuffle8(x, H, W, 3, 3, pad_b, pad_r, unshuf_, kChSrc, main_));
    last_kernels_ += L.kernels;
    st = cuda_status(L.first, "compress: pad_and_unshuffle_8");
    if (st == kOk) st = run_phase(kEncAnalysis, main_);
    if (st == kOk) st = cuda_status(cudaEventRecord(ev_phase_, main_), "compress");
    if (st == kOk) st = run_phase(kEncSynthesis, main_);
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    if (st != kOk) {
        return st;
    }
    // the four steps' symbols and z to the host while the decoder runs (worker,
    // dmci_proxy.cpp:818-846)
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
    cudaStreamWaitEvent(copy_, ev_phase_, 0);
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
    *x_hat = x_hat_;
    last_count_ = total;
    return kOk;
}

int IntraCodec::decompress(const uint8_t* bytes, size_t n, int qp, int height, int width, int ecp,
                           cudaStream_t caller, const __half** x_hat)
{
    if (!ready_) {
        set_last_error("decompress: set_param has not been called");
        return kNotReady;
    }
    if (qp < 0 || qp >= kQpNum || ecp < 1 || ecp > kMaxEcParallel || n > 0x7fffffff ||
        (n > 0 && bytes == nullptr) || height <= 0 || width <= 0) {
        set_last_error("decompress: bad qp, ec_parallel, stream or picture size");
        return kInvalidArgument;
    }
    int st = allocate(ceil_to(height, 16), ceil_to(width, 16));
    if (st != kOk) {
        return st;
    }
    last_kernels_ = 0;
    cudaEventRecord(ev_in_, caller);
    cudaStreamWaitEvent(main_, ev_in_, 0);
    cudaStreamWaitEvent(copy_, ev_in_, 0);
    set_qp(qp, main_);
    // z first (worker DecodeZ, dmci_proxy.cpp:846-857)
    RansDecoderSession dec;
    std::string err;
    if (!dec.begin(bytes, static_cast<int>(n), ecp, &err) ||
        !dec.decode_z(tables_, z_num_, qp * kChZ, kChZ, z_host_, &err)) {
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
    // one CPU round trip per step (worker DecodeY, dmci_proxy.cpp:857-870)
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
        *x_hat = x_hat_;
        last_count_ = total;
    }
    cudaEventRecord(ev_out_, main_);
    cudaStreamWaitEvent(caller, ev_out_, 0);
    return st;
}

}  // namespace dcvc
