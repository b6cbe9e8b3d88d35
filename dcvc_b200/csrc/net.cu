#include "net.h"

#include <cuda_fp8.h>

#include <cmath>

#include "elementwise.cuh"
#include "ffn_sm100.cuh"
#include "gemm_sm100.cuh"

namespace dcvc {

cudaError_t gemm_sm100(int dtype, const void* A, int lda, const void* W, const GemmParams& p,
                       int epi, int bn, cudaStream_t stream);
int gemm_bn_for(int dtype, int epi, const GemmParams& p, cudaStream_t stream);

// ------------------------------------------------------------------------------ arena

void* DeviceArena::alloc(size_t bytes)
{
    void* p = nullptr;
    const size_t b = (bytes + 255) & ~size_t(255);
    if (cudaMalloc(&p, b == 0 ? 256 : b) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    blocks_.push_back(p);
    bytes_ += b;
    return p;
}

void DeviceArena::clear()
{
    for (void* p : blocks_) {
        cudaFree(p);
    }
    blocks_.clear();
    bytes_ = 0;
}

// ------------------------------------------------------------------------------ parameters

const HostTensor* ParamBuilder::get(const std::string& name, size_t ndim_min)
{
    auto it = sd_.find(name);
    if (it == sd_.end()) {
        fail("missing state-dict entry '" + name + "'");
        return nullptr;
    }
    if (it->second.shape.size() < ndim_min) {
        fail("state-dict entry '" + name + "' has too few dimensions");
        return nullptr;
    }
    return &it->second;
}

const __half* ParamBuilder::upload_half(const std::vector<float>& v)
{
    std::vector<__half> h(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        h[i] = __float2half_rn(v[i]);
    }
    __half* d = arena_.alloc_n<__half>(v.size());
    if (d == nullptr || cudaMemcpy(d, h.data(), h.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess) {
        fail("device allocation/copy of parameters failed");
        return nullptr;
    }
    return d;
}

const __half* ParamBuilder::upload_act(const std::vector<float>& v, int dtype)
{
    if (dtype == 0) {
        return upload_half(v);
    }
    std::vector<__nv_bfloat16> h(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        h[i] = __float2bfloat16_rn(v[i]);
    }
    __nv_bfloat16* d = arena_.alloc_n<__nv_bfloat16>(v.size());
    if (d == nullptr || cudaMemcpy(d, h.data(), h.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess) {
        fail("device allocation/copy of parameters failed");
        return nullptr;
    }
    return reinterpret_cast<const __half*>(d);
}

const __half* ParamBuilder::bf16_rows(const std::string& name, int* rows, int* cols)
{
    const HostTensor* t = get(name, 2);
    if (t == nullptr) {
        return nullptr;
    }
    *rows = static_cast<int>(t->shape[0]);
    *cols = static_cast<int>(t->numel() / t->shape[0]);
    return upload_act(t->data, 1);
}

const float* ParamBuilder::upload_float(const std::vector<float>& v)
{
    float* d = arena_.alloc_n<float>(v.size());
    if (d == nullptr || cudaMemcpy(d, v.data(), v.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        fail("device allocation/copy of parameters failed");
        return nullptr;
    }
    return d;
}

const __half* ParamBuilder::half_rows(const std::string& name, int* rows, int* cols)
{
    const HostTensor* t = get(name, 2);
    if (t == nullptr) {
        return nullptr;
    }
    *rows = static_cast<int>(t->shape[0]);
    *cols = static_cast<int>(t->numel() / t->shape[0]);
    return upload_half(t->data);
}

Lin ParamBuilder::lin(const std::string& prefix, bool bias)
{
    Lin l;
    const HostTensor* w = get(prefix + "weight", 2);
    if (w == nullptr) {
        return l;
    }
    l.cout = static_cast<int>(w->shape[0]);
    l.cin = static_cast<int>(w->numel() / w->shape[0]);
    if (w->numel() != static_cast<int64_t>(l.cout) * l.cin ||
        (w->shape.size() == 4 && (w->shape[2] != 1 || w->shape[3] != 1))) {
        fail("'" + prefix + "weight' is not a 1x1 convolution");
        return l;
    }
    l.dtype = dtype_;
    l.w = upload_act(w->data, dtype_);
    if (bias) {
        const HostTensor* b = get(prefix + "bias");
        if (b != nullptr) {
            l.b = upload_float(b->data);
        }
    }
    return l;
}

Dcb ParamBuilder::dcb(const std::string& p, bool shortcut)
{
    Dcb d;
    d.shortcut = shortcut;
    d.dtype = dtype_;
    if (has(p + "adaptor.weight")) {
        d.adaptor = true;
        d.ad = lin(p + "adaptor.");
    }
    d.dc1 = lin(p + "dc.0.");
    const HostTensor* dw = get(p + "dc.2.weight", 4);
    const HostTensor* dwb = get(p + "dc.2.bias");
    const HostTensor* w3 = get(p + "dc.3.weight", 2);
    const HostTensor* b3 = get(p + "dc.3.bias");
    if (dw == nullptr || dwb == nullptr || w3 == nullptr || b3 == nullptr) {
        return d;
    }
    d.cdc = static_cast<int>(dw->shape[0]);
    d.C = static_cast<int>(w3->shape[0]);
    if (dw->shape[1] != 1 || dw->shape[2] != 3 || dw->shape[3] != 3) {
        fail("'" + p + "dc.2.weight' is not a depthwise 3x3");
        return d;
    }
    // depthwise weight [c, 1, 3, 3] -> tap-major [9][c]
    std::vector<float> dwt(9 * static_cast<size_t>(d.cdc));
    for (int c = 0; c < d.cdc; ++c) {
        for (int k = 0; k < 9; ++k) {
            dwt[static_cast<size_t>(k) * d.cdc + c] = dw->data[static_cast<size_t>(c) * 9 + k];
        }
    }
    d.dw = upload_float(dwt);
    // dc.3 bias with the depthwise bias folded in: b3 + W3 . b2 (layers_proxy.cpp:175-178)
    std::vector<float> fb(d.C);
    for (int o = 0; o < d.C; ++o) {
        double s = b3->data[o];
        for (int c = 0; c < d.cdc; ++c) {
            s += static_cast<double>(w3->data[static_cast<size_t>(o) * d.cdc + c]) * dwb->data[c];
        }
        fb[o] = static_cast<float>(s);
    }
    d.dc2.cin = d.cdc;
    d.dc2.cout = d.C;
    d.dc2.dtype = dtype_;
    d.dc2.w = upload_act(w3->data, dtype_);
    d.dc2.b = upload_float(fb);
    d.ffn1 = lin(p + "ffn.0.");
    if (fp8_ && ok()) {
        // E4M3 rows with per-row scales max|w| / 448 (the FP8 form's quad GEMM)
        const HostTensor* w1 = get(p + "ffn.0.weight", 2);
        if (w1 != nullptr) {
            const int rows = static_cast<int>(w1->shape[0]);
            const int cols = static_cast<int>(w1->numel() / rows);
            std::vector<uint8_t> q(w1->data.size());
            std::vector<float> ws(rows);
            for (int r = 0; r < rows; ++r) {
                float mx = 0.f;
                for (int c = 0; c < cols; ++c) {
                    mx = std::max(mx, std::fabs(w1->data[static_cast<size_t>(r) * cols + c]));
                }
                const float sc = mx > 0.f ? mx / 448.f : 1.f;
                for (int c = 0; c < cols; ++c) {
                    q[static_cast<size_t>(r) * cols + c] = static_cast<uint8_t>(__nv_cvt_float_to_fp8(
                        w1->data[static_cast<size_t>(r) * cols + c] / sc, __NV_SATFINITE, __NV_E4M3));
                }
                ws[r] = sc * kFp8ActScale;
            }
            uint8_t* dq = arena_.alloc_n<uint8_t>(q.size());
            if (dq == nullptr || cudaMemcpy(dq, q.data(), q.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
                fail("device allocation/copy of parameters failed");
            }
            d.ffn1_w8 = dq;
            d.ffn1_ws = upload_float(ws);
        }
    }
    d.ffn2 = lin(p + "ffn.2.");
    d.cffn = d.ffn2.cin;
    d.cin = d.adaptor ? d.ad.cin : d.C;
    if (ok() && (d.dc1.cin != d.C || d.dc1.cout != d.cdc || d.ffn1.cout != 4 * d.cffn ||
                 d.ffn1.cin != d.C || d.ffn2.cout != d.C || (d.adaptor && d.ad.cout != d.C))) {
        fail("inconsistent DepthConvBlock shapes under '" + p + "'");
    }
    return d;
}

DownBlock ParamBuilder::down(const std::string& p, bool shortcut)
{
    DownBlock b;
    const HostTensor* w = get(p + "down.weight", 2);
    const HostTensor* bias = get(p + "down.bias");
    if (w == nullptr || bias == nullptr) {
        return b;
    }
    const int cout = static_cast<int>(w->shape[0]);
    const int k4 = static_cast<int>(w->numel() / cout);
    const int cin = k4 / 4;
    // K index c*4 + dy*2 + dx (pixel_unshuffle order) -> (dy*2 + dx)*cin + c
    std::vector<float> pw(static_cast<size_t>(cout) * k4);
    for (int o = 0; o < cout; ++o) {
        for (int c = 0; c < cin; ++c) {
            for (int s = 0; s < 4; ++s) {
                pw[static_cast<size_t>(o) * k4 + s * cin + c] =
                    w->data[static_cast<size_t>(o) * k4 + c * 4 + s];
            }
        }
    }
    b.down.cin = k4;
    b.down.cout = cout;
    b.down.dtype = dtype_;
    b.down.w = upload_act(pw, dtype_);
    b.down.b = upload_float(bias->data);
    b.dcb = dcb(p + "conv.", shortcut);
    return b;
}

UpBlock ParamBuilder::up(const std::string& p, bool shortcut)
{
    UpBlock b;
    b.up = subpel(p + "up.");
    b.dcb = dcb(p + "conv.", shortcut);
    return b;
}

Lin ParamBuilder::subpel(const std::string& p)
{
    Lin b;
    const HostTensor* w = get(p + "conv.0.weight", 2);
    if (w == nullptr) {
        return b;
    }
    const int n4 = static_cast<int>(w->shape[0]);
    const int kin = static_cast<int>(w->numel() / n4);  // cin (1x1) or 9 * cin (3x3)
    const int cout = n4 / 4;
    const bool k3 = w->shape.size() == 4 && w->shape[2] == 3 && w->shape[3] == 3;
    if (w->shape.size() == 4 && !k3 && (w->shape[2] != 1 || w->shape[3] != 1)) {
        fail("'" + p + "conv.0.weight' is neither 1x1 nor 3x3");
        return b;
    }
    const int cin = k3 ? kin / 9 : kin;
    // row c*4 + dy*2 + dx (pixel_shuffle order) -> (dy*2 + dx)*cout + c; a 3x3 kernel's K axis
    // [c][ky][kx] -> (ky*3 + kx)*cin + c to match the stride-1 patches
    std::vector<float> pw(static_cast<size_t>(n4) * kin);
    for (int c = 0; c < cout; ++c) {
        for (int s4 = 0; s4 < 4; ++s4) {
            const float* src = w->data.data() + static_cast<size_t>(c * 4 + s4) * kin;
            float* dst = pw.data() + static_cast<size_t>(s4 * cout + c) * kin;
            if (!k3) {
                std::copy(src, src + kin, dst);
            } else {
                for (int ci = 0; ci < cin; ++ci) {
                    for (int t = 0; t < 9; ++t) {
                        dst[t * cin + ci] = src[ci * 9 + t];
                    }
                }
            }
        }
    }
    b.cin = kin;
    b.cout = n4;
    b.dtype = dtype_;
    b.w = upload_act(pw, dtype_);
    if (has(p + "conv.0.bias")) {
        const HostTensor* bias = get(p + "conv.0.bias");
        if (bias == nullptr || bias->numel() != n4) {
            fail("'" + p + "conv.0.bias' does not match its weight");
            return b;
        }
        std::vector<float> pb(n4);
        for (int c = 0; c < cout; ++c) {
            for (int s4 = 0; s4 < 4; ++s4) {
                pb[s4 * cout + c] = bias->data[c * 4 + s4];
            }
        }
        b.b = upload_float(pb);
    }
    return b;
}

Lin ParamBuilder::conv3x3s2(const std::string& p)
{
    Lin l;
    const HostTensor* w = get(p + "weight", 4);
    const HostTensor* b = get(p + "bias");
    if (w == nullptr || b == nullptr) {
        return l;
    }
    const int cout = static_cast<int>(w->shape[0]);
    const int cin = static_cast<int>(w->shape[1]);
    if (w->shape[2] != 3 || w->shape[3] != 3) {
        fail("'" + p + "weight' is not 3x3");
        return l;
    }
    // [o][c][ky][kx] -> [o][(ky*3 + kx)*cin + c]
    std::vector<float> pw(static_cast<size_t>(cout) * 9 * cin);
    for (int o = 0; o < cout; ++o) {
        for (int c = 0; c < cin; ++c) {
            for (int k = 0; k < 9; ++k) {
                pw[(static_cast<size_t>(o) * 9 + k) * cin + c] =
                    w->data[(static_cast<size_t>(o) * cin + c) * 9 + k];
            }
        }
    }
    l.cin = 9 * cin;
    l.cout = cout;
    l.dtype = dtype_;
    l.w = upload_act(pw, dtype_);
    l.b = upload_float(b->data);
    return l;
}

// ------------------------------------------------------------------------------ execution

void gemm(Launch& L, const Lin& lin, int epi, const __half* x, int ldx, int M, __half* out,
          int ldo, const __half* res, int ldr, const __half* q, int sub_w, const __half* res2,
          int ldr2, int q_rows)
{
    GemmParams p{};
    p.M = M;
    p.N = lin.cout;
    p.K = lin.cin;
    p.bias = lin.b;
    p.res = res;
    p.ldr = ldr;
    p.res2 = res2;
    p.ldr2 = ldr2;
    p.qscale = q;
    p.out = out;
    p.ldo = ldo;
    p.sub_w = sub_w;
    p.sub_cout = epi == kEpiSubpel ? lin.cout / 4 : 0;
    p.q_rows = q != nullptr ? q_rows : 0;
    p.err = L.err_word;
    // the autotuned width of this shape (tuned here on first sight when tuning is enabled and
    // the phase runs eagerly), else the library's rule
    const int bn = gemm_bn_for(lin.dtype, epi, p, L.s);
    L.note(gemm_sm100(lin.dtype, x, ldx, lin.w, p, epi, bn, L.s));
}

void run_dcb(Launch& L, const Dcb& d, const __half* x, int ldx, int H, int W, __half* out, int ldo,
             Scratch& s, const __half* q, int img_h)
{
    // per-image factors in a packed batch: one row of q per image of img_h x W pixels
    const int q_rows = (img_h > 0 && img_h < H) ? img_h * W : 0;
    const int M = H * W;
    const __half* xin = x;
    int ldin = ldx;
    if (d.adaptor) {
        gemm(L, d.ad, kEpiBias, x, ldx, M, s.t0, d.C);
        xin = s.t0;
        ldin = d.C;
    }
    gemm(L, d.dc1, kEpiBiasWsilu, xin, ldin, M, s.t1, d.cdc);
    // d3x3 + conv1x1_bias_shortcut: one streaming GEMM launch whose operand producer computes the
    // depthwise 3x3, or two launches
    const bool stream_dc2 = gemm_stream_form_enabled() && gemm_stream_eligible(kEpiBiasRes, M, d.C, d.cdc);
    const bool dw_fused = stream_dc2 && gemm_dw_fusion_enabled() && d.dc2.dtype == d.dtype;
    if (!dw_fused) {
        L.note(launch_dwconv3x3(s.t1, H, W, d.cdc, d.cdc, d.dw, s.t2, d.cdc, L.s, d.dtype, img_h));
    }
    // the FP8 form: the streaming residual GEMM also writes the E4M3 operand of the quad GEMM
    const bool fp8_quad = d.ffn1_w8 != nullptr && s.t5 != nullptr;
    const bool out8 = fp8_quad && stream_dc2 && d.C % 16 == 0;
    bool t5_ready = false;
    if (dw_fused || out8) {
        GemmParams p{};
        p.M = M;
        p.N = d.C;
        p.K = d.cdc;
        p.bias = d.dc2.b;
        p.res = xin;
        p.ldr = ldin;
        p.out = s.t3;
        p.ldo = d.C;
        p.err = L.err_word;
        if (out8) {
            p.out8 = s.t5;
            p.ldo8 = d.C;
            p.out8_inv_scale = 1.0f / kFp8ActScale;
            t5_ready = true;
        }
        if (dw_fused) {
            p.dw_weight = d.dw;
            p.dw_h = H;
            p.dw_w = W;
            p.dw_img_h = img_h > 0 ? img_h : H;
        }
        L.note(gemm_sm100(d.dc2.dtype, dw_fused ? s.t1 : s.t2, d.cdc, d.dc2.w, p, kEpiBiasRes, kBlockNStream,
                          L.s));
    } else {
        gemm(L, d.dc2, kEpiBiasRes, s.t2, d.cdc, M, s.t3, d.C, xin, ldin);
    }
    if (!d.shortcut && d.dtype == 0 && (q == nullptr || q_rows == 0) &&
        ffn_sm100_preferred(d.C, d.cffn, d.ffn1.cout)) {
        // the ConvFFN as one kernel, the quad output kept on chip (ffn_sm100.cu)
        FfnParams fp{M, d.C, d.cffn, d.ffn1.b, d.ffn2.b, q, out, ldo, L.err_word, 0};
        L.note(ffn_sm100(s.t3, d.C, d.ffn1.w, d.ffn2.w, fp, L.s));
        return;
    }
    if (d.ffn1_w8 != nullptr && s.t5 != nullptr) {
        // the FP8 form: E4M3 copy of the dc output, quad GEMM on kind::f8f6f4
        if (!t5_ready) {
            L.note(launch_quantize_fp8(s.t3, d.dtype, d.C, 1.0f / kFp8ActScale, s.t5, d.C, M, d.C, L.s));
        }
        GemmParams p{};
        p.M = M;
        p.N = d.ffn1.cout;
        p.K = d.ffn1.cin;
        p.bias = d.ffn1.b;
        p.wscale = d.ffn1_ws;
        p.out = s.t4;
        p.ldo = d.cffn;
        p.err = L.err_word;
        L.note(gemm_sm100(kDtypeF8, s.t5, d.C, d.ffn1_w8, p, kEpiQuad, 0, L.s));
    } else {
        gemm(L, d.ffn1, kEpiQuad, s.t3, d.C, M, s.t4, d.cffn);
    }
    if (d.shortcut) {
        // conv1x1_bias_shortcut2 (layers_proxy.cpp:89-91): ffn + ffn input + block input
        gemm(L, d.ffn2, kEpiBiasRes2, s.t4, d.cffn, M, out, ldo, s.t3, d.C, nullptr, 0, xin, ldin);
        return;
    }
    if (q != nullptr) {
        gemm(L, d.ffn2, kEpiBiasResQ, s.t4, d.cffn, M, out, ldo, s.t3, d.C, q, 0, nullptr, 0,
             q_rows);
    } else {
        gemm(L, d.ffn2, kEpiBiasRes, s.t4, d.cffn, M, out, ldo, s.t3, d.C);
    }
}

}  // namespace dcvc
