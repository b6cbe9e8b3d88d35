"""Parameter layout and seeded initialisation of the DCVC-UF HT-S video model and the intra model.

The module tree mirrors the reference's nn.Module structure (src/models/video_model_ht.py:26-
351, src/layers/layers.py:92-188, src/models/image_model.py:15-140) only as far as parameter
names, shapes, registration order and initialisation go: building it under
torch.manual_seed(s) consumes the random stream exactly as the reference constructor does
(default Conv2d init, then BitEstimator normals, then xavier_normal_ over modules(),
common_model.py:49-54), so `hts_state_dict(seed)` equals the reference `DMC().state_dict()`
for the same seed.  There is no forward here: the codec runs in libdcvc_b200.so.
"""
import torch
from torch import nn

# HT-S sizes (video_model_ht.py:16-23)
FRAME_DELAY = 8
CH_SRC_INTRA = 3 * 8 * 8
CH_SRC = CH_SRC_INTRA * FRAME_DELAY
CH_Y = 256
CH_Z = 128
CH_D = 512
CH_M = 512
CH_RECON = 256
QP_NUM = 64
# intra model sizes (image_model.py:11-14)
CH_ENC_DEC_INTRA = 384
# Residual-branch scale of the calibrated variants (see calibrated_hts_state_dict).
CALIBRATION_ALPHA = 0.1


class _Act(nn.Module):
    """Parameter-free placeholder (WSiLU / WSiLUChunkAdd / PixelShuffle) keeping indices aligned."""


class DCB(nn.Module):
    """DepthConvBlock parameters (layers.py:128-159)."""

    def __init__(self, in_ch, out_ch, dcb2=False, force_adaptor=False):
        super().__init__()
        self.adaptor = nn.Conv2d(in_ch, out_ch, 1) if (in_ch != out_ch or force_adaptor) else None
        r = 2 if dcb2 else 1
        self.dc = nn.Sequential(
            nn.Conv2d(out_ch, out_ch // r, 1), _Act(),
            nn.Conv2d(out_ch // r, out_ch // r, 3, padding=1, groups=out_ch // r),
            nn.Conv2d(out_ch // r, out_ch, 1))
        self.ffn = nn.Sequential(nn.Conv2d(out_ch, out_ch * 4 // r, 1), _Act(),
                                 nn.Conv2d(out_ch // r, out_ch, 1))


class Subpel(nn.Module):
    """SubpelConv2x (layers.py:92-103)."""

    def __init__(self, in_ch, out_ch, k=1, padding=0, force_bias=False):
        super().__init__()
        self.conv = nn.Sequential(
            nn.Conv2d(in_ch, out_ch * 4, k, padding=padding, bias=(k > 1) or force_bias), _Act())


class RBUp(nn.Module):
    """ResidualBlockUpsample (layers.py:162-173)."""

    def __init__(self, in_ch, out_ch, dcb2=False, force_bias=False):
        super().__init__()
        self.up = Subpel(in_ch, out_ch, 1, force_bias=force_bias)
        self.conv = DCB(out_ch, out_ch, dcb2=dcb2)


class RBDown(nn.Module):
    """ResidualBlockWithStride2 (layers.py:176-188)."""

    def __init__(self, in_ch, out_ch, dcb2=False):
        super().__init__()
        self.down = nn.Conv2d(in_ch * 4, out_ch, 1)
        self.conv = DCB(out_ch, out_ch, dcb2=dcb2)


class BitEstimator(nn.Module):
    """entropy_models.py:103-113."""

    def __init__(self, qp_num, channel):
        super().__init__()
        self.h = nn.Parameter(nn.init.normal_(torch.empty([qp_num, channel, 4]), 0, 0.01))
        self.b = nn.Parameter(nn.init.normal_(torch.empty([qp_num, channel, 4]), 0, 0.01))
        self.a = nn.Parameter(nn.init.normal_(torch.empty([qp_num, channel, 3]), 0, 0.01))


def _seq(*mods):
    return nn.Sequential(*mods)


class _Wrap(nn.Module):
    def __init__(self, **kw):
        super().__init__()
        for k, v in kw.items():
            setattr(self, k, v)


def _init_xavier(model):
    for m in model.modules():
        if isinstance(m, nn.Conv2d):
            nn.init.xavier_normal_(m.weight, 1.)
            if m.bias is not None:
                nn.init.constant_(m.bias, 0.)


class HTSModel(nn.Module):
    """Parameter tree of DMC(ModelStructure.HTS) (video_model_ht.py:320-351)."""

    def __init__(self):
        super().__init__()
        self.bit_estimator_z = BitEstimator(QP_NUM, CH_Z)
        d = lambda i, o: DCB(i, o, dcb2=True)  # noqa: E731
        self.feature_adaptor_i = _Wrap(conv=_seq(d(CH_SRC_INTRA, CH_M), *[d(CH_M, CH_M) for _ in range(3)]))
        self.feature_adaptor_m = _Wrap(conv=_seq(d(CH_M + CH_D, CH_M), *[d(CH_M, CH_M) for _ in range(5)]))
        self.feature_extractor = _Wrap(conv=_seq(d(CH_M, CH_D), *[d(CH_D, CH_D) for _ in range(4)]))
        enc = _Wrap(conv1=_seq(d(CH_SRC + CH_D, CH_D), *[d(CH_D, CH_D) for _ in range(5)]))
        enc.down = nn.Conv2d(CH_D, CH_Y, 3, stride=2, padding=1)
        self.encoder = enc
        self.hyper_encoder = _Wrap(conv=_seq(DCB(CH_Y, CH_Y), RBDown(CH_Y, CH_Y), RBDown(CH_Y, CH_Z)))
        self.hyper_decoder = _Wrap(conv=_seq(RBUp(CH_Z, CH_Y), RBUp(CH_Y, CH_Y), DCB(CH_Y, CH_Y)))
        self.temporal_prior_encoder = _Wrap(conv=RBDown(CH_D, CH_Y * 2))
        pf = [DCB(CH_Y * 3, CH_Y * 3) for _ in range(3)]
        self.y_prior_fusion = _Wrap(conv=_seq(*pf, nn.Conv2d(CH_Y * 3, CH_Y * 3, 1)))
        self.y_spatial_prior_reduction = nn.Conv2d(CH_Y * 3, CH_Y, 1)
        for k in (1, 2, 3):
            setattr(self, f"y_spatial_prior_adaptor_{k}", DCB(CH_Y * 2, CH_Y * 2, force_adaptor=True))
        sp = [DCB(CH_Y * 2, CH_Y * 2) for _ in range(3)]
        self.y_spatial_prior = _Wrap(conv=_seq(*sp, nn.Conv2d(CH_Y * 2, CH_Y, 1)))
        dec = _Wrap(up=Subpel(CH_Y, CH_D, 1))
        dec.conv1 = _seq(d(CH_D * 2, CH_D), *[d(CH_D, CH_D) for _ in range(6)])
        self.decoder = dec
        rh = _Wrap(conv1=nn.ModuleList([_seq(DCB(CH_D, CH_D)) for _ in range(FRAME_DELAY // 2)]))
        rh.conv2 = nn.ModuleList([
            _seq(DCB(CH_D, CH_RECON), DCB(CH_RECON, CH_RECON), DCB(CH_RECON, CH_RECON),
                 nn.Conv2d(CH_RECON, CH_SRC_INTRA, 1)) for _ in range(FRAME_DELAY)])
        self.recon_head = rh
        self.q_encoder = nn.Parameter(torch.ones((QP_NUM, CH_D)))
        self.q_decoder = nn.Parameter(torch.ones((QP_NUM, CH_D)))
        self.q_feature = nn.Parameter(torch.ones((QP_NUM, CH_D)))
        _init_xavier(self)


class HTLModel(nn.Module):
    """Parameter tree of DMC(ModelStructure.HTL) (video_model_ht.py:24-351 with is_hts False):
    plain (not dcb2) DepthConvBlocks, a 3x3 sub-pixel decoder up-sampling with bias, biased
    hyper-decoder up-sampling, and resampling blocks with the default shortcut."""

    def __init__(self):
        super().__init__()
        self.bit_estimator_z = BitEstimator(QP_NUM, CH_Z)
        self.feature_adaptor_i = _Wrap(conv=_seq(DCB(CH_SRC_INTRA, CH_M), DCB(CH_M, CH_M), DCB(CH_M, CH_M)))
        self.feature_adaptor_m = _Wrap(conv=_seq(DCB(CH_M + CH_D, CH_M), *[DCB(CH_M, CH_M) for _ in range(9)]))
        self.feature_extractor = _Wrap(conv=_seq(DCB(CH_M, CH_D), DCB(CH_D, CH_D)))
        enc = _Wrap(conv1=_seq(DCB(CH_SRC + CH_D, CH_D), *[DCB(CH_D, CH_D) for _ in range(6)]))
        enc.down = nn.Conv2d(CH_D, CH_Y, 3, stride=2, padding=1)
        self.encoder = enc
        self.hyper_encoder = _Wrap(conv=_seq(DCB(CH_Y, CH_Y), RBDown(CH_Y, CH_Y), RBDown(CH_Y, CH_Z)))
        self.hyper_decoder = _Wrap(conv=_seq(RBUp(CH_Z, CH_Y, force_bias=True),
                                             RBUp(CH_Y, CH_Y, force_bias=True), DCB(CH_Y, CH_Y)))
        self.temporal_prior_encoder = _Wrap(conv=RBDown(CH_D, CH_Y * 2))
        pf = [DCB(CH_Y * 3, CH_Y * 3) for _ in range(3)]
        self.y_prior_fusion = _Wrap(conv=_seq(*pf, nn.Conv2d(CH_Y * 3, CH_Y * 3, 1)))
        self.y_spatial_prior_reduction = nn.Conv2d(CH_Y * 3, CH_Y, 1)
        for k in (1, 2, 3):
            setattr(self, f"y_spatial_prior_adaptor_{k}", DCB(CH_Y * 2, CH_Y * 2, force_adaptor=True))
        sp = [DCB(CH_Y * 2, CH_Y * 2) for _ in range(3)]
        self.y_spatial_prior = _Wrap(conv=_seq(*sp, nn.Conv2d(CH_Y * 2, CH_Y * 2, 1)))
        dec = _Wrap(up=Subpel(CH_Y, CH_D, 3, padding=1, force_bias=True))
        dec.conv1 = _seq(DCB(CH_D * 2, CH_D), *[DCB(CH_D, CH_D) for _ in range(10)])
        self.decoder = dec
        self.recon_head = _Wrap(conv=nn.ModuleList([
            _seq(DCB(CH_D, CH_RECON), *[DCB(CH_RECON, CH_RECON) for _ in range(4)],
                 nn.Conv2d(CH_RECON, CH_SRC_INTRA, 1)) for _ in range(FRAME_DELAY)]))
        self.q_encoder = nn.Parameter(torch.ones((QP_NUM, CH_D)))
        self.q_decoder = nn.Parameter(torch.ones((QP_NUM, CH_D)))
        self.q_feature = nn.Parameter(torch.ones((QP_NUM, CH_D)))
        _init_xavier(self)


def htl_state_dict(seed=0, dtype=torch.float32):
    """State dict of a random-init HT-L model, equal to the reference DMC(ModelStructure.HTL)
    under torch.manual_seed(seed) (fp32 CPU; cast to `dtype`)."""
    return _seeded(HTLModel, seed, dtype)


def calibrated_htl_state_dict(seed=0, dtype=torch.float32, alpha=CALIBRATION_ALPHA):
    """The seed-`seed` HT-L weights with the residual-branch output convolutions scaled by
    `alpha` (see calibrated_hts_state_dict)."""
    sd = htl_state_dict(seed, torch.float32)
    for k in list(sd):
        if k.endswith(("dc.3.weight", "ffn.2.weight")):
            sd[k] = sd[k] * alpha
    return {k: v.to(dtype) for k, v in sd.items()}


def perturbed_htl_state_dict(seed=0, dtype=torch.float32, q_jitter=0.25, calibrated=True):
    """Seed-`seed` HT-L weights with non-trivial per-QP quant vectors."""
    sd = calibrated_htl_state_dict(seed) if calibrated else htl_state_dict(seed, torch.float32)
    g = torch.Generator().manual_seed(seed + 23)
    for k in ("q_encoder", "q_decoder", "q_feature"):
        sd[k] = 1.0 + q_jitter * (torch.rand(sd[k].shape, generator=g) * 2 - 1)
    return {k: v.to(dtype) for k, v in sd.items()}


# LD model sizes (video_model_ld.py:11-16)
LD_CH_Y, LD_CH_Z, LD_CH_D, LD_CH_M = 128, 128, 256, 256


class LDModel(nn.Module):
    """Parameter tree of the low-delay model DMC (video_model_ld.py:18-213): one frame per call,
    dcb2 DepthConvBlocks, resampling blocks without shortcut, a means-only spatial prior."""

    def __init__(self):
        super().__init__()
        y, z, dd, m = LD_CH_Y, LD_CH_Z, LD_CH_D, LD_CH_M
        d = lambda i, o: DCB(i, o, dcb2=True)  # noqa: E731
        self.bit_estimator_z = BitEstimator(QP_NUM, z)
        self.feature_adaptor_i = _Wrap(conv=_seq(d(CH_SRC_INTRA, m), d(m, m), d(m, m), d(m, m)))
        self.feature_adaptor_m = _Wrap(conv=_seq(d(m + dd, m), d(m, m), d(m, m), d(m, m)))
        self.feature_extractor = _Wrap(conv=_seq(*[d(m, m) for _ in range(5)]))
        enc = _Wrap(conv1=_seq(d(CH_SRC_INTRA + m, dd), d(dd, dd)))
        enc.conv2 = d(dd, dd)
        enc.down = nn.Conv2d(dd, y, 3, stride=2, padding=1)
        self.encoder = enc
        self.hyper_encoder = _Wrap(conv=_seq(d(y, z), RBDown(z, z, dcb2=True), RBDown(z, z, dcb2=True)))
        self.hyper_decoder = _Wrap(conv=_seq(RBUp(z, z, dcb2=True), RBUp(z, z, dcb2=True), d(z, y)))
        self.temporal_prior_encoder = _Wrap(conv=RBDown(m, y * 2, dcb2=True))
        self.y_prior_fusion = _Wrap(conv=_seq(d(y * 3, y * 3), d(y * 3, y * 3), d(y * 3, y * 3),
                                              nn.Conv2d(y * 3, y * 3, 1)))
        self.y_spatial_prior = _Wrap(conv=_seq(d(y * 4, y * 2), d(y * 2, y * 2), nn.Conv2d(y * 2, y, 1)))
        dec = _Wrap(up=Subpel(y, dd, 1))
        dec.conv1 = _seq(d(dd + m, dd), d(dd, dd), d(dd, dd))
        dec.conv2 = nn.Conv2d(dd, dd, 1)
        self.decoder = dec
        rh = _Wrap(conv=_seq(d(dd, dd), d(dd, dd), d(dd, dd)))
        rh.head = nn.Conv2d(dd, CH_SRC_INTRA, 1)
        self.recon_head = rh
        self.q_encoder = nn.Parameter(torch.ones((QP_NUM, dd)))
        self.q_decoder = nn.Parameter(torch.ones((QP_NUM, dd)))
        self.q_feature = nn.Parameter(torch.ones((QP_NUM, y * 2)))
        _init_xavier(self)


def ld_state_dict(seed=0, dtype=torch.float32):
    """State dict of a random-init LD model, equal to the reference video_model_ld.DMC() under
    torch.manual_seed(seed) (fp32 CPU; cast to `dtype`)."""
    return _seeded(LDModel, seed, dtype)


def calibrated_ld_state_dict(seed=0, dtype=torch.float32, alpha=CALIBRATION_ALPHA):
    """The seed-`seed` LD weights with the residual-branch output convolutions scaled by
    `alpha` (see calibrated_hts_state_dict)."""
    sd = ld_state_dict(seed, torch.float32)
    for k in list(sd):
        if k.endswith(("dc.3.weight", "ffn.2.weight")):
            sd[k] = sd[k] * alpha
    return {k: v.to(dtype) for k, v in sd.items()}


def perturbed_ld_state_dict(seed=0, dtype=torch.float32, q_jitter=0.25, calibrated=True):
    """Seed-`seed` LD weights with non-trivial per-QP quant vectors."""
    sd = calibrated_ld_state_dict(seed) if calibrated else ld_state_dict(seed, torch.float32)
    g = torch.Generator().manual_seed(seed + 29)
    for k in ("q_encoder", "q_decoder", "q_feature"):
        sd[k] = 1.0 + q_jitter * (torch.rand(sd[k].shape, generator=g) * 2 - 1)
    return {k: v.to(dtype) for k, v in sd.items()}


class DMCIModel(nn.Module):
    """Parameter tree of DMCI, the intra model (image_model.py:15-140).  Its resampling blocks
    keep the reference's default shortcut (layers.py:162-188), which has no parameters."""

    def __init__(self):
        super().__init__()
        self.bit_estimator_z = BitEstimator(QP_NUM, CH_Z)
        c = CH_ENC_DEC_INTRA
        enc = _Wrap(enc_1=DCB(CH_SRC_INTRA, c))
        enc.enc_2 = _seq(*[DCB(c, c) for _ in range(6)], nn.Conv2d(c, CH_Y, 3, stride=2, padding=1))
        self.enc = enc
        self.hyper_enc = _Wrap(conv=_seq(DCB(CH_Y, CH_Z), RBDown(CH_Z, CH_Z), RBDown(CH_Z, CH_Z)))
        self.hyper_dec = _Wrap(conv=_seq(RBUp(CH_Z, CH_Z), RBUp(CH_Z, CH_Z), DCB(CH_Z, CH_Y)))
        self.y_prior_fusion = _Wrap(conv=_seq(DCB(CH_Y, CH_Y * 2), DCB(CH_Y * 2, CH_Y * 2),
                                              DCB(CH_Y * 2, CH_Y * 2), nn.Conv2d(CH_Y * 2, CH_Y * 2, 1)))
        self.y_spatial_prior_reduction = nn.Conv2d(CH_Y * 2, CH_Y, 1)
        for k in (1, 2, 3):
            setattr(self, f"y_spatial_prior_adaptor_{k}", DCB(CH_Y * 2, CH_Y * 2, force_adaptor=True))
        sp = [DCB(CH_Y * 2, CH_Y * 2) for _ in range(3)]
        self.y_spatial_prior = _Wrap(conv=_seq(*sp, nn.Conv2d(CH_Y * 2, CH_Y * 2, 1)))
        dec = _Wrap(dec_1=_seq(RBUp(CH_Y, c), *[DCB(c, c) for _ in range(12)]))
        dec.dec_2 = DCB(c, CH_SRC_INTRA)
        self.dec = dec
        self.q_scale_enc = nn.Parameter(torch.ones((QP_NUM, c)))
        self.q_scale_dec = nn.Parameter(torch.ones((QP_NUM, c)))
        self.q_scale_y_enc = nn.Parameter(torch.ones((QP_NUM, CH_Y)))
        self.q_scale_y_dec = nn.Parameter(torch.ones((QP_NUM, CH_Y)))
        _init_xavier(self)


def _seeded(cls, seed, dtype):
    state = torch.random.get_rng_state()
    try:
        torch.manual_seed(seed)
        model = cls()
    finally:
        torch.random.set_rng_state(state)
    return {k: v.detach().to(dtype) for k, v in model.state_dict().items()}


def dmci_state_dict(seed=0, dtype=torch.float32):
    """State dict of a random-init intra model, equal to the reference DMCI() under
    torch.manual_seed(seed) (fp32 CPU; cast to `dtype`)."""
    return _seeded(DMCIModel, seed, dtype)


def hts_state_dict(seed=0, dtype=torch.float32):
    """State dict of a random-init HT-S model, equal to the reference DMC() under
    torch.manual_seed(seed) (fp32 CPU; cast to `dtype`)."""
    return _seeded(HTSModel, seed, dtype)



def calibrated_hts_state_dict(seed=0, dtype=torch.float32, alpha=CALIBRATION_ALPHA):
    """The seed-`seed` random-init weights with the output convolution of every residual branch
    (dc.3 and ffn.2 of each DepthConvBlock) scaled by `alpha`.

    The plain random init is numerically unstable: every DepthConvBlock adds its branch to its
    input at full gain, so activations grow by orders of magnitude per block and the temporal
    memory by about 1e14 per chunk (in FP64 as well), and any FP16 implementation overflows in
    the first chunk.  With alpha = 0.1 activations stay O(1) across chunks and 10-20 % of the y
    latents are coded, a realistic entropy-coding load.  Architecture, shapes and FLOPs are
    unchanged."""
    sd = hts_state_dict(seed, torch.float32)
    for k in list(sd):
        if k.endswith(("dc.3.weight", "ffn.2.weight")):
            sd[k] = sd[k] * alpha
    return {k: v.to(dtype) for k, v in sd.items()}


def calibrated_dmci_state_dict(seed=0, dtype=torch.float32, alpha=CALIBRATION_ALPHA):
    """The seed-`seed` intra weights with the residual-branch output convolutions scaled by
    `alpha`, for the reason given in calibrated_hts_state_dict."""
    sd = dmci_state_dict(seed, torch.float32)
    for k in list(sd):
        if k.endswith(("dc.3.weight", "ffn.2.weight")):
            sd[k] = sd[k] * alpha
    return {k: v.to(dtype) for k, v in sd.items()}


def perturbed_dmci_state_dict(seed=0, dtype=torch.float32, q_jitter=0.25, calibrated=True):
    """Seed-`seed` intra weights with non-trivial per-QP quant vectors."""
    sd = calibrated_dmci_state_dict(seed) if calibrated else dmci_state_dict(seed, torch.float32)
    g = torch.Generator().manual_seed(seed + 19)
    for k in ("q_scale_enc", "q_scale_dec", "q_scale_y_enc", "q_scale_y_dec"):
        sd[k] = 1.0 + q_jitter * (torch.rand(sd[k].shape, generator=g) * 2 - 1)
    return {k: v.to(dtype) for k, v in sd.items()}


def perturbed_hts_state_dict(seed=0, dtype=torch.float32, q_jitter=0.25, calibrated=True):
    """Seed-`seed` weights (calibrated by default) with non-trivial per-QP quant vectors (the
    random init sets them to ones, which hides QP dependence); used by tests that must see
    QP-specific behaviour."""
    sd = calibrated_hts_state_dict(seed) if calibrated else hts_state_dict(seed, torch.float32)
    g = torch.Generator().manual_seed(seed + 17)
    for k in ("q_encoder", "q_decoder", "q_feature"):
        sd[k] = 1.0 + q_jitter * (torch.rand(sd[k].shape, generator=g) * 2 - 1)
    return {k: v.to(dtype) for k, v in sd.items()}
