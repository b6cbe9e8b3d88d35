"""ORACLE (test infrastructure only; never imported by the product).

CPU restatement of the reference's low-delay (LD) video codec as its CUDA proxy runs it
(src/layers/extensions/inference/dmc_ld_proxy.cpp:420-566 compress / decompress, :639-655 the
memory update), in float64 or float32 PyTorch CPU ops, reading the weights from a state dict.
Used by tests/ (PSNR / bpp / symbol agreement against the GPU path); the sub-networks are pinned
against the reference nn.Modules by tests/golden/ld_modules_golden.npz.

One frame per call.  Network math follows src/models/video_model_ld.py (Decoder :24-40, Encoder
:43-59, FeatureAdaptorI/M :62-89, FeatureExtractor :92-106, HyperDecoder/Encoder :109-134,
PriorFusion :137-148 with the temporal parameters scaled by q_feature, ReconHead :151-166,
SpatialPrior :169-179, TemporalPriorEncoder :182-188).  The temporal parameters are computed
right after every memory update (dmc_ld_proxy.cpp:407-418, 470-475, 509-515); the entropy model
is the 2-phase checkerboard of common_model.py:157-172, 212-229 (phase p codes channel half g at
the 2x2 positions with (h + w + g + p) even), with the proxy's skip threshold, clamps and a final
x max(q_dec, 0.5) (process_with_mask_no_scale*, stream.cu:548-683); the symbols of both phases
form one NHWC segment with the scales of the prior fusion, followed by z.
"""
import numpy as np
import torch
import torch.nn.functional as F

from hts_oracle import (HtsOracle, ec_parallel_for, rans_decode, rans_encode, round_half_away,
                        scale_index)

CH_Y, CH_Z = 128, 128


def mask_2x(phase, C, H, W, dtype):
    g = torch.arange(C) // (C // 2)
    hw = (torch.arange(H)[:, None] + torch.arange(W)[None, :])
    return (((hw[None] + g[:, None, None] + phase) % 2) == 0).to(dtype)[None]


class LdOracle(HtsOracle):
    """One stream of the LD codec on the CPU."""

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.temporal = None

    # ---- sub-networks (video_model_ld.py)
    def encoder(self, x, ctx, q_enc):
        f = torch.cat((F.pixel_unshuffle(x, 8), ctx), dim=1)
        f = self.seq("encoder.conv1.", 2, f)
        f = self.dcb("encoder.conv2.", f, q_enc)
        return self.conv("encoder.down.", f, stride=2, padding=1)

    def hyper_encoder(self, y):
        z = self.dcb("hyper_encoder.conv.0.", y)
        z = self.rb_down("hyper_encoder.conv.1.", z)
        return self.rb_down("hyper_encoder.conv.2.", z)

    def hyper_decoder(self, z_hat):
        h = self.rb_up("hyper_decoder.conv.0.", z_hat)
        h = self.rb_up("hyper_decoder.conv.1.", h)
        return self.dcb("hyper_decoder.conv.2.", h)

    def temporal_prior_ld(self, memory):
        return self.rb_down("temporal_prior_encoder.conv.", memory)

    def prior_fusion_ld(self, hyper, temporal, q_feat):
        x = self.seq("y_prior_fusion.conv.", 3, torch.cat((hyper, temporal * q_feat), dim=1))
        return self.conv("y_prior_fusion.conv.3.", x)

    def spatial_prior_ld(self, y_hat, common):
        x = self.seq("y_spatial_prior.conv.", 2, torch.cat((y_hat, common), dim=1))
        return self.conv("y_spatial_prior.conv.2.", x)

    def decoder(self, y_hat, ctx, q_dec):
        up = self.subpel("decoder.up.", y_hat)
        f = self.seq("decoder.conv1.", 3, torch.cat((up, ctx), dim=1))
        return self.conv("decoder.conv2.", f) * q_dec

    def feature_adaptor_i(self, f):
        return self.seq("feature_adaptor_i.conv.", 4, f)

    def feature_adaptor_m(self, memory, feature):
        return self.seq("feature_adaptor_m.conv.", 4, torch.cat((memory, feature), dim=1))

    def feature_extractor(self, memory):
        return self.seq("feature_extractor.conv.", 5, memory)

    def recon_head_out(self, feature):
        """ReconHead.forward(for_reset=True): the 192-channel head before pixel_shuffle."""
        return self.conv("recon_head.head.", self.seq("recon_head.conv.", 3, feature))

    # ---- public API mirroring DMCLDProxy
    def add_ref_feature_from_frame(self, frame, apply_adaptor=True):
        self.feature_i = F.pixel_unshuffle(frame.to("cpu", self.dtype), 8)
        if apply_adaptor:
            self.memory = self.feature_adaptor_i(self.feature_i)
            self.ctx = self.feature_extractor(self.memory)
            self.temporal = self.temporal_prior_ld(self.memory)
        self.memory_has_value = bool(apply_adaptor)

    def set_temporal_state(self, memory):
        """Tests: the temporal memory the next frame is coded with (already updated)."""
        self.memory = memory.to(self.dtype)
        self.ctx = self.feature_extractor(self.memory)
        self.temporal = self.temporal_prior_ld(self.memory)
        self._memory_ready = True

    def entropy_params_ld(self, z_hat, qp, H16, W16):
        hyper = self.hyper_decoder(z_hat)[:, :, :H16, :W16]
        common = self.prior_fusion_ld(hyper, self.temporal, self.q("q_feature", qp))
        q_dec, scales, means = common.chunk(3, 1)
        return common, torch.clamp_min(q_dec, 0.5), scales, means

    @torch.no_grad()
    def compress(self, x, qp, reset_feature_memory, padding_b, padding_r, ec_parallel=None):
        x = F.pad(x.to("cpu", self.dtype), (0, padding_r, 0, padding_b), mode="replicate")
        y = self.encoder(x, self.ctx, self.q("q_encoder", qp))
        _, C, H16, W16 = y.shape
        ph, pw = (-H16) % 4, (-W16) % 4
        y_pad = F.pad(y, (0, pw, 0, ph), mode="replicate") if (ph or pw) else y
        z = self.hyper_encoder(y_pad)
        z_hat = torch.clamp(round_half_away(z), -64, 63)
        common, q_dec, scales, means = self.entropy_params_ld(z_hat, qp, H16, W16)
        y = y / q_dec
        y_q = torch.zeros_like(y)
        y_hat = torch.zeros_like(y)
        for k in range(2):
            if k == 1:
                means = self.spatial_prior_ld(y_hat, common)
            m = mask_2x(k, C, H16, W16, self.dtype)
            s_hat = scales * m
            m_hat = means * m
            q = round_half_away((y - m_hat) * m) * (s_hat > self.thr).to(self.dtype)
            q = torch.clamp(q, -128, 127)
            y_q = y_q + q
            y_hat = y_hat + (q + m_hat)
        y_hat = y_hat * q_dec
        s_nhwc = scales[0].permute(1, 2, 0).reshape(-1).numpy()
        q_nhwc = y_q[0].permute(1, 2, 0).reshape(-1).numpy().astype(np.int64)
        cond = s_nhwc > self.thr
        idx = scale_index(s_nhwc)
        sym = ((q_nhwc << 8) + idx.astype(np.int64)).astype(np.int16)[cond]
        z_i8 = z_hat[0].permute(1, 2, 0).reshape(-1).numpy().astype(np.int8)
        ecp = ec_parallel or ec_parallel_for(sym.size)
        data = rans_encode(self.cdf_z, self.len_z, self.cdf_y, self.len_y, sym, z_i8,
                           qp * CH_Z, CH_Z, ecp)
        feature = self.decoder(y_hat, self.ctx, self.q("q_decoder", qp))
        if reset_feature_memory:
            self.memory = self.feature_adaptor_i(self.recon_head_out(feature))
        else:
            self.memory = self.feature_adaptor_m(self.memory, feature)
        self.ctx = self.feature_extractor(self.memory)
        self.temporal = self.temporal_prior_ld(self.memory)
        return {"bit_stream": data, "ec_parallel": ecp, "y_q": y_q, "y_hat": y_hat,
                "z_hat": z_hat, "symbols": sym, "feature": feature}

    @torch.no_grad()
    def decompress(self, bit_stream, qp, height, width, ec_parallel, reset_feature_memory):
        Hp, Wp = (height + 15) // 16 * 16, (width + 15) // 16 * 16
        H16, W16 = Hp // 16, Wp // 16
        H64, W64 = (height + 63) // 64, (width + 63) // 64
        if getattr(self, "_memory_ready", False):
            self._memory_ready = False
        else:
            if self.memory_has_value:
                self.memory = self.feature_adaptor_m(self.memory, self.feature_p)
            else:
                self.memory = self.feature_adaptor_i(self.feature_i)
            self.temporal = self.temporal_prior_ld(self.memory)
        n_z = CH_Z * H64 * W64
        _, z_i8 = rans_decode(self.cdf_z, self.len_z, self.cdf_y, self.len_y, bit_stream,
                              np.zeros(0, np.uint8), n_z, qp * CH_Z, CH_Z, ec_parallel)
        z_hat = torch.from_numpy(z_i8.astype(np.float64)).to(self.dtype)
        z_hat = z_hat.reshape(H64, W64, CH_Z).permute(2, 0, 1)[None]
        common, q_dec, scales, means = self.entropy_params_ld(z_hat, qp, H16, W16)
        s_nhwc = scales[0].permute(1, 2, 0).reshape(-1).numpy()
        cond = s_nhwc > self.thr
        idx = scale_index(s_nhwc)[cond]
        y_dec, _ = rans_decode(self.cdf_z, self.len_z, self.cdf_y, self.len_y, bit_stream,
                               np.ascontiguousarray(idx, np.uint8), n_z, qp * CH_Z, CH_Z,
                               ec_parallel)
        full = np.zeros(s_nhwc.size, np.float64)
        full[cond] = y_dec
        C = scales.shape[1]
        y_q = torch.from_numpy(full).to(self.dtype).reshape(H16, W16, C).permute(2, 0, 1)[None]
        self.ctx = self.feature_extractor(self.memory)
        y_hat = torch.zeros_like(y_q)
        for k in range(2):
            if k == 1:
                means = self.spatial_prior_ld(y_hat, common)
            m = mask_2x(k, C, H16, W16, self.dtype)
            y_hat = y_hat + (y_q + means) * m
        y_hat = y_hat * q_dec
        feature = self.decoder(y_hat, self.ctx, self.q("q_decoder", qp))
        head = self.recon_head_out(feature)
        x_hat = torch.clamp(F.pixel_shuffle(head, 8), -0.5, 0.5)
        self.feature_p = feature
        self.feature_i = head
        self.memory_has_value = not reset_feature_memory
        return {"x_hat": x_hat, "y_q": y_q, "y_hat": y_hat, "z_hat": z_hat}
