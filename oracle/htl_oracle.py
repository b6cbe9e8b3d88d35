"""ORACLE (test infrastructure only; never imported by the product).

CPU restatement of the reference's DCVC-UF HT-L chunk codec as its CUDA proxy runs it
(src/layers/extensions/inference/dmc_htl_proxy.cpp:583-916 compress / decompress, :503-582 the
entropy worker), in float64 or float32 PyTorch CPU ops, reading the weights from a state dict.
Used by tests/ (PSNR / bpp / symbol agreement against the GPU path); the sub-networks are pinned
against the reference nn.Modules by tests/golden/htl_modules_golden.npz.

HT-L is the HT-S dataflow (temporal memory, prior fusion into q_dec | scales | means, y divided
by max(q_dec, 0.5)) with the HT-L modules of src/models/video_model_ht.py (is_hts False: plain
DepthConvBlocks, the 3x3 biased sub-pixel decoder up-sampling :41, biased hyper-decoder
up-sampling :167-181, resampling blocks with their default shortcut :184-198, :307-317, the
per-frame recon heads :215-275) and the intra model's 4-step coding: the spatial prior over
cat(y_hat so far, reduced params) gives the scales and means of steps 1-3
(common_model.py:231-290 with spatial_prior_has_scales), every step codes the quarter of the
channels active at each 2x2 position, the payload holds the steps' symbols in the order 3, 2, 1,
0 then z, and the reconstruction is (y_hat so far + step 3) x max(q_dec, 0.5)
(dmc_htl_proxy.cpp:606-689, 864-909).
"""
import numpy as np
import torch
import torch.nn.functional as F

from hts_oracle import (HtsOracle, RansSegmentDecoder, checker_mask, ec_parallel_for,
                        rans_encode_segments, round_half_away, scale_index)
from intra_oracle import nhwc, quarter_part

CH_Y, CH_Z = 256, 128


class HtlOracle(HtsOracle):
    """One stream of the HT-L codec on the CPU."""

    # ---- sub-networks (video_model_ht.py, is_hts False)
    def encoder(self, x, ctx, q_enc):
        f = torch.cat((F.pixel_unshuffle(x, 8), ctx), dim=1)
        f = self.seq("encoder.conv1.", 7, f, q_enc)
        return self.conv("encoder.down.", f, stride=2, padding=1)

    def hyper_encoder(self, y):
        z = self.dcb("hyper_encoder.conv.0.", y)
        z = self.rb_down("hyper_encoder.conv.1.", z, shortcut=True)
        return self.rb_down("hyper_encoder.conv.2.", z, shortcut=True)

    def hyper_decoder(self, z_hat):
        h = self.rb_up("hyper_decoder.conv.0.", z_hat, shortcut=True)
        h = self.rb_up("hyper_decoder.conv.1.", h, shortcut=True)
        return self.dcb("hyper_decoder.conv.2.", h)

    def temporal_prior(self, memory, q_feat):
        return self.rb_down("temporal_prior_encoder.conv.", memory * q_feat, shortcut=True)

    def spatial_prior(self, k, y_hat, reduced):
        x = self.dcb(f"y_spatial_prior_adaptor_{k}.", torch.cat((y_hat, reduced), dim=1))
        x = self.seq("y_spatial_prior.conv.", 3, x)
        return self.conv("y_spatial_prior.conv.3.", x)

    def decoder(self, y_hat, ctx, q_dec):
        up = F.pixel_shuffle(self.conv("decoder.up.conv.0.", y_hat, padding=1), 2)
        return self.seq("decoder.conv1.", 11, torch.cat((up, ctx), dim=1), q_dec)

    def feature_adaptor_i(self, f):
        return self.seq("feature_adaptor_i.conv.", 3, f)

    def feature_adaptor_m(self, memory, feature):
        return self.seq("feature_adaptor_m.conv.", 10, torch.cat((memory, feature), dim=1))

    def feature_extractor(self, memory):
        return self.seq("feature_extractor.conv.", 2, memory)

    def recon_head_frame(self, i, feature):
        out = self.seq(f"recon_head.conv.{i}.", 5, feature)
        return self.conv(f"recon_head.conv.{i}.5.", out)

    def recon_head(self, feature):
        frames = []
        head7 = None
        for i in range(8):
            h = self.recon_head_frame(i, feature)
            if i == 7:
                head7 = h
            frames.append(torch.clamp(F.pixel_shuffle(h, 8), -0.5, 0.5))
        return frames, head7

    def recon_head_reset(self, feature):
        return self.recon_head_frame(7, feature)

    # ---- public API mirroring DMCHTLProxy
    @torch.no_grad()
    def compress(self, x, qp, reset_feature_memory, padding_b, padding_r, ec_parallel=None):
        x = F.pad(x.to("cpu", self.dtype), (0, padding_r, 0, padding_b), mode="replicate")
        y = self.encoder(x, self.ctx, self.q("q_encoder", qp))
        _, C, H16, W16 = y.shape
        ph, pw = (-H16) % 4, (-W16) % 4
        y_pad = F.pad(y, (0, pw, 0, ph), mode="replicate") if (ph or pw) else y
        z = self.hyper_encoder(y_pad)
        z_hat = torch.clamp(round_half_away(z), -64, 63)
        temporal = self.temporal_prior(self.memory, self.q("q_feature", qp))
        common, q_dec, scales, means = self.entropy_params(z_hat, temporal, H16, W16)
        y = y / q_dec
        reduced = self.conv("y_spatial_prior_reduction.", common)
        so_far = torch.zeros_like(y)
        y_q = torch.zeros_like(y)
        segs = []
        for k in range(4):
            if k > 0:
                scales, means = self.spatial_prior(k, so_far, reduced).chunk(2, 1)
            m = checker_mask(k, C, H16, W16, self.dtype)
            s_hat = scales * m
            m_hat = means * m
            q = round_half_away((y - m_hat) * m) * (s_hat > self.thr).to(self.dtype)
            q = torch.clamp(q, -128, 127)
            y_q = y_q + q
            step = q + m_hat
            if k < 3:
                so_far = so_far + step
            else:
                y_hat = (so_far + step) * q_dec
            s_part = nhwc(quarter_part(scales, m)).numpy()
            q_part = nhwc(quarter_part(q, m)).numpy().astype(np.int64)
            cond = s_part > self.thr
            idx = scale_index(s_part)
            segs.append(((q_part << 8) + idx.astype(np.int64)).astype(np.int16)[cond])
        z_i8 = z_hat[0].permute(1, 2, 0).reshape(-1).numpy().astype(np.int8)
        total = sum(s.size for s in segs)
        ecp = ec_parallel or ec_parallel_for(total)
        data = rans_encode_segments(self.cdf_z, self.len_z, self.cdf_y, self.len_y, segs[::-1],
                                    z_i8, qp * CH_Z, CH_Z, ecp)
        feature = self.decoder(y_hat, self.ctx, self.q("q_decoder", qp))
        if reset_feature_memory:
            self.memory = self.feature_adaptor_i(self.recon_head_reset(feature))
        else:
            self.memory = self.feature_adaptor_m(self.memory, feature)
        self.ctx = self.feature_extractor(self.memory)
        return {"bit_stream": data, "ec_parallel": ecp, "y_q": y_q, "y_hat": y_hat,
                "z_hat": z_hat, "symbols": segs, "feature": feature}

    @torch.no_grad()
    def decompress(self, bit_stream, qp, height, width, ec_parallel, reset_feature_memory):
        Hp, Wp = (height + 15) // 16 * 16, (width + 15) // 16 * 16
        H16, W16 = Hp // 16, Wp // 16
        H64, W64 = (height + 63) // 64, (width + 63) // 64
        if getattr(self, "_memory_ready", False):
            self._memory_ready = False
        elif self.memory_has_value:
            self.memory = self.feature_adaptor_m(self.memory, self.feature_p)
        else:
            self.memory = self.feature_adaptor_i(self.feature_i)
        temporal = self.temporal_prior(self.memory, self.q("q_feature", qp))
        dec = RansSegmentDecoder(self.cdf_z, self.len_z, self.cdf_y, self.len_y, bit_stream,
                                 ec_parallel)
        try:
            z_i8 = dec.decode_z(CH_Z * H64 * W64, qp * CH_Z, CH_Z)
            z_hat = torch.from_numpy(z_i8.astype(np.float64)).to(self.dtype)
            z_hat = z_hat.reshape(H64, W64, CH_Z).permute(2, 0, 1)[None]
            common, q_dec, scales, means = self.entropy_params(z_hat, temporal, H16, W16)
            reduced = self.conv("y_spatial_prior_reduction.", common)
            self.ctx = self.feature_extractor(self.memory)
            C = CH_Y
            so_far = torch.zeros(1, C, H16, W16, dtype=self.dtype)
            y_q = torch.zeros_like(so_far)
            for k in range(4):
                if k > 0:
                    scales, means = self.spatial_prior(k, so_far, reduced).chunk(2, 1)
                m = checker_mask(k, C, H16, W16, self.dtype)
                s_part = nhwc(quarter_part(scales, m)).numpy()
                cond = s_part > self.thr
                vals = dec.decode_y(scale_index(s_part)[cond])
                full = np.zeros(s_part.size, np.float64)
                full[cond] = vals
                part = torch.from_numpy(full).to(self.dtype).reshape(H16, W16, C // 4)
                part = part.permute(2, 0, 1)[None].repeat(1, 4, 1, 1)
                y_q = y_q + part * m
                step = (part + means) * m
                if k < 3:
                    so_far = so_far + step
                else:
                    y_hat = (so_far + step) * q_dec
        finally:
            dec.close()
        feature = self.decoder(y_hat, self.ctx, self.q("q_decoder", qp))
        frames, head7 = self.recon_head(feature)
        self.feature_p = feature
        self.feature_i = head7
        self.memory_has_value = not reset_feature_memory
        return {"x_hat": frames, "y_q": y_q, "y_hat": y_hat, "z_hat": z_hat}
