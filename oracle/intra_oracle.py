"""ORACLE (test infrastructure only; never imported by the product).

CPU restatement of the reference's intra (DMCI) codec as its CUDA proxy runs it
(src/layers/extensions/inference/dmci_proxy.cpp:296-602 compress / decompress, :804-880 the
entropy worker), written with plain PyTorch CPU ops in float64 or float32, reading the weights
from a state dict.  Used by tests/ (PSNR / bpp / symbol agreement against the GPU path); the
sub-networks are pinned against the reference nn.Modules by tests/golden/intra_modules_golden.npz
and the coder by tests/golden/rans_segments_golden.npz.

Network math follows src/models/image_model.py (IntraEncoder :50-69, IntraHyperEncoder :85-95,
IntraHyperDecoder :72-82, IntraYPriorFusion :112-123, IntraSpatialPrior :98-109, IntraDecoder
:21-47) on the layers of src/layers/layers.py, with the resampling blocks' default shortcut
(layers.py:162-188).  The proxy-only steps: the decoder output is clamped to [-0.5, 0.5]
(dmci_proxy.cpp:30, pixel_shuffle_8 with clamp); the latent is scaled by q_scale_y_enc before
the 4-step coding and the reconstruction by q_scale_y_dec after it (dmci_proxy.cpp:326,
392-393); every step quantises one quarter of the channels per 2x2 position with the skip
threshold and clamp [-128, 127] (stream.cu:548-683), takes the scales and means of steps 1-3
from the spatial prior over cat(y_hat so far, reduced params) (dmci_proxy.cpp:343-393), and
codes the step's quarter-channel part in NHWC order (single_part_for_writing_4x, stream.cu:
931-962; build_index_enc, stream.cu:126-173); the payload holds the steps' symbols in the
order 3, 2, 1, 0 and then z (dmci_proxy.cpp:818-846).
"""
import numpy as np
import torch
import torch.nn.functional as F

from hts_oracle import (HtsOracle, RansSegmentDecoder, checker_mask, ec_parallel_for,
                        rans_encode_segments, round_half_away, scale_index)

CH_Y, CH_Z = 256, 128


def quarter_part(t, mask):
    """The active quarter of each 2x2 position: [1, C, H, W] -> [C/4, H, W]."""
    C = t.shape[1]
    return (t * mask)[0].reshape(4, C // 4, *t.shape[2:]).sum(0)


def nhwc(t):
    return t.permute(1, 2, 0).reshape(-1)


class IntraOracle(HtsOracle):
    """The intra codec on the CPU.  `sd`: DMCI state dict plus the four CDF entries."""

    # ---- sub-networks (image_model.py)
    def encoder(self, x, q_enc):
        f = self.dcb("enc.enc_1.", F.pixel_unshuffle(x, 8), q_enc)
        f = self.seq("enc.enc_2.", 6, f)
        return self.conv("enc.enc_2.6.", f, stride=2, padding=1)

    def hyper_encoder(self, y):
        z = self.dcb("hyper_enc.conv.0.", y)
        z = self.rb_down("hyper_enc.conv.1.", z, shortcut=True)
        return self.rb_down("hyper_enc.conv.2.", z, shortcut=True)

    def hyper_decoder(self, z_hat):
        h = self.rb_up("hyper_dec.conv.0.", z_hat, shortcut=True)
        h = self.rb_up("hyper_dec.conv.1.", h, shortcut=True)
        return self.dcb("hyper_dec.conv.2.", h)

    def prior_fusion(self, h):
        return self.conv("y_prior_fusion.conv.3.", self.seq("y_prior_fusion.conv.", 3, h))

    def spatial_prior(self, k, y_hat, reduced):
        x = self.dcb(f"y_spatial_prior_adaptor_{k}.", torch.cat((y_hat, reduced), dim=1))
        x = self.seq("y_spatial_prior.conv.", 3, x)
        return self.conv("y_spatial_prior.conv.3.", x)

    def decoder_features(self, y_hat, q_dec):
        """IntraDecoder.forward up to and including pixel_shuffle (no clamp)."""
        out = self.rb_up("dec.dec_1.0.", y_hat, shortcut=True)
        out = self.seq("dec.dec_1.", 13, out, q_dec, start=1)
        return F.pixel_shuffle(self.dcb("dec.dec_2.", out), 8)

    def decoder(self, y_hat, q_dec):
        return torch.clamp(self.decoder_features(y_hat, q_dec), -0.5, 0.5)

    def seq(self, prefix, n, x, quant=None, start=0):
        for i in range(start, n):
            x = self.dcb(f"{prefix}{i}.", x, quant if i == n - 1 else None)
        return x

    def entropy_params(self, z_hat, H16, W16):
        params = self.prior_fusion(self.hyper_decoder(z_hat))[:, :, :H16, :W16]
        scales, means = params.chunk(2, 1)
        return params, scales, means

    # ---- public API mirroring DMCIProxy
    @torch.no_grad()
    def compress(self, x, qp, padding_b, padding_r, ec_parallel=None):
        x = F.pad(x.to("cpu", self.dtype), (0, padding_r, 0, padding_b), mode="replicate")
        y = self.encoder(x, self.q("q_scale_enc", qp))
        _, C, H16, W16 = y.shape
        ph, pw = (-H16) % 4, (-W16) % 4
        y_pad = F.pad(y, (0, pw, 0, ph), mode="replicate") if (ph or pw) else y
        z = self.hyper_encoder(y_pad)
        z_hat = torch.clamp(round_half_away(z), -64, 63)
        params, scales, means = self.entropy_params(z_hat, H16, W16)
        y = y * self.q("q_scale_y_enc", qp)
        reduced = self.conv("y_spatial_prior_reduction.", params)
        so_far = torch.zeros_like(y)
        y_q = torch.zeros_like(y)
        segs, conds, idxs = [], [], []
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
                y_hat = (so_far + step) * self.q("q_scale_y_dec", qp)
            s_part = nhwc(quarter_part(scales, m)).numpy()
            q_part = nhwc(quarter_part(q, m)).numpy().astype(np.int64)
            cond = s_part > self.thr
            idx = scale_index(s_part)
            segs.append(((q_part << 8) + idx.astype(np.int64)).astype(np.int16)[cond])
            conds.append(cond)
            idxs.append(idx)
        z_i8 = z_hat[0].permute(1, 2, 0).reshape(-1).numpy().astype(np.int8)
        total = sum(s.size for s in segs)
        ecp = ec_parallel or ec_parallel_for(total)
        data = rans_encode_segments(self.cdf_z, self.len_z, self.cdf_y, self.len_y, segs[::-1],
                                    z_i8, qp * CH_Z, CH_Z, ecp)
        x_hat = self.decoder(y_hat, self.q("q_scale_dec", qp))
        return {"bit_stream": data, "ec_parallel": ecp, "x_hat": x_hat, "y_q": y_q,
                "y_hat": y_hat, "z_hat": z_hat, "symbols": segs, "cond": conds, "idx": idxs}

    @torch.no_grad()
    def decompress(self, bit_stream, qp, height, width, ec_parallel):
        Hp, Wp = (height + 15) // 16 * 16, (width + 15) // 16 * 16
        H16, W16 = Hp // 16, Wp // 16
        H64, W64 = (height + 63) // 64, (width + 63) // 64
        dec = RansSegmentDecoder(self.cdf_z, self.len_z, self.cdf_y, self.len_y, bit_stream,
                                 ec_parallel)
        try:
            z_i8 = dec.decode_z(CH_Z * H64 * W64, qp * CH_Z, CH_Z)
            z_hat = torch.from_numpy(z_i8.astype(np.float64)).to(self.dtype)
            z_hat = z_hat.reshape(H64, W64, CH_Z).permute(2, 0, 1)[None]
            params, scales, means = self.entropy_params(z_hat, H16, W16)
            reduced = self.conv("y_spatial_prior_reduction.", params)
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
                    y_hat = (so_far + step) * self.q("q_scale_y_dec", qp)
        finally:
            dec.close()
        x_hat = self.decoder(y_hat, self.q("q_scale_dec", qp))
        return {"x_hat": x_hat, "y_q": y_q, "y_hat": y_hat, "z_hat": z_hat}
