"""CDF tables of the entropy models, built as the reference's update() builds them.

Restates GaussianEncoder.update and BitEstimator.update (src/models/entropy_models.py:114-217)
with the same FP32 torch operations in the same order, and quantises each pmf with this
package's pmf_to_quantized_cdf (the C++ port of py_rans.cpp:35-94) unless the caller passes
another quantiser with the same contract (list of floats -> list of ints).  The resulting int32
tables equal the reference model's `gaussian_encoder` / `bit_estimator_z` CDF info bit for bit.
The native library is loaded only when the default quantiser is used.
"""
import math

import torch
import torch.nn.functional as F

MAX_ENTROPY_CODING_VALUE = 8
SCALE_MIN, SCALE_MAX, SCALE_LEVEL = 0.11, 16.0, 128


def _reorder_prob(prob):
    """0, +1, -1, +2, -2, ... order, tail mass last (entropy_models.py:46-57)."""
    length = prob.size(0)
    out = prob.clone()
    center = (length - 1) // 2
    out[0] = prob[center]
    for i in range(1, center + 1):
        out[2 * i - 1] = prob[center + i]
        out[2 * i - 0] = prob[center - i]
    return out


def _default_quantizer():
    from .MLCodec_extensions_cpp import pmf_to_quantized_cdf
    return pmf_to_quantized_cdf


def _pmf_to_cdf(pmf, tail_mass, pmf_length, max_length, quantize=None):
    quantize = quantize or _default_quantizer()
    cdf = torch.zeros((len(pmf_length), max_length + 2), dtype=torch.int32)
    for i, p in enumerate(pmf):
        prob = torch.cat((p[: pmf_length[i]], tail_mass[i]), dim=0)
        q = quantize(_reorder_prob(prob).tolist())
        q = torch.IntTensor(q)
        cdf[i, : q.size(0)] = q
    return cdf


def gaussian_tables(quantize=None):
    """(quantized_cdf [128, 19] int32, cdf_length [128] int32) of the Gaussian scale tables."""
    scale_table = torch.exp(torch.linspace(math.log(SCALE_MIN), math.log(SCALE_MAX), SCALE_LEVEL))
    zeros = torch.zeros_like(scale_table)
    sym_range = zeros + MAX_ENTROPY_CODING_VALUE
    dist = torch.distributions.normal.Normal(0., scale_table)
    for i in range(MAX_ENTROPY_CODING_VALUE, 1, -1):
        probs = torch.squeeze(dist.cdf(zeros + i))
        sym_range = torch.where(probs > 0.999, i, sym_range)
    sym_range = sym_range.int()
    pmf_length = 2 * sym_range + 1
    max_length = 2 * MAX_ENTROPY_CODING_VALUE + 1
    samples = (torch.arange(max_length, device=sym_range.device) - sym_range[:, None]).float()
    dist = torch.distributions.normal.Normal(0., scale_table[:, None])
    upper = dist.cdf(samples + 0.5)
    lower = dist.cdf(samples - 0.5)
    pmf = upper - lower
    tail_mass = 2 * lower[:, :1]
    cdf = _pmf_to_cdf(pmf, tail_mass, pmf_length, max_length, quantize)
    return cdf.numpy(), (pmf_length + 2).reshape(-1).int().numpy()


def _bit_estimator_prob(x, h, b, a):
    # layers.py:13-19
    for i in range(4):
        x = x * F.softplus(h[:, :, i:i + 1, None]) + b[:, :, i:i + 1, None]
        if i != 3:
            x = x + torch.tanh(x) * torch.tanh(a[:, :, i:i + 1, None])
    return torch.sigmoid(x)


@torch.inference_mode()
def bit_estimator_tables(h, b, a, quantize=None):
    """(quantized_cdf [qp_num * ch, 19], cdf_length [qp_num * ch]) from the bit estimator
    parameters h, b [qp, ch, 4] and a [qp, ch, 3] (FP32, as BitEstimator.update runs them)."""
    h, b, a = h.float().cpu(), b.float().cpu(), a.float().cpu()
    qp_num, channel = h.shape[0], h.shape[1]
    index = torch.arange(qp_num, dtype=torch.int32)
    hs, bs, as_ = (torch.index_select(t, 0, index) for t in (h, b, a))
    fwd = lambda x: _bit_estimator_prob(x, hs, bs, as_)  # noqa: E731
    zeros = torch.zeros((qp_num, channel, 1, 1))
    sym_range = zeros + MAX_ENTROPY_CODING_VALUE
    for i in range(MAX_ENTROPY_CODING_VALUE, 1, -1):
        neg = fwd(zeros - i)
        pos = fwd(zeros + i)
        sym_range = torch.where(torch.logical_and(neg < 0.001, pos > 0.999), i, sym_range)
    sym_range = sym_range.int()
    pmf_length = sym_range * 2 + 1
    max_length = MAX_ENTROPY_CODING_VALUE * 2 + 1
    samples = torch.arange(max_length)[None, None, None, :] - sym_range
    lower = fwd(samples - 0.5)
    upper = fwd(samples + 0.5)
    pmf = (upper - lower)[:, :, 0, :]
    upper = fwd(sym_range.float())
    tail_mass = lower[:, :, 0, :1] + (1.0 - upper[:, :, 0, -1:])
    pmf = pmf.reshape([-1, max_length])
    tail_mass = tail_mass.reshape([-1, 1])
    pmf_length = pmf_length.reshape([-1])
    cdf = _pmf_to_cdf(pmf, tail_mass, pmf_length, max_length, quantize)
    return cdf.numpy(), (pmf_length + 2).reshape(-1).int().numpy()


def add_cdf_to_state_dict(state_dict, quantize=None):
    """Adds the four CDF entries the proxies read (common_model.py:64-70)."""
    qy, ly = gaussian_tables(quantize)
    qz, lz = bit_estimator_tables(state_dict["bit_estimator_z.h"], state_dict["bit_estimator_z.b"],
                                  state_dict["bit_estimator_z.a"], quantize)
    out = dict(state_dict)
    out["gaussian_encoder.quantized_cdf"] = torch.from_numpy(qy)
    out["gaussian_encoder.cdf_length"] = torch.from_numpy(ly)
    out["bit_estimator_z.quantized_cdf"] = torch.from_numpy(qz)
    out["bit_estimator_z.cdf_length"] = torch.from_numpy(lz)
    return out
