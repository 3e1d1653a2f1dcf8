"""Precision form on the CPU: storage of the micro-image texels, and the FP32
NCC error of the reference's raw moments and of shifted moments against an
FP64 evaluation of the same taps and samples (the oracle in both FP32 modes is
what the device computes bit for bit; the FP64 side takes the FP32 path's
sample points, so only the accumulation differs)."""
import numpy as np
import pytest
import torch

from scenes import random_hypotheses


def test_eight_bit_texels_are_exact_in_fp16_and_bf16():
    """The raw frame is 8-bit: every texel value 0..255 is exact in FP16 (11-bit
    significand) and in BF16 (8-bit significand, integers up to 256), so holding
    the texels in either format computes exactly what the 8-bit tiles compute.
    The device keeps them as 8-bit tiles: one byte per texel, half of FP16's
    gather bytes and a quarter of the reference's float textures."""
    v = torch.arange(256, dtype=torch.float32)
    assert torch.equal(v.to(torch.float16).to(torch.float32), v)
    assert torch.equal(v.to(torch.bfloat16).to(torch.float32), v)
    # and the bilinear samples of 8-bit texels (multiples of 1/256 below 256)
    # need 16 fraction bits: FP16/BF16 texel storage must not hold samples
    s = torch.tensor([255.0 + 255.0 / 256.0], dtype=torch.float32)
    assert s.to(torch.float16).item() != s.item() and s.to(torch.bfloat16).item() != s.item()


def _errors(oracle, pfd, shifted):
    w = pfd.make_workload(300, 220, 23.2, 6, seed=9, max_nb=8)
    P = pfd.PmParams(base=23.2, patch_size=15, sigma_spatial=3.0, sigma_color=12.0)
    rs = np.random.RandomState(3)
    vids, pxy, planes = random_hypotheses(rs, w.centers.shape[0], w.mi, 4000, 23.2 / 2)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, shifted=shifted)
    c32, _ = orc.cost_vectors(P, vids, pxy, planes)
    c64 = orc.ncc_fp64_batch(P, vids, pxy, planes, sampling=2)
    both = (c32 < 2) & (c64 < 2)
    return np.abs(c32.astype(np.float64) - c64)[both]


def test_shifted_moments_cut_the_fp32_error(pfd, oracle):
    ref = _errors(oracle, pfd, False)
    sh = _errors(oracle, pfd, True)
    assert ref.size > 2000 and sh.size == ref.size
    assert np.median(sh) < np.median(ref) / 10
    assert np.percentile(sh, 99) < 1e-5
    assert np.mean(sh <= 1e-5) > 0.995
    assert np.mean(ref <= 1e-5) < 0.9          # the raw moments do lose digits
