"""Polar-format preparation (focusing.polar_format_phase_history) against a
per-pulse restatement of the reference's MATLAB lines
(matlab/focusalg_PF.m:33-35, matlab/formSARImage.m:217-220,341)."""
import math

import numpy as np

from uncc_sar_focusing_b200 import focusing as F


def reference_modulation(ph, chirp_deg, adf, center_deg):
    # formSARImage.m: Ts0 = 1/ADF; chirpRates_rad = ChirpRate*pi/180;
    # centerFreq_rad = DesCntrFreq*pi/180; freq_scales per pulse;
    # focusalg_PF.m: phdata(:, p) .* exp((-2j*pi/numPulses) * freq_scales)
    Np, K = ph.shape
    out = np.empty_like(ph, dtype=np.complex128)
    ts0 = 1.0 / adf
    center_rad = center_deg * math.pi / 180.0
    for p in range(Np):
        chirp_rad = chirp_deg[p] * math.pi / 180.0
        scales = 1.0 + (chirp_rad * ts0 / center_rad) * np.linspace(-K / 2, K / 2 - 1, K)
        out[p] = ph[p] * np.exp((-2j * math.pi / Np) * scales)
    return out


def test_polar_format_modulation_matches_the_reference_lines():
    rng = np.random.default_rng(0)
    Np, K = 37, 64
    ph = (rng.standard_normal((Np, K)) + 1j * rng.standard_normal((Np, K))).astype(np.complex64)
    chirp = rng.uniform(1e12, 3e12, Np)
    adf, center = 5e7, 9.6e9
    got = F.polar_format_phase_history(ph, chirp, adf, center)
    want = reference_modulation(ph.astype(np.complex128), chirp, adf, center)
    assert got.dtype == np.complex64 and got.shape == ph.shape
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()


def test_polar_format_accepts_torch_and_a_single_rate():
    import torch

    rng = np.random.default_rng(1)
    ph = (rng.standard_normal((8, 16)) + 1j * rng.standard_normal((8, 16))).astype(np.complex64)
    a = F.polar_format_phase_history(ph, 2e12, 5e7, 9.6e9)
    b = F.polar_format_phase_history(torch.as_tensor(ph), 2e12, 5e7, 9.6e9)
    assert isinstance(b, torch.Tensor) and b.dtype == torch.complex64
    assert np.allclose(a, b.numpy(), rtol=1e-6, atol=1e-6)
