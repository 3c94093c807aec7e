"""Autofocus building blocks on CPU: PGA restores an injected azimuth phase
error (the reference's own PGA self-test, src/autofocus/cpu/autofocus_cpu.cpp:
547-633, here on an FP64-oracle image), the focus metrics rank a focused image
above a defocused one, and the cubic motion model evaluates its polynomial."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from uncc_sar_focusing_b200 import autofocus as AF
from uncc_sar_focusing_b200 import scenes as S


@pytest.fixture(scope="module")
def focused():
    sc = S.point_target_scene(K=64, Np=64, n=64, spacing=0.12, nfft=512, snr_db=30.0, seed=12, n_targets=4,
                              extent=5.0)
    return torch.as_tensor(O.focus_fp64(sc)[0].astype(np.complex64))


def defocus(img, seed=0, amp=6.0):
    n = img.shape[-1]
    rng = np.random.default_rng(seed)
    x = np.linspace(-1, 1, n)
    phi = amp * (rng.uniform(0.5, 1.0) * x ** 2 + rng.uniform(-0.5, 0.5) * x ** 3)
    X = torch.fft.fft(img, dim=-1) * torch.exp(1j * torch.as_tensor(phi, dtype=torch.float64)).to(torch.complex64)
    return torch.fft.ifft(X, dim=-1)


def test_pga_restores_an_injected_phase_error(focused):
    bad = defocus(focused)
    e_good, e_bad = float(AF.entropy(focused)), float(AF.entropy(bad))
    assert e_bad > e_good + 0.3
    fixed, phi, rms = AF.pga(bad, max_iter=30)
    e_fixed = float(AF.entropy(fixed))
    assert e_fixed < e_good + 0.2 * (e_bad - e_good), (e_good, e_bad, e_fixed)
    assert rms[-1] < rms[0]


@pytest.mark.parametrize("n", [64, 63])
def test_pga_iteration_matches_the_reference_steps(focused, n):
    """One PGA iteration's phase estimate equals an independent numpy
    restatement of matlab/PGA.m:150-212 (1-based indexing written out), on an
    even and an odd azimuth length."""
    bad = defocus(focused)[:, :n].contiguous()
    _, phi, _ = AF.pga(bad, max_iter=1)
    want = O.pga_step_reference(bad.numpy())
    assert np.abs(phi.numpy() - want).max() < 1e-5, np.abs(phi.numpy() - want).max()


def test_focus_metrics_rank_focus(focused):
    bad = defocus(focused, seed=3)
    assert float(AF.entropy(focused)) < float(AF.entropy(bad))
    from uncc_sar_focusing_b200 import autograd as A

    assert float(A.image_sharpness(focused)) < float(A.image_sharpness(bad))
    batch = torch.stack([focused, bad])[:, None]
    e = AF.batch_entropy(batch)
    assert torch.allclose(e, torch.stack([AF.entropy(focused), AF.entropy(bad)]), rtol=1e-5)


def test_cubic_motion_model():
    Np = 33
    base = [torch.linspace(0, 1, Np, dtype=torch.float64) * s for s in (1.0, 2.0, 3.0)]
    m = AF.CubicMotion(*base)
    theta = torch.tensor([[0.1, 0.2, 0.3, 0.4], [0.0, -1.0, 0.0, 0.5], [1.0, 0.0, 0.0, 0.0]], dtype=torch.float64)
    tau = np.linspace(-1, 1, Np)
    want = np.stack([b.numpy() for b in base]) + S.cubic_track_error(theta.numpy(), tau)
    assert np.allclose(m.track(theta).numpy(), want, atol=1e-12)


def test_motion_error_scene_respects_the_peak():
    sc = S.motion_error_scene(K=16, Np=64, n=8, peak=1.5, walk_sigma=0.0, seed=3)
    cub = S.cubic_track_error(sc.true_cubic, S.slow_time(64))
    assert np.allclose(np.abs(cub).max(axis=1), 1.5)
    assert np.allclose(sc.true_error, cub)


def test_reference_dft_cost_matches_the_reference_loops():
    # direct transcription of dft2DCalculation's loops (sincospif DFT, corner test, mirrored rows)
    rng = np.random.default_rng(1)
    img = torch.as_tensor((rng.standard_normal((12, 10)) + 1j * rng.standard_normal((12, 10))).astype(np.complex64))
    u8 = AF.reference_u8_image(img).numpy().astype(np.float64)
    nx, ny = u8.shape
    out = 0.0
    hh, hw = ny // 2, nx // 2
    threshold = int((hh * hh + hw * hw) * (0.35 * 0.35))
    for dft_x in range(nx):
        d1 = [sum(u8[x, yy] * np.exp(-2j * np.pi * dft_x * x / nx) for x in range(nx)) for yy in range(ny)]
        d2 = [sum(np.exp(-2j * np.pi * dy * yy / ny) * d1[yy] for yy in range(ny)) for dy in range(ny)]
        for y in range(hh):
            r = dft_x * dft_x + y * y
            r2 = (nx - dft_x - 1) ** 2 + y * y
            if r < threshold or r2 < threshold:
                out += abs(d2[y]) + abs(d2[ny - y - 1])
    assert abs(AF.reference_dft_cost(img) - (-out)) < 1e-6 * abs(out)
