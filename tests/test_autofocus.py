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
    ran = rms[torch.isfinite(rms)]
    assert ran[-1] < ran[0]


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


PGA_GOLDEN = ["pga_cpp_64x64", "pga_cpp_64x63_edges"]


def load_pga_golden(name):
    import os

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    return d["image"], int(d["iterations"]), d["ref_out"], d["ref_rms"]


@pytest.mark.parametrize("name", PGA_GOLDEN)
def test_pga_cpp_restatement_pinned_to_reference_golden(name):
    """The oracle's restatement of the reference's C++ PGA routine
    (autofocus_cpu.cpp:250-474) against that routine's own compiled output
    (tests/golden, written by make_golden.py --pga): per-iteration rms to the
    6 decimals the routine prints, image to float rounding."""
    img, iters, ref_out, ref_rms = load_pga_golden(name)
    out, _, rms = O.pga_cpp_reference(img, iters)
    assert len(rms) == len(ref_rms)
    assert np.abs(np.asarray(rms) - ref_rms).max() < 2e-6
    assert O.rel_l2(out, ref_out) < 1e-5


@pytest.mark.skipif(not O.ref_pga_available(), reason="oracle/_ref/libref_pga.so not built")
def test_pga_cpp_restatement_matches_compiled_reference_live(focused):
    bad = defocus(focused, seed=5).numpy()
    out_ref = O.ref_pga(bad, 3)
    out, _, _ = O.pga_cpp_reference(bad, 3)
    assert O.rel_l2(out, out_ref) < 1e-5


@pytest.mark.parametrize("name", PGA_GOLDEN)
def test_pga_reference_cpp_semantics_matches_reference_golden(name):
    img, iters, ref_out, ref_rms = load_pga_golden(name)
    out, _, rms = AF.pga(torch.as_tensor(img), max_iter=iters, semantics="reference_cpp")
    ran = rms[torch.isfinite(rms)].numpy()
    assert len(ran) == len(ref_rms)
    assert np.abs(ran - ref_rms).max() < 2e-5
    assert O.rel_l2(out.numpy(), ref_out) < 1e-4


def test_pga_batches_equal_single_images(focused):
    imgs = torch.stack([defocus(focused, seed=s) for s in range(3)])
    for sem in ("matlab", "reference_cpp"):
        out_b, phi_b, rms_b = AF.pga(imgs, max_iter=6, semantics=sem)
        for i in range(3):
            out_1, phi_1, rms_1 = AF.pga(imgs[i], max_iter=6, semantics=sem)
            assert torch.allclose(out_b[i], out_1, atol=1e-5 * float(out_1.abs().max()))
            assert torch.allclose(phi_b[i], phi_1, atol=1e-9)


def test_unwrap_matches_numpy():
    rng = np.random.default_rng(4)
    p = np.cumsum(rng.uniform(-5, 5, (3, 50)), axis=1)
    p[1, 7] = p[1, 6] + np.pi  # an exact +pi jump is kept
    assert np.allclose(AF._unwrap(torch.as_tensor(p)).numpy(), np.unwrap(p), atol=1e-12)


def column_entropy_transcription(img: np.ndarray, dyn: float = 70.0) -> float:
    """cuCalculateColumnEntropy (gridSearchErrorFunctions.cuh:341-447) as its
    loops read: one 'column' per x index (the x-major image's ny pixels), the
    8-bit dB pixels against the image maximum, a 256-bin histogram, H_x =
    -sum p log2 p, cost sum_x (100 if H_x == 0 else -H_x) / width."""
    nx, ny = img.shape
    mag = np.abs(img).astype(np.float32)
    max_val = mag.max()
    total = 0.0
    for x in range(nx):
        hist = [0] * 256
        for y in range(ny):
            with np.errstate(divide="ignore"):  # log10(0) = -inf maps to pixel 0, as on the device
                pixelf = np.float32(255.0 / dyn) * (np.float32(20.0) * np.log10(mag[x, y] / max_val)
                                                    + np.float32(dyn))
            hist[0 if pixelf < 0 else int(pixelf)] += 1
        h = 0.0
        for c in hist:
            if c:
                p = c / ny
                h -= p * np.log2(p)
        total += 100.0 if h == 0.0 else -h
    return total / nx


def test_reference_column_entropy_matches_the_reference_loops():
    rng = np.random.default_rng(2)
    imgs = (rng.standard_normal((3, 9, 14)) + 1j * rng.standard_normal((3, 9, 14))).astype(np.complex64)
    imgs[1, 4, :] = 0.0  # an all-zero line: H_x = 0, the routine's +100 penalty
    got = AF.reference_column_entropies(torch.as_tensor(imgs)).numpy()
    want = [column_entropy_transcription(im) for im in imgs]
    assert np.allclose(got, want, rtol=0, atol=1e-9), (got, want)


def test_reference_dft_costs_batch_equals_single():
    rng = np.random.default_rng(6)
    imgs = torch.as_tensor((rng.standard_normal((4, 12, 10)) + 1j * rng.standard_normal((4, 12, 10))).astype(
        np.complex64))
    batch = AF.reference_dft_costs(imgs)
    for i in range(4):
        assert abs(float(batch[i]) - AF.reference_dft_cost(imgs[i])) < 1e-9 * abs(float(batch[i]))


def test_autofocus_state_round_trips_through_npz(tmp_path):
    rng = np.random.default_rng(3)
    st = AF.AutofocusState(theta=rng.standard_normal((3, 4)), exp_avg=rng.standard_normal((3, 4)),
                           exp_avg_sq=rng.random((3, 4)), step=17.0, iters_done=17, total_iters=300, lr=0.02)
    path = str(tmp_path / "state.npz")
    st.save(path)
    back = AF.AutofocusState.load(path)
    for name in ("theta", "exp_avg", "exp_avg_sq"):
        assert np.array_equal(getattr(back, name), getattr(st, name))
    assert (back.step, back.iters_done, back.total_iters, back.lr) == (17.0, 17, 300, 0.02)
