"""PGA as a device-resident GPU stage (autofocus.pga on CUDA tensors).

* MATLAB semantics (matlab/PGA.m:153-239): one iteration's phase estimate on
  the GPU against the oracle's restatement with PGA.m's 1-based indexing
  written out, even and odd azimuth lengths (1e-5 rad, as the CPU test).
* The reference C++ routine's semantics (src/autofocus/cpu/autofocus_cpu.cpp:
  250-474): several iterations on the GPU against that routine's own compiled
  output (golden fixtures from make_golden.py --pga, and live where
  oracle/_ref/libref_pga.so is present): per-iteration rms and image.
* No host read-back inside the loop: the whole call runs under
  torch.cuda.set_sync_debug_mode("error"), which raises on any operation
  that synchronises with the host.
* A batch of images equals the images one at a time.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def focused():
    sc = S.point_target_scene(K=64, Np=64, n=64, spacing=0.12, nfft=512, snr_db=30.0, seed=12, n_targets=4,
                              extent=5.0)
    return O.focus_fp64(sc)[0].astype(np.complex64)


def defocus(img, seed=0, amp=6.0):
    n = img.shape[-1]
    rng = np.random.default_rng(seed)
    x = np.linspace(-1, 1, n)
    phi = amp * (rng.uniform(0.5, 1.0) * x ** 2 + rng.uniform(-0.5, 0.5) * x ** 3)
    return np.fft.ifft(np.fft.fft(img, axis=-1) * np.exp(1j * phi), axis=-1).astype(np.complex64)


@pytest.mark.parametrize("n", [64, 63])
def test_matlab_semantics_phase_estimate_matches_oracle(torch_cuda, focused, n):
    from uncc_sar_focusing_b200 import autofocus as AF

    torch = torch_cuda
    bad = np.ascontiguousarray(defocus(focused)[:, :n])
    _, phi, _ = AF.pga(torch.as_tensor(bad).cuda(), max_iter=1)
    want = O.pga_step_reference(bad)
    assert np.abs(phi.cpu().numpy() - want).max() < 1e-5


@pytest.mark.parametrize("name", ["pga_cpp_64x64", "pga_cpp_64x63_edges"])
def test_reference_cpp_semantics_matches_the_compiled_routine(torch_cuda, name):
    from uncc_sar_focusing_b200 import autofocus as AF

    torch = torch_cuda
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    iters = int(d["iterations"])
    out, _, rms = AF.pga(torch.as_tensor(d["image"]).cuda(), max_iter=iters, semantics="reference_cpp")
    rms = rms.cpu().numpy()
    ran = rms[np.isfinite(rms)]
    assert len(ran) == len(d["ref_rms"])
    assert np.abs(ran - d["ref_rms"]).max() < 2e-5
    assert O.rel_l2(out.cpu().numpy(), d["ref_out"]) < 1e-4
    if O.ref_pga_available():
        live = O.ref_pga(d["image"], iters)
        assert O.rel_l2(out.cpu().numpy(), live) < 1e-4


@pytest.mark.parametrize("semantics", ["matlab", "reference_cpp"])
def test_pga_loop_never_waits_for_the_host(torch_cuda, focused, semantics):
    from uncc_sar_focusing_b200 import autofocus as AF

    torch = torch_cuda
    imgs = torch.as_tensor(np.stack([defocus(focused, seed=s) for s in range(4)])).cuda()
    AF.pga(imgs, max_iter=2, semantics=semantics)  # warm-up: FFT plans, kernels
    torch.cuda.synchronize()
    torch.cuda.set_sync_debug_mode("error")
    try:
        out, phi, rms = AF.pga(imgs, max_iter=20, semantics=semantics)
    finally:
        torch.cuda.set_sync_debug_mode("default")
    torch.cuda.synchronize()
    assert torch.isfinite(out).all()


@pytest.mark.parametrize("semantics", ["matlab", "reference_cpp"])
def test_batch_equals_single_images(torch_cuda, focused, semantics):
    from uncc_sar_focusing_b200 import autofocus as AF

    torch = torch_cuda
    imgs = torch.as_tensor(np.stack([defocus(focused, seed=s) for s in range(3)])).cuda()
    out_b, phi_b, rms_b = AF.pga(imgs, max_iter=8, semantics=semantics)
    for i in range(3):
        out_1, phi_1, rms_1 = AF.pga(imgs[i], max_iter=8, semantics=semantics)
        assert torch.allclose(out_b[i], out_1, atol=1e-5 * float(out_1.abs().max()))
        assert torch.allclose(phi_b[i], phi_1, atol=1e-9)


def test_matlab_semantics_restores_an_injected_phase_error(torch_cuda, focused):
    from uncc_sar_focusing_b200 import autofocus as AF

    torch = torch_cuda
    good = torch.as_tensor(focused).cuda()
    bad = torch.as_tensor(defocus(focused)).cuda()
    fixed, _, _ = AF.pga(bad, max_iter=30)
    e_good, e_bad, e_fixed = (float(AF.entropy(v)) for v in (good, bad, fixed))
    assert e_fixed < e_good + 0.2 * (e_bad - e_good)
