"""Range tapers and caller-supplied range weights through the C ABI.

The plan's per-sample factor (taper x 1/nfft x fftshift twiddle) is built on
the host and applied by the range-compression kernels, so every taper and any
caller vector costs nothing per sample.  Each is checked here against the FP64
oracle's range compression on both range-compression paths (the fused kernel,
nfft = R K with K in {256, 512, 1024}, and taper / cuFFT / pair rows for other
shapes, e.g. the point-target configuration's K = 424, nfft = 3392) and in
both precisions.  Tolerances as the other range-compression parity tests:
2e-6 (mixed), 1e-13 (FP64) relative L2.
"""
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu
TOL = {"mixed": 2e-6, "fp64": 1e-13}


@pytest.fixture(scope="module")
def F():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from uncc_sar_focusing_b200 import focusing

    return focusing


def scene(K, nfft, window):
    sc = S.point_target_scene(K=K, Np=20, n=32, spacing=0.2, nfft=nfft, snr_db=20.0, seed=9, n_targets=3,
                              extent=5.0)
    sc.window = window
    return sc


SHAPES = [(256, 2048, True), (424, 3392, False)]


@pytest.mark.parametrize("window", ["taylor", "hamming", "none"])
@pytest.mark.parametrize("K,nfft,fused", SHAPES)
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_window_matches_oracle(F, window, K, nfft, fused, precision):
    sc = scene(K, nfft, window)
    want = O.range_compress_fp64(sc.phase_history, nfft, O.window_for(window, K))
    with F.Plan.for_scene(sc, precision) as plan:
        assert plan.info["fused_range_compression"] == int(fused and precision == "mixed")
        plan.range_compress(sc.phase_history)
        got = plan.range_profiles()
    assert O.rel_l2(got, want) < TOL[precision]


def caller_weights(K):
    """A Taylor taper times a range reference function (a linear-FM
    deramp), as a caller matching in range would pass it."""
    k = np.arange(K)
    return O.taylor(K) * np.exp(1j * np.pi * 0.37 * (k - K / 2) ** 2 / K)


@pytest.mark.parametrize("K,nfft,fused", SHAPES)
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_caller_weights_match_oracle_and_reset(F, K, nfft, fused, precision):
    sc = scene(K, nfft, "hamming")
    w = caller_weights(K)
    want = O.range_compress_fp64(sc.phase_history, nfft, w)
    want_hamming = O.range_compress_fp64(sc.phase_history, nfft, O.hamming(K))
    with F.Plan.for_scene(sc, precision) as plan:
        plan.set_range_weights(w)
        plan.range_compress(sc.phase_history)
        got = plan.range_profiles()
        plan.set_range_weights(None)  # back to the plan's Hamming taper
        plan.range_compress(sc.phase_history)
        back = plan.range_profiles()
    assert O.rel_l2(got, want) < TOL[precision]
    assert O.rel_l2(back, want_hamming) < TOL[precision]


def test_caller_weights_reach_the_matched_filter(F):
    sc = S.point_target_scene(K=32, Np=12, n=12, spacing=0.25, nfft=256, snr_db=None, seed=10, n_targets=2,
                              extent=2.0)
    sc.window = "none"
    w = caller_weights(sc.num_range_samples)
    weighted = sc.phase_history.astype(np.complex128) * w[None, :]
    want = O.mf_fp64(dataclasses.replace(sc, phase_history=weighted))
    with F.Plan.for_scene(sc, "fp64") as plan:
        plan.set_range_weights(w)
        got = plan.matched_filter(sc.phase_history, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)
    assert O.rel_l2(got, want) < 1e-9


def test_rejects_non_finite_weights(F):
    sc = scene(256, 2048, "hamming")
    w = caller_weights(256)
    w[7] = np.nan
    with F.Plan.for_scene(sc, "mixed") as plan:
        with pytest.raises(Exception):
            plan.set_range_weights(w)
