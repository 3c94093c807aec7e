"""The reference-facing shim: cuda_focus_SAR_image<float,float> and
<double,double> exported by libsarbp_compat.so, called exactly as the
reference's MATLAB front-end calls it (tests/native/compat_probe.cpp,
compiled against the reference's headers), checked against the FP64 oracle.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu
PROBE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native", "_build", "libcompat_probe.so")


@pytest.fixture(scope="module")
def probe():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(PROBE):
        pytest.skip("compat probe not built (needs the reference headers at build time)")
    L = ctypes.CDLL(PROBE)
    for name, t in (("compat_focus_f32", np.float32), ("compat_focus_f64", np.float64)):
        p = np.ctypeslib.ndpointer(dtype=t, flags="C_CONTIGUOUS")
        sc = ctypes.c_float if t == np.float32 else ctypes.c_double
        getattr(L, name).argtypes = ([ctypes.c_int, ctypes.c_int] + [p] * 6 + [ctypes.c_int] * 3 + [sc] * 4 + [p, p])
        getattr(L, name).restype = ctypes.c_int
    return L


def run(probe, sc, dtype):
    K, Np = sc.num_range_samples, sc.num_pulses
    freq = (sc.start_freq[0] + np.arange(K) * sc.delta_freq).astype(dtype)
    ph = np.ascontiguousarray(sc.phase_history.astype(np.complex64 if dtype == np.float32 else np.complex128))
    geo = [np.ascontiguousarray(v, dtype=dtype) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range)]
    g = sc.grid
    img = np.zeros((g.nx, g.ny), dtype=np.complex64 if dtype == np.float32 else np.complex128)
    mw = np.zeros(1, dtype=dtype)
    fn = probe.compat_focus_f32 if dtype == np.float32 else probe.compat_focus_f64
    assert fn(K, Np, ph.view(dtype).reshape(-1), freq, *geo, sc.nfft, g.nx, g.ny, g.x0, g.y0, g.wx, g.wy,
              img.view(dtype).reshape(-1), mw) == 0
    return img, float(mw[0])


@pytest.mark.parametrize("nfft_factor", [1, 4])
def test_reference_symbols_focus_like_the_oracle(probe, nfft_factor):
    sc = S.point_target_scene(K=64, Np=48, n=40, spacing=0.2, nfft=64 * nfft_factor, snr_db=20.0, seed=21,
                              n_targets=4, extent=6.0)
    sc.window = "none"  # the reference applies no taper
    for dtype, tol in ((np.float32, 1e-4), (np.float64, 1e-9)):
        img, max_wy = run(probe, sc, dtype)
        assert abs(max_wy - sc.max_wr) < 1e-3 * sc.max_wr
        # the same inputs the caller handed over: SAR_Aperture<T> holds positions,
        # slant range and frequencies as T, and max_Wy_m comes from its statistics
        geo = [np.asarray(v, dtype=dtype).astype(np.float64) for v in (sc.ant_x, sc.ant_y, sc.ant_z,
                                                                         sc.slant_range)]
        f0 = np.full(sc.num_pulses, float(dtype(sc.start_freq[0])))
        want = O.bp_fp64(O.range_compress_fp64(sc.phase_history, sc.nfft, None), *geo, f0, max_wy, sc.grid)[0]
        assert O.rel_l2(img, want) < tol, (dtype, O.rel_l2(img, want))


def test_repeated_calls_reuse_the_plan_and_agree(probe):
    sc = S.point_target_scene(K=32, Np=24, n=24, spacing=0.3, nfft=128, snr_db=None, seed=2, n_targets=2)
    sc.window = "none"
    a, _ = run(probe, sc, np.float32)
    b, _ = run(probe, sc, np.float32)
    assert np.array_equal(a, b)
