"""The reference's raw-array callback API (include/charlotte_sar_api.hpp:
sph_sar_data_callback_gpu<float>, :261-316) running unchanged on top of the
engine: tests/native/callback_probe.cpp calls it with Sandia-style arrays; the
header's own code derives the frequencies (StartF + k ChirpRate / ADF), picks
the full-scene grid and calls cuda_focus_SAR_image, which libsarbp_compat.so
provides, then writes an 8-bit BMP.  The BMP must equal the image the engine
forms through its own API from the same arrays and the same float-rounded
aperture parameters the header computes, mapped to 8 bits as writeBMPFile
does (uncc_sar_globals.hpp:66-117): at most 1% of pixels off, by one level.
"""
import ctypes
import os

import numpy as np
import pytest

from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu

PROBE = os.path.join(os.path.dirname(__file__), "native", "_build", "libcallback_probe.so")
CLIGHT = 299792458.0


@pytest.fixture(scope="module")
def F():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(PROBE):
        pytest.skip("callback probe not built (needs the reference headers at build time)")
    from uncc_sar_focusing_b200 import focusing

    return focusing


def read_bmp(path):
    b = open(path, "rb").read()
    assert b[:2] == b"BM"
    off = int.from_bytes(b[10:14], "little")
    w = int.from_bytes(b[18:22], "little")
    h = int.from_bytes(b[22:26], "little")
    assert int.from_bytes(b[28:30], "little") == 24
    stride = (3 * w + 3) // 4 * 4
    rows = [np.frombuffer(b, np.uint8, 3 * w, off + r * stride)[::3] for r in range(h)]
    return np.stack(rows[::-1])  # stored bottom-up: row r of the file is image row h - 1 - r


def test_sph_callback_runs_unchanged_on_the_engine(F, tmp_path):
    import torch

    from uncc_sar_focusing_b200 import autofocus as AF

    sc = S.point_target_scene(K=64, Np=48, n=40, spacing=0.2, snr_db=20.0, seed=3, n_targets=4, extent=6.0)
    K, Np = sc.num_range_samples, sc.num_pulses
    adf = np.float32(2.0e6)
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    samples = f32(sc.phase_history.view(np.float32))  # interleaved re, im, K per pulse
    start, chirp = f32(sc.start_freq), f32(np.full(Np, sc.delta_freq * float(adf)))
    x, y, z = f32(sc.ant_x), f32(sc.ant_y), f32(sc.ant_z)

    L = ctypes.CDLL(PROBE)
    P = ctypes.POINTER(ctypes.c_float)
    L.probe_callback_grid.argtypes = [ctypes.c_float, P, ctypes.c_int, P, P, P, P, P, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    L.probe_callback_gpu.argtypes = [ctypes.c_char_p, ctypes.c_float, P, ctypes.c_int, P, P, P, P, P, ctypes.c_int]
    p = lambda a: a.ctypes.data_as(P)  # noqa: E731
    dims, geom = (ctypes.c_int * 3)(), (ctypes.c_double * 5)()
    assert L.probe_callback_grid(adf, p(samples), K, p(start), p(chirp), p(x), p(y), p(z), Np, dims, geom) == 0
    nx, ny, nfft = dims
    bmp = str(tmp_path / "callback.bmp")
    assert L.probe_callback_gpu(bmp.encode(), adf, p(samples), K, p(start), p(chirp), p(x), p(y), p(z), Np) == 0
    got = read_bmp(bmp)
    assert got.shape == (ny, nx)

    # the aperture as the header builds it, in float: R0 = |antenna|,
    # deltaF = ChirpRate / ADF, max_Wy = c / (2 mean deltaF)
    r0 = np.sqrt(x * x + y * y + z * z).astype(np.float32)
    mean_df = np.float32(np.mean((chirp / adf).astype(np.float32).astype(np.float64)))
    max_wy = np.float32(CLIGHT / (2.0 * np.float64(mean_df)))
    assert abs(float(max_wy) - geom[4]) <= 1e-6 * geom[4]
    grid = S.Grid(nx=nx, ny=ny, wx=geom[2], wy=geom[3], x0=geom[0], y0=geom[1])
    with F.Plan(K, Np, nfft, float(max_wy), grid, precision="mixed", window=None) as plan:
        img = plan.focus(sc.phase_history, *(a.astype(np.float64) for a in (x, y, z, r0, start)))
    u8 = AF.reference_u8_image(torch.as_tensor(img[0])).numpy()  # [nx, ny]
    want = u8[:, ::-1].T  # writeBMPFile: row y shows column ny - 1 - y
    diff = np.abs(got.astype(int) - want.astype(int))
    assert diff.max() <= 1 and (diff > 0).mean() < 0.01, (diff.max(), (diff > 0).mean())
