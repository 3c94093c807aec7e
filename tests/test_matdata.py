"""MAT-file ingest (uncc_sar_focusing_b200.matdata): the GOTCHA and Sandia
layouts the reference reads with matio (include/uncc_sar_matio.hpp:133-196),
completed as initialize_SAR_Aperture_Data does
(include/uncc_sar_focusing.hpp:224-393).  Files are written with the module's
own writers from synthetic point-target scenes, read back, and focused by the
FP64 oracle next to the original scene."""
import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import matdata as M
from uncc_sar_focusing_b200 import scenes as S


def small():
    return S.point_target_scene(K=48, Np=40, n=24, spacing=0.2, nfft=384, snr_db=20.0, seed=11, n_targets=3,
                                extent=3.0)


def freqs(sc):
    return sc.start_freq[0] + np.arange(sc.num_range_samples) * sc.delta_freq


def test_gotcha_round_trip(tmp_path):
    sc = small()
    f = tmp_path / "gotcha.mat"
    th = np.linspace(-2.0, 2.0, sc.num_pulses)
    M.save_gotcha(str(f), sc.phase_history, freqs(sc), sc.ant_x, sc.ant_y, sc.ant_z, r0=sc.slant_range,
                  th=th, phi=np.full(sc.num_pulses, 30.0), r_correct=np.zeros(sc.num_pulses),
                  ph_correct=np.ones(sc.num_pulses))
    ap = M.load(str(f))
    assert ap.layout == "gotcha" and ap.phase_history.shape == sc.phase_history.shape
    np.testing.assert_array_equal(ap.phase_history, sc.phase_history)
    for a in ("ant_x", "ant_y", "ant_z", "slant_range"):
        np.testing.assert_array_equal(getattr(ap, a), getattr(sc, a))
    # one frequency vector for every pulse: start = min(freq), step = |f1 - f0|
    np.testing.assert_array_equal(ap.start_freq, np.full(sc.num_pulses, freqs(sc).min()))
    assert ap.max_wr == pytest.approx(sc.max_wr, rel=1e-9)
    np.testing.assert_array_equal(ap.extra["th"], th)
    assert set(ap.extra) == {"th", "phi", "af_r_correct", "af_ph_correct"}
    got = O.focus_fp64(ap.to_scene(sc.grid, nfft=sc.nfft))
    assert O.rel_l2(got, O.focus_fp64(sc)) < 1e-9


def test_gotcha_per_pulse_frequencies_and_missing_r0(tmp_path):
    sc = small()
    fmat = np.tile(freqs(sc)[:, None], (1, sc.num_pulses))  # K x Np
    f = tmp_path / "gotcha_fmat.mat"
    M.save_gotcha(str(f), sc.phase_history, fmat, sc.ant_x, sc.ant_y, sc.ant_z)
    ap = M.load(str(f))
    assert ap.freq.shape == (sc.num_pulses, sc.num_range_samples)
    np.testing.assert_array_equal(ap.start_freq, sc.start_freq)
    # no r0 in the file: |antenna| (uncc_sar_focusing.hpp:311-321)
    np.testing.assert_allclose(ap.slant_range, np.sqrt(sc.ant_x ** 2 + sc.ant_y ** 2 + sc.ant_z ** 2), rtol=0)


def test_sandia_derived_frequencies(tmp_path):
    sc = small()
    adf = 2.5e6
    chirp = np.full(sc.num_pulses, sc.delta_freq * adf)
    f = tmp_path / "sandia.mat"
    M.save_sandia(str(f), sc.phase_history, sc.start_freq, chirp, adf, sc.ant_x, sc.ant_y, sc.ant_z)
    ap = M.load(str(f))
    assert ap.layout == "sandia"
    # freq = StartF + k ChirpRate / ADF (uncc_sar_focusing.hpp:297-300)
    want = sc.start_freq[:, None] + np.arange(sc.num_range_samples)[None, :] * (chirp / adf)[:, None]
    np.testing.assert_array_equal(ap.freq, want)
    assert ap.max_wr == pytest.approx(sc.max_wr, rel=1e-12)
    got = O.focus_fp64(ap.to_scene(sc.grid, nfft=sc.nfft))
    assert O.rel_l2(got, O.focus_fp64(sc)) < 1e-9  # slant range |antenna| = radius to rounding


def test_rejections(tmp_path):
    import scipy.io

    sc = small()
    bad = tmp_path / "real.mat"
    M.save_gotcha(str(bad), sc.phase_history.real, freqs(sc), sc.ant_x, sc.ant_y, sc.ant_z)
    with pytest.raises(ValueError, match="complex"):
        M.load(str(bad))
    other = tmp_path / "other.mat"
    scipy.io.savemat(str(other), {"something": np.zeros(3)})
    with pytest.raises(ValueError, match="neither"):
        M.load(str(other))
    neg = tmp_path / "neg.mat"
    M.save_sandia(str(neg), sc.phase_history, sc.start_freq, -np.ones(sc.num_pulses), 1e6, sc.ant_x, sc.ant_y,
                  sc.ant_z)
    with pytest.raises(ValueError, match="increase"):
        M.load(str(neg))
    # a -v7.3 header (HDF5 container): text, subsystem offset, version 0x0200, endian mark
    v73 = tmp_path / "v73.mat"
    head = b"MATLAB 7.3 MAT-file, Platform: GLNXA64".ljust(116, b" ") + b"\x00" * 8 + b"\x00\x02IM"
    v73.write_bytes(head + b"\x89HDF\r\n\x1a\n" + b"\x00" * 64)
    with pytest.raises(ValueError, match="7.3"):
        M.load(str(v73))
