"""MAT ingest against files written independently of the reader's own
writer: tests/matv5.py writes the GOTCHA `data` and Sandia `sph_MATData`
structs byte by byte from the MAT level-5 format, field by field as the
reference reads them (include/uncc_sar_matio.hpp:133-196: data.fp,
data.freq, data.x/y/z, data.r0, data.th, data.phi, data.af.r_correct /
ph_correct; sph_MATData.Data.SampleData, .StartF, .ChirpRate,
.radarCoordinateFrame.x/y/z, sph_MATData.preamble.ADF), in MATLAB's shapes
(K x Np phase history, single-precision complex as the collected data; 1 x Np
and Np x 1 vectors).  matdata.load reads them; the CPU tests compare every
field with the scene they came from, the GPU tests focus the loaded aperture
with the engine against the FP64 oracle image of the original scene."""
import numpy as np
import pytest

import matv5
from oracle import oracle as O
from uncc_sar_focusing_b200 import matdata as M
from uncc_sar_focusing_b200 import scenes as S

TOL = 1e-4  # mixed-precision image against the FP64 oracle


def scene():
    return S.point_target_scene(K=64, Np=48, n=32, spacing=0.2, nfft=512, snr_db=20.0, seed=21, n_targets=3,
                                extent=4.0)


def freqs(sc):
    return sc.start_freq[0] + np.arange(sc.num_range_samples) * sc.delta_freq


def write_gotcha(path, sc):
    Np = sc.num_pulses
    matv5.write(path, {"data": {
        "fp": sc.phase_history.T.astype(np.complex64),            # K x Np, single complex
        "freq": freqs(sc)[:, None],                                # K x 1
        "x": sc.ant_x[None, :], "y": sc.ant_y[None, :], "z": sc.ant_z[None, :],  # 1 x Np
        "r0": sc.slant_range[None, :],
        "th": np.linspace(-2.0, 2.0, Np)[None, :], "phi": np.full((1, Np), 30.0),
        "af": {"r_correct": np.zeros((1, Np)), "ph_correct": np.zeros((1, Np))},
    }})


def write_sandia(path, sc, adf=2.5e6):
    Np = sc.num_pulses
    matv5.write(path, {"sph_MATData": {
        "preamble": {"ADF": adf},
        "Data": {
            "SampleData": sc.phase_history.T.astype(np.complex64),  # K x Np
            "StartF": sc.start_freq[:, None],                        # Np x 1
            "ChirpRate": np.full((Np, 1), sc.delta_freq * adf),
            "radarCoordinateFrame": {"x": sc.ant_x[:, None], "y": sc.ant_y[:, None], "z": sc.ant_z[:, None]},
        },
    }})


def test_gotcha_fields_from_an_independent_file(tmp_path):
    sc = scene()
    p = str(tmp_path / "gotcha_v5.mat")
    write_gotcha(p, sc)
    ap = M.load(p)
    assert ap.layout == "gotcha"
    np.testing.assert_array_equal(ap.phase_history, sc.phase_history)
    for a in ("ant_x", "ant_y", "ant_z", "slant_range"):
        np.testing.assert_array_equal(getattr(ap, a), getattr(sc, a))
    np.testing.assert_array_equal(ap.start_freq, np.full(sc.num_pulses, freqs(sc)[0]))
    assert ap.max_wr == pytest.approx(sc.max_wr, rel=1e-9)
    assert set(ap.extra) == {"th", "phi", "af_r_correct", "af_ph_correct"}
    assert O.rel_l2(O.focus_fp64(ap.to_scene(sc.grid, nfft=sc.nfft)), O.focus_fp64(sc)) < 1e-9


def test_sandia_fields_from_an_independent_file(tmp_path):
    sc = scene()
    p = str(tmp_path / "sandia_v5.mat")
    write_sandia(p, sc)
    ap = M.load(p)
    assert ap.layout == "sandia"
    np.testing.assert_array_equal(ap.phase_history, sc.phase_history)
    np.testing.assert_array_equal(ap.start_freq, sc.start_freq)
    assert ap.max_wr == pytest.approx(sc.max_wr, rel=1e-12)
    assert O.rel_l2(O.focus_fp64(ap.to_scene(sc.grid, nfft=sc.nfft)), O.focus_fp64(sc)) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["gotcha", "sandia"])
def test_engine_focuses_an_independent_file(tmp_path, layout):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from uncc_sar_focusing_b200 import focusing

    sc = scene()
    p = str(tmp_path / f"{layout}.mat")
    (write_gotcha if layout == "gotcha" else write_sandia)(p, sc)
    loaded = M.load(p).to_scene(sc.grid, nfft=sc.nfft)
    want = O.focus_fp64(sc)
    with focusing.Plan.for_scene(loaded, "mixed") as plan:
        got = plan.focus(loaded.phase_history, loaded.ant_x, loaded.ant_y, loaded.ant_z, loaded.slant_range,
                         loaded.start_freq)
        plan.check()
    assert O.rel_l2(got, want) < TOL
