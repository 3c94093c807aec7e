"""The oracle, pinned before it is trusted (CPU only).

* its FFT against numpy's FFT (including Bluestein lengths);
* its float instantiation against the reference's run_bp<float>, bit for bit,
  through the committed golden fixtures and, where the reference sources are
  present, through oracle/_ref compiled from them;
* its FP64 instantiation against the reference's run_bp<double> (which keeps
  the differential range in float, cpuBackProjection.hpp:65, hence the
  tolerance) and against known answers: a point target focuses at its pixel
  with zero phase and the expected gain, and the operator is linear.
"""
import numpy as np
import pytest

import golden_cases as G
from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12, 53, 64, 127, 131, 255, 424, 512, 2042, 3392, 4096])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign in (-1, +1):
        y = O.dft(x, sign)
        ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
        assert np.abs(y - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_range_compress_fp64_matches_numpy_definition():
    rng = np.random.default_rng(0)
    Np, K, nfft = 7, 53, 424
    ph = (rng.standard_normal((Np, K)) + 1j * rng.standard_normal((Np, K))).astype(np.complex64)
    w = O.hamming(K)
    got = O.range_compress_fp64(ph, nfft, w)
    want = np.fft.fftshift(np.fft.ifft(ph.astype(np.complex128) * w[None, :], nfft, axis=1), axes=1)
    assert np.abs(got - want).max() < 1e-13


@pytest.mark.parametrize("name", G.names())
def test_ref32_oracle_bit_exact_against_golden(name):
    sc, d = G.load(name)
    ph, _ = O.pad_for_reference(sc)
    rc = O.range_compress_ref32(ph)
    g = sc.grid
    img = O.bp_ref32(rc, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, d["ref_start_f_f32"],
                     float(d["ref_max_wy_f32"]), g.nx, g.ny, g.x0, g.y0, g.wx, g.wy)
    assert np.array_equal(img, d["ref_img_f32"])


@pytest.mark.parametrize("name", G.names())
def test_ref64_oracle_bit_exact_against_golden(name):
    sc, d = G.load(name)
    ph, _ = O.pad_for_reference(sc, np.float64)
    rc = O.range_compress_ref64(ph)
    g = sc.grid
    img = O.bp_ref64(rc, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, d["ref_start_f_f64"],
                     float(d["ref_max_wy_f64"]), g.nx, g.ny, g.x0, g.y0, g.wx, g.wy)
    assert np.array_equal(img, d["ref_img_f64"])


@pytest.mark.parametrize("name", G.names())
def test_fp64_oracle_against_reference_double_golden(name):
    sc, d = G.load(name)
    img = O.focus_fp64(sc)[0]
    # run_bp<double> rounds dR to float and truncates the real part of the
    # complex product through a float temporary (uncc_complex.hpp:187); the
    # FP64 oracle is the same operation sequence without those roundings
    assert O.rel_l2(img, d["ref_img_f64"]) < 3e-4
    assert O.rel_l2(d["ref_img_f32"], img) > 1e-3  # the float path is visibly worse


@pytest.mark.skipif(not O.ref_available(), reason="reference not compiled here (oracle/_ref absent)")
def test_ref32_oracle_bit_exact_against_live_reference():
    sc = S.point_target_scene(K=40, Np=33, n=20, spacing=0.3, nfft=160, snr_db=15.0, seed=123, n_targets=6,
                              extent=5.0)
    ref, maxwy, sf = O.reference_focus(sc, "f32")
    ph, _ = O.pad_for_reference(sc)
    rc = O.range_compress_ref32(ph)
    g = sc.grid
    img = O.bp_ref32(rc, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sf, maxwy, g.nx, g.ny, g.x0, g.y0, g.wx,
                     g.wy)
    assert np.array_equal(img, ref)


def test_point_target_known_answer():
    # one unit target at a pixel centre: every pulse adds the range-profile
    # peak sum_k w_k / Nfft with zero phase
    K, Np, nfft = 64, 32, 512
    sc = S.point_target_scene(K=K, Np=Np, n=33, spacing=0.2, nfft=nfft, snr_db=None, seed=0, n_targets=1)
    sc.targets[:] = 0.0
    freqs = sc.start_freq[0] + np.arange(K) * sc.delta_freq
    ant = np.stack([sc.ant_x, sc.ant_y, sc.ant_z], 1)
    sc.phase_history = S.synthesize_phase_history(freqs, ant, sc.slant_range, sc.targets, sc.amplitudes)
    img = O.focus_fp64(sc)[0]
    peak = np.unravel_index(np.argmax(np.abs(img)), img.shape)
    assert peak == (16, 16)
    gain = Np * O.hamming(K).sum() / nfft
    assert abs(np.angle(img[peak])) < 1e-3
    assert 0.97 * gain < abs(img[peak]) <= gain * 1.0001


def test_fp64_oracle_is_linear():
    sc = S.point_target_scene(K=48, Np=24, n=16, spacing=0.3, nfft=256, snr_db=None, seed=3)
    a = O.focus_fp64(sc)
    ph0 = sc.phase_history.copy()
    rng = np.random.default_rng(9)
    other = (rng.standard_normal(ph0.shape) + 1j * rng.standard_normal(ph0.shape)).astype(np.complex64)
    sc.phase_history = other
    b = O.focus_fp64(sc)
    sc.phase_history = (ph0.astype(np.complex128) * 2.0 - 0.5j * other.astype(np.complex128)).astype(
        np.complex128)
    c = O.focus_fp64(sc)
    assert O.rel_l2(c, 2.0 * a - 0.5j * b) < 1e-6  # complex64 rounding of the combined input


def test_pixel_subset_matches_full_image():
    sc = S.point_target_scene(K=48, Np=24, n=20, spacing=0.3, nfft=256, snr_db=20.0, seed=4)
    full = O.focus_fp64(sc).ravel()
    pix = np.array([0, 5, 77, 211, 399], dtype=np.int64)
    sub = O.focus_fp64(sc, pixels=pix)
    assert np.array_equal(sub, full[pix])


def test_fp64_gradient_oracle_matches_central_differences():
    # L = Re(sum conj(G) img): its gradient is exactly what the adjoint returns
    sc = S.point_target_scene(K=64, Np=12, n=20, spacing=0.25, nfft=512, snr_db=None, seed=3, n_targets=3,
                              extent=4.0)
    rc = O.range_compress_fp64(sc.phase_history, sc.nfft, O.hamming(sc.num_range_samples))
    rng = np.random.default_rng(0)
    G = rng.standard_normal((1, 20, 20)) + 1j * rng.standard_normal((1, 20, 20))
    ga, gr = O.bp_grad_fp64(rc, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq, sc.max_wr,
                            sc.grid, G)

    def L(ax, ay, az, r0):
        img = O.bp_fp64(rc, ax, ay, az, r0, sc.start_freq, sc.max_wr, sc.grid)
        return float(np.real(np.sum(np.conj(G) * img)))

    h = 1e-6  # central-difference truncation ~ h^2 (2 pi k)^3 / 6 stays below 1e-5 relative
    for p in (0, 5, 11):
        scale = np.abs(ga[:, p]).max()
        base = [sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range]
        for axis in range(4):
            up, dn = list(base), list(base)
            up[axis] = base[axis].copy()
            dn[axis] = base[axis].copy()
            up[axis][p] += h
            dn[axis][p] -= h
            fd = (L(*up) - L(*dn)) / (2 * h)
            want = ga[axis][p] if axis < 3 else gr[p]
            assert abs(fd - want) < 2e-5 * scale, (p, axis, fd, want)


# ---- matched filter (cpuBackProjection.hpp:165-228, matlab/mfBasic.m:73-89) ----

def _mf_scene(**kw):
    from uncc_sar_focusing_b200 import scenes as S

    args = dict(K=32, Np=24, n=16, spacing=0.1, nfft=256, snr_db=None, seed=5, n_targets=2, extent=1.0)
    args.update(kw)
    return S.point_target_scene(**args)


def test_mf_oracle_matches_direct_sum():
    from uncc_sar_focusing_b200 import scenes as S

    sc = _mf_scene(K=8, Np=5, n=4, spacing=0.3, nfft=64, n_targets=1, extent=0.5, seed=6)
    ph = sc.phase_history.astype(complex) * O.window_for(sc.window, 8)
    img = np.zeros((4, 4), complex)
    for ix, x in enumerate(sc.grid.axis("x")):
        for iy, y in enumerate(sc.grid.axis("y")):
            for p in range(sc.num_pulses):
                dR = np.sqrt((sc.ant_x[p] - x) ** 2 + (sc.ant_y[p] - y) ** 2 + sc.ant_z[p] ** 2) - sc.slant_range[p]
                f = sc.start_freq[p] + np.arange(8) * sc.delta_freq
                img[ix, iy] += np.sum(ph[p] * np.exp(1j * 4 * np.pi * f * dR / S.CLIGHT))
    assert O.rel_l2(O.mf_fp64(sc)[0], img) < 1e-12


@pytest.mark.skipif(not O.ref_available(), reason="reference not compiled here")
def test_mf_oracle_pinned_to_reference_run_mf():
    """The reference's run_mf<double> starts at pulse 2 (cpuBackProjection.hpp:
    216-218); with the same start the oracle matches it to its float dR."""
    sc = _mf_scene()
    ref = O.reference_mf(sc)
    assert O.rel_l2(O.mf_fp64(sc, first_pulse=2)[0], ref) < 3e-5
    assert O.rel_l2(O.mf_fp64(sc)[0], ref) > 0.05  # the skipped pulses matter


def test_mf_is_nfft_times_bp_up_to_interpolation():
    sc = _mf_scene(K=64, Np=48, n=32, spacing=0.15, nfft=512, snr_db=20.0, seed=3, n_targets=4, extent=4.0)
    assert O.rel_l2(O.focus_fp64(sc) * sc.nfft, O.mf_fp64(sc)) < 0.03


def test_taylor_window_matches_scipy():
    """The oracle's Taylor taper (matlab/rangeCompress.m:11, taylorwin(K, 5,
    -35), not normalised) against scipy's independent implementation."""
    from scipy.signal import windows

    for n in (1, 2, 7, 64, 424, 512, 1001):
        want = windows.taylor(n, nbar=5, sll=35, norm=False)
        assert np.allclose(O.taylor(n), want, rtol=0, atol=1e-12), n


def test_complex_range_weights_oracle_is_the_weighted_transform():
    """Range compression with complex per-sample weights equals the plain
    oracle transform of the weighted phase history (numpy FFT in FP64)."""
    rng = np.random.default_rng(3)
    ph = (rng.standard_normal((5, 48)) + 1j * rng.standard_normal((5, 48))).astype(np.complex64)
    w = rng.standard_normal(48) + 1j * rng.standard_normal(48)
    got = O.range_compress_fp64(ph, 200, w)
    x = np.zeros((5, 200), dtype=np.complex128)
    x[:, :48] = ph.astype(np.complex128) * w[None, :]
    want = np.fft.fftshift(np.fft.ifft(x, axis=1), axes=1)
    assert np.abs(got - want).max() < 1e-13 * np.abs(want).max() * 200
