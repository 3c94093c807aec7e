"""TEST INFRASTRUCTURE (the oracle), not product code.

ctypes binding of oracle/liboracle.so (the project's CPU restatement of the
reference backprojection, oracle/bp_oracle.c), of oracle/_ref/libref_bp*.so
(the reference's own run_bp compiled from its sources by oracle/Makefile) and
of oracle/_ref/libref_gpu.so (the reference's own GPU kernels, built from
their header by the same Makefile, launched by oracle/ref_gpu_harness.cu).
Only tests/, __graft_entry__.smoke() and bench.py's reference legs (the CPU
baseline, the reference arm, the reference-GPU timing) import this module:
as the checker, or as the reference being timed, never as the product.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}

_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_c = ctypes


def build() -> None:
    """Compile liboracle.so, and the reference harness when the environment
    names a reference checkout (SARBP_REFERENCE; make is a no-op when
    everything is up to date)."""
    import subprocess

    ref = os.environ.get("SARBP_REFERENCE", "")
    if ref and not os.path.isdir(os.path.join(ref, "src")):
        raise RuntimeError(f"SARBP_REFERENCE={ref} is not a reference checkout (no src/ directory)")
    targets = ["all"] if ref else [os.path.join(HERE, "liboracle.so")]
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_range_compress_fp64.argtypes = [_c.c_int, _c.c_int, _c.c_int, _f32p, _c.c_void_p, _f64p]
        L.oracle_range_compress_fp64_cw.argtypes = [_c.c_int, _c.c_int, _c.c_int, _f32p, _f64p, _f64p]
        L.oracle_range_compress_ref32.argtypes = [_c.c_int, _c.c_int, _f32p, _f32p]
        bp_geo = [_f64p] * 5 + [_c.c_double] + [_c.c_int] * 3 + [_c.c_double] * 6
        L.oracle_bp_fp64.argtypes = [_c.c_int, _c.c_int, _f64p] + bp_geo + [_f64p]
        L.oracle_bp_fp64_pixels.argtypes = [_c.c_int, _c.c_int, _f64p] + bp_geo + [_c.c_longlong, _i64p, _f64p]
        L.oracle_bp_ref32.argtypes = ([_c.c_int, _c.c_int, _f32p] + [_f32p] * 5 + [_c.c_float, _c.c_int, _c.c_int]
                                      + [_c.c_float] * 4 + [_f32p])
        L.oracle_range_compress_ref64.argtypes = [_c.c_int, _c.c_int, _f64p, _f64p]
        L.oracle_bp_ref64.argtypes = ([_c.c_int, _c.c_int, _f64p] + [_f64p] * 5 + [_c.c_double, _c.c_int, _c.c_int]
                                      + [_c.c_double] * 4 + [_f64p])
        L.oracle_bp_grad_fp64.argtypes = ([_c.c_int, _c.c_int, _f64p] + bp_geo + [_f64p] * 5)
        L.oracle_dft_c128.argtypes = [_c.c_int, _f64p, _f64p, _c.c_int]
        L.oracle_mf_fp64.argtypes = ([_c.c_int, _c.c_int, _f64p] + [_f64p] * 5 + [_c.c_double] + [_c.c_int] * 3
                                     + [_c.c_double] * 6 + [_c.c_int, _f64p])
        for f in ("oracle_range_compress_fp64", "oracle_range_compress_fp64_cw", "oracle_range_compress_ref32", "oracle_bp_fp64",
                  "oracle_bp_fp64_pixels", "oracle_bp_ref32", "oracle_dft_c128", "oracle_range_compress_ref64",
                  "oracle_bp_ref64", "oracle_bp_grad_fp64", "oracle_mf_fp64"):
            getattr(L, f).restype = _c.c_int
        _LIB = L
    return _LIB


def ref_available(fast: bool = False) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_bp_fast.so" if fast else "libref_bp.so"))


def ref_lib(fast: bool = False):
    key = "fast" if fast else "strict"
    if key not in _REF:
        path = os.path.join(HERE, "_ref", "libref_bp_fast.so" if fast else "libref_bp.so")
        L = ctypes.CDLL(path)
        L.ref_focus_bp_f32.argtypes = ([_c.c_int, _c.c_int] + [_f32p] * 6 + [_c.c_int, _c.c_int]
                                       + [_c.c_float] * 4 + [_f32p, _f32p, _f32p])
        L.ref_focus_bp_f64.argtypes = ([_c.c_int, _c.c_int] + [_f64p] * 6 + [_c.c_int, _c.c_int]
                                       + [_c.c_double] * 4 + [_f64p, _f64p, _f64p])
        L.ref_focus_mf_f64.argtypes = ([_c.c_int, _c.c_int] + [_f64p] * 6 + [_c.c_int, _c.c_int]
                                       + [_c.c_double] * 4 + [_f64p])
        L.ref_focus_mf_f64.restype = _c.c_int
        L.ref_focus_bp_f32.restype = _c.c_int
        L.ref_focus_bp_f64.restype = _c.c_int
        _REF[key] = L
    return _REF[key]


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def hamming(K: int) -> np.ndarray:
    """0.54 - 0.46 cos(2 pi k / (K-1)) (the taper of matlab/formImage3DSAR.m:115-116)."""
    k = np.arange(K, dtype=np.float64)
    return 0.54 - 0.46 * np.cos(2.0 * np.pi * k / (K - 1))


def taylor(n: int, nbar: int = 5, sll: float = -35.0) -> np.ndarray:
    """Taylor window, not normalised (the taper of matlab/rangeCompress.m:11,
    taylorwin(K, 5, -35)): w = 1 + 2 sum_{m<nbar} F_m cos(2 pi m x),
    x = (k - n/2 + 1/2)/n, with the coefficients F_m of Carrara, Goodman and
    Majewski, "Spotlight Synthetic Aperture Radar" (1995)."""
    if n <= 1:
        return np.ones(max(n, 0))
    A = np.arccosh(10.0 ** (-sll / 20.0)) / np.pi
    sig2 = nbar ** 2 / (A ** 2 + (nbar - 0.5) ** 2)
    i = np.arange(1, nbar, dtype=np.float64)
    x = (np.arange(n, dtype=np.float64) - 0.5 * n + 0.5) / n
    w = np.ones(n)
    for m in range(1, nbar):
        num = np.prod(1.0 - (m * m / sig2) / (A ** 2 + (i - 0.5) ** 2))
        den = np.prod(1.0 - m * m / i[i != m] ** 2)
        w += 2.0 * ((-1) ** (m + 1)) * num / (2.0 * den) * np.cos(2.0 * np.pi * m * x)
    return w


def window_for(name: Optional[str], K: int) -> Optional[np.ndarray]:
    if name in (None, "none"):
        return None
    if name == "hamming":
        return hamming(K)
    if name == "taylor":
        return taylor(K)
    raise ValueError(name)


def dft(x: np.ndarray, sign: int) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    _check(lib().oracle_dft_c128(x.shape[0], x.view(np.float64), out.view(np.float64), sign), "dft")
    return out


def range_compress_fp64(ph: np.ndarray, nfft: int, window: Optional[np.ndarray] = None) -> np.ndarray:
    ph = np.ascontiguousarray(ph, dtype=np.complex64)
    Np, K = ph.shape
    out = np.empty((Np, nfft), dtype=np.complex128)
    if window is not None and np.iscomplexobj(window):
        cw = np.ascontiguousarray(window, dtype=np.complex128)
        _check(lib().oracle_range_compress_fp64_cw(K, Np, nfft, ph.view(np.float32).reshape(-1),
                                                   cw.view(np.float64), out.view(np.float64).reshape(-1)),
               "range_compress_fp64_cw")
        return out
    wptr = None
    if window is not None:
        window = np.ascontiguousarray(window, dtype=np.float64)
        wptr = window.ctypes.data
    _check(lib().oracle_range_compress_fp64(K, Np, nfft, ph.view(np.float32).reshape(-1), wptr,
                                            out.view(np.float64).reshape(-1)), "range_compress_fp64")
    return out


def _geo(ax, ay, az, r0, f0):
    return [np.ascontiguousarray(v, dtype=np.float64) for v in (ax, ay, az, r0, f0)]


def bp_fp64(rc: np.ndarray, ax, ay, az, r0, f0, max_wr: float, grid) -> np.ndarray:
    rc = np.ascontiguousarray(rc, dtype=np.complex128)
    Np, nfft = rc.shape
    out = np.empty((grid.nz, grid.nx, grid.ny), dtype=np.complex128)
    _check(lib().oracle_bp_fp64(Np, nfft, rc.view(np.float64).reshape(-1), *_geo(ax, ay, az, r0, f0),
                                float(max_wr), grid.nx, grid.ny, grid.nz, grid.x0, grid.y0, grid.z0, grid.wx,
                                grid.wy, grid.wz, out.view(np.float64).reshape(-1)), "bp_fp64")
    return out


def bp_fp64_pixels(rc: np.ndarray, ax, ay, az, r0, f0, max_wr: float, grid, pix: np.ndarray) -> np.ndarray:
    rc = np.ascontiguousarray(rc, dtype=np.complex128)
    Np, nfft = rc.shape
    pix = np.ascontiguousarray(pix, dtype=np.int64)
    out = np.empty(pix.shape[0], dtype=np.complex128)
    _check(lib().oracle_bp_fp64_pixels(Np, nfft, rc.view(np.float64).reshape(-1), *_geo(ax, ay, az, r0, f0),
                                       float(max_wr), grid.nx, grid.ny, grid.nz, grid.x0, grid.y0, grid.z0,
                                       grid.wx, grid.wy, grid.wz, pix.shape[0], pix,
                                       out.view(np.float64).reshape(-1)), "bp_fp64_pixels")
    return out


def bp_grad_fp64(rc: np.ndarray, ax, ay, az, r0, f0, max_wr: float, grid, G: np.ndarray):
    """dL/d(ant_x, ant_y, ant_z) [3, Np] and dL/dR0 [Np] of a loss with upstream
    image gradient G (complex, [nz, nx, ny])."""
    rc = np.ascontiguousarray(rc, dtype=np.complex128)
    Np, nfft = rc.shape
    G = np.ascontiguousarray(G, dtype=np.complex128)
    out = np.zeros((4, Np), dtype=np.float64)
    _check(lib().oracle_bp_grad_fp64(Np, nfft, rc.view(np.float64).reshape(-1), *_geo(ax, ay, az, r0, f0),
                                     float(max_wr), grid.nx, grid.ny, grid.nz, grid.x0, grid.y0, grid.z0, grid.wx,
                                     grid.wy, grid.wz, G.view(np.float64).reshape(-1), out[0], out[1], out[2],
                                     out[3]), "bp_grad_fp64")
    return out[:3], out[3]


def focus_fp64(scene, pixels: Optional[np.ndarray] = None) -> np.ndarray:
    """FP64 oracle image of a scenes.Scene (window, zero pad to Nfft, IFFT,
    fftshift, then BP).  With pixels, only those flat indices are formed."""
    w = window_for(scene.window, scene.num_range_samples)
    rc = range_compress_fp64(scene.phase_history, scene.nfft, w)
    args = (rc, scene.ant_x, scene.ant_y, scene.ant_z, scene.slant_range, scene.start_freq, scene.max_wr,
            scene.grid)
    if pixels is None:
        return bp_fp64(*args)
    return bp_fp64_pixels(*args, pixels)


def pad_for_reference(scene, dtype=np.float32, pulses: Optional[slice] = None):
    """The reference has no zero pad or window (cpuBackProjection.hpp:107-110):
    feed it w.*ph zero-padded from K to Nfft and freq extended at the same step."""
    K = scene.num_range_samples
    w = window_for(scene.window, K)
    ph = scene.phase_history[pulses if pulses is not None else slice(None)].astype(np.complex128)
    if w is not None:
        ph = ph * w[None, :]
    padded = np.zeros((ph.shape[0], scene.nfft), dtype=np.complex128)
    padded[:, :K] = ph
    freq = scene.start_freq[0] + np.arange(scene.nfft, dtype=np.float64) * scene.delta_freq
    ctype = np.complex64 if dtype == np.float32 else np.complex128
    return padded.astype(ctype), freq.astype(dtype)


def range_compress_ref32(ph_padded: np.ndarray) -> np.ndarray:
    ph_padded = np.ascontiguousarray(ph_padded, dtype=np.complex64)
    Np, nfft = ph_padded.shape
    out = np.empty_like(ph_padded)
    _check(lib().oracle_range_compress_ref32(nfft, Np, ph_padded.view(np.float32).reshape(-1),
                                             out.view(np.float32).reshape(-1)), "range_compress_ref32")
    return out


def bp_ref32(rc: np.ndarray, ax, ay, az, r0, f0, max_wr: float, nx: int, ny: int, x0: float, y0: float,
             wx: float, wy: float) -> np.ndarray:
    rc = np.ascontiguousarray(rc, dtype=np.complex64)
    Np, nfft = rc.shape
    out = np.empty((nx, ny), dtype=np.complex64)
    geo = [np.ascontiguousarray(v, dtype=np.float32) for v in (ax, ay, az, r0, f0)]
    _check(lib().oracle_bp_ref32(Np, nfft, rc.view(np.float32).reshape(-1), *geo, np.float32(max_wr), nx, ny,
                                 np.float32(x0), np.float32(y0), np.float32(wx), np.float32(wy),
                                 out.view(np.float32).reshape(-1)), "bp_ref32")
    return out


def range_compress_ref64(ph_padded: np.ndarray) -> np.ndarray:
    ph_padded = np.ascontiguousarray(ph_padded, dtype=np.complex128)
    Np, nfft = ph_padded.shape
    out = np.empty_like(ph_padded)
    _check(lib().oracle_range_compress_ref64(nfft, Np, ph_padded.view(np.float64).reshape(-1),
                                             out.view(np.float64).reshape(-1)), "range_compress_ref64")
    return out


def bp_ref64(rc: np.ndarray, ax, ay, az, r0, f0, max_wr: float, nx: int, ny: int, x0: float, y0: float,
             wx: float, wy: float) -> np.ndarray:
    rc = np.ascontiguousarray(rc, dtype=np.complex128)
    Np, nfft = rc.shape
    out = np.empty((nx, ny), dtype=np.complex128)
    _check(lib().oracle_bp_ref64(Np, nfft, rc.view(np.float64).reshape(-1), *_geo(ax, ay, az, r0, f0),
                                 float(max_wr), nx, ny, float(x0), float(y0), float(wx), float(wy),
                                 out.view(np.float64).reshape(-1)), "bp_ref64")
    return out


def reference_focus(scene, precision: str = "f32", fast: bool = False, pulses: Optional[slice] = None):
    """Run the reference's focus_SAR_image<T,T> (run_bp) on a scene.

    Returns (image [nx, ny], max_Wy_m the reference derived, startF it used)."""
    dtype = np.float32 if precision == "f32" else np.float64
    sl = pulses if pulses is not None else slice(None)
    ph, freq = pad_for_reference(scene, dtype, sl)
    ph = np.ascontiguousarray(ph)
    geo = [np.ascontiguousarray(v[sl], dtype=dtype) for v in (scene.ant_x, scene.ant_y, scene.ant_z,
                                                              scene.slant_range)]
    Np, nfft = ph.shape
    g = scene.grid
    img = np.empty((g.nx, g.ny), dtype=np.complex64 if dtype == np.float32 else np.complex128)
    max_wy = np.zeros(1, dtype=dtype)
    start_f = np.zeros(Np, dtype=dtype)
    L = ref_lib(fast)
    fn = L.ref_focus_bp_f32 if dtype == np.float32 else L.ref_focus_bp_f64
    _check(fn(nfft, Np, ph.view(dtype).reshape(-1), freq, *geo, g.nx, g.ny, g.x0, g.y0, g.wx, g.wy,
              img.view(dtype).reshape(-1), max_wy, start_f), "reference focus_SAR_image")
    return img, float(max_wy[0]), start_f


def ref_gpu_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_gpu.so"))


def reference_gpu_focus(scene, reps: int = 3):
    """The reference's own GPU kernels (cuifft, cufftNormalize_1DBatch,
    cufftShift_1DBatch, backprojection_loop<float>; oracle/ref_gpu_harness.cu)
    on a scene, timed with CUDA events.  Float geometry as SAR_Aperture<float>
    holds it; the phase history tapered and zero-padded to Nfft (the reference
    has neither).  Returns (image [nx, ny] complex64, fft_ms, bp_ms); raises
    ValueError, before any GPU work, for a scene that reaches the swath's
    lower edge (the reference kernel would read index -1 there)."""
    if "gpu" not in _REF:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_gpu.so"))
        L.ref_gpu_focus.argtypes = ([_f32p, _c.c_int, _c.c_int] + [_f32p] * 5 + [_c.c_double, _c.c_int, _c.c_int]
                                    + [_c.c_double] * 4 + [_c.c_int, _f32p, _c.POINTER(_c.c_double),
                                                           _c.POINTER(_c.c_double)])
        L.ref_gpu_focus.restype = _c.c_int
        _REF["gpu"] = L
    if scene.grid.nz != 1 or scene.grid.z0 != 0.0:
        raise ValueError("the reference kernel images the z = 0 plane only")
    ph, _ = pad_for_reference(scene, np.float32)
    ph = np.ascontiguousarray(ph)
    Np, nfft = ph.shape
    geo = [np.ascontiguousarray(v, dtype=np.float32) for v in (scene.ant_x, scene.ant_y, scene.ant_z,
                                                               scene.slant_range, scene.start_freq)]
    g = scene.grid
    img = np.empty((g.nx, g.ny), dtype=np.complex64)
    fft_ms, bp_ms = _c.c_double(0.0), _c.c_double(0.0)
    rc = _REF["gpu"].ref_gpu_focus(ph.view(np.float32).reshape(-1), nfft, Np, *geo, float(scene.max_wr), g.nx, g.ny,
                                   g.x0, g.y0, g.wx, g.wy, int(reps), img.view(np.float32).reshape(-1),
                                   _c.byref(fft_ms), _c.byref(bp_ms))
    if rc == -2:
        raise ValueError("scene reaches the swath's lower edge: the reference kernel would read index -1")
    _check(rc, "reference GPU focus")
    return img, fft_ms.value, bp_ms.value


def mf_fp64(scene, first_pulse: int = 0) -> np.ndarray:
    """FP64 matched-filter image of a scenes.Scene ([nz, nx, ny]): taper w
    applied to the phase history, freq_k = f0_p + k dF, all pulses from
    first_pulse on (matlab/mfBasic.m:73-89)."""
    w = window_for(scene.window, scene.num_range_samples)
    ph = scene.phase_history.astype(np.complex128)
    if w is not None:
        ph = ph * w[None, :]
    ph = np.ascontiguousarray(ph)
    g = scene.grid
    out = np.empty((g.nz, g.nx, g.ny), dtype=np.complex128)
    _check(lib().oracle_mf_fp64(scene.num_pulses, scene.num_range_samples, ph.view(np.float64).reshape(-1),
                                *_geo(scene.ant_x, scene.ant_y, scene.ant_z, scene.slant_range, scene.start_freq),
                                float(scene.delta_freq), g.nx, g.ny, g.nz, g.x0, g.y0, g.z0, g.wx, g.wy, g.wz,
                                int(first_pulse), out.view(np.float64).reshape(-1)), "mf_fp64")
    return out


def reference_mf(scene) -> np.ndarray:
    """The reference's run_mf<double> (focus_SAR_image with MATCHED_FILTER) on a
    scene ([nx, ny]); the taper is applied beforehand, as for backprojection."""
    K = scene.num_range_samples
    w = window_for(scene.window, K)
    ph = scene.phase_history.astype(np.complex128)
    if w is not None:
        ph = ph * w[None, :]
    ph = np.ascontiguousarray(ph)
    freq = scene.start_freq[0] + np.arange(K, dtype=np.float64) * scene.delta_freq
    geo = [np.ascontiguousarray(v, dtype=np.float64) for v in (scene.ant_x, scene.ant_y, scene.ant_z,
                                                               scene.slant_range)]
    g = scene.grid
    img = np.empty((g.nx, g.ny), dtype=np.complex128)
    _check(ref_lib().ref_focus_mf_f64(K, scene.num_pulses, ph.view(np.float64).reshape(-1), freq, *geo, g.nx, g.ny,
                                      g.x0, g.y0, g.wx, g.wy, img.view(np.float64).reshape(-1)), "reference run_mf")
    return img


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def peak_phase_error(a: np.ndarray, b: np.ndarray) -> float:
    """Phase difference (rad) at the magnitude peak of b."""
    b = np.asarray(b)
    i = int(np.argmax(np.abs(b).ravel()))
    return float(abs(np.angle(np.asarray(a).ravel()[i] * np.conj(b.ravel()[i]))))


def pga_step_reference(img: np.ndarray, db_down: float = 30.0) -> np.ndarray:
    """One iteration of the reference's PGA (matlab/PGA.m:150-212), restated
    with its 1-based MATLAB indexing written out, in double: the estimated,
    detrended azimuth phase error phi_error_est_detrended [Nx] of an image
    [Ny range lines][Nx azimuth samples]."""
    img = np.asarray(img, dtype=np.complex128)
    ny, nx = img.shape
    c = int(np.ceil(nx / 2.0))  # center_az_idx (1-based), :150
    f = np.zeros_like(img)
    for row in range(ny):  # :157-164
        m = int(np.argmax(np.abs(img[row]))) + 1  # 1-based max index
        f[row] = np.roll(img[row], 1 + c - m)  # circshift(img_af(row,:), 1 + c - m)
    avg = np.sum(np.conj(img) * img, axis=0).real  # :167
    avg_db = 10.0 * np.log10(avg / avg.max())
    cutoff = avg_db.max() - abs(db_down)
    left_part = np.nonzero(avg_db[:c] - cutoff < 0)[0]  # 1..c (1-based)
    right_part = np.nonzero(avg_db[c:] - cutoff < 0)[0]  # c+1..end
    leftidx = (left_part[-1] + 1) + 1 if left_part.size else 1  # 1-based, :172-177
    rightidx = (right_part[0] + 1) + c - 1 if right_part.size else nx
    mask = np.zeros(nx)
    mask[leftidx - 1:rightidx] = 1.0  # window_mask_row(leftidx:rightidx) = 1
    g = f * mask[None, :]
    G = np.fft.fft(np.fft.ifftshift(g, axes=1), axis=1)  # :195-196
    G_dot = np.diff(G, axis=1)
    phi_dot = np.sum(np.imag(np.conj(G[:, :-1]) * G_dot), axis=0) / np.sum(np.abs(G[:, :-1]) ** 2, axis=0)
    phi = np.unwrap(np.concatenate([[0.0], np.cumsum(phi_dot)]))  # :204
    x = np.arange(nx, dtype=np.float64)
    coeffs = np.polyfit(x, phi, 1)  # :209-212
    return phi - (coeffs[0] * x + coeffs[1])


def ref_pga_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_pga.so"))


def ref_pga(img: np.ndarray, iters: int) -> np.ndarray:
    """The reference's own compiled C++ PGA, autofocus<float>()
    (src/autofocus/cpu/autofocus_cpu.cpp:250-474, built into
    oracle/_ref/libref_pga.so), on an image [range lines][azimuth samples];
    returns the corrected image (complex64, same layout).  The routine prints
    one rms line per iteration on stdout."""
    if "pga" not in _REF:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_pga.so"))
        L.ref_pga_f32.argtypes = [_c.c_void_p, _c.c_int, _c.c_int, _c.c_int]
        L.ref_pga_f32.restype = _c.c_int
        _REF["pga"] = L
    rows, n = img.shape
    # the routine's layout: range fastest, index r + p * numRange
    data = np.ascontiguousarray(np.asarray(img, dtype=np.complex64).T)
    _check(_REF["pga"].ref_pga_f32(data.ctypes.data, n, rows, int(iters)), "ref_pga_f32")
    return np.ascontiguousarray(data.T)


def pga_cpp_reference(img: np.ndarray, iters: int, rms_stop: float = 0.1):
    """The reference's C++ PGA routine autofocus() (autofocus_cpu.cpp:250-474)
    restated in double, step for step, on an image [range lines][azimuth
    samples] (n azimuth samples).  Per iteration:
      * each range line circularly shifted so that its largest sample (first
        of equal maxima) lands at index n - n//2 (valarray cshift(n/2 + max),
        :266-285);
      * window from the non-coherent azimuth power of the UNSHIFTED image in
        dB against its maximum (:290-305): leftIdx = the last i < n//2 below
        -30 dB, rightIdx = the first i < n//2 with sample i + n//2 below -30 dB
        -- the index i itself, not i + n//2, as the routine has it (:307-311)
        -- defaults 0 and n; samples [0, leftIdx) and [rightIdx, n) zeroed;
      * G = forward FFT of fftshift(line), fftshift = cshift((n+1)//2)
        (:323-339, cpuBackProjection_fft.hpp:81-84);
      * phi_dot[p+1] = sum_r Im(conj(G_p) (G_{p+1} - G_p)) / sum_r |G_p|^2,
        phi = cumulative sum, no unwrap (:342-371);
      * least-squares line removed (:377-402); rms = sqrt(mean(phi^2)); stop
        before correcting when rms < 0.1 (:406-414);
      * each range line: forward FFT, times exp(-j phi), inverse FFT with the
        1/n scale (:418-445).
    Returns (corrected image complex128, [phi per applied iteration], [rms])."""
    x = np.asarray(img, dtype=np.complex128).copy()
    rows, n = x.shape
    h = n // 2
    col = np.arange(n)
    phis, rmss = [], []
    for _ in range(int(iters)):
        peak = np.argmax(np.abs(x), axis=1)
        shifted = np.take_along_axis(x, (col[None, :] + h + peak[:, None]) % n, axis=1)
        avg = np.sum((np.conj(x) * x).real, axis=0)
        avg_db = 10.0 * np.log10(avg / avg.max())
        left, right = -1, -1
        for i in range(h):
            if avg_db[i] < -30.0:
                left = i
            if avg_db[i + h] < -30.0 and right == -1:
                right = i
        left = 0 if left == -1 else left
        right = n if right == -1 else right
        shifted[:, :left] = 0.0
        shifted[:, right:] = 0.0
        G = np.fft.fft(np.roll(shifted, -((n + 1) // 2), axis=1), axis=1)
        num = np.sum(np.imag(np.conj(G[:, :-1]) * (G[:, 1:] - G[:, :-1])), axis=0)
        den = np.sum(np.abs(G[:, :-1]) ** 2, axis=0)
        phi = np.cumsum(np.concatenate([[0.0], num / den]))
        i = np.arange(n, dtype=np.float64)
        sx, sy, sxy, sxx = i.sum(), phi.sum(), (i * phi).sum(), (i * i).sum()
        d = n * sxx - sx * sx
        phi = phi - ((n * sxy - sx * sy) / d * i + (sy * sxx - sx * sxy) / d)
        rms = float(np.sqrt(np.mean(phi ** 2)))
        rmss.append(rms)
        if rms < rms_stop:
            break
        phis.append(phi)
        x = np.fft.ifft(np.fft.fft(x, axis=1) * np.exp(-1j * phi)[None, :], axis=1)
    return x, phis, rmss
