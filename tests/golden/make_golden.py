"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's CPU backprojection (run_bp via focus_SAR_image<float,float>
and <double,double>, src/cpuBackProjection/cpuBackProjection.hpp:95-163,230-262),
compiled from its own sources by oracle/Makefile into oracle/_ref/, on small
seeded point-target scenes, and stores inputs and outputs as .npz.  The GPU box
has no reference sources, so these files are how the oracle stays pinned there.
With --pga it writes the PGA fixtures instead: the reference's C++ PGA routine
(autofocus<float>(), src/autofocus/cpu/autofocus_cpu.cpp:250-474, compiled into
oracle/_ref/libref_pga.so) on seeded defocused images, with the rms values it
prints per iteration.

    python tests/golden/make_golden.py          # backprojection fixtures
    python tests/golden/make_golden.py --pga    # PGA fixtures
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from uncc_sar_focusing_b200 import scenes as S  # noqa: E402

CASES = {
    # name: point_target_scene kwargs
    "pt_k64_np48_32x32": dict(K=64, Np=48, n=32, spacing=0.25, nfft=512, snr_db=None, seed=5, n_targets=3,
                              extent=6.0),
    "pt_k53_np40_24x40_noise": dict(K=53, Np=40, n=24, spacing=0.3, nfft=424, snr_db=20.0, seed=11,
                                    n_targets=4, extent=5.0),
    "pt_k32_np64_16x16_hamming_odd": dict(K=32, Np=64, n=16, spacing=0.4, nfft=255, snr_db=None, seed=7,
                                          n_targets=2, extent=4.0),
}


def scene_for(name: str) -> S.Scene:
    kw = dict(CASES[name])
    sc = S.point_target_scene(**kw)
    if name == "pt_k53_np40_24x40_noise":
        sc.grid = S.Grid(nx=24, ny=40, x0=0.3, y0=-0.2, wx=23 * 0.3, wy=39 * 0.2)
    return sc


PGA_CASES = {
    # name: (azimuth samples, edge attenuation: columns at each end scaled by 1e-3, iterations)
    "pga_cpp_64x64": (64, 0, 4),
    "pga_cpp_64x63_edges": (63, 6, 12),
}


def pga_input(n: int, edge: int) -> np.ndarray:
    """A seeded point-target image (FP64 oracle, 64 range lines) defocused by a
    quadratic + cubic azimuth phase error; `edge` columns at each azimuth end
    attenuated 60 dB so that the -30 dB window of PGA cuts them."""
    sc = S.point_target_scene(K=64, Np=64, n=64, spacing=0.12, nfft=512, snr_db=30.0, seed=12, n_targets=4,
                              extent=5.0)
    img = O.focus_fp64(sc)[0][:, :n].astype(np.complex128)
    x = np.linspace(-1.0, 1.0, n)
    phi = 4.0 * x ** 2 + 1.5 * x ** 3
    img = np.fft.ifft(np.fft.fft(img, axis=1) * np.exp(1j * phi)[None, :], axis=1)
    if edge:
        img[:, :edge] *= 1e-3
        img[:, n - edge:] *= 1e-3
    return img.astype(np.complex64)


def run_ref_pga(img: np.ndarray, iters: int):
    """The reference's compiled autofocus<float>() on img, with the rms values
    it prints captured from file descriptor 1."""
    import tempfile

    sys.stdout.flush()
    saved = os.dup(1)
    with tempfile.TemporaryFile(mode="w+") as tmp:
        os.dup2(tmp.fileno(), 1)
        try:
            out = O.ref_pga(img, iters)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        tmp.seek(0)
        rms = [float(line.split("=")[1]) for line in tmp.read().splitlines() if line.startswith("rms =")]
    return out, np.asarray(rms)


def write_pga(out_dir: str) -> None:
    for name, (n, edge, iters) in PGA_CASES.items():
        img = pga_input(n, edge)
        out, rms = run_ref_pga(img, iters)
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), image=img, iterations=iters, ref_out=out,
                            ref_rms=rms)
        print(name, "written", len(rms), "iterations")


def main() -> None:
    if not O.ref_available():
        O.build()
    out_dir = os.path.dirname(os.path.abspath(__file__))
    if "--pga" in sys.argv:
        write_pga(out_dir)
        return
    for name in CASES:
        sc = scene_for(name)
        img32, maxwy32, sf32 = O.reference_focus(sc, "f32")
        img64, maxwy64, sf64 = O.reference_focus(sc, "f64")
        g = sc.grid
        np.savez_compressed(
            os.path.join(out_dir, name + ".npz"),
            phase_history=sc.phase_history, ant_x=sc.ant_x, ant_y=sc.ant_y, ant_z=sc.ant_z,
            slant_range=sc.slant_range, start_freq=sc.start_freq, delta_freq=sc.delta_freq, nfft=sc.nfft,
            window=sc.window, grid=np.array([g.nx, g.ny, g.nz], dtype=np.int64),
            grid_geom=np.array([g.x0, g.y0, g.z0, g.wx, g.wy, g.wz], dtype=np.float64),
            ref_img_f32=img32, ref_max_wy_f32=maxwy32, ref_start_f_f32=sf32,
            ref_img_f64=img64, ref_max_wy_f64=maxwy64, ref_start_f_f64=sf64)
        print(name, "written")


if __name__ == "__main__":
    main()
