"""Seeded synthetic stepped-frequency phase histories.

The scene model is the reference's point-target synthesis
(matlab/formImagePointTargetBP.m:44-81):

    ph[p, k] = sum_t A_t * exp(-j * 4*pi * f_k * (|a_p - x_t| - R0_p) / c)

with f_k = linspace(fc - BW/2, fc + BW/2, K) (:45), antenna positions on a
circular track a_p = R * (cos el cos az_p, cos el sin az_p, sin el) (sph2cart,
:50-52), R0_p = R (:88) and per-pulse start frequency f_0 (:94).  Antenna and
target positions are float64; the phase history is rounded to complex64 like
the reference's SAR_Aperture<float>::sampleData (include/uncc_sar_focusing.hpp:68).
Noise is circular complex Gaussian at the requested SNR.

The named configurations are the workloads the engine is measured on: a
point-target scene (424 x 512, 256^2 image), a large scene (1024 x 2048, 2000
Rayleigh scatterers, 1024^2 image), a volumetric multi-pass scene, a
motion-error autofocus scene and a batched scene.  No public dataset is used;
the reference's real-data paths (include/uncc_sar_globals.hpp:35-47) are not
available, so every input is generated here from a seed.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Sequence

import numpy as np

CLIGHT = 299792458.0  # include/uncc_sar_focusing.hpp:34


@dataclasses.dataclass
class Grid:
    """Image grid: pixel i along x sits at x0 - wx/2 + i*wx/(nx-1) (linspace),
    the same rule as cpuBackProjection.hpp:55-62; nz == 1 means the plane z = z0.
    Images are laid out [nz][nx][ny] (x-major within a slice, img[x*Ny + y])."""

    nx: int
    ny: int
    nz: int = 1
    x0: float = 0.0
    y0: float = 0.0
    z0: float = 0.0
    wx: float = 0.0
    wy: float = 0.0
    wz: float = 0.0

    @property
    def npix(self) -> int:
        return self.nx * self.ny * self.nz

    def axis(self, which: str) -> np.ndarray:
        n, c, w = {"x": (self.nx, self.x0, self.wx), "y": (self.ny, self.y0, self.wy),
                   "z": (self.nz, self.z0, self.wz)}[which]
        if n == 1:
            return np.array([c], dtype=np.float64)
        return (c - 0.5 * w) + np.arange(n, dtype=np.float64) * (w / (n - 1))


@dataclasses.dataclass
class Scene:
    """One aperture plus its image-formation parameters."""

    name: str
    phase_history: np.ndarray  # complex64 [Np, K], frequency fastest
    ant_x: np.ndarray  # float64 [Np]
    ant_y: np.ndarray
    ant_z: np.ndarray
    slant_range: np.ndarray  # R0, float64 [Np]
    start_freq: np.ndarray  # f0, float64 [Np]
    delta_freq: float  # Hz
    nfft: int
    grid: Grid
    window: str = "hamming"
    targets: Optional[np.ndarray] = None  # float64 [T, 3]
    amplitudes: Optional[np.ndarray] = None  # complex128 [T]
    seed: int = 0

    @property
    def num_pulses(self) -> int:
        return int(self.phase_history.shape[0])

    @property
    def num_range_samples(self) -> int:
        return int(self.phase_history.shape[1])

    @property
    def max_wr(self) -> float:
        """Range-profile extent c / (2 dF) (SAR_ImageFormationParameters::update,
        include/uncc_sar_focusing.hpp:429)."""
        return CLIGHT / (2.0 * self.delta_freq)

    @property
    def pixel_pulses(self) -> int:
        return self.grid.npix * self.num_pulses


def circular_track(num_pulses: int, radius: float, el_deg, az_center_deg: float, az_span_deg: float):
    """Antenna phase centres on a circle (formImagePointTargetBP.m:47-52)."""
    az = np.deg2rad(np.linspace(az_center_deg - az_span_deg / 2.0, az_center_deg + az_span_deg / 2.0,
                                num_pulses))
    el = np.deg2rad(np.broadcast_to(np.asarray(el_deg, dtype=np.float64), az.shape))
    x = radius * np.cos(el) * np.cos(az)
    y = radius * np.cos(el) * np.sin(az)
    z = radius * np.sin(el)
    return x, y, z


def synthesize_phase_history(freqs: np.ndarray, ant: np.ndarray, r0: np.ndarray, targets: np.ndarray,
                             amps: np.ndarray, device: Optional[str] = None) -> np.ndarray:
    """sum_t A_t exp(-j 4 pi f_k dR_pt / c) in float64, returned as complex64 [Np, K].

    device=None computes with numpy; device="cuda" uses torch float64 on the
    GPU (input generation only, for the large scenes)."""
    npulse = ant.shape[0]
    K = freqs.shape[0]
    if device is None:
        out = np.zeros((npulse, K), dtype=np.complex128)
        kf = (-4.0 * math.pi / CLIGHT) * freqs[None, :]
        for t in range(targets.shape[0]):
            d = ant - targets[t][None, :]
            dR = np.sqrt(np.sum(d * d, axis=1)) - r0
            out += amps[t] * np.exp(1j * (dR[:, None] * kf))
        return out.astype(np.complex64)
    import torch

    dev = torch.device(device)
    f = torch.as_tensor(freqs, dtype=torch.float64, device=dev)
    a = torch.as_tensor(ant, dtype=torch.float64, device=dev)
    r = torch.as_tensor(r0, dtype=torch.float64, device=dev)
    tg = torch.as_tensor(targets, dtype=torch.float64, device=dev)
    am = torch.as_tensor(amps, dtype=torch.complex128, device=dev)
    acc_re = torch.zeros((npulse, K), dtype=torch.float64, device=dev)
    acc_im = torch.zeros((npulse, K), dtype=torch.float64, device=dev)
    kf = (-4.0 * math.pi / CLIGHT) * f
    chunk = max(1, int(2**28 // max(1, npulse * K)))
    for t0 in range(0, tg.shape[0], chunk):
        t1 = min(tg.shape[0], t0 + chunk)
        d = a[:, None, :] - tg[None, t0:t1, :]
        dR = torch.sqrt((d * d).sum(-1)) - r[:, None]  # [Np, T]
        ph = dR[:, :, None] * kf[None, None, :]  # [Np, T, K]
        c, s = torch.cos(ph), torch.sin(ph)
        ar, ai = am[t0:t1].real[None, :, None], am[t0:t1].imag[None, :, None]
        acc_re += (ar * c - ai * s).sum(1)
        acc_im += (ar * s + ai * c).sum(1)
    out = torch.complex(acc_re, acc_im).to(torch.complex64).cpu().numpy()
    return out


def add_noise(ph: np.ndarray, snr_db: Optional[float], rng: np.random.Generator) -> np.ndarray:
    if snr_db is None:
        return ph
    p_sig = float(np.mean(np.abs(ph.astype(np.complex128)) ** 2))
    sigma2 = p_sig * 10.0 ** (-snr_db / 10.0)
    noise = (rng.standard_normal(ph.shape) + 1j * rng.standard_normal(ph.shape)) * math.sqrt(sigma2 / 2.0)
    return (ph.astype(np.complex128) + noise).astype(np.complex64)


def make_scene(name: str, *, fc: float, bw: float, K: int, Np: int, radius: float, el_deg,
               az_center_deg: float, az_span_deg: float, targets: np.ndarray, amps: np.ndarray,
               nfft: int, grid: Grid, snr_db: Optional[float], seed: int, window: str = "hamming",
               device: Optional[str] = None, rng: Optional[np.random.Generator] = None) -> Scene:
    rng = rng if rng is not None else np.random.default_rng(seed)
    freqs = np.linspace(fc - bw / 2.0, fc + bw / 2.0, K)
    ax, ay, az = circular_track(Np, radius, el_deg, az_center_deg, az_span_deg)
    r0 = np.full(Np, float(radius))
    ant = np.stack([ax, ay, az], axis=1)
    ph = synthesize_phase_history(freqs, ant, r0, targets, amps, device=device)
    ph = add_noise(ph, snr_db, rng)
    return Scene(name=name, phase_history=np.ascontiguousarray(ph), ant_x=ax, ant_y=ay, ant_z=az,
                 slant_range=r0, start_freq=np.full(Np, freqs[0]), delta_freq=float(freqs[1] - freqs[0]),
                 nfft=nfft, grid=grid, window=window, targets=targets, amplitudes=amps, seed=seed)


def point_target_scene(K: int = 424, Np: int = 512, n: int = 256, spacing: float = 0.08, n_targets: int = 5,
                       nfft: Optional[int] = None, snr_db: Optional[float] = 20.0, seed: int = 1,
                       az_span_deg: float = 4.0, radius: float = 10e3, el_deg: float = 30.0,
                       fc: float = 9.6e9, bw: float = 600e6, extent: float = 20.0,
                       device: Optional[str] = None) -> Scene:
    """Point-target scene: X-band stepped frequency, circular aperture, unit
    targets uniform over an extent x extent metre patch at z = 0, 8x range
    upsampling and a Hamming taper by default."""
    rng = np.random.default_rng(seed)
    tg = np.zeros((n_targets, 3))
    tg[:, :2] = rng.uniform(-extent / 2.0, extent / 2.0, size=(n_targets, 2))
    amps = np.ones(n_targets, dtype=np.complex128)
    w = spacing * (n - 1)
    grid = Grid(nx=n, ny=n, wx=w, wy=w)
    return make_scene("point_targets", fc=fc, bw=bw, K=K, Np=Np, radius=radius, el_deg=el_deg,
                      az_center_deg=0.0, az_span_deg=az_span_deg, targets=tg, amps=amps,
                      nfft=nfft if nfft is not None else 8 * K, grid=grid, snr_db=snr_db, seed=seed,
                      device=device, rng=rng)


def large_scene(K: int = 1024, Np: int = 2048, n: int = 1024, n_targets: int = 2000, extent: float = 100.0,
                nfft: Optional[int] = None, seed: int = 2, device: Optional[str] = None) -> Scene:
    """Large scene: fc 9.6 GHz, 640 MHz, 30 deg of azimuth at 8 km and 45 deg
    elevation; Rayleigh(sigma=1) amplitudes with uniform phase; n x n image
    over extent metres; Nfft = 8K unless given."""
    rng = np.random.default_rng(seed)
    tg = np.zeros((n_targets, 3))
    tg[:, :2] = rng.uniform(-extent / 2.0, extent / 2.0, size=(n_targets, 2))
    amps = rng.rayleigh(1.0, n_targets) * np.exp(1j * rng.uniform(0.0, 2.0 * math.pi, n_targets))
    grid = Grid(nx=n, ny=n, wx=extent, wy=extent)
    return make_scene("large", fc=9.6e9, bw=640e6, K=K, Np=Np, radius=8e3, el_deg=45.0, az_center_deg=0.0,
                      az_span_deg=30.0, targets=tg, amps=amps, nfft=nfft if nfft is not None else 8 * K,
                      grid=grid, snr_db=None, seed=seed, device=device, rng=rng)


def volumetric_scene(K: int = 512, pulses_per_pass: int = 1024, elevations: Sequence[float] = tuple(
        30.0 + 0.2 * i for i in range(8)), nx: int = 256, ny: int = 256, nz: int = 64, cube: float = 10.0,
                     n_targets: int = 500, nfft: Optional[int] = None, seed: int = 3, radius: float = 10e3,
                     device: Optional[str] = None) -> Scene:
    """Multi-pass circular collection over a cube; scatterers on random planar
    facets; voxel output [nz][nx][ny]."""
    rng = np.random.default_rng(seed)
    n_facets = 10
    per = int(math.ceil(n_targets / n_facets))
    pts = []
    for _ in range(n_facets):
        c = rng.uniform(-cube / 2.0, cube / 2.0, 3) * 0.6
        nrm = rng.standard_normal(3)
        nrm /= np.linalg.norm(nrm)
        u = np.cross(nrm, [0.0, 0.0, 1.0] if abs(nrm[2]) < 0.9 else [1.0, 0.0, 0.0])
        u /= np.linalg.norm(u)
        v = np.cross(nrm, u)
        s, t = rng.uniform(-cube / 5.0, cube / 5.0, (2, per))
        pts.append(c[None, :] + s[:, None] * u[None, :] + t[:, None] * v[None, :])
    tg = np.clip(np.concatenate(pts)[:n_targets], -cube / 2.0, cube / 2.0)
    amps = rng.rayleigh(1.0, n_targets) * np.exp(1j * rng.uniform(0.0, 2.0 * math.pi, n_targets))
    el = np.repeat(np.asarray(elevations, dtype=np.float64), pulses_per_pass)
    npass = len(elevations)
    az = np.tile(np.linspace(-180.0, 180.0, pulses_per_pass, endpoint=False), npass)
    Np = npass * pulses_per_pass
    freqs = np.linspace(9.6e9 - 300e6, 9.6e9 + 300e6, K)
    ax = radius * np.cos(np.deg2rad(el)) * np.cos(np.deg2rad(az))
    ay = radius * np.cos(np.deg2rad(el)) * np.sin(np.deg2rad(az))
    azz = radius * np.sin(np.deg2rad(el))
    r0 = np.full(Np, radius)
    ph = synthesize_phase_history(freqs, np.stack([ax, ay, azz], 1), r0, tg, amps, device=device)
    grid = Grid(nx=nx, ny=ny, nz=nz, wx=cube, wy=cube, wz=cube)
    return Scene(name="volumetric", phase_history=ph, ant_x=ax, ant_y=ay, ant_z=azz, slant_range=r0,
                 start_freq=np.full(Np, freqs[0]), delta_freq=float(freqs[1] - freqs[0]),
                 nfft=nfft if nfft is not None else 8 * K, grid=grid, targets=tg, amplitudes=amps, seed=seed)


def slow_time(num_pulses: int) -> np.ndarray:
    """Normalised slow time tau in [-1, 1] over the aperture."""
    return np.linspace(-1.0, 1.0, num_pulses)


def cubic_track_error(coeffs: np.ndarray, tau: np.ndarray) -> np.ndarray:
    """[3, Np] position error sum_n c[axis, n] tau^n, n = 0..3 (c is [3, 4])."""
    powers = np.stack([tau ** n for n in range(4)])  # [4, Np]
    return np.asarray(coeffs, dtype=np.float64) @ powers


def motion_error_scene(K: int = 512, Np: int = 1024, n: int = 512, spacing: float = 0.08, peak: float = 1.5,
                       walk_sigma: float = 1e-3, seed: int = 4, snr_db: Optional[float] = 20.0,
                       n_targets: int = 5, extent: float = 20.0, device: Optional[str] = None) -> Scene:
    """Autofocus scene: the point-target geometry (9.6 GHz, 600 MHz, 4 deg at
    10 km, 30 deg elevation) with Np pulses of K samples, where the phase
    history is synthesised from the TRUE antenna track and the scene carries
    the MEASURED track (ant_x/y/z) the focuser is given:
        true = measured + e(tau),  e = cubic in slow time per axis (seeded,
        max |e| <= peak metres on each axis) + Gaussian random walk
        (walk_sigma metres per pulse).
    The true cubic coefficients and the full error are attached as
    scene.true_cubic [3, 4] and scene.true_error [3, Np]."""
    rng = np.random.default_rng(seed)
    tg = np.zeros((n_targets, 3))
    tg[:, :2] = rng.uniform(-extent / 2.0, extent / 2.0, size=(n_targets, 2))
    amps = np.ones(n_targets, dtype=np.complex128)
    fc, bw, radius, el = 9.6e9, 600e6, 10e3, 30.0
    freqs = np.linspace(fc - bw / 2.0, fc + bw / 2.0, K)
    ax, ay, az = circular_track(Np, radius, el, 0.0, 4.0)
    measured = np.stack([ax, ay, az])
    tau = slow_time(Np)
    coeffs = rng.uniform(-1.0, 1.0, size=(3, 4))
    cub = cubic_track_error(coeffs, tau)
    coeffs = coeffs * (peak / np.abs(cub).max(axis=1, keepdims=True))
    walk = np.cumsum(rng.normal(0.0, walk_sigma, size=(3, Np)), axis=1)
    err = cubic_track_error(coeffs, tau) + walk
    true = measured + err
    r0 = np.full(Np, radius)
    ph = synthesize_phase_history(freqs, true.T.copy(), r0, tg, amps, device=device)
    ph = add_noise(ph, snr_db, rng)
    w = spacing * (n - 1)
    sc = Scene(name="motion_error", phase_history=np.ascontiguousarray(ph), ant_x=ax, ant_y=ay, ant_z=az,
               slant_range=r0, start_freq=np.full(Np, freqs[0]), delta_freq=float(freqs[1] - freqs[0]),
               nfft=8 * K, grid=Grid(nx=n, ny=n, wx=w, wy=w), targets=tg, amplitudes=amps, seed=seed)
    sc.true_cubic = coeffs
    sc.true_error = err
    return sc
