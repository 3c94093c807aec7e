"""MAT-file ingest of phase-history data, without matio.

The reference reads two layouts with matio (include/uncc_sar_matio.hpp:
133-196, read_MAT_Variables :250-285) and completes the aperture in
initialize_SAR_Aperture_Data (include/uncc_sar_focusing.hpp:224-393):

* GOTCHA (AFRL, `data` struct): data.fp (K x Np complex, frequency fastest),
  data.freq (K, or K x Np), data.x / .y / .z (antenna, Np), data.r0 (slant
  range to scene centre, Np), data.th, data.phi (angles), data.af.r_correct
  and data.af.ph_correct (autofocus corrections, carried along, not used for
  focusing, as in the reference).
* Sandia (`sph_MATData` struct): Data.SampleData (K x Np complex),
  Data.StartF, Data.ChirpRate (Np), Data.radarCoordinateFrame.x / .y / .z,
  preamble.ADF (A/D sample rate): freq[k] = StartF + k ChirpRate / ADF, the
  derived-frequency path of :281-307.

Completion as the reference does it: a K-vector of frequencies is shared by
every pulse with start frequency min(freq) and step |freq[1] - freq[0]|
(:246-280); a missing slant range becomes |antenna| (:311-321); the range
extent is max_wr = c / (2 mean deltaF) (SAR_ImageFormationParameters::update,
:430).  Files are read with scipy.io (MAT levels 4 and 5, which covers the
-v6 and -v7 formats); -v7.3 files are HDF5 and need an HDF5 reader this
package does not carry: load() rejects them with a message to re-save with
-v7.  `save_gotcha` / `save_sandia` write the same layouts (fixtures and
converters).
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Optional

import numpy as np

from . import scenes as S

CLIGHT = S.CLIGHT


@dataclasses.dataclass
class MatAperture:
    layout: str                      # "gotcha" or "sandia"
    phase_history: np.ndarray        # complex64 [Np, K]
    ant_x: np.ndarray                # float64 [Np]
    ant_y: np.ndarray
    ant_z: np.ndarray
    slant_range: np.ndarray          # float64 [Np]
    start_freq: np.ndarray           # float64 [Np]
    delta_freq: np.ndarray           # float64 [Np], Hz per sample
    freq: np.ndarray                 # float64 [Np, K]
    extra: Dict[str, np.ndarray] = dataclasses.field(default_factory=dict)  # th, phi, af_*

    @property
    def num_pulses(self) -> int:
        return int(self.phase_history.shape[0])

    @property
    def num_range_samples(self) -> int:
        return int(self.phase_history.shape[1])

    @property
    def mean_delta_freq(self) -> float:
        return float(np.mean(self.delta_freq))

    @property
    def max_wr(self) -> float:
        """Range extent of the profiles, c / (2 mean deltaF) (m)."""
        return CLIGHT / (2.0 * self.mean_delta_freq)

    def to_scene(self, grid: S.Grid, nfft: Optional[int] = None, window: Optional[str] = "hamming") -> S.Scene:
        """A scenes.Scene for the focusing engine (nfft defaults to 8 K, the
        zero-padding of matlab/formImage3DSAR.m:115-116)."""
        K = self.num_range_samples
        return S.Scene(name=f"mat:{self.layout}", phase_history=np.ascontiguousarray(self.phase_history),
                       ant_x=self.ant_x, ant_y=self.ant_y, ant_z=self.ant_z, slant_range=self.slant_range,
                       start_freq=self.start_freq, delta_freq=self.mean_delta_freq,
                       nfft=int(nfft) if nfft else 8 * K, grid=grid, window=window)


def _vec(a) -> np.ndarray:
    return np.asarray(a, dtype=np.float64).reshape(-1)


def _field(obj, path: str):
    for part in path.split("."):
        if obj is None:
            return None
        if isinstance(obj, dict):
            obj = obj.get(part)
        else:
            obj = getattr(obj, part, None)
    return obj


def _complex_kxnp(a, name: str) -> np.ndarray:
    a = np.asarray(a)
    if not np.iscomplexobj(a):
        raise ValueError(f"{name} is not complex-valued")
    if a.ndim == 1:
        a = a[:, None]
    return np.ascontiguousarray(a.T.astype(np.complex64))  # MATLAB K x Np -> [Np, K]


def _from_gotcha(d) -> MatAperture:
    ph = _complex_kxnp(_field(d, "fp"), "data.fp")
    Np, K = ph.shape
    ax, ay, az = (_vec(_field(d, a)) for a in ("x", "y", "z"))
    if not (ax.size == ay.size == az.size == Np):
        raise ValueError(f"antenna positions hold {ax.size}/{ay.size}/{az.size} values for {Np} pulses")
    freq = np.asarray(_field(d, "freq"), dtype=np.float64)
    if freq.ndim <= 1 or 1 in freq.shape:
        f = freq.reshape(-1)
        if f.size != K:
            raise ValueError(f"data.freq holds {f.size} values for {K} samples per pulse")
        fmat = np.tile(f, (Np, 1))
        start = np.full(Np, f.min())
        step = np.full(Np, abs(f[1] - f[0]) if K > 1 else 0.0)
    else:
        if freq.shape != (K, Np):
            raise ValueError(f"data.freq is {freq.shape}, expected ({K}, {Np})")
        fmat = np.ascontiguousarray(freq.T)
        start = fmat.min(axis=1)
        step = np.abs(fmat[:, 1] - fmat[:, 0]) if K > 1 else np.zeros(Np)
    r0 = _field(d, "r0")
    r0 = _vec(r0) if r0 is not None and np.size(r0) == Np else np.sqrt(ax * ax + ay * ay + az * az)
    extra = {}
    for key, path in (("th", "th"), ("phi", "phi"), ("af_r_correct", "af.r_correct"),
                      ("af_ph_correct", "af.ph_correct")):
        v = _field(d, path)
        if v is not None:
            extra[key] = _vec(v)
    return MatAperture("gotcha", ph, ax, ay, az, r0, start, step, fmat, extra)


def _from_sandia(s) -> MatAperture:
    ph = _complex_kxnp(_field(s, "Data.SampleData"), "sph_MATData.Data.SampleData")
    Np, K = ph.shape
    ax, ay, az = (_vec(_field(s, f"Data.radarCoordinateFrame.{a}")) for a in ("x", "y", "z"))
    start = _vec(_field(s, "Data.StartF"))
    chirp = _vec(_field(s, "Data.ChirpRate"))
    adf = _vec(_field(s, "preamble.ADF"))
    if not (ax.size == ay.size == az.size == start.size == chirp.size == Np) or adf.size != 1:
        raise ValueError("Sandia fields do not hold one value per pulse (ADF: one value)")
    step = chirp / adf[0]
    if not np.all(step > 0):
        raise ValueError("non-positive ChirpRate / ADF: frequencies must increase along a pulse")
    fmat = start[:, None] + np.arange(K)[None, :] * step[:, None]
    r0 = np.sqrt(ax * ax + ay * ay + az * az)
    return MatAperture("sandia", ph, ax, ay, az, r0, start, step, fmat, {})


def load(path: str) -> MatAperture:
    """Read a GOTCHA or Sandia phase-history MAT file."""
    import scipy.io

    with open(path, "rb") as fh:
        head = fh.read(128)
    if len(head) == 128 and head[124:126] in (b"\x00\x02", b"\x02\x00"):
        raise ValueError(f"{path} is a MAT -v7.3 (HDF5) file; re-save it with save(..., '-v7')")
    m = scipy.io.loadmat(path, squeeze_me=True, struct_as_record=False)
    if "sph_MATData" in m:
        return _from_sandia(m["sph_MATData"])
    if "data" in m:
        return _from_gotcha(m["data"])
    raise ValueError(f"{path}: neither a GOTCHA `data` nor a Sandia `sph_MATData` struct "
                     f"(variables: {sorted(k for k in m if not k.startswith('__'))})")


def save_gotcha(path: str, phase_history, freq, ant_x, ant_y, ant_z, r0=None, th=None, phi=None,
                r_correct=None, ph_correct=None) -> None:
    """Write the GOTCHA layout (phase_history [Np, K] -> data.fp K x Np)."""
    import scipy.io

    d = {"fp": np.asarray(phase_history).T, "freq": np.asarray(freq, dtype=np.float64),
         "x": _vec(ant_x), "y": _vec(ant_y), "z": _vec(ant_z)}
    if r0 is not None:
        d["r0"] = _vec(r0)
    if th is not None:
        d["th"] = _vec(th)
    if phi is not None:
        d["phi"] = _vec(phi)
    if r_correct is not None or ph_correct is not None:
        d["af"] = {"r_correct": _vec(r_correct if r_correct is not None else []),
                   "ph_correct": _vec(ph_correct if ph_correct is not None else [])}
    scipy.io.savemat(path, {"data": d}, do_compression=True)


def save_sandia(path: str, phase_history, start_freq, chirp_rate, adf, ant_x, ant_y, ant_z) -> None:
    """Write the Sandia layout (phase_history [Np, K] -> Data.SampleData K x Np)."""
    import scipy.io

    s = {"Data": {"SampleData": np.asarray(phase_history).T, "StartF": _vec(start_freq),
                  "ChirpRate": _vec(chirp_rate),
                  "radarCoordinateFrame": {"x": _vec(ant_x), "y": _vec(ant_y), "z": _vec(ant_z)}},
         "preamble": {"ADF": float(adf)}}
    scipy.io.savemat(path, {"sph_MATData": s}, do_compression=True)
