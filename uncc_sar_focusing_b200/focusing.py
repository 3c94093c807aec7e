"""Python front-end of the C ABI (include/sarbp.h).

`Plan` owns a sarbp_plan: device buffers and the FFT plan for one aperture
shape and image grid.  Arrays may be numpy arrays (host memory: the call
copies in and out and synchronises) or CUDA torch tensors (device memory:
the call is enqueued on torch's current stream and returns immediately).
Torch is only the device-memory and stream provider here; all computation
happens in libsarbp.so.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _native as N
from .scenes import CLIGHT, Grid, Scene

_PRECISION = {"mixed": N.PRECISION_MIXED, "fp64": N.PRECISION_FP64}
_WINDOW = {None: N.WINDOW_NONE, "none": N.WINDOW_NONE, "hamming": N.WINDOW_HAMMING, "taylor": N.WINDOW_TAYLOR}


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x, dtype, count: Optional[int] = None):
    """(pointer, memory kind, keep-alive) of a numpy array or CUDA tensor."""
    if _is_torch(x):
        import torch

        want = {np.float64: torch.float64, np.complex64: torch.complex64, np.complex128: torch.complex128}[dtype]
        if not x.is_cuda:
            raise ValueError("torch tensors passed to the engine must live on a CUDA device")
        if x.dtype != want or not x.is_contiguous():
            raise ValueError(f"expected a contiguous {want} tensor, got {x.dtype}")
        if count is not None and x.numel() < count:
            raise ValueError(f"tensor has {x.numel()} elements, need {count}")
        return ctypes.c_void_p(x.data_ptr()), N.MEMORY_DEVICE, x
    a = np.ascontiguousarray(x, dtype=dtype)
    if count is not None and a.size < count:
        raise ValueError(f"array has {a.size} elements, need {count}")
    return ctypes.c_void_p(a.ctypes.data), N.MEMORY_HOST, a


def _stream(*arrays):
    if any(_is_torch(a) for a in arrays):
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(0)


class Plan:
    """Device state for focusing apertures of K samples x <= num_pulses
    pulses onto one grid (sarbp_plan_create)."""

    def __init__(self, num_range_samples: int, num_pulses: int, nfft: int, max_wr: float, grid: Grid,
                 precision: str = "mixed", window: Optional[str] = "hamming", device: int = -1):
        self.K = int(num_range_samples)
        self.np_cap = int(num_pulses)
        self.nfft = int(nfft)
        self.grid = grid
        self.precision = precision
        self.image_dtype = np.complex128 if precision == "fp64" else np.complex64
        d = N.PlanDesc()
        d.num_range_samples = self.K
        d.num_pulses = self.np_cap
        d.nfft = self.nfft
        d.max_wr = float(max_wr)
        d.grid = N.Grid(grid.nx, grid.ny, grid.nz, grid.x0, grid.y0, grid.z0, grid.wx, grid.wy, grid.wz)
        d.precision = _PRECISION[precision]
        d.window = _WINDOW[window]
        d.device = int(device)
        self._desc = d
        h = ctypes.c_void_p()
        N.check(N.lib().sarbp_plan_create(ctypes.byref(d), ctypes.byref(h)), "sarbp_plan_create")
        self._h = h
        self.num_pulses_ready = 0

    @classmethod
    def for_scene(cls, scene: Scene, precision: str = "mixed", device: int = -1) -> "Plan":
        return cls(scene.num_range_samples, scene.num_pulses, scene.nfft, scene.max_wr, scene.grid,
                   precision=precision, window=scene.window, device=device)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().sarbp_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def workspace_bytes(self) -> int:
        v = ctypes.c_size_t()
        N.check(N.lib().sarbp_plan_workspace_bytes(self._h, ctypes.byref(v)), "sarbp_plan_workspace_bytes")
        return int(v.value)

    @property
    def info(self) -> dict:
        """Tiling the plan chose (sarbp_plan_get_info)."""
        v = N.PlanInfo()
        N.check(N.lib().sarbp_plan_get_info(self._h, ctypes.byref(v)), "sarbp_plan_get_info")
        return {f: getattr(v, f) for f, _ in N.PlanInfo._fields_ if f != "reserved"}

    def image_shape(self):
        g = self.grid
        return (g.nz, g.nx, g.ny)

    def new_image(self, device: Optional[str] = None):
        if device is None:
            return np.zeros(self.image_shape(), dtype=self.image_dtype)
        import torch

        dt = torch.complex128 if self.precision == "fp64" else torch.complex64
        return torch.zeros(self.image_shape(), dtype=dt, device=device)

    # -- entry points -------------------------------------------------------
    def set_range_weights(self, weights) -> None:
        """Complex per-sample range weights (a taper, a range reference
        function, or both; length K) in place of the plan's window; None
        restores the window (sarbp_plan_set_range_weights)."""
        if weights is None:
            N.check(N.lib().sarbp_plan_set_range_weights(self._h, None), "sarbp_plan_set_range_weights")
            return
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.complex128).reshape(-1))
        if w.shape[0] != self.K:
            raise ValueError(f"range weights need {self.K} values, got {w.shape[0]}")
        N.check(N.lib().sarbp_plan_set_range_weights(self._h, ctypes.c_void_p(w.ctypes.data)),
                "sarbp_plan_set_range_weights")

    def range_compress(self, phase_history) -> None:
        n = int(phase_history.shape[0])
        p, mem, keep = _ptr(phase_history, np.complex64, n * self.K)
        st = N.lib().sarbp_range_compress(self._h, p, n, mem, _stream(phase_history))
        N.check(st, "sarbp_range_compress")
        self.num_pulses_ready = n

    def range_profiles(self, out=None):
        n = self.num_pulses_ready
        dt = np.complex128 if self.precision == "fp64" else np.complex64
        if out is None:
            out = np.empty((n, self.nfft), dtype=dt)
        p, mem, keep = _ptr(out, dt, n * self.nfft)
        N.check(N.lib().sarbp_get_range_profiles(self._h, p, mem, _stream(out)), "sarbp_get_range_profiles")
        return out

    def _geometry(self, ant_x, ant_y, ant_z, slant_range, start_freq):
        n = int(ant_x.shape[0])
        ptrs = [_ptr(v, np.float64, n) for v in (ant_x, ant_y, ant_z, slant_range, start_freq)]
        mems = {m for _, m, _ in ptrs}
        if len(mems) != 1:
            raise ValueError("geometry arrays must all be host arrays or all CUDA tensors")
        g = N.Geometry(ptrs[0][0], ptrs[1][0], ptrs[2][0], ptrs[3][0], ptrs[4][0], n, mems.pop())
        return g, [k for _, _, k in ptrs]

    def backproject(self, ant_x, ant_y, ant_z, slant_range, start_freq, out=None, accumulate: bool = False,
                    checked: bool = False):
        geo, keep = self._geometry(ant_x, ant_y, ant_z, slant_range, start_freq)
        if out is None:
            out = self.new_image(None if geo.memory == N.MEMORY_HOST else "cuda")
        ip, imem, ikeep = _ptr(out, self.image_dtype, int(np.prod(self.image_shape())))
        flags = (N.ACCUMULATE if accumulate else 0) | (N.CHECKED if checked else 0)
        st = N.lib().sarbp_backproject(self._h, ctypes.byref(geo), ip, imem, flags,
                                       _stream(out, ant_x))
        N.check(st, "sarbp_backproject")
        if imem == N.MEMORY_HOST and ikeep is not out:
            np.copyto(out, ikeep.reshape(out.shape))
        return out

    def backproject_hypotheses(self, ant_x, ant_y, ant_z, slant_range, start_freq, out=None, accumulate=False):
        """Images for H antenna-track hypotheses at once: geometry arrays
        [H, Np] (hypothesis-major), images [H, nz, nx, ny]
        (sarbp_backproject_hypotheses)."""
        H, n = int(ant_x.shape[0]), int(ant_x.shape[1])
        flat = [v.reshape(-1) for v in (ant_x, ant_y, ant_z, slant_range, start_freq)]
        ptrs = [_ptr(v, np.float64, H * n) for v in flat]
        mems = {m for _, m, _ in ptrs}
        if len(mems) != 1:
            raise ValueError("geometry arrays must all be host arrays or all CUDA tensors")
        geo = N.Geometry(ptrs[0][0], ptrs[1][0], ptrs[2][0], ptrs[3][0], ptrs[4][0], n, mems.pop())
        shape = (H,) + tuple(self.image_shape())
        if out is None:
            if geo.memory == N.MEMORY_HOST:
                out = np.zeros(shape, dtype=np.complex64)
            else:
                import torch

                out = torch.zeros(shape, dtype=torch.complex64, device=ant_x.device)
        ip, imem, ikeep = _ptr(out, np.complex64, int(np.prod(shape)))
        st = N.lib().sarbp_backproject_hypotheses(self._h, ctypes.byref(geo), H, ip, imem,
                                                  N.ACCUMULATE if accumulate else 0, _stream(out, ant_x))
        N.check(st, "sarbp_backproject_hypotheses")
        if imem == N.MEMORY_HOST and ikeep is not out:
            np.copyto(out, ikeep.reshape(out.shape))
        return out

    def backproject_adjoint(self, ant_x, ant_y, ant_z, slant_range, start_freq, grad_image, accumulate=False):
        """dL/d(ant_x, ant_y, ant_z) as a [3, Np] array and dL/dR0 [Np] for a
        real loss L whose image gradient is grad_image = dL/dRe + j dL/dIm
        (sarbp_backproject_adjoint, on the plan's current range profiles)."""
        geo, keep = self._geometry(ant_x, ant_y, ant_z, slant_range, start_freq)
        gp, gmem, gkeep = _ptr(grad_image, np.complex64, int(np.prod(self.image_shape())))
        n = geo.num_pulses
        if gmem == N.MEMORY_DEVICE:
            import torch

            gant = torch.zeros((3, n), dtype=torch.float64, device=grad_image.device)
            gr0 = torch.zeros(n, dtype=torch.float64, device=grad_image.device)
            optr = (ctypes.c_void_p(gant.data_ptr()), ctypes.c_void_p(gr0.data_ptr()))
        else:
            gant = np.zeros((3, n), dtype=np.float64)
            gr0 = np.zeros(n, dtype=np.float64)
            optr = (ctypes.c_void_p(gant.ctypes.data), ctypes.c_void_p(gr0.ctypes.data))
        st = N.lib().sarbp_backproject_adjoint(self._h, ctypes.byref(geo), gp, gmem, optr[0], optr[1], gmem,
                                               N.ACCUMULATE if accumulate else 0, _stream(grad_image, ant_x))
        N.check(st, "sarbp_backproject_adjoint")
        return gant, gr0

    def focus(self, phase_history, ant_x, ant_y, ant_z, slant_range, start_freq, out=None):
        geo, keep = self._geometry(ant_x, ant_y, ant_z, slant_range, start_freq)
        if int(phase_history.shape[0]) != geo.num_pulses:
            raise ValueError("phase history and geometry disagree on the pulse count")
        pp, pmem, pkeep = _ptr(phase_history, np.complex64, geo.num_pulses * self.K)
        ap = N.Aperture(pp, pmem, geo)
        if out is None:
            out = self.new_image(None if pmem == N.MEMORY_HOST and geo.memory == N.MEMORY_HOST else "cuda")
        ip, imem, ikeep = _ptr(out, self.image_dtype, int(np.prod(self.image_shape())))
        st = N.lib().sarbp_focus(self._h, ctypes.byref(ap), ip, imem, _stream(out, phase_history, ant_x))
        N.check(st, "sarbp_focus")
        self.num_pulses_ready = geo.num_pulses
        if imem == N.MEMORY_HOST and ikeep is not out:
            np.copyto(out, ikeep.reshape(out.shape))
        return out

    # -- pipelined host-buffer focusing ---------------------------------------
    def focus_submit(self, phase_history, ant_x, ant_y, ant_z, slant_range, start_freq, out) -> int:
        """Queue range compression + backprojection of a host aperture into
        the host image `out` and return its ticket (sarbp_focus_submit).
        Upload, kernels and download of successive submissions overlap when
        the arrays are page-locked (e.g. numpy views of pinned torch tensors).
        Neither the inputs nor `out` may be touched until `focus_wait` covers
        the ticket; `out` must be a C-contiguous array of the plan's image
        dtype and shape, written in place."""
        if _is_torch(out) or not isinstance(out, np.ndarray) or out.dtype != self.image_dtype \
                or not out.flags.c_contiguous or out.size != int(np.prod(self.image_shape())):
            raise ValueError(f"out must be a C-contiguous {np.dtype(self.image_dtype)} numpy array "
                             f"of shape {self.image_shape()}")
        geo, keep = self._geometry(ant_x, ant_y, ant_z, slant_range, start_freq)
        if geo.memory != N.MEMORY_HOST:
            raise ValueError("focus_submit takes host (numpy) geometry arrays")
        if int(phase_history.shape[0]) != geo.num_pulses:
            raise ValueError("phase history and geometry disagree on the pulse count")
        pp, pmem, pkeep = _ptr(phase_history, np.complex64, geo.num_pulses * self.K)
        if pmem != N.MEMORY_HOST:
            raise ValueError("focus_submit takes a host (numpy) phase history")
        ap = N.Aperture(pp, pmem, geo)
        t = ctypes.c_ulonglong()
        st = N.lib().sarbp_focus_submit(self._h, ctypes.byref(ap), ctypes.c_void_p(out.ctypes.data),
                                        ctypes.byref(t))
        N.check(st, "sarbp_focus_submit")
        inflight = self.__dict__.setdefault("_inflight", {})
        inflight[t.value] = (keep, pkeep, out)
        # the library collected everything older than its two staging slots
        for old in [k for k in inflight if k + 2 <= t.value]:
            inflight.pop(old)
        self.num_pulses_ready = geo.num_pulses
        return t.value

    def focus_wait(self, ticket: int = 0) -> None:
        """Wait for every submission up to `ticket` (0: all) and raise the
        first error one of them recorded (sarbp_focus_wait)."""
        st = N.lib().sarbp_focus_wait(self._h, ctypes.c_ulonglong(int(ticket)))
        inflight = self.__dict__.get("_inflight", {})
        for old in [k for k in inflight if ticket == 0 or k <= ticket]:
            inflight.pop(old)
        N.check(st, "sarbp_focus_wait")

    def matched_filter(self, phase_history, ant_x, ant_y, ant_z, slant_range, start_freq, out=None):
        """Matched-filter image on the plan's grid (sarbp_matched_filter):
        nfft times the backprojection image up to its interpolation error."""
        geo, keep = self._geometry(ant_x, ant_y, ant_z, slant_range, start_freq)
        if int(phase_history.shape[0]) != geo.num_pulses:
            raise ValueError("phase history and geometry disagree on the pulse count")
        pp, pmem, pkeep = _ptr(phase_history, np.complex64, geo.num_pulses * self.K)
        ap = N.Aperture(pp, pmem, geo)
        if out is None:
            out = self.new_image(None if pmem == N.MEMORY_HOST and geo.memory == N.MEMORY_HOST else "cuda")
        ip, imem, ikeep = _ptr(out, self.image_dtype, int(np.prod(self.image_shape())))
        st = N.lib().sarbp_matched_filter(self._h, ctypes.byref(ap), ip, imem, _stream(out, phase_history, ant_x))
        N.check(st, "sarbp_matched_filter")
        if imem == N.MEMORY_HOST and ikeep is not out:
            np.copyto(out, ikeep.reshape(out.shape))
        return out

    def check(self) -> None:
        """Synchronise and raise if a kernel recorded an error."""
        import torch

        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream) if torch.cuda.is_available() else None
        N.check(N.lib().sarbp_plan_check(self._h, s), "sarbp_plan_check")


def _desc(K: int, num_pulses: int, nfft: int, max_wr: float, grid: Grid, precision: str, window, device: int):
    d = N.PlanDesc()
    d.num_range_samples = int(K)
    d.num_pulses = int(num_pulses)
    d.nfft = int(nfft)
    d.max_wr = float(max_wr)
    d.grid = N.Grid(grid.nx, grid.ny, grid.nz, grid.x0, grid.y0, grid.z0, grid.wx, grid.wy, grid.wz)
    d.precision = _PRECISION[precision]
    d.window = _WINDOW[window]
    d.device = int(device)
    return d


class Batch:
    """Independent scenes of uneven sizes focused together (sarbp_batch_*):
    one backprojection launch over all scenes' tiles, replayed as a captured
    CUDA graph.  Inputs and images are CUDA torch tensors; calls run on
    torch's current stream."""

    def __init__(self, scenes, device: int = -1):
        self.grids = [sc.grid for sc in scenes]
        self.K = [sc.num_range_samples for sc in scenes]
        descs = (N.PlanDesc * len(scenes))(*[
            _desc(sc.num_range_samples, sc.num_pulses, sc.nfft, sc.max_wr, sc.grid, "mixed", sc.window, device)
            for sc in scenes])
        h = ctypes.c_void_p()
        N.check(N.lib().sarbp_batch_create(descs, len(scenes), ctypes.byref(h)), "sarbp_batch_create")
        self._h = h
        self.n = len(scenes)
        self._keep = None

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().sarbp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def new_images(self, device="cuda"):
        import torch

        return [torch.zeros((g.nz, g.nx, g.ny), dtype=torch.complex64, device=device) for g in self.grids]

    def _args(self, apertures, images):
        if len(apertures) != self.n or len(images) != self.n:
            raise ValueError(f"need {self.n} apertures and images")
        aps = (N.Aperture * self.n)()
        keep = []
        for i, (ap, img) in enumerate(zip(apertures, images)):
            ph, ax, ay, az, r0, f0 = ap
            n = int(ax.shape[0])
            pp, pmem, pk = _ptr(ph, np.complex64, n * self.K[i])
            gp = [_ptr(v, np.float64, n) for v in (ax, ay, az, r0, f0)]
            ip, imem, ik = _ptr(img, np.complex64, int(np.prod(img.shape)))
            if pmem != N.MEMORY_DEVICE or imem != N.MEMORY_DEVICE or any(m != N.MEMORY_DEVICE for _, m, _ in gp):
                raise ValueError("batch inputs and images must be CUDA tensors")
            aps[i] = N.Aperture(pp, pmem, N.Geometry(gp[0][0], gp[1][0], gp[2][0], gp[3][0], gp[4][0], n,
                                                     N.MEMORY_DEVICE))
            keep.append((pk, ik, [k for _, _, k in gp]))
        imgs = (ctypes.c_void_p * self.n)(*[ctypes.c_void_p(img.data_ptr()) for img in images])
        return aps, imgs, keep

    def focus(self, apertures, images) -> None:
        """apertures: per scene (phase_history [Np, K] complex64, ant_x,
        ant_y, ant_z, slant_range, start_freq [Np] float64), CUDA tensors;
        images: per scene complex64 [nz, nx, ny] CUDA tensors."""
        aps, imgs, keep = self._args(apertures, images)
        st = N.lib().sarbp_batch_focus(self._h, aps, imgs, _stream(images[0]))
        N.check(st, "sarbp_batch_focus")
        self._keep = keep

    def wait(self):
        """Wait for the last focus; per-image completion times (ms after the
        call's start, GPU clock) as a numpy array."""
        ms = (ctypes.c_double * self.n)()
        N.check(N.lib().sarbp_batch_wait(self._h, ms), "sarbp_batch_wait")
        return np.array(ms[:], dtype=np.float64)

    def autotune(self, apertures, images) -> float:
        aps, imgs, keep = self._args(apertures, images)
        best = ctypes.c_double()
        st = N.lib().sarbp_batch_autotune(self._h, aps, imgs, _stream(images[0]), ctypes.byref(best))
        N.check(st, "sarbp_batch_autotune")
        return float(best.value)

    def set_schedule(self, per_tile: Optional[bool]) -> None:
        """True: one CTA per tile in scene order; False: units split over the
        resident CTAs; None: automatic."""
        v = -1 if per_tile is None else int(bool(per_tile))
        N.check(N.lib().sarbp_batch_set_schedule(self._h, v), "sarbp_batch_set_schedule")

    @property
    def info(self) -> dict:
        v = N.BatchInfo()
        N.check(N.lib().sarbp_batch_get_info(self._h, ctypes.byref(v)), "sarbp_batch_get_info")
        return {f: getattr(v, f) for f, _ in N.BatchInfo._fields_ if f != "reserved"}


def focus_scene(scene: Scene, precision: str = "mixed") -> np.ndarray:
    """Focus a scene through host buffers (sarbp_focus on host memory)."""
    with Plan.for_scene(scene, precision) as plan:
        return plan.focus(scene.phase_history, scene.ant_x, scene.ant_y, scene.ant_z, scene.slant_range,
                          scene.start_freq)


def polar_format_phase_history(phase_history, chirp_rate, adc_rate: float, center_freq: float):
    """The reference's polar-format algorithm is backprojection of a phase
    history whose pulses are first modulated (matlab/focusalg_PF.m:33-35; the
    rest of that file is focusalg_BP's): pulse p of Np is multiplied by
    exp(-2j pi s_pk / Np) with frequency scales
    s_pk = 1 + (chirp_rate_p / (adc_rate * center_freq)) (k - K/2), k = 0..K-1
    (matlab/formSARImage.m:217-220,341, where the degree-to-radian factors of
    the chirp rate and centre frequency cancel).  Returns the modulated phase
    history ([Np, K] complex64, numpy array or torch tensor like the input);
    focus it with Plan.focus / sarbp_focus as any other.

    chirp_rate: per-pulse chirp rates [Np] (or one value), in the units of
    adc_rate * center_freq (Sandia: ChirpRate, ADF, DesCntrFreq)."""
    np_, K = int(phase_history.shape[0]), int(phase_history.shape[1])
    rates = np.broadcast_to(np.asarray(chirp_rate, dtype=np.float64), (np_,))
    k = np.arange(K, dtype=np.float64) - K / 2.0
    scales = 1.0 + (rates[:, None] / (adc_rate * center_freq)) * k[None, :]
    mod = np.exp((-2j * np.pi / np_) * scales)
    if isinstance(phase_history, np.ndarray):
        return (phase_history.astype(np.complex128) * mod).astype(np.complex64)
    import torch

    m = torch.as_tensor(mod, dtype=torch.complex128, device=phase_history.device)
    return (phase_history.to(torch.complex128) * m).to(torch.complex64)
