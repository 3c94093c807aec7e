"""ctypes binding of lib/libsarbp.so (include/sarbp.h).

The library is the product: there is no Python or CPU fallback.  Loading
fails with a RuntimeError when it has not been built.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsarbp.so")
ABI_VERSION = 1  # SARBP_ABI_VERSION of the include/sarbp.h these structures mirror
COMPAT_PATH = os.path.join(HERE, "lib", "libsarbp_compat.so")

SARBP_OK = 0
SARBP_ERR_INVALID_ARGUMENT = 1
SARBP_ERR_NULL_POINTER = 2
SARBP_ERR_UNSUPPORTED = 3
SARBP_ERR_OUT_OF_MEMORY = 4
SARBP_ERR_CUDA = 5
SARBP_ERR_CUFFT = 6
SARBP_ERR_NOT_FINITE = 7
SARBP_ERR_KERNEL_TIMEOUT = 8
SARBP_ERR_KERNEL_BOUNDS = 9
SARBP_ERR_NO_DEVICE = 10

PRECISION_MIXED = 0
PRECISION_FP64 = 1
WINDOW_NONE = 0
WINDOW_HAMMING = 1
WINDOW_TAYLOR = 2
MEMORY_HOST = 0
MEMORY_DEVICE = 1
ACCUMULATE = 1
CHECKED = 2

# Every symbol include/sarbp.h declares (tests check the library exports them).
EXPORTED = (
    "sarbp_abi_version", "sarbp_status_string", "sarbp_plan_create", "sarbp_plan_destroy",
    "sarbp_plan_workspace_bytes", "sarbp_range_compress", "sarbp_get_range_profiles", "sarbp_backproject",
    "sarbp_focus", "sarbp_focus_image", "sarbp_plan_check", "sarbp_backproject_noalloc",
    "sarbp_backproject_adjoint", "sarbp_backproject_hypotheses", "sarbp_focus_submit", "sarbp_focus_wait", "sarbp_plan_get_info",
    "sarbp_batch_create", "sarbp_batch_destroy", "sarbp_batch_focus", "sarbp_batch_wait", "sarbp_batch_autotune",
    "sarbp_batch_get_info", "sarbp_batch_set_schedule", "sarbp_matched_filter", "sarbp_plan_set_range_weights",
    "sarbp_test_fail_device_alloc", "sarbp_test_drop_window_copy", "sarbp_image_entropy_work_bytes",
    "sarbp_image_entropy", "sarbp_image_entropy_grad",
)


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("x0", ctypes.c_double), ("y0", ctypes.c_double), ("z0", ctypes.c_double),
                ("wx", ctypes.c_double), ("wy", ctypes.c_double), ("wz", ctypes.c_double)]


class PlanDesc(ctypes.Structure):
    _fields_ = [("num_range_samples", ctypes.c_int), ("num_pulses", ctypes.c_int), ("nfft", ctypes.c_int),
                ("max_wr", ctypes.c_double), ("grid", Grid), ("precision", ctypes.c_int),
                ("window", ctypes.c_int), ("device", ctypes.c_int), ("reserved", ctypes.c_int * 4)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("tile_mx", ctypes.c_int), ("stage_pulses", ctypes.c_int), ("window_bins", ctypes.c_int),
                ("resident_ctas", ctypes.c_int), ("tiles", ctypes.c_longlong), ("smem_bytes", ctypes.c_longlong),
                ("kernels_per_backproject", ctypes.c_int), ("fused_range_compression", ctypes.c_int),
                ("reserved", ctypes.c_int * 4)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("num_scenes", ctypes.c_int), ("tile_mx", ctypes.c_int), ("stage_pulses", ctypes.c_int),
                ("max_window_bins", ctypes.c_int), ("resident_ctas", ctypes.c_int), ("graph", ctypes.c_int),
                ("tiles", ctypes.c_longlong), ("units", ctypes.c_longlong), ("smem_bytes", ctypes.c_longlong),
                ("workspace_bytes", ctypes.c_longlong), ("per_tile", ctypes.c_int), ("reserved", ctypes.c_int * 3)]


class Geometry(ctypes.Structure):
    _fields_ = [("ant_x", ctypes.c_void_p), ("ant_y", ctypes.c_void_p), ("ant_z", ctypes.c_void_p),
                ("slant_range", ctypes.c_void_p), ("start_freq", ctypes.c_void_p),
                ("num_pulses", ctypes.c_int), ("memory", ctypes.c_int)]


class Aperture(ctypes.Structure):
    _fields_ = [("phase_history", ctypes.c_void_p), ("phase_history_memory", ctypes.c_int),
                ("geometry", Geometry)]


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m uncc_sar_focusing_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
        L.sarbp_abi_version.restype = i
        if L.sarbp_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI version {L.sarbp_abi_version()}, these bindings mirror "
                               f"version {ABI_VERSION} (include/sarbp.h): rebuild the library")
        L.sarbp_status_string.restype = ctypes.c_char_p
        L.sarbp_status_string.argtypes = [i]
        L.sarbp_plan_create.argtypes = [P(PlanDesc), P(vp)]
        L.sarbp_plan_destroy.argtypes = [vp]
        L.sarbp_plan_workspace_bytes.argtypes = [vp, P(ctypes.c_size_t)]
        L.sarbp_range_compress.argtypes = [vp, vp, i, i, vp]
        L.sarbp_get_range_profiles.argtypes = [vp, vp, i, vp]
        L.sarbp_backproject.argtypes = [vp, P(Geometry), vp, i, i, vp]
        L.sarbp_focus.argtypes = [vp, P(Aperture), vp, i, vp]
        L.sarbp_focus_image.argtypes = [P(PlanDesc), P(Aperture), vp, i]
        L.sarbp_plan_check.argtypes = [vp, vp]
        L.sarbp_backproject_noalloc.argtypes = [P(PlanDesc), vp, P(Geometry), vp, i, vp]
        L.sarbp_backproject_adjoint.argtypes = [vp, P(Geometry), vp, i, vp, vp, i, i, vp]
        L.sarbp_backproject_hypotheses.argtypes = [vp, P(Geometry), i, vp, i, i, vp]
        L.sarbp_focus_submit.argtypes = [vp, P(Aperture), vp, P(ctypes.c_ulonglong)]
        L.sarbp_focus_wait.argtypes = [vp, ctypes.c_ulonglong]
        L.sarbp_plan_get_info.argtypes = [vp, P(PlanInfo)]
        L.sarbp_batch_create.argtypes = [P(PlanDesc), i, P(vp)]
        L.sarbp_batch_destroy.argtypes = [vp]
        L.sarbp_batch_focus.argtypes = [vp, P(Aperture), P(vp), vp]
        L.sarbp_batch_wait.argtypes = [vp, P(ctypes.c_double)]
        L.sarbp_batch_autotune.argtypes = [vp, P(Aperture), P(vp), vp, P(ctypes.c_double)]
        L.sarbp_batch_get_info.argtypes = [vp, P(BatchInfo)]
        L.sarbp_batch_set_schedule.argtypes = [vp, i]
        L.sarbp_matched_filter.argtypes = [vp, P(Aperture), vp, i, vp]
        L.sarbp_plan_set_range_weights.argtypes = [vp, vp]
        L.sarbp_test_fail_device_alloc.argtypes = [i]
        L.sarbp_test_drop_window_copy.argtypes = [vp, i]
        L.sarbp_image_entropy_work_bytes.argtypes = []
        L.sarbp_image_entropy.argtypes = [vp, ctypes.c_longlong, vp, vp, vp]
        L.sarbp_image_entropy_grad.argtypes = [vp, ctypes.c_longlong, vp, vp, vp, vp]
        for name in EXPORTED:
            if name != "sarbp_status_string":
                getattr(L, name).restype = i
        L.sarbp_image_entropy_work_bytes.restype = ctypes.c_size_t
        _LIB = L
    return _LIB


class SarbpError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        msg = lib().sarbp_status_string(status).decode()
        super().__init__(f"{what}: {msg} (status {status})")


def check(status: int, what: str) -> None:
    if status != SARBP_OK:
        raise SarbpError(status, what)
