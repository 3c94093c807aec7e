"""The C ABI without a GPU: the library loads, exports every entry point
include/sarbp.h declares, and rejects bad arguments with status codes before
touching a device (no compute calls here)."""
import ctypes
import os
import re

import pytest

from uncc_sar_focusing_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"SARBP_API\s+[\w\s\*]*?\b(sarbp_\w+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    names = declared("sarbp.h")
    assert len(names) >= 10
    lib = N.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(N.EXPORTED)


def test_bindings_mirror_the_header_abi_version():
    import re

    from uncc_sar_focusing_b200 import _native as N

    hdr = open(os.path.join(ROOT, "include", "sarbp.h")).read()
    assert int(re.search(r"#define SARBP_ABI_VERSION (\d+)", hdr).group(1)) == N.ABI_VERSION


def test_abi_version_and_status_strings():
    lib = N.lib()
    assert lib.sarbp_abi_version() == 1
    for code in range(0, 11):
        assert lib.sarbp_status_string(code).decode() not in ("", "unknown status")
    assert lib.sarbp_status_string(999).decode() == "unknown status"


def desc(**kw):
    d = N.PlanDesc()
    d.num_range_samples, d.num_pulses, d.nfft, d.max_wr = 64, 32, 256, 15.0
    d.grid = N.Grid(32, 32, 1, 0.0, 0.0, 0.0, 5.0, 5.0, 0.0)
    d.precision, d.window, d.device = N.PRECISION_MIXED, N.WINDOW_HAMMING, -1
    for k, v in kw.items():
        if k.startswith("g_"):
            setattr(d.grid, k[2:], v)
        else:
            setattr(d, k, v)
    return d


@pytest.mark.parametrize("kw", [dict(nfft=32), dict(num_range_samples=0), dict(num_pulses=0), dict(max_wr=0.0),
                                dict(max_wr=float("nan")), dict(g_nx=0), dict(g_wx=-1.0),
                                dict(g_x0=float("inf")), dict(precision=7), dict(window=9)])
def test_plan_create_rejects_invalid_descriptions(kw):
    h = ctypes.c_void_p()
    assert N.lib().sarbp_plan_create(ctypes.byref(desc(**kw)), ctypes.byref(h)) == N.SARBP_ERR_INVALID_ARGUMENT
    assert not h.value


def test_null_pointers_are_reported():
    lib = N.lib()
    h = ctypes.c_void_p()
    assert lib.sarbp_plan_create(None, ctypes.byref(h)) == N.SARBP_ERR_NULL_POINTER
    assert lib.sarbp_plan_create(ctypes.byref(desc()), None) == N.SARBP_ERR_NULL_POINTER
    assert lib.sarbp_plan_destroy(None) == N.SARBP_ERR_NULL_POINTER
    assert lib.sarbp_focus(None, None, None, 0, None) == N.SARBP_ERR_NULL_POINTER
    assert lib.sarbp_backproject(None, None, None, 0, 0, None) == N.SARBP_ERR_NULL_POINTER
    assert lib.sarbp_range_compress(None, None, 0, 0, None) == N.SARBP_ERR_NULL_POINTER
    assert lib.sarbp_focus_submit(None, None, None, None) == N.SARBP_ERR_NULL_POINTER
    assert lib.sarbp_focus_wait(None, 0) == N.SARBP_ERR_NULL_POINTER


def test_no_device_is_a_status_not_a_crash():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert N.lib().sarbp_plan_create(ctypes.byref(desc()), ctypes.byref(h)) == N.SARBP_ERR_NO_DEVICE


def test_compat_library_exports_the_reference_symbols():
    if not os.path.exists(N.COMPAT_PATH):
        pytest.skip("shim not built (needs the reference headers)")
    syms = os.popen(f"nm -D {N.COMPAT_PATH}").read()
    # cuda_focus_SAR_image<float,float> and <double,double>, as libcuda_sar_focusing.cu:26-32 exports them
    assert "_Z20cuda_focus_SAR_imageIffEvRK12SAR_ApertureIT_ERK28SAR_ImageFormationParametersIT0_ERSt8valarrayI11unccComplexIS1_EE" in syms
    assert "_Z20cuda_focus_SAR_imageIddEvRK12SAR_ApertureIT_ERK28SAR_ImageFormationParametersIT0_ERSt8valarrayI11unccComplexIS1_EE" in syms
