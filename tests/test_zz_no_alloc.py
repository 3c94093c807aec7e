"""sarbp_backproject_noalloc through the C ABI, against sarbp_backproject.

The entry point exists for callers that must not allocate device memory when
they form an image (a pulse-callback loop that cannot stall on cudaMalloc's
device-wide synchronisation, or an application that owns all GPU memory
through its own pool).  It reuses one fixed device array for its scratch, so
the test makes two calls in a row with different sizes -- the second must not
see anything the first left behind -- and compares each with the plan-based
entry point on the same range profiles and geometry, within the mixed
precision tolerance of the other parity tests.  Kept in its own file, named
to be collected last.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import _native as N
from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu
MIXED_TOL = 1e-4


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def reference_and_inputs(torch, sc):
    """Range profiles and image from the plan-based entry points, plus the
    device inputs for the allocation-free call."""
    from uncc_sar_focusing_b200 import focusing

    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    geo = [dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)]
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        rc = torch.empty((sc.num_pulses, sc.nfft), dtype=torch.complex64, device="cuda")
        plan.range_profiles(out=rc)
        want = plan.backproject(*geo, out=plan.new_image("cuda"))
        torch.cuda.synchronize()
        plan.check()
        desc = plan._desc
    return desc, rc, geo, want.cpu().numpy()


def call_noalloc(torch, desc, rc, geo, shape, flags=0, start=None):
    if start is None:
        out = torch.full(shape, complex(7.0, -3.0), dtype=torch.complex64, device="cuda")  # stale contents
    else:
        out = torch.as_tensor(start).cuda()
    g = N.Geometry(*(ctypes.c_void_p(v.data_ptr()) for v in geo), geo[0].numel(), N.MEMORY_DEVICE)
    st = N.lib().sarbp_backproject_noalloc(ctypes.byref(desc), ctypes.c_void_p(rc.data_ptr()), ctypes.byref(g),
                                           ctypes.c_void_p(out.data_ptr()), flags,
                                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, out.cpu().numpy()


def limit_scene(num_pulses):
    """A 64-sample, nfft-256 scene whose staged rows are 744 entries each.

    The call picks 32 x 64-pixel tiles here: with lambda = nfft / max_wr =
    16.26 bins/m and a tile half-diagonal of hypot(3.2, 6.4) m the window is
    2 x (ceil(16.26 x 7.155) + 3) + 2 = 242 entries, the guard bands 244
    entries each side, so a row is 256 + 2 x 244 = 744 entries.  The scratch
    holds 2^21 - 1 entries after the error word: 2818 rows fit (2,096,592
    entries), 2819 do not (2,097,336)."""
    sc = S.point_target_scene(K=64, Np=num_pulses, n=40, spacing=0.2, nfft=256, snr_db=None, seed=33,
                              n_targets=2)
    lam = sc.nfft / sc.max_wr
    w = int(np.ceil(lam * np.hypot(0.5 * 32 * 0.2, 0.5 * 64 * 0.2))) + 3
    assert 2 * w + 2 == 242, "scene no longer gives the 744-entry rows this test is sized for"
    return sc


def test_noalloc_matches_plan_entry_point_on_two_calls_in_a_row(torch_cuda):
    torch = torch_cuda
    big = S.point_target_scene(K=128, Np=96, n=80, spacing=0.1, nfft=1024, snr_db=20.0, seed=31, n_targets=4)
    small = S.point_target_scene(K=64, Np=40, n=40, spacing=0.2, nfft=256, snr_db=None, seed=32, n_targets=3,
                                 extent=5.0)
    small.grid = S.Grid(nx=37, ny=45, x0=0.4, y0=-0.3, wx=36 * 0.2, wy=44 * 0.17)
    for sc in (big, small):
        desc, rc, geo, want = reference_and_inputs(torch, sc)
        st, got = call_noalloc(torch, desc, rc, geo, want.shape)
        assert st == N.SARBP_OK, N.lib().sarbp_status_string(st)
        assert O.rel_l2(got, want) < MIXED_TOL
        assert np.isfinite(got).all()


def test_noalloc_runs_on_the_device_its_descriptor_names(torch_cuda):
    torch = torch_cuda
    sc = S.point_target_scene(K=64, Np=40, n=40, spacing=0.2, nfft=256, snr_db=None, seed=35, n_targets=3)
    desc, rc, geo, want = reference_and_inputs(torch, sc)
    desc.device = torch.cuda.current_device()
    st, got = call_noalloc(torch, desc, rc, geo, want.shape)
    assert st == N.SARBP_OK, N.lib().sarbp_status_string(st)
    assert O.rel_l2(got, want) < MIXED_TOL
    desc.device = torch.cuda.device_count()  # no such device
    st, _ = call_noalloc(torch, desc, rc, geo, want.shape)
    assert st == N.SARBP_ERR_INVALID_ARGUMENT


def test_noalloc_accumulates_into_the_callers_image(torch_cuda):
    torch = torch_cuda
    sc = S.point_target_scene(K=64, Np=40, n=40, spacing=0.2, nfft=256, snr_db=None, seed=34, n_targets=3)
    desc, rc, geo, want = reference_and_inputs(torch, sc)
    rng = np.random.default_rng(5)
    start = (rng.standard_normal(want.shape) + 1j * rng.standard_normal(want.shape)).astype(np.complex64)
    start *= np.float32(np.abs(want).max())
    st, got = call_noalloc(torch, desc, rc, geo, want.shape, flags=N.ACCUMULATE, start=start)
    assert st == N.SARBP_OK, N.lib().sarbp_status_string(st)
    assert O.rel_l2(got - start, want) < MIXED_TOL


def test_noalloc_serves_the_largest_request_its_scratch_holds(torch_cuda):
    torch = torch_cuda
    desc, rc, geo, want = reference_and_inputs(torch, limit_scene(2818))
    st, got = call_noalloc(torch, desc, rc, geo, want.shape)
    assert st == N.SARBP_OK, N.lib().sarbp_status_string(st)
    assert O.rel_l2(got, want) < MIXED_TOL


def test_noalloc_rejects_requests_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    sc = limit_scene(2819)
    desc, rc, geo, want = reference_and_inputs(torch, sc)
    st, _ = call_noalloc(torch, desc, rc, geo, want.shape)
    assert st == N.SARBP_ERR_UNSUPPORTED
