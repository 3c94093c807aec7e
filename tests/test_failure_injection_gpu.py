"""Failure detection on the GPU, without a GPU fault.

* Device allocations: `sarbp_test_fail_device_alloc(n)` makes the n-th
  allocation from now fail as if the device were out of memory.  Failing
  each allocation of a plan's creation in turn must return
  SARBP_ERR_OUT_OF_MEMORY with everything allocated before it released; the
  adjoint's first-use allocation must fail the same way and succeed on the
  next call.
* Bounded device waits: `sarbp_test_drop_window_copy(plan, p)` makes the
  producing warp of pulse p expect its range-bin window's bytes without
  issuing the copy, so that stage's mbarrier phase never completes (a flag
  that nothing sets).  The kernels' waits give up after about two seconds,
  every warp leaves, and the call returns SARBP_ERR_KERNEL_TIMEOUT; the CUDA
  context stays usable and the same plan focuses correctly once the hook is
  off.  No wait in the kernels is unbounded, so the test cannot hang a GPU.
"""
import ctypes
import time

import numpy as np
import pytest

from uncc_sar_focusing_b200 import _native as N
from uncc_sar_focusing_b200 import focusing
from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture
def disarm():
    yield
    N.lib().sarbp_test_fail_device_alloc(-1)


def small_scene():
    return S.point_target_scene(K=64, Np=40, n=40, spacing=0.2, nfft=256, snr_db=None, seed=41, n_targets=3)


def free_bytes(torch):
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_each_allocation_of_plan_creation_fails_cleanly(torch_cuda, disarm):
    torch = torch_cuda
    sc = small_scene()
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        desc = plan._desc
    before = free_bytes(torch)
    failures = 0
    for n in range(64):
        N.lib().sarbp_test_fail_device_alloc(n)
        h = ctypes.c_void_p()
        st = N.lib().sarbp_plan_create(ctypes.byref(desc), ctypes.byref(h))
        if st == N.SARBP_OK:
            # every allocation of the creation got through: the hook is still armed
            N.lib().sarbp_test_fail_device_alloc(-1)
            N.lib().sarbp_plan_destroy(h)
            break
        assert st == N.SARBP_ERR_OUT_OF_MEMORY, N.lib().sarbp_status_string(st)
        assert not h.value
        # nothing the failed creation allocated is left behind
        assert abs(free_bytes(torch) - before) < (4 << 20)
        failures += 1
    assert failures >= 7  # staging, geometry, FFT, pair rows, factors, image, error word at least
    # a plan created afterwards works
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        img = plan.focus(sc.phase_history, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)
    assert np.isfinite(img).all() and np.abs(img).max() > 0


def test_first_use_allocation_of_the_adjoint_fails_then_succeeds(torch_cuda, disarm):
    sc = small_scene()
    geo = (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        img = plan.focus(sc.phase_history, *geo)
        N.lib().sarbp_test_fail_device_alloc(0)
        with pytest.raises(N.SarbpError) as e:
            plan.backproject_adjoint(*geo, img)
        assert e.value.status == N.SARBP_ERR_OUT_OF_MEMORY
        N.lib().sarbp_test_fail_device_alloc(-1)
        gant, gr0 = plan.backproject_adjoint(*geo, img)
    assert np.isfinite(gant).all() and np.abs(gr0).max() > 0


def test_a_window_copy_that_never_lands_times_out_and_the_plan_recovers(torch_cuda):
    torch = torch_cuda
    sc = small_scene()
    geo = (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        want = plan.focus(sc.phase_history, *geo)
        grad_want = [np.asarray(v) for v in plan.backproject_adjoint(*geo, want)]
        assert N.lib().sarbp_test_drop_window_copy(plan._h, 3) == N.SARBP_OK
        t0 = time.perf_counter()
        with pytest.raises(N.SarbpError) as e:
            plan.focus(sc.phase_history, *geo)
        assert e.value.status == N.SARBP_ERR_KERNEL_TIMEOUT
        with pytest.raises(N.SarbpError) as e:
            plan.backproject_adjoint(*geo, want)
        assert e.value.status == N.SARBP_ERR_KERNEL_TIMEOUT
        assert time.perf_counter() - t0 < 60.0
        # the context is usable and the plan works again without the hook
        assert float(torch.ones(4, device="cuda").sum().item()) == 4.0
        assert N.lib().sarbp_test_drop_window_copy(plan._h, -1) == N.SARBP_OK
        got = plan.focus(sc.phase_history, *geo)
        grad_got = [np.asarray(v) for v in plan.backproject_adjoint(*geo, want)]
    assert np.array_equal(got, want)
    for a, b in zip(grad_got, grad_want):
        assert np.array_equal(a, b)


def test_drop_hook_is_refused_on_fp64_plans(torch_cuda):
    sc = small_scene()
    with focusing.Plan.for_scene(sc, "fp64") as plan:
        assert N.lib().sarbp_test_drop_window_copy(plan._h, 0) == N.SARBP_ERR_UNSUPPORTED
