"""Pipelined host-buffer focusing (sarbp_focus_submit / sarbp_focus_wait).

Each submission runs the same kernels on the same inputs as the synchronous
sarbp_focus, so its image must equal that call's bit for bit; the mixed path
is also held to the FP64 oracle's 1e-4 relative L2 on every aperture of the
stream.
"""
import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from uncc_sar_focusing_b200 import focusing

    return focusing


def scene(seed, Np=48):
    return S.point_target_scene(K=64, Np=Np, n=40, spacing=0.2, nfft=512, snr_db=20.0, seed=seed, n_targets=4,
                                extent=6.0)


def args(sc):
    return (sc.phase_history, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)


def pinned_like(a):
    import torch

    t = torch.empty(a.shape, dtype={np.complex64: torch.complex64, np.float64: torch.float64,
                                    np.complex128: torch.complex128}[a.dtype.type], pin_memory=True)
    v = t.numpy()
    v[...] = a
    return v, t


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_stream_of_apertures_matches_synchronous_focus(F, precision):
    scenes = [scene(seed) for seed in range(5)]
    with F.Plan.for_scene(scenes[0], precision) as plan:
        want = [plan.focus(*args(sc)) for sc in scenes]
        keep, outs, tickets = [], [], []
        for sc in scenes:
            pinned = [pinned_like(np.ascontiguousarray(a)) for a in args(sc)]
            keep.append(pinned)
            out, t = pinned_like(plan.new_image())
            keep.append(t)
            outs.append(out)
            tickets.append(plan.focus_submit(*[v for v, _ in pinned], out=out))
        assert tickets == list(range(1, 6))
        plan.focus_wait()
    for sc, got, ref in zip(scenes, outs, want):
        np.testing.assert_array_equal(got, ref)
        if precision == "mixed":
            assert O.rel_l2(got, O.focus_fp64(sc)) < 1e-4


def test_pageable_buffers_and_fewer_pulses(F):
    """Pageable host memory (no overlap, same result) and apertures shorter
    than the plan's pulse capacity."""
    big, short = scene(7, Np=48), scene(8, Np=48)
    for name in ("phase_history", "ant_x", "ant_y", "ant_z", "slant_range", "start_freq"):
        setattr(short, name, np.ascontiguousarray(getattr(short, name)[:30]))
    with F.Plan.for_scene(big, "mixed") as plan:
        want_big = plan.focus(*args(big))
        want_short = plan.focus(*args(short))
        out_big, out_short = plan.new_image(), plan.new_image()
        t1 = plan.focus_submit(*args(big), out=out_big)
        t2 = plan.focus_submit(*args(short), out=out_short)
        plan.focus_wait(t1)
        np.testing.assert_array_equal(out_big, want_big)
        plan.focus_wait(t2)
        np.testing.assert_array_equal(out_short, want_short)


def test_other_calls_wait_for_outstanding_submissions(F):
    a, b = scene(11), scene(12)
    with F.Plan.for_scene(a, "mixed") as plan:
        want_a = plan.focus(*args(a))
        want_b = plan.focus(*args(b))
        out = plan.new_image()
        plan.focus_submit(*args(a), out=out)
        # a synchronous call on the same plan drains the pipeline first
        got_b = plan.focus(*args(b))
        np.testing.assert_array_equal(out, want_a)
        np.testing.assert_array_equal(got_b, want_b)
        plan.focus_wait()


def test_submit_errors(F):
    a = scene(13)
    with F.Plan.for_scene(a, "mixed") as plan:
        plan.focus_wait()  # nothing submitted: fine
        with pytest.raises(F.N.SarbpError):
            plan.focus_wait(5)  # beyond the last ticket
        bad = a.ant_x.copy()
        bad[3] = np.nan
        with pytest.raises(F.N.SarbpError):
            plan.focus_submit(a.phase_history, bad, a.ant_y, a.ant_z, a.slant_range, a.start_freq,
                              out=plan.new_image())
        with pytest.raises(ValueError):
            plan.focus_submit(*args(a), out=np.zeros((1, 2, 3), np.complex64))
        out = plan.new_image()
        plan.focus_wait(plan.focus_submit(*args(a), out=out))
        np.testing.assert_array_equal(out, plan.focus(*args(a)))


def test_plan_info_reports_the_split(F):
    import torch  # noqa: F401

    sc = scene(21)
    with F.Plan.for_scene(sc, "mixed") as plan:
        info = plan.info
        assert info["tile_mx"] in (1, 2, 4, 8) and info["stage_pulses"] >= 1
        assert info["resident_ctas"] > 0 and info["window_bins"] >= 4
        split = info["tiles"] % info["resident_ctas"] != 0
        assert info["kernels_per_backproject"] == (2 if split else 1)


@pytest.mark.parametrize("nx,mx_mixed", [(96, 4), (256, 8), (200, 8), (40, 8)])
def test_tile_height_follows_row_padding(F, nx, mx_mixed):
    """Mixed plans take 64-row tiles unless padding the rows to a multiple of
    64 adds more than 15% over padding to 32 (96 rows: 128 vs 96); FP64
    plans keep at most 32-row tiles.  Either way the image matches FP64."""
    sc = S.point_target_scene(K=64, Np=24, n=40, spacing=0.2, nfft=512, snr_db=None, seed=31, n_targets=3,
                              extent=6.0)
    sc.grid = S.Grid(nx=nx, ny=48, wx=(nx - 1) * 0.1, wy=47 * 0.1)
    with F.Plan.for_scene(sc, "mixed") as plan:
        assert plan.info["tile_mx"] == mx_mixed
        img = plan.focus(*args(sc))
    with F.Plan.for_scene(sc, "fp64") as p64:
        assert p64.info["tile_mx"] <= 4
        ref = p64.focus(*args(sc))
    assert O.rel_l2(img, ref) < 1e-4
