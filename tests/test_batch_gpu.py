"""Batches of uneven scenes (sarbp_batch_*): one backprojection launch over the
tiles of all scenes, replayed as a captured CUDA graph.

Every image of a batch is held to the FP64 oracle's 1e-4 relative L2 (the
accuracy target) and to the single-scene plan within 1e-5 (same kernel
arithmetic: the plan is given the batch's tile shape, and the batch splits the
pulse sums at other places, so the sums differ in rounding only).
"""
import os

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


# (K, Np, n, spacing, nfft, window, seed): sizes that are not tile multiples,
# different range sample counts, FFT lengths, pulse counts and tapers
SHAPES = [
    (64, 48, 40, 0.2, 512, "hamming", 1),
    (53, 96, 70, 0.15, 424, "hamming", 2),
    (40, 32, 33, 0.25, 256, None, 3),
    (80, 64, 128, 0.12, 640, "hamming", 4),
    (64, 20, 17, 0.3, 512, None, 5),
]


def make(shape):
    K, Np, n, sp, nfft, win, seed = shape
    sc = S.point_target_scene(K=K, Np=Np, n=n, spacing=sp, nfft=nfft, snr_db=20.0, seed=seed, n_targets=4,
                              extent=0.5 * sp * n)
    sc.window = win
    return sc


def dev_args(sc, n=None):
    import torch

    n = sc.num_pulses if n is None else n
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a[:n])).cuda()  # noqa: E731
    return (d(sc.phase_history), d(sc.ant_x), d(sc.ant_y), d(sc.ant_z), d(sc.slant_range), d(sc.start_freq))


def single(F, sc, n=None, tile=None):
    """The same scene through its own plan.  With tile = the batch's (rows / 8,
    stage pulses), the plan uses the batch's tile shape (SARBP_TILE override),
    so the two FP32 paths share their tile-centre bases and agree to ~1e-6;
    plans with another tile height differ at the 1e-5 level (both stay within
    1e-4 of FP64)."""
    n = sc.num_pulses if n is None else n
    old = os.environ.get("SARBP_TILE")
    if tile is not None:
        os.environ["SARBP_TILE"] = f"{tile[0]},{tile[1]}"
    try:
        with F.Plan.for_scene(sc, "mixed") as plan:
            return plan.focus(sc.phase_history[:n], sc.ant_x[:n], sc.ant_y[:n], sc.ant_z[:n], sc.slant_range[:n],
                              sc.start_freq[:n])
    finally:
        if old is None:
            os.environ.pop("SARBP_TILE", None)
        else:
            os.environ["SARBP_TILE"] = old


def batch_tile(batch):
    info = batch.info
    return info["tile_mx"], info["stage_pulses"]


def test_uneven_batch_matches_oracle_and_single_plans(F):
    import torch

    scenes = [make(s) for s in SHAPES]
    with F.Batch(scenes) as batch:
        imgs = batch.new_images()
        batch.focus([dev_args(sc) for sc in scenes], imgs)
        ms = batch.wait()
        info = batch.info
        tile = batch_tile(batch)
    assert info["num_scenes"] == len(scenes) and info["resident_ctas"] > 0
    assert np.isfinite(ms).all() and (ms > 0).all()
    for sc, img in zip(scenes, imgs):
        got = img.cpu().numpy()
        assert O.rel_l2(got, O.focus_fp64(sc)) < 1e-4
        assert O.rel_l2(got, single(F, sc, tile=tile)) < 1e-5
    torch.cuda.synchronize()


@pytest.mark.parametrize("per_tile", [False, True])
def test_both_schedules(F, per_tile):
    scenes = [make(s) for s in SHAPES]
    with F.Batch(scenes) as batch:
        batch.set_schedule(per_tile)
        imgs = batch.new_images()
        batch.focus([dev_args(sc) for sc in scenes], imgs)
        ms = batch.wait()
        assert batch.info["per_tile"] == int(per_tile)
        tile = batch_tile(batch)
    assert np.isfinite(ms).all() and (ms > 0).all()
    for sc, img in zip(scenes, imgs):
        assert O.rel_l2(img.cpu().numpy(), single(F, sc, tile=tile)) < 1e-5


def test_graph_replay_with_new_buffers_and_pulse_counts(F):
    scenes = [make(s) for s in SHAPES[:3]]
    others = [make(s[:-1] + (s[-1] + 10,)) for s in SHAPES[:3]]
    with F.Batch(scenes) as batch:
        imgs = batch.new_images()
        batch.focus([dev_args(sc) for sc in scenes], imgs)
        batch.wait()
        assert batch.info["graph"] == 1
        tile = batch_tile(batch)
        # same shapes, new tensors: the replayed graph reads the new table
        imgs2 = batch.new_images()
        batch.focus([dev_args(sc) for sc in others], imgs2)
        batch.wait()
        for sc, img in zip(others, imgs2):
            assert O.rel_l2(img.cpu().numpy(), single(F, sc, tile=tile)) < 1e-5
        # fewer pulses in one scene: new unit count, re-captured
        cut = [None, scenes[1].num_pulses // 2, None]
        imgs3 = batch.new_images()
        batch.focus([dev_args(sc, c) for sc, c in zip(scenes, cut)], imgs3)
        batch.wait()
        for sc, c, img in zip(scenes, cut, imgs3):
            assert O.rel_l2(img.cpu().numpy(), single(F, sc, c, tile=tile)) < 1e-5


def test_autotune_keeps_results(F):
    scenes = [make(s) for s in SHAPES]
    args = [dev_args(sc) for sc in scenes]
    with F.Batch(scenes) as batch:
        imgs = batch.new_images()
        best = batch.autotune(args, imgs)
        assert best > 0.0
        info = batch.info
        assert (info["tile_mx"], info["stage_pulses"]) in [(8, 8), (8, 4), (4, 8), (4, 4), (2, 8), (2, 4), (1, 8),
                                                           (1, 4)]
        imgs = batch.new_images()
        batch.focus(args, imgs)
        batch.wait()
    for sc, img in zip(scenes, imgs):
        assert O.rel_l2(img.cpu().numpy(), O.focus_fp64(sc)) < 1e-4


def test_batch_argument_errors(F):
    import torch

    scenes = [make(s) for s in SHAPES[:2]]
    with F.Batch(scenes) as batch:
        imgs = batch.new_images()
        host = [(sc.phase_history, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq) for sc in scenes]
        with pytest.raises(ValueError):
            batch.focus(host, imgs)  # host memory
        too_many = [dev_args(sc) for sc in scenes]
        big = make(SHAPES[0][:1] + (SHAPES[0][1] * 2,) + SHAPES[0][2:])
        too_many[0] = dev_args(big)  # more pulses than the scene was created for
        with pytest.raises(F.N.SarbpError):
            batch.focus(too_many, imgs)
        batch.focus([dev_args(sc) for sc in scenes], imgs)
        batch.wait()
    torch.cuda.synchronize()


def test_fused_range_compression_scenes_in_a_batch(F):
    """Scenes whose nfft = R K has a fused range-compression kernel (K = 256,
    512) take it inside the batch's graph, next to a scene on the cuFFT path."""
    shapes = [(256, 24, 40, 0.2, 2048, "hamming", 21), (512, 16, 33, 0.25, 4096, None, 22),
              (64, 20, 17, 0.3, 512, None, 23)]
    scenes = [make(s) for s in shapes]
    with F.Batch(scenes) as batch:
        for _ in range(2):  # capture, then replay
            imgs = batch.new_images()
            batch.focus([dev_args(sc) for sc in scenes], imgs)
            batch.wait()
        assert batch.info["graph"] == 1
        tile = batch_tile(batch)
    for sc, img in zip(scenes, imgs):
        got = img.cpu().numpy()
        assert O.rel_l2(got, O.focus_fp64(sc)) < 1e-4
        assert O.rel_l2(got, single(F, sc, tile=tile)) < 1e-5


def test_batch_at_the_batched_configurations_sizes(F):
    """Scenes of the batched configuration's size range (512 samples, Nfft
    4096, 0.1 m pixels; 128^2 x 256 pulses up to 1024^2 x 2048 pulses) in
    one batch: every image against the FP64 CPU oracle (3.1e9 pixel-pulses
    on the host's cores)."""
    import torch

    shapes = [(128, 256, 5), (384, 1024, 60), (700, 777, 200), (1024, 2048, 500), (200, 1500, 30)]
    scenes = [S.point_target_scene(K=512, Np=npulse, n=n, spacing=0.1, n_targets=nt, nfft=4096, seed=200 + i,
                                   extent=0.08 * n, device="cuda") for i, (n, npulse, nt) in enumerate(shapes)]
    with F.Batch(scenes) as batch:
        imgs = batch.new_images()
        batch.focus([dev_args(sc) for sc in scenes], imgs)
        batch.wait()
    errs = [O.rel_l2(img.cpu().numpy(), O.focus_fp64(sc)) for sc, img in zip(scenes, imgs)]
    print("batched-configuration sizes vs FP64 oracle:", ["%.2e" % e for e in errs])
    assert max(errs) < 1e-4, errs
    torch.cuda.empty_cache()
