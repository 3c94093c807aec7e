"""Hypothesis batches and the gradient autofocus pipeline on the GPU."""
import copy

import numpy as np
import pytest

from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_hypothesis_batch_equals_single_images(torch_cuda):
    torch = torch_cuda
    from uncc_sar_focusing_b200 import focusing

    sc = S.point_target_scene(K=64, Np=48, n=40, spacing=0.2, nfft=512, snr_db=20.0, seed=3, n_targets=4)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    H = 5
    rng = np.random.default_rng(0)
    tracks = [np.stack([sc.ant_x, sc.ant_y, sc.ant_z]) + rng.normal(0, 0.01, (3, sc.num_pulses)) for _ in range(H)]
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        r0 = dev(np.tile(sc.slant_range, (H, 1)))
        f0 = dev(np.tile(sc.start_freq, (H, 1)))
        ax, ay, az = (dev(np.stack([t[i] for t in tracks])) for i in range(3))
        batch = plan.backproject_hypotheses(ax, ay, az, r0, f0)
        host = plan.backproject_hypotheses(ax.cpu().numpy(), ay.cpu().numpy(), az.cpu().numpy(), r0.cpu().numpy(),
                                           f0.cpu().numpy())
        for h in range(H):
            one = plan.backproject(ax[h].contiguous(), ay[h].contiguous(), az[h].contiguous(), r0[h].contiguous(),
                                   f0[h].contiguous())
            torch.cuda.synchronize()
            assert torch.equal(batch[h], one)
            assert np.array_equal(host[h], one.cpu().numpy())


def test_hypothesis_batch_full_size_against_oracle(torch_cuda):
    """The autofocus configuration at full size (1024 pulses x 512 samples,
    512^2 image): 8 track hypotheses in one launch, the first and the last
    against the FP64 CPU oracle on every pixel, all 8 against single calls.
    At this size a single image's tiles are split over the resident CTAs and
    their pulse stages summed in a rotated order, so the two agree to
    rounding, not bit for bit (the small-scene test above has one CTA per
    tile in both and is bit-exact)."""
    torch = torch_cuda
    from oracle import oracle as O
    from uncc_sar_focusing_b200 import focusing

    sc = S.motion_error_scene(device="cuda")
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    H = 8
    rng = np.random.default_rng(1)
    ramp = np.linspace(-1.0, 1.0, sc.num_pulses)
    tracks = [np.stack([sc.ant_x, sc.ant_y, sc.ant_z]) + rng.normal(0, 0.02, (3, 1)) * ramp for _ in range(H)]
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        r0 = dev(np.tile(sc.slant_range, (H, 1)))
        f0 = dev(np.tile(sc.start_freq, (H, 1)))
        ax, ay, az = (dev(np.stack([t[i] for t in tracks])) for i in range(3))
        batch = plan.backproject_hypotheses(ax, ay, az, r0, f0)
        for h in range(H):
            one = plan.backproject(ax[h].contiguous(), ay[h].contiguous(), az[h].contiguous(), r0[h].contiguous(),
                                   f0[h].contiguous())
            torch.cuda.synchronize()
            d = float((batch[h] - one).abs().pow(2).sum().sqrt() / one.abs().pow(2).sum().sqrt())
            assert d < 1e-6, (h, d)
        plan.check()
        got = batch.cpu().numpy()
    errs = []
    for h in (0, H - 1):
        sh = copy.copy(sc)
        sh.ant_x, sh.ant_y, sh.ant_z = (np.ascontiguousarray(v) for v in tracks[h])
        errs.append(O.rel_l2(got[h].reshape(-1), O.focus_fp64(sh).reshape(-1)))
    print("hypotheses 0 and 7 vs FP64 oracle:", ["%.2e" % e for e in errs])
    assert max(errs) < 1e-4, errs
    torch.cuda.empty_cache()


def test_gradient_autofocus_pipeline_recovers_focus(torch_cuda):
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autofocus as AF
    from uncc_sar_focusing_b200 import autograd as A
    from uncc_sar_focusing_b200 import focusing

    sc = S.motion_error_scene(K=128, Np=256, n=128, spacing=0.16, peak=0.3, walk_sigma=5e-4, seed=9,
                              device="cuda")
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ax, ay, az, r0, f0 = (dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        ent = lambda x, y, z, r=r0: float(A.image_entropy(plan.backproject(x, y, z, r, f0)))  # noqa: E731
        e_measured = ent(ax, ay, az)
        e_true = ent(*(dev(getattr(sc, a) + sc.true_error[i]) for i, a in enumerate(("ant_x", "ant_y", "ant_z"))))
        out = AF.focus_motion_error(plan, ax, ay, az, r0, f0, cubic_iters=200, los_iters=150)
        e_final = min(out["entropy_cubic"], out["entropy_los"], out["entropy_pga"])
    assert e_measured > e_true + 0.5
    # the pipeline closes at least 90% of the entropy gap between the measured and the true track
    assert e_final < e_true + 0.1 * (e_measured - e_true), (e_measured, e_true, out["entropy_cubic"],
                                                             out["entropy_los"], out["entropy_pga"])
    times = [t for t, _, _ in out["timeline"]]
    assert times == sorted(times)


def test_captured_descent_matches_eager(torch_cuda):
    """Descent steps replayed from a captured CUDA graph take the same steps
    as the eager loop (same kernels, same capturable Adam): entropy histories
    and the chosen parameters agree."""
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autofocus as AF
    from uncc_sar_focusing_b200 import focusing

    sc = S.motion_error_scene(K=128, Np=256, n=128, spacing=0.16, peak=0.3, walk_sigma=5e-4, seed=10,
                              device="cuda")
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ax, ay, az, r0, f0 = (dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        motion = AF.CubicMotion(ax, ay, az)
        g = AF.gradient_autofocus(plan, motion, r0, f0, iters=25, graph=True)
        e = AF.gradient_autofocus(plan, motion, r0, f0, iters=25, graph=False)
        eg = np.array([h["entropy"] for h in g.history])
        ee = np.array([h["entropy"] for h in e.history])
        assert np.allclose(eg, ee, rtol=1e-6, atol=0)
        assert torch.allclose(g.theta, e.theta, rtol=1e-6, atol=1e-9)
        rg, hg, _ = AF.line_of_sight_autofocus(plan, ax, ay, az, r0, f0, iters=15, graph=True)
        re_, he, _ = AF.line_of_sight_autofocus(plan, ax, ay, az, r0, f0, iters=15, graph=False)
        assert np.allclose([h["entropy"] for h in hg], [h["entropy"] for h in he], rtol=1e-6, atol=0)
        assert torch.allclose(rg, re_, rtol=0, atol=1e-9)


def test_gradient_autofocus_resumes_from_a_saved_state(torch_cuda, tmp_path):
    """A descent split in two, the first part's state written to .npz and
    read back for the second, reaches the coefficients and Adam moments of
    the whole run (same schedule positions, same optimiser state)."""
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autofocus as AF
    from uncc_sar_focusing_b200 import focusing

    sc = S.motion_error_scene(K=128, Np=256, n=128, spacing=0.16, peak=0.3, walk_sigma=5e-4, seed=11,
                              device="cuda")
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ax, ay, az, r0, f0 = (dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        motion = AF.CubicMotion(ax, ay, az)
        whole = AF.gradient_autofocus(plan, motion, r0, f0, iters=30, graph=False)
        first = AF.gradient_autofocus(plan, motion, r0, f0, iters=12, total_iters=30, graph=False)
        first.state.save(str(tmp_path / "autofocus.npz"))
        state = AF.AutofocusState.load(str(tmp_path / "autofocus.npz"))
        assert state.iters_done == 12 and state.total_iters == 30
        second = AF.gradient_autofocus(plan, motion, r0, f0, iters=18, resume=state, graph=False)
    assert second.history[0]["iter"] == 12 and second.state.iters_done == 30
    assert second.state.step == whole.state.step == 30
    for name in ("theta", "exp_avg", "exp_avg_sq"):
        a, b = getattr(second.state, name), getattr(whole.state, name)
        assert np.allclose(a, b, rtol=1e-12, atol=0), (name, np.abs(a - b).max())
    # the entropies of the second part are the whole run's last 18
    assert np.allclose([h["entropy"] for h in second.history], [h["entropy"] for h in whole.history[12:]],
                       rtol=1e-12, atol=0)


def test_gradient_autofocus_stops_on_a_plateau(torch_cuda):
    """With a plateau tolerance the descent ends at a check once the best
    entropy gained less than the tolerance over the last check_every steps;
    the steps it ran are the whole run's first steps."""
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autofocus as AF
    from uncc_sar_focusing_b200 import focusing

    sc = S.motion_error_scene(K=128, Np=256, n=128, spacing=0.16, peak=0.3, walk_sigma=5e-4, seed=12,
                              device="cuda")
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ax, ay, az, r0, f0 = (dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        motion = AF.CubicMotion(ax, ay, az)
        full = AF.gradient_autofocus(plan, motion, r0, f0, iters=200, graph=False)
        early = AF.gradient_autofocus(plan, motion, r0, f0, iters=200, graph=False, plateau=1e-2, check_every=20)
    n = early.images_formed
    assert n % 20 == 0 and 40 <= n < 200  # the first check that can stop is after 40 steps
    e_full = np.array([h["entropy"] for h in full.history])
    e_early = np.array([h["entropy"] for h in early.history])
    assert len(e_early) == n
    assert np.allclose(e_early, e_full[:n], rtol=1e-12, atol=0)
    best = np.minimum.accumulate(e_full)
    assert best[n - 21] - best[n - 1] < 1e-2  # the check that stopped it
    assert all(best[k - 21] - best[k - 1] >= 1e-2 for k in range(40, n, 20))  # the earlier checks did not


def test_reference_costs_on_the_gpu_match_the_transcriptions(torch_cuda):
    """The reference's two grid-search costs, batched on the device, against
    direct transcriptions of the reference's loops (dft2DCalculation,
    gridSearchErrorFunctions_dft.cuh:112-203,320-335; cuCalculateColumnEntropy,
    gridSearchErrorFunctions.cuh:341-447) run on the CPU."""
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autofocus as AF

    import test_autofocus as T

    rng = np.random.default_rng(8)
    imgs = (rng.standard_normal((3, 12, 10)) + 1j * rng.standard_normal((3, 12, 10))).astype(np.complex64)
    imgs[2, 5, :] = 0.0
    dft = AF.reference_dft_costs(torch.as_tensor(imgs).cuda()).cpu().numpy()
    col = AF.reference_column_entropies(torch.as_tensor(imgs).cuda()).cpu().numpy()
    for i in range(3):
        u8 = AF.reference_u8_image(torch.as_tensor(imgs[i])).numpy().astype(np.float64)
        nx, ny = u8.shape
        hh, hw = ny // 2, nx // 2
        threshold = int((hh * hh + hw * hw) * (0.35 * 0.35))
        out = 0.0
        for dft_x in range(nx):
            d1 = [sum(u8[x, yy] * np.exp(-2j * np.pi * dft_x * x / nx) for x in range(nx)) for yy in range(ny)]
            d2 = [sum(np.exp(-2j * np.pi * dy * yy / ny) * d1[yy] for yy in range(ny)) for dy in range(ny)]
            for y in range(hh):
                if dft_x * dft_x + y * y < threshold or (nx - dft_x - 1) ** 2 + y * y < threshold:
                    out += abs(d2[y]) + abs(d2[ny - y - 1])
        assert abs(dft[i] + out) < 1e-6 * out
        assert abs(col[i] - T.column_entropy_transcription(imgs[i])) < 1e-9


def test_grid_search_with_the_reference_cost_improves_focus(torch_cuda):
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autofocus as AF
    from uncc_sar_focusing_b200 import focusing

    sc = S.motion_error_scene(K=128, Np=256, n=96, spacing=0.16, peak=0.3, walk_sigma=0.0, seed=11,
                              device="cuda")
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ax, ay, az, r0, f0 = (dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        motion = AF.CubicMotion(ax, ay, az)
        before = AF.focus_metrics(plan.backproject(ax, ay, az, r0, f0))
        res = AF.grid_search_autofocus(plan, motion, r0, f0, span=0.3, points=3, levels=3, batch=243)
        a = motion.track(res.theta)
        after = AF.focus_metrics(plan.backproject(a[0].contiguous(), a[1].contiguous(), a[2].contiguous(), r0, f0))
    assert res.images_formed == 3 * 3 ** 6
    assert [h["cost"] for h in res.history] == ["reference_dft"] * 3
    assert after["reference_dft_cost"] < before["reference_dft_cost"]
    assert abs(after["reference_dft_cost"] - res.history[-1]["score"]) < 1e-6 * abs(after["reference_dft_cost"])
