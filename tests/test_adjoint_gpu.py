"""The adjoint backprojection kernel (sarbp_backproject_adjoint) and its torch
autograd wrapper against the FP64 gradient oracle and finite differences."""
import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S

pytestmark = pytest.mark.gpu
GRAD_TOL = 1e-3  # relative to the largest gradient component


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def grads_vs_oracle(torch, sc, seed=0):
    from uncc_sar_focusing_b200 import focusing

    g = sc.grid
    rng = np.random.default_rng(seed)
    G = (rng.standard_normal((g.nz, g.nx, g.ny)) + 1j * rng.standard_normal((g.nz, g.nx, g.ny))).astype(np.complex64)
    w = O.window_for(sc.window, sc.num_range_samples)
    rc = O.range_compress_fp64(sc.phase_history, sc.nfft, w)
    want_a, want_r = O.bp_grad_fp64(rc, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq, sc.max_wr, g,
                                    G.astype(np.complex128))
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(sc.phase_history)
        got_a, got_r = plan.backproject_adjoint(sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq, G)
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
        da, dr = plan.backproject_adjoint(*(dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range,
                                                              sc.start_freq)), dev(G))
        torch.cuda.synchronize()
        # device and host buffers give the same result
        assert np.allclose(da.cpu().numpy(), got_a, rtol=1e-12, atol=1e-9)
    scale = max(np.abs(want_a).max(), np.abs(want_r).max())
    return np.abs(got_a - want_a).max() / scale, np.abs(got_r - want_r).max() / scale


def test_adjoint_matches_fp64_gradient_oracle(torch_cuda):
    sc = S.point_target_scene(K=96, Np=64, n=48, spacing=0.15, nfft=768, snr_db=20.0, seed=5, n_targets=4,
                              extent=5.0)
    ea, er = grads_vs_oracle(torch_cuda, sc)
    assert ea < GRAD_TOL and er < GRAD_TOL, (ea, er)


def test_adjoint_odd_grid_and_swath_edges(torch_cuda):
    sc = S.point_target_scene(K=32, Np=40, n=8, spacing=1.0, nfft=64, snr_db=None, seed=6, n_targets=2)
    sc.grid = S.Grid(nx=45, ny=37, wx=44 * 0.9, wy=36 * 1.3, x0=3.0, y0=-2.0)
    ea, er = grads_vs_oracle(torch_cuda, sc, seed=1)
    assert ea < GRAD_TOL and er < GRAD_TOL, (ea, er)


def test_adjoint_partial_last_stage(torch_cuda):
    # 37 pulses: the last pulse stage of every tile is partly empty
    sc = S.point_target_scene(K=64, Np=37, n=40, spacing=0.2, nfft=256, snr_db=None, seed=9, n_targets=3,
                              extent=5.0)
    ea, er = grads_vs_oracle(torch_cuda, sc, seed=3)
    assert ea < GRAD_TOL and er < GRAD_TOL, (ea, er)


def test_adjoint_large_config(torch_cuda):
    """The large configuration at full size (1024 x 2048 pulses, 1024^2
    image, Nfft 8192) with a random upstream gradient: every pulse's dL/d
    antenna xyz and dL/dR0 against the FP64 gradient oracle."""
    sc = S.large_scene(device="cuda")
    ea, er = grads_vs_oracle(torch_cuda, sc, seed=4)
    print(f"large configuration adjoint vs FP64 gradient oracle: antenna {ea:.2e}, R0 {er:.2e} of max")
    assert ea < GRAD_TOL and er < GRAD_TOL, (ea, er)
    torch_cuda.cuda.empty_cache()


def test_adjoint_near_field(torch_cuda):
    sc = S.point_target_scene(K=64, Np=32, n=64, spacing=0.1, nfft=512, snr_db=None, seed=7, n_targets=3,
                              radius=60.0)
    ea, er = grads_vs_oracle(torch_cuda, sc, seed=2)
    assert ea < GRAD_TOL and er < GRAD_TOL, (ea, er)


def test_entropy_gradient_through_autograd_matches_finite_differences(torch_cuda):
    torch = torch_cuda
    from uncc_sar_focusing_b200 import autograd as A
    from uncc_sar_focusing_b200 import focusing

    sc = S.point_target_scene(K=96, Np=48, n=40, spacing=0.15, nfft=768, snr_db=None, seed=8, n_targets=3,
                              extent=4.0)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ax, ay, az, r0, f0 = (dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    with focusing.Plan.for_scene(sc, "mixed") as plan, focusing.Plan.for_scene(sc, "fp64") as p64:
        plan.range_compress(dev(sc.phase_history))
        p64.range_compress(dev(sc.phase_history))
        axg = ax.clone().requires_grad_(True)
        azg = az.clone().requires_grad_(True)
        img = A.backproject(plan, axg, ay, azg, r0, f0)
        E = A.image_entropy(img)
        E.backward()

        def entropy64(x, z):
            im = p64.backproject(x, ay, z, r0, f0, out=p64.new_image("cuda"))
            w = im.real ** 2 + im.imag ** 2
            p = w / w.sum()
            return float(-(p * torch.log(p.clamp_min(1e-300))).sum())

        h = 1e-6
        scale = max(axg.grad.abs().max().item(), azg.grad.abs().max().item())
        for p in (0, 17, 47):
            for which in ("x", "z"):
                up_x, dn_x, up_z, dn_z = ax.clone(), ax.clone(), az.clone(), az.clone()
                if which == "x":
                    up_x[p] += h
                    dn_x[p] -= h
                else:
                    up_z[p] += h
                    dn_z[p] -= h
                fd = (entropy64(up_x, up_z) - entropy64(dn_x, dn_z)) / (2 * h)
                got = (axg.grad if which == "x" else azg.grad)[p].item()
                assert abs(fd - got) < 2e-3 * scale, (p, which, fd, got)
