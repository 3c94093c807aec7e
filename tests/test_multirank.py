"""Pixel sharding across ranks, on CPU with the gloo backend (world size 2):
the slabs of the full grid, each formed independently (FP64 oracle), gather
into exactly the single-process image; timings reduce to the max over ranks;
the sharded entropy-gradient step reproduces the whole image's entropy and
per-pulse geometry gradient; weak-scaling grids keep per-rank work fixed."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S
from uncc_sar_focusing_b200 import sharding as SH


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def scene():
    sc = S.point_target_scene(K=48, Np=24, n=16, spacing=0.3, nfft=256, snr_db=20.0, seed=4, n_targets=3)
    sc.grid = S.Grid(nx=14, ny=21, x0=0.2, y0=-0.4, wx=13 * 0.3, wy=20 * 0.25)
    return sc


def worker(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = scene()
        full = sc.grid
        sc.grid = SH.slab_grid(full, rank, world)
        slab = torch.as_tensor(O.focus_fp64(sc))
        img = SH.gather_slabs(slab, full)
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            np.save(out_path, img.numpy())
            assert t.item() == world
    finally:
        dist.destroy_process_group()


def grad_worker(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = scene()
        full = sc.grid
        sc.grid = SH.slab_grid(full, rank, world)
        slab = torch.as_tensor(O.focus_fp64(sc))
        rc = O.range_compress_fp64(sc.phase_history, sc.nfft, O.window_for(sc.window, sc.num_range_samples))

        def adjoint(G):
            return O.bp_grad_fp64(rc, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq, sc.max_wr,
                                  sc.grid, G.numpy().astype(np.complex128))

        E, ga, gr = SH.sharded_entropy_gradient(slab, adjoint)
        if rank == 0:
            np.savez(out_path, E=E.item(), ga=ga.numpy(), gr=gr.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_entropy_gradient_matches_the_whole_image(tmp_path):
    """Sharded gradient autofocus step: two scalar all-reduces and one of the
    per-pulse gradients reproduce the single-process entropy and geometry
    gradient (image gradient by torch autograd here, FP64 oracle adjoint)."""
    out = str(tmp_path / "grad.npz")
    mp.start_processes(grad_worker, args=(2, free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    sc = scene()
    img = O.focus_fp64(sc)
    re = torch.tensor(img.real, requires_grad=True)
    im = torch.tensor(img.imag, requires_grad=True)
    w = re ** 2 + im ** 2
    p = w / w.sum()
    E = -(p * torch.log(p)).sum()
    E.backward()
    G = (re.grad + 1j * im.grad).numpy()
    rc = O.range_compress_fp64(sc.phase_history, sc.nfft, O.window_for(sc.window, sc.num_range_samples))
    want_a, want_r = O.bp_grad_fp64(rc, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq, sc.max_wr,
                                    sc.grid, G)
    assert abs(float(got["E"]) - E.item()) <= 1e-12 * abs(E.item())
    scale = max(np.abs(want_a).max(), np.abs(want_r).max())
    assert np.abs(got["ga"] - want_a).max() <= 1e-9 * scale
    assert np.abs(got["gr"] - want_r).max() <= 1e-9 * scale


def test_two_rank_slabs_gather_to_the_full_image(tmp_path):
    out = str(tmp_path / "img.npy")
    mp.start_processes(worker, args=(2, free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    sc = scene()
    want = O.focus_fp64(sc)
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("n,world", [(21, 2), (1024, 8), (7, 7), (10, 3)])
def test_slab_bounds_partition(n, world):
    spans = [SH.slab_bounds(n, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def test_slab_pixel_positions_match_the_full_grid():
    full = S.Grid(nx=5, ny=23, x0=1.0, y0=-3.0, wx=4.0, wy=11.0)
    ys = full.axis("y")
    got = np.concatenate([SH.slab_grid(full, r, 4).axis("y") for r in range(4)])
    assert np.allclose(got, ys, atol=1e-12)


def test_weak_scaling_grid_keeps_per_rank_work():
    per = S.Grid(nx=1024, ny=1024, wx=100.0, wy=100.0)
    full = SH.weak_scaling_grid(per, 8)
    for r in range(8):
        g = SH.slab_grid(full, r, 8)
        assert g.ny == 1024 and abs(g.wy - 100.0) < 1e-9


def nccl_worker(rank, world, port, out_path):
    from uncc_sar_focusing_b200 import focusing

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=rank, world_size=world, device_id=torch.device("cuda:0"))
    try:
        sc = S.point_target_scene(K=96, Np=48, n=40, spacing=0.15, nfft=768, snr_db=None, seed=8, n_targets=3,
                                  extent=4.0)
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
        geo = [dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)]
        with focusing.Plan.for_scene(sc, "mixed") as plan:
            img = plan.focus(dev(sc.phase_history), *geo, out=plan.new_image("cuda"))
            E, ga, gr = SH.sharded_entropy_gradient(img, lambda G: plan.backproject_adjoint(*geo, G))
            torch.cuda.synchronize()
            np.savez(out_path, E=E.item(), ga=ga.cpu().numpy(), gr=gr.cpu().numpy(), img=img.cpu().numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_entropy_gradient_on_the_engine_with_nccl(tmp_path):
    """The same step on the GPU engine over NCCL (one rank: every collective
    runs, on device tensors): entropy and gradient equal the engine's own
    autograd path on the whole image."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from uncc_sar_focusing_b200 import autograd as A
    from uncc_sar_focusing_b200 import focusing

    out = str(tmp_path / "nccl.npz")
    mp.start_processes(nccl_worker, args=(1, free_port(), out), nprocs=1, join=True, start_method="spawn")
    got = np.load(out)
    sc = S.point_target_scene(K=96, Np=48, n=40, spacing=0.15, nfft=768, snr_db=None, seed=8, n_targets=3,
                              extent=4.0)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ax, ay, az, r0, f0 = (dev(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(dev(sc.phase_history))
        axg, ayg, azg, r0g = (t.clone().requires_grad_(True) for t in (ax, ay, az, r0))
        img = A.backproject(plan, axg, ayg, azg, r0g, f0)
        E = A.image_entropy(img)
        E.backward()
        want_a = torch.stack([axg.grad, ayg.grad, azg.grad]).cpu().numpy()
        want_r = r0g.grad.cpu().numpy()
    assert np.allclose(got["img"], img.detach().cpu().numpy(), rtol=0, atol=1e-6 * np.abs(got["img"]).max())
    assert abs(float(got["E"]) - E.item()) <= 1e-5 * abs(E.item())
    scale = max(np.abs(want_a).max(), np.abs(want_r).max())
    assert np.abs(got["ga"] - want_a).max() <= 1e-3 * scale
    assert np.abs(got["gr"] - want_r).max() <= 1e-3 * scale
