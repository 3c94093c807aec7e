"""Pixel sharding across ranks, on CPU with the gloo backend (world size 2):
the slabs of the full grid, each formed independently (FP64 oracle), gather
into exactly the single-process image; timings reduce to the max over ranks;
weak-scaling grids keep per-rank work fixed."""
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
