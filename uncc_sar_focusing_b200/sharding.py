"""Pixel sharding across ranks (one process per GPU).

Backprojection pixels are independent and every rank needs the whole
aperture, so the image is cut into contiguous slabs along y (the fast axis
of the x-major layout) with no exchange on the data path; the reference has
no distributed mode at all.  `slab_grid` gives rank r its slab as a grid of
its own, on exactly the pixel positions of the full grid; `gather_slabs`
assembles the full image on every rank with one all_gather (used when a
caller wants the whole image; the throughput bench does not gather).

Gradient autofocus on a sharded image has one real exchange per step:
`sharded_entropy_gradient` all-reduces the image power and sum p log p
(two scalars) so every rank can form its slab's upstream gradient, runs the
adjoint on its slab, and all-reduces the 4 Np per-pulse gradients.
"""
from __future__ import annotations

import dataclasses
from typing import Tuple

from .scenes import Grid


def slab_bounds(n: int, rank: int, world: int) -> Tuple[int, int]:
    """[start, stop) of rank's share of n indices, sizes differing by at most one."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def slab_grid(grid: Grid, rank: int, world: int) -> Grid:
    """Rank's slab of `grid` along y: columns [start, stop) of the full grid,
    as a Grid whose pixel j sits where full-grid pixel start + j sits."""
    start, stop = slab_bounds(grid.ny, rank, world)
    n = stop - start
    if n < 1:
        raise ValueError(f"rank {rank} of {world} gets no columns of a {grid.ny}-column grid")
    dy = grid.wy / (grid.ny - 1) if grid.ny > 1 else 0.0
    y_first = (grid.y0 - 0.5 * grid.wy if grid.ny > 1 else grid.y0) + start * dy
    wy = (n - 1) * dy
    return dataclasses.replace(grid, ny=n, y0=y_first + 0.5 * wy, wy=wy)


def weak_scaling_grid(per_rank: Grid, world: int) -> Grid:
    """The full grid whose world slabs each have per_rank's size and spacing,
    centred where per_rank is centred (weak scaling: fixed work per rank)."""
    dy = per_rank.wy / (per_rank.ny - 1) if per_rank.ny > 1 else 0.0
    ny = per_rank.ny * world
    return dataclasses.replace(per_rank, ny=ny, wy=(ny - 1) * dy)


def gather_slabs(slab, grid: Grid, group=None):
    """All-gather every rank's [nz, nx, ny_r] slab into the full [nz, nx, ny]
    image (torch tensors; slabs may differ in width by one column)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    widths = [slab_bounds(grid.ny, r, world) for r in range(world)]
    wmax = max(b - a for a, b in widths)
    pad = torch.zeros(slab.shape[:-1] + (wmax,), dtype=slab.dtype, device=slab.device)
    pad[..., : slab.shape[-1]] = slab
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[..., : b - a] for p, (a, b) in zip(parts, widths)], dim=-1)


def sharded_entropy_gradient(slab, adjoint, group=None):
    """Entropy of the whole image and its gradient with respect to the
    per-pulse geometry, when every rank holds one slab of the image.

    E = -sum_q p_q log p_q with p_q = |I_q|^2 / S, S = sum_q |I_q|^2 over all
    ranks' pixels, so dE/d|I_q|^2 = -(log p_q + E) / S and the upstream
    gradient of pixel q (dE/dRe + j dE/dIm) is G_q = -2 (log p_q + E) I_q / S:
    after two scalar all-reduces (S and sum p log p) each rank forms G on its
    own slab.  `adjoint(G)` returns this rank's (grad_ant [3, Np],
    grad_r0 [Np]) for its slab (e.g. Plan.backproject_adjoint bound to the
    geometry, or the FP64 oracle); the per-pulse gradients are sums over
    pixels, so one all-reduce of 4 Np doubles gives the whole image's.

    slab: complex tensor [nz, nx, ny_r].  Returns (E, grad_ant, grad_r0),
    the same on every rank (float64 tensors on slab's device).  Collectives
    run on `group` (default: the world); with NCCL, slab lives on this rank's
    GPU."""
    import torch
    import torch.distributed as dist

    w = slab.real.double() ** 2 + slab.imag.double() ** 2
    S = w.sum().reshape(1)
    dist.all_reduce(S, group=group)
    p = w / S
    logp = torch.log(p.clamp_min(1e-300))
    plogp = (p * logp).sum().reshape(1)
    dist.all_reduce(plogp, group=group)
    E = -plogp
    G = (-2.0 * (logp + E) / S) * slab.to(torch.complex128)
    grad_ant, grad_r0 = adjoint(G.to(slab.dtype))
    grad_ant = torch.as_tensor(grad_ant, dtype=torch.float64, device=slab.device)
    grad_r0 = torch.as_tensor(grad_r0, dtype=torch.float64, device=slab.device)
    n = grad_r0.numel()
    packed = torch.cat([grad_ant.reshape(-1), grad_r0.reshape(-1)])
    dist.all_reduce(packed, group=group)
    return E[0], packed[: 3 * n].reshape(3, n), packed[3 * n:]
