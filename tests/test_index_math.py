"""CPU proof that the backprojection kernels stay inside their buffers.

Re-derives, in numpy, the window geometry the host code in
uncc_sar_focusing_b200/csrc/api.cu chooses (window half-width W, window size,
guard band, row stride) and the per-(tile, pulse) window start the kernels in
bp_mixed.cu / bp_fp64.cu compute, then checks for every tile, pulse and pixel
of the scenes that
  * each bulk copy [ws, ws + wsize) lies inside the guarded row
    [-guard, nfft + guard), and
  * every pixel's bin relative to its window start has floor in
    [0, wsize - 2], so the pair entry read from shared memory is in the
    window, both for the exact range and for the far-field expansion the
    mixed kernel uses.
This runs before any kernel touches a GPU.
"""
import math

import numpy as np
import pytest

from uncc_sar_focusing_b200 import scenes as S


def plan_geometry(scene, mx):
    g = scene.grid
    lam = scene.nfft / scene.max_wr
    dx = g.wx / (g.nx - 1) if g.nx > 1 else 0.0
    dy = g.wy / (g.ny - 1) if g.ny > 1 else 0.0
    hx, hy = 0.5 * 8 * mx * dx, 0.5 * 64 * dy
    hd = math.sqrt(hx * hx + hy * hy)
    W = int(math.ceil(lam * hd)) + 3
    wsize = 2 * W + 2
    guard = wsize + 2
    return dict(lam=lam, dx=dx, dy=dy, hd=hd, W=W, wsize=wsize, guard=guard,
                left=g.x0 - 0.5 * g.wx if g.nx > 1 else g.x0, bottom=g.y0 - 0.5 * g.wy if g.ny > 1 else g.y0)


def check_scene(scene, mx):
    P = plan_geometry(scene, mx)
    g = scene.grid
    TX, TY = 8 * mx, 64
    nfft = scene.nfft
    ant = np.stack([scene.ant_x, scene.ant_y, scene.ant_z], 1)
    # pixel offsets of a tile relative to its centre (integers)
    ii, jj = np.meshgrid(np.arange(TX) - TX // 2, np.arange(TY) - TY // 2, indexing="ij")
    worst_lo, worst_hi = np.inf, -np.inf
    for tx0 in range(0, g.nx, TX):
        for ty0 in range(0, g.ny, TY):
            c = np.array([P["left"] + (tx0 + TX // 2) * P["dx"], P["bottom"] + (ty0 + TY // 2) * P["dy"], g.z0])
            v = ant - c[None, :]
            rc = np.linalg.norm(v, axis=1)
            D = rc - scene.slant_range
            bc = D * P["lam"] + nfft / 2
            ws = np.floor(bc).astype(np.int64) - P["W"]
            active = ~((ws + P["wsize"] - 2 <= 0) | (ws + 1 >= nfft - 1))
            # bulk copy source range inside the guarded row
            assert np.all(ws[active] >= -P["guard"])
            assert np.all(ws[active] + P["wsize"] <= nfft + P["guard"])
            # exact bins of every tile pixel
            px = c[0] + ii * P["dx"]
            py = c[1] + jj * P["dy"]
            d = np.sqrt((ant[:, 0, None, None] - px[None]) ** 2 + (ant[:, 1, None, None] - py[None]) ** 2 +
                        (ant[:, 2, None, None] - g.z0) ** 2)
            B = (d - scene.slant_range[:, None, None]) * P["lam"] + nfft / 2 - ws[:, None, None]
            # far-field expansion used by the mixed kernel
            u = v / rc[:, None]
            t = u[:, 0, None, None] * (ii * P["dx"])[None] + u[:, 1, None, None] * (jj * P["dy"])[None]
            e = (ii * P["dx"]) ** 2 + (jj * P["dy"]) ** 2 - t * t
            gg = e * (0.5 / rc[:, None, None] + t * 0.5 / rc[:, None, None] ** 2)
            B2 = (bc - ws)[:, None, None] - P["lam"] * t + P["lam"] * gg
            for Bx in (B, B2):
                f = np.floor(Bx[active])
                worst_lo = min(worst_lo, f.min())
                worst_hi = max(worst_hi, f.max())
    assert worst_lo >= 0, worst_lo
    assert worst_hi <= P["wsize"] - 2, (worst_hi, P["wsize"])
    return worst_lo, worst_hi, P


@pytest.mark.parametrize("mx", [1, 2, 4])
def test_point_target_config_indices(mx):
    sc = S.point_target_scene(K=424, Np=64, n=256, spacing=0.08, snr_db=None, n_targets=1)
    lo, hi, P = check_scene(sc, mx)
    assert lo >= 1 and hi <= P["wsize"] - 3  # at least one entry of margin on each side


def test_large_config_indices():
    sc = S.large_scene(K=64, Np=48, n=1024, n_targets=1)
    sc.nfft = 8 * 1024  # the large configuration's range sampling (max_wr from 640 MHz over 1024 samples)
    sc.delta_freq = 640e6 / 1023
    check_scene(sc, 4)


def test_swath_edge_and_odd_grid_indices():
    # scene wider than the swath: tiles whose windows cross the range edges
    sc = S.point_target_scene(K=32, Np=40, n=8, spacing=1.0, nfft=64, snr_db=None, n_targets=1)
    sc.grid = S.Grid(nx=70, ny=45, wx=69 * 0.9, wy=44 * 1.3, x0=3.0, y0=-2.0)
    check_scene(sc, 4)
    check_scene(sc, 1)


def test_near_field_indices():
    sc = S.point_target_scene(K=64, Np=32, n=64, spacing=0.1, nfft=512, snr_db=None, n_targets=1, radius=60.0)
    check_scene(sc, 4)
