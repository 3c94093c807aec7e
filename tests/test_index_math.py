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
            # each pulse's tight window (make_geo, bp_tile.cuh): half-width
            # wp = min(W, ceil(|gam| TX/2 + |eta| 32 + lam hd^2 / (2 (Rc - hd))) + 3)
            # (W for near-field pulses), copied to entries [W - wp, W + wp + 2)
            k = 2.0 * scene.start_freq / 299792458.0
            near = (rc < 16 * P["hd"]) | (rc ** 3 < k * 0.625 * P["hd"] ** 4 / 1e-7)
            gam, eta = -P["lam"] * u[:, 0] * P["dx"], -P["lam"] * u[:, 1] * P["dy"]
            span = np.abs(gam) * (TX // 2) + np.abs(eta) * 32 + P["lam"] * P["hd"] ** 2 / (2 * (rc - P["hd"]))
            wp = np.where(near | (span >= P["W"]), P["W"], np.minimum(P["W"], np.ceil(span).astype(np.int64) + 3))
            for Bx in (B, B2):
                f = np.floor(Bx)[active]
                lo_ok = f >= (P["W"] - wp)[active, None, None]
                hi_ok = f <= (P["W"] + wp)[active, None, None]
                assert lo_ok.all() and hi_ok.all(), "a pixel's bin falls outside its pulse's tight window"
            tight_frac = float(np.mean((2 * wp + 2) / P["wsize"]))
            P["tight_frac"] = min(P.get("tight_frac", 1.0), tight_frac)
    assert worst_lo >= 0, worst_lo
    assert worst_hi <= P["wsize"] - 2, (worst_hi, P["wsize"])
    return worst_lo, worst_hi, P


@pytest.mark.parametrize("mx", [1, 2, 4, 8])
def test_point_target_config_indices(mx):
    sc = S.point_target_scene(K=424, Np=64, n=256, spacing=0.08, snr_db=None, n_targets=1)
    lo, hi, P = check_scene(sc, mx)
    assert lo >= 1 and hi <= P["wsize"] - 3  # at least one entry of margin on each side


@pytest.mark.parametrize("mx", [4, 8])
def test_large_config_indices(mx):
    sc = S.large_scene(K=64, Np=48, n=1024, n_targets=1)
    sc.nfft = 8 * 1024  # the large configuration's range sampling (max_wr from 640 MHz over 1024 samples)
    sc.delta_freq = 640e6 / 1023
    _, _, P = check_scene(sc, mx)
    if mx == 8:
        assert P["tight_frac"] < 0.7  # the tight windows copy and rewrite about 40% fewer entries


def test_volumetric_config_indices():
    sc = S.volumetric_scene(K=16, pulses_per_pass=24, elevations=(30.0, 31.4), nx=256, ny=256, nz=1,
                            n_targets=1)
    sc.nfft = 8 * 512
    sc.delta_freq = 600e6 / 511
    check_scene(sc, 8)


def test_swath_edge_and_odd_grid_indices():
    # scene wider than the swath: tiles whose windows cross the range edges
    sc = S.point_target_scene(K=32, Np=40, n=8, spacing=1.0, nfft=64, snr_db=None, n_targets=1)
    sc.grid = S.Grid(nx=70, ny=45, wx=69 * 0.9, wy=44 * 1.3, x0=3.0, y0=-2.0)
    check_scene(sc, 8)
    check_scene(sc, 4)
    check_scene(sc, 1)


def test_near_field_indices():
    sc = S.point_target_scene(K=64, Np=32, n=64, spacing=0.1, nfft=512, snr_db=None, n_targets=1, radius=60.0)
    check_scene(sc, 4)
    check_scene(sc, 8)


# ---- work split of the forward kernels (tile::sk_lo / sk_owner / sk_slot) ----

def sk_lo(c, units, G):
    return c * units // G


def sk_owner(u, units, G):
    c = u * G // units
    while c + 1 < G and sk_lo(c + 1, units, G) <= u:
        c += 1
    while c > 0 and sk_lo(c, units, G) > u:
        c -= 1
    return c


def simulate_split(tiles, stages, G):
    """Replay the kernels' unit loop: which (tile, stage range) each CTA
    accumulates, where it flushes, and what the fix-up kernel reads."""
    units = tiles * stages
    covered = np.zeros(units, dtype=np.int64)
    stored_whole = {}
    slot_writes = {}
    for c in range(G):
        lo, hi = sk_lo(c, units, G), sk_lo(c + 1, units, G)
        n = hi - lo
        seg, seg_first, seg_units = 0, lo % stages, []
        for i in range(n):
            u = lo + i
            t, b = divmod(u, stages)
            covered[u] += 1
            seg_units.append(u)
            if i + 1 == n or (u + 1) // stages != t:
                if seg_first == 0 and b == stages - 1:
                    assert t not in stored_whole
                    stored_whole[t] = c
                else:
                    slot = 2 * c + (1 if seg > 0 else 0)
                    assert slot not in slot_writes, "two segments share a partial slot"
                    slot_writes[slot] = (t, tuple(seg_units))
                seg += 1
                seg_first = 0
                seg_units = []
    assert (covered == 1).all()
    # fix-up: tiles on several CTAs sum the slots of their CTAs
    for t in range(tiles):
        c0, c1 = sk_owner(t * stages, units, G), sk_owner(t * stages + stages - 1, units, G)
        if c0 == c1:
            assert stored_whole.get(t) == c0
            continue
        assert t not in stored_whole
        got = []
        for c in range(c0, c1 + 1):
            slot = 2 * c if sk_lo(c, units, G) >= t * stages else 2 * c + 1
            tt, us = slot_writes.pop(slot)
            assert tt == t
            got.extend(us)
        assert got == list(range(t * stages, (t + 1) * stages)), "fix-up must add every stage once, in order"
    assert not slot_writes, "a partial slot nobody reads"


@pytest.mark.parametrize("tiles,stages,G", [
    (512, 256, 296), (512, 256, 148), (32, 64, 296), (1, 7, 5), (7, 1, 3), (1024, 256, 296),
    (8192, 128, 296), (3, 3, 9), (17, 5, 17), (296, 10, 296), (512, 256, 512),
])
def test_work_split_covers_every_unit_once(tiles, stages, G):
    simulate_split(tiles, stages, min(G, tiles * stages))


def test_work_split_random_shapes():
    rng = np.random.default_rng(5)
    for _ in range(200):
        tiles, stages = int(rng.integers(1, 60)), int(rng.integers(1, 40))
        G = int(rng.integers(1, tiles * stages + 1))
        simulate_split(tiles, stages, G)


def test_unit_cursor_matches_division():
    """tile::UnitCursor.advance (carry chain b -> ty -> tx -> iz -> hyp) walks
    units in the same order as the division-based decomposition of u."""
    for tiles_y, tiles_x, nz, nhyp, stages in [(16, 32, 1, 1, 256), (3, 2, 4, 5, 7), (1, 1, 1, 3, 1), (5, 1, 2, 1, 3)]:
        units = tiles_y * tiles_x * nz * nhyp * stages

        def decompose(u):
            t, b = divmod(u, stages)
            r, ty = divmod(t, tiles_y)
            q, tx = divmod(r, tiles_x)
            hyp, iz = divmod(q, nz)
            return [b, ty, tx, iz, hyp]

        for start in sorted({0, 1, units // 3, units - 2, units - 1}):
            cur = decompose(start)
            for u in range(start, min(units, start + 3 * stages + 5)):
                assert cur == decompose(u)
                b, ty, tx, iz, hyp = cur
                b += 1
                if b == stages:
                    b, ty = 0, ty + 1
                    if ty == tiles_y:
                        ty, tx = 0, tx + 1
                        if tx == tiles_x:
                            tx, iz = 0, iz + 1
                            if iz == nz:
                                iz, hyp = 0, hyp + 1
                cur = [b, ty, tx, iz, hyp]


def stage_rotation(t, stages, units, G):
    """SceneCursor::set_rot (bp_mixed.cu): unit t S + b of tile t processes
    pulse stage (b + rot_t) mod S, rot_t = t S - lo(owner of unit t S)."""
    first = t * stages
    return (first - sk_lo(sk_owner(first, units, G), units, G)) % stages


@pytest.mark.parametrize("tiles,stages,G", [
    (256, 256, 296), (512, 256, 296), (1024, 256, 296), (32, 64, 296), (17, 5, 17), (3, 3, 9), (7, 1, 3),
    (8192, 128, 296), (256, 256, 256),
])
def test_stage_rotation_walks_resident_ctas_in_step(tiles, stages, G):
    """Every tile still processes each of its pulse stages exactly once, and
    a CTA works on stage k mod S at its local step k, except on its first
    (partial) tile, which runs lo(c) - lo(owner of that tile) stages off: the
    CTAs resident together stage nearby pulses through L2."""
    units = tiles * stages
    G = min(G, units)
    for t in range(tiles):
        r = stage_rotation(t, stages, units, G)
        assert sorted((b + r) % stages for b in range(stages)) == list(range(stages))
    for c in range(G):
        lo, hi = sk_lo(c, units, G), sk_lo(c + 1, units, G)
        for k, u in enumerate(range(lo, hi)):
            t, b = divmod(u, stages)
            stage = (b + stage_rotation(t, stages, units, G)) % stages
            off = (stage - k) % stages
            owner = sk_owner(t * stages, units, G)
            if owner == c:
                assert off == 0
            else:
                assert k < stages and off == (lo - sk_lo(owner, units, G)) % stages
