"""Motion-error autofocus on top of the backprojection engine.

* `CubicMotion`: per-axis cubic in normalised slow time, 12 coefficients
  (the reference's grid search fits linear or quadratic tracks with a velocity
  scale, src/autofocus/autofocus_gpu.cu:315-416 and
  gridSearchErrorFunctions_dft.cuh:279-291; the same family one degree higher).
* `gradient_autofocus`: minimises image entropy over the coefficients with the
  gradient from the adjoint backprojection kernel (autograd.backproject).
* `grid_search_autofocus`: the reference's search scheme restated on this
  engine -- a box of `points` samples per searched coefficient around the
  current estimate, every grid point imaged (hypothesis batches of
  sarbp_backproject_hypotheses), the best kept, the box halved, repeated
  (autofocus_gpu.cu:843-952, the halving at :938-939).  The reference's own
  implementation cannot run these sizes (Np <= 200, Nx <= 500 per
  gridSearchErrorFunctions_dft.cuh:37,41,275-277) and depends on the
  un-vendored cuGridSearch, so the comparison uses this restatement.
* `pga`: phase gradient autofocus as matlab/PGA.m:153-239 (circular shift of
  the brightest azimuth sample to the centre, -30 dB window, azimuth FFT,
  phi_dot = sum Im(conj(G) dG) / sum |G|^2, integrate, unwrap, remove the
  linear trend, apply exp(-j phi) in the azimuth-frequency domain), on the GPU
  with torch FFTs.
* focus metrics: entropy, sharpness, and the reference's own grid-search
  cost (2-D DFT low-frequency energy of the 8-bit dB image,
  gridSearchErrorFunctions_dft.cuh:102-109,112-203,320-335).
"""
from __future__ import annotations

import dataclasses
import math
import time
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import autograd as A
from .focusing import Plan


def slow_time(num_pulses: int, device=None) -> torch.Tensor:
    return torch.linspace(-1.0, 1.0, num_pulses, dtype=torch.float64, device=device)


class CubicMotion:
    """Track correction a(theta) = a_measured + theta @ [1, tau, tau^2, tau^3]
    per axis; theta is [3, 4] (12 coefficients, metres)."""

    def __init__(self, ant_x, ant_y, ant_z):
        self.base = torch.stack([ant_x, ant_y, ant_z])  # [3, Np]
        tau = slow_time(self.base.shape[1], self.base.device)
        self.powers = torch.stack([tau ** n for n in range(4)])  # [4, Np]

    def track(self, theta: torch.Tensor) -> torch.Tensor:
        return self.base + theta @ self.powers


def entropy(img: torch.Tensor) -> torch.Tensor:
    return A.image_entropy(img)


def batch_entropy(imgs: torch.Tensor) -> torch.Tensor:
    """Entropy of each image of a [H, ...] batch."""
    w = (imgs.real.float() ** 2 + imgs.imag.float() ** 2).reshape(imgs.shape[0], -1)
    p = w / w.sum(dim=1, keepdim=True)
    return -(p * torch.log(p.clamp_min(1e-30))).sum(dim=1)


def reference_u8_image(img: torch.Tensor, dyn_range_db: float = 70.0) -> torch.Tensor:
    """The reference's 8-bit dB mapping (gridSearchErrorFunctions_dft.cuh:
    102-109): (255/dyn) (20 log10(|p|/max) + dyn), negative values to 0,
    then truncation to unsigned char."""
    mag = img.abs().float()
    pixelf = (255.0 / dyn_range_db) * (20.0 * torch.log10(mag / mag.max()) + dyn_range_db)
    return torch.where(pixelf < 0, torch.zeros_like(pixelf), torch.trunc(pixelf))


def reference_dft_cost(img: torch.Tensor, dyn_range_db: float = 70.0, percentage: float = 0.35) -> float:
    """The reference grid search's focus cost restated
    (gridSearchErrorFunctions_dft.cuh:112-203,320-335): the 2-D DFT F of the
    8-bit image (x-major [Nx][Ny]), and for every x and every y < Ny/2 whose
    squared index distance to the (0, 0) or (Nx-1, 0) corner is below
    int((Ny/2)^2 + (Nx/2)^2) * percentage^2, |F[x][y]| + |F[x][Ny-1-y]| summed;
    the cost is minus that sum.  The reference kernel computes this for one
    image per CUDA block with Nx <= 500; here any size, with torch's FFT."""
    u8 = reference_u8_image(img.reshape(img.shape[-2], img.shape[-1]), dyn_range_db).double()
    F = torch.fft.fft2(u8).abs()
    nx, ny = F.shape
    hh, hw = ny // 2, nx // 2
    threshold = int((hh * hh + hw * hw) * (percentage * percentage))
    x = torch.arange(nx, device=F.device)[:, None]
    y = torch.arange(hh, device=F.device)[None, :]
    r = x * x + y * y
    r2 = (nx - x - 1) * (nx - x - 1) + y * y
    mask = (r < threshold) | (r2 < threshold)
    vals = F[:, :hh] + F[:, ny - 1 - torch.arange(hh, device=F.device)]
    return -float((vals * mask).sum())


def _descend(step, iters: int, lr_at, lr: torch.Tensor, record, graph: bool, warm: int = 10):
    """Run `iters` descent steps; `step()` does one (forward, entropy,
    backward, optimiser step) on static tensors.  With graph=True the first
    `warm` steps run eagerly (they initialise the optimiser state and every
    lazily allocated buffer, and the first steps, where a descent from a
    metre-scale error gains the most, do not wait for the capture) and the
    rest replay one CUDA graph captured right after them
    (capture_begin/capture_end on a side stream: the capture itself executes
    nothing).  Before step it the learning-rate tensor holds
    lr_at(it); after it `record(it)` copies the step's outputs on the device.
    Returns (seconds, completion events; events[0] = start), the events on
    the GPU clock, the capture included in the wall time."""
    events = [torch.cuda.Event(enable_timing=True) for _ in range(iters + 1)]
    cur = torch.cuda.current_stream()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    side = torch.cuda.Stream() if graph else cur
    side.wait_stream(cur)
    g = None
    with torch.cuda.stream(side):
        events[0].record()
        for it in range(iters):
            lr.fill_(lr_at(it))
            if graph and g is None and it == warm:
                g = torch.cuda.CUDAGraph()
                g.capture_begin()
                step()
                g.capture_end()
            if g is not None:
                g.replay()
            else:
                step()
            record(it)
            events[it + 1].record()
    cur.wait_stream(side)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    del g
    return seconds, events


@dataclasses.dataclass
class AutofocusResult:

    theta: torch.Tensor
    history: List[dict]
    seconds: float
    images_formed: int


def gradient_autofocus(plan: Plan, motion: CubicMotion, slant_range, start_freq, iters: int = 200,
                       lr: float = 0.02, theta0: Optional[torch.Tensor] = None, coarse_to_fine: bool = True,
                       log_every: int = 1, graph: bool = True) -> AutofocusResult:
    """Adam on the 12 coefficients, loss = image entropy, gradient through the
    adjoint backprojection.  With coarse_to_fine the step size decays from
    `lr` metres to lr/100 (cosine, as CosineAnnealingLR), which lets the first
    steps cross the large blur of a metre-scale track error and the last ones
    settle.  Each step is replayed from a captured CUDA graph (graph=False:
    eager); entropies and parameters stay on the device and the steps are
    timed with CUDA events, so the host never waits inside the loop."""
    dev = motion.base.device
    start = theta0.clone() if theta0 is not None else torch.zeros((3, 4), dtype=torch.float64, device=dev)
    theta = start.clone().requires_grad_(True)
    lr_t = torch.tensor(lr, dtype=torch.float64, device=dev)
    opt = torch.optim.Adam([theta], lr=lr_t, capturable=True)
    eta_min = lr / 100.0

    def lr_at(it):
        return eta_min + 0.5 * (lr - eta_min) * (1.0 + math.cos(math.pi * it / iters)) if coarse_to_fine else lr

    e_out = torch.zeros((), dtype=torch.float64, device=dev)
    theta_pre = torch.zeros_like(start)

    def step():
        opt.zero_grad(set_to_none=False)
        theta_pre.copy_(theta.detach())
        a = motion.track(theta)
        img = A.backproject(plan, a[0].contiguous(), a[1].contiguous(), a[2].contiguous(), slant_range,
                            start_freq)
        E = A.image_entropy(img)
        E.backward()
        e_out.copy_(E.detach())
        opt.step()

    ents = torch.empty(iters, dtype=torch.float64, device=dev)
    thetas = torch.empty((iters, 3, 4), dtype=torch.float64, device=dev)

    def record(it):
        ents[it] = e_out
        thetas[it] = theta_pre

    seconds, events = _descend(step, iters, lr_at, lr_t, record, graph)
    e_host = ents.cpu().tolist()
    best = min(range(iters), key=lambda i: e_host[i])
    hist = [{"iter": it, "entropy": e_host[it], "t": events[0].elapsed_time(events[it + 1]) * 1e-3}
            for it in range(iters) if (log_every and (it % log_every == 0 or it == iters - 1)) or not log_every]
    return AutofocusResult(theta=thetas[best].clone(), history=hist, seconds=seconds, images_formed=iters)


def grid_search_autofocus(plan: Plan, motion: CubicMotion, slant_range, start_freq, span: float,
                          coeffs: Sequence[tuple] = ((0, 2), (0, 3), (1, 2), (1, 3), (2, 2), (2, 3)),
                          points: int = 5, levels: int = 4, batch: int = 256,
                          theta0: Optional[torch.Tensor] = None, deadline_s: Optional[float] = None,
                          target_entropy: Optional[float] = None) -> AutofocusResult:
    """Exhaustive multiresolution search: `points` samples in +-span around
    the estimate for each searched coefficient (axis, power), every
    combination imaged and scored by entropy, the best kept, span halved,
    `levels` times.  Stops early at `deadline_s` or once `target_entropy` is
    reached (time-to-target measurement)."""
    dev = motion.base.device
    theta = theta0.clone() if theta0 is not None else torch.zeros((3, 4), dtype=torch.float64, device=dev)
    Np = motion.base.shape[1]
    hist = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    formed = 0
    best_e = float("inf")
    ncoef = len(coeffs)
    offsets1d = torch.linspace(-1.0, 1.0, points, dtype=torch.float64, device=dev)
    mesh = torch.stack(torch.meshgrid(*([offsets1d] * ncoef), indexing="ij"), dim=-1).reshape(-1, ncoef)
    r0 = slant_range.reshape(1, -1)
    f0 = start_freq.reshape(1, -1)
    done = False
    for level in range(levels):
        s = span / (2 ** level)
        best_level = (float("inf"), None)
        for b0 in range(0, mesh.shape[0], batch):
            cand = mesh[b0:b0 + batch] * s  # [H, ncoef]
            H = cand.shape[0]
            th = theta.unsqueeze(0).repeat(H, 1, 1)
            for j, (ax_i, pw) in enumerate(coeffs):
                th[:, ax_i, pw] = theta[ax_i, pw] + cand[:, j]
            tracks = motion.base.unsqueeze(0) + th @ motion.powers  # [H, 3, Np]
            imgs = plan.backproject_hypotheses(tracks[:, 0].contiguous(), tracks[:, 1].contiguous(),
                                               tracks[:, 2].contiguous(), r0.expand(H, Np).contiguous(),
                                               f0.expand(H, Np).contiguous())
            ent = batch_entropy(imgs)
            formed += H
            k = int(torch.argmin(ent))
            if float(ent[k]) < best_level[0]:
                best_level = (float(ent[k]), th[k].clone())
            if deadline_s is not None and time.perf_counter() - t0 > deadline_s:
                done = True
                break
        if best_level[1] is not None and best_level[0] < best_e:
            best_e = best_level[0]
            theta = best_level[1]
        hist.append({"level": level, "entropy": best_e, "t": time.perf_counter() - t0, "images": formed})
        if done or (target_entropy is not None and best_e <= target_entropy):
            break
    torch.cuda.synchronize()
    return AutofocusResult(theta=theta, history=hist, seconds=time.perf_counter() - t0, images_formed=formed)


def pga(img: torch.Tensor, max_iter: int = 30, db_down: float = 30.0, rms_stop: float = 0.1,
        az_axis: int = -1):
    """Phase gradient autofocus of a 2-D complex image (matlab/PGA.m:153-239).
    Returns (corrected image, accumulated phase correction, rms history)."""
    x = img.to(torch.complex64)
    if az_axis not in (-1, x.dim() - 1):
        x = x.transpose(az_axis, -1)
    rows, n = x.shape[-2], x.shape[-1]
    c = (n + 1) // 2  # MATLAB center_az_idx = ceil(n/2) (1-based)
    center = c - 1  # its 0-based index: the window splits at [0, c) / [c, n)
    col = torch.arange(n, device=x.device)
    total = torch.zeros(n, dtype=torch.float64, device=x.device)
    rms_hist = []
    for _ in range(max_iter):
        # brightest azimuth sample of each range line to 0-based index c:
        # circshift(row, 1 + c - m) with m the 1-based peak (:159-164)
        peak = torch.argmax(x.abs(), dim=-1)
        idx = (col[None, :] - (c - peak)[:, None]) % n
        f = torch.gather(x, -1, idx)
        # -30 dB window from the non-coherent average of the image (:167-188)
        avg = (x.real ** 2 + x.imag ** 2).sum(dim=0)
        avg_db = 10.0 * torch.log10(avg / avg.max() + 1e-30)
        cutoff = avg_db.max() - abs(db_down)
        below_left = torch.nonzero(avg_db[:center + 1] - cutoff < 0).flatten()
        below_right = torch.nonzero(avg_db[center + 1:] - cutoff < 0).flatten()
        left = int(below_left[-1]) + 1 if below_left.numel() else 0
        right = int(below_right[0]) + center if below_right.numel() else n - 1
        mask = ((col >= left) & (col <= right)).to(f.real.dtype)
        g = f * mask[None, :]
        # azimuth FFT of the ifftshifted lines, phase-gradient estimate (:195-201)
        G = torch.fft.fft(torch.fft.ifftshift(g, dim=-1), dim=-1).to(torch.complex128)
        dG = G[:, 1:] - G[:, :-1]
        num = (G[:, :-1].conj() * dG).imag.sum(dim=0)
        den = (G[:, :-1].abs() ** 2).sum(dim=0).clamp_min(1e-300)
        phi_dot = num / den
        phi = torch.cat([torch.zeros(1, dtype=torch.float64, device=x.device), torch.cumsum(phi_dot, 0)])
        phi = torch.from_numpy(np.unwrap(phi.cpu().numpy())).to(x.device)
        # remove the linear trend (:209-212)
        xs = torch.arange(n, dtype=torch.float64, device=x.device)
        A_ = torch.stack([xs, torch.ones_like(xs)], dim=1)
        coef = torch.linalg.lstsq(A_, phi[:, None]).solution[:, 0]
        phi = phi - (coef[0] * xs + coef[1])
        rms = float(torch.sqrt(torch.mean(phi ** 2)))
        rms_hist.append(rms)
        total = total + phi
        # apply exp(-j phi) in the azimuth-frequency domain (:229-232)
        X = torch.fft.fft(x, dim=-1) * torch.exp(-1j * phi).to(torch.complex64)[None, :]
        x = torch.fft.ifft(X, dim=-1)
        if rms < rms_stop:
            break
    if az_axis not in (-1, x.dim() - 1):
        x = x.transpose(az_axis, -1)
    return x, total, rms_hist


def line_of_sight_autofocus(plan: Plan, ant_x, ant_y, ant_z, slant_range, start_freq, iters: int = 200,
                            lr: float = 2e-3, graph: bool = True) -> tuple:
    """Second stage: one slant-range offset per pulse (the line-of-sight part
    of a track error that no low-order polynomial represents, e.g. a random
    walk), entropy minimised with the adjoint's dL/dR0, steps replayed from a
    captured CUDA graph as in gradient_autofocus.  Returns (best slant range
    tensor, history, seconds)."""
    dev = slant_range.device
    dr = torch.zeros_like(slant_range, requires_grad=True)
    lr_t = torch.tensor(lr, dtype=torch.float64, device=dev)
    opt = torch.optim.Adam([dr], lr=lr_t, capturable=True)
    e_out = torch.zeros((), dtype=torch.float64, device=dev)
    r_pre = torch.zeros_like(slant_range)

    def step():
        opt.zero_grad(set_to_none=False)
        r = slant_range + dr
        r_pre.copy_(r.detach())
        E = A.image_entropy(A.backproject(plan, ant_x, ant_y, ant_z, r, start_freq))
        E.backward()
        e_out.copy_(E.detach())
        opt.step()

    ents = torch.empty(iters, dtype=torch.float64, device=dev)
    ranges = torch.empty((iters,) + tuple(slant_range.shape), dtype=slant_range.dtype, device=dev)

    def record(it):
        ents[it] = e_out
        ranges[it] = r_pre

    seconds, events = _descend(step, iters, lambda it: lr, lr_t, record, graph)
    e_host = ents.cpu().tolist()
    best = min(range(iters), key=lambda i: e_host[i])
    hist = [{"iter": it, "entropy": e_host[it], "t": events[0].elapsed_time(events[it + 1]) * 1e-3}
            for it in range(iters)]
    return ranges[best].clone().contiguous(), hist, seconds


def focus_motion_error(plan: Plan, ant_x, ant_y, ant_z, slant_range, start_freq, cubic_iters: int = 300,
                       cubic_lr: float = 0.02, los_iters: int = 200, los_lr: float = 2e-3,
                       pga_iters: int = 30) -> dict:
    """Gradient autofocus pipeline on the plan's range profiles:
    (1) the 12 cubic track coefficients, (2) a per-pulse line-of-sight
    correction, both by entropy descent through the adjoint backprojection,
    (3) PGA, the reference's own phase-only refinement.  Returns the corrected
    geometry, the final image and a timeline of (seconds, entropy)."""
    motion = CubicMotion(ant_x, ant_y, ant_z)
    t_start = time.perf_counter()
    timeline = []
    r1 = gradient_autofocus(plan, motion, slant_range, start_freq, iters=cubic_iters, lr=cubic_lr, log_every=0)
    running = float("inf")
    for h in r1.history:
        running = min(running, h["entropy"])
        timeline.append((h["t"], running, "cubic"))
    a = motion.track(r1.theta)
    ax, ay, az = (a[i].contiguous() for i in range(3))
    t1 = time.perf_counter() - t_start
    r0, h2, s2 = line_of_sight_autofocus(plan, ax, ay, az, slant_range, start_freq, iters=los_iters, lr=los_lr)
    for h in h2:
        running = min(running, h["entropy"])
        timeline.append((t1 + h["t"], running, "line_of_sight"))
    img = plan.backproject(ax, ay, az, r0, start_freq, out=plan.new_image(ax.device))
    t2 = time.perf_counter() - t_start
    img_pga, phi, rms = pga(img[0], max_iter=pga_iters)
    torch.cuda.synchronize()
    e_pga = float(A.image_entropy(img_pga))
    t3 = time.perf_counter() - t_start
    timeline.append((t3, min(running, e_pga), "pga"))
    final = img_pga if e_pga <= running else img[0]
    return {"theta": r1.theta, "ant": (ax, ay, az), "slant_range": r0, "image": final, "timeline": timeline,
            "entropy_cubic": min(h["entropy"] for h in r1.history), "entropy_los": min(h["entropy"] for h in h2),
            "entropy_pga": e_pga, "seconds": t3, "pga_iterations": len(rms)}


def time_to_entropy(timeline, target: float) -> Optional[float]:
    """First time in a (seconds, best entropy, stage) timeline at or below target."""
    for t, e, _ in timeline:
        if e <= target:
            return t
    return None
