"""Motion-error autofocus on top of the backprojection engine.

* `CubicMotion`: per-axis cubic in normalised slow time, 12 coefficients
  (the reference's grid search fits linear or quadratic tracks with a velocity
  scale, src/autofocus/autofocus_gpu.cu:315-416 and
  gridSearchErrorFunctions_dft.cuh:279-291; the same family one degree higher).
* `gradient_autofocus`: minimises image entropy over the coefficients with the
  gradient from the adjoint backprojection kernel (autograd.backproject).
* `grid_search_autofocus`: the reference's search scheme restated on this
  engine -- a box of `points` samples per searched coefficient around the
  current estimate (by default the reference's own: slope and quadratic term
  per axis), every grid point imaged (hypothesis batches of
  sarbp_backproject_hypotheses) and scored with the reference's DFT cost,
  the best kept, the box halved, repeated (autofocus_gpu.cu:843-952, the
  halving at :938-939).  The reference's own
  implementation cannot run these sizes (Np <= 200, Nx <= 500 per
  gridSearchErrorFunctions_dft.cuh:37,41,275-277) and depends on the
  un-vendored cuGridSearch, so the comparison uses this restatement.
* `pga`: phase gradient autofocus as matlab/PGA.m:153-239 (circular shift of
  the brightest azimuth sample to the centre, -30 dB window, azimuth FFT,
  phi_dot = sum Im(conj(G) dG) / sum |G|^2, integrate, unwrap, remove the
  linear trend, apply exp(-j phi) in the azimuth-frequency domain), or as the
  reference's C++ routine (src/autofocus/cpu/autofocus_cpu.cpp:250-474), on
  the GPU with torch FFTs, batched, with no host read-back inside the loop.
* focus metrics: entropy, sharpness, and the reference's own grid-search
  costs, batched on the device: the 2-D DFT low-frequency energy of the 8-bit
  dB image (gridSearchErrorFunctions_dft.cuh:102-109,112-203,320-335) and the
  column-histogram entropy (gridSearchErrorFunctions.cuh:341-447).
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
    then truncation to unsigned char; max over each image of a batch
    [..., nx, ny]."""
    mag = img.abs().float()
    mx = mag.amax(dim=(-2, -1), keepdim=True)
    pixelf = (255.0 / dyn_range_db) * (20.0 * torch.log10(mag / mx) + dyn_range_db)
    return torch.where(pixelf < 0, torch.zeros_like(pixelf), torch.trunc(pixelf))


def reference_dft_costs(imgs: torch.Tensor, dyn_range_db: float = 70.0, percentage: float = 0.35) -> torch.Tensor:
    """The reference grid search's focus cost for each image of a batch
    [..., nx, ny] (x-major), on the device (gridSearchErrorFunctions_dft.cuh:
    112-203, 320-335): the 2-D DFT F of the 8-bit dB image, and for every x
    and every y < ny/2 whose squared index distance to the (0, 0) or
    (nx-1, 0) corner is below int((ny/2)^2 + (nx/2)^2) * percentage^2,
    |F[x][y]| + |F[x][ny-1-y]| summed; the cost is minus that sum.  The
    reference evaluates this DFT directly, one image per CUDA block with
    nx <= 500 (its local arrays); here any size, the DFT as a batched FFT."""
    u8 = reference_u8_image(imgs, dyn_range_db).double()
    F = torch.fft.fft2(u8).abs()
    nx, ny = F.shape[-2], F.shape[-1]
    hh, hw = ny // 2, nx // 2
    threshold = int((hh * hh + hw * hw) * (percentage * percentage))
    x = torch.arange(nx, device=F.device)[:, None]
    y = torch.arange(hh, device=F.device)[None, :]
    mask = ((x * x + y * y) < threshold) | (((nx - x - 1) ** 2 + y * y) < threshold)
    vals = F[..., :, :hh] + F[..., :, ny - 1 - torch.arange(hh, device=F.device)]
    return -(vals * mask).sum(dim=(-2, -1))


def reference_dft_cost(img: torch.Tensor, dyn_range_db: float = 70.0, percentage: float = 0.35) -> float:
    """reference_dft_costs of one image [nx, ny] as a float."""
    return float(reference_dft_costs(img.reshape(img.shape[-2], img.shape[-1]), dyn_range_db, percentage))


def reference_column_entropies(imgs: torch.Tensor, dyn_range_db: float = 70.0) -> torch.Tensor:
    """The reference's other grid-search cost, cuCalculateColumnEntropy
    (src/autofocus/gridSearchErrorFunctions.cuh:341-447), for each image of a
    batch [..., nx, ny], on the device: the 8-bit dB image against the
    image's maximum, a 256-bin histogram of each x line (ny pixels), its
    entropy H_x = -sum p log2 p, and the cost sum_x (100 if H_x == 0 else
    -H_x) / nx, as the routine returns it (the search minimises it)."""
    u8 = reference_u8_image(imgs, dyn_range_db).long()
    lead = u8.shape[:-1]  # [..., nx]
    ny = u8.shape[-1]
    flat = u8.reshape(-1, ny)
    counts = torch.zeros((flat.shape[0], 256), dtype=torch.float64, device=u8.device)
    counts.scatter_add_(1, flat, torch.ones_like(flat, dtype=torch.float64))
    p = counts / ny
    h = -(torch.where(p > 0, p * torch.log2(p.clamp_min(1e-300)), torch.zeros_like(p))).sum(dim=1)
    h = h.reshape(lead)
    per_line = torch.where(h == 0, torch.full_like(h, 100.0), -h)
    return per_line.mean(dim=-1)


def focus_metrics(img: torch.Tensor) -> dict:
    """Shannon entropy of the normalised intensity (the gradient pipeline's
    loss) and the reference's two grid-search costs of one image."""
    x = img.reshape(img.shape[-2], img.shape[-1])
    return {"shannon_entropy": float(A.image_entropy(x)), "reference_dft_cost": reference_dft_cost(x),
            "reference_column_entropy_cost": float(reference_column_entropies(x))}


def _descend(step, iters: int, lr_at, lr: torch.Tensor, record, graph: bool, warm: int = 10, stop=None,
             check_every: int = 25):
    """Run up to `iters` descent steps; `step()` does one (forward, entropy,
    backward, optimiser step) on static tensors.  With graph=True the first
    `warm` steps run eagerly (they initialise the optimiser state and every
    lazily allocated buffer, and the first steps, where a descent from a
    metre-scale error gains the most, do not wait for the capture) and the
    rest replay one CUDA graph captured right after them
    (capture_begin/capture_end on a side stream: the capture itself executes
    nothing).  Before step it the learning-rate tensor holds
    lr_at(it); after it `record(it)` copies the step's outputs on the device.
    `stop(n)`, when given, is asked after every `check_every` steps (n steps
    done; it may read the recorded outputs, one host wait) and ends the
    descent when true.  Returns (seconds, completion events; events[0] =
    start, steps run), the events on the GPU clock, the capture included in
    the wall time."""
    events = [torch.cuda.Event(enable_timing=True) for _ in range(iters + 1)]
    done = 0
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
            done = it + 1
            if stop is not None and done % check_every == 0 and done < iters and stop(done):
                break
    cur.wait_stream(side)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    del g
    return seconds, events, done


@dataclasses.dataclass
class AutofocusState:
    """Where a gradient autofocus run stopped: the last iterate of the 12
    coefficients, Adam's moments and step count, and the schedule position
    (`iters_done` of `total_iters` steps), enough to resume it exactly."""

    theta: np.ndarray       # [3, 4] float64
    exp_avg: np.ndarray     # [3, 4] Adam first moment
    exp_avg_sq: np.ndarray  # [3, 4] Adam second moment
    step: float             # Adam step count
    iters_done: int
    total_iters: int
    lr: float

    def save(self, path: str) -> None:
        """Write the state to an .npz file."""
        np.savez(path, theta=self.theta, exp_avg=self.exp_avg, exp_avg_sq=self.exp_avg_sq,
                 step=np.float64(self.step), iters_done=np.int64(self.iters_done),
                 total_iters=np.int64(self.total_iters), lr=np.float64(self.lr))

    @classmethod
    def load(cls, path: str) -> "AutofocusState":
        with np.load(path) as z:
            return cls(theta=z["theta"].copy(), exp_avg=z["exp_avg"].copy(), exp_avg_sq=z["exp_avg_sq"].copy(),
                       step=float(z["step"]), iters_done=int(z["iters_done"]), total_iters=int(z["total_iters"]),
                       lr=float(z["lr"]))


@dataclasses.dataclass
class AutofocusResult:

    theta: torch.Tensor
    history: List[dict]
    seconds: float
    images_formed: int
    state: Optional[AutofocusState] = None  # the last iterate, to resume from


def gradient_autofocus(plan: Plan, motion: CubicMotion, slant_range, start_freq, iters: int = 200,
                       lr: float = 0.02, theta0: Optional[torch.Tensor] = None, coarse_to_fine: bool = True,
                       log_every: int = 1, graph: bool = True, resume: Optional[AutofocusState] = None,
                       total_iters: Optional[int] = None, plateau: Optional[float] = None,
                       check_every: int = 25) -> AutofocusResult:
    """Adam on the 12 coefficients, loss = image entropy, gradient through the
    adjoint backprojection.  With coarse_to_fine the step size decays from
    `lr` metres to lr/100 (cosine, as CosineAnnealingLR), which lets the first
    steps cross the large blur of a metre-scale track error and the last ones
    settle.  Each step is replayed from a captured CUDA graph (graph=False:
    eager); entropies and parameters stay on the device and the steps are
    timed with CUDA events, so the host never waits inside the loop.

    Checkpoints: the result's `state` holds the last iterate and Adam's
    moments; `resume=state` continues from it (its learning rate and
    schedule position), so a run of n steps split into parts that save and
    resume their state reaches the same coefficients as the whole run.  The
    cosine schedule spans `total_iters` steps (default: this call's steps,
    or the resumed run's total).

    Early stop: with `plateau` set, the descent ends (before `iters` steps)
    once the best entropy has improved by less than `plateau` nats over the
    last `check_every` steps (one host read of the entropies per check)."""
    dev = motion.base.device
    done = 0
    if resume is not None:
        lr = resume.lr
        done = resume.iters_done
        total = resume.total_iters if total_iters is None else int(total_iters)
        start = torch.as_tensor(resume.theta, dtype=torch.float64, device=dev)
    else:
        total = iters if total_iters is None else int(total_iters)
        start = theta0.clone() if theta0 is not None else torch.zeros((3, 4), dtype=torch.float64, device=dev)
    theta = start.clone().requires_grad_(True)
    lr_t = torch.tensor(lr, dtype=torch.float64, device=dev)
    opt = torch.optim.Adam([theta], lr=lr_t, capturable=True)
    if resume is not None:
        st = opt.state[theta]
        # Adam's own lazy state: a scalar step tensor of the default scalar
        # type on the device (capturable), moments of the parameter's type
        step_dtype = torch.float64 if torch.get_default_dtype() == torch.float64 else torch.float32
        st["step"] = torch.tensor(resume.step, dtype=step_dtype, device=dev)
        st["exp_avg"] = torch.as_tensor(resume.exp_avg, dtype=torch.float64, device=dev).clone()
        st["exp_avg_sq"] = torch.as_tensor(resume.exp_avg_sq, dtype=torch.float64, device=dev).clone()
    eta_min = lr / 100.0

    def lr_at(it):
        k = done + it
        return eta_min + 0.5 * (lr - eta_min) * (1.0 + math.cos(math.pi * k / total)) if coarse_to_fine else lr

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

    stop = None
    if plateau is not None:
        def stop(n):
            if n <= check_every:
                return False
            return float(ents[:n - check_every].min() - ents[:n].min()) < plateau

    seconds, events, ran = _descend(step, iters, lr_at, lr_t, record, graph, stop=stop, check_every=check_every)
    e_host = ents[:ran].cpu().tolist()
    best = min(range(ran), key=lambda i: e_host[i])
    hist = [{"iter": done + it, "entropy": e_host[it], "t": events[0].elapsed_time(events[it + 1]) * 1e-3}
            for it in range(ran) if (log_every and (it % log_every == 0 or it == ran - 1)) or not log_every]
    ost = opt.state[theta]
    state = AutofocusState(theta=theta.detach().cpu().numpy().copy(), exp_avg=ost["exp_avg"].cpu().numpy().copy(),
                           exp_avg_sq=ost["exp_avg_sq"].cpu().numpy().copy(), step=float(ost["step"]),
                           iters_done=done + ran, total_iters=total, lr=lr)
    return AutofocusResult(theta=thetas[best].clone(), history=hist, seconds=seconds, images_formed=ran,
                           state=state)


# The reference's quadratic search varies, per axis, the slope and the
# quadratic coefficient of the track over pulse index (5 points each) and a
# common velocity scale of the slopes (autofocus_gpu.cu:1010-1030,
# gridSearchErrorFunctions_dft.cuh:279-291); the constant terms stay fixed.
# On the cubic model that is powers 1 and 2 of slow time on each axis (the
# velocity scale multiplies every slope: a direction the slope axes span).
REFERENCE_SEARCH_COEFFS = ((0, 1), (0, 2), (1, 1), (1, 2), (2, 1), (2, 2))


def grid_search_autofocus(plan: Plan, motion: CubicMotion, slant_range, start_freq, span: float,
                          coeffs: Sequence[tuple] = REFERENCE_SEARCH_COEFFS, points: int = 5, levels: int = 4,
                          batch: int = 256, theta0: Optional[torch.Tensor] = None,
                          deadline_s: Optional[float] = None, target_entropy: Optional[float] = None,
                          cost: str = "reference_dft") -> AutofocusResult:
    """Exhaustive multiresolution search (autofocus_gpu.cu:1032-1118, halving
    at :938-939): `points` samples in +-span around the estimate for each
    searched coefficient (axis, power), every combination imaged
    (sarbp_backproject_hypotheses) and scored -- by the reference's own cost
    (cost="reference_dft", reference_dft_costs) or by the Shannon entropy
    (cost="entropy") -- the best kept, the box halved, `levels` times.  The
    best score, its coefficients and its image's Shannon entropy stay on the
    device across batches (no host read-back inside a level); each level ends
    with one read for the history.  Stops after the level at which
    `deadline_s` has passed or `target_entropy` (Shannon) is reached."""
    if cost not in ("reference_dft", "entropy"):
        raise ValueError(cost)
    dev = motion.base.device
    theta = theta0.clone() if theta0 is not None else torch.zeros((3, 4), dtype=torch.float64, device=dev)
    Np = motion.base.shape[1]
    hist = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    formed = 0
    ncoef = len(coeffs)
    offsets1d = torch.linspace(-1.0, 1.0, points, dtype=torch.float64, device=dev)
    mesh = torch.stack(torch.meshgrid(*([offsets1d] * ncoef), indexing="ij"), dim=-1).reshape(-1, ncoef)
    r0 = slant_range.reshape(1, -1)
    f0 = start_freq.reshape(1, -1)
    ax_i = torch.tensor([a for a, _ in coeffs], device=dev)
    pw_i = torch.tensor([p for _, p in coeffs], device=dev)
    best_score = torch.full((), float("inf"), dtype=torch.float64, device=dev)
    best_ent = torch.full((), float("inf"), dtype=torch.float64, device=dev)
    done = False
    for level in range(levels):
        s = span / (2 ** level)
        centre = theta.clone()
        for b0 in range(0, mesh.shape[0], batch):
            cand = mesh[b0:b0 + batch] * s  # [H, ncoef]
            H = cand.shape[0]
            th = centre.unsqueeze(0).repeat(H, 1, 1)
            th[:, ax_i, pw_i] = centre[ax_i, pw_i].unsqueeze(0) + cand
            tracks = motion.base.unsqueeze(0) + th @ motion.powers  # [H, 3, Np]
            imgs = plan.backproject_hypotheses(tracks[:, 0].contiguous(), tracks[:, 1].contiguous(),
                                               tracks[:, 2].contiguous(), r0.expand(H, Np).contiguous(),
                                               f0.expand(H, Np).contiguous())
            ent = batch_entropy(imgs)
            score = reference_dft_costs(imgs[:, 0]) if cost == "reference_dft" else ent
            formed += H
            k = torch.argmin(score)
            better = score[k] < best_score
            best_score = torch.where(better, score[k], best_score)
            best_ent = torch.where(better, ent[k].double(), best_ent)
            theta = torch.where(better, th[k], theta)
            if deadline_s is not None and time.perf_counter() - t0 > deadline_s:
                done = True
                break
        e = float(best_ent)  # one read per level, for the history
        hist.append({"level": level, "entropy": e, "score": float(best_score), "cost": cost,
                     "t": time.perf_counter() - t0, "images": formed})
        if done or (target_entropy is not None and e <= target_entropy):
            break
    torch.cuda.synchronize()
    return AutofocusResult(theta=theta, history=hist, seconds=time.perf_counter() - t0, images_formed=formed)


def _unwrap(phi: torch.Tensor) -> torch.Tensor:
    """numpy.unwrap along the last axis on the device: jumps of more than pi
    between neighbours replaced by their value modulo 2 pi (in (-pi, pi],
    +pi kept for positive jumps of exactly pi), accumulated."""
    d = phi[..., 1:] - phi[..., :-1]
    dd = torch.remainder(d + math.pi, 2.0 * math.pi) - math.pi
    dd = torch.where((dd == -math.pi) & (d > 0), torch.full_like(dd, math.pi), dd)
    corr = torch.where(d.abs() < math.pi, torch.zeros_like(d), dd - d)
    return torch.cat([phi[..., :1], phi[..., 1:] + torch.cumsum(corr, -1)], dim=-1)


def _detrend(phi: torch.Tensor) -> torch.Tensor:
    """phi minus its least-squares line over the sample index (last axis)."""
    n = phi.shape[-1]
    i = torch.arange(n, dtype=phi.dtype, device=phi.device)
    sx, sxx = float(n * (n - 1) / 2), float((n - 1) * n * (2 * n - 1) / 6)
    sy, sxy = phi.sum(-1, keepdim=True), (phi * i).sum(-1, keepdim=True)
    d = n * sxx - sx * sx
    return phi - ((n * sxy - sx * sy) / d * i + (sy * sxx - sx * sxy) / d)


def _pga_estimate_matlab(x: torch.Tensor, col: torch.Tensor, db_down: float) -> torch.Tensor:
    """One phase-error estimate of matlab/PGA.m:153-212 for a batch [B, rows, n]."""
    n = x.shape[-1]
    c = (n + 1) // 2  # MATLAB center_az_idx = ceil(n/2) (1-based)
    center = c - 1  # its 0-based index: the window splits at [0, c) / [c, n)
    # brightest azimuth sample of each range line to 0-based index c:
    # circshift(row, 1 + c - m) with m the 1-based peak (:159-164)
    peak = torch.argmax(x.abs(), dim=-1, keepdim=True)
    f = torch.gather(x, -1, (col - (c - peak)) % n)
    # -30 dB window from the non-coherent average of the image (:167-188)
    avg = (x.real.double() ** 2 + x.imag.double() ** 2).sum(dim=-2)
    avg_db = 10.0 * torch.log10(avg / avg.amax(-1, keepdim=True) + 1e-30)
    below = avg_db - (avg_db.amax(-1, keepdim=True) - abs(db_down)) < 0
    left = torch.where(below & (col <= center), col, -1).amax(-1, keepdim=True) + 1
    right = torch.where(below & (col > center), col, n).amin(-1, keepdim=True) - 1
    g = f * ((col >= left) & (col <= right)).unsqueeze(-2)
    # azimuth FFT of the ifftshifted lines, phase-gradient estimate (:195-201)
    G = torch.fft.fft(torch.fft.ifftshift(g, dim=-1), dim=-1).to(torch.complex128)
    num = (G[..., :-1].conj() * (G[..., 1:] - G[..., :-1])).imag.sum(dim=-2)
    den = (G[..., :-1].abs() ** 2).sum(dim=-2).clamp_min(1e-300)
    phi = torch.cumsum(torch.cat([torch.zeros_like(num[..., :1]), num / den], dim=-1), dim=-1)
    # unwrap (:204), remove the linear trend (:209-212)
    return _detrend(_unwrap(phi))


def _pga_estimate_cpp(x: torch.Tensor, col: torch.Tensor) -> torch.Tensor:
    """One phase-error estimate of the reference's C++ PGA routine
    (src/autofocus/cpu/autofocus_cpu.cpp:250-402) for a batch [B, rows, n]:
    peak to index n - n//2 (cshift(n/2 + max)), -30 dB window from the
    unshifted image with the routine's own right-edge index (the position i
    in the second half's loop, not i + n/2: :307-311), G = FFT(cshift((n+1)/2)
    of the line), phi_dot normalised by sum |G|^2, cumulative sum without
    unwrap, least-squares line removed."""
    n = x.shape[-1]
    h = n // 2
    peak = torch.argmax(x.abs(), dim=-1, keepdim=True)
    f = torch.gather(x, -1, (col + h + peak) % n)
    avg = (x.real.double() ** 2 + x.imag.double() ** 2).sum(dim=-2)
    below = 10.0 * torch.log10(avg / avg.amax(-1, keepdim=True)) < -30.0
    first = col < h
    left = torch.where(below & first, col, -1).amax(-1, keepdim=True)
    left = torch.where(left < 0, torch.zeros_like(left), left)
    below_hi = torch.roll(below, -h, dims=-1)  # below[i + h] at position i (i < h)
    right = torch.where(below_hi & first, col, n).amin(-1, keepdim=True)
    g = f * ((col >= left) & (col < right)).unsqueeze(-2)
    G = torch.fft.fft(torch.roll(g, -((n + 1) // 2), dims=-1), dim=-1).to(torch.complex128)
    num = (G[..., :-1].conj() * (G[..., 1:] - G[..., :-1])).imag.sum(dim=-2)
    den = (G[..., :-1].abs() ** 2).sum(dim=-2)
    phi = torch.cumsum(torch.cat([torch.zeros_like(num[..., :1]), num / den], dim=-1), dim=-1)
    return _detrend(phi)


def pga(img: torch.Tensor, max_iter: int = 30, db_down: float = 30.0, rms_stop: float = 0.1,
        az_axis: int = -1, semantics: str = "matlab"):
    """Phase gradient autofocus, kept as the reference's own second-stage
    method, for one image [rows, n] or a batch [..., rows, n] (azimuth along
    `az_axis`), entirely on the device: every iteration is a fixed sequence
    of kernels with no host read-back, and an image whose rms has reached
    `rms_stop` stops changing (a per-image mask) instead of ending the loop,
    so a batch runs max_iter iterations without the host waiting.

    semantics="matlab": matlab/PGA.m:153-239 (correction applied, then the
    loop ends once rms < rms_stop).  semantics="reference_cpp": the
    reference's C++ routine autofocus() (autofocus_cpu.cpp:250-474; the rms
    test comes before the correction, threshold 0.1 there).

    Returns (corrected image(s), accumulated phase correction [..., n],
    rms per iteration [..., max_iter] with NaN after an image stopped)."""
    if semantics not in ("matlab", "reference_cpp"):
        raise ValueError(semantics)
    x = img.to(torch.complex64)
    if az_axis not in (-1, x.dim() - 1):
        x = x.transpose(az_axis, -1)
    single = x.dim() == 2
    if single:
        x = x.unsqueeze(0)
    lead = x.shape[:-2]
    x = x.reshape((-1,) + tuple(x.shape[-2:])).contiguous()
    B, n = x.shape[0], x.shape[-1]
    col = torch.arange(n, device=x.device)
    total = torch.zeros((B, n), dtype=torch.float64, device=x.device)
    rms_hist = torch.full((B, max_iter), float("nan"), dtype=torch.float64, device=x.device)
    active = torch.ones((B, 1), dtype=torch.bool, device=x.device)
    for it in range(max_iter):
        phi = _pga_estimate_matlab(x, col, db_down) if semantics == "matlab" else _pga_estimate_cpp(x, col)
        rms = torch.sqrt(torch.mean(phi ** 2, dim=-1, keepdim=True))
        keep_on = rms >= rms_stop
        # matlab: this iteration's correction is applied, then the image stops;
        # reference_cpp: an image below the threshold stops before correcting
        apply = active if semantics == "matlab" else active & keep_on
        phi = torch.where(apply, phi, torch.zeros_like(phi))
        rms_hist[:, it:it + 1] = torch.where(active, rms, torch.full_like(rms, float("nan")))
        total += phi
        # apply exp(-j phi) in the azimuth-frequency domain (PGA.m:229-232)
        X = torch.fft.fft(x, dim=-1) * torch.exp(-1j * phi).to(torch.complex64).unsqueeze(-2)
        x = torch.fft.ifft(X, dim=-1)
        active = active & keep_on
    x = x.reshape(tuple(lead) + tuple(x.shape[-2:]))
    total = total.reshape(tuple(lead) + (n,))
    rms_hist = rms_hist.reshape(tuple(lead) + (max_iter,))
    if single:
        x, total, rms_hist = x[0], total[0], rms_hist[0]
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

    seconds, events, _ = _descend(step, iters, lambda it: lr, lr_t, record, graph)
    e_host = ents.cpu().tolist()
    best = min(range(iters), key=lambda i: e_host[i])
    hist = [{"iter": it, "entropy": e_host[it], "t": events[0].elapsed_time(events[it + 1]) * 1e-3}
            for it in range(iters)]
    return ranges[best].clone().contiguous(), hist, seconds


def focus_motion_error(plan: Plan, ant_x, ant_y, ant_z, slant_range, start_freq, cubic_iters: int = 300,
                       cubic_lr: float = 0.02, los_iters: int = 200, los_lr: float = 2e-3,
                       pga_iters: int = 30, cubic_plateau: Optional[float] = 2e-3) -> dict:
    """Gradient autofocus pipeline on the plan's range profiles:
    (1) the 12 cubic track coefficients, (2) a per-pulse line-of-sight
    correction, both by entropy descent through the adjoint backprojection,
    (3) PGA, the reference's own phase-only refinement.  The cubic stage runs
    up to `cubic_iters` steps and stops early once its best entropy gains
    less than `cubic_plateau` nats per 25 steps (None: all steps): a low-order
    track reaches its floor well before the line-of-sight stage, which does
    most of the work (on the bench's autofocus scene it plateaus near 8.59
    after about 100 steps, and the final entropy after 100, 150 or 300 cubic
    steps is 6.223-6.225).  Returns the corrected geometry, the final image
    and a timeline of (seconds, entropy)."""
    motion = CubicMotion(ant_x, ant_y, ant_z)
    t_start = time.perf_counter()
    timeline = []
    r1 = gradient_autofocus(plan, motion, slant_range, start_freq, iters=cubic_iters, lr=cubic_lr, log_every=0,
                            plateau=cubic_plateau)
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
    e_pga = float(A.image_entropy(img_pga))
    t3 = time.perf_counter() - t_start
    timeline.append((t3, min(running, e_pga), "pga"))
    final = img_pga if e_pga <= running else img[0]
    return {"theta": r1.theta, "ant": (ax, ay, az), "slant_range": r0, "image": final, "timeline": timeline,
            "entropy_cubic": min(h["entropy"] for h in r1.history), "entropy_los": min(h["entropy"] for h in h2),
            "entropy_pga": e_pga, "seconds": t3, "pga_iterations": int(torch.isfinite(rms).sum()),
            "cubic_steps": r1.images_formed}


def time_to_entropy(timeline, target: float) -> Optional[float]:
    """First time in a (seconds, best entropy, stage) timeline at or below target."""
    for t, e, _ in timeline:
        if e <= target:
            return t
    return None
