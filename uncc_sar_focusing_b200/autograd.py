"""Backprojection as a differentiable torch operation.

`backproject(plan, ant_x, ant_y, ant_z, slant_range, start_freq)` forms the
image from the plan's current range profiles (sarbp_backproject) and, on
backward, returns the gradient with respect to the antenna positions and the
slant range through the hand-written adjoint kernel
(sarbp_backproject_adjoint).  Geometry tensors are float64 on the GPU; the
image is complex64.  The plan's range profiles must not change between the
forward and the backward call.  Nothing per pixel-pulse is saved for
backward: the adjoint recomputes every range.

The autofocus objectives of this package (image entropy, sharpness) are
plain torch functions of the image, so any of them composes with this
operation; the reference's own focus metric is a non-differentiable 2-D DFT
of an 8-bit dB image (src/autofocus/gridSearchErrorFunctions_dft.cuh:112-203).
"""
from __future__ import annotations

import torch

from .focusing import Plan


class _Backproject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, plan: Plan, ant_x, ant_y, ant_z, slant_range, start_freq):
        img = plan.backproject(ant_x, ant_y, ant_z, slant_range, start_freq, out=plan.new_image(ant_x.device))
        ctx.plan = plan
        ctx.save_for_backward(ant_x, ant_y, ant_z, slant_range, start_freq)
        return img

    @staticmethod
    def backward(ctx, grad_img):
        ax, ay, az, r0, f0 = ctx.saved_tensors
        g = grad_img.to(torch.complex64).contiguous()
        gant, gr0 = ctx.plan.backproject_adjoint(ax.detach(), ay.detach(), az.detach(), r0.detach(), f0.detach(), g)
        return None, gant[0], gant[1], gant[2], gr0, None


def backproject(plan: Plan, ant_x, ant_y, ant_z, slant_range, start_freq):
    return _Backproject.apply(plan, ant_x, ant_y, ant_z, slant_range, start_freq)


def image_entropy(img: torch.Tensor) -> torch.Tensor:
    """Shannon entropy of the normalised intensity, -sum p log p with
    p = |I|^2 / sum |I|^2 (lower = sharper)."""
    w = img.real.float() ** 2 + img.imag.float() ** 2
    p = w / w.sum()
    return -(p * torch.log(p.clamp_min(1e-30))).sum()


def image_sharpness(img: torch.Tensor) -> torch.Tensor:
    """-sum |I|^4 / (sum |I|^2)^2 (lower = sharper)."""
    w = img.real.float() ** 2 + img.imag.float() ** 2
    return -(w * w).sum() / w.sum() ** 2
