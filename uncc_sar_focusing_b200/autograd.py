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
functions of the image that compose with this operation: the entropy of a
complex64 CUDA image runs as the library's fused kernels
(sarbp_image_entropy and its gradient), other inputs and the sharpness as
torch operations.  The reference's own focus metric is a non-differentiable
2-D DFT of an 8-bit dB image (src/autofocus/gridSearchErrorFunctions_dft.cuh:
112-203).
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as N
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


class _Entropy(torch.autograd.Function):
    """E = -sum p log p of a complex64 CUDA image through the library's
    kernels: two launches forward (FP64 sums in a fixed order), one backward;
    the sums travel from forward to backward in a small device buffer."""

    @staticmethod
    def forward(ctx, img):
        x = img.contiguous()
        with torch.cuda.device(x.device):
            work = torch.empty(N.lib().sarbp_image_entropy_work_bytes() // 8, dtype=torch.float64, device=x.device)
            e = torch.empty((), dtype=torch.float32, device=x.device)
            stream = torch.cuda.current_stream(x.device).cuda_stream
            N.check(N.lib().sarbp_image_entropy(ctypes.c_void_p(x.data_ptr()), x.numel(),
                                                ctypes.c_void_p(work.data_ptr()), ctypes.c_void_p(e.data_ptr()),
                                                ctypes.c_void_p(stream)), "sarbp_image_entropy")
        ctx.save_for_backward(x, work)
        ctx.shape = img.shape
        return e

    @staticmethod
    def backward(ctx, grad_e):
        x, work = ctx.saved_tensors
        with torch.cuda.device(x.device):
            g = grad_e.detach().to(device=x.device, dtype=torch.float32).contiguous()
            grad = torch.empty_like(x)
            stream = torch.cuda.current_stream(x.device).cuda_stream
            N.check(N.lib().sarbp_image_entropy_grad(ctypes.c_void_p(x.data_ptr()), x.numel(),
                                                     ctypes.c_void_p(work.data_ptr()), ctypes.c_void_p(g.data_ptr()),
                                                     ctypes.c_void_p(grad.data_ptr()), ctypes.c_void_p(stream)),
                    "sarbp_image_entropy_grad")
        return grad.reshape(ctx.shape)


def image_entropy(img: torch.Tensor) -> torch.Tensor:
    """Shannon entropy of the normalised intensity, -sum p log p with
    p = |I|^2 / sum |I|^2 (lower = sharper).  Complex64 CUDA images: the
    library's kernels (sums in FP64); otherwise torch operations in FP32."""
    if img.is_cuda and img.dtype == torch.complex64 and img.numel() > 0:
        return _Entropy.apply(img)
    return image_entropy_torch(img)


def image_entropy_torch(img: torch.Tensor) -> torch.Tensor:
    """image_entropy as torch operations (any device and complex dtype)."""
    w = img.real.float() ** 2 + img.imag.float() ** 2
    p = w / w.sum()
    return -(p * torch.log(p.clamp_min(1e-30))).sum()


def image_sharpness(img: torch.Tensor) -> torch.Tensor:
    """-sum |I|^4 / (sum |I|^2)^2 (lower = sharper)."""
    w = img.real.float() ** 2 + img.imag.float() ** 2
    return -(w * w).sum() / w.sum() ** 2
