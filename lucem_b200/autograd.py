"""Reverse-mode differentiation of the Gaussian family and of Richardson-Lucy.

The reference's operators are forward-only; these torch.autograd Functions
make them differentiable with hand-written backward kernels:

* the Gaussian filters' input gradients run the adjoint passes
  (lucem_gaussian_blur_adjoint: reversed taps plus the fold of the halo reads
  for every pad mode); DoG, LoG, unsharp and gradient magnitude compose them;
* Richardson-Lucy's gradients with respect to the PSF and the observation run
  the reverse pass through the unrolled iterations on the FFT passes
  (lucem_richardson_lucy_backward), recomputing the iterates from checkpoints
  kept every `checkpoint_every` iterations;
* fft_convolve (the deconvolution's forward model) has its own backward.

The forward of each Function is the same fused kernel the plain operator
runs.  Inputs must be float32 CUDA tensors where a gradient is wanted.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import ops

__all__ = [
    "gaussian_blur", "difference_of_gaussians", "gaussian_laplace", "gaussian_grad_mag", "unsharp_mask",
    "richardson_lucy", "fft_convolve",
]


class _GaussianBlur(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, kw):
        ctx.kw = kw
        return ops.gaussian_blur(x.contiguous(), **kw)

    @staticmethod
    def backward(ctx, g):
        kw = dict(ctx.kw)
        kw.pop("cval", None)
        return ops.gaussian_blur_adjoint(g.contiguous(), **kw), None


def gaussian_blur(x: torch.Tensor, sigmas, *, orders=None, mode="reflect", cval=0.0, truncate=4.0, radii=None,
                  axes=None, channel_axis=None, input_scale=1.0) -> torch.Tensor:
    """Differentiable ops.gaussian_blur (same arguments)."""
    kw = dict(sigmas=sigmas, orders=orders, mode=mode, cval=cval, truncate=truncate, radii=radii, axes=axes,
              channel_axis=channel_axis, input_scale=input_scale)
    return _GaussianBlur.apply(x, kw)


class _DoG(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, low, high, kw):
        ctx.low, ctx.high, ctx.kw = low, high, kw
        return ops.difference_of_gaussians(x.contiguous(), low, high, **kw)

    @staticmethod
    def backward(ctx, g):
        kw = dict(ctx.kw)
        kw.pop("cval", None)
        g = g.contiguous()
        lo = ops.gaussian_blur_adjoint(g, ctx.low, **kw)
        hi = ops.gaussian_blur_adjoint(g, ctx.high, **kw)
        return lo - hi, None, None, None


def difference_of_gaussians(x: torch.Tensor, low_sigmas, high_sigmas, *, mode="reflect", cval=0.0, truncate=4.0,
                            axes=None, channel_axis=None, input_scale=1.0) -> torch.Tensor:
    """Differentiable ops.difference_of_gaussians: G(low) x - G(high) x."""
    kw = dict(mode=mode, cval=cval, truncate=truncate, axes=axes, channel_axis=channel_axis,
              input_scale=input_scale)
    return _DoG.apply(x, low_sigmas, high_sigmas, kw)


class _Laplace(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, sigmas, kw):
        ctx.sigmas, ctx.kw, ctx.ndim = sigmas, kw, x.dim()
        return ops.gaussian_laplace(x.contiguous(), sigmas, **kw)

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous()
        out = None
        for a in range(ctx.ndim):
            orders = [0] * ctx.ndim
            orders[a] = 2
            t = ops.gaussian_blur_adjoint(g, ctx.sigmas, orders=orders, mode=ctx.kw["mode"],
                                          truncate=ctx.kw["truncate"])
            out = t if out is None else out + t
        return out, None, None


def gaussian_laplace(x: torch.Tensor, sigmas, *, mode="reflect", cval=0.0, truncate=4.0) -> torch.Tensor:
    """Differentiable ops.gaussian_laplace: the sum over axes of the
    second-derivative Gaussian along that axis."""
    return _Laplace.apply(x, sigmas, dict(mode=mode, cval=cval, truncate=truncate))


class _GradMag(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, sigmas, kw):
        x = x.contiguous()
        out = ops.gaussian_grad_mag(x, sigmas, **kw)
        ctx.sigmas, ctx.kw = sigmas, kw
        ctx.save_for_backward(x, out)
        return out

    @staticmethod
    def backward(ctx, g):
        x, mag = ctx.saved_tensors
        kw = ctx.kw
        # d|grad| / dx = sum_a D_a^T (g * d_a / |grad|), 0 where |grad| = 0.
        w = torch.where(mag > 0, g / torch.where(mag > 0, mag, torch.ones_like(mag)), torch.zeros_like(mag))
        out = None
        for a in range(x.dim()):
            orders = [0] * x.dim()
            orders[a] = 1
            d = ops.gaussian_blur(x, ctx.sigmas, orders=orders, mode=kw["mode"], cval=kw["cval"],
                                  truncate=kw["truncate"])
            t = ops.gaussian_blur_adjoint((w * d).contiguous(), ctx.sigmas, orders=orders, mode=kw["mode"],
                                          truncate=kw["truncate"])
            out = t if out is None else out + t
        return out, None, None


def gaussian_grad_mag(x: torch.Tensor, sigmas, *, mode="reflect", cval=0.0, truncate=4.0) -> torch.Tensor:
    """Differentiable ops.gaussian_grad_mag."""
    return _GradMag.apply(x, sigmas, dict(mode=mode, cval=cval, truncate=truncate))


class _Unsharp(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, sigmas, amount, kw):
        ctx.sigmas, ctx.amount, ctx.kw = sigmas, float(amount), kw
        return ops.unsharp_mask(x.contiguous(), sigmas, amount, **kw)

    @staticmethod
    def backward(ctx, g):
        kw = dict(ctx.kw)
        kw.pop("cval", None)
        scale = kw.pop("input_scale", 1.0)
        g = g.contiguous()
        blurred = ops.gaussian_blur_adjoint(g, ctx.sigmas, input_scale=scale, **kw)
        return (1.0 + ctx.amount) * scale * g - ctx.amount * blurred, None, None, None


def unsharp_mask(x: torch.Tensor, sigmas, amount: float, *, mode="reflect", cval=0.0, truncate=4.0, axes=None,
                 channel_axis=None, input_scale=1.0) -> torch.Tensor:
    """Differentiable ops.unsharp_mask: (1 + amount) x - amount G x."""
    kw = dict(mode=mode, cval=cval, truncate=truncate, axes=axes, channel_axis=channel_axis,
              input_scale=input_scale)
    return _Unsharp.apply(x, sigmas, amount, kw)


class _RichardsonLucy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, psf, kw):
        x = x.contiguous()
        psf = psf.contiguous()
        ctx.kw = kw
        ctx.save_for_backward(x, psf)
        # A leading batch axis goes to the library as it is: one call, the
        # volumes in the same launches.
        return ops.richardson_lucy(x, psf, num_iter=kw["num_iter"], clip=False, filter_epsilon=kw["filter_epsilon"],
                                   mode="constant", grid=kw["grid"], workspace=kw["workspace"])

    @staticmethod
    def backward(ctx, g):
        x, psf = ctx.saved_tensors
        kw = ctx.kw
        need_x, need_p = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        gp, gx = ops.richardson_lucy_backward(x, psf, g.contiguous(), num_iter=kw["num_iter"],
                                              filter_epsilon=kw["filter_epsilon"], grid=kw["grid"],
                                              checkpoint_every=kw["checkpoint_every"], need_psf=need_p,
                                              need_input=need_x, workspace=kw["workspace"])
        return gx, gp, None


def richardson_lucy(x: torch.Tensor, psf: torch.Tensor, *, num_iter: int = 30,
                    filter_epsilon: Optional[float] = None, grid=None, checkpoint_every: int = 5,
                    workspace: Optional[ops.Workspace] = None) -> torch.Tensor:
    """Differentiable ops.richardson_lucy with clip off and zero padding
    (mode "constant"), with respect to the observation and the PSF (through
    its normalisation).  `x` may carry one leading batch axis (one PSF for the
    batch).  The backward recomputes iterates from checkpoints kept every
    `checkpoint_every` iterations."""
    kw = dict(num_iter=int(num_iter), filter_epsilon=filter_epsilon, grid=grid,
              checkpoint_every=int(checkpoint_every), workspace=workspace)
    return _RichardsonLucy.apply(x, psf, kw)


class _FftConvolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, psf, grid):
        x = x.contiguous()
        psf = psf.contiguous()
        ctx.grid = grid
        ctx.save_for_backward(x, psf)
        return ops.fft_convolve(x, psf, grid=grid)

    @staticmethod
    def backward(ctx, g):
        x, psf = ctx.saved_tensors
        gp, gx = ops.fft_convolve_backward(x, psf, g.contiguous(), grid=ctx.grid,
                                           need_psf=ctx.needs_input_grad[1], need_input=ctx.needs_input_grad[0])
        return gx, gp, None


def fft_convolve(x: torch.Tensor, psf: torch.Tensor, *, grid=None) -> torch.Tensor:
    """Differentiable ops.fft_convolve (zero padding, PSF as given)."""
    return _FftConvolve.apply(x, psf, grid)
