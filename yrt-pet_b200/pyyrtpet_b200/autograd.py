"""Differentiable TOF Siddon projection as a torch.autograd.Function.

forward(x) = A x for a fixed set of list-mode events; backward(g) = A^T g,
computed by the hand-written back-projection kernel (the ray traversal is
recomputed, no system matrix is stored).  A batch of images (B, nt, nz, ny,
nx) may share one event set or use one event set per batch element.
"""
from __future__ import annotations

from typing import Sequence, Union

import torch

from .core import DeviceEvents, DeviceProjector


class SiddonProjectFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, projector: DeviceProjector,
                events: Union[DeviceEvents, Sequence[DeviceEvents]]):
        batched = x.dim() == 5
        xs = x if batched else x[None]
        evs = events if isinstance(events, (list, tuple)) else [events] * xs.shape[0]
        if len(evs) != xs.shape[0]:
            raise RuntimeError("one event set per batch element expected")
        outs = []
        for b in range(xs.shape[0]):
            xb = xs[b].detach().contiguous().float()
            outs.append(projector.forward(xb, evs[b]))
        ctx.projector = projector
        ctx.events = evs
        ctx.batched = batched
        ctx.shape = xs.shape
        y = torch.stack(outs) if batched else outs[0]
        return y

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        gs = g if ctx.batched else g[None]
        grads = []
        for b in range(gs.shape[0]):
            img = torch.zeros(ctx.shape[1:], dtype=torch.float32, device=g.device)
            ctx.projector.backward(gs[b].contiguous().float(), ctx.events[b],
                                   img=img)
            grads.append(img)
        gx = torch.stack(grads) if ctx.batched else grads[0]
        return gx, None, None


def project(x, projector, events):
    return SiddonProjectFn.apply(x, projector, events)


class PoissonNLLFn(torch.autograd.Function):
    """List-mode Poisson negative log-likelihood sum_j s_j x_j - sum_e
    log(max(y_e, eps)), y = A x, and its gradient s - A^T (1/y) from one fused
    traversal per event (yrtb_em_step_model): the EM kernel's forward sum is
    y (written per event for the loss) and its back projection of 1/y is the
    gradient's data term.  The loss is identical to poisson_nll's (same
    forward sums, FP64 reductions); the gradient equals its autograd gradient
    for non-negative images up to the order of the FP32 atomic sums.  The
    gradient is computed with the loss, so a loss that is never
    differentiated still pays for it."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, projector: DeviceProjector,
                events: Union[DeviceEvents, Sequence[DeviceEvents]],
                sens_image: torch.Tensor, eps: float):
        batched = x.dim() == 5
        xs = x if batched else x[None]
        evs = events if isinstance(events, (list, tuple)) else [events] * xs.shape[0]
        if len(evs) != xs.shape[0]:
            raise RuntimeError("one event set per batch element expected")
        sens = sens_image.reshape(xs.shape[1:]).float()
        losses, grads = [], []
        for b in range(xs.shape[0]):
            xb = xs[b].detach().contiguous().float()
            y = torch.empty(evs[b].count, dtype=torch.float32, device=x.device)
            bp = torch.zeros_like(xb)
            projector.em_step(xb, bp, evs[b], denom_threshold=eps, model=y)
            lin = (sens.double() * xb.double()).sum()
            losses.append(lin - torch.log(y.double().clamp_min(eps)).sum())
            grads.append(sens - bp)
        ctx.save_for_backward(torch.stack(grads))
        ctx.batched = batched
        return torch.stack(losses) if batched else losses[0]

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        (grad,) = ctx.saved_tensors
        gs = g.reshape(-1, *([1] * (grad.dim() - 1))).to(grad.dtype)
        gx = gs * grad
        return (gx if ctx.batched else gx[0]), None, None, None, None


def poisson_nll_fused(x, projector, events, sens_image, eps: float = 1e-12):
    """poisson_nll with the loss and gradient of one fused pass (PoissonNLLFn)."""
    return PoissonNLLFn.apply(x, projector, events, sens_image, eps)


def poisson_nll(x, projector, events, sens_image, eps: float = 1e-12):
    """List-mode Poisson negative log-likelihood:
    sum_j s_j x_j - sum_e log(y_e) with y = A x.  Both reductions run in
    FP64 (millions of terms); the projections and gradients stay FP32."""
    y = project(x, projector, events).double()
    xd = x.double()
    if x.dim() == 5:
        lin = (sens_image[None].double() * xd).sum(dim=tuple(range(1, x.dim())))
        return lin - torch.log(y.clamp_min(eps)).sum(dim=-1)
    return (sens_image.double() * xd).sum() - torch.log(y.clamp_min(eps)).sum()
