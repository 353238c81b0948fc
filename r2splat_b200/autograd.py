"""``torch.autograd`` interface to the explicit CT operators.

``rasterize`` and ``voxelize`` wrap ``rasterize_fwd``/``rasterize_bwd`` and
``voxelize_fwd``/``voxelize_bwd`` (the reference's explicit API,
``r2splat/explicit.py:102-351``) in ``torch.autograd.Function``s. Gradients
flow to means, quats, scales, densities and, when given, beta and uncertainty;
cameras, volume extent and centre are constants, as in the explicit API.

With ``recompute=True`` the forward keeps only its (validated) inputs and the
backward rebuilds what the VJP reads:
* rasterize: the parameter transform and the projection (packed records and
  tile rectangles). The record-parallel VJP walks each record's tile
  rectangle, so the intersection lists are neither stored nor rebuilt.
* voxelize: the parameter transform, the voxel mapping and the scan of the
  per-primitive tile-box layer counts. The record-parallel voxel VJP walks
  each primitive's tile box, so here too the intersection lists are neither
  stored nor rebuilt.

That trades a projection for the memory of the saved lists and records
between forward and backward. Without ``recompute``
the explicit context from the forward is kept and consumed by the first
backward; a second backward (``retain_graph=True``) rebuilds it.
"""

from __future__ import annotations

from typing import Optional, Sequence, Union

import torch

from . import _fused, explicit
from ._validation import _options

Tensor = torch.Tensor


def _vjp_context(kind, shape, primitives, buffers, eps, detach_variance):
    return explicit._context(kind, shape, primitives, buffers, [], eps, "primitive", detach_variance)


class _Rasterize(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, quats, scales, densities, beta, uncertainty, viewmats, Ks, image_size, eps, radius_clip,
                detach_variance, recompute):
        output, context = explicit.rasterize_fwd(
            means.detach(), quats.detach(), scales.detach(), densities.detach(), viewmats, Ks, image_size,
            beta=None if beta is None else beta.detach(),
            uncertainty=None if uncertainty is None else uncertainty.detach(),
            eps=eps, radius_clip=radius_clip, detach_variance=detach_variance)
        ctx.has_variance = uncertainty is not None
        ctx.kept = None if recompute else context
        ctx.shape = context.shape
        ctx.eps = context.eps
        ctx.radius_clip = _options(beta, eps, radius_clip, detach_variance)[1]
        ctx.detach_variance = detach_variance
        ctx.cameras = (context.buffers["viewmats"], context.buffers["Ks"])
        ctx.save_for_backward(*context.primitives)
        if recompute:
            context.buffers.clear()
        return output

    @staticmethod
    def backward(ctx, *grads):
        v_image = grads[0]
        v_variance = grads[1] if ctx.has_variance else None
        context, ctx.kept = ctx.kept, None
        primitives = ctx.saved_tensors
        if context is None or context.used:
            means, quats, scales, densities, beta, _ = primitives
            viewmats, Ks = ctx.cameras
            _, height, width = ctx.shape
            with torch.cuda.device(means.device):
                state = _fused.raster_vjp_state(means, quats, scales, densities, viewmats, Ks, width, height, beta,
                                                ctx.eps, ctx.radius_clip)
            context = _vjp_context("rasterize", ctx.shape, primitives,
                                   {"viewmats": viewmats, "Ks": Ks, "state": state}, ctx.eps, ctx.detach_variance)
        g = explicit.rasterize_bwd(context, v_image, v_variance)
        return (g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty) + (None,) * 7


class _Voxelize(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, quats, scales, densities, beta, uncertainty, volume_shape, volume_extent, volume_center,
                eps, radius_clip, detach_variance, recompute):
        output, context = explicit.voxelize_fwd(
            means.detach(), quats.detach(), scales.detach(), densities.detach(), volume_shape,
            volume_extent=volume_extent, volume_center=volume_center,
            beta=None if beta is None else beta.detach(),
            uncertainty=None if uncertainty is None else uncertainty.detach(),
            eps=eps, radius_clip=radius_clip, detach_variance=detach_variance)
        ctx.has_variance = uncertainty is not None
        ctx.kept = None if recompute else context
        ctx.shape = context.shape
        ctx.eps = context.eps
        ctx.radius_clip = _options(beta, eps, radius_clip, detach_variance)[1]
        ctx.detach_variance = detach_variance
        ctx.volume = (context.buffers["extent"], context.buffers["center"])
        ctx.save_for_backward(*context.primitives)
        if recompute:
            context.buffers.clear()
        return output

    @staticmethod
    def backward(ctx, *grads):
        v_volume = grads[0]
        v_variance = grads[1] if ctx.has_variance else None
        context, ctx.kept = ctx.kept, None
        primitives = ctx.saved_tensors
        if context is None or context.used:
            means, quats, scales, densities, beta, uncertainty = primitives
            extent, center = ctx.volume
            with torch.cuda.device(means.device):
                state = _fused.voxel_vjp_state(means, quats, scales, densities, ctx.shape, extent, center, beta,
                                               uncertainty, ctx.eps, ctx.radius_clip)
            context = _vjp_context("voxelize", ctx.shape, primitives,
                                   {"extent": extent, "center": center, "state": state}, ctx.eps,
                                   ctx.detach_variance)
        g = explicit.voxelize_bwd(context, v_volume, v_variance)
        return (g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty) + (None,) * 7


def rasterize(means: Tensor, quats: Tensor, scales: Tensor, densities: Tensor, viewmats: Tensor, Ks: Tensor,
              image_size: Sequence[int], *, beta: Optional[Tensor] = None, uncertainty: Optional[Tensor] = None,
              eps: float = 1.0e-8, radius_clip: Optional[float] = None, detach_variance: bool = False,
              recompute: bool = False) -> Union[Tensor, tuple[Tensor, Tensor]]:
    """Differentiable projection: the image (or (image, variance) with uncertainty)."""
    return _Rasterize.apply(means, quats, scales, densities, beta, uncertainty, viewmats, Ks, image_size, eps,
                            radius_clip, detach_variance, recompute)


def voxelize(means: Tensor, quats: Tensor, scales: Tensor, densities: Tensor, volume_shape: Sequence[int], *,
             volume_extent: Union[Tensor, Sequence[float]],
             volume_center: Union[Tensor, Sequence[float]] = (0.0, 0.0, 0.0), beta: Optional[Tensor] = None,
             uncertainty: Optional[Tensor] = None, eps: float = 1.0e-8, radius_clip: Optional[float] = None,
             detach_variance: bool = False, recompute: bool = False) -> Union[Tensor, tuple[Tensor, Tensor]]:
    """Differentiable voxelization: the volume (or (volume, variance) with uncertainty)."""
    return _Voxelize.apply(means, quats, scales, densities, beta, uncertainty, volume_shape, volume_extent,
                           volume_center, eps, radius_clip, detach_variance, recompute)


__all__ = ["rasterize", "voxelize"]
