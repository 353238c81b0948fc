"""Explicit CUDA forward/VJP calls for physical primitive parameters.

Same public contract as the reference's ``r2splat/explicit.py``:
``rasterize_fwd`` (:102-188), ``rasterize_bwd`` (:191-242), ``voxelize_fwd``
(:245-311), ``voxelize_bwd`` (:314-351), the one-shot context with tensor
version guards (:37-99) and ``ParameterGradients`` (:25-34). Forward returns
``(output, context)`` without recording an autograd graph; backward consumes
the context once and returns gradients without writing ``.grad``. Geometry is
constant; activations and loss derivatives belong to the caller.

The device work runs through the fused sm_100a pipelines in ``_fused``.
``backward_mode`` is accepted for compatibility: "pixel" and "primitive" give
the same VJP here (one tile kernel serves both; they differ only in float
summation order in the reference).
"""

from __future__ import annotations

import contextlib
from dataclasses import dataclass
from typing import Optional, Sequence, Union

import torch

from . import _fused
from ._validation import (FOCAL, HOMOGENEOUS_ROW, PINHOLE, POSITIVE, _constant, _options, _primitives, _shape,
                          _tensor, _value_check, _vector, deferred_value_checks)

Tensor = torch.Tensor
Output = Union[Tensor, tuple[Tensor, Tensor]]
_PRIMITIVE_NAMES = ("means", "quats", "scales", "densities", "beta", "uncertainty")


@dataclass
class ParameterGradients:
    """VJP tensors matching the physical inputs; absent optional inputs give None."""

    means: Tensor
    quats: Tensor
    scales: Tensor
    densities: Tensor
    beta: Optional[Tensor] = None
    uncertainty: Optional[Tensor] = None


@dataclass
class _Context:
    kind: str
    shape: tuple
    primitives: tuple
    buffers: dict
    versions: tuple
    eps: float
    backward_mode: str
    detach_variance: bool
    used: bool = False


@contextlib.contextmanager
def _resolving(checks):
    """Resolves pending input checks after the block's device work is enqueued.

    A failing check is raised in preference to an error of the block itself.
    Checks already resolved inside the block (before a host read) are not
    evaluated again.
    """
    try:
        yield
    except BaseException:
        failure = checks.resolve()
        if failure is not None:
            raise failure from None
        raise
    checks.check()


def _mode(value):
    value = str(value).lower()
    if value not in ("pixel", "primitive"):
        raise ValueError("backward_mode must be 'pixel' or 'primitive'")
    return value


def _context(kind, shape, primitives, buffers, originals, eps, mode, detach_variance):
    """Snapshots the version counter of every input and saved tensor."""
    watched, seen = [], set()
    entries = list(originals) + list(zip(_PRIMITIVE_NAMES, primitives)) + [
        (name, value) for name, value in buffers.items() if isinstance(value, Tensor)]
    for name, value in entries:
        if isinstance(value, Tensor) and id(value) not in seen:
            try:
                version = value._version
            except RuntimeError as error:
                raise ValueError("explicit contexts require tensors with version counters") from error
            watched.append((name, value, version))
            seen.add(id(value))
    return _Context(kind, shape, primitives, buffers, tuple(watched), eps, mode, detach_variance)


def _check_context(context, kind):
    if not isinstance(context, _Context) or context.kind != kind:
        raise TypeError(f"expected a context returned by {kind}_fwd")
    if context.used:
        raise RuntimeError("this context has already been consumed by backward")
    for name, value, version in context.versions:
        if value._version != version:
            raise RuntimeError(f"saved input {name} was modified in-place after forward")


def _adjoint(name, value, context):
    return None if value is None else _tensor(name, value, context.shape, context.primitives[0])


def _zero_gradients(context):
    return ParameterGradients(*(None if value is None else torch.zeros_like(value) for value in context.primitives))


def _consume(context, gradients):
    context.used = True
    context.primitives = ()
    context.buffers.clear()
    context.versions = ()
    return gradients


@torch.no_grad()
def rasterize_fwd(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    densities: Tensor,
    viewmats: Tensor,
    Ks: Tensor,
    image_size: Sequence[int],
    *,
    beta: Optional[Tensor] = None,
    uncertainty: Optional[Tensor] = None,
    eps: float = 1.0e-8,
    radius_clip: Optional[float] = None,
    detach_variance: bool = False,
    backward_mode: str = "primitive",
) -> tuple[Output, _Context]:
    """Project physical primitives, returning a detached image and VJP context.

    World-to-camera ``viewmats [C,4,4]`` and pinhole ``Ks [C,3,3]`` are
    constant. Output is ``[C,height,width]`` or ``(image, variance)`` with
    uncertainty. No input needs requires_grad.
    """
    return _rasterize_fwd(means, quats, scales, densities, viewmats, Ks, image_size, beta, uncertainty, eps,
                          radius_clip, detach_variance, backward_mode, None)


def rasterize_fwd_with_loss(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    densities: Tensor,
    viewmats: Tensor,
    Ks: Tensor,
    image_size: Sequence[int],
    target: Tensor,
    *,
    loss: str = "mse",
    loss_weight: float = 1.0,
    beta: Optional[Tensor] = None,
    uncertainty: Optional[Tensor] = None,
    eps: float = 1.0e-8,
    radius_clip: Optional[float] = None,
    detach_variance: bool = False,
    backward_mode: str = "primitive",
) -> tuple[Output, _Context, Tensor, Tensor, Tensor]:
    """``rasterize_fwd`` with the mean image loss against ``target`` fused into the tile kernel.

    No reference counterpart: the reference's fit loop (examples/optimize.py)
    computes the image loss and its gradient with separate passes after the
    forward; its L1 form is ``image_loss_l1_fwd/bwd`` (Loss.cpp:12-113). Here
    the tile kernel's epilogue writes them while the image is in registers.

    ``target`` is ``[C,height,width]`` with the primitives' device and dtype.
    ``loss`` is "mse" (``weight * mean((image - target)^2)``, gradient
    ``(image - target) * (2 weight / numel)``) or "l1" (``weight * mean|image -
    target|``, gradient ``weight * sign(image - target) / numel``, the
    reference's L1 backward with an upstream gradient of one). The loss is on
    the image only; with ``uncertainty`` the variance is returned as usual.

    Returns ``(output, context, v_image, loss, loss_value)``: ``v_image`` is
    the adjoint to pass to ``rasterize_bwd``; ``loss`` is the weighted mean
    (0-dim) and ``loss_value`` the unweighted one, both summed in fp64 in a
    fixed order.
    """
    if loss not in _fused.IMAGE_LOSS_KINDS:
        raise ValueError('loss must be "mse" or "l1"')
    weight = float(loss_weight)
    if not (weight == weight and abs(weight) != float("inf")):
        raise ValueError("loss_weight must be finite")
    return _rasterize_fwd(means, quats, scales, densities, viewmats, Ks, image_size, beta, uncertainty, eps,
                          radius_clip, detach_variance, backward_mode, (target, loss, weight))


def _rasterize_fwd(means, quats, scales, densities, viewmats, Ks, image_size, beta, uncertainty, eps, radius_clip,
                   detach_variance, backward_mode, image_loss):
    originals = list(zip(
        ("means", "quats", "scales", "densities", "viewmats", "Ks", "beta", "uncertainty"),
        (means, quats, scales, densities, viewmats, Ks, beta, uncertainty),
    ))
    with deferred_value_checks(pending=True) as checks:
        height, width = _shape("image_size", image_size, 2)
        primitives = _primitives(means, quats, scales, densities, beta, uncertainty)
        means, quats, scales, densities, beta, uncertainty = primitives
        eps, radius_clip = _options(beta, eps, radius_clip, detach_variance)
        mode = _mode(backward_mode)
        # Check the originals: a contiguous copy under no_grad drops requires_grad.
        for name, value in (("viewmats", viewmats), ("Ks", Ks)):
            if isinstance(value, Tensor):
                _constant(name, value)
        viewmats = _constant("viewmats", _tensor("viewmats", viewmats, (None, 4, 4), means))
        cameras = viewmats.shape[0]
        if cameras == 0:
            raise ValueError("viewmats must contain at least one camera")
        if cameras * max(height * width, means.shape[0]) > 2**31 - 1 or cameras > 65535:
            raise ValueError("camera batch exceeds CUDA indexing or grid limits")
        if max(height, width) > 16 * 65535:
            raise ValueError("image_size exceeds CUDA grid limits")
        Ks = _constant("Ks", _tensor("Ks", Ks, (cameras, 3, 3), means))
        _value_check(Ks, FOCAL, ValueError, "Ks must have positive fx and fy")
        _value_check(Ks, PINHOLE, ValueError, "Ks must be pinhole intrinsics with zero skew and last row [0, 0, 1]")
        _value_check(viewmats, HOMOGENEOUS_ROW, ValueError, "viewmats must have homogeneous last row [0, 0, 0, 1]")
        if image_loss is not None:
            target = _constant("target", _tensor("target", image_loss[0], (cameras, height, width), means))
            image_loss = (target,) + tuple(image_loss[1:])
    shape = (cameras, height, width)
    buffers = {"viewmats": viewmats, "Ks": Ks}
    loss_out = None
    if means.shape[0] == 0:
        checks.check()
        image = means.new_zeros(shape)
        output = image if uncertainty is None else (image, image.clone())
        if image_loss is not None:
            # No primitives, no intersections: every tile list is empty.
            tile = _fused.RASTER_TILE
            offsets = torch.zeros((cameras * ((height + tile - 1) // tile) * ((width + tile - 1) // tile),),
                                  dtype=torch.int32, device=means.device)
            with torch.cuda.device(means.device):
                loss_out = _fused.render_image_loss(None, None, False, offsets, None, 0, 1, width, height, tile,
                                                    image_loss[0], image_loss[1], image_loss[2], image, None,
                                                    means.device)
    else:
        with _resolving(checks), torch.cuda.device(means.device):
            # The input checks resolve just before the intersection count is read.
            result = _fused.raster_forward(means, quats, scales, densities, viewmats, Ks, width, height, beta,
                                           uncertainty, eps, radius_clip, image_loss=image_loss,
                                           before_count=checks.check)
        output, state = result[0], result[1]
        if image_loss is not None:
            loss_out = result[2]
        buffers.update(state=state, covars=state.covars, records=state.records, offsets=state.offsets,
                       isect_ids=state.isect_ids, flatten_ids=state.flatten_ids, ratio=state.ratio)
    context = _context("rasterize", shape, primitives, buffers, originals, eps, mode, detach_variance)
    if image_loss is None:
        return output, context
    return (output, context) + tuple(loss_out)


@torch.no_grad()
def rasterize_bwd(context: _Context, v_image: Optional[Tensor], v_variance: Optional[Tensor] = None
                  ) -> ParameterGradients:
    """Consume a projection context and return physical-parameter gradients.

    Adjoint tensors match the output's shape, device, and dtype. None denotes
    a zero adjoint, including variance-only losses. Inputs must remain unchanged.
    """
    _check_context(context, "rasterize")
    means, quats, scales, densities, beta, uncertainty = context.primitives
    if v_variance is not None and uncertainty is None:
        raise ValueError("v_variance requires uncertainty in the forward call")
    with deferred_value_checks(pending=True) as checks:
        v_image = _adjoint("v_image", v_image, context)
        v_variance = _adjoint("v_variance", v_variance, context)
    if means.shape[0] == 0 or (v_image is None and v_variance is None):
        checks.check()
        return _consume(context, _zero_gradients(context))
    b = context.buffers
    # The VJP is enqueued before the adjoint checks resolve; on a failure its
    # result is dropped and the context stays unconsumed.
    with _resolving(checks), torch.cuda.device(means.device):
        grads = _fused.raster_backward(b["state"], means, quats, scales, densities, beta, uncertainty,
                                       b["viewmats"], b["Ks"], context.eps, v_image, v_variance,
                                       context.detach_variance)
    return _consume(context, ParameterGradients(*grads))


@torch.no_grad()
def voxelize_fwd(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    densities: Tensor,
    volume_shape: Sequence[int],
    *,
    volume_extent: Union[Tensor, Sequence[float]],
    volume_center: Union[Tensor, Sequence[float]] = (0.0, 0.0, 0.0),
    beta: Optional[Tensor] = None,
    uncertainty: Optional[Tensor] = None,
    eps: float = 1.0e-8,
    radius_clip: Optional[float] = None,
    detach_variance: bool = False,
    backward_mode: str = "primitive",
) -> tuple[Output, _Context]:
    """Sample physical primitives, returning a detached volume and VJP context.

    ``volume_shape`` and output use ``[depth,height,width]``; physical extent
    and center use xyz order. With uncertainty, output is ``(volume, variance)``.
    """
    originals = list(zip(
        ("means", "quats", "scales", "densities", "volume_extent", "volume_center", "beta", "uncertainty"),
        (means, quats, scales, densities, volume_extent, volume_center, beta, uncertainty),
    ))
    with deferred_value_checks(pending=True) as checks:
        depth, height, width = _shape("volume_shape", volume_shape, 3)
        if max(height, width) > 8 * 65535:
            raise ValueError("volume_shape exceeds CUDA grid limits")
        primitives = _primitives(means, quats, scales, densities, beta, uncertainty)
        means, quats, scales, densities, beta, uncertainty = primitives
        eps, radius_clip = _options(beta, eps, radius_clip, detach_variance)
        mode = _mode(backward_mode)
        for name, value in (("volume_extent", volume_extent), ("volume_center", volume_center)):
            if isinstance(value, Tensor):
                _constant(name, value)
        extent = _vector("volume_extent", volume_extent, means)
        center = _vector("volume_center", volume_center, means)
        _value_check(extent, POSITIVE, ValueError, "volume_extent must contain positive physical lengths")
    shape = (depth, height, width)
    buffers = {"extent": extent, "center": center}
    if means.shape[0] == 0:
        checks.check()
        volume = means.new_zeros(shape)
        output = volume if uncertainty is None else (volume, volume.clone())
    else:
        with _resolving(checks), torch.cuda.device(means.device):
            output, state = _fused.voxel_forward(means, quats, scales, densities, shape, extent, center, beta,
                                                 uncertainty, eps, radius_clip, before_count=checks.check)
        buffers.update(state=state, covars=state.covars, records=state.records, offsets=state.offsets,
                       isect_ids=state.isect_ids, flatten_ids=state.flatten_ids)
    context = _context("voxelize", shape, primitives, buffers, originals, eps, mode, detach_variance)
    return output, context


@torch.no_grad()
def voxelize_bwd(context: _Context, v_volume: Optional[Tensor], v_variance: Optional[Tensor] = None
                 ) -> ParameterGradients:
    """Consume a volume context and return gradients without updating inputs."""
    _check_context(context, "voxelize")
    means, quats, scales, densities, beta, uncertainty = context.primitives
    if v_variance is not None and uncertainty is None:
        raise ValueError("v_variance requires uncertainty in the forward call")
    with deferred_value_checks(pending=True) as checks:
        v_volume = _adjoint("v_volume", v_volume, context)
        v_variance = _adjoint("v_variance", v_variance, context)
    if means.shape[0] == 0 or (v_volume is None and v_variance is None):
        checks.check()
        return _consume(context, _zero_gradients(context))
    b = context.buffers
    with _resolving(checks), torch.cuda.device(means.device):
        grads = _fused.voxel_backward(b["state"], means, quats, scales, beta, uncertainty, b["extent"],
                                      b["center"], context.eps, v_volume, v_variance, context.detach_variance)
    return _consume(context, ParameterGradients(*grads))


# rasterize_fwd_with_loss is an extension outside the reference's surface: it is
# reached as r2splat_b200.explicit.rasterize_fwd_with_loss and not re-exported.
__all__ = ["ParameterGradients", "rasterize_fwd", "rasterize_bwd", "voxelize_fwd", "voxelize_bwd"]
